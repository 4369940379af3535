"""Copies whitelisted functions out of the reference's .cu files into oracle/_ref/gen/ so that
g++ can compile them with shim.h. TEST INFRASTRUCTURE ONLY: it runs in the container that has the
reference sources; its outputs stay in the git-ignored oracle/_ref/ and are never committed.

Host launchers (``hd_*``, which use the ``<<<...>>>`` launch syntax) and the kernels that need a
whole CTA in lock-step (shared-memory reductions) are not taken.
"""
import os
import re
import sys

SRC = os.path.join(os.environ.get("STEADYSCAN_REFERENCE_SOURCE", "/root/reference/setup/source"), "task")
WANT = {
    "task_updategradients.cu": ["d_updateGradients"],
    "task_filldiagonals.cu": ["d_insertValue", "d_fillDiagonals"],
    "task_filljtr.cu": ["d_fillJTr"],
    "task_expandresults.cu": ["d_expandResults"],
    "task_calcerrval.cu": ["d_calcBaseErrval"],
    "task_correlation.cu": ["d_globalCorrelation", "d_clearImage", "d_swapWIDiff"],
    "task_linesearch.cu": ["d_addDeltaP", "d_reduceDeltaP", "d_setNewP", "d_checkMovement"],
}


def functions(text):
    """Yields (name, start, end) of each top-level function definition preceded by template<...>."""
    for m in re.finditer(r"template\s*<[^>]*>\s*(?:__\w+__\s+)*(?:inline\s+)?[\w:<>\*\s]+?\b(\w+)\s*\(", text):
        name = m.group(1)
        i = text.find("{", m.end())
        semi = text.find(";", m.end())
        if i < 0 or (0 <= semi < i):
            continue
        depth, j = 0, i
        while j < len(text):
            if text[j] == "{":
                depth += 1
            elif text[j] == "}":
                depth -= 1
                if depth == 0:
                    break
            j += 1
        yield name, m.start(), j + 1


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    for fname, names in WANT.items():
        text = open(os.path.join(SRC, fname)).read()
        found = {n: text[a:b] for n, a, b in functions(text) if n in names}
        missing = [n for n in names if n not in found]
        if missing:
            sys.exit(f"{fname}: functions not found: {missing}")
        with open(os.path.join(out_dir, fname.replace(".cu", ".gen.inc")), "w") as f:
            f.write(f"// extracted from setup/source/task/{fname} by oracle/ref_pin/extract.py\n")
            for n in names:
                f.write(found[n] + "\n\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(__file__), "..", "_ref", "gen"))
