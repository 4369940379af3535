"""Copies the reference's task layer (Task, MainIteration, the kernels and their host launchers, the
filters, CudaHelper, ParameterOrganizer, Configuration) from the reference tree into
oracle/_ref/run/, rewritten so that g++ compiles it against the host CUDA runtime of hostcuda.h:
TEST INFRASTRUCTURE ONLY. It runs where the reference sources are; its outputs stay in the
git-ignored oracle/_ref/ and are never committed.

Rewrites (mechanical; the code itself is the reference's):
* ``kernel<<<grid, block, smem>>>( args )`` becomes ``SS_LAUNCH( grid, block, smem, kernel( args ) )``;
* ``extern __shared__ T a[]`` becomes ``SS_EXTERN_SHARED T a[]`` (one buffer per emulated block) and
  ``__shared__`` becomes ``SS_SHARED`` (a static shared by the block's emulated threads);
* before d_linesearch's launch the first knot of every frame but the first is copied from p to pnew
  (``ss_refrun_sync_boundary``): with the blocks run in order this fixes the race on that knot
  (task_linesearch.cu:50-54, 98-99) as the oracle does, and every trial knot is written before any
  thread warps its column with the next thread's knot (task_linesearch.cu:52-53, lock step);
* in d_linesearch (task_linesearch.cu) the two reads of the block-wide flag ``sharedResult`` that
  are followed by a reset of the flag without a barrier (``if( sharedResult ) break;`` and
  ``if( !sharedResult ) return;``) read it through ``ss_lockstep_read``: every thread of the block
  reads before any thread goes on, as the threads of one warp do in lock step (the test cases keep
  a frame's blocks within one warp, frameW <= 32), and after a trial with no block present every
  thread clears the flag before any thread's movement check sets it again (a lock-step point after
  the clear: without it a later thread's clear erased an earlier thread's report of movement, and
  the search of a frame whose moving knots run first stopped early);
* the includes of ``mex.h``, the Eigen headers and the timing/printing helpers are left out by the
  reference's own switches (``_DEBUG``, EIGENINCLUDE unset in the force-included configuration).
"""
import os
import re
import sys

SRC = os.environ.get("STEADYSCAN_REFERENCE_SOURCE", "/root/reference/setup/source")

FILES = [
    "task/task.cpp", "task/task_allocate.cu", "task/task_applyparameters.cu", "task/task_calcerrval.cu",
    "task/task_correlation.cu", "task/task_expandresults.cu", "task/task_filldiagonals.cu", "task/task_filljtr.cu",
    "task/task_generatesubsparseoffset.cu", "task/task_linesearch.cu", "task/task_maskinactive.cu",
    "task/task_updategradients.cu", "task/mainiteration/mainiteration.cpp", "task/solver/cusolversolver.cu",
    "task/filter/smearingfilter.cpp", "task/filter/rangefilter.cpp", "task/filter/nofilter.cpp",
    "task/filter/medianfilter.cpp", "task/filter/d_medianfilter.cu", "helper/cudahelper/cudahelper.cu",
    "interface/parameterorganizer/parameterorganizer.cpp", "mex/configuration.cpp", "interface/stopcriterion.cpp",
]

LAUNCH = re.compile(r"([A-Za-z_][\w:]*(?:\s*<[^<>;]*>)?)\s*<<<(.*?)>>>\s*\(", re.S)


def rewrite_launches(text):
    out, pos = [], 0
    for m in LAUNCH.finditer(text):
        # the argument list of the launch: up to the matching parenthesis
        i, depth = m.end(), 1
        while depth:
            depth += {"(": 1, ")": -1}.get(text[i], 0)
            i += 1
        args = text[m.end():i - 1]
        cfg = [c.strip() for c in split_top(m.group(2))]
        while len(cfg) < 3:
            cfg.append("0")
        out.append(text[pos:m.start()])
        out.append(f"SS_LAUNCH( {cfg[0]}, {cfg[1]}, {cfg[2]}, {m.group(1).strip()}( {args} ) )")
        pos = i
    out.append(text[pos:])
    return "".join(out)


def split_top(s):
    parts, depth, cur = [], 0, ""
    for ch in s:
        if ch in "([<":
            depth += 1
        elif ch in ")]>":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    parts.append(cur)
    return parts


def transform(rel, text):
    text = edit(rel, text)
    text = rewrite_launches(text)
    text = text.replace("extern __shared__", "SS_EXTERN_SHARED")
    text = re.sub(r"\b__shared__\b", "SS_SHARED", text)
    return text


def edit(rel, text):
    edits = []
    if rel.endswith("task_linesearch.cu"):
        edits = [("\td_linesearch<T> <<<", "\tss_refrun_sync_boundary( mem );\n\td_linesearch<T> <<<"),
                 # every thread's trial knot is written before any thread warps its column, which
                 # reads the next thread's knot (lock step within the warp)
                 ("\t\t\td_addDeltaP<T>( mem, idx );\n", "\t\t\td_addDeltaP<T>( mem, idx );\n\t\t\tss_lockstep_point();\n"),
                 # every thread clears the flag before any thread's movement check sets it again
                 ("\t\t\tif( sharedResult ) break;\n\t\t\tsharedResult = false;\n",
                  "\t\t\tif( ss_lockstep_read( sharedResult ) ) break;\n\t\t\tsharedResult = false;\n"
                  "\t\t\tss_lockstep_point();\n"),
                 ("if( !sharedResult ) return;", "if( !ss_lockstep_read( sharedResult ) ) return;"),
                 # thread idx == 0 updates the errval that the block's threads compare with
                 ("if( errvalNew < mem->errval[shift * mem->nFrames + blockIdx.x] ) {",
                  "if( errvalNew < ss_lockstep_read( mem->errval[shift * mem->nFrames + blockIdx.x] ) ) {")]
    elif rel.endswith("task_correlation.cu"):
        # d_blockReduce reads the other threads' partial sums with no barrier before its first step
        edits = [("__device__ void d_blockReduce( T* arr, int numElements2 ) {",
                  "__device__ void d_blockReduce( T* arr, int numElements2 ) {\n\tss_lockstep_point();"),
                 # d_frameCorrelation: every thread reads the reduced means before thread 0 overwrites
                 # their slots with its second-pass sums
                 ("\tT divSumB = buffB[0] / static_cast<T>( buffC[0] );\n",
                  "\tT divSumB = buffB[0] / static_cast<T>( buffC[0] );\n\tss_lockstep_point();\n")]
    for a, b in edits:
        if a not in text:
            sys.exit(f"{rel}: pattern not found: {a}")
        text = text.replace(a, b)
    return text


def main(out_dir):
    # every source and header keeps its place, so the reference's relative includes resolve in the copy
    for root, _, names in os.walk(SRC):
        for name in names:
            if not name.endswith((".h", ".cuh", ".cu", ".cpp")):
                continue
            rel = os.path.relpath(os.path.join(root, name), SRC)
            if rel.startswith("mk" + os.sep):
                continue
            with open(os.path.join(SRC, rel), errors="replace") as f:
                text = f.read()
            dst = os.path.join(out_dir, rel)
            os.makedirs(os.path.dirname(dst), exist_ok=True)
            with open(dst, "w") as f:
                f.write(f"// rewritten from setup/source/{rel} by oracle/ref_pin/run_transform.py\n")
                f.write(transform(rel, text))
    with open(os.path.join(out_dir, "sources.list"), "w") as f:
        f.write("\n".join(FILES) + "\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(__file__), "..", "_ref", "run"))
