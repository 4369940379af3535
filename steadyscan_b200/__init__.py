"""B200-native align_group_to_template (SteadyScan motion estimator).

The estimator runs as hand-written sm_100a CUDA kernels behind the C-ABI declared in
``include/steadyscan_b200.h`` (library ``steadyscan_b200/libsteadyscan_b200.so``). This package
holds the host-side mirror of the reference's MEX interface (:mod:`steadyscan_b200.api`), the
caller-side preparation of its inputs (:mod:`steadyscan_b200.prep`) and synthetic workloads
(:mod:`steadyscan_b200.synth`).
"""
__version__ = "0.1.0"
