"""B200 NDT scan-to-map registration (DAPHNE ndt_mapping align path).

Python side of the package: the ctypes binding of the C ABI in
include/ndt_b200.h (`ndt`), the synthetic workload generator (`synth`) and the
DAPHNE .dat format (`datfile`).  The compute path is the CUDA library built
from csrc/ into _build/libndt_b200.so; there is no CPU fallback.
"""
from . import autotune, datfile, ec, learned, ndt, posenet, shard, synth, voxel_filter  # noqa: F401
