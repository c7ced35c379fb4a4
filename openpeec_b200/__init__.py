"""B200 (sm_100a) frequency-sweep hot path of the OpenPEEC PEEC solver.

The compute lives in libpeec_b200.so (hand-written CUDA + C ABI, include/peec_b200.h);
this package is the host-side mirror: problem containers, the .peec subset reader and
geometry builder, and ctypes bindings of the C ABI.
"""
from .problem import Problem  # noqa: F401
