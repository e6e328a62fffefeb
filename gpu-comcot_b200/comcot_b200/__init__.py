"""comcot_b200: B200-native COMCOT time-stepping hot path (host side).

The compute path is libgcomcot.so (CUDA for sm_100a behind the reference's C
ABI); this package holds its ctypes binding, the once-per-run set-up
(precompute), seeded synthetic inputs, the reference-driver mirror and the
ensemble / serving front ends.
"""
from . import precompute, synth  # noqa: F401
from ._lib import LIB_PATH, load  # noqa: F401
