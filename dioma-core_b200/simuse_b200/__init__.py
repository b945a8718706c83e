"""simuse_b200 — B200-native SiMuse simulation step behind the reference's
``Network`` builder/step API.

The compute path is ``libsimuse_b200.so`` (hand-written CUDA for sm_100a,
C ABI in include/simuse_b200.h); this package is a thin ctypes mirror of the
reference's Rust API (crates/SiMuse/crates/pillars/src/api/net/network/) so
tests and tools read like the reference's own.  There is no CPU fallback:
importing the package fails loudly when the library is missing.
"""
from ._lib import SimuseError, lib, library_path  # noqa: F401
from .network import (  # noqa: F401
    GPEA,
    HH,
    IZH,
    LIF,
    W_BF16,
    W_F32,
    W_FP8,
    Network,
    Pool,
)
from .kuramoto import KuramotoBatch  # noqa: F401,E402
from .sweep import Sweep  # noqa: F401,E402
from .synaptic import SynapticBrain  # noqa: F401,E402
from . import taas  # noqa: F401,E402
