"""oraclev8_b200 — B200 (sm_100a) backend for the Oracle V8 LH82 anelastic step.

The package mirrors the reference's solver interface (oracle_v8.solver):
OperatorConfig, the step components and RK3Integrator keep their call
signatures; fields are CUDA torch tensors and every operator runs in the
hand-written kernels of liboracle_b200.so (C ABI: include/oracle_b200.h).
There is no CPU fallback.
"""
from .backend import GPU_AVAILABLE, asarray, to_numpy, wrap_base  # noqa: F401
from .build import LIB as LIBRARY_PATH  # noqa: F401

__version__ = "0.1.0"
