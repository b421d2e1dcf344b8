"""B200 (sm_100a) implementation of NNPEngine's short-range force step.

The compute lives in ``lib/libnnpe.so`` (CUDA kernels behind the C ABI of ``include/nnpe.h``);
this package holds the Python mirror of the reference interfaces (``engine``), the seeded
system generators in the reference's file formats (``systems``) and the in-tree build
(``build``).
"""
from .systems import System, water_box, lj_mixture  # noqa: F401
