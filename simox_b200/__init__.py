"""B200-native force / charge / integrate path of SIMOX (sm_100a CUDA + cuFFT).

The compute path is ``libsimox_b200.so`` (sources in ``csrc/``), reached
through the C ABI of ``include/simox_gpu.h``.  ``api.Simox`` mirrors the
reference's per-step subroutines; ``systems`` generates seeded inputs.
"""
from . import _abi  # noqa: F401

__all__ = ["api", "systems", "build"]
