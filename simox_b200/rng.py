"""The library's seeded counter-based random numbers in Python (host side):
the SplitMix64 output mix (Steele, Lea & Flood, OOPSLA 2014) applied to
(seed, stream a, counter b), 53 bits scaled into [0, 1) -- the same function
the GPU kernels of VINIT and the stochastic thermostat evaluate, so host-side
draws (the O2 insertion of the oxidation mode) come from the same family.
Streams in use: (1 << 62) | atom for VINIT, (step << 32) | atom for the
thermostat, (1 << 63) | event for O2 insertion."""
from __future__ import annotations

_M64 = (1 << 64) - 1
_G = 0x9E3779B97F4A7C15


def _mix64(z: int) -> int:
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def uniform(seed: int, a: int, b: int) -> float:
    """Draw number b of stream a under seed, in [0, 1)."""
    z = _mix64((_mix64((seed + _G * (a + 1)) & _M64) + _G * (b + 1)) & _M64)
    return (z >> 11) * (1.0 / 9007199254740992.0)
