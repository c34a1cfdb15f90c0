"""Standard synthetic sea states used by the tests and the benchmark.

No dataset is involved: every workload is a seeded descriptor (or a seeded
list of them) in the shapes the reference's own benchmark and tests use.
Random draws come from PCG32 (the generator the library itself uses for h0),
restated here in vectorised numpy so seeded lists are reproducible anywhere.
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

from . import OceanDesc, FoamDesc

_MULT = np.uint64(6364136223846793005)
_MASK = (1 << 64) - 1


class Pcg32:
    """PCG32 XSH-RR (seed, stream) with the reference's seeding rule."""

    def __init__(self, seed: int, stream: int = 0):
        self.inc = ((stream << 1) | 1) & _MASK
        self.state = 0
        self.next_u32()
        self.state = (self.state + seed) & _MASK
        self.next_u32()

    def next_u32(self) -> int:
        old = self.state
        self.state = (old * 6364136223846793005 + self.inc) & _MASK
        xs = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xs >> rot) | (xs << ((32 - rot) & 31))) & 0xFFFFFFFF

    def next_open01(self) -> float:
        return (self.next_u32() + 0.5) * (1.0 / 4294967296.0)

    def many_u32(self, count: int) -> np.ndarray:
        """The next `count` outputs, vectorised (identical to repeated next_u32)."""
        block = 4096
        first = np.empty(min(block, count), dtype=np.uint64)
        s = self.state
        for i in range(first.size):
            first[i] = s
            s = (s * 6364136223846793005 + self.inc) & _MASK
        # Affine map of `block` steps: s -> A*s + C (mod 2^64).
        a, c = 1, 0
        for _ in range(block):
            a, c = (a * 6364136223846793005) & _MASK, (c * 6364136223846793005 + self.inc) & _MASK
        A, Cc = np.uint64(a), np.uint64(c)
        states = np.empty(count, dtype=np.uint64)
        cur = first
        pos = 0
        with np.errstate(over="ignore"):
            while pos < count:
                take = min(block, count - pos)
                states[pos:pos + take] = cur[:take]
                pos += take
                cur = cur * A + Cc
        # Advance the scalar state past the consumed outputs.
        last = int(states[count - 1])
        self.state = (last * 6364136223846793005 + self.inc) & _MASK
        with np.errstate(over="ignore"):
            xs = (((states >> np.uint64(18)) ^ states) >> np.uint64(27)) & np.uint64(0xFFFFFFFF)
            rot = states >> np.uint64(59)
            out = (xs >> rot) | (xs << ((np.uint64(32) - rot) & np.uint64(31)))
        return (out & np.uint64(0xFFFFFFFF)).astype(np.uint32)


# ---------------------------------------------------------------------------
# Sea states
# ---------------------------------------------------------------------------
def single_patch_256() -> Tuple[OceanDesc, float]:
    """One 256^2 patch, 200 m, 12 m/s, gamma 3.3, deep water, choppiness 1,
    seed 1337, evaluated at t = 10 s."""
    return OceanDesc(size=256, patch_length=200.0, wind_speed=12.0, peak_enhancement=3.3,
                     choppiness=1.0, seed=1337), 10.0


def bench_update_patch(n: int = 512, seed: int = 1337) -> OceanDesc:
    """The reference bench_update descriptor (bench/bench_update.cpp:91-102):
    200 m, 12 m/s, wind direction 0.4, choppiness 1."""
    return OceanDesc(size=n, patch_length=200.0, wind_speed=12.0, wind_direction=0.4,
                     choppiness=1.0, seed=seed)


def foam_patch_512(seed: int = 7) -> OceanDesc:
    """512^2, 250 m, 22 m/s, choppiness 1.5, orbital velocity on (needed by
    the persistent foam that rides on it)."""
    return OceanDesc(size=512, patch_length=250.0, wind_speed=22.0, choppiness=1.5, seed=seed,
                     compute_velocity=True)


FOAM_DT = 1.0 / 60.0


def foam_desc() -> FoamDesc:
    return FoamDesc()


def cascade_3x256() -> List[OceanDesc]:
    """Three 256^2 cascades of 800 / 150 / 25 m at 15 m/s over 30 m of water,
    velocity on, seeds 1 / 2 / 3."""
    return [OceanDesc(size=256, patch_length=L, wind_speed=15.0, depth=30.0, seed=s,
                      compute_velocity=True) for L, s in ((800.0, 1), (150.0, 2), (25.0, 3))]


def cascade_query_points(count: int = 1_000_000, extent: float = 800.0) -> np.ndarray:
    """(count, 2) float32 points uniform over [0, extent)^2 from PCG32(3, 0)."""
    u = Pcg32(3, 0).many_u32(2 * count).astype(np.float64)
    xz = ((u + 0.5) * (1.0 / 4294967296.0) * extent).astype(np.float32)
    return xz.reshape(count, 2)


def ensemble_64(count: int = 64) -> List[OceanDesc]:
    """`count` independent sea states from PCG32(42, 0): N from
    {64, 128, 256, 512, 1024}, wind 5-25 m/s, direction in [0, 2pi),
    choppiness 0.5-1.8, patch 50-1000 m; seed 1000 + i."""
    r = Pcg32(42, 0)
    sizes = (64, 128, 256, 512, 1024)
    out = []
    for i in range(count):
        n = sizes[r.next_u32() % 5]
        u_w, u_d, u_c, u_l = (r.next_open01() for _ in range(4))
        out.append(OceanDesc(size=n, patch_length=50.0 + 950.0 * u_l, wind_speed=5.0 + 20.0 * u_w,
                             wind_direction=2.0 * math.pi * u_d, choppiness=0.5 + 1.3 * u_c,
                             seed=1000 + i))
    return out
