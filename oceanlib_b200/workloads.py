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


# ---------------------------------------------------------------------------
# Serving loop: sessions, moving sources, Poisson arrivals
# ---------------------------------------------------------------------------
SERVE_DT = 1.0 / 60.0
SERVE_FIELD_EXTENT = 64.0


def serving_sessions(count: int = 256):
    """`count` sessions from PCG32(5, 0): ocean N from {128, 256, 512} (the
    other ocean fields at their defaults, seed 5000 + i), each with a 512^2
    interaction field over 64 m with a radius-6 stencil. Returns
    (ocean descriptors, interaction descriptor)."""
    from .interaction import InteractionDesc

    r = Pcg32(5, 0)
    sizes = (128, 256, 512)
    oceans = [OceanDesc(size=sizes[r.next_u32() % 3], seed=5000 + i) for i in range(count)]
    field = InteractionDesc(size=512, extent=SERVE_FIELD_EXTENT, kernel_radius=6)
    return oceans, field


class DiscPaths:
    """`per_session` continuous disc sources per session on seeded random-walk
    paths: radius U(0.5, 4) m, speed U(0, 8) m/s, heading turning by
    U(-0.4, 0.4) rad per frame, reflected off an 8 m margin inside the field.
    `frame(s)` returns session s's sources for its next update (positions at
    the frame start, velocities for the substep motion) and advances them."""

    def __init__(self, sessions: int, per_session: int = 32, seed: int = 17,
                 extent: float = SERVE_FIELD_EXTENT, dt: float = SERVE_DT):
        from .serve import DISTURBANCE_DTYPE

        rng = np.random.default_rng(seed)
        shape = (sessions, per_session)
        self.dt = dt
        self.lo, self.hi = 8.0, extent - 8.0
        self.x = rng.uniform(self.lo, self.hi, shape)
        self.z = rng.uniform(self.lo, self.hi, shape)
        self.radius = rng.uniform(0.5, 4.0, shape)
        self.speed = rng.uniform(0.0, 8.0, shape)
        self.heading = rng.uniform(0.0, 2.0 * math.pi, shape)
        self.strength = rng.uniform(0.05, 0.4, shape)
        self.turn = np.random.default_rng(seed + 1)
        self.dtype = DISTURBANCE_DTYPE

    def frame(self, s: int) -> np.ndarray:
        vx = self.speed[s] * np.cos(self.heading[s])
        vz = self.speed[s] * np.sin(self.heading[s])
        out = np.zeros(self.x.shape[1], self.dtype)
        out["world_x"] = self.x[s]
        out["world_z"] = self.z[s]
        out["radius"] = self.radius[s]
        out["strength"] = self.strength[s]
        out["velocity_x"] = vx
        out["velocity_z"] = vz
        out["kind"] = 1  # continuous
        # advance: move, reflect at the margin, turn
        x = self.x[s] + vx * self.dt
        z = self.z[s] + vz * self.dt
        hx = (x < self.lo) | (x > self.hi)
        hz = (z < self.lo) | (z > self.hi)
        h = self.heading[s]
        h = np.where(hx, math.pi - h, h)
        h = np.where(hz, -h, h)
        self.x[s] = np.clip(x, self.lo, self.hi)
        self.z[s] = np.clip(z, self.lo, self.hi)
        self.heading[s] = h + self.turn.uniform(-0.4, 0.4, h.shape)
        return out


def serving_points(sets: int = 16, count: int = 4096, seed: int = 23,
                   extent: float = SERVE_FIELD_EXTENT) -> np.ndarray:
    """`sets` seeded (count, 2) float32 point sets uniform over the field."""
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, extent, (sets, count, 2)).astype(np.float32)


def poisson_arrivals(sessions: int, rate: float, duration: float, p_update: float = 0.5,
                     seed: int = 29):
    """A Poisson process of mean `rate` requests/s over `duration` s: sorted
    arrival times, the session of each, and whether it is an update (else a
    height query)."""
    rng = np.random.default_rng(seed)
    n = int(rng.poisson(rate * duration))
    times = np.sort(rng.uniform(0.0, duration, n))
    sess = rng.integers(0, sessions, n)
    upd = rng.random(n) < p_update
    return times, sess, upd
