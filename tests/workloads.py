"""Test cases shared by the golden-fixture generator and the tests."""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from oceanlib_b200 import OceanDesc, FoamDesc
from oceanlib_b200 import workloads as W


def desc_to_json(d: OceanDesc) -> dict:
    return dataclasses.asdict(d)


def desc_from_json(j: dict) -> OceanDesc:
    return OceanDesc(**j)


# Small grids: full arrays are stored. Covers every size class of the kernels'
# shape table below 128, velocity, finite depth, swell, choppiness 0 (J == 1
# exactly), a degenerate foam threshold and a large absolute time.
SMALL_CASES = [
    (OceanDesc(size=16, patch_length=50.0, wind_speed=8.0, seed=3), (0.0, 1.5, 97.25)),
    (OceanDesc(size=32, patch_length=100.0, wind_speed=12.0, wind_direction=0.4, seed=555,
               compute_velocity=True), (0.0, 4.0, 3600.0)),
    (OceanDesc(size=64, patch_length=200.0, wind_speed=12.0, depth=30.0, swell=0.6,
               choppiness=0.0, seed=11), (10.0,)),
    (OceanDesc(size=64, patch_length=80.0, wind_speed=20.0, choppiness=1.8, foam_threshold=0.0,
               seed=99, compute_velocity=True), (1e5,)),
]

# Full sizes: only sha256 of the reference's bytes is stored.
_s256, _t256 = W.single_patch_256()
HASH_CASES = [
    (_s256, (_t256, 0.0, 3600.0)),
    (W.bench_update_patch(512), (100.0, 100.0137, 1e4)),
    (W.foam_patch_512(), (0.0, 1.0 / 60.0, 1e3, 1e4, 1e5)),
    (OceanDesc(size=128, patch_length=150.0, wind_speed=15.0, depth=30.0, seed=2,
               compute_velocity=True), (5.0,)),
    (OceanDesc(size=1024, patch_length=1000.0, wind_speed=25.0, wind_direction=2.0, choppiness=1.2,
               seed=5), (42.0,)),
    # Above the persistent kernel's range: the three-pass schedule.
    (OceanDesc(size=2048, patch_length=2000.0, wind_speed=18.0, wind_direction=0.9, choppiness=1.4,
               seed=2048, compute_velocity=True), (7.5, 1e4)),
    (OceanDesc(size=4096, patch_length=4000.0, wind_speed=10.0, wind_direction=2.6, choppiness=0.9,
               seed=4096, compute_velocity=True), (3.0,)),
    (OceanDesc(size=4096, patch_length=600.0, wind_speed=21.0, wind_direction=-1.2, depth=40.0,
               seed=77), (250.0,)),
]

# Persistent foam on the foam patch: 120 frames at 60 Hz.
FOAM_CASE = (W.foam_patch_512(), W.foam_desc(), 120, 1.0 / 60.0)

# Config 2's full run: 1000 frames at 60 Hz from t = 0 (frame k at t = k/60,
# then FoamField::update(1/60)), foam checked at these frames.
FOAM_LONG_CASE = (W.foam_patch_512(), W.foam_desc(), 1000, 1.0 / 60.0)
FOAM_LONG_CHECKPOINTS = (250, 500, 1000)

# The rest of FoamField on the foam patch: foam_at and coverage after 30
# frames, then set_desc to FOAM_RETUNE for 20 more frames (fixed_dt and
# max_substeps given here differ from the field's and must be ignored), then
# clear() and one more frame.
FOAM_QUERY_FRAMES = (30, 20)
FOAM_RETUNE = FoamDesc(decay=1.2, source_gain=0.5, advect_scale=0.5, wind_drift_x=3.0, wind_drift_z=-2.0,
                       fixed_dt=1.0 / 30.0, max_substeps=1)

# World queries on the single 256 patch at t = 10.
QUERY_CASE = (_s256, _t256, 4096)

# Three 256^2 cascades (800 / 150 / 25 m, 30 m depth, velocity on) at t = 10,
# queried at the first 4096 points of the seeded uniform stream over the
# 800 m tile plus a few far / negative points.
CASCADE_CASE = (W.cascade_3x256(), 10.0, 4096)


def interaction_script():
    """A 128^2, 32 m interaction field driven for 12 frames at 60 Hz: an
    impulse, a moving continuous source, a second impulse, a Neumann
    obstruction block from frame 3 and a recentre at frame 8. Returns
    (desc, [(frame, action, args)]) with actions applied before each frame's
    update in list order."""
    from oceanlib_b200.interaction import Disturbance, InteractionDesc

    desc = InteractionDesc(size=128, extent=32.0, kernel_radius=6, absorb_cells=12)
    n = desc.size
    mask = np.zeros((n, n), np.uint8)
    mask[70:84, 40:52] = 1
    moving = Disturbance(world_x=16.0, world_z=16.0, radius=1.0, strength=0.2, velocity_y=-0.5,
                         velocity_x=2.0, velocity_z=-0.5, kind=1)
    script = [
        (0, "add", Disturbance(world_x=10.0, world_z=12.0, radius=0.6, strength=0.3)),
        (3, "obstruct", mask.ravel()),
        (5, "add", Disturbance(world_x=22.0, world_z=9.0, radius=0.8, strength=-0.2, velocity_y=0.4)),
        (8, "recenter", (18.0, 17.0)),
    ]
    for f in range(12):
        script.append((f, "add_moving", moving))
    script.sort(key=lambda a: (a[0], a[1] != "obstruct", a[1] != "recenter"))
    return desc, script, 12, 1.0 / 60.0


def run_interaction(field, script, frames, dt, on_frame=None):
    """Drive any object with add / update / set_obstruction / recenter."""
    by_frame = {}
    for f, action, arg in script:
        by_frame.setdefault(f, []).append((action, arg))
    for f in range(frames):
        for action, arg in by_frame.get(f, []):
            if action in ("add", "add_moving"):
                field.add(arg)
            elif action == "obstruct":
                field.set_obstruction(arg)
            elif action == "recenter":
                field.recenter(*arg)
        field.update(dt)
        if on_frame is not None:
            on_frame(f, field)


def cascade_points(count: int) -> np.ndarray:
    pts = W.cascade_query_points(count - 4)
    edge = np.array([[-5.0, -7.5], [1600.0, 2400.0], [0.0, 0.0], [799.999, 0.001]], np.float32)
    return np.concatenate([pts, edge]).astype(np.float32)


def query_points(desc: OceanDesc, count: int) -> np.ndarray:
    """Seeded points over three tiles (negative coordinates included) plus
    edge cases: cell corners, the tile seam, far-away points."""
    rng = np.random.default_rng(1234)
    L = desc.patch_length
    pts = rng.uniform(-1.5 * L, 1.5 * L, size=(count - 8, 2)).astype(np.float32)
    cell = L / desc.size
    edge = np.array([[0, 0], [L, L], [-L, 0], [cell, 2 * cell], [L - 1e-3, 0.5],
                     [1e4 * L, -1e4 * L], [-0.0, 0.0], [3 * cell, -5 * cell]], dtype=np.float32)
    return np.concatenate([pts, edge]).astype(np.float32)


def pack_patterns():
    """Float bit patterns for the RGBA16F pack: every upper half-word with a
    few low half-words (all exponents, subnormals, infinities, NaNs) plus
    seeded random words, as (texels, 4) float32, and a seeded alpha plane."""
    hi = np.arange(1 << 16, dtype=np.uint32) << 16
    lows = np.array([0, 1, 0x0FFF, 0x1000, 0x1001, 0x2000, 0x3000, 0xFFFF, 0x8000, 0x7FFF, 0xE000, 0xF000],
                    np.uint32)
    bits = (hi[:, None] | lows[None, :]).reshape(-1)
    rng = np.random.default_rng(2024)
    bits = np.concatenate([bits, rng.integers(0, 2 ** 32, 1 << 20, dtype=np.uint64).astype(np.uint32)])
    bits = bits[: len(bits) // 4 * 4]
    src = bits.view(np.float32).reshape(-1, 4)
    alpha = rng.standard_normal(src.shape[0]).astype(np.float32)
    return src, alpha
