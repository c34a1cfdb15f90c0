"""GPU iWave interaction field through the C ABI.

Bars: stencil taps, timestep and stability limit bit-identical to the
reference's builder; stepping (stencil, damping, obstruction, finalize) and
recentering bit-exact against the oracle from the same state; the whole
scripted run with sources bit-exact against the reference. Source stamps take
the correctly rounded exponential (double precision, rounded once), which is
glibc's expf wherever glibc rounds to nearest, and a parallel double
reduction for the stamp mean, whose float value equals the reference's
sequential sum's.
"""
from pathlib import Path

import numpy as np
import pytest

import oceanlib_b200 as ob
from oceanlib_b200 import abi, workloads as W
from oceanlib_b200.interaction import (Disturbance, InteractionDesc, InteractionField,
                                       sample_combined_many)
from oracle import iwave as OI
from tests.workloads import interaction_script, run_interaction

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.fixture(autouse=True)
def _device(cuda_device):
    yield


def test_stencil_taps_and_limits_match_reference():
    g = np.load(GOLDEN / "ref_interaction.npz")
    desc, _, _, _ = interaction_script()
    f = InteractionField(desc)
    assert np.array_equal(bits(f.taps()), bits(g["taps"]))
    assert np.float32(f.fixed_dt) == g["fixed_dt"]
    assert np.float32(f.dt_limit) == g["dt_limit"]
    assert np.float32(f.dispersion_error) == g["dispersion_error"]
    f.close()


def _random_state(n, seed):
    rng = np.random.default_rng(seed)
    cur = (rng.standard_normal(n * n) * 0.05).astype(np.float32)
    old = (cur + rng.standard_normal(n * n) * 0.001).astype(np.float32)
    return cur, old


@pytest.mark.parametrize("obstruction", [None, abi.OCEAN_OBSTRUCTION_NEUMANN,
                                         abi.OCEAN_OBSTRUCTION_DIRICHLET])
def test_stepping_bit_exact_from_a_state(obstruction):
    desc = InteractionDesc(size=128, extent=32.0, kernel_radius=6, absorb_cells=12,
                           obstruction=obstruction or 0)
    f = InteractionField(desc)
    orc = OI.OracleInteraction(desc, f.taps(), f.fixed_dt)
    cur, old = _random_state(desc.size, 3)
    f.set_state(cur, old)
    orc.set_state(cur, old)
    if obstruction is not None:
        mask = np.zeros((128, 128), np.uint8)
        mask[30:50, 60:64] = 1
        mask[100:128, 0:10] = 1
        f.set_obstruction(mask)
        orc.set_obstruction(mask)
    for k in range(6):
        f.update(1.0 / 60.0 if k != 3 else 3.0 / 60.0)
        orc.update(1.0 / 60.0 if k != 3 else 3.0 / 60.0)
        assert f.last_substeps == orc.last_substeps
        assert np.array_equal(bits(f.buffers()["field"]), bits(orc.out)), k
    c2, o2 = f.get_state()
    oc, oo = orc.state()
    assert np.array_equal(bits(c2), bits(oc)) and np.array_equal(bits(o2), bits(oo))
    f.close()


def test_recenter_is_an_exact_integer_shift():
    desc = InteractionDesc(size=64, extent=16.0, kernel_radius=3, absorb_cells=4)
    f = InteractionField(desc)
    orc = OI.OracleInteraction(desc, f.taps(), f.fixed_dt)
    cur, old = _random_state(64, 8)
    f.set_state(cur, old)
    orc.set_state(cur, old)
    for target in ((10.0, 7.0), (3.2, 15.9), (200.0, -50.0)):
        moved = f.recenter(*target)
        assert moved == orc.recenter(*target)
        assert np.array_equal(bits(f.buffers()["field"]), bits(orc.out)), target
        b = f.buffers()
        assert b["origin_x"] == np.float32(orc.origin[0]) * orc.cell
    f.close()


def test_scripted_run_with_sources_bit_exact_against_reference():
    # Sources, obstruction, recentre and stepping over 12 frames: every word
    # of every frame equals the reference's. The stamps' exponential is the
    # correctly rounded one on the device; the reference's glibc expf rounds
    # to nearest at every stamp cell of this script (checked on the CPU by
    # tests/test_oracle_iwave.py), so the stamps agree bit for bit.
    g = np.load(GOLDEN / "ref_interaction.npz")
    desc, script, frames, dt = interaction_script()
    f = InteractionField(desc)
    got = []
    run_interaction(f, script, frames, dt, lambda k, fld: got.append(fld.buffers()["field"].copy()))
    for k in range(frames):
        same = bits(got[k]) == bits(g["fields"][k])
        assert same.all(), (k, int(np.count_nonzero(~same)), same.size)
    # queries on this field: single == batched, and close to the reference
    s = f.sample_many(g["xz"])
    one = f.sample_at(float(g["xz"][5, 0]), float(g["xz"][5, 1]))
    assert np.float32(one["height"]) == s[5, 0]
    assert np.array_equal(bits(s), bits(g["samples"]))
    assert abs(f.energy() - float(g["energy"])) <= 1e-10 * abs(float(g["energy"]))
    f.close()


def test_queue_overflow_and_zero_step_updates_keep_impulses():
    desc = InteractionDesc(size=64, extent=16.0, kernel_radius=3, absorb_cells=4, max_sources=2)
    f = InteractionField(desc)
    for k in range(5):
        f.add(Disturbance(world_x=8.0, world_z=8.0, kind=abi.OCEAN_SOURCE_IMPULSE))
    assert f.dropped == 3
    f.update(0.0)  # no step: impulses are kept
    assert f.last_substeps == 0
    f.update(1.0 / 60.0)
    assert f.last_substeps == 1
    assert np.abs(f.buffers()["field"][:, 0]).max() > 0.0
    f.update(10.0)
    assert f.last_clamped and f.last_substeps == desc.max_substeps
    f.close()


def test_combined_surface_composes_ocean_and_field():
    desc_o, t = W.single_patch_256()
    oc = ob.Ocean(desc_o)
    oc.update(t)
    f = InteractionField(InteractionDesc(size=128, extent=32.0))
    f.add(Disturbance(world_x=16.0, world_z=16.0, radius=1.0, strength=0.5))
    for _ in range(20):
        f.update(1.0 / 60.0)
    rng = np.random.default_rng(4)
    xz = rng.uniform(0.0, 32.0, (4096, 2)).astype(np.float32)
    comb = sample_combined_many(oc, f, xz)
    base = oc.sample_many(xz)
    e = f.sample_many(xz)
    # heights and vertical velocity add exactly; the normal composes via slopes
    f32 = np.float32
    assert np.array_equal(bits(comb[:, 0]), bits((base[:, 0] + e[:, 0]).astype(f32)))
    assert np.array_equal(bits(comb[:, 8]), bits((base[:, 8] + e[:, 3]).astype(f32)))
    up = base[:, 4] > f32(1e-6)
    inv = (f32(1.0) / base[:, 4]).astype(f32)
    sx = (-base[:, 3] * inv + e[:, 1]).astype(f32)
    sz = (-base[:, 5] * inv + e[:, 2]).astype(f32)
    il = (f32(1.0) / np.sqrt((sx * sx + sz * sz + f32(1.0)).astype(f32))).astype(f32)
    assert np.array_equal(bits(comb[up, 4]), bits(il[up]))
    assert np.array_equal(bits(comb[up, 3]), bits((-sx * il).astype(f32)[up]))
    # the single-point reference entry point agrees with the batch
    import ctypes as C

    one = abi.SurfaceEx()
    ob.lib().ocean_sample_combined(oc.handle, f.handle, float(xz[7, 0]), float(xz[7, 1]), C.byref(one))
    assert np.float32(one.height) == comb[7, 0]
    f.close()
    oc.close()


def _oracle_tables(mask):
    n = mask.shape[0]
    nearest = np.empty(n * n, np.uint32)
    solid = np.empty(n * n, np.uint32)
    count = OI.oracle().or_iwave_nearest(n, np.ascontiguousarray(mask, np.uint8).ctypes.data,
                                         nearest.ctypes.data, solid.ctypes.data)
    return solid[:count], nearest


@pytest.mark.parametrize("n", [64, 256])
def test_obstruction_tables_built_on_device_match_the_reference_bfs(n):
    # The device BFS (obstruction.cu) against the oracle's restatement of the
    # reference's queue BFS (src/interaction.cpp:255-292), table for table:
    # blobs, noise, a checkerboard, one fluid cell in a solid grid (n - 1 + n - 1
    # levels deep, so the order keys are re-ranked), an all-solid grid (no
    # fluid reachable) and an all-fluid one.
    rng = np.random.default_rng(n)
    masks = []
    m = np.zeros((n, n), np.uint8)
    for _ in range(6):
        x, z = rng.integers(0, n, 2)
        w, h = rng.integers(2, n // 3, 2)
        m[z:z + h, x:x + w] = 1
    masks.append(m)
    masks.append((rng.random((n, n)) < 0.45).astype(np.uint8))
    masks.append(((np.arange(n)[:, None] + np.arange(n)[None, :]) % 2).astype(np.uint8))
    one = np.ones((n, n), np.uint8)
    one[n // 3, (2 * n) // 3] = 0
    masks.append(one)
    masks.append(np.ones((n, n), np.uint8))
    masks.append(np.zeros((n, n), np.uint8))
    f = InteractionField(InteractionDesc(size=n, extent=float(n) / 4.0, kernel_radius=3, absorb_cells=4))
    for k, mask in enumerate(masks):
        f.set_obstruction(mask)
        solid, nearest = f.obstruction_tables()
        want_solid, want_nearest = _oracle_tables(mask)
        assert np.array_equal(solid, want_solid), k
        assert np.array_equal(nearest, want_nearest), k
    f.close()
