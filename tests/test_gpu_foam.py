"""GPU parity of the rest of ocean::FoamField on a persistent-foam batch:
foam_at, coverage, set_desc and clear (src/foam.cpp:254-313), against the
reference FoamField's own results (tests/golden/ref_foam.json), and the
reference's foam property tests (tests/test_foam.cpp:71-194) run on the
device: decay at the stated rate, advection by whole cells exact, a lap of
the patch returns the field bit for bit.

Bar: bit-exact for fields and foam_at; coverage within 1e-12 relative (the
reference sums in index order, the device in a fixed tree).
"""
import hashlib
import json
import math
from pathlib import Path

import numpy as np
import pytest

import oceanlib_b200 as ob
from tests.workloads import FOAM_CASE, FOAM_QUERY_FRAMES, FOAM_RETUNE, query_points

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


class Frames:
    """update_host of a one-ocean foam batch into reusable host arrays."""

    def __init__(self, batch, n):
        self.batch = batch
        self.disp = np.empty((n * n, 4), np.float32)
        self.nrm = np.empty_like(self.disp)
        self.vel = np.empty_like(self.disp)
        self.foam = np.empty(n * n, np.float32)

    def step(self, t, dt):
        self.batch.update_host([t], dt, self.disp, self.nrm, self.vel, self.foam)
        return self.foam


@pytest.fixture(autouse=True)
def _exact_level(cuda_device):
    ob.force_simd_level(None)
    yield
    ob.force_simd_level(None)


def test_foam_at_coverage_set_desc_and_clear_match_reference():
    g = json.loads((GOLDEN / "ref_foam.json").read_text())
    desc, foam, _, dt = FOAM_CASE
    first, second = FOAM_QUERY_FRAMES
    batch = ob.OceanBatch([desc], foam=foam)
    fr = Frames(batch, desc.size)
    for k in range(first):
        fr.step((k + 1) * dt, dt)
    assert sha(fr.foam) == g["field"]
    assert sha(batch.foam_at_many(0, query_points(desc, 4096))) == g["at"]
    assert abs(batch.foam_coverage(0) - g["coverage"]) <= 1e-12 * g["coverage"]

    batch.set_foam_desc(FOAM_RETUNE)
    kept = batch.foam_desc()
    assert kept.fixed_dt == np.float32(foam.fixed_dt) and kept.max_substeps == foam.max_substeps
    assert kept.decay == np.float32(FOAM_RETUNE.decay)
    for k, want in zip(range(first, first + second), g["retuned"]):
        fr.step((k + 1) * dt, dt)
        assert batch.last_foam_substeps == want["substeps"], k
        assert sha(fr.foam) == want["field"], k
    assert abs(batch.foam_coverage(0) - g["coverage_retuned"]) <= 1e-12 * g["coverage_retuned"]

    batch.foam_clear()
    assert batch.foam_coverage(0) == g["coverage_cleared"] == 0.0
    fr.step((first + second + 1) * dt, dt)
    assert sha(fr.foam) == g["after_clear"]
    batch.close()


def foam_ocean(n=128):
    # tests/test_foam.cpp:24-35
    return ob.OceanDesc(size=n, patch_length=200.0, wind_speed=16.0, choppiness=1.4, foam_threshold=0.9,
                        seed=31337, compute_velocity=True)


def test_foam_decays_at_the_stated_rate():
    # tests/test_foam.cpp:71-113: build foam, switch the source off, and the
    # coverage falls as exp(-decay t) with the ocean held still.
    fd = ob.FoamDesc(decay=0.5, source_gain=6.0, advect_scale=0.0)
    batch = ob.OceanBatch([foam_ocean()], foam=fd)
    fr = Frames(batch, 128)
    for _ in range(120):
        fr.step(20.0, 1.0 / 60.0)
    built = batch.foam_coverage(0)
    assert built > 1e-4
    batch.set_foam_desc(ob.FoamDesc(decay=0.5, source_gain=0.0, advect_scale=0.0))
    for _ in range(120):
        fr.step(20.0, 1.0 / 60.0)
    after = batch.foam_coverage(0)
    expected = built * math.exp(-0.5 * 2.0)
    assert abs(after / expected - 1.0) < 1e-3, (built, after, expected)
    assert after > 0.0
    batch.close()


def _drift_one_cell_per_step():
    cell = np.float32(200.0) / np.float32(128.0)
    dt = np.float32(1.0) / np.float32(60.0)
    return float(cell / dt), float(dt)


def test_foam_is_advected_exactly_by_whole_cells_and_wraps_after_a_lap():
    # tests/test_foam.cpp:115-194: a drift of exactly one cell per step is a
    # pure relabelling (bilinear weights 1 and 0), so 5 steps shift the field
    # by 5 cells bit for bit, and N steps bring it back to where it started.
    drift, dt = _drift_one_cell_per_step()
    for steps in (5, 128):
        fd = ob.FoamDesc(decay=0.0, source_gain=5.0, advect_scale=0.0, fixed_dt=dt)
        batch = ob.OceanBatch([foam_ocean()], foam=fd)
        fr = Frames(batch, 128)
        for _ in range(60):
            fr.step(20.0, dt)
        before = fr.foam.reshape(128, 128).copy()
        assert before.mean() > 1e-4
        batch.set_foam_desc(ob.FoamDesc(decay=0.0, source_gain=0.0, advect_scale=0.0, wind_drift_x=drift))
        for _ in range(steps):
            fr.step(20.0, dt)
        after = fr.foam.reshape(128, 128)
        assert np.array_equal(bits(after), bits(np.roll(before, steps, axis=1))), steps
        batch.close()


def test_foam_members_need_a_persistent_foam_batch():
    batch = ob.OceanBatch([foam_ocean(64)])
    for call in (batch.foam_clear, lambda: batch.foam_coverage(0),
                 lambda: batch.set_foam_desc(ob.FoamDesc()),
                 lambda: batch.foam_at_many(0, np.zeros((4, 2), np.float32))):
        with pytest.raises(ob.OceanError):
            call()
    batch.close()
