"""The persistent kernel's task plans (0 default; 1 single-row tasks at
N = 256 and 512, 64 lanes a sequence with single-row tasks at N = 1024) and
intermediate ring depths (2 or 3 oceans in flight) and both publish timings
of a finished row task: every combination gives
the reference's bits, with and without velocity and with persistent foam,
and the batch autotuner keeps a combination that exists."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import oceanlib_b200 as ob
import oracle as O
from oceanlib_b200 import workloads as W
from tests.workloads import FOAM_CASE

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(autouse=True)
def _device(cuda_device):
    ob.force_simd_level(None)
    yield


@pytest.mark.parametrize("n", [256, 512, 1024])
@pytest.mark.parametrize("velocity", [False, True])
def test_every_plan_is_bit_exact(n, velocity):
    descs = [ob.OceanDesc(size=n, patch_length=0.6 * n + 40.0, wind_speed=13.0 + k, wind_direction=0.5 * k,
                          choppiness=1.1, seed=70 + k, compute_velocity=velocity) for k in range(3)]
    batch = ob.OceanBatch(descs)
    assert batch.plan_count == 2
    cells = n * n
    assert batch.deferred_publish == velocity  # the default: deferred with velocity
    for plan, slots, defer in ((1, 3, True), (1, 2, False), (0, 2, True), (0, 3, False)):
        batch.set_plan(plan)
        batch.set_ring_slots(slots)
        batch.set_deferred_publish(defer)
        assert batch.plan == plan and batch.ring_slots == slots and batch.deferred_publish == defer
        disp = np.empty((3 * cells, 4), np.float32)
        nrm = np.empty_like(disp)
        vel = np.empty_like(disp) if velocity else None
        batch.update_host([21.5], 0.0, disp, nrm, vel)
        for k, d in enumerate(descs):
            od, on, ov = O.update(d, 21.5)
            sl = slice(k * cells, (k + 1) * cells)
            assert np.array_equal(bits(disp[sl]), bits(od)), (n, plan, k)
            assert np.array_equal(bits(nrm[sl]), bits(on)), (n, plan, k)
            if velocity:
                assert np.array_equal(bits(vel[sl]), bits(ov)), (n, plan, k)
    with pytest.raises(ValueError):
        batch.set_plan(2)
    with pytest.raises(ValueError):
        batch.set_ring_slots(4)
    with pytest.raises(ValueError):
        batch.set_ring_slots(1)  # one slot: the queue would not be deadlock-free
    batch.close()


def test_single_row_plan_with_persistent_foam_matches_reference_foamfield():
    # The foam patch's first 24 frames under plan 1 (single-row tasks) give
    # the reference FoamField's bits, frame by frame.
    golden = json.loads((GOLDEN / "ref_hashes.json").read_text())["foam"]
    desc, foam, _, dt = FOAM_CASE
    cells = desc.size * desc.size
    batch = ob.OceanBatch([desc], foam=foam)
    batch.set_plan(1)
    disp = np.empty((cells, 4), np.float32)
    nrm = np.empty_like(disp)
    vel = np.empty_like(disp)
    fo = np.empty(cells, np.float32)
    for k in range(24):
        batch.update_host([(k + 1) * dt], dt, disp, nrm, vel, fo)
        assert sha(fo) == golden["hashes"][k], k
    batch.close()


def test_batch_autotuner_keeps_an_existing_plan():
    batch = ob.OceanBatch([W.bench_update_patch(512, seed=1337 + b) for b in range(8)])
    ms = batch.autotune_plan()
    assert len(ms) == 2 and all(m > 0 for m in ms)
    assert batch.plan == int(np.argmin(ms))
    assert batch.ring_slots in (2, 3)
    small = ob.OceanBatch([ob.OceanDesc(size=64, seed=3)])
    assert small.plan_count == 1 and len(small.autotune_plan()) == 1  # the publish timing is still a choice
    small.close()
    batch.close()


@pytest.mark.parametrize("defer", [False, True])
def test_publish_timing_many_oceans_many_frames(defer):
    # 24 oceans of 256^2 with velocity, 3 ring slots: the queue's counters
    # carry every ocean through the ring eight times a frame; four frames
    # under each publish timing give the oracle's bits for every ocean.
    n, count = 256, 24
    descs = [ob.OceanDesc(size=n, patch_length=150.0 + 7.0 * k, wind_speed=9.0 + 0.5 * k,
                          wind_direction=0.3 * k, choppiness=1.2, seed=300 + k, compute_velocity=True)
             for k in range(count)]
    batch = ob.OceanBatch(descs)
    batch.set_deferred_publish(defer)
    cells = n * n
    disp = np.empty((count * cells, 4), np.float32)
    nrm = np.empty_like(disp)
    vel = np.empty_like(disp)
    for f in range(4):
        t = 3.0 + 0.75 * f
        batch.update_host([t], 0.0, disp, nrm, vel)
        for k in (0, 7, 13, count - 1) if f < 3 else range(count):
            od, on, ov = O.update(descs[k], t)
            sl = slice(k * cells, (k + 1) * cells)
            assert np.array_equal(bits(disp[sl]), bits(od)), (defer, f, k)
            assert np.array_equal(bits(nrm[sl]), bits(on)), (defer, f, k)
            assert np.array_equal(bits(vel[sl]), bits(ov)), (defer, f, k)
    batch.close()
