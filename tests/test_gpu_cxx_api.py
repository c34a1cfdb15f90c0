"""The reference's C++ API (include/ocean/ocean.hpp, foam.hpp, cascade.hpp,
interaction.hpp) and its C header path (include/ocean/ocean.h), exercised by
native programs written against those headers and linked against
libocean_b200.so (tests/native/): the relink check of the drop-in boundary.

Bars, all bit for bit:
* ocean::Ocean frame buffers and sample_at against the oracle (which is
  pinned to the reference);
* ocean::FoamField after 30 frames against the oracle's FoamField run, and
  foam_at at the same points; coverage within 1e-12;
* ocean::CascadeStack::sample_at against the reference's own CascadeStack
  records (tests/golden/ref_cascade.npz), a level's buffers and queries
  against the oracle;
* WaterSurface over an Ocean equal to ocean_sample_combined, over a
  CascadeStack equal to the reference's composition of the two samples.
The C program checks the C ABI from C (four parallel_for dispatches per
update, NULL-handle no-ops, an interaction session).
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oceanlib_b200 as ob
import oracle as O
from oceanlib_b200 import workloads as W
from tests.native.build_native import build
from tests.test_oracle_pins import run_oracle_foam
from tests.workloads import CASCADE_CASE

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def load(d, name, cols=None):
    a = np.fromfile(d / name, dtype=np.float32)
    return a.reshape(-1, cols) if cols else a


def compose(s, e):
    """WaterSurface::sample_at's composition (src/interaction.cpp:863-900) in
    float32, one operation at a time."""
    f = np.float32
    out = s.copy()
    out[:, 0] = (s[:, 0] + e[:, 0]).astype(f)
    out[:, 8] = (s[:, 8] + e[:, 3]).astype(f)
    up = s[:, 4] > f(1e-6)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = (f(1.0) / s[:, 4]).astype(f)
        sx = ((-s[:, 3] * inv).astype(f) + e[:, 1]).astype(f)
        sz = ((-s[:, 5] * inv).astype(f) + e[:, 2]).astype(f)
        ln = np.sqrt((((sx * sx).astype(f) + (sz * sz).astype(f)).astype(f) + f(1.0)).astype(f)).astype(f)
        il = (f(1.0) / ln).astype(f)
    out[up, 3] = (-sx * il).astype(f)[up]
    out[up, 4] = il[up]
    out[up, 5] = (-sz * il).astype(f)[up]
    return out


def test_cxx_api_program_against_oracle_and_reference(cuda_device, tmp_path):
    exe = build()["ocean_api_check"]
    rng = np.random.default_rng(77)
    xz = rng.uniform(-90.0, 170.0, size=(257, 2)).astype(np.float32)
    xz.tofile(tmp_path / "xz.bin")
    g = np.load(GOLDEN / "ref_cascade.npz")
    g["xz"].astype(np.float32).tofile(tmp_path / "cascade_xz.bin")
    res = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    rep = dict(line.split(" = ", 1) for line in (tmp_path / "report.txt").read_text().splitlines())
    assert rep["done"] == "1"
    for key in ("height_at_matches_sample_at", "move_keeps_buffers", "c_handle_buffers_match",
                "invalid_size_throws", "foam_without_velocity_throws", "interaction_crater",
                "interaction_dt_ok", "interaction_recentered", "water_surface_matches_c_combined",
                "water_surface_height_is_sum"):
        assert rep[key] == "1", key
    assert float(rep["time_after_construction"]) == 0.0
    assert float(rep["time"]) == 3.25
    assert rep["hook_dispatches_per_update"] == "4"

    # Ocean: the frame and the queries.
    desc = ob.OceanDesc(size=64, patch_length=80.0, wind_speed=14.0, wind_direction=0.7, choppiness=1.3,
                        seed=4242, compute_velocity=True)
    d, n, v = O.update(desc, 3.25)
    assert np.array_equal(bits(load(tmp_path, "ocean_disp.bin", 4)), bits(d))
    assert np.array_equal(bits(load(tmp_path, "ocean_normal.bin", 4)), bits(n))
    assert np.array_equal(bits(load(tmp_path, "ocean_vel.bin", 4)), bits(v))
    assert np.array_equal(bits(load(tmp_path, "ocean_queries.bin", 10)),
                          bits(O.sample_many(64, 80.0, d, n, v, xz)))

    # FoamField: 30 frames at 60 Hz.
    dt = 1.0 / 60.0
    want = run_oracle_foam(desc, W.foam_desc(), [(k / 60.0, dt) for k in range(1, 31)])[-1]
    assert np.array_equal(bits(load(tmp_path, "foam.bin")), bits(want))
    assert rep["foam_size"] == "64" and rep["foam_last_substeps"] == "1"
    assert abs(float(rep["foam_coverage"]) - float(want.astype(np.float64).mean())) < 1e-12
    d30, n30, _ = O.update(desc, 30 / 60.0)
    assert np.array_equal(bits(load(tmp_path, "foam_at.bin")),
                          bits(O.foam_at_many(64, 80.0, d30, n30, want, xz)))
    assert float(rep["foam_cleared_coverage"]) == 0.0

    # CascadeStack: the reference's records, a level's frame and queries.
    levels, t, _ = CASCADE_CASE
    assert rep["cascade_levels"] == "3" and float(rep["cascade_time"]) == t
    assert float(rep["cascade_level_time"]) == t
    assert np.array_equal(bits(load(tmp_path, "cascade_queries.bin", 10)), bits(g["out"]))
    d2, n2, v2 = O.update(levels[2], t)
    assert np.array_equal(bits(load(tmp_path, "cascade_level2_disp.bin", 4)), bits(d2))
    assert np.array_equal(bits(load(tmp_path, "cascade_level2_queries.bin", 10)),
                          bits(O.sample_many(256, 25.0, d2, n2, v2, xz)))

    # WaterSurface over the cascade: the reference's composition of the
    # cascade sample and the interaction sample.
    frames = [O.update(l, t) for l in levels]
    cas = O.cascade_sample_many(levels, frames, xz)
    inter = load(tmp_path, "water_cascade_interaction.bin", 4)
    assert np.array_equal(bits(load(tmp_path, "water_cascade_queries.bin", 10)), bits(compose(cas, inter)))


def test_c_header_program_runs(cuda_device):
    exe = build()["c_header_check"]
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, f"check {res.returncode} failed: {res.stdout}{res.stderr}"
    assert "c header check ok" in res.stdout
