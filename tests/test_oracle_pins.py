"""Pins the CPU oracle (oracle/ocean_oracle.c) before anything trusts it.

* against the reference's own known answers (the PCG32 KAT of
  tests/test_rng.cpp:17-20 and the FFT-vs-DFT bound of tests/test_fft.cpp:166);
* against golden fixtures produced by the reference itself
  (tests/golden/make_golden.py, compiled from the reference's sources);
* live against the reference library when it is built here.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from oceanlib_b200 import workloads as W
from tests.workloads import (FOAM_CASE, FOAM_QUERY_FRAMES, HASH_CASES, QUERY_CASE, SMALL_CASES,
                             desc_from_json, query_points)

GOLDEN = Path(__file__).resolve().parent / "golden"


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_pcg32_known_answers():
    # seed 42, stream 54: the canonical pcg32 demo outputs (tests/test_rng.cpp:17-20)
    want = [0xA15C02B7, 0x7B47F409, 0xBA1D3330, 0x83D2F293,
            0xBFA4784B, 0xCBED606E, 0xBFC6A3AD, 0x812FFF6D]
    assert O.pcg32(42, 54, 8).tolist() == want
    r = W.Pcg32(42, 54)
    assert [r.next_u32() for _ in range(8)] == want
    # the vectorised generator continues the same stream
    r1, r2 = W.Pcg32(3, 0), W.Pcg32(3, 0)
    scalar = [r1.next_u32() for _ in range(10000)]
    assert r2.many_u32(10000).tolist() == scalar
    assert r1.next_u32() == r2.next_u32()


def test_oracle_matches_reference_small_grids():
    g = np.load(GOLDEN / "ref_small.npz")
    meta = json.loads(bytes(g["meta"]).decode())
    for i, m in enumerate(meta):
        desc = desc_from_json(m["desc"])
        tables = O.spectrum(desc)
        assert np.array_equal(bits(tables), bits(g[f"c{i}_tables"])), f"tables case {i}"
        for j, t in enumerate(m["times"]):
            d, n, v = O.update(desc, t, tables)
            assert np.array_equal(bits(d), bits(g[f"c{i}_t{j}_disp"])), (i, t)
            assert np.array_equal(bits(n), bits(g[f"c{i}_t{j}_normal"])), (i, t)
            if v is not None:
                assert np.array_equal(bits(v), bits(g[f"c{i}_t{j}_vel"])), (i, t)


def test_choppiness_zero_gives_unit_jacobian():
    # tests/test_simulation.cpp:275-296: lambda = 0 => J == 1 exactly.
    desc, times = SMALL_CASES[2]
    _, n, _ = O.update(desc, times[0])
    assert np.all(n[:, 3] == 1.0)


def test_oracle_matches_reference_hashes_full_size():
    # Sizes up to 2048 (a 4096^2 oracle frame takes tens of seconds; the GPU
    # suite checks those digests against the device directly).
    golden = json.loads((GOLDEN / "ref_hashes.json").read_text())
    for case in golden["cases"]:
        desc = desc_from_json(case["desc"])
        if desc.size > 2048:
            continue
        tables = O.spectrum(desc)
        assert sha(np.stack([tables[0], tables[1]], axis=1)) == case["h0"], desc
        for fr in case["frames"]:
            d, n, v = O.update(desc, fr["t"], tables)
            assert sha(d) == fr["disp"], (desc.size, fr["t"])
            assert sha(n) == fr["normal"], (desc.size, fr["t"])
            if v is not None:
                assert sha(v) == fr["vel"], (desc.size, fr["t"])


class FoamAccumulator:
    """FoamField::update's fixed-step accumulator (src/foam.cpp:218-252)."""

    def __init__(self, fixed_dt, max_substeps):
        self.step = float(np.float32(fixed_dt))
        self.max = max_substeps
        self.accum = 0.0

    def steps(self, dt):
        dt = float(np.float32(dt)) if dt > 0 else 0.0
        self.accum += dt
        eps = self.step * 1e-6
        s = int((self.accum + eps) / self.step) if self.accum + eps >= self.step else 0
        if s > self.max:
            s, self.accum = self.max, 0.0
        else:
            self.accum = max(0.0, self.accum - s * self.step)
        return s


def run_oracle_foam(desc, foam, frames):
    """The oracle's foam state after each (t, dt) frame, stepped as the
    reference's FoamField is (fixed substeps from an accumulator)."""
    n = desc.size
    tables = O.spectrum(desc)
    cur = np.zeros(n * n, np.float32)
    acc = FoamAccumulator(foam.fixed_dt, foam.max_substeps)
    fdt = np.float32(foam.fixed_dt)
    decay = np.exp(np.float32(-np.float32(foam.decay) * fdt), dtype=np.float32)
    gain = np.float32(np.float32(foam.source_gain) * fdt)
    cell = np.float32(np.float32(desc.patch_length) / np.float32(n))
    out = []
    for t, dt in frames:
        d, _, v = O.update(desc, t, tables)
        for _ in range(acc.steps(dt)):
            cur = O.foam_step(n, cell, fdt, decay, gain, foam.advect_scale, foam.wind_drift_x,
                              foam.wind_drift_z, d, v, cur)
        out.append(cur)
    return out


def test_oracle_foam_matches_reference():
    golden = json.loads((GOLDEN / "ref_hashes.json").read_text())["foam"]
    desc, foam, frames, dt = FOAM_CASE
    # 24 frames keep the CPU suite fast; the GPU test checks all of them.
    got = run_oracle_foam(desc, foam, [((k + 1) * dt, dt) for k in range(24)])
    for k in range(24):
        assert sha(got[k]) == golden["hashes"][k], k


def test_oracle_foam_at_and_coverage_match_reference():
    # FoamField::foam_at (src/foam.cpp:291-305) and coverage (:307-313) after
    # 30 frames of the foam patch, against the reference's own results.
    g = json.loads((GOLDEN / "ref_foam.json").read_text())
    desc, foam, _, dt = FOAM_CASE
    first, _ = FOAM_QUERY_FRAMES
    field = run_oracle_foam(desc, foam, [((k + 1) * dt, dt) for k in range(first)])[-1]
    assert sha(field) == g["field"]
    d, n, _ = O.update(desc, first * dt)
    at = O.foam_at_many(desc.size, desc.patch_length, d, n, field, query_points(desc, 4096))
    assert sha(at) == g["at"]
    # The reference sums in index order; any other order differs by rounding.
    assert abs(float(field.astype(np.float64).mean()) - g["coverage"]) <= 1e-12 * g["coverage"]


def test_oracle_queries_match_reference():
    g = np.load(GOLDEN / "ref_queries.npz")
    desc, t, count = QUERY_CASE
    d, n, v = O.update(desc, t)
    assert np.array_equal(g["xz"], query_points(desc, count))
    res = O.sample_many(desc.size, desc.patch_length, d, n, v, g["xz"])
    assert np.array_equal(bits(res), bits(g["out"]))


def test_fft_matches_fp64_direct_dft():
    # tests/test_fft.cpp:138-169: 2-D transform vs the O(N^4) direct sum < 1e-6
    # relative to the peak.
    rng = np.random.default_rng(5)
    n = 32
    re = rng.standard_normal(n * n).astype(np.float32)
    im = rng.standard_normal(n * n).astype(np.float32)
    fr, fi = O.fft_2d(re, im, +1)
    xs = np.tile(np.arange(n), n)
    ys = np.repeat(np.arange(n), n)
    dr, di = O.dft_points(re, im, xs, ys)
    err = np.sqrt((fr - dr) ** 2 + (fi - di) ** 2).max()
    scale = np.sqrt(dr ** 2 + di ** 2).max()
    assert err / scale < 1e-6


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
def test_oracle_matches_live_reference_random_descriptors():
    rng = np.random.default_rng(77)
    from oceanlib_b200 import OceanDesc

    for k in range(6):
        desc = OceanDesc(size=int(rng.choice([16, 32, 64, 128])),
                         patch_length=float(rng.uniform(20, 900)),
                         wind_speed=float(rng.uniform(0, 30)),
                         fetch=float(rng.uniform(1e3, 5e5)),
                         wind_direction=float(rng.uniform(-7, 7)),
                         peak_enhancement=float(rng.uniform(1, 7)),
                         swell=float(rng.uniform(0, 1)),
                         depth=float(rng.choice([0.0, 5.0, 40.0])),
                         choppiness=float(rng.uniform(0, 2)),
                         seed=int(rng.integers(0, 2 ** 63)),
                         compute_velocity=bool(k % 2))
        t = float(rng.uniform(0, 1e4))
        ro = O.RefOcean(desc)
        ro.update(t)
        rd, rn, rv = ro.buffers()
        d, n, v = O.update(desc, t)
        assert np.array_equal(bits(d), bits(rd))
        assert np.array_equal(bits(n), bits(rn))
        if v is not None:
            assert np.array_equal(bits(v), bits(rv))
        xz = rng.uniform(-2 * desc.patch_length, 2 * desc.patch_length, (256, 2)).astype(np.float32)
        assert np.array_equal(bits(ro.sample_many(xz)),
                              bits(O.sample_many(desc.size, desc.patch_length, d, n, v, xz)))


def oracle_cascade(levels, t, xz):
    """CascadeStack::sample_at (src/cascade.cpp:82-153) composed from the
    oracle's per-level queries, in float32, in the reference's order."""
    f32 = np.float32
    acc = {k: np.zeros(len(xz), f32) for k in ("h", "ox", "oz", "nx", "ny", "nz", "vx", "vy", "vz")}
    transparency = np.ones(len(xz), f32)
    for d in levels:
        disp, nrm, vel = O.update(d, t)
        s = O.sample_many(d.size, d.patch_length, disp, nrm, vel, xz)
        for k, col in (("h", 0), ("ox", 1), ("oz", 2), ("nx", 3), ("ny", 4), ("nz", 5),
                       ("vx", 7), ("vy", 8), ("vz", 9)):
            acc[k] = (acc[k] + s[:, col]).astype(f32)
        transparency = (transparency * (f32(1.0) - s[:, 6])).astype(f32)
    len2 = (acc["nx"] * acc["nx"] + acc["ny"] * acc["ny"] + acc["nz"] * acc["nz"]).astype(f32)
    out = np.zeros((len(xz), 10), f32)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = (f32(1.0) / np.sqrt(len2)).astype(f32)
    pos = len2 > 0
    out[:, 3] = np.where(pos, acc["nx"] * inv, f32(0.0))
    out[:, 4] = np.where(pos, acc["ny"] * inv, f32(1.0))
    out[:, 5] = np.where(pos, acc["nz"] * inv, f32(0.0))
    out[:, 0], out[:, 1], out[:, 2] = acc["h"], acc["ox"], acc["oz"]
    out[:, 6] = (f32(1.0) - transparency).astype(f32)
    out[:, 7], out[:, 8], out[:, 9] = acc["vx"], acc["vy"], acc["vz"]
    return out


def test_oracle_cascade_matches_reference():
    from tests.workloads import CASCADE_CASE

    g = np.load(GOLDEN / "ref_cascade.npz")
    levels, t, count = CASCADE_CASE
    got = oracle_cascade(levels, t, g["xz"])
    assert np.array_equal(bits(got), bits(g["out"]))


def test_pack_rgba16_matches_reference_viewer_pack():
    # examples/viewer/half.hpp: the oracle's RGBA16F pack against the sha256 of
    # the reference's own pack over every exponent, subnormals, infinities and
    # NaNs, with and without the separate alpha plane.
    from tests.workloads import pack_patterns

    golden = json.loads((GOLDEN / "ref_pack.json").read_text())
    src, alpha = pack_patterns()
    assert src.shape[0] == golden["texels"]
    assert sha(O.pack_rgba16(src)) == golden["plain"]
    assert sha(O.pack_rgba16(src, alpha)) == golden["alpha"]


def test_oracle_cascade_restatement_matches_reference():
    # The C restatement of CascadeStack::sample_at (or_cascade_sample_many)
    # at the reference's 4 fixed-point steps: the reference's own records.
    from tests.workloads import CASCADE_CASE

    g = np.load(GOLDEN / "ref_cascade.npz")
    levels, t, count = CASCADE_CASE
    frames = [O.update(d, t) for d in levels]
    got = O.cascade_sample_many(levels, frames, g["xz"], iterations=4, tolerance=0.0)
    assert np.array_equal(bits(got), bits(g["out"]))


def test_oracle_converged_inversion_is_a_fixed_point():
    # Config 3's converged mode (steps until both parameter coordinates move
    # by <= 1e-6 m, at most 64): where the surface has not folded the
    # iteration is a contraction, so 200 steps no longer move the answer
    # (float32 rounding aside), while 4 steps (the reference) still differ.
    from tests.workloads import CASCADE_CASE

    levels, t, _ = CASCADE_CASE
    frames = [O.update(d, t) for d in levels]
    xz = W.cascade_query_points(20_000)
    conv = O.cascade_sample_many(levels, frames, xz, iterations=64, tolerance=1e-6)
    more = O.cascade_sample_many(levels, frames, xz, iterations=200, tolerance=0.0)
    four = O.cascade_sample_many(levels, frames, xz, iterations=4, tolerance=0.0)
    dh = np.abs(conv[:, 0].astype(np.float64) - more[:, 0])
    assert np.quantile(dh, 0.999) < 1e-5
    assert np.abs(four[:, 0] - conv[:, 0]).max() > 0.0


def test_fp64_foam_run_tracks_the_fp32_foam():
    # The FP64 foam yardstick (oracle/fp64_foam.py) against the oracle's FP32
    # FoamField on a small choppy patch: the two stay within a few 1e-6.
    import oceanlib_b200 as ob
    from oracle.fp64_foam import fp64_foam_run

    desc = ob.OceanDesc(size=64, patch_length=60.0, wind_speed=20.0, choppiness=1.6, seed=21,
                        compute_velocity=True)
    foam = W.foam_desc()
    dt = 1.0 / 60.0
    f64 = fp64_foam_run(desc, foam, 40, dt, [10, 40], device="cpu", threads=4)
    f32 = run_oracle_foam(desc, foam, [((k + 1) * dt, dt) for k in range(40)])
    for k in (10, 40):
        err = np.abs(f32[k - 1].astype(np.float64) - f64[k])
        assert err.max() < 2e-5, (k, err.max())
        assert f32[k - 1].max() > 0.1  # the patch does foam
