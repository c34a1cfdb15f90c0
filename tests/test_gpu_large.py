"""GPU parity at N = 2048 and 4096, the reference's largest sizes
(src/ocean.cpp:28-59), which run the three-pass schedule (rows, columns in
place, finalize) instead of the persistent frame kernel.

Bar: bit-exact, as at the other sizes. 4096^2 frames and every h0 table are
checked against sha256 digests of the reference's own output bytes
(tests/golden/ref_hashes.json, which the parity suite also walks); 2048^2
frames, persistent foam and the ensemble against the oracle; the fast (FMA)
form within max-abs 1e-5 x field RMS per output channel.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import oceanlib_b200 as ob
import oracle as O
from oceanlib_b200 import abi
from oceanlib_b200.serve import OceanServer
from tests.test_oracle_pins import run_oracle_foam
from tests.workloads import desc_from_json

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
FAST_TOL = 1e-5  # max-abs error / field RMS, per output channel (fast form)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def large_cases():
    golden = json.loads((GOLDEN / "ref_hashes.json").read_text())
    return [c for c in golden["cases"] if c["desc"]["size"] > 1024]


@pytest.fixture(autouse=True)
def _exact_level(cuda_device):
    ob.force_simd_level(None)
    yield
    ob.force_simd_level(None)


def test_large_h0_tables_and_frames_bit_exact_against_reference_digests():
    cases = large_cases()
    assert sorted({c["desc"]["size"] for c in cases}) == [2048, 4096]
    for case in cases:
        desc = desc_from_json(case["desc"])
        batch = ob.OceanBatch([desc])
        h0, _ = batch.read_spectrum(0)
        assert sha(h0) == case["h0"], desc.size
        cells = desc.size ** 2
        disp = np.empty((cells, 4), np.float32)
        nrm = np.empty_like(disp)
        vel = np.empty_like(disp) if desc.compute_velocity else None
        for fr in case["frames"]:
            batch.update_host([fr["t"]], 0.0, disp, nrm, vel)
            assert sha(disp) == fr["disp"], (desc.size, fr["t"])
            assert sha(nrm) == fr["normal"], (desc.size, fr["t"])
            if vel is not None:
                assert sha(vel) == fr["vel"], (desc.size, fr["t"])
        batch.close()


def test_2048_matches_oracle_with_and_without_velocity():
    for vel in (False, True):
        desc = ob.OceanDesc(size=2048, patch_length=1500.0, wind_speed=13.0, wind_direction=0.3,
                            choppiness=1.6, seed=31 + vel, compute_velocity=vel)
        oc = ob.Ocean(desc)
        oc.update(123.456)
        b = oc.buffers()
        od, on, ov = O.update(desc, 123.456)
        assert np.array_equal(bits(b["displacement"]), bits(od)), vel
        assert np.array_equal(bits(b["normal"]), bits(on)), vel
        if vel:
            assert np.array_equal(bits(b["velocity"]), bits(ov))
        oc.close()


def test_2048_fast_form_within_tolerance():
    desc = ob.OceanDesc(size=2048, patch_length=1800.0, wind_speed=17.0, choppiness=1.2, seed=8,
                        compute_velocity=True)
    b = ob.OceanBatch([desc], form=abi.OCEAN_FFT_FAST)
    cells = desc.size ** 2
    disp = np.empty((cells, 4), np.float32)
    nrm = np.empty_like(disp)
    vel = np.empty_like(disp)
    b.update_host([40.0], 0.0, disp, nrm, vel)
    b.close()
    od, on, ov = O.update(desc, 40.0)
    for name, got, ref in (("disp", disp, od), ("normal", nrm, on), ("vel", vel, ov)):
        for ch in range(4):
            err = float(np.abs(got[:, ch].astype(np.float64) - ref[:, ch]).max())
            rms = float(np.sqrt(np.mean(ref[:, ch].astype(np.float64) ** 2)))
            if (name == "disp" and ch == 3) or rms == 0.0:
                # foam (a clamped ramp, mostly 0) and the zero velocity w
                assert err <= FAST_TOL, (name, ch, err)
            else:
                assert err <= FAST_TOL * rms, (name, ch, err / rms)


def test_2048_persistent_foam_matches_oracle_foam_steps():
    # The finalize pass fuses the first substep; the second frame's dt of
    # 2.5 fixed steps runs two (one fused, one stand-alone).
    desc = ob.OceanDesc(size=2048, patch_length=900.0, wind_speed=22.0, choppiness=1.5, seed=7,
                        compute_velocity=True)
    foam = ob.FoamDesc()
    dts = (1.0 / 60.0, 2.5 / 60.0)
    batch = ob.OceanBatch([desc], foam=foam)
    cells = desc.size ** 2
    disp = np.empty((cells, 4), np.float32)
    nrm, vel = np.empty_like(disp), np.empty_like(disp)
    fo = np.empty(cells, np.float32)
    frames = [(sum(dts[:k + 1]), dt) for k, dt in enumerate(dts)]
    got = []
    for t, dt in frames:
        batch.update_host([t], dt, disp, nrm, vel, fo)
        got.append((fo.copy(), batch.last_foam_substeps))
    batch.close()
    ref = run_oracle_foam(desc, foam, frames)
    assert [s for _, s in got] == [1, 2]
    for k, (f, _) in enumerate(got):
        assert np.array_equal(bits(f), bits(ref[k])), k
    assert float(got[-1][0].max()) > 0.0  # the case does make foam


def test_2048_batch_chunking_and_mixed_size_ensemble():
    descs = [ob.OceanDesc(size=2048, patch_length=1000.0 + 100.0 * k, wind_speed=9.0 + 4.0 * k,
                          seed=50 + k) for k in range(3)]
    cells = 2048 * 2048
    outs = []
    for chunk in (1, 3):
        batch = ob.OceanBatch(descs, chunk=chunk)
        d = np.empty((3, cells, 4), np.float32)
        n = np.empty_like(d)
        batch.update_host([5.0, 6.0, 7.0], 0.0, d, n)
        outs.append((d, n))
        batch.close()
    assert np.array_equal(bits(outs[0][0]), bits(outs[1][0]))
    assert np.array_equal(bits(outs[0][1]), bits(outs[1][1]))
    # An ensemble holding a 2048^2 ocean beside smaller ones.
    small = ob.OceanDesc(size=256, patch_length=300.0, wind_speed=12.0, seed=3)
    ens = ob.OceanEnsemble([small, descs[1], small], autotune=True)
    ens.update(6.0)
    ens.synchronize()
    d1, n1 = ens.read(1)
    ens.close()
    assert np.array_equal(bits(d1), bits(outs[0][0][1]))
    assert np.array_equal(bits(n1), bits(outs[0][1][1]))


def test_serving_rejects_sizes_above_1024():
    # The serving loop batches sessions into persistent frame launches.
    srv = OceanServer()
    with pytest.raises(ValueError):
        srv.open_session(ob.OceanDesc(size=2048, patch_length=1000.0))
    srv.close()
