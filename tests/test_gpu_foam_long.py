"""Config 2's full run: the 512^2 foam patch (250 m, 22 m/s, choppiness 1.5,
velocity on) with persistent foam for 1000 frames at dt = 1/60 s from t = 0.

* The FP32 form's foam plane is bit-identical to the reference FoamField's
  (src/foam.cpp:218-252) at frames 250, 500 and 1000: sha256 of the plane and
  its coverage, from tests/golden/ref_foam_long.json (made by the reference).
* The tensor-core form's foam drift over the run is stated against the FP32
  form and against an FP64 run (oracle/fp64_foam.py: the reference's FP32
  spectra, everything after them in double) as max-abs and mean-abs
  difference at each checkpoint, beside the FP32 form's own drift against
  FP64. Bar: the tensor form drifts from FP64 by no more than twice the FP32
  form's drift in the mean, and by under 1e-3 anywhere.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import oceanlib_b200 as ob
from oceanlib_b200 import abi
from tests.workloads import FOAM_LONG_CASE, FOAM_LONG_CHECKPOINTS

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_form(form):
    desc, foam, frames, dt = FOAM_LONG_CASE
    cells = desc.size * desc.size
    batch = ob.OceanBatch([desc], foam=foam, form=form)
    disp = np.empty((cells, 4), np.float32)
    nrm = np.empty_like(disp)
    vel = np.empty_like(disp)
    out = {}
    for k in range(1, frames + 1):
        if k in FOAM_LONG_CHECKPOINTS:
            fo = np.empty(cells, np.float32)
            batch.update_host([k * dt], dt, disp, nrm, vel, fo)
            assert batch.last_foam_substeps == 1
            out[k] = (fo, batch.foam_coverage(0))
        else:
            batch.update([k * dt], dt)
    batch.close()
    return out


def test_thousand_frames_foam_fp32_bit_exact_and_tensor_drift(cuda_device):
    from oracle.fp64_foam import fp64_foam_run

    golden = json.loads((GOLDEN / "ref_foam_long.json").read_text())
    desc, foam, frames, dt = FOAM_LONG_CASE
    assert golden["frames"] == frames
    exact = run_form(abi.OCEAN_FFT_EXACT)
    for k in FOAM_LONG_CHECKPOINTS:
        g = golden["checkpoints"][str(k)]
        fo, cov = exact[k]
        assert sha(fo) == g["sha"], f"frame {k}"
        assert abs(cov - g["coverage"]) < 1e-12, k
    tensor = run_form(abi.OCEAN_FFT_TENSOR)
    fp64 = fp64_foam_run(desc, foam, frames, dt, FOAM_LONG_CHECKPOINTS, device="cuda")
    rows = []
    for k in FOAM_LONG_CHECKPOINTS:
        e32 = exact[k][0].astype(np.float64)
        tc = tensor[k][0].astype(np.float64)
        ref = fp64[k]
        d_tc_32 = np.abs(tc - e32)
        d_tc_64 = np.abs(tc - ref)
        d_32_64 = np.abs(e32 - ref)
        rows.append((k, d_tc_32.max(), d_tc_32.mean(), d_tc_64.max(), d_tc_64.mean(), d_32_64.max(),
                     d_32_64.mean(), ref.mean()))
        assert d_tc_64.mean() <= 2.0 * d_32_64.mean() + 1e-9, k
        assert d_tc_64.max() < 1e-3, k
    print("\nfoam drift over the 1000-frame run (max-abs / mean-abs):")
    print("frame | tensor vs FP32 | tensor vs FP64 | FP32 vs FP64 | FP64 coverage")
    for k, a, b, c, d, e, f, cov in rows:
        print(f"{k:5d} | {a:.3e} / {b:.3e} | {c:.3e} / {d:.3e} | {e:.3e} / {f:.3e} | {cov:.6f}")
