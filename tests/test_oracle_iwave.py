"""Pins the iWave part of the oracle (oracle/ocean_oracle.c or_iwave_*,
orchestrated by oracle/iwave.py) against the reference InteractionField:
golden fields made by the reference (tests/golden/make_golden.py) and, when
the reference library is built here, a live run."""
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from oracle import iwave as OI
from tests.workloads import interaction_script, run_interaction

GOLDEN = Path(__file__).resolve().parent / "golden"


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_oracle_interaction_matches_reference_golden():
    g = np.load(GOLDEN / "ref_interaction.npz")
    desc, script, frames, dt = interaction_script()
    orc = OI.OracleInteraction(desc, g["taps"], float(g["fixed_dt"]))
    got = []
    run_interaction(orc, script, frames, dt, lambda f, fld: got.append(fld.out.copy()))
    for f in range(frames):
        assert np.array_equal(bits(got[f]), bits(g["fields"][f])), f"frame {f}"


def test_stencil_is_d4_symmetric_with_zero_sum():
    # tests/test_iwave_kernel.cpp: D4 symmetry and zero sum (symbol 0 at k = 0)
    g = np.load(GOLDEN / "ref_interaction.npz")
    taps = g["taps"].astype(np.float64)
    w = int(round(np.sqrt(taps.size)))
    t = taps.reshape(w, w)
    assert np.array_equal(t, t.T) and np.array_equal(t, t[::-1, :]) and np.array_equal(t, t[:, ::-1])
    assert abs(t.sum()) < 1e-5 * np.abs(t).max()
    # dispersion error bound at P = 6 (tests/test_iwave_kernel.cpp:170)
    assert g["stats"][2] < 0.15


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
def test_oracle_interaction_matches_live_reference_dirichlet_and_clamp():
    from oceanlib_b200.interaction import Disturbance, InteractionDesc

    desc = InteractionDesc(size=64, extent=20.0, kernel_radius=4, absorb_cells=8, obstruction=1,
                           max_substeps=3)
    cell = float(np.float32(desc.extent) / np.float32(desc.size))
    taps, _ = OI.ref_taps(desc.kernel_radius, cell, desc.depth)
    r = OI.RefInteraction(desc)
    orc = OI.OracleInteraction(desc, taps, r.fixed_dt)
    mask = np.zeros((64, 64), np.uint8)
    mask[10:20, 30:34] = 1
    for fld in (r, orc):
        fld.set_obstruction(mask)
        fld.add(Disturbance(world_x=6.0, world_z=7.0, radius=0.5, strength=0.4))
        fld.update(1.0 / 60.0)
        fld.update(0.2)  # clamped to max_substeps
        fld.add(Disturbance(world_x=9.0, world_z=5.0, radius=0.7, strength=0.1, kind=1, velocity_x=3.0))
        fld.update(1.0 / 30.0)
        fld.recenter(12.0, 8.0)
        fld.update(1.0 / 60.0)
    assert np.array_equal(bits(r.field()), bits(orc.out))


def _stamp_arguments(desc, script, frames, dt):
    """Every e^-u argument the scripted run's source stamps evaluate
    (src/interaction.cpp:322-378, float arithmetic in the reference's order),
    collected by running the oracle with its inject call observed."""
    import math

    f32 = np.float32
    args = []
    real = OI.OracleInteraction._inject

    def observe(self, d, sub_time, scale):
        cell = f32(self.cell)
        radius = f32(d.radius)
        sigma = radius if radius > f32(0.25) * cell else f32(0.25) * cell
        inv2s2 = f32(f32(1.0) / (f32(2.0) * sigma * sigma))
        wx = f32(f32(d.world_x) + f32(f32(d.velocity_x) * f32(sub_time)))
        wz = f32(f32(d.world_z) + f32(f32(d.velocity_z) * f32(sub_time)))
        gx = f32(f32(wx - f32(f32(self.origin[0]) * cell)) / cell)
        gz = f32(f32(wz - f32(f32(self.origin[1]) * cell)) / cell)
        rad = int(math.ceil(f32(f32(4.0) * sigma) / cell))
        fx, fz = int(math.floor(gx)), int(math.floor(gz))
        x0, x1 = max(0, fx - rad), min(self.n - 1, fx + rad)
        z0, z1 = max(0, fz - rad), min(self.n - 1, fz + rad)
        if x1 >= x0 and z1 >= z0:
            px = ((np.arange(x0, x1 + 1, dtype=f32) + f32(0.5)).astype(f32) - gx).astype(f32)
            pz = ((np.arange(z0, z1 + 1, dtype=f32) + f32(0.5)).astype(f32) - gz).astype(f32)
            r2 = ((px * px)[None, :].astype(f32) + (pz * pz)[:, None].astype(f32)).astype(f32)
            r2 = ((r2 * cell).astype(f32) * cell).astype(f32)
            args.append((r2 * inv2s2).astype(f32).ravel())
        return real(self, d, sub_time, scale)

    g = np.load(GOLDEN / "ref_interaction.npz")
    orc = OI.OracleInteraction(desc, g["taps"], float(g["fixed_dt"]))
    orc._inject = observe.__get__(orc)
    run_interaction(orc, script, frames, dt)
    return np.concatenate(args)


def test_reference_expf_rounds_to_nearest_on_the_scripted_stamps():
    # The device's stamps take e^-u in double precision rounded once to float
    # (correctly rounded). The reference calls the host libm's expf, which
    # rounds to nearest except on a small fraction of arguments. On every
    # argument the scripted run's stamps evaluate the two agree, which is why
    # the GPU test can compare that run bit for bit.
    import ctypes
    import ctypes.util

    libm = ctypes.CDLL(ctypes.util.find_library("m"))
    libm.expf.restype = ctypes.c_float
    libm.expf.argtypes = [ctypes.c_float]
    desc, script, frames, dt = interaction_script()
    u = _stamp_arguments(desc, script, frames, dt)
    assert u.size > 10_000
    host = np.array([libm.expf(float(-x)) for x in u], np.float32)
    rounded = np.exp(-u.astype(np.float64)).astype(np.float32)
    assert np.array_equal(bits(host), bits(rounded))
