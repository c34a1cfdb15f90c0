"""Test infrastructure: persistent foam run in FP64, the yardstick for foam drift.

A FoamField (src/foam.cpp:89-139, :218-252) riding on an ocean whose frames
are computed in FP64 from the reference's FP32 evolved spectra: the same
definition as ``oracle.fp64_frame`` (the evolve stays the reference's FP32
arithmetic, everything after it - the inverse transforms, the finalize, the
foam source, the semi-Lagrangian step and its decay - runs in double). Frames
over many hundred steps make numpy too slow, so the transforms and the foam
step run in torch float64 on whatever device the caller names (a GPU in the
tests; the CPU works, slowly). The evolve is the C oracle's, evaluated on a
thread pool ahead of the device work.

Only tests/ use this module.
"""
from __future__ import annotations

import concurrent.futures as cf
import math

import numpy as np

from . import evolve, spectrum


class FoamAccumulator:
    """FoamField::update's substep rule (src/foam.cpp:218-252): a double
    accumulator with a relative epsilon, backlog discarded at max_substeps."""

    def __init__(self, fixed_dt: float, max_substeps: int):
        self.step = float(np.float32(fixed_dt))
        self.max = int(max_substeps)
        self.accum = 0.0

    def steps(self, dt: float) -> int:
        dt = float(np.float32(dt))
        if not dt > 0.0:
            dt = 0.0
        self.accum += dt
        eps = self.step * 1e-6
        s = int((self.accum + eps) / self.step) if self.accum + eps >= self.step else 0
        if s > self.max:
            s, self.accum = self.max, 0.0
        else:
            self.accum = max(0.0, self.accum - s * self.step)
        return s


def _frame64(torch, fields32: np.ndarray, n: int, lam: float, thr: float, device):
    """(foam source, velocity x, velocity z) of one frame in FP64 (N, N)."""
    f = torch.from_numpy(fields32).to(device=device, dtype=torch.float64)
    z = torch.complex(f[0::2], f[1::2]).reshape(-1, n, n)
    g = torch.fft.ifft2(z) * float(n * n)  # unnormalised inverse, sign +
    jxx, jzz, jxz = g[2].imag, g[3].real, g[3].imag
    axx = 1.0 + lam * jxx
    azz = 1.0 + lam * jzz
    axz = lam * jxz
    jac = axx * azz - axz * axz
    inv_thr = 1.0 / thr if thr > 1e-6 else 0.0
    src = torch.clamp((thr - jac) * inv_thr, 0.0, 1.0)
    return src, g[4].real, g[5].real


def _sample_wrap(torch, f, u, v, n: int):
    """Periodic bilinear fetch (src/foam.cpp:22-41) in FP64."""
    fu = torch.floor(u)
    fv = torch.floor(v)
    tu = u - fu
    tv = v - fv
    x0 = torch.remainder(fu.long(), n)
    z0 = torch.remainder(fv.long(), n)
    x1 = (x0 + 1) % n
    z1 = (z0 + 1) % n
    flat = f.reshape(-1)
    a = flat[z0 * n + x0]
    b = flat[z0 * n + x1]
    c = flat[z1 * n + x0]
    d = flat[z1 * n + x1]
    return a * (1 - tu) * (1 - tv) + b * tu * (1 - tv) + c * (1 - tu) * tv + d * tu * tv


def fp64_foam_run(desc, foam, frames: int, dt: float, checkpoints, device="cuda", threads: int = 8):
    """Frames k = 1 .. frames at t = k * dt, each followed by FoamField::update(dt);
    returns {k: foam plane (N*N,) float64} for k in checkpoints."""
    import torch

    n = desc.size
    tables = spectrum(desc)
    lam = float(np.float32(desc.choppiness))
    thr = float(np.float32(desc.foam_threshold))
    fixed = float(np.float32(foam.fixed_dt))
    decay = math.exp(-float(np.float32(foam.decay)) * fixed)
    gain = float(np.float32(foam.source_gain)) * fixed
    scale = float(np.float32(foam.advect_scale))
    drift_x = float(np.float32(foam.wind_drift_x))
    drift_z = float(np.float32(foam.wind_drift_z))
    inv_cell = 1.0 / (float(np.float32(desc.patch_length)) / n)
    zz, xx = torch.meshgrid(torch.arange(n, dtype=torch.float64, device=device),
                            torch.arange(n, dtype=torch.float64, device=device), indexing="ij")
    cur = torch.zeros((n, n), dtype=torch.float64, device=device)
    acc = FoamAccumulator(foam.fixed_dt, foam.max_substeps)
    want = set(int(c) for c in checkpoints)
    out = {}
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        ahead = 2 * threads
        pending = {k: ex.submit(evolve, desc, k * dt, tables) for k in range(1, min(frames, ahead) + 1)}
        for k in range(1, frames + 1):
            fields = pending.pop(k).result()
            if k + ahead <= frames:
                pending[k + ahead] = ex.submit(evolve, desc, (k + ahead) * dt, tables)
            src, vx_field, vz_field = _frame64(torch, fields, n, lam, thr, device)
            for _ in range(acc.steps(dt)):
                vx = vx_field * scale + drift_x
                vz = vz_field * scale + drift_z
                su = xx - vx * fixed * inv_cell
                sv = zz - vz * fixed * inv_cell
                f = _sample_wrap(torch, cur, su, sv, n)
                cur = torch.clamp(f * decay + src * gain, 0.0, 1.0)
            if k in want:
                out[k] = cur.reshape(-1).cpu().numpy().copy()
    return out
