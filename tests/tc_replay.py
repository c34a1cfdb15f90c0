"""A numpy replay of the tensor-core DFT form's arithmetic (CPU, test only).

It follows csrc/tc_dft.cuh step by step for the 512-point four-step DFT
(512 = 16 x 32): each operand row scaled so its maximum lies in
[2^29, 2^30), cut into four signed 8-bit digits (halves rounded up), the
DFT matrices at 2^30 likewise; the digit-pair levels 0..3 summed exactly
(float64 matrix products of integers below 2^22 are exact) and combined in
FP32 as the engine does; the FP32 twiddle step Z = Y W, either with each
product and the sum rounded (three roundings) or by Kahan's difference of
products (about one); then the 2-D frame (rows, FP32 intermediate, columns)
and the FP32 finalize. Used to check the precision design of the tensor
form against FP64 without a GPU. Fused multiply-adds are emulated in float64
and rounded once to FP32 (a product of two FP32 values is exact in float64).
"""
from __future__ import annotations

import numpy as np

import oracle as O

_SCALE = np.array([2.0 ** 24, 2.0 ** 16, 2.0 ** 8, 1.0])


def _f32(a):
    return np.asarray(a, np.float64).astype(np.float32).astype(np.float64)


def _fma32(a, b, c):
    return _f32(np.asarray(a, np.float64) * np.asarray(b, np.float64) + np.asarray(c, np.float64))


def _digits_int(q):
    """Signed 8-bit digits of integers |q| < 2^31 (halves up), as float64."""
    d0 = (q + (1 << 23)) >> 24
    r = q - (d0 << 24)
    d1 = (r + (1 << 15)) >> 16
    r = r - (d1 << 16)
    d2 = (r + (1 << 7)) >> 8
    d3 = r - (d2 << 8)
    return np.stack([d0, d1, d2, d3], -1).astype(np.float64)


def _digits_operand(x):
    """The engine's operand split of FP32 values x (float64 array): the nearest
    integer of the remaining value at each weight, halves up (y + 1/2 rounded
    once to FP32, then floor), exact residuals."""
    def nearest_half_up(v, s):
        return np.floor(_f32(v * s + 0.5))
    t0 = nearest_half_up(x, 2.0 ** -24)
    x1 = _fma32(t0, -2.0 ** 24, x)
    t1 = nearest_half_up(x1, 2.0 ** -16)
    x2 = _fma32(t1, -2.0 ** 16, x1)
    t2 = nearest_half_up(x2, 2.0 ** -8)
    x3 = _fma32(t2, -2.0 ** 8, x2)
    t3 = nearest_half_up(x3, 1.0)
    return np.stack([t0, t1, t2, t3], -1)


def _dft_matrix_digits(npt: int) -> np.ndarray:
    """Real block DFT matrix [[C, -S], [S, C]] (rows = outputs) at 2^30, digits."""
    k2 = 2 * npt
    j = np.arange(k2)[:, None]
    k = np.arange(k2)[None, :]
    qo, kk, p, nn = j // npt, j % npt, k // npt, k % npt
    ang = 2.0 * np.pi * ((nn * kk) % npt) / npt
    v = np.where(qo == p, np.cos(ang), np.where(qo == 0, -np.sin(ang), np.sin(ang)))
    return _digits_int(np.rint(v * 2.0 ** 30).astype(np.int64))


_B1 = _dft_matrix_digits(16)
_B3 = _dft_matrix_digits(32)
_TWC = np.cos(2.0 * np.pi * np.arange(256) / 512).astype(np.float32).astype(np.float64)
_TWS = np.sin(2.0 * np.pi * np.arange(256) / 512).astype(np.float32).astype(np.float64)


def _gemm(a, b):
    """The engine's exact digit-slice GEMM of rows a (FP32 values) with the
    digit matrix b, levels 0..3 combined in FP32 largest first."""
    m = np.abs(a).max(axis=1)
    ex = np.where(m > 0, np.floor(np.log2(np.where(m > 0, m, 1.0))), 0).astype(np.int64)
    e = np.where(m > 0, 29 - ex, 0)
    ad = _digits_operand(_f32(a * (2.0 ** e)[:, None]))
    lv = []
    for L in range(4):
        d = np.zeros((a.shape[0], b.shape[0]))
        for i in range(L + 1):
            d += ad[:, :, i] @ b[:, :, L - i].T
        lv.append(d * (2.0 ** (18 - 8 * L - e))[:, None])
    y = _f32(lv[0] + lv[1])  # each weighted level is exact
    y = _f32(y + lv[2])
    return _f32(y + lv[3])


def _dft512(x: np.ndarray, kahan: bool) -> np.ndarray:
    shape = x.shape
    xs = x.reshape(-1, 16, 32)  # [sequence, n1, n2]
    a1 = np.concatenate([xs.real.transpose(0, 2, 1), xs.imag.transpose(0, 2, 1)], axis=2).reshape(-1, 32)
    y = _gemm(a1, _B1).reshape(-1, 32, 32)  # [sequence, n2, (re k1 | im k1)]
    yr, yi = y[:, :, :16], y[:, :, 16:]
    e = np.arange(32)[:, None] * np.arange(16)[None, :]
    wr, wi = _TWC[e & 255], _TWS[e & 255]
    neg = (e & 256) != 0
    wr, wi = np.where(neg, -wr, wr), np.where(neg, -wi, wi)
    if kahan:
        def dop(a, b, c, d):
            w = _f32(c * d)
            return _f32(_fma32(a, b, -w) + _fma32(-c, d, w))
        zr, zi = dop(yr, wr, yi, wi), dop(yr, wi, -yi, wr)
    else:
        zr = _f32(_f32(yr * wr) - _f32(yi * wi))
        zi = _f32(_f32(yr * wi) + _f32(yi * wr))
    a3 = np.concatenate([zr.transpose(0, 2, 1), zi.transpose(0, 2, 1)], axis=2).reshape(-1, 64)
    xo = _gemm(a3, _B3).reshape(-1, 16, 64)  # [sequence, k1, (re k2 | im k2)]
    return (xo[:, :, :32] + 1j * xo[:, :, 32:]).transpose(0, 2, 1).reshape(shape)


def frame(desc, t: float, kahan: bool = True) -> dict:
    """displacement (x, y, z) and normal (x, y, z, w) of one 512^2 frame as the
    tensor form computes them (float32 arrays, (N, N, 3) and (N, N, 4))."""
    n = desc.size
    assert n == 512, "the tensor-core form is built for N = 512"
    f = O.evolve(desc, t).astype(np.float64)
    planes = f.shape[0] // 2
    z = (f[0::2] + 1j * f[1::2]).reshape(planes, n, n)
    rows = _dft512(z, kahan)  # along x; the intermediate is FP32
    g = np.swapaxes(_dft512(np.swapaxes(rows, 1, 2).copy(), kahan), 1, 2)
    gr, gi = g.real.astype(np.float32), g.imag.astype(np.float32)
    h, dx, dz, hx, hz, jxx, jzz, jxz = gr[0], gi[0], gr[1], gi[1], gr[2], gi[2], gr[3], gi[3]
    lam = np.float32(desc.choppiness)
    one = np.float32(1.0)
    axx = one + lam * jxx
    azz = one + lam * jzz
    axz = lam * jxz
    jac = axx * azz - axz * axz
    nx = -(hx * azz - axz * hz)
    ny = jac
    nz = -(axx * hz - hx * axz)
    ln2 = nx * nx + ny * ny + nz * nz
    inv = np.where(ln2 > 0, one / np.sqrt(np.where(ln2 > 0, ln2, one)), np.float32(0))
    return {"displacement": np.stack([lam * dx, h, lam * dz], -1),
            "normal": np.stack([nx * inv, ny * inv, nz * inv, jac], -1)}


def channel_errors(got: dict, ref: dict) -> dict:
    """max |e| / RMS of the FP64 frame per channel."""
    out = {}
    for k in got:
        for c in range(got[k].shape[-1]):
            r = ref[k][..., c]
            out[f"{k}.{'xyzw'[c]}"] = float(np.abs(got[k][..., c].astype(np.float64) - r).max()
                                            / np.sqrt(np.mean(r * r)))
    return out
