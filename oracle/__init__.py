"""Test infrastructure: the CPU checkers for oceanlib_b200.

Two libraries, both built by oracle/Makefile:

* ``liboracle.so``           - ocean_oracle.c, a plain-C restatement of the
                               reference's per-frame path (the oracle).
* ``_ref/libocean_ref.so``   - the reference oceanlib itself, compiled from its
                               own sources, behind ref_shim.cpp. Used to pin the
                               oracle and as the timed CPU baseline.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package. Nothing in oceanlib_b200 may.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libocean_ref.so"
# The reference checkout: $OCEAN_REF_SRC, else a "reference" directory beside
# this repository.
REF_SRC = Path(os.environ.get("OCEAN_REF_SRC", str(HERE.parent.parent / "reference")))


class OrDesc(C.Structure):
    _fields_ = [
        ("n", C.c_uint32),
        ("patch_length", C.c_float),
        ("wind_speed", C.c_float),
        ("fetch", C.c_float),
        ("wind_direction", C.c_float),
        ("peak_enhancement", C.c_float),
        ("swell", C.c_float),
        ("small_wave_cutoff", C.c_float),
        ("gravity", C.c_float),
        ("depth", C.c_float),
        ("choppiness", C.c_float),
        ("foam_threshold", C.c_float),
        ("seed", C.c_uint64),
        ("velocity", C.c_int32),
    ]


class OrefFoamDesc(C.Structure):
    _fields_ = [(n, C.c_float) for n in
                ("decay", "source_gain", "advect_scale", "wind_drift_x", "wind_drift_z", "fixed_dt")] + \
               [("max_substeps", C.c_uint32), ("thread_count", C.c_uint32)]


def build(quiet: bool = True) -> None:
    """Compile the oracle (and, when the reference sources are present, the
    reference library) in place."""
    cmd = ["make", "-s", "-C", str(HERE), f"REF={REF_SRC}"]
    subprocess.run(cmd, check=True, capture_output=quiet)


_oracle: Optional[C.CDLL] = None
_ref: Optional[C.CDLL] = None

_F = C.POINTER(C.c_float)
_P = C.c_void_p


def oracle() -> C.CDLL:
    global _oracle
    if _oracle is None:
        if not ORACLE_SO.exists():
            build()
        l = C.CDLL(str(ORACLE_SO))
        sig = {
            "or_pcg32_fill": (None, [C.c_uint64, C.c_uint64, C.c_uint32, _P]),
            "or_mix64": (C.c_uint64, [C.c_uint64]),
            "or_row_gaussians": (None, [C.c_uint64, C.c_uint32, C.c_uint32, _P]),
            "or_build_spectrum": (None, [C.POINTER(OrDesc), _P]),
            "or_evolve": (None, [C.POINTER(OrDesc), _P, C.c_double, _P]),
            "or_fft_1d": (None, [C.c_uint32, _P, _P, C.c_int]),
            "or_fft_2d": (None, [C.c_uint32, _P, _P, C.c_int]),
            "or_finalize": (None, [C.POINTER(OrDesc), _P, _P, _P, _P]),
            "or_update": (None, [C.POINTER(OrDesc), _P, C.c_double, _P, _P, _P, _P]),
            "or_sample_many": (None, [C.c_uint32, C.c_float, _P, _P, _P, _P, C.c_uint64, _P]),
            "or_cascade_sample_many": (None, [C.c_uint32, _P, _P, _P, _P, _P, _P, C.c_uint64, C.c_int,
                                              C.c_float, _P]),
            "or_foam_step": (None, [C.c_uint32] + [C.c_float] * 7 + [_P, _P, _P, _P]),
            "or_foam_at_many": (None, [C.c_uint32, C.c_float, _P, _P, _P, _P, C.c_uint64, _P]),
            "or_dft2d_points": (None, [C.c_uint32, _P, _P, C.c_uint32, _P, _P, _P, _P]),
            "or_dft2d_full": (None, [C.c_uint32, _P, _P, _P, _P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _oracle = l
    return _oracle


def ref_available() -> bool:
    if REF_SO.exists():
        return True
    if (REF_SRC / "src" / "ocean.cpp").exists():
        try:
            build()
        except Exception:
            return False
    return REF_SO.exists()


def ref() -> C.CDLL:
    """The reference library (raises if it was never built)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(f"{REF_SO} not built (reference sources absent)")
        l = C.CDLL(str(REF_SO))
        sig = {
            "oref_c_create": (_P, [_P, C.POINTER(C.c_int)]),
            "oref_c_destroy": (None, [_P]),
            "oref_c_update": (None, [_P, C.c_double]),
            "oref_c_get_buffers": (None, [_P, _P]),
            "oref_c_get_velocity": (_F, [_P]),
            "oref_c_height_at": (C.c_float, [_P, C.c_float, C.c_float]),
            "oref_c_sample_ex": (None, [_P, C.c_float, C.c_float, _P]),
            "oref_c_sample_many": (None, [_P, _P, C.c_uint64, _P]),
            "oref_c_desc_init": (None, [_P]),
            "oref_c_force_simd_level": (C.c_char_p, [C.c_char_p]),
            "oref_c_simd_level": (C.c_char_p, []),
            "oref_stage_create": (_P, [_P]),
            "oref_stage_destroy": (None, [_P]),
            "oref_stage_tables": (None, [_P, _P]),
            "oref_stage_evolve": (None, [_P, C.c_double]),
            "oref_stage_fft": (None, [_P]),
            "oref_stage_plane_count": (C.c_int, [_P]),
            "oref_stage_get_fields": (None, [_P, _P]),
            "oref_stage_set_fields": (None, [_P, _P]),
            "oref_stage_finalize": (None, [_P, _P, _P, _P]),
            "oref_fft_1d": (None, [C.c_uint32, _P, _P, C.c_int]),
            "oref_fft_2d": (None, [C.c_uint32, _P, _P, C.c_int]),
            "oref_pcg32": (None, [C.c_uint64, C.c_uint64, C.c_uint32, _P]),
            "oref_row_gaussians": (None, [C.c_uint64, C.c_uint32, C.c_uint32, _P]),
            "oref_foam_create": (_P, [_P, C.POINTER(OrefFoamDesc), C.POINTER(C.c_int)]),
            "oref_foam_destroy": (None, [_P]),
            "oref_foam_update": (None, [_P, C.c_float]),
            "oref_foam_data": (_F, [_P]),
            "oref_foam_last_substeps": (C.c_uint32, [_P]),
            "oref_foam_coverage": (C.c_double, [_P]),
            "oref_foam_at": (C.c_float, [_P, C.c_float, C.c_float]),
            "oref_foam_clear": (None, [_P]),
            "oref_foam_set_desc": (C.c_int, [_P, C.POINTER(OrefFoamDesc)]),
            "oref_cascade_create": (_P, [_P, C.c_uint32, C.POINTER(C.c_int)]),
            "oref_cascade_destroy": (None, [_P]),
            "oref_cascade_update": (None, [_P, C.c_double]),
            "oref_cascade_sample_many": (None, [_P, _P, C.c_uint64, _P]),
            "oref_time_updates": (C.c_double, [_P, _P, C.c_uint32, C.c_uint32, C.c_double,
                                               C.c_double, C.c_float]),
            "oref_hardware_concurrency": (C.c_uint32, []),
            "oref_pack_rgba16": (None, [_P, _P, _P, C.c_uint64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _ref = l
    return _ref


# ---------------------------------------------------------------------------
# Descriptor plumbing. `desc` is any object with the OceanDesc attribute names
# used by oceanlib_b200.OceanDesc (size, patch_length, wind_speed, ...).
# ---------------------------------------------------------------------------
def or_desc(desc) -> OrDesc:
    d = OrDesc()
    d.n = desc.size
    d.patch_length = desc.patch_length
    d.wind_speed = desc.wind_speed
    d.fetch = desc.fetch
    d.wind_direction = desc.wind_direction
    d.peak_enhancement = desc.peak_enhancement
    d.swell = desc.swell
    d.small_wave_cutoff = desc.small_wave_cutoff
    d.gravity = desc.gravity
    d.depth = desc.depth
    d.choppiness = desc.choppiness
    d.foam_threshold = desc.foam_threshold
    d.seed = desc.seed
    d.velocity = 1 if desc.compute_velocity else 0
    return d


def c_desc_bytes(desc) -> C.Array:
    """The reference's `ocean_desc` for `desc`, built through the reference's
    own ocean_desc_init, as raw bytes (96 on LP64)."""
    from oceanlib_b200.abi import OceanDescC  # layout only

    d = OceanDescC()
    ref().oref_c_desc_init(C.byref(d))
    d.size = desc.size
    d.patch_length = desc.patch_length
    s = d.spectrum
    s.wind_speed = desc.wind_speed
    s.fetch = desc.fetch
    s.wind_direction = desc.wind_direction
    s.peak_enhancement = desc.peak_enhancement
    s.swell = desc.swell
    s.small_wave_cutoff = desc.small_wave_cutoff
    s.gravity = desc.gravity
    d.water_depth = desc.depth
    d.choppiness = desc.choppiness
    d.foam_threshold = desc.foam_threshold
    d.seed = desc.seed
    d.compute_velocity = 1 if desc.compute_velocity else 0
    d.thread_count = getattr(desc, "thread_count", 0)
    return d


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


# ---------------------------------------------------------------------------
# Oracle (C restatement) helpers
# ---------------------------------------------------------------------------
def spectrum(desc) -> np.ndarray:
    """(8, N*N) float32 tables: h0_re, h0_im, h0c_re, h0c_im, omega, kx, kz, k_inv."""
    n = desc.size
    t = np.empty((8, n * n), dtype=np.float32)
    d = or_desc(desc)
    oracle().or_build_spectrum(C.byref(d), t.ctypes.data)
    return t


def update(desc, t: float, tables: Optional[np.ndarray] = None):
    """One frame on the CPU oracle -> (disp (N*N,4), normal (N*N,4), velocity or None)."""
    n = desc.size
    if tables is None:
        tables = spectrum(desc)
    d = or_desc(desc)
    planes = 12 if desc.compute_velocity else 8
    fields = np.empty((planes, n * n), dtype=np.float32)
    disp = np.empty((n * n, 4), dtype=np.float32)
    normal = np.empty((n * n, 4), dtype=np.float32)
    vel = np.empty((n * n, 4), dtype=np.float32) if desc.compute_velocity else None
    oracle().or_update(C.byref(d), tables.ctypes.data, float(t), fields.ctypes.data,
                       disp.ctypes.data, normal.ctypes.data, _ptr(vel))
    return disp, normal, vel


def evolve(desc, t: float, tables: Optional[np.ndarray] = None) -> np.ndarray:
    n = desc.size
    if tables is None:
        tables = spectrum(desc)
    d = or_desc(desc)
    fields = np.empty((12 if desc.compute_velocity else 8, n * n), dtype=np.float32)
    oracle().or_evolve(C.byref(d), tables.ctypes.data, float(t), fields.ctypes.data)
    return fields


def fft_2d(re: np.ndarray, im: np.ndarray, sign: int = +1):
    re = np.ascontiguousarray(re, dtype=np.float32).copy()
    im = np.ascontiguousarray(im, dtype=np.float32).copy()
    oracle().or_fft_2d(int(round(np.sqrt(re.size))), re.ctypes.data, im.ctypes.data, sign)
    return re, im


def fft_1d(re: np.ndarray, im: np.ndarray, sign: int = +1):
    re = np.ascontiguousarray(re, dtype=np.float32).copy()
    im = np.ascontiguousarray(im, dtype=np.float32).copy()
    oracle().or_fft_1d(re.size, re.ctypes.data, im.ctypes.data, sign)
    return re, im


def sample_many(n: int, patch_length: float, disp, normal, vel, xz: np.ndarray) -> np.ndarray:
    xz = np.ascontiguousarray(xz, dtype=np.float32)
    out = np.empty((xz.shape[0], 10), dtype=np.float32)
    oracle().or_sample_many(n, patch_length, disp.ctypes.data, normal.ctypes.data, _ptr(vel),
                            xz.ctypes.data, xz.shape[0], out.ctypes.data)
    return out


def cascade_sample_many(levels, frames, xz: np.ndarray, iterations: int = 4,
                        tolerance: float = 0.0) -> np.ndarray:
    """CascadeStack::sample_at (src/cascade.cpp:80-153) at the points xz
    (count x 2) over `levels` (descriptors) with their frames [(disp, normal,
    velocity or None)], each level inverted with `iterations` fixed-point
    steps stopping once both coordinates move by <= tolerance (0: never).
    iterations=4, tolerance=0 is the reference. (count, 10) float32."""
    k = len(levels)
    pts = np.ascontiguousarray(xz, dtype=np.float32).reshape(-1, 2)
    keep = [tuple(np.ascontiguousarray(a, np.float32) if a is not None else None for a in f) for f in frames]
    ns = (C.c_uint32 * k)(*[d.size for d in levels])
    ls = (C.c_float * k)(*[d.patch_length for d in levels])
    arr = lambda j: (C.c_void_p * k)(*[(f[j].ctypes.data if f[j] is not None else None) for f in keep])
    out = np.empty((pts.shape[0], 10), dtype=np.float32)
    oracle().or_cascade_sample_many(k, ns, ls, arr(0), arr(1), arr(2), pts.ctypes.data, pts.shape[0],
                                    int(iterations), float(tolerance), out.ctypes.data)
    return out


def foam_step(n, cell, dt, decay, gain, scale, drift_x, drift_z, disp, vel, cur) -> np.ndarray:
    nxt = np.empty(n * n, dtype=np.float32)
    oracle().or_foam_step(n, cell, dt, decay, gain, scale, drift_x, drift_z, disp.ctypes.data,
                          vel.ctypes.data, np.ascontiguousarray(cur, np.float32).ctypes.data,
                          nxt.ctypes.data)
    return nxt


def foam_at_many(n: int, patch_length: float, disp, normal, foam, xz: np.ndarray) -> np.ndarray:
    """FoamField::foam_at (src/foam.cpp:291-305) at the points xz (count x 2)."""
    pts = np.ascontiguousarray(xz, dtype=np.float32).reshape(-1, 2)
    d = np.ascontiguousarray(disp, np.float32)
    nm = np.ascontiguousarray(normal, np.float32)
    f = np.ascontiguousarray(foam, np.float32)
    out = np.empty(pts.shape[0], np.float32)
    oracle().or_foam_at_many(n, patch_length, d.ctypes.data, nm.ctypes.data, f.ctypes.data, pts.ctypes.data,
                             pts.shape[0], out.ctypes.data)
    return out


def dft_points(re: np.ndarray, im: np.ndarray, xs, ys):
    """FP64 direct inverse DFT of one complex field at points (xs[i], ys[i])."""
    n = int(round(np.sqrt(re.size)))
    xs = np.ascontiguousarray(xs, dtype=np.uint32)
    ys = np.ascontiguousarray(ys, dtype=np.uint32)
    o_re = np.empty(xs.size, dtype=np.float64)
    o_im = np.empty(xs.size, dtype=np.float64)
    oracle().or_dft2d_points(n, np.ascontiguousarray(re, np.float32).ctypes.data,
                             np.ascontiguousarray(im, np.float32).ctypes.data, xs.size,
                             xs.ctypes.data, ys.ctypes.data, o_re.ctypes.data, o_im.ctypes.data)
    return o_re, o_im


def fp64_fields(desc, t: float) -> np.ndarray:
    """The evolved spectra (or_evolve, FP32 as the reference builds them)
    inverse-transformed in FP64: (planes, N, N) complex128, unnormalised,
    sign + (src/core/fft.cpp). numpy's complex128 FFT stands in for the
    direct sum; dft_points gives the direct sum at chosen points to check it."""
    n = desc.size
    f = evolve(desc, t).astype(np.float64)
    planes = f.shape[0] // 2
    z = (f[0::2] + 1j * f[1::2]).reshape(planes, n, n)
    return np.fft.ifft2(z, axes=(1, 2)) * (n * n)


def fp64_frame(desc, t: float) -> dict:
    """One update's outputs in FP64 from fp64_fields, through the finalize
    arithmetic of src/core/evolve.cpp:238-327 (and :186-203 for velocity):
    displacement (lambda Dx, h, lambda Dz, foam), normal (n / |n|, J),
    velocity (ux, uy, uz, 0). Arrays (N, N, 4) float64."""
    g = fp64_fields(desc, t)
    h, dx = g[0].real, g[0].imag
    dz, hx = g[1].real, g[1].imag
    hz, jxx = g[2].real, g[2].imag
    jzz, jxz = g[3].real, g[3].imag
    lam = float(desc.choppiness)
    axx = 1.0 + lam * jxx
    azz = 1.0 + lam * jzz
    axz = lam * jxz
    jac = axx * azz - axz * axz
    nx = -(hx * azz - axz * hz)
    ny = jac
    nz = -(axx * hz - hx * axz)
    ln = np.sqrt(nx * nx + ny * ny + nz * nz)
    inv = np.where(ln > 0, 1.0 / np.where(ln > 0, ln, 1.0), 0.0)
    thr = float(desc.foam_threshold)
    foam = np.clip((thr - jac) * (1.0 / thr if thr > 1e-6 else 0.0), 0.0, 1.0)
    out = {"displacement": np.stack([lam * dx, h, lam * dz, foam], axis=-1),
           "normal": np.stack([nx * inv, ny * inv, nz * inv, jac], axis=-1)}
    if g.shape[0] > 4:
        out["velocity"] = np.stack([g[4].real, g[4].imag, g[5].real, np.zeros_like(h)], axis=-1)
    return out


def pack_rgba16(src: np.ndarray, alpha: Optional[np.ndarray] = None) -> np.ndarray:
    """The viewer's RGBA16F upload pack restated (examples/viewer/half.hpp:58-112):
    binary32 -> binary16 round-to-nearest-even, overflow to infinity, a NaN
    becomes sign | 0x7E00; alpha from `alpha` when given. (cells, 4) uint16."""
    src = np.ascontiguousarray(src, dtype=np.float32).reshape(-1, 4).copy()
    if alpha is not None:
        src[:, 3] = np.ascontiguousarray(alpha, dtype=np.float32).reshape(-1)
    with np.errstate(over="ignore"):
        h = src.astype(np.float16).view(np.uint16)
    nan = np.isnan(src)
    h[nan] = ((src.view(np.uint32)[nan] >> 16) & 0x8000).astype(np.uint16) | np.uint16(0x7E00)
    return h


def ref_pack_rgba16(src: np.ndarray, alpha: Optional[np.ndarray] = None) -> np.ndarray:
    """The reference's own scalar pack (examples/viewer/half.hpp:99-112)."""
    src = np.ascontiguousarray(src, dtype=np.float32).reshape(-1, 4)
    cells = src.shape[0]
    out = np.empty((cells, 4), np.uint16)
    a = None if alpha is None else np.ascontiguousarray(alpha, dtype=np.float32).reshape(-1)
    ref().oref_pack_rgba16(out.ctypes.data, src.ctypes.data, None if a is None else a.ctypes.data, cells)
    return out


def pcg32(seed: int, stream: int, count: int) -> np.ndarray:
    out = np.empty(count, dtype=np.uint32)
    oracle().or_pcg32_fill(seed, stream, count, out.ctypes.data)
    return out


def row_gaussians(seed: int, row: int, pairs: int) -> np.ndarray:
    out = np.empty(2 * pairs, dtype=np.float32)
    oracle().or_row_gaussians(seed, row, pairs, out.ctypes.data)
    return out


# ---------------------------------------------------------------------------
# Reference helpers
# ---------------------------------------------------------------------------
class RefOcean:
    """The reference ocean::Ocean behind its own C ABI."""

    def __init__(self, desc):
        self.desc = desc
        self._cd = c_desc_bytes(desc)
        st = C.c_int(-1)
        self.h = ref().oref_c_create(C.byref(self._cd), C.byref(st))
        if not self.h:
            raise ValueError(f"reference rejected descriptor (status {st.value})")
        self.n = desc.size

    def update(self, t: float) -> None:
        ref().oref_c_update(self.h, float(t))

    def buffers(self):
        from oceanlib_b200.abi import Buffers

        b = Buffers()
        ref().oref_c_get_buffers(self.h, C.byref(b))
        cells = self.n * self.n
        disp = np.ctypeslib.as_array(b.displacement, shape=(cells * 4,)).reshape(cells, 4).copy()
        normal = np.ctypeslib.as_array(b.normal, shape=(cells * 4,)).reshape(cells, 4).copy()
        v = ref().oref_c_get_velocity(self.h)
        vel = np.ctypeslib.as_array(v, shape=(cells * 4,)).reshape(cells, 4).copy() if v else None
        return disp, normal, vel

    def sample_many(self, xz: np.ndarray) -> np.ndarray:
        xz = np.ascontiguousarray(xz, dtype=np.float32)
        out = np.empty((xz.shape[0], 10), dtype=np.float32)
        ref().oref_c_sample_many(self.h, xz.ctypes.data, xz.shape[0], out.ctypes.data)
        return out

    def close(self):
        if self.h:
            ref().oref_c_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefFoam:
    """The reference ocean::FoamField over a RefOcean."""

    def __init__(self, ocean: RefOcean, foam_desc, thread_count: int = 0):
        d = OrefFoamDesc()
        for k in ("decay", "source_gain", "advect_scale", "wind_drift_x", "wind_drift_z", "fixed_dt"):
            setattr(d, k, getattr(foam_desc, k))
        d.max_substeps = foam_desc.max_substeps
        d.thread_count = thread_count
        st = C.c_int(-1)
        self.h = ref().oref_foam_create(ocean.h, C.byref(d), C.byref(st))
        if not self.h:
            raise ValueError("reference FoamField rejected")
        self.n = ocean.n
        self._ocean = ocean

    def update(self, dt: float) -> None:
        ref().oref_foam_update(self.h, dt)

    def data(self) -> np.ndarray:
        p = ref().oref_foam_data(self.h)
        return np.ctypeslib.as_array(p, shape=(self.n * self.n,)).copy()

    @property
    def last_substeps(self) -> int:
        return ref().oref_foam_last_substeps(self.h)

    def coverage(self) -> float:
        return ref().oref_foam_coverage(self.h)

    def foam_at_many(self, xz: np.ndarray) -> np.ndarray:
        pts = np.ascontiguousarray(xz, dtype=np.float32).reshape(-1, 2)
        return np.array([ref().oref_foam_at(self.h, float(x), float(z)) for x, z in pts], np.float32)

    def clear(self) -> None:
        ref().oref_foam_clear(self.h)

    def set_desc(self, foam_desc) -> None:
        d = OrefFoamDesc()
        for k in ("decay", "source_gain", "advect_scale", "wind_drift_x", "wind_drift_z", "fixed_dt"):
            setattr(d, k, getattr(foam_desc, k))
        d.max_substeps = foam_desc.max_substeps
        if ref().oref_foam_set_desc(self.h, C.byref(d)) != 0:
            raise ValueError("reference FoamField::set_desc rejected the descriptor")

    def close(self):
        if self.h:
            ref().oref_foam_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_stage(desc):
    """Reference internal stages: returns (tables (8,N*N), callable evolve, ...)."""
    cd = c_desc_bytes(desc)
    h = ref().oref_stage_create(C.byref(cd))
    return h


def ref_tables(desc) -> np.ndarray:
    h = ref_stage(desc)
    try:
        t = np.empty((8, desc.size * desc.size), dtype=np.float32)
        ref().oref_stage_tables(h, t.ctypes.data)
        return t
    finally:
        ref().oref_stage_destroy(h)


def ref_evolve_fields(desc, t: float, transform: bool = False) -> np.ndarray:
    h = ref_stage(desc)
    try:
        ref().oref_stage_evolve(h, float(t))
        if transform:
            ref().oref_stage_fft(h)
        planes = ref().oref_stage_plane_count(h)
        f = np.empty((planes, desc.size * desc.size), dtype=np.float32)
        ref().oref_stage_get_fields(h, f.ctypes.data)
        return f
    finally:
        ref().oref_stage_destroy(h)


def ref_pcg32(seed: int, stream: int, count: int) -> np.ndarray:
    out = np.empty(count, dtype=np.uint32)
    ref().oref_pcg32(seed, stream, count, out.ctypes.data)
    return out


def ref_fft_2d(re: np.ndarray, im: np.ndarray, sign: int = +1):
    re = np.ascontiguousarray(re, dtype=np.float32).copy()
    im = np.ascontiguousarray(im, dtype=np.float32).copy()
    ref().oref_fft_2d(int(round(np.sqrt(re.size))), re.ctypes.data, im.ctypes.data, sign)
    return re, im


def ref_fft_1d(re: np.ndarray, im: np.ndarray, sign: int = +1):
    re = np.ascontiguousarray(re, dtype=np.float32).copy()
    im = np.ascontiguousarray(im, dtype=np.float32).copy()
    ref().oref_fft_1d(re.size, re.ctypes.data, im.ctypes.data, sign)
    return re, im
