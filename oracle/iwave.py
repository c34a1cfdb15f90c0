"""Test infrastructure: iWave interaction field checkers.

* RefInteraction    - the reference's InteractionField through its C ABI
                      (oracle/_ref/libocean_ref.so).
* OracleInteraction - the field restated: ocean_oracle.c's step, finalize,
                      damping, source stamp and BFS, orchestrated here exactly
                      as InteractionField::update / recenter / set_obstruction
                      do (src/interaction.cpp:531-723).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import oracle, ref

_P = C.c_void_p
_bound = False


def _bind():
    global _bound
    if _bound:
        return
    o = oracle()
    sig = {
        "or_iwave_damping": (None, [C.c_uint32, C.c_float, C.c_uint32, C.c_float, _P, _P]),
        "or_iwave_step": (None, [C.c_uint32, C.c_uint32, C.c_size_t, _P, _P, _P, C.c_float, _P, _P]),
        "or_iwave_finalize": (None, [C.c_uint32, C.c_size_t, _P, _P, C.c_float, C.c_float, _P]),
        "or_iwave_inject": (None, [C.c_uint32, C.c_size_t, C.c_float, C.c_int32, C.c_int32, C.c_float,
                                   _P, C.c_float, C.c_float, _P, _P]),
        "or_iwave_nearest": (C.c_uint32, [C.c_uint32, _P, _P, _P]),
        "or_iwave_obstruction": (None, [C.c_uint32, C.c_size_t, _P, C.c_uint32, _P, C.c_int, _P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(o, name)
        f.restype = res
        f.argtypes = args
    if True:
        r = ref()
        rsig = {
            "oref_iwave_taps": (C.c_int, [C.c_uint32, C.c_double, C.c_double, _P, _P]),
            "oref_i_create": (_P, [_P, C.POINTER(C.c_int)]),
            "oref_i_destroy": (None, [_P]),
            "oref_i_desc_init": (None, [_P]),
            "oref_i_add": (None, [_P, _P]),
            "oref_i_update": (None, [_P, C.c_float]),
            "oref_i_recenter": (C.c_int, [_P, C.c_float, C.c_float]),
            "oref_i_set_obstruction": (None, [_P, _P]),
            "oref_i_buffers": (None, [_P, _P]),
            "oref_i_sample_many": (None, [_P, _P, C.c_uint64, _P]),
            "oref_i_fixed_dt": (C.c_float, [_P]),
            "oref_i_dt_limit": (C.c_float, [_P]),
            "oref_i_dispersion_error": (C.c_float, [_P]),
            "oref_i_energy": (C.c_double, [_P]),
            "oref_i_dropped": (C.c_uint64, [_P]),
            "oref_sample_combined_many": (None, [_P, _P, _P, C.c_uint64, _P]),
            "oref_i_time_updates": (C.c_double, [_P, _P, C.c_uint32, C.c_uint32, C.c_float]),
        }
        for name, (res, args) in rsig.items():
            f = getattr(r, name)
            f.restype = res
            f.argtypes = args
    _bound = True


def _bind_oracle_only():
    global _bound
    o = oracle()
    if getattr(o, "_iwave_bound", False):
        return
    try:
        _bind()
    except FileNotFoundError:
        # reference library absent: bind the oracle functions only
        sig = {
            "or_iwave_damping": (None, [C.c_uint32, C.c_float, C.c_uint32, C.c_float, _P, _P]),
            "or_iwave_step": (None, [C.c_uint32, C.c_uint32, C.c_size_t, _P, _P, _P, C.c_float, _P, _P]),
            "or_iwave_finalize": (None, [C.c_uint32, C.c_size_t, _P, _P, C.c_float, C.c_float, _P]),
            "or_iwave_inject": (None, [C.c_uint32, C.c_size_t, C.c_float, C.c_int32, C.c_int32, C.c_float,
                                       _P, C.c_float, C.c_float, _P, _P]),
            "or_iwave_nearest": (C.c_uint32, [C.c_uint32, _P, _P, _P]),
            "or_iwave_obstruction": (None, [C.c_uint32, C.c_size_t, _P, C.c_uint32, _P, C.c_int, _P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(o, name)
            f.restype = res
            f.argtypes = args
    o._iwave_bound = True


def ref_taps(radius: int, cell: float, depth: float):
    _bind()
    w = 2 * radius + 1
    taps = np.empty(w * w, np.float32)
    stats = np.empty(3, np.float64)
    assert ref().oref_iwave_taps(radius, cell, depth, taps.ctypes.data, stats.ctypes.data) == 0
    return taps, stats


def _c_desc(desc):
    from oceanlib_b200.abi import InteractionDescC

    d = InteractionDescC()
    ref().oref_i_desc_init(C.byref(d))
    for k in ("size", "extent", "kernel_radius", "damping", "absorb_cells", "fixed_dt",
              "max_substeps", "max_sources", "gravity", "obstruction"):
        setattr(d, k, getattr(desc, k))
    d.water_depth = desc.depth
    return d


class RefInteraction:
    """The reference InteractionField (its C ABI), same method names as
    oceanlib_b200.interaction.InteractionField."""

    def __init__(self, desc):
        _bind()
        self.desc = desc
        self._cd = _c_desc(desc)
        st = C.c_int(-1)
        self.h = ref().oref_i_create(C.byref(self._cd), C.byref(st))
        if not self.h:
            raise ValueError(f"reference rejected interaction descriptor ({st.value})")
        self.size = desc.size

    def add(self, d):
        ref().oref_i_add(self.h, C.byref(d.to_c()))

    def update(self, dt):
        ref().oref_i_update(self.h, dt)

    def recenter(self, x, z):
        return bool(ref().oref_i_recenter(self.h, x, z))

    def set_obstruction(self, mask):
        if mask is None:
            ref().oref_i_set_obstruction(self.h, None)
        else:
            m = np.ascontiguousarray(mask, np.uint8)
            ref().oref_i_set_obstruction(self.h, m.ctypes.data)

    def field(self) -> np.ndarray:
        from oceanlib_b200.abi import InteractionBuffers

        b = InteractionBuffers()
        ref().oref_i_buffers(self.h, C.byref(b))
        n = b.size * b.size
        return np.ctypeslib.as_array(b.field, shape=(4 * n,)).reshape(n, 4).copy()

    def sample_many(self, xz):
        xz = np.ascontiguousarray(xz, np.float32)
        out = np.empty((xz.shape[0], 4), np.float32)
        ref().oref_i_sample_many(self.h, xz.ctypes.data, xz.shape[0], out.ctypes.data)
        return out

    @property
    def fixed_dt(self):
        return ref().oref_i_fixed_dt(self.h)

    @property
    def dt_limit(self):
        return ref().oref_i_dt_limit(self.h)

    @property
    def dispersion_error(self):
        return ref().oref_i_dispersion_error(self.h)

    def energy(self):
        return ref().oref_i_energy(self.h)

    @property
    def dropped(self):
        return ref().oref_i_dropped(self.h)

    def close(self):
        if self.h:
            ref().oref_i_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OracleInteraction:
    """The field restated on the CPU. `taps`, `fixed_dt` come from the caller
    (the reference's builder or the library's) so this class checks the
    per-substep arithmetic only."""

    def __init__(self, desc, taps: np.ndarray, dt: float):
        _bind_oracle_only()
        self.desc = desc
        self.n = n = desc.size
        self.p = p = desc.kernel_radius
        self.cell = np.float32(np.float32(desc.extent) / np.float32(n))
        self.stride = (n + 2 * p + 15) & ~15
        self.rows = n + 2 * p
        self.dt = np.float32(dt)
        self.taps = np.ascontiguousarray(taps, np.float32)
        self.planes = [np.zeros(self.rows * self.stride, np.float32) for _ in range(2)]
        self.cur, self.old = 0, 1
        self.c1 = np.empty(n * n, np.float32)
        self.c2 = np.empty(n * n, np.float32)
        oracle().or_iwave_damping(n, desc.damping, desc.absorb_cells, self.dt, self.c1.ctypes.data,
                                  self.c2.ctypes.data)
        self.out = np.zeros((n * n, 4), np.float32)
        self.queue = []
        self.accum = 0.0
        self.origin = [0, 0]
        self.mask = np.zeros(n * n, np.uint8)
        self.has_mask = False
        self.solid = np.zeros(n * n, np.uint32)
        self.nearest = np.zeros(n * n, np.uint32)
        self.solid_count = 0
        self.last_substeps = 0
        self.finalize()

    def _ptr(self, which):
        off = (self.p * self.stride + self.p) * 4
        return self.planes[which].ctypes.data + off

    def add(self, d):
        if len(self.queue) >= self.desc.max_sources:
            return
        self.queue.append(d)

    def _inject(self, d, sub_time, scale):
        arr = np.array([d.world_x, d.world_z, d.radius, d.strength, d.velocity_y, d.velocity_x,
                        d.velocity_z], np.float32)
        oracle().or_iwave_inject(self.n, self.stride, self.cell, self.origin[0], self.origin[1],
                                 self.dt, arr.ctypes.data, sub_time, scale, self._ptr(self.cur),
                                 self._ptr(self.old))

    def substep(self):
        if self.has_mask and self.solid_count:
            oracle().or_iwave_obstruction(self.n, self.stride, self.solid.ctypes.data, self.solid_count,
                                          self.nearest.ctypes.data,
                                          1 if self.desc.obstruction == 1 else 0, self._ptr(self.cur))
        gdt2 = np.float32(np.float32(self.desc.gravity) * self.dt * self.dt)
        oracle().or_iwave_step(self.n, self.p, self.stride, self.taps.ctypes.data, self.c1.ctypes.data,
                               self.c2.ctypes.data, gdt2, self._ptr(self.cur), self._ptr(self.old))
        self.cur, self.old = self.old, self.cur

    def finalize(self):
        oracle().or_iwave_finalize(self.n, self.stride, self._ptr(self.cur), self._ptr(self.old),
                                   np.float32(np.float32(0.5) / self.cell),
                                   np.float32(np.float32(1.0) / self.dt), self.out.ctypes.data)

    def update(self, dt):
        # src/interaction.cpp:531-587
        dt = float(np.float32(dt)) if dt > 0 else 0.0
        self.accum += dt
        step = float(self.dt)
        steps = int(self.accum / step) if self.accum >= step else 0
        if steps > self.desc.max_substeps:
            steps = self.desc.max_substeps
            self.accum = 0.0
        else:
            self.accum -= steps * step
        self.last_substeps = steps
        if steps == 0:
            self.queue = [d for d in self.queue if d.kind == 0]
            return
        for s in range(steps):
            sub_time = np.float32(np.float32(s) * self.dt)
            for d in self.queue:
                if d.kind == 0:
                    if s == 0:
                        self._inject(d, 0.0, 1.0)
                else:
                    self._inject(d, sub_time, self.dt)
            self.substep()
        self.queue = []
        self.finalize()

    def set_obstruction(self, mask):
        if mask is None:
            self.mask[:] = 0
            self.has_mask = False
            self.solid_count = 0
            return
        self.mask[:] = np.asarray(mask, np.uint8).ravel()
        self.has_mask = True
        self._rebuild()

    def _rebuild(self):
        self.solid_count = 0
        if not self.has_mask:
            return
        self.solid_count = oracle().or_iwave_nearest(self.n, self.mask.ctypes.data, self.nearest.ctypes.data,
                                                     self.solid.ctypes.data)

    def recenter(self, wx, wz):
        # src/interaction.cpp:601-705
        half = np.float32(np.float32(0.5) * np.float32(self.desc.extent))
        tx = int(_lround(float((np.float32(wx) - half) / self.cell)))
        tz = int(_lround(float((np.float32(wz) - half) / self.cell)))
        dx, dz = tx - self.origin[0], tz - self.origin[1]
        if dx == 0 and dz == 0:
            return False
        self.origin = [tx, tz]
        n = self.n
        if abs(dx) >= n or abs(dz) >= n:
            for pl in self.planes:
                pl[:] = 0
            self.mask[:] = 0
        else:
            for which in (self.cur, self.old):
                g = self.planes[which].reshape(self.rows, self.stride)
                inner = g[self.p:self.p + n, self.p:self.p + n].copy()
                moved = np.zeros_like(inner)
                zs = slice(max(0, -dz), min(n, n - dz))
                xs = slice(max(0, -dx), min(n, n - dx))
                moved[zs, xs] = inner[zs.start + dz:zs.stop + dz, xs.start + dx:xs.stop + dx]
                g[self.p:self.p + n, self.p:self.p + n] = moved
            if self.has_mask:
                m = self.mask.reshape(n, n)
                moved = np.zeros_like(m)
                zs = slice(max(0, -dz), min(n, n - dz))
                xs = slice(max(0, -dx), min(n, n - dx))
                moved[zs, xs] = m[zs.start + dz:zs.stop + dz, xs.start + dx:xs.stop + dx]
                self.mask[:] = moved.ravel()
        self._rebuild()
        self.finalize()
        return True

    def state(self):
        n = self.n
        out = []
        for which in (self.cur, self.old):
            g = self.planes[which].reshape(self.rows, self.stride)
            out.append(g[self.p:self.p + n, self.p:self.p + n].copy().ravel())
        return out

    def set_state(self, cur, old):
        n = self.n
        for which, src in ((self.cur, cur), (self.old, old)):
            g = self.planes[which].reshape(self.rows, self.stride)
            g[self.p:self.p + n, self.p:self.p + n] = np.asarray(src, np.float32).reshape(n, n)
        self.finalize()


def _lround(v: float) -> int:
    # std::lround: half away from zero
    return int(math.floor(v + 0.5)) if v >= 0 else -int(math.floor(-v + 0.5))
