"""oceanlib_b200 - the B200 (sm_100a) ocean library, Python host side.

Mirrors the reference's ocean::Ocean / OceanDesc interface (include/ocean/
ocean.hpp of DarshanVShah/oceanlib) over the C ABI in include/ocean_b200.h:

    desc = OceanDesc(size=256, patch_length=200.0, wind_speed=12.0)
    ocean = Ocean(desc)            # ValueError on a malformed descriptor
    ocean.update(10.0)             # absolute time; pure function of (seed, desc, t)
    b = ocean.buffers()            # numpy views of the RGBA32F host mirror
    ocean.height_at(3.0, 4.0)      # fixed-point inversion, on the GPU

and adds OceanBatch for many oceans per launch. All compute runs in
libocean_b200.so on the GPU; importing this package without the built library
raises, there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

from . import abi
from .abi import OceanDescC, FoamDescC, BatchDescC, SurfaceEx, DeviceBuffers

# The in-tree build; OCEANLIB_B200_LIBRARY names another build of the same
# library (e.g. one compiled with different flags) to load instead.
_LIB_PATH = Path(os.environ.get("OCEANLIB_B200_LIBRARY", str(Path(__file__).resolve().parent / "libocean_b200.so")))
_lib: Optional[C.CDLL] = None


class OceanError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} ({status})")


def lib() -> C.CDLL:
    """The loaded C-ABI library (loaded once, with every signature bound)."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise ImportError(
                f"{_LIB_PATH} is missing: build it with `python -m oceanlib_b200.build`")
        l = C.CDLL(str(_LIB_PATH))
        for name, (res, args) in abi.SIGNATURES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def library_path() -> Path:
    return _LIB_PATH


def status_string(status: int) -> str:
    return lib().ocean_status_string(status).decode()


def _check(status: int, what: str) -> None:
    if status != abi.OCEAN_OK:
        raise OceanError(status, what)


# ---------------------------------------------------------------------------
# Descriptors
# ---------------------------------------------------------------------------
@dataclass
class OceanDesc:
    """ocean::OceanDesc (include/ocean/ocean.hpp:39-130) flattened: the
    SpectrumDesc fields sit beside the grid fields."""

    size: int = 256
    patch_length: float = 200.0
    wind_speed: float = 10.0
    fetch: float = 100000.0
    wind_direction: float = 0.0
    peak_enhancement: float = 3.3
    swell: float = 0.0
    small_wave_cutoff: float = 0.5
    gravity: float = 9.81
    depth: float = 0.0
    choppiness: float = 1.0
    foam_threshold: float = 0.5
    seed: int = 1337
    compute_velocity: bool = False
    thread_count: int = 0

    def to_c(self) -> OceanDescC:
        d = OceanDescC()
        lib().ocean_desc_init(C.byref(d))
        d.size = self.size
        d.patch_length = self.patch_length
        s = d.spectrum
        s.wind_speed = self.wind_speed
        s.fetch = self.fetch
        s.wind_direction = self.wind_direction
        s.peak_enhancement = self.peak_enhancement
        s.swell = self.swell
        s.small_wave_cutoff = self.small_wave_cutoff
        s.gravity = self.gravity
        d.water_depth = self.depth
        d.choppiness = self.choppiness
        d.foam_threshold = self.foam_threshold
        d.seed = self.seed
        d.compute_velocity = 1 if self.compute_velocity else 0
        d.thread_count = self.thread_count
        return d


@dataclass
class FoamDesc:
    """ocean::FoamDesc (include/ocean/foam.hpp:38-74)."""

    decay: float = 0.35
    source_gain: float = 4.0
    advect_scale: float = 1.0
    wind_drift_x: float = 0.0
    wind_drift_z: float = 0.0
    fixed_dt: float = 1.0 / 60.0
    max_substeps: int = 4

    def to_c(self) -> FoamDescC:
        f = FoamDescC()
        lib().ocean_foam_desc_init(C.byref(f))
        f.decay = self.decay
        f.source_gain = self.source_gain
        f.advect_scale = self.advect_scale
        f.wind_drift_x = self.wind_drift_x
        f.wind_drift_z = self.wind_drift_z
        f.fixed_dt = self.fixed_dt
        f.max_substeps = self.max_substeps
        return f


SURFACE_FIELDS = ("height", "offset_x", "offset_z", "normal_x", "normal_y", "normal_z", "foam",
                  "velocity_x", "velocity_y", "velocity_z")


def _host_view(ptr, count: int) -> np.ndarray:
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float)), shape=(count,))


# ---------------------------------------------------------------------------
# Single ocean (the reference-shaped handle)
# ---------------------------------------------------------------------------
class Ocean:
    """One ocean patch on the current CUDA device; see ocean::Ocean."""

    def __init__(self, desc: OceanDesc | OceanDescC):
        cd = desc.to_c() if isinstance(desc, OceanDesc) else desc
        st = C.c_int(-1)
        h = lib().ocean_create(C.byref(cd), C.byref(st))
        if not h:
            if st.value == abi.OCEAN_ERROR_INVALID_ARG:
                raise ValueError(f"invalid ocean descriptor ({status_string(st.value)})")
            raise OceanError(st.value, "ocean_create")
        self._h = h
        self.size = cd.size
        self.patch_length = cd.patch_length
        self.velocity_on = bool(cd.compute_velocity)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().ocean_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> int:
        return self._h

    def update(self, time: float) -> None:
        lib().ocean_update(self._h, float(time))

    def update_async(self, time: float, stream: int = 0) -> None:
        _check(lib().ocean_update_async(self._h, float(time), C.c_void_p(stream)), "ocean_update_async")

    def refresh_host(self) -> None:
        _check(lib().ocean_refresh_host(self._h), "ocean_refresh_host")

    @property
    def time(self) -> float:
        return lib().ocean_get_time(self._h)

    def buffers(self) -> dict:
        """Numpy views (N*N, 4) of the host mirror; rewritten by update()."""
        b = lib().ocean_get_buffers(self._h)
        n = b.size * b.size
        out = {"displacement": _host_view(b.displacement, 4 * n).reshape(n, 4),
               "normal": _host_view(b.normal, 4 * n).reshape(n, 4),
               "size": b.size, "patch_length": b.patch_length}
        v = lib().ocean_get_velocity(self._h)
        out["velocity"] = _host_view(v, 4 * n).reshape(n, 4) if v else None
        return out

    def device_buffers(self) -> DeviceBuffers:
        d = DeviceBuffers()
        _check(lib().ocean_get_device_buffers(self._h, C.byref(d)), "ocean_get_device_buffers")
        return d

    def height_at(self, x: float, z: float) -> float:
        return lib().ocean_height_at(self._h, x, z)

    def sample_at(self, x: float, z: float) -> dict:
        s = SurfaceEx()
        lib().ocean_sample_ex(self._h, x, z, C.byref(s))
        return {k: getattr(s, k) for k in SURFACE_FIELDS}

    def sample_many(self, xz: np.ndarray) -> np.ndarray:
        """(count, 2) float32 world positions -> (count, 10) float32 records in
        SURFACE_FIELDS order, computed on the GPU."""
        xz = np.ascontiguousarray(xz, dtype=np.float32)
        out = np.empty((xz.shape[0], 10), dtype=np.float32)
        _check(lib().ocean_sample_many(self._h, xz.ctypes.data, xz.shape[0], out.ctypes.data),
               "ocean_sample_many")
        return out


# ---------------------------------------------------------------------------
# Batches
# ---------------------------------------------------------------------------
class OceanBatch:
    """Many same-size oceans advanced together (one row and one column launch
    per chunk of oceans)."""

    def __init__(self, descs: Sequence[OceanDesc], *, form: int = abi.OCEAN_FFT_EXACT,
                 foam: Optional[FoamDesc] = None, chunk: int = 0,
                 schedule: int = abi.OCEAN_SCHEDULE_PERSISTENT):
        arr = (OceanDescC * len(descs))(*[d.to_c() for d in descs])
        bd = BatchDescC()
        lib().ocean_batch_desc_init(C.byref(bd))
        bd.oceans = arr
        bd.count = len(descs)
        bd.fft_form = form
        bd.persistent_foam = 1 if foam is not None else 0
        if foam is not None:
            bd.foam = foam.to_c()
        bd.chunk = chunk
        bd.schedule = schedule
        st = C.c_int(-1)
        h = lib().ocean_batch_create(C.byref(bd), C.byref(st))
        if not h:
            if st.value == abi.OCEAN_ERROR_INVALID_ARG:
                raise ValueError(f"invalid batch descriptor ({status_string(st.value)})")
            raise OceanError(st.value, "ocean_batch_create")
        self._h = h
        self._keep = arr
        self.count = len(descs)
        self.size = descs[0].size
        self.velocity_on = bool(descs[0].compute_velocity)
        self.foam_on = foam is not None

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().ocean_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> int:
        return self._h

    def update(self, times, foam_dt: float = 0.0, stream: int = 0) -> None:
        t = np.ascontiguousarray(np.atleast_1d(np.asarray(times, dtype=np.float64)))
        per = 1 if t.size > 1 else 0
        if per and t.size != self.count:
            raise ValueError("times must hold one value or one per ocean")
        _check(lib().ocean_batch_update(self._h, t.ctypes.data, per, float(foam_dt),
                                        C.c_void_p(stream)), "ocean_batch_update")

    def update_host(self, times, foam_dt: float, disp: np.ndarray, normal: np.ndarray,
                    velocity: Optional[np.ndarray] = None, foam: Optional[np.ndarray] = None) -> None:
        t = np.ascontiguousarray(np.atleast_1d(np.asarray(times, dtype=np.float64)))
        per = 1 if t.size > 1 else 0
        ptr = lambda a: None if a is None else a.ctypes.data
        _check(lib().ocean_batch_update_host(self._h, t.ctypes.data, per, float(foam_dt),
                                             ptr(disp), ptr(normal), ptr(velocity), ptr(foam)),
               "ocean_batch_update_host")

    def update_host_rgba16(self, times, foam_dt: float, disp: Optional[np.ndarray],
                           normal: Optional[np.ndarray] = None,
                           velocity: Optional[np.ndarray] = None) -> None:
        """The frame with its outputs narrowed to RGBA16F on the device (uint16
        arrays of binary16 bits, count * N * N * 4); with persistent foam the
        displacement alpha carries the foam, as the reference viewer packs it."""
        t = np.ascontiguousarray(np.atleast_1d(np.asarray(times, dtype=np.float64)))
        per = 1 if t.size > 1 else 0
        for a in (disp, normal, velocity):
            if a is not None and (a.dtype != np.uint16 or not a.flags.c_contiguous):
                raise ValueError("RGBA16F outputs are contiguous uint16 arrays")
        ptr = lambda a: None if a is None else a.ctypes.data
        _check(lib().ocean_batch_update_host_rgba16(self._h, t.ctypes.data, per, float(foam_dt),
                                                    ptr(disp), ptr(normal), ptr(velocity)),
               "ocean_batch_update_host_rgba16")

    def synchronize(self) -> None:
        _check(lib().ocean_batch_synchronize(self._h), "ocean_batch_synchronize")

    def device_buffers(self, index: int) -> DeviceBuffers:
        d = DeviceBuffers()
        _check(lib().ocean_batch_get_device_buffers(self._h, index, C.byref(d)),
               "ocean_batch_get_device_buffers")
        return d

    @property
    def last_foam_substeps(self) -> int:
        return lib().ocean_batch_last_foam_substeps(self._h)

    def set_profiling(self, on: bool) -> None:
        _check(lib().ocean_batch_set_profiling(self._h, 1 if on else 0), "ocean_batch_set_profiling")

    def read_profile(self) -> dict:
        p = abi.PassProfile()
        _check(lib().ocean_batch_read_profile(self._h, C.byref(p)), "ocean_batch_read_profile")
        return {k: getattr(p, k) for k, _ in abi.PassProfile._fields_}

    @property
    def plan_count(self) -> int:
        return lib().ocean_batch_plan_count(self._h)

    @property
    def plan(self) -> int:
        return lib().ocean_batch_plan(self._h)

    def set_plan(self, plan: int) -> None:
        """Pick the persistent kernel's task plan (0 default, 1 the alternative)."""
        st = lib().ocean_batch_set_plan(self._h, int(plan))
        if st == abi.OCEAN_ERROR_INVALID_ARG:
            raise ValueError(f"plan {plan} is not available for this batch")
        _check(st, "ocean_batch_set_plan")

    @property
    def ring_slots(self) -> int:
        return lib().ocean_batch_ring_slots(self._h)

    def set_ring_slots(self, slots: int) -> None:
        """Intermediate ring depth of the persistent kernel: 2 or 3 oceans in
        flight (as allocated; 1 for a batch of one ocean)."""
        st = lib().ocean_batch_set_ring_slots(self._h, int(slots))
        if st == abi.OCEAN_ERROR_INVALID_ARG:
            raise ValueError(f"{slots} ring slots are not available for this batch")
        _check(st, "ocean_batch_set_ring_slots")

    @property
    def deferred_publish(self) -> bool:
        return lib().ocean_batch_deferred_publish(self._h) == 1

    def set_deferred_publish(self, defer: bool) -> None:
        """When the persistent kernel announces a finished row task: once the
        CTA's next task has staged its inputs (True), or before that task
        (False). Same bits either way."""
        _check(lib().ocean_batch_set_deferred_publish(self._h, 1 if defer else 0),
               "ocean_batch_set_deferred_publish")

    def autotune_plan(self) -> list:
        """Time every (plan, ring slots, publish) combination, keep the
        fastest; each plan's best ms per frame (empty for a batch that runs the
        per-chunk passes, with nothing to choose)."""
        ms = np.full(max(1, self.plan_count), -1.0, np.float64)
        _check(lib().ocean_batch_autotune_plan(self._h, ms.ctypes.data), "ocean_batch_autotune_plan")
        return [float(m) for m in ms[: self.plan_count] if m >= 0.0]

    @property
    def launch_count(self) -> int:
        return lib().ocean_batch_launch_count(self._h)

    # The rest of ocean::FoamField (persistent foam batches only).
    def foam_clear(self) -> None:
        """FoamField::clear: every ocean's foam to zero, accumulator reset."""
        _check(lib().ocean_batch_foam_clear(self._h), "ocean_batch_foam_clear")

    def set_foam_desc(self, foam: "FoamDesc") -> None:
        """FoamField::set_desc: decay, gain, advect scale and drift from the
        next update on (fixed_dt and max_substeps stay as created)."""
        f = foam.to_c()
        _check(lib().ocean_batch_foam_set_desc(self._h, C.byref(f)), "ocean_batch_foam_set_desc")

    def foam_desc(self) -> FoamDescC:
        f = FoamDescC()
        _check(lib().ocean_batch_foam_get_desc(self._h, C.byref(f)), "ocean_batch_foam_get_desc")
        return f

    def foam_at_many(self, index: int, xz: np.ndarray) -> np.ndarray:
        """FoamField::foam_at at world points xz (count x 2 float32)."""
        pts = np.ascontiguousarray(xz, dtype=np.float32).reshape(-1, 2)
        out = np.empty(pts.shape[0], np.float32)
        _check(lib().ocean_batch_foam_at_many(self._h, index, pts.ctypes.data, pts.shape[0], out.ctypes.data),
               "ocean_batch_foam_at_many")
        return out

    def foam_coverage(self, index: int = 0) -> float:
        """FoamField::coverage: mean foam over the patch."""
        v = C.c_double(0.0)
        _check(lib().ocean_batch_foam_coverage(self._h, index, C.byref(v)), "ocean_batch_foam_coverage")
        return v.value

    def read_spectrum(self, index: int):
        n = self.size
        h0 = np.empty((n * n, 2), dtype=np.float32)
        wk = np.empty((n * n, 2), dtype=np.float32)
        _check(lib().ocean_batch_read_spectrum(self._h, index, h0.ctypes.data, wk.ctypes.data),
               "ocean_batch_read_spectrum")
        return h0, wk


class OceanEnsemble:
    """Independent sea states of uneven size, advanced together: one stream
    and one persistent kernel per size, schedule chosen by the autotuner.
    `form` (an OCEAN_FFT_* value) overrides the process-wide form; with the
    tensor-core form, sizes outside 64..512 run the exact FP32 form."""

    def __init__(self, descs: Sequence[OceanDesc], autotune: bool = True, form: Optional[int] = None):
        arr = (OceanDescC * len(descs))(*[d.to_c() for d in descs])
        st = C.c_int(-1)
        if form is None:
            h = lib().ocean_ensemble_create(arr, len(descs), 1 if autotune else 0, C.byref(st))
        else:
            h = lib().ocean_ensemble_create_form(arr, len(descs), 1 if autotune else 0, int(form), C.byref(st))
        if not h:
            if st.value == abi.OCEAN_ERROR_INVALID_ARG:
                raise ValueError(f"invalid ensemble ({status_string(st.value)})")
            raise OceanError(st.value, "ocean_ensemble_create")
        self._h = h
        self.descs = list(descs)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().ocean_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def update(self, time: float, stream: int = 0) -> None:
        _check(lib().ocean_ensemble_update(self._h, float(time), C.c_void_p(stream)), "ocean_ensemble_update")

    def set_graph(self, enable: bool) -> None:
        """Replay the frame as one CUDA graph (default) or issue each call."""
        _check(lib().ocean_ensemble_set_graph(self._h, 1 if enable else 0), "ocean_ensemble_set_graph")

    def synchronize(self) -> None:
        _check(lib().ocean_ensemble_synchronize(self._h), "ocean_ensemble_synchronize")

    SEQUENTIAL, CONCURRENT, ONE_LAUNCH = 0, 1, 2

    def set_schedule(self, schedule: int) -> None:
        """Force a schedule: SEQUENTIAL, CONCURRENT (SM shares by work) or
        ONE_LAUNCH (every size in one persistent launch)."""
        st = lib().ocean_ensemble_set_schedule(self._h, int(schedule))
        if st == abi.OCEAN_ERROR_INVALID_ARG:
            raise ValueError(f"schedule {schedule} is not available for these oceans")
        _check(st, "ocean_ensemble_set_schedule")

    @property
    def schedule_kind(self) -> int:
        return lib().ocean_ensemble_schedule(self._h)

    def device_buffers(self, index: int) -> DeviceBuffers:
        d = DeviceBuffers()
        _check(lib().ocean_ensemble_device_buffers(self._h, index, C.byref(d)), "ocean_ensemble_device_buffers")
        return d

    def read(self, index: int):
        """(displacement, normal) of ocean `index` copied to host arrays."""
        d = self.device_buffers(index)
        n = d.size * d.size
        disp = np.empty((n, 4), np.float32)
        nrm = np.empty((n, 4), np.float32)
        _check(lib().ocean_copy_to_host(disp.ctypes.data, d.displacement, disp.nbytes), "copy")
        _check(lib().ocean_copy_to_host(nrm.ctypes.data, d.normal, nrm.nbytes), "copy")
        return disp, nrm

    @property
    def schedule(self) -> str:
        n = int(lib().ocean_ensemble_describe(self._h, None, 0))
        buf = C.create_string_buffer(n + 1)
        lib().ocean_ensemble_describe(self._h, buf, n + 1)
        return buf.value.decode()


class CascadeStack:
    """ocean::CascadeStack (include/ocean/cascade.hpp:45-92): several ocean
    levels summed at query time, updated together on the GPU. `form` (an
    OCEAN_FFT_* value) overrides the process-wide form."""

    def __init__(self, levels: Sequence[OceanDesc], form: Optional[int] = None):
        arr = (OceanDescC * len(levels))(*[d.to_c() for d in levels])
        st = C.c_int(-1)
        if form is None:
            h = lib().ocean_cascade_create(arr, len(levels), C.byref(st))
        else:
            h = lib().ocean_cascade_create_form(arr, len(levels), int(form), C.byref(st))
        if not h:
            if st.value == abi.OCEAN_ERROR_INVALID_ARG:
                raise ValueError(f"invalid cascade ({status_string(st.value)})")
            raise OceanError(st.value, "ocean_cascade_create")
        self._h = h
        self.levels = list(levels)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().ocean_cascade_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> int:
        return self._h

    def update(self, time: float, stream: int = 0) -> None:
        _check(lib().ocean_cascade_update(self._h, float(time), C.c_void_p(stream)),
               "ocean_cascade_update")

    def synchronize(self) -> None:
        _check(lib().ocean_cascade_synchronize(self._h), "ocean_cascade_synchronize")

    @property
    def time(self) -> float:
        return lib().ocean_cascade_get_time(self._h)

    def device_buffers(self, level: int) -> DeviceBuffers:
        d = DeviceBuffers()
        _check(lib().ocean_cascade_level_device_buffers(self._h, level, C.byref(d)),
               "ocean_cascade_level_device_buffers")
        return d

    def sample_many(self, xz: np.ndarray, iterations: int = 4, tolerance: float = 0.0) -> np.ndarray:
        """(count, 2) host points -> (count, 10) records (SURFACE_FIELDS order)."""
        xz = np.ascontiguousarray(xz, dtype=np.float32)
        out = np.empty((xz.shape[0], 10), dtype=np.float32)
        _check(lib().ocean_cascade_sample_many(self._h, xz.ctypes.data, xz.shape[0], out.ctypes.data,
                                               iterations, tolerance, 0, None),
               "ocean_cascade_sample_many")
        return out

    def sample_many_device(self, xz_ptr: int, count: int, out_ptr: int, iterations: int = 4,
                           tolerance: float = 0.0, stream: int = 0) -> None:
        """Device-resident queries: `xz_ptr` -> count float2, `out_ptr` -> count
        records of 10 floats; queued on `stream`."""
        _check(lib().ocean_cascade_sample_many(self._h, C.c_void_p(xz_ptr), count, C.c_void_p(out_ptr),
                                               iterations, tolerance, 1, C.c_void_p(stream)),
               "ocean_cascade_sample_many")


def force_simd_level(name: Optional[str]) -> str:
    r = lib().ocean_force_simd_level(None if name is None else name.encode())
    return r.decode()


def simd_level() -> str:
    return lib().ocean_simd_level().decode()


def version() -> tuple:
    a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
    lib().ocean_version(C.byref(a), C.byref(b), C.byref(c))
    return (a.value, b.value, c.value)
