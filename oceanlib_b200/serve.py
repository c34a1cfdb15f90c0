"""The serving loop over the C ABI (ocean_server_*): many sessions, each an
ocean and optionally an interaction field, with update and height requests
batched on the GPU as they arrive.

    srv = OceanServer(hbm_budget=120e9)
    sid = srv.open_session(OceanDesc(size=256), InteractionDesc(size=512))
    t1 = srv.submit_update(sid, time=1 / 60, dt=1 / 60, sources=disturbances)
    out = np.empty(4096, np.float32)
    t2 = srv.submit_query(sid, xz, out)   # sees the update above
    srv.wait(t2)                           # out now holds the heights
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import OceanDesc, OceanError, _check, abi, lib, status_string
from .abi import DisturbanceC, ServerDescC, ServerStatsC
from .interaction import InteractionDesc

# numpy mirror of ocean_disturbance (7 floats + int32, 32 bytes)
DISTURBANCE_DTYPE = np.dtype([("world_x", "<f4"), ("world_z", "<f4"), ("radius", "<f4"),
                              ("strength", "<f4"), ("velocity_y", "<f4"), ("velocity_x", "<f4"),
                              ("velocity_z", "<f4"), ("kind", "<i4")])
assert DISTURBANCE_DTYPE.itemsize == C.sizeof(DisturbanceC)


def session_bytes(ocean: OceanDesc, field: Optional[InteractionDesc] = None) -> int:
    """Device bytes one session of these descriptors holds."""
    oc = ocean.to_c()
    fc = field.to_c() if field is not None else None
    return int(lib().ocean_server_session_bytes(C.byref(oc), C.byref(fc) if fc is not None else None))


class OceanServer:
    def __init__(self, hbm_budget: Optional[float] = None, max_inflight: int = 2,
                 max_batch_requests: int = 4096, max_batch_points: int = 1 << 20,
                 max_query_points: int = 65536, form: int = abi.OCEAN_FFT_EXACT):
        d = ServerDescC()
        lib().ocean_server_desc_init(C.byref(d))
        if hbm_budget is not None:
            d.hbm_budget = int(hbm_budget)
        d.max_inflight = max_inflight
        d.max_batch_requests = max_batch_requests
        d.max_batch_points = max_batch_points
        d.max_query_points = max_query_points
        d.fft_form = form
        st = C.c_int(-1)
        h = lib().ocean_server_create(C.byref(d), C.byref(st))
        if not h:
            if st.value == abi.OCEAN_ERROR_INVALID_ARG:
                raise ValueError(f"invalid server descriptor ({status_string(st.value)})")
            raise OceanError(st.value, "ocean_server_create")
        self._h = h
        self.desc = d
        self._keep = {}  # ticket -> arrays the library writes later
        self._ticket = C.c_uint64(0)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().ocean_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> int:
        return self._h

    def open_session(self, ocean: OceanDesc, field: Optional[InteractionDesc] = None) -> int:
        oc = ocean.to_c()
        fc = field.to_c() if field is not None else None
        sid = C.c_uint64(0)
        st = lib().ocean_server_open_session(self._h, C.byref(oc), C.byref(fc) if fc is not None else None,
                                             C.byref(sid))
        if st == abi.OCEAN_ERROR_INVALID_ARG:
            raise ValueError(f"invalid session descriptor ({status_string(st)})")
        if st == abi.OCEAN_ERROR_OUT_OF_MEMORY:
            raise MemoryError("session larger than the whole HBM budget")
        _check(st, "ocean_server_open_session")
        return int(sid.value)

    def close_session(self, sid: int) -> None:
        _check(lib().ocean_server_close_session(self._h, sid), "ocean_server_close_session")

    def state(self, sid: int) -> int:
        return int(lib().ocean_server_session_state(self._h, sid))

    def submit_update(self, sid: int, time: float, dt: float, sources: Optional[np.ndarray] = None) -> int:
        """`sources`: a DISTURBANCE_DTYPE array (copied before returning)."""
        if sources is None or len(sources) == 0:
            ptr, n = None, 0
        else:
            sources = np.ascontiguousarray(sources, dtype=DISTURBANCE_DTYPE)
            ptr, n = sources.ctypes.data, len(sources)
        st = lib().ocean_server_submit_update(self._h, sid, float(time), float(dt), ptr, n,
                                              C.byref(self._ticket))
        _check(st, "ocean_server_submit_update")
        return int(self._ticket.value)

    def submit_query(self, sid: int, xz: np.ndarray, out: np.ndarray) -> int:
        """Heights at xz[count, 2] land in out[count] (float32, kept alive here
        until the ticket is waited on)."""
        xz = np.ascontiguousarray(xz, dtype=np.float32).reshape(-1, 2)
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.size < len(xz):
            raise ValueError("out must be a contiguous float32 array with one entry per point")
        st = lib().ocean_server_submit_query(self._h, sid, xz.ctypes.data, len(xz), out.ctypes.data,
                                             C.byref(self._ticket))
        _check(st, "ocean_server_submit_query")
        t = int(self._ticket.value)
        self._keep[t] = out
        return t

    def wait(self, ticket: int, timeout_ms: int = 60000) -> int:
        st = int(lib().ocean_server_wait(self._h, ticket, timeout_ms))
        if st != abi.OCEAN_ERROR_TIMEOUT:
            self._keep.pop(ticket, None)
        return st

    def drain(self, timeout_ms: int = 600000) -> None:
        _check(lib().ocean_server_drain(self._h, timeout_ms), "ocean_server_drain")
        self._keep.clear()

    def read_session(self, sid: int, ocean_size: int, field_size: int = 0):
        """(displacement, normal, field) of a session after its requests so far."""
        disp = np.empty((ocean_size, ocean_size, 4), np.float32)
        normal = np.empty_like(disp)
        field = np.empty((field_size, field_size, 4), np.float32) if field_size else None
        st = lib().ocean_server_read_session(self._h, sid, disp.ctypes.data, normal.ctypes.data,
                                             field.ctypes.data if field is not None else None)
        _check(st, "ocean_server_read_session")
        return disp, normal, field

    def stats(self) -> dict:
        s = ServerStatsC()
        _check(lib().ocean_server_get_stats(self._h, C.byref(s)), "ocean_server_get_stats")
        return {k: getattr(s, k) for k, _ in ServerStatsC._fields_}

    def latency_samples(self):
        """(submit_ms, latency_ms, kind) arrays of every request completed since
        the last reset (kind 0 = update, 1 = query)."""
        n = int(lib().ocean_server_latency_samples(self._h, None, None, None, 0))
        sub = np.empty(n, np.float64)
        lat = np.empty(n, np.float64)
        kind = np.empty(n, np.int32)
        m = int(lib().ocean_server_latency_samples(self._h, sub.ctypes.data, lat.ctypes.data,
                                                   kind.ctypes.data, n))
        m = min(m, n)
        return sub[:m], lat[:m], kind[:m]

    def reset_stats(self) -> None:
        _check(lib().ocean_server_reset_stats(self._h), "ocean_server_reset_stats")
