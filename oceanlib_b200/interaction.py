"""ocean::InteractionField (include/ocean/interaction.hpp:232-346) over the C
ABI: an iWave height field stepped on the GPU, plus the combined surface
query (WaterSurface, include/ocean/interaction.hpp:374-398)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import OceanError, _check, abi, lib, status_string
from .abi import DisturbanceC, InteractionDescC, InteractionSample, SurfaceEx


@dataclass
class InteractionDesc:
    """ocean::InteractionDesc defaults (include/ocean/interaction.hpp:64-139)."""

    size: int = 256
    extent: float = 64.0
    kernel_radius: int = 6
    damping: float = 0.20
    absorb_cells: int = 16
    fixed_dt: float = 0.0
    max_substeps: int = 8
    max_sources: int = 64
    gravity: float = 9.81
    depth: float = 0.0
    obstruction: int = abi.OCEAN_OBSTRUCTION_NEUMANN

    def to_c(self) -> InteractionDescC:
        d = InteractionDescC()
        lib().ocean_interaction_desc_init(C.byref(d))
        for k in ("size", "extent", "kernel_radius", "damping", "absorb_cells", "fixed_dt",
                  "max_substeps", "max_sources", "gravity", "obstruction"):
            setattr(d, k, getattr(self, k))
        d.water_depth = self.depth
        return d


@dataclass
class Disturbance:
    """ocean::Disturbance (include/ocean/interaction.hpp:159-186)."""

    world_x: float = 0.0
    world_z: float = 0.0
    radius: float = 0.35
    strength: float = 0.25
    velocity_y: float = 0.0
    velocity_x: float = 0.0
    velocity_z: float = 0.0
    kind: int = abi.OCEAN_SOURCE_IMPULSE

    def to_c(self) -> DisturbanceC:
        d = DisturbanceC()
        for k in ("world_x", "world_z", "radius", "strength", "velocity_y", "velocity_x",
                  "velocity_z", "kind"):
            setattr(d, k, getattr(self, k))
        return d


class InteractionField:
    def __init__(self, desc: InteractionDesc):
        cd = desc.to_c()
        st = C.c_int(-1)
        h = lib().ocean_interaction_create(C.byref(cd), C.byref(st))
        if not h:
            if st.value == abi.OCEAN_ERROR_INVALID_ARG:
                raise ValueError(f"invalid interaction descriptor ({status_string(st.value)})")
            raise OceanError(st.value, "ocean_interaction_create")
        self._h = h
        self.desc = desc
        self.size = desc.size

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().ocean_interaction_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> int:
        return self._h

    def add(self, d: Disturbance) -> None:
        lib().ocean_interaction_add(self._h, C.byref(d.to_c()))

    def update(self, dt: float) -> None:
        lib().ocean_interaction_update(self._h, dt)

    def recenter(self, x: float, z: float) -> bool:
        return bool(lib().ocean_interaction_recenter(self._h, x, z))

    def set_obstruction(self, mask: Optional[np.ndarray]) -> None:
        if mask is None:
            lib().ocean_interaction_set_obstruction(self._h, None)
            return
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        lib().ocean_interaction_set_obstruction(self._h, m.ctypes.data)

    def buffers(self) -> dict:
        b = lib().ocean_interaction_get_buffers(self._h)
        n = b.size * b.size
        field = np.ctypeslib.as_array(b.field, shape=(4 * n,)).reshape(n, 4)
        return {"field": field, "size": b.size, "extent": b.extent, "origin_x": b.origin_x,
                "origin_z": b.origin_z}

    def sample_at(self, x: float, z: float) -> dict:
        s = InteractionSample()
        lib().ocean_interaction_sample_at(self._h, x, z, C.byref(s))
        return {k: getattr(s, k) for k, _ in InteractionSample._fields_}

    def sample_many(self, xz: np.ndarray) -> np.ndarray:
        xz = np.ascontiguousarray(xz, dtype=np.float32)
        out = np.empty((xz.shape[0], 4), dtype=np.float32)
        _check(lib().ocean_interaction_sample_many(self._h, xz.ctypes.data, xz.shape[0], out.ctypes.data),
               "ocean_interaction_sample_many")
        return out

    @property
    def fixed_dt(self) -> float:
        return lib().ocean_interaction_fixed_dt(self._h)

    @property
    def dt_limit(self) -> float:
        return lib().ocean_interaction_dt_limit(self._h)

    @property
    def dispersion_error(self) -> float:
        return lib().ocean_interaction_dispersion_error(self._h)

    @property
    def dropped(self) -> int:
        return lib().ocean_interaction_dropped(self._h)

    @property
    def last_substeps(self) -> int:
        return lib().ocean_interaction_last_substeps(self._h)

    @property
    def last_clamped(self) -> bool:
        return bool(lib().ocean_interaction_last_clamped(self._h))

    def energy(self) -> float:
        return lib().ocean_interaction_energy(self._h)

    def taps(self) -> np.ndarray:
        w = 2 * self.desc.kernel_radius + 1
        t = np.empty(w * w, dtype=np.float32)
        _check(lib().ocean_interaction_kernel_taps(self._h, t.ctypes.data), "ocean_interaction_kernel_taps")
        return t

    def obstruction_tables(self):
        """(solid cells in index order, nearest-fluid index per cell) as the
        device built them for the current obstruction."""
        n = self.size
        solid = np.empty(n * n, np.uint32)
        nearest = np.empty(n * n, np.uint32)
        count = C.c_uint32(0)
        _check(lib().ocean_interaction_obstruction_tables(self._h, solid.ctypes.data, nearest.ctypes.data,
                                                          C.byref(count)), "ocean_interaction_obstruction_tables")
        return solid[:count.value].copy(), nearest

    def get_state(self):
        n = self.size
        cur = np.empty(n * n, np.float32)
        old = np.empty(n * n, np.float32)
        _check(lib().ocean_interaction_get_state(self._h, cur.ctypes.data, old.ctypes.data),
               "ocean_interaction_get_state")
        return cur, old

    def set_state(self, cur: np.ndarray, old: np.ndarray) -> None:
        cur = np.ascontiguousarray(cur, np.float32)
        old = np.ascontiguousarray(old, np.float32)
        _check(lib().ocean_interaction_set_state(self._h, cur.ctypes.data, old.ctypes.data),
               "ocean_interaction_set_state")


def sample_combined_many(ocean, field: InteractionField, xz: np.ndarray) -> np.ndarray:
    """FFT ocean plus interaction field at (count, 2) points -> (count, 10)."""
    xz = np.ascontiguousarray(xz, dtype=np.float32)
    out = np.empty((xz.shape[0], 10), dtype=np.float32)
    _check(lib().ocean_sample_combined_many(ocean.handle, field.handle, xz.ctypes.data, xz.shape[0],
                                            out.ctypes.data), "ocean_sample_combined_many")
    return out
