"""ctypes mirror of include/ocean_b200.h (the reference C ABI's structs plus the
GPU extensions). Pure layout: importing this module touches no library."""
from __future__ import annotations

import ctypes as C

OCEAN_OK = 0
OCEAN_ERROR_INVALID_ARG = 1
OCEAN_ERROR_OUT_OF_MEMORY = 2
OCEAN_ERROR_UNKNOWN = 3
OCEAN_ERROR_DEVICE = 4
OCEAN_ERROR_TIMEOUT = 5

OCEAN_FFT_EXACT = 0
OCEAN_FFT_FAST = 1
OCEAN_FFT_TENSOR = 2
OCEAN_FFT_PRECISE = 3

OCEAN_SCHEDULE_PERSISTENT = 0
OCEAN_SCHEDULE_CHUNKED = 1

TASK_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_uint32)
PARALLEL_FOR_FN = C.CFUNCTYPE(None, C.c_void_p, TASK_FN, C.c_void_p, C.c_uint32)


class SpectrumDesc(C.Structure):
    _fields_ = [
        ("wind_speed", C.c_float),
        ("fetch", C.c_float),
        ("wind_direction", C.c_float),
        ("peak_enhancement", C.c_float),
        ("swell", C.c_float),
        ("small_wave_cutoff", C.c_float),
        ("gravity", C.c_float),
    ]


class OceanDescC(C.Structure):
    """`ocean_desc` (include/ocean/ocean.h:85-134 in the reference)."""

    _fields_ = [
        ("struct_size", C.c_size_t),
        ("size", C.c_uint32),
        ("patch_length", C.c_float),
        ("spectrum", SpectrumDesc),
        ("choppiness", C.c_float),
        ("foam_threshold", C.c_float),
        ("seed", C.c_uint64),
        ("parallel_for", C.c_void_p),
        ("parallel_for_user", C.c_void_p),
        ("thread_count", C.c_uint32),
        ("water_depth", C.c_float),
        ("compute_velocity", C.c_int32),
    ]


class Buffers(C.Structure):
    _fields_ = [
        ("displacement", C.POINTER(C.c_float)),
        ("normal", C.POINTER(C.c_float)),
        ("size", C.c_uint32),
        ("patch_length", C.c_float),
    ]


class Surface(C.Structure):
    _fields_ = [(n, C.c_float) for n in
                ("height", "offset_x", "offset_z", "normal_x", "normal_y", "normal_z", "foam")]


class SurfaceEx(C.Structure):
    _fields_ = [(n, C.c_float) for n in
                ("height", "offset_x", "offset_z", "normal_x", "normal_y", "normal_z", "foam",
                 "velocity_x", "velocity_y", "velocity_z")]


class DeviceBuffers(C.Structure):
    _fields_ = [
        ("displacement", C.c_void_p),
        ("normal", C.c_void_p),
        ("velocity", C.c_void_p),
        ("foam", C.c_void_p),
        ("size", C.c_uint32),
        ("patch_length", C.c_float),
    ]


class FoamDescC(C.Structure):
    """Mirrors ocean::FoamDesc (include/ocean/foam.hpp:38-74)."""

    _fields_ = [
        ("struct_size", C.c_size_t),
        ("decay", C.c_float),
        ("source_gain", C.c_float),
        ("advect_scale", C.c_float),
        ("wind_drift_x", C.c_float),
        ("wind_drift_z", C.c_float),
        ("fixed_dt", C.c_float),
        ("max_substeps", C.c_uint32),
    ]


class BatchDescC(C.Structure):
    _fields_ = [
        ("struct_size", C.c_size_t),
        ("oceans", C.POINTER(OceanDescC)),
        ("count", C.c_uint32),
        ("fft_form", C.c_int32),
        ("persistent_foam", C.c_int32),
        ("foam", FoamDescC),
        ("chunk", C.c_uint32),
        ("schedule", C.c_int32),
    ]


class InteractionDescC(C.Structure):
    """`ocean_interaction_desc` (include/ocean/ocean.h:300-318 in the reference)."""

    _fields_ = [
        ("struct_size", C.c_size_t),
        ("size", C.c_uint32),
        ("extent", C.c_float),
        ("kernel_radius", C.c_uint32),
        ("damping", C.c_float),
        ("absorb_cells", C.c_uint32),
        ("fixed_dt", C.c_float),
        ("max_substeps", C.c_uint32),
        ("max_sources", C.c_uint32),
        ("gravity", C.c_float),
        ("water_depth", C.c_float),
        ("obstruction", C.c_int32),
        ("parallel_for", C.c_void_p),
        ("parallel_for_user", C.c_void_p),
        ("thread_count", C.c_uint32),
    ]


class DisturbanceC(C.Structure):
    _fields_ = [(n, C.c_float) for n in
                ("world_x", "world_z", "radius", "strength", "velocity_y", "velocity_x",
                 "velocity_z")] + [("kind", C.c_int32)]


class InteractionBuffers(C.Structure):
    _fields_ = [
        ("field", C.POINTER(C.c_float)),
        ("size", C.c_uint32),
        ("extent", C.c_float),
        ("origin_x", C.c_float),
        ("origin_z", C.c_float),
    ]


class InteractionSample(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("height", "slope_x", "slope_z", "velocity_y")]


OCEAN_OBSTRUCTION_NEUMANN = 0
OCEAN_OBSTRUCTION_DIRICHLET = 1
OCEAN_SOURCE_IMPULSE = 0
OCEAN_SOURCE_CONTINUOUS = 1


class PassProfile(C.Structure):
    _fields_ = [
        ("row_launches", C.c_uint64),
        ("col_launches", C.c_uint64),
        ("foam_launches", C.c_uint64),
        ("row_ms", C.c_double),
        ("col_ms", C.c_double),
        ("foam_ms", C.c_double),
        ("frame_launches", C.c_uint64),
        ("frame_ms", C.c_double),
    ]


class ServerDescC(C.Structure):
    _fields_ = [
        ("struct_size", C.c_size_t),
        ("hbm_budget", C.c_uint64),
        ("max_inflight", C.c_uint32),
        ("max_batch_requests", C.c_uint32),
        ("max_batch_points", C.c_uint32),
        ("max_query_points", C.c_uint32),
        ("fft_form", C.c_int32),
        ("reserved", C.c_uint32),
    ]


OCEAN_SESSION_WAITING = 0
OCEAN_SESSION_ACTIVE = 1
OCEAN_SESSION_CLOSED = 2


class ServerStatsC(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "sessions_active", "sessions_waiting", "sessions_closed", "bytes_in_use", "hbm_budget",
        "requests_submitted", "requests_completed", "requests_failed", "updates_completed",
        "queries_completed", "query_points_completed", "batches", "kernel_launches",
        "bytes_staging")] + \
        [(n, C.c_double) for n in (
            "mean_batch_requests", "latency_p50_ms", "latency_p99_ms", "latency_max_ms",
            "update_p50_ms", "update_p99_ms", "query_p50_ms", "query_p99_ms", "gpu_busy_ms",
            "wall_ms", "dispatch_max_ms")] + [("staging_growths", C.c_uint64)]


# Every function include/ocean_b200.h declares, with its ctypes signature.
SIGNATURES = {
    "ocean_dft_batch": (C.c_int, [C.c_uint32, C.c_uint32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ocean_batch_update_host_rgba16": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_float, C.c_void_p,
                                                 C.c_void_p, C.c_void_p]),
    "ocean_pack_rgba16": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    "ocean_server_desc_init": (None, [C.POINTER(ServerDescC)]),
    "ocean_server_create": (C.c_void_p, [C.POINTER(ServerDescC), C.POINTER(C.c_int)]),
    "ocean_server_destroy": (None, [C.c_void_p]),
    "ocean_server_session_bytes": (C.c_uint64, [C.POINTER(OceanDescC), C.POINTER(InteractionDescC)]),
    "ocean_server_open_session": (C.c_int, [C.c_void_p, C.POINTER(OceanDescC), C.POINTER(InteractionDescC),
                                            C.POINTER(C.c_uint64)]),
    "ocean_server_close_session": (C.c_int, [C.c_void_p, C.c_uint64]),
    "ocean_server_session_state": (C.c_int, [C.c_void_p, C.c_uint64]),
    "ocean_server_submit_update": (C.c_int, [C.c_void_p, C.c_uint64, C.c_double, C.c_float, C.c_void_p,
                                             C.c_uint32, C.POINTER(C.c_uint64)]),
    "ocean_server_submit_query": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint32, C.c_void_p,
                                            C.POINTER(C.c_uint64)]),
    "ocean_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32]),
    "ocean_server_drain": (C.c_int, [C.c_void_p, C.c_uint32]),
    "ocean_server_read_session": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ocean_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(ServerStatsC)]),
    "ocean_server_reset_stats": (C.c_int, [C.c_void_p]),
    "ocean_server_latency_samples": (C.c_uint64, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64]),
    "ocean_status_string": (C.c_char_p, [C.c_int]),
    "ocean_desc_init": (None, [C.POINTER(OceanDescC)]),
    "ocean_create": (C.c_void_p, [C.POINTER(OceanDescC), C.POINTER(C.c_int)]),
    "ocean_destroy": (None, [C.c_void_p]),
    "ocean_update": (None, [C.c_void_p, C.c_double]),
    "ocean_get_buffers": (Buffers, [C.c_void_p]),
    "ocean_get_time": (C.c_double, [C.c_void_p]),
    "ocean_height_at": (C.c_float, [C.c_void_p, C.c_float, C.c_float]),
    "ocean_sample_at": (Surface, [C.c_void_p, C.c_float, C.c_float]),
    "ocean_sample_ex": (None, [C.c_void_p, C.c_float, C.c_float, C.POINTER(SurfaceEx)]),
    "ocean_get_velocity": (C.POINTER(C.c_float), [C.c_void_p]),
    "ocean_simd_level": (C.c_char_p, []),
    "ocean_force_simd_level": (C.c_char_p, [C.c_char_p]),
    "ocean_version": (None, [C.POINTER(C.c_uint32)] * 3),
    "ocean_get_device_buffers": (C.c_int, [C.c_void_p, C.POINTER(DeviceBuffers)]),
    "ocean_update_async": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p]),
    "ocean_refresh_host": (C.c_int, [C.c_void_p]),
    "ocean_sample_many": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "ocean_foam_desc_init": (None, [C.POINTER(FoamDescC)]),
    "ocean_batch_desc_init": (None, [C.POINTER(BatchDescC)]),
    "ocean_batch_create": (C.c_void_p, [C.POINTER(BatchDescC), C.POINTER(C.c_int)]),
    "ocean_batch_destroy": (None, [C.c_void_p]),
    "ocean_batch_count": (C.c_uint32, [C.c_void_p]),
    "ocean_batch_update": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_float, C.c_void_p]),
    "ocean_batch_update_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_float,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ocean_batch_get_device_buffers": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(DeviceBuffers)]),
    "ocean_batch_last_foam_substeps": (C.c_uint32, [C.c_void_p]),
    "ocean_batch_synchronize": (C.c_int, [C.c_void_p]),
    "ocean_batch_read_spectrum": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "ocean_batch_foam_clear": (C.c_int, [C.c_void_p]),
    "ocean_batch_foam_set_desc": (C.c_int, [C.c_void_p, C.POINTER(FoamDescC)]),
    "ocean_batch_foam_get_desc": (C.c_int, [C.c_void_p, C.POINTER(FoamDescC)]),
    "ocean_batch_foam_at_many": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p]),
    "ocean_batch_foam_coverage": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double)]),
    "ocean_batch_set_profiling": (C.c_int, [C.c_void_p, C.c_int32]),
    "ocean_batch_read_profile": (C.c_int, [C.c_void_p, C.POINTER(PassProfile)]),
    "ocean_batch_launch_count": (C.c_uint64, [C.c_void_p]),
    "ocean_batch_set_plan": (C.c_int, [C.c_void_p, C.c_int32]),
    "ocean_batch_plan": (C.c_int32, [C.c_void_p]),
    "ocean_batch_plan_count": (C.c_int32, [C.c_void_p]),
    "ocean_batch_set_ring_slots": (C.c_int, [C.c_void_p, C.c_int32]),
    "ocean_batch_ring_slots": (C.c_int32, [C.c_void_p]),
    "ocean_batch_set_deferred_publish": (C.c_int, [C.c_void_p, C.c_int32]),
    "ocean_batch_deferred_publish": (C.c_int32, [C.c_void_p]),
    "ocean_batch_autotune_plan": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ocean_frame_static_scratch": (C.c_int, [C.c_uint32, C.c_float, C.c_double, C.c_float,
                                             C.c_float, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p]),
    "ocean_frame_static_scratch_status": (C.c_int, [C.c_void_p]),
    "ocean_check_static_scratch_status": (C.c_int, [C.c_uint32]),
    "ocean_ensemble_create": (C.c_void_p, [C.POINTER(OceanDescC), C.c_uint32, C.c_int32,
                                           C.POINTER(C.c_int)]),
    "ocean_ensemble_create_form": (C.c_void_p, [C.POINTER(OceanDescC), C.c_uint32, C.c_int32, C.c_int32,
                                                C.POINTER(C.c_int)]),
    "ocean_ensemble_destroy": (None, [C.c_void_p]),
    "ocean_ensemble_count": (C.c_uint32, [C.c_void_p]),
    "ocean_ensemble_update": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p]),
    "ocean_ensemble_synchronize": (C.c_int, [C.c_void_p]),
    "ocean_ensemble_set_schedule": (C.c_int, [C.c_void_p, C.c_int32]),
    "ocean_ensemble_schedule": (C.c_int32, [C.c_void_p]),
    "ocean_ensemble_set_graph": (C.c_int, [C.c_void_p, C.c_int32]),
    "ocean_ensemble_device_buffers": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(DeviceBuffers)]),
    "ocean_ensemble_describe": (C.c_uint64, [C.c_void_p, C.c_char_p, C.c_uint64]),
    "ocean_cascade_create":(C.c_void_p, [C.POINTER(OceanDescC), C.c_uint32, C.POINTER(C.c_int)]),
    "ocean_cascade_create_form": (C.c_void_p, [C.POINTER(OceanDescC), C.c_uint32, C.c_int32, C.POINTER(C.c_int)]),
    "ocean_cascade_destroy": (None, [C.c_void_p]),
    "ocean_cascade_update": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p]),
    "ocean_cascade_level_count": (C.c_uint32, [C.c_void_p]),
    "ocean_cascade_get_time": (C.c_double, [C.c_void_p]),
    "ocean_cascade_level_device_buffers": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(DeviceBuffers)]),
    "ocean_cascade_synchronize": (C.c_int, [C.c_void_p]),
    "ocean_cascade_sample_many": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                            C.c_int32, C.c_float, C.c_int32, C.c_void_p]),
    "ocean_interaction_desc_init": (None, [C.POINTER(InteractionDescC)]),
    "ocean_interaction_create": (C.c_void_p, [C.POINTER(InteractionDescC), C.POINTER(C.c_int)]),
    "ocean_interaction_destroy": (None, [C.c_void_p]),
    "ocean_interaction_add": (None, [C.c_void_p, C.POINTER(DisturbanceC)]),
    "ocean_interaction_dropped": (C.c_uint64, [C.c_void_p]),
    "ocean_interaction_update": (None, [C.c_void_p, C.c_float]),
    "ocean_interaction_recenter": (C.c_int32, [C.c_void_p, C.c_float, C.c_float]),
    "ocean_interaction_set_obstruction": (None, [C.c_void_p, C.c_void_p]),
    "ocean_interaction_get_buffers": (InteractionBuffers, [C.c_void_p]),
    "ocean_interaction_sample_at": (None, [C.c_void_p, C.c_float, C.c_float, C.POINTER(InteractionSample)]),
    "ocean_interaction_height_at": (C.c_float, [C.c_void_p, C.c_float, C.c_float]),
    "ocean_interaction_fixed_dt": (C.c_float, [C.c_void_p]),
    "ocean_interaction_dt_limit": (C.c_float, [C.c_void_p]),
    "ocean_interaction_dispersion_error": (C.c_float, [C.c_void_p]),
    "ocean_sample_combined": (None, [C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.POINTER(SurfaceEx)]),
    "ocean_interaction_device_field": (C.c_void_p, [C.c_void_p]),
    "ocean_interaction_obstruction_tables": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]),
    "ocean_interaction_last_shift": (None, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "ocean_interaction_last_substeps": (C.c_uint32, [C.c_void_p]),
    "ocean_interaction_last_clamped": (C.c_int32, [C.c_void_p]),
    "ocean_interaction_energy": (C.c_double, [C.c_void_p]),
    "ocean_interaction_get_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "ocean_interaction_set_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "ocean_interaction_kernel_taps": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ocean_interaction_sample_many": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "ocean_sample_combined_many": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "ocean_check_bounded_wait": (C.c_int, [C.c_uint32]),
    "ocean_copy_to_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "ocean_device_arch": (C.c_char_p, []),
}
