"""The C-ABI library without a GPU: it loads, exports every symbol the header
declares, keeps the reference's struct layouts, and its host-side behaviour
(status codes, NULL tolerance, struct_size versioning, level forcing) matches
the reference's C ABI tests (tests/test_c_api.cpp). No device work is done
without a GPU: a descriptor that passes the checks then fails to create. Where
a GPU is present, the valid-size test does create, then destroy, its oceans."""
import ctypes as C
import json
import re
from pathlib import Path

import pytest

import oceanlib_b200 as ob
from oceanlib_b200 import abi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "ocean_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"OCEAN_API\s+[^;(]*?\b(ocean_\w+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = ob.lib()
    names = declared_functions()
    assert len(names) >= 29
    for name in names:
        assert hasattr(lib, name), name
        assert name in abi.SIGNATURES, f"{name} missing from the ctypes mirror"
    assert set(abi.SIGNATURES) == set(names)


def test_reference_abi_symbols_present():
    # The 15 ocean_* entry points of the reference's C ABI (include/ocean/ocean.h)
    # that cover the ocean update path keep their names.
    ref_names = ["ocean_status_string", "ocean_desc_init", "ocean_create", "ocean_destroy",
                 "ocean_update", "ocean_get_buffers", "ocean_get_time", "ocean_height_at",
                 "ocean_sample_at", "ocean_sample_ex", "ocean_get_velocity", "ocean_simd_level",
                 "ocean_force_simd_level", "ocean_version"]
    for n in ref_names:
        assert n in declared_functions()


def test_struct_layouts_match_reference_header():
    layout = json.loads((ROOT / "tests" / "golden" / "abi_layout.json").read_text())
    assert C.sizeof(abi.OceanDescC) == layout["sizeof.ocean_desc"]
    assert C.sizeof(abi.SpectrumDesc) == layout["sizeof.ocean_spectrum_desc"]
    assert C.sizeof(abi.Buffers) == layout["sizeof.ocean_buffers"]
    assert C.sizeof(abi.Surface) == layout["sizeof.ocean_surface"]
    assert C.sizeof(abi.SurfaceEx) == layout["sizeof.ocean_surface_ex"]
    for key, off in layout.items():
        if key.startswith("ocean_desc."):
            assert getattr(abi.OceanDescC, key.split(".")[1]).offset == off, key
        if key.startswith("ocean_buffers."):
            assert getattr(abi.Buffers, key.split(".")[1]).offset == off, key


def test_status_strings_and_version():
    assert ob.status_string(abi.OCEAN_OK) == "ok"
    for s in range(1, 6):
        assert len(ob.status_string(s)) > 0
    assert ob.version() == (1, 0, 0)
    assert len(ob.simd_level()) > 0
    assert ob.lib().ocean_device_arch() == b"sm_100a"


def test_desc_init_defaults_match_reference():
    d = abi.OceanDescC()
    ob.lib().ocean_desc_init(C.byref(d))
    assert d.struct_size == C.sizeof(abi.OceanDescC)
    assert (d.size, d.patch_length) == (256, 200.0)
    assert d.spectrum.wind_speed == 10.0 and d.spectrum.fetch == 100000.0
    assert abs(d.spectrum.peak_enhancement - 3.3) < 1e-6
    assert abs(d.spectrum.gravity - 9.81) < 1e-6 and d.spectrum.small_wave_cutoff == 0.5
    assert d.choppiness == 1.0 and d.foam_threshold == 0.5 and d.seed == 1337
    assert d.water_depth == 0.0 and d.compute_velocity == 0 and not d.parallel_for


@pytest.mark.parametrize("size", [16, 1024, 2048, 4096])
def test_every_reference_size_passes_validation(size):
    # src/ocean.cpp:28-59: N is a power of two in [16, 4096]. Past the
    # descriptor checks, a create without a GPU fails on the device instead.
    d = abi.OceanDescC()
    ob.lib().ocean_desc_init(C.byref(d))
    d.size = size
    st = C.c_int(-1)
    h = ob.lib().ocean_create(C.byref(d), C.byref(st))
    assert st.value != abi.OCEAN_ERROR_INVALID_ARG
    if h:
        ob.lib().ocean_destroy(h)


@pytest.mark.parametrize("mutate", [
    lambda d: setattr(d, "size", 100),            # not a power of two
    lambda d: setattr(d, "size", 8),              # below 16
    lambda d: setattr(d, "size", 8192),           # above 4096
    lambda d: setattr(d, "patch_length", 0.0),
    lambda d: setattr(d.spectrum, "gravity", -1.0),
    lambda d: setattr(d.spectrum, "fetch", 0.0),
    lambda d: setattr(d.spectrum, "wind_speed", -1.0),
    lambda d: setattr(d.spectrum, "peak_enhancement", 0.5),
    lambda d: setattr(d, "choppiness", -0.1),
    lambda d: setattr(d, "struct_size", 0),
    lambda d: setattr(d, "struct_size", C.sizeof(abi.OceanDescC) + 8),
])
def test_invalid_descriptor_is_rejected_before_any_device_work(mutate):
    # src/ocean.cpp:28-59 and src/c_api.cpp:46-60 (tests/test_c_api.cpp:97-141)
    d = abi.OceanDescC()
    ob.lib().ocean_desc_init(C.byref(d))
    mutate(d)
    st = C.c_int(-1)
    assert not ob.lib().ocean_create(C.byref(d), C.byref(st))
    assert st.value == abi.OCEAN_ERROR_INVALID_ARG
    assert not ob.lib().ocean_create(None, C.byref(st))
    assert st.value == abi.OCEAN_ERROR_INVALID_ARG
    # a NULL status pointer is allowed
    assert not ob.lib().ocean_create(C.byref(d), None)


def test_null_handles_are_tolerated():
    # tests/test_c_api.cpp:205-225
    lib = ob.lib()
    lib.ocean_destroy(None)
    lib.ocean_update(None, 1.0)
    b = lib.ocean_get_buffers(None)
    assert not b.displacement and not b.normal and b.size == 0
    assert lib.ocean_get_time(None) == 0.0
    assert lib.ocean_height_at(None, 1.0, 2.0) == 0.0
    s = lib.ocean_sample_at(None, 0.0, 0.0)
    assert s.normal_y == 1.0 and s.height == 0.0
    ex = abi.SurfaceEx()
    lib.ocean_sample_ex(None, 0.0, 0.0, C.byref(ex))
    assert ex.normal_y == 1.0
    lib.ocean_sample_ex(None, 0.0, 0.0, None)
    assert not lib.ocean_get_velocity(None)
    lib.ocean_batch_destroy(None)
    assert lib.ocean_batch_count(None) == 0
    assert lib.ocean_batch_update(None, None, 0, 0.0, None) == abi.OCEAN_ERROR_INVALID_ARG
    assert lib.ocean_get_device_buffers(None, None) == abi.OCEAN_ERROR_INVALID_ARG
    # the FoamField members of a batch
    inval = abi.OCEAN_ERROR_INVALID_ARG
    assert lib.ocean_batch_foam_clear(None) == inval
    assert lib.ocean_batch_foam_set_desc(None, None) == inval
    assert lib.ocean_batch_foam_get_desc(None, None) == inval
    assert lib.ocean_batch_foam_at_many(None, 0, None, 0, None) == inval
    v = C.c_double(-1.0)
    assert lib.ocean_batch_foam_coverage(None, 0, C.byref(v)) == inval and v.value == -1.0


def test_force_simd_level_semantics():
    # tests/test_c_api.cpp:409-433
    assert ob.force_simd_level("scalar") == "scalar"
    assert ob.simd_level() == "scalar"
    assert ob.force_simd_level("SCALAR") == "scalar"
    assert ob.force_simd_level("not-a-real-level") == "scalar"
    assert ob.force_simd_level("fast") == "fast"
    assert ob.force_simd_level("precise") == "precise"  # the FP64-block form
    assert ob.force_simd_level(None) == "sm_100a"


def test_batch_descriptor_validation_is_host_side():
    lib = ob.lib()
    bd = abi.BatchDescC()
    lib.ocean_batch_desc_init(C.byref(bd))
    st = C.c_int(-1)
    assert not lib.ocean_batch_create(C.byref(bd), C.byref(st))  # no oceans
    assert st.value == abi.OCEAN_ERROR_INVALID_ARG
    bd.fft_form = 7
    assert not lib.ocean_batch_create(C.byref(bd), C.byref(st))
    assert st.value == abi.OCEAN_ERROR_INVALID_ARG
    # mixed sizes are refused
    descs = (abi.OceanDescC * 2)()
    for d in descs:
        lib.ocean_desc_init(C.byref(d))
    descs[1].size = 128
    lib.ocean_batch_desc_init(C.byref(bd))
    bd.oceans = descs
    bd.count = 2
    assert not lib.ocean_batch_create(C.byref(bd), C.byref(st))
    assert st.value == abi.OCEAN_ERROR_INVALID_ARG
    # foam needs velocity
    descs[1].size = 256
    bd.persistent_foam = 1
    assert not lib.ocean_batch_create(C.byref(bd), C.byref(st))
    assert st.value == abi.OCEAN_ERROR_INVALID_ARG


def test_ensemble_and_cascade_forms_are_validated_host_side():
    # ocean_ensemble_create_form / ocean_cascade_create_form refuse an unknown
    # form (and empty input) before any device work.
    lib = ob.lib()
    descs = (abi.OceanDescC * 2)()
    for d in descs:
        lib.ocean_desc_init(C.byref(d))
    st = C.c_int(-1)
    assert not lib.ocean_ensemble_create_form(descs, 2, 0, 7, C.byref(st))
    assert st.value == abi.OCEAN_ERROR_INVALID_ARG
    assert not lib.ocean_ensemble_create_form(None, 0, 0, abi.OCEAN_FFT_TENSOR, C.byref(st))
    assert st.value == abi.OCEAN_ERROR_INVALID_ARG
    assert not lib.ocean_cascade_create_form(descs, 2, 7, C.byref(st))
    assert st.value == abi.OCEAN_ERROR_INVALID_ARG
    assert not lib.ocean_cascade_create_form(None, 0, abi.OCEAN_FFT_EXACT, C.byref(st))
    assert st.value == abi.OCEAN_ERROR_INVALID_ARG


def test_reference_header_paths_compile_and_link():
    # include/ocean/ocean.h as C99 (-pedantic -Werror) and include/ocean/*.hpp
    # as C++20, each in a program linked against libocean_b200.so: C and C++
    # code written against the reference's headers builds and links here.
    # (The GPU test runs both programs.)
    from tests.native.build_native import build

    exes = build()
    for path in exes.values():
        assert path.exists()
