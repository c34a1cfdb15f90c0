"""The allocation-free frame entry point, ocean_frame_static_scratch.

It exists for callers that may not call cudaMalloc themselves or have the
library call it for them - an engine whose GPU memory belongs to its own
allocator and budget, or a real-time thread that cannot take cudaMalloc's
implicit synchronisation. Such a caller hands in its own device buffers for
the spectrum tables and the outputs, and the frame keeps its intermediate in
the library's fixed static device array.

Checked here against the regular batch entry point, bit for bit (the bar
every exact-form test in this suite uses), on two calls in a row so that the
second call runs over the contents the first left in the shared array. This
file is named to be collected last; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import oceanlib_b200 as ob
from oceanlib_b200 import abi, workloads as W

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _small(size, velocity):
    return lambda: ob.OceanDesc(size=size, patch_length=40.0 * size / 16, wind_speed=11.0,
                                choppiness=1.3, seed=900 + size, compute_velocity=velocity)


# 16 and 64 take other stage offsets and lane layouts than 256 and 512
# (single sequences vs pairs, one or several stage blocks).
@pytest.mark.parametrize("make", [W.foam_patch_512, lambda: W.single_patch_256()[0],
                                  _small(16, True), _small(16, False), _small(64, True),
                                  _small(64, False)],
                         ids=["512_velocity", "256_plain", "16_velocity", "16_plain",
                              "64_velocity", "64_plain"])
def test_static_scratch_frame_matches_batch_entry_point(cuda_device, make):
    import torch

    desc = make()
    n = desc.size
    cells = n * n
    batch = ob.OceanBatch([desc])
    h0, wk = batch.read_spectrum(0)
    # The caller's own device buffers (allocated here by the test, as the
    # caller's allocator would).
    h0_d = torch.from_numpy(h0).cuda()
    wk_d = torch.from_numpy(wk).cuda()
    disp_d = torch.empty((cells, 4), dtype=torch.float32, device="cuda")
    nrm_d = torch.empty_like(disp_d)
    vel_d = torch.empty_like(disp_d) if desc.compute_velocity else None
    stream = torch.cuda.current_stream()

    want_d = np.empty((cells, 4), np.float32)
    want_n = np.empty_like(want_d)
    want_v = np.empty_like(want_d) if desc.compute_velocity else None
    for t in (10.0, 10.0 + 1.0 / 60.0):
        st = ob.lib().ocean_frame_static_scratch(
            n, desc.patch_length, t, desc.choppiness, desc.foam_threshold,
            h0_d.data_ptr(), wk_d.data_ptr(), disp_d.data_ptr(), nrm_d.data_ptr(),
            None if vel_d is None else vel_d.data_ptr(), C.c_void_p(stream.cuda_stream))
        assert st == abi.OCEAN_OK, ob.status_string(st)
        st = ob.lib().ocean_frame_static_scratch_status(C.c_void_p(stream.cuda_stream))
        assert st == abi.OCEAN_OK, ob.status_string(st)
        torch.cuda.synchronize()
        batch.update_host([t], 0.0, want_d, want_n, want_v)
        assert np.array_equal(_bits(disp_d.cpu().numpy()), _bits(want_d)), t
        assert np.array_equal(_bits(nrm_d.cpu().numpy()), _bits(want_n)), t
        if vel_d is not None:
            assert np.array_equal(_bits(vel_d.cpu().numpy()), _bits(want_v)), t
    batch.close()


def test_static_scratch_rejects_sizes_beyond_its_array(cuda_device):
    lib = ob.lib()
    for bad in (1024, 2048, 100, 8):
        st = lib.ocean_frame_static_scratch(bad, 100.0, 1.0, 1.0, 0.5, 16, 16, 16, 16, None, None)
        assert st == abi.OCEAN_ERROR_INVALID_ARG, bad
    st = lib.ocean_frame_static_scratch(256, 100.0, 1.0, 1.0, 0.5, None, 16, 16, 16, None, None)
    assert st == abi.OCEAN_ERROR_INVALID_ARG
    # Buffers off a 16-byte boundary are refused before anything is queued
    # (the values are never dereferenced: the call returns first).
    for k in range(5):
        ptrs = [4096, 4096, 4096, 4096, 4096]
        ptrs[k] += 8
        st = lib.ocean_frame_static_scratch(256, 100.0, 1.0, 1.0, 0.5, *ptrs, None)
        assert st == abi.OCEAN_ERROR_INVALID_ARG, k


def test_static_scratch_status_reports_a_bounded_wait_that_gave_up(cuda_device):
    """The frame's h0-copy wait, run on an mbarrier nothing arrives at with the
    static array's status word as its error word, gives up after 50 ms; the
    status query then reports OCEAN_ERROR_TIMEOUT, the device stays usable,
    and the next frame call clears the word."""
    import torch

    lib = ob.lib()
    assert lib.ocean_check_static_scratch_status(50) == abi.OCEAN_ERROR_TIMEOUT
    assert lib.ocean_frame_static_scratch_status(None) == abi.OCEAN_ERROR_TIMEOUT
    desc = _small(16, False)()
    batch = ob.OceanBatch([desc])
    h0, wk = batch.read_spectrum(0)
    h0_d = torch.from_numpy(h0).cuda()
    wk_d = torch.from_numpy(wk).cuda()
    out = torch.empty((2, 16 * 16, 4), dtype=torch.float32, device="cuda")
    st = lib.ocean_frame_static_scratch(16, desc.patch_length, 1.0, desc.choppiness, desc.foam_threshold,
                                        h0_d.data_ptr(), wk_d.data_ptr(), out[0].data_ptr(),
                                        out[1].data_ptr(), None, None)
    assert st == abi.OCEAN_OK
    assert lib.ocean_frame_static_scratch_status(None) == abi.OCEAN_OK
    batch.close()
