"""The serving loop's C ABI without a GPU: struct layouts against the C
compiler's view of the header, descriptor defaults, session sizing and NULL
handling. No device work is done."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import pytest

import oceanlib_b200 as ob
from oceanlib_b200 import abi, serve
from oceanlib_b200 import workloads as W
from oceanlib_b200.interaction import InteractionDesc

ROOT = Path(__file__).resolve().parents[1]


def c_layout(tmp_path, struct, fields):
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ocean_b200.h"', "int main(void) {",
             f'printf("%zu\\n", sizeof({struct}));']
    lines += [f'printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    lines += ["return 0; }"]
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    return vals[0], vals[1:]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
@pytest.mark.parametrize("cls,struct", [(abi.ServerDescC, "ocean_server_desc"),
                                        (abi.ServerStatsC, "ocean_server_stats")])
def test_server_structs_match_the_header(tmp_path, cls, struct):
    names = [n for n, _ in cls._fields_]
    size, offs = c_layout(tmp_path, struct, names)
    assert C.sizeof(cls) == size
    assert [getattr(cls, n).offset for n in names] == offs


def test_server_desc_defaults():
    d = abi.ServerDescC()
    ob.lib().ocean_server_desc_init(C.byref(d))
    assert d.struct_size == C.sizeof(abi.ServerDescC)
    assert d.hbm_budget == 120_000_000_000
    assert d.max_inflight == 2 and d.max_batch_requests == 4096
    assert d.max_batch_points == 1 << 20 and d.max_query_points == 65536
    assert d.fft_form == abi.OCEAN_FFT_EXACT


def test_session_bytes_is_the_sum_of_its_buffers():
    def r256(b):
        return (b + 255) // 256 * 256

    for n, vel in ((128, False), (512, False), (256, True)):
        od = ob.OceanDesc(size=n, compute_velocity=vel)
        cells = n * n
        ocean = r256(8 * cells) * 2 + r256(4 * n) + r256(16 * cells) * (3 if vel else 2)
        assert serve.session_bytes(od) == ocean
        fd = InteractionDesc(size=512, kernel_radius=6)
        stride = (512 + 12 + 15) // 16 * 16
        field = 2 * r256((512 + 12) * stride * 4) + r256(16 * 512 * 512)
        assert serve.session_bytes(od, fd) == ocean + field
    # the serving workload: 256 sessions fit the 120 GB budget many times over
    oceans, fd = W.serving_sessions()
    total = sum(serve.session_bytes(o, fd) for o in oceans)
    assert 2.5e9 < total < 4e9


def test_null_server_handles_are_tolerated():
    lib = ob.lib()
    lib.ocean_server_destroy(None)
    t = C.c_uint64(0)
    assert lib.ocean_server_submit_update(None, 1, 0.0, 0.0, None, 0, C.byref(t)) == abi.OCEAN_ERROR_INVALID_ARG
    assert lib.ocean_server_submit_query(None, 1, None, 0, None, C.byref(t)) == abi.OCEAN_ERROR_INVALID_ARG
    assert lib.ocean_server_wait(None, 1, 0) == abi.OCEAN_ERROR_INVALID_ARG
    assert lib.ocean_server_drain(None, 0) == abi.OCEAN_ERROR_INVALID_ARG
    assert lib.ocean_server_session_state(None, 1) == abi.OCEAN_SESSION_CLOSED
    assert lib.ocean_server_close_session(None, 1) == abi.OCEAN_ERROR_INVALID_ARG
    s = abi.ServerStatsC()
    assert lib.ocean_server_get_stats(None, C.byref(s)) == abi.OCEAN_ERROR_INVALID_ARG
    # a bad struct_size is refused before any device work
    d = abi.ServerDescC()
    lib.ocean_server_desc_init(C.byref(d))
    d.struct_size = 0
    st = C.c_int(-1)
    assert not lib.ocean_server_create(C.byref(d), C.byref(st))
    assert st.value == abi.OCEAN_ERROR_INVALID_ARG


def test_poisson_arrivals_and_paths_are_seeded():
    a = W.poisson_arrivals(256, 20000.0, 0.5)
    b = W.poisson_arrivals(256, 20000.0, 0.5)
    assert all((x == y).all() for x, y in zip(a, b))
    times, sess, upd = a
    assert abs(len(times) - 10000) < 400 and (sess < 256).all() and 0.45 < upd.mean() < 0.55
    p = W.DiscPaths(3, seed=5)
    f0 = p.frame(1)
    assert len(f0) == 32 and (f0["kind"] == abi.OCEAN_SOURCE_CONTINUOUS).all()
    assert (f0["radius"] >= 0.5).all() and (f0["radius"] <= 4.0).all()
    speed = (f0["velocity_x"] ** 2 + f0["velocity_z"] ** 2) ** 0.5
    assert (speed <= 8.0 + 1e-5).all()
