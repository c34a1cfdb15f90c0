"""The serving loop on the GPU: each session's results are the same alone,
in a mix of sessions batched together, and through the single-session
handles (Ocean + InteractionField + the combined query); admission waits
for the HBM budget and resumes when a session closes."""
import threading
import time

import numpy as np
import pytest

import oceanlib_b200 as ob
from oceanlib_b200 import abi
from oceanlib_b200 import workloads as W
from oceanlib_b200.interaction import Disturbance, InteractionField, sample_combined_many
from oceanlib_b200.serve import OceanServer, session_bytes

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _device(cuda_device):
    ob.force_simd_level(None)
    yield


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def scripts(count, frames=5, seed=3):
    """Per session: frames x (update with its 32 moving sources), with height
    queries before the first update, after update 2 and after the last."""
    paths = W.DiscPaths(count, seed=seed)
    pts = W.serving_points(sets=4, count=1000)
    out = []
    for s in range(count):
        sc = [("query", pts[s % 4])]
        for f in range(frames):
            sc.append(("update", (f + 1) * W.SERVE_DT, W.SERVE_DT, paths.frame(s)))
            if f == 2 or f == frames - 1:
                sc.append(("query", pts[(s + f) % 4]))
        out.append(sc)
    return out


def run_server(oceans, field, picks, sc, order_seed=None, threads=1, form=abi.OCEAN_FFT_EXACT):
    """Opens `picks` sessions, submits their scripts (interleaved at random
    when order_seed is given, keeping each session's own order), drains, and
    returns {session: (heights list, disp, normal, field)}."""
    srv = OceanServer(form=form)
    sid = {k: srv.open_session(oceans[k], field) for k in picks}
    heights = {k: [] for k in picks}
    steps = [(k, i) for k in picks for i in range(len(sc[k]))]
    if order_seed is not None:
        rng = np.random.default_rng(order_seed)
        pos = {k: 0 for k in picks}
        steps = []
        live = list(picks)
        while live:
            k = live[rng.integers(len(live))]
            steps.append((k, pos[k]))
            pos[k] += 1
            if pos[k] == len(sc[k]):
                live.remove(k)

    def submit(chunk):
        for k, i in chunk:
            item = sc[k][i]
            if item[0] == "update":
                srv.submit_update(sid[k], item[1], item[2], item[3])
            else:
                out = np.empty(len(item[1]), np.float32)
                heights[k].append(out)
                srv.submit_query(sid[k], item[1], out)

    if threads == 1:
        submit(steps)
    else:
        # each thread owns a subset of the sessions (its order kept)
        groups = [[st for st in steps if picks.index(st[0]) % threads == t] for t in range(threads)]
        ts = [threading.Thread(target=submit, args=(g,)) for g in groups]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
    srv.drain()
    res = {}
    for k in picks:
        d, n, f = srv.read_session(sid[k], oceans[k].size, field.size)
        res[k] = (heights[k], d, n, f)
    st = srv.stats()
    srv.close()
    return res, st


def run_standalone(ocean_desc, field_desc, sc):
    ocean = ob.Ocean(ocean_desc)
    fld = InteractionField(field_desc)
    heights = []
    for item in sc:
        if item[0] == "update":
            ocean.update(item[1])
            for row in item[3]:
                fld.add(Disturbance(**{k: row[k].item() for k in row.dtype.names}))
            fld.update(item[2])
        else:
            heights.append(sample_combined_many(ocean, fld, item[1])[:, 0].copy())
    b = ocean.buffers()
    d, n = b["displacement"].copy(), b["normal"].copy()
    f = fld.buffers()["field"].copy()
    ocean.close()
    fld.close()
    return heights, d, n, f


def test_results_are_the_same_alone_in_the_mix_and_standalone():
    oceans, field = W.serving_sessions(12)
    sizes = {o.size for o in oceans}
    assert sizes == {128, 256, 512}
    sc = scripts(12)
    picks = [next(i for i, o in enumerate(oceans) if o.size == n) for n in (128, 256, 512)]
    alone = {k: run_server(oceans, field, [k], sc)[0][k] for k in picks}
    mix, st = run_server(oceans, field, list(range(12)), sc, order_seed=5)
    mix_mt, _ = run_server(oceans, field, list(range(12)), sc, order_seed=9, threads=3)
    assert st["requests_failed"] == 0
    assert st["batches"] >= 1 and st["updates_completed"] == 12 * 5
    for k in picks:
        ref = run_standalone(oceans[k], field, sc[k])
        for got in (alone[k], mix[k], mix_mt[k]):
            assert len(got[0]) == len(ref[0]) == 3
            for h, r in zip(got[0], ref[0]):
                assert np.array_equal(bits(h), bits(r)), oceans[k].size
            assert np.array_equal(bits(got[1]), bits(ref[1].reshape(got[1].shape)))
            assert np.array_equal(bits(got[2]), bits(ref[2].reshape(got[2].shape)))
            assert np.array_equal(bits(got[3]), bits(ref[3].reshape(got[3].shape)))
        # the field actually moved and the ocean is not at rest
        assert np.abs(ref[3][..., 0]).max() > 1e-4
        assert np.abs(ref[1][..., 1]).max() > 0.1


def test_admission_waits_for_the_budget_and_resumes_on_close():
    desc = ob.OceanDesc(size=128, seed=77)
    b = session_bytes(desc)
    # the 128^2 frame kernel's shared tables: intermediate ring + twiddles
    kind = (3 * 128 * 128 * 4 * 8 + 255) // 256 * 256 + (127 * 8 + 255) // 256 * 256
    srv = OceanServer(hbm_budget=2 * b + kind)
    s1 = srv.open_session(desc)
    s2 = srv.open_session(ob.OceanDesc(size=128, seed=78))
    s3 = srv.open_session(ob.OceanDesc(size=128, seed=79))
    pts = W.serving_points(sets=1, count=256, extent=200.0)[0]
    out = np.empty(256, np.float32)
    t_up = srv.submit_update(s3, 2.5, 0.0)
    t_q = srv.submit_query(s3, pts, out)
    deadline = time.time() + 20
    while srv.state(s2) != abi.OCEAN_SESSION_ACTIVE and time.time() < deadline:
        time.sleep(0.01)
    assert srv.state(s1) == abi.OCEAN_SESSION_ACTIVE and srv.state(s2) == abi.OCEAN_SESSION_ACTIVE
    assert srv.state(s3) == abi.OCEAN_SESSION_WAITING
    assert srv.wait(t_q, 200) == abi.OCEAN_ERROR_TIMEOUT
    st = srv.stats()
    assert st["sessions_waiting"] == 1 and st["bytes_in_use"] <= 2 * b + kind
    srv.close_session(s1)
    assert srv.wait(t_up, 20000) == abi.OCEAN_OK
    assert srv.wait(t_q, 20000) == abi.OCEAN_OK
    assert srv.state(s3) == abi.OCEAN_SESSION_ACTIVE
    assert srv.state(s1) == abi.OCEAN_SESSION_CLOSED
    o = ob.Ocean(ob.OceanDesc(size=128, seed=79))
    o.update(2.5)
    ref = o.sample_many(pts)[:, 0]
    assert np.array_equal(bits(out), bits(ref))
    o.close()
    srv.close()


def test_bad_requests_are_refused():
    srv = OceanServer(hbm_budget=10_000_000)
    with pytest.raises(MemoryError):
        srv.open_session(ob.OceanDesc(size=1024))
    with pytest.raises(ValueError):
        srv.open_session(ob.OceanDesc(size=100))
    sid = srv.open_session(ob.OceanDesc(size=64))
    with pytest.raises(ob.OceanError):
        srv.submit_update(sid + 7, 1.0, 0.0)
    assert srv.wait(12345, 0) == abi.OCEAN_ERROR_INVALID_ARG
    srv.close_session(sid)
    with pytest.raises(ob.OceanError):
        srv.submit_update(sid, 1.0, 0.0)  # closing: no new requests
    srv.drain()
    srv.close()


def test_poisson_load_completes_with_batching():
    oceans, field = W.serving_sessions(32)
    srv = OceanServer()
    sids = [srv.open_session(o, field) for o in oceans]
    paths = W.DiscPaths(32)
    pts = W.serving_points(sets=4)
    times, sess, upd = W.poisson_arrivals(32, 20000.0, 0.2)
    frame = [0] * 32
    outs = []
    t0 = time.perf_counter()
    for t, s, u in zip(times, sess, upd):
        while time.perf_counter() - t0 < t:
            pass
        if u:
            frame[s] += 1
            srv.submit_update(sids[s], frame[s] * W.SERVE_DT, W.SERVE_DT, paths.frame(s))
        else:
            o = np.empty(4096, np.float32)
            outs.append(o)
            srv.submit_query(sids[s], pts[len(outs) % 4], o)
    srv.drain()
    st = srv.stats()
    srv.close()
    assert st["requests_completed"] == len(times) and st["requests_failed"] == 0
    assert st["mean_batch_requests"] > 1.0
    assert 0.0 < st["latency_p50_ms"] <= st["latency_p99_ms"] <= st["latency_max_ms"]
    assert all(np.isfinite(o).all() for o in outs)


def test_tensor_form_sessions_match_tensor_form_batches():
    # The serving loop in the tensor-core form (config 5's sizes 128, 256 and
    # 512 all have it): each session's ocean, batched with the others, equals
    # a tensor-form batch of that ocean alone at the same time, bit for bit;
    # a size without the form is refused when the session opens.
    oceans, field = W.serving_sessions(6)
    sc = scripts(6, frames=3)
    mix, st = run_server(oceans, field, list(range(6)), sc, order_seed=4, form=abi.OCEAN_FFT_TENSOR)
    assert st["requests_failed"] == 0 and st["updates_completed"] == 6 * 3
    for k in range(6):
        t_last = [item[1] for item in sc[k] if item[0] == "update"][-1]
        n = oceans[k].size
        b = ob.OceanBatch([oceans[k]], form=abi.OCEAN_FFT_TENSOR)
        d = np.empty((n * n, 4), np.float32)
        nrm = np.empty_like(d)
        b.update_host([t_last], 0.0, d, nrm)
        b.close()
        assert np.array_equal(bits(mix[k][1]), bits(d.reshape(mix[k][1].shape))), n
        assert np.array_equal(bits(mix[k][2]), bits(nrm.reshape(mix[k][2].shape))), n
    srv = OceanServer(form=abi.OCEAN_FFT_TENSOR)
    with pytest.raises((ValueError, ob.OceanError)):
        srv.open_session(ob.OceanDesc(size=1024, seed=3), field)
    srv.close()


def test_precise_form_sessions_match_precise_form_batches():
    # The serving loop in the precise form (FP64 stage blocks): each
    # session's ocean, batched with sessions of other sizes in one launch,
    # equals a precise-form batch of that ocean alone, bit for bit.
    oceans, field = W.serving_sessions(6)
    sc = scripts(6, frames=2)
    mix, st = run_server(oceans, field, list(range(6)), sc, order_seed=7, form=abi.OCEAN_FFT_PRECISE)
    assert st["requests_failed"] == 0 and st["updates_completed"] == 6 * 2
    for k in range(6):
        t_last = [item[1] for item in sc[k] if item[0] == "update"][-1]
        n = oceans[k].size
        b = ob.OceanBatch([oceans[k]], form=abi.OCEAN_FFT_PRECISE)
        d = np.empty((n * n, 4), np.float32)
        nrm = np.empty_like(d)
        b.update_host([t_last], 0.0, d, nrm)
        b.close()
        assert np.array_equal(bits(mix[k][1]), bits(d.reshape(mix[k][1].shape))), n
        assert np.array_equal(bits(mix[k][2]), bits(nrm.reshape(mix[k][2].shape))), n
