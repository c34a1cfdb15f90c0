"""Benchmark: batched 512^2 ocean updates per second on B200.

Workload (one "step" = one frame of every ocean in the batch): the 512^2
foam patch - 250 m, 22 m/s wind, choppiness 1.5, orbital velocity on and
persistent advected foam (1 substep of 1/60 s per frame) - replicated over
`--batch` independent sea states (seeds 7, 8, ...), frames at t = k/60 s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One JSON line on stdout (rank 0). `value` is device-timed (CUDA events on
the launching stream, inputs resident in HBM); `e2e` is the same metric
through ocean_batch_update_host with pinned host buffers, the copies of every
output inside the timed region. Under torchrun every rank runs its own batch
(no data-path collective: the oceans are independent), and the time is the
max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# `value` is the plain FP32 form (bit-identical to the reference); the
# tensor-core form's throughput sits beside it in "tensor_core_form", the
# precise form's (FP64 stage blocks: like the tensor form, within 2e-6 of
# FP64) in "precise_form", and the serving loop's request latency in "p99_ms".
METRIC = "512^2 ocean updates/s: batched TC-FFT vs plain FP32 @<=2e-6 rel err; p99 ms"
UNIT = "updates/s"
N = 512
CELLS = N * N
# Algorithmic bytes per 512^2 update with velocity and persistent foam:
# read h0 (8 B/cell), write displacement + normal + velocity RGBA32F
# (48 B/cell), read + write the foam plane (8 B/cell) = 64 B/cell.
ALG_BYTES_PER_CELL = 64
# Split between the passes: the row pass reads h0 (8 B/cell); the column pass
# writes the three RGBA32F outputs and reads/writes foam (56 B/cell).
COL_ALG_BYTES_PER_CELL = 56
ROW_ALG_BYTES_PER_CELL = 8
# The reference bench_update unit (velocity and foam off): h0 read 8 B +
# displacement and normal RGBA32F written 32 B.
PLAIN_ALG_BYTES_PER_CELL = 40
L2_BYTES = 126 * 2 ** 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--batch", type=int, default=64, help="oceans per GPU")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--schedule", default="persistent", choices=["persistent", "chunked"])
    ap.add_argument("--form", default="exact", choices=["exact", "fast", "tensor", "precise"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the secondary workloads")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--extra", default=None,
                    choices=["bench_update_512", "cascade", "iwave", "ensemble", "serving", "large_sizes"],
                    help="run only this secondary workload and print its JSON object")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def rank_seeds(rank: int, batch: int, base: int = 7):
    """Seeds of the oceans rank `rank` owns: replicas never share a sea state,
    so the ranks' work is disjoint and needs no exchange."""
    return [base + rank * batch + b for b in range(batch)]


def max_over_ranks(value: float, dist, device) -> float:
    """The slowest rank's time (every rank takes this same collective)."""
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        j = json.loads(p.read_text())
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def smi_id(local: int) -> str:
    """nvidia-smi --id for the CUDA device (PCI bus id, so CUDA_VISIBLE_DEVICES
    remapping cannot point the sampler at another GPU)."""
    import torch

    p = torch.cuda.get_device_properties(local)
    try:
        return f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
    except AttributeError:
        return str(local)


def profile_traffic():
    """ncu DRAM bytes per column-pass launch from the committed profile summary."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return None
    return None


# ---------------------------------------------------------------------------
# Reference CPU implementation (the reference compiled from its own sources)
# ---------------------------------------------------------------------------
def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), as the reference's
    bench_update prints it beside its figures."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_rate(seconds: float, warm: int = 2, threads: int = 0):
    """Updates/s of the reference's own Ocean + FoamField on this host's cores
    for the same workload, sequential frames of one ocean with its built-in
    thread pool over all hardware threads (threads = 0, the reference's
    threaded path) or over `threads` threads."""
    import oracle as O
    from oceanlib_b200 import workloads as W

    desc = W.foam_patch_512()
    desc.thread_count = threads
    ro = O.RefOcean(desc)
    rf = O.RefFoam(ro, W.foam_desc(), thread_count=threads)
    cores = threads if threads > 0 else int(O.ref().oref_hardware_concurrency())
    dt = W.FOAM_DT
    frame = 0
    for _ in range(warm):
        frame += 1
        ro.update(frame * dt)
        rf.update(dt)
    done = 0
    t0 = time.perf_counter()
    while True:
        frame += 1
        ro.update(frame * dt)
        rf.update(dt)
        done += 1
        el = time.perf_counter() - t0
        if el >= seconds and done >= 3:
            break
    return done / el, cores, done


REF_TIMED_S = 2.5  # seconds the reference arm's timed steps span together


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    import oracle as O
    from oceanlib_b200 import workloads as W

    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference library not built"}))
        return
    desc = W.foam_patch_512()
    ro = O.RefOcean(desc)
    rf = O.RefFoam(ro, W.foam_desc())
    cores = int(O.ref().oref_hardware_concurrency())
    dt = W.FOAM_DT
    # Warm-up: at least W x 4 frames and 0.5 s, so the reference's thread pool
    # is running at speed; its rate sets the frames per step.
    frame = 0
    t0 = time.perf_counter()
    while True:
        frame += 1
        ro.update(frame * dt)
        rf.update(dt)
        el = time.perf_counter() - t0
        if frame >= args.warmup * 4 and el >= 0.5:
            break
    rate = frame / el
    # Frames of one ocean per step (a bounded sample of the batch frame):
    # enough for the K timed steps to span about REF_TIMED_S seconds, so the
    # figure is a steady rate and not a start-up transient.
    per_step = max(4, int(np.ceil(rate * REF_TIMED_S / max(1, args.steps))))
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for _ in range(per_step):
            frame += 1
            ro.update(frame * dt)
            rf.update(dt)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = per_step * args.steps / total
    ms = [1000.0 * t for t in times]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "foam_patch_512 (N=512, L=250 m, U=22 m/s, choppiness 1.5, "
                               "velocity + persistent foam, dt=1/60 s)",
                   "sample": f"{per_step} frames of one ocean per step"},
        "latency_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99))},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{per_step * args.steps} sequential frames of one 512^2 ocean, "
                                   f"reference thread pool over {cores} hardware threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# Secondary workloads (reported under "extra"; not the headline metric)
# ---------------------------------------------------------------------------
def bench_cascade(torch, queries: int = 1_000_000, frames: int = 50):
    """3 x 256^2 cascades (800/150/25 m, 30 m depth, velocity on): frames of
    all levels, then `queries` device-resident summed queries per frame, each
    timed back to back on the device (a frame is tens of microseconds, so a
    per-frame host synchronisation would time the host's enqueue as well)."""
    import oceanlib_b200 as ob
    from oceanlib_b200 import workloads as W

    cs = ob.CascadeStack(W.cascade_3x256())
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    with torch.cuda.stream(stream):
        xz = torch.from_numpy(W.cascade_query_points(queries)).cuda()
        out = torch.empty((queries, 10), dtype=torch.float32, device="cuda")
    for k in range(3):
        cs.update(k / 60.0, stream=sh)
        cs.sample_many_device(xz.data_ptr(), queries, out.data_ptr(), stream=sh)
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    for k in range(frames):
        cs.update(1.0 + k / 60.0, stream=sh)
    e1.record(stream)
    for k in range(frames):
        cs.sample_many_device(xz.data_ptr(), queries, out.data_ptr(), stream=sh)
    e2.record(stream)
    torch.cuda.synchronize()
    upd_ms = e0.elapsed_time(e1)
    q_ms = e1.elapsed_time(e2)
    res = {"workload": "cascade_3x256 + 1M summed queries (4 fixed-point steps)",
           "cascade_frames_per_s": frames / (upd_ms / 1000.0),
           "queries_per_s": queries * frames / (q_ms / 1000.0),
           "query_ms_per_1M": q_ms / frames * (1_000_000 / queries)}
    # converged inversion (to 1e-6 m, at most 64 steps)
    e1.record(stream)
    cs.sample_many_device(xz.data_ptr(), queries, out.data_ptr(), iterations=64, tolerance=1e-6, stream=sh)
    e2.record(stream)
    torch.cuda.synchronize()
    res["converged_queries_per_s"] = queries / (e1.elapsed_time(e2) / 1000.0)
    cs.close()
    # The same levels in the tensor-core form.
    from oceanlib_b200 import abi

    cs = ob.CascadeStack(W.cascade_3x256(), form=abi.OCEAN_FFT_TENSOR)
    for k in range(3):
        cs.update(k / 60.0, stream=sh)
    torch.cuda.synchronize()
    e0.record(stream)
    for k in range(frames):
        cs.update(1.0 + k / 60.0, stream=sh)
    e1.record(stream)
    torch.cuda.synchronize()
    res["tensor_core_form"] = {"cascade_frames_per_s": frames / (e0.elapsed_time(e1) / 1000.0)}
    cs.close()
    return res


def bench_large_sizes(torch, frames: int = 10):
    """N = 2048 and 4096, the reference's largest sizes (three launches per
    frame): device time per update with velocity on, oceans resident in HBM,
    frames back to back."""
    import oceanlib_b200 as ob

    res = {}
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    for n, count in ((2048, 4), (4096, 1)):
        descs = [ob.OceanDesc(size=n, patch_length=0.8 * n, wind_speed=15.0, seed=9 + k, compute_velocity=True)
                 for k in range(count)]
        b = ob.OceanBatch(descs)
        for k in range(3):
            b.update([1.0 + k / 60.0], stream=sh)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(frames):
            b.update([2.0 + k / 60.0], stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / frames
        alg = 56 * n * n  # h0 in; displacement, normal and velocity out
        res[str(n)] = {"workload": f"{count} x {n}^2, L = {0.8 * n:.0f} m, U = 15 m/s, velocity on",
                       "updates_per_s": count * 1000.0 / ms, "ms_per_frame": ms,
                       "gpu_launches_per_frame": 3, "alg_bytes_per_update": alg,
                       "achieved_gbs": alg * count / (ms / 1000.0) / 1e9}
        b.close()
    return res


def bench_large_reference(seconds: float = 2.0):
    """The reference Ocean at the same large descriptors, its thread pool over
    all hardware threads."""
    import oracle as O
    from oceanlib_b200 import OceanDesc

    res = {}
    for n in (2048, 4096):
        ro = O.RefOcean(OceanDesc(size=n, patch_length=0.8 * n, wind_speed=15.0, seed=9, compute_velocity=True))
        ro.update(1.0)
        t0 = time.perf_counter()
        k = 0
        while time.perf_counter() - t0 < seconds / 2 or k < 2:
            ro.update(2.0 + k / 60.0)
            k += 1
        res[str(n)] = {"updates_per_s": k / (time.perf_counter() - t0), "frames": k,
                       "threads": int(O.ref().oref_hardware_concurrency())}
        ro.close()
    return res


def bench_ensemble(torch, frames: int = 30):
    """64 seeded sea states of uneven N (64..1024), schedule picked by the
    autotuner; one frame = every ocean advanced once."""
    import oceanlib_b200 as ob
    from oceanlib_b200 import workloads as W

    descs = W.ensemble_64()
    ens = ob.OceanEnsemble(descs, autotune=True)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream

    def timed(graph: bool):
        ens.set_graph(graph)
        for k in range(3):
            ens.update(k / 60.0, stream=sh)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for k in range(frames):
            ens.update(1.0 + k / 60.0, stream=sh)
        b.record(stream)
        torch.cuda.synchronize()
        # host cost of issuing one frame, with the GPU idle
        host = []
        for k in range(10):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ens.update(2.0 + k / 60.0, stream=sh)
            host.append((time.perf_counter() - t0) * 1e6)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / frames, float(np.median(host))

    ms_calls, host_calls = timed(False)
    ms, host_graph = timed(True)  # the default: one graph replay per frame
    cells = sum(d.size * d.size for d in descs)
    res = {"workload": "ensemble_64 (N in 64..1024, seeded, velocity off)",
           "frames_per_s": 1000.0 / ms, "ms_per_frame": ms,
           "ocean_updates_per_s": len(descs) * 1000.0 / ms,
           "cells_per_s": cells * 1000.0 / ms,
           "equiv_512sq_updates_per_s": cells / (512 * 512) * 1000.0 / ms,
           "schedule": ens.schedule,
           "cuda_graph": {"ms_per_frame": ms, "host_us_per_update": host_graph},
           "per_call_launches": {"ms_per_frame": ms_calls, "host_us_per_update": host_calls}}
    # Every schedule forced in turn (graph replay), beside the autotuner's pick.
    per = {}
    for name, kind in (("sequential", ob.OceanEnsemble.SEQUENTIAL),
                       ("concurrent_work_shares", ob.OceanEnsemble.CONCURRENT),
                       ("one_launch", ob.OceanEnsemble.ONE_LAUNCH)):
        try:
            ens.set_schedule(kind)
        except ValueError:
            continue
        per[name] = timed(True)[0]
    res["schedules_ms_per_frame"] = per
    ens.close()
    # The same sea states in the tensor-core form (N = 64..512 on the tensor
    # cores, N = 1024 in the exact form), schedule again by the autotuner.
    from oceanlib_b200 import abi

    ens = ob.OceanEnsemble(descs, autotune=True, form=abi.OCEAN_FFT_TENSOR)
    ms_tc, _ = timed(True)
    res["tensor_core_form"] = {"ms_per_frame": ms_tc, "ocean_updates_per_s": len(descs) * 1000.0 / ms_tc,
                               "equiv_512sq_updates_per_s": cells / (512 * 512) * 1000.0 / ms_tc,
                               "schedule": ens.schedule}
    ens.close()
    # And in the precise form (every size, FP64 stage blocks), autotuned.
    ens = ob.OceanEnsemble(descs, autotune=True, form=abi.OCEAN_FFT_PRECISE)
    ms_pr, _ = timed(True)
    res["precise_form"] = {"ms_per_frame": ms_pr, "ocean_updates_per_s": len(descs) * 1000.0 / ms_pr,
                           "equiv_512sq_updates_per_s": cells / (512 * 512) * 1000.0 / ms_pr,
                           "schedule": ens.schedule}
    ens.close()
    return res


def bench_plain_update(torch, batch: int = 64, steps: int = 60, cpu_seconds: float = 0.0):
    """The reference bench_update unit of work (bench/bench_update.cpp:91-102,
    :72): 512^2, 200 m, 12 m/s, wind direction 0.4, choppiness 1, velocity
    and foam off (4 packed complex FFT fields); `batch` oceans with seeds
    1337 + b, step i at t = 100 + 0.0137 i. Algorithmic bytes: h0 read 8 B +
    displacement and normal RGBA32F written 32 B = 40 B/cell."""
    import oceanlib_b200 as ob
    from oceanlib_b200 import abi
    from oceanlib_b200 import workloads as W

    descs = [W.bench_update_patch(512, seed=1337 + b) for b in range(batch)]
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    alg_update = PLAIN_ALG_BYTES_PER_CELL * CELLS
    peak, peak_kind = measured_peaks()
    out = {"workload": "bench_update_512 (N=512, L=200 m, U=12 m/s, dir 0.4, choppiness 1, "
                       "velocity and foam off; seeds 1337+b, t = 100 + 0.0137 i)",
           "oceans_per_launch": batch, "alg_bytes_per_update": alg_update}

    def run(form):
        b = ob.OceanBatch(descs, form=form)
        step = [0]

        def one():
            b.update([100.0 + step[0] * 0.0137], stream=sh)
            step[0] += 1

        for _ in range(5):
            one()
        torch.cuda.synchronize()
        b.set_profiling(True)
        b.read_profile()
        l0 = b.launch_count
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        ev[0].record(stream)
        for i in range(steps):
            one()
            ev[i + 1].record(stream)
        torch.cuda.synchronize()
        prof = b.read_profile()
        b.set_profiling(False)
        launches = b.launch_count - l0
        total_ms = ev[0].elapsed_time(ev[-1])
        step_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]
        res = {"value": batch * steps / (total_ms / 1000.0), "unit": UNIT,
               "ms_per_step": total_ms / steps, "gpu_launches": int(launches),
               "latency_ms": {"p50": float(np.percentile(step_ms, 50)),
                              "p99": float(np.percentile(step_ms, 99))}}
        if prof["frame_launches"] > 0:
            launch_ms = prof["frame_ms"] / prof["frame_launches"]
            alg = alg_update * batch * steps / prof["frame_launches"]
            ach = alg / (launch_ms / 1000.0) / 1e9
            res["roofline"] = {"bound": "hbm", "kernel": "frame_kernel", "achieved": ach,
                               "peak": peak, "unit": "GB/s", "frac": ach / peak,
                               "peak_kind": peak_kind, "alg_bytes_per_launch": alg,
                               "avg_launch_ms": launch_ms}
        return b, res

    b, out["fp32"] = run(abi.OCEAN_FFT_EXACT)
    # end to end: displacement + normal copied to pinned host memory every step
    pinned = [torch.empty((batch, CELLS, 4), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    disp, nrm = (t.numpy() for t in pinned)
    for i in range(2):
        b.update_host([100.0 + i * 0.0137], 0.0, disp, nrm)
    e2e_steps = max(3, steps // 3)
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        b.update_host([100.0 + i * 0.0137], 0.0, disp, nrm)
    e2e_s = time.perf_counter() - t0
    out["e2e"] = {"value": batch * e2e_steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 8,
                  "d2h_bytes_per_step": batch * CELLS * 32,
                  "api": "ocean_batch_update_host (pinned host buffers)"}
    b.close()
    del pinned
    tb, out["tensor_core_form"] = run(abi.OCEAN_FFT_TENSOR)
    tb.close()
    out["tensor_core_form"]["vs_plain_fp32"] = out["tensor_core_form"]["value"] / out["fp32"]["value"]
    pb, out["precise_form"] = run(abi.OCEAN_FFT_PRECISE)
    pb.close()
    out["precise_form"]["vs_plain_fp32"] = out["precise_form"]["value"] / out["fp32"]["value"]
    if cpu_seconds > 0:
        import oracle as O

        ro = O.RefOcean(W.bench_update_patch(512))
        cores = int(O.ref().oref_hardware_concurrency())
        for i in range(2):
            ro.update(i * 0.013)
        done, t0 = 0, time.perf_counter()
        while True:
            ro.update(100.0 + done * 0.0137)
            done += 1
            el = time.perf_counter() - t0
            if el >= cpu_seconds and done >= 3:
                break
        out["reference_cpu"] = {"value": done / el, "unit": UNIT, "cores": cores,
                                "kind": "reference",
                                "sample": f"{done} sequential updates of one 512^2 ocean, "
                                          f"reference thread pool over {cores} hardware threads"}
    return out


def bench_cascade_reference(seconds: float = 4.0):
    import ctypes as C

    import oracle as O
    from oceanlib_b200 import workloads as W
    from oceanlib_b200.abi import OceanDescC

    levels = W.cascade_3x256()
    arr = (OceanDescC * 3)(*[O.c_desc_bytes(d) for d in levels])
    st = C.c_int(-1)
    h = O.ref().oref_cascade_create(arr, 3, C.byref(st))
    t0 = time.perf_counter()
    frames = 0
    while time.perf_counter() - t0 < seconds / 2 or frames < 2:
        O.ref().oref_cascade_update(h, 1.0 + frames / 60.0)
        frames += 1
    upd = frames / (time.perf_counter() - t0)
    xz = W.cascade_query_points(20_000)
    out = np.empty((xz.shape[0], 10), np.float32)
    t0 = time.perf_counter()
    reps = 0
    while time.perf_counter() - t0 < seconds / 2 or reps < 1:
        O.ref().oref_cascade_sample_many(h, xz.ctypes.data, xz.shape[0], out.ctypes.data)
        reps += 1
    q = reps * xz.shape[0] / (time.perf_counter() - t0)
    O.ref().oref_cascade_destroy(h)
    return {"cascade_frames_per_s": upd, "queries_per_s": q, "query_threads": 1,
            "update_threads": int(O.ref().oref_hardware_concurrency())}


def iwave_sources(extent: float, count: int = 32, seed: int = 11):
    """`count` continuous disc sources, radius 0.5-4 m, speed 0-8 m/s."""
    from oceanlib_b200.interaction import Disturbance

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        sp, hd = rng.uniform(0, 8), rng.uniform(0, 2 * np.pi)
        out.append(Disturbance(world_x=float(rng.uniform(0.2, 0.8) * extent),
                               world_z=float(rng.uniform(0.2, 0.8) * extent),
                               radius=float(rng.uniform(0.5, 4.0)), strength=0.05, velocity_y=-0.1,
                               velocity_x=float(sp * np.cos(hd)), velocity_z=float(sp * np.sin(hd)),
                               kind=1))
    return out


def bench_iwave(updates: int = 60):
    """A 512^2, 64 m iWave field (P = 6) with 32 moving disc sources, one
    1/60 s substep per update, through the reference-shaped update call (which
    also refreshes the host mirror)."""
    from oceanlib_b200.interaction import InteractionDesc, InteractionField

    desc = InteractionDesc(size=512, extent=64.0, kernel_radius=6, max_sources=64)
    f = InteractionField(desc)
    src = iwave_sources(desc.extent)
    for _ in range(5):
        for d in src:
            f.add(d)
        f.update(1.0 / 60.0)
    t0 = time.perf_counter()
    for _ in range(updates):
        for d in src:
            f.add(d)
        f.update(1.0 / 60.0)
    el = time.perf_counter() - t0
    f.close()
    return {"workload": "iwave 512^2 x 64 m, P=6, 32 moving disc sources, dt=1/60 s",
            "updates_per_s": updates / el, "ms_per_update": 1000.0 * el / updates,
            "includes": "source stamps, 169-tap step, finalize, 4 MiB host mirror copy"}


def bench_iwave_reference(updates: int = 20):
    import ctypes as C

    import oracle as O
    from oracle import iwave as OI
    from oceanlib_b200.interaction import InteractionDesc

    desc = InteractionDesc(size=512, extent=64.0, kernel_radius=6, max_sources=64)
    r = OI.RefInteraction(desc)
    src = iwave_sources(desc.extent)
    arr = (type(src[0].to_c()) * len(src))(*[d.to_c() for d in src])
    O.ref().oref_i_time_updates(r.h, arr, len(src), 3, 1.0 / 60.0)
    el = O.ref().oref_i_time_updates(r.h, arr, len(src), updates, 1.0 / 60.0)
    return {"updates_per_s": updates / el, "ms_per_update": 1000.0 * el / updates,
            "threads": int(O.ref().oref_hardware_concurrency())}


def _serve_script(paths, sess, upd, pts, frames):
    """Pre-built requests (session, frame number or 0, sources or None,
    points or None); `frames` holds each session's last frame and advances."""
    out = []
    for i, (s, u) in enumerate(zip(sess.tolist(), upd.tolist())):
        if u:
            frames[s] += 1
            out.append((s, frames[s], paths.frame(s), None))
        else:
            out.append((s, 0, None, pts[i % len(pts)]))
    return out


def _serve_run(srv, sids, script, times):
    """Submits `script` at the arrival `times` (open loop; None = as fast as
    possible), drains, returns the wall seconds from the first submission to
    the last result."""
    import numpy as np

    from oceanlib_b200 import workloads as W

    outs = [np.empty(4096, np.float32) for _ in range(256)]
    t0 = time.perf_counter()
    for i, (s, f, src, xz) in enumerate(script):
        if times is not None:
            while time.perf_counter() - t0 < times[i]:
                pass
        if src is not None:
            srv.submit_update(sids[s], f * W.SERVE_DT, W.SERVE_DT, src)
        else:
            srv.submit_query(sids[s], xz, outs[i % 256])
    srv.drain()
    return time.perf_counter() - t0


def bench_serving(rate: float = 20000.0, seconds: float = 3.0):
    """The serving loop: 256 sessions (ocean N in {128, 256, 512}, a 512^2
    interaction field with 32 moving disc sources each), update and
    4096-point height requests arriving as a Poisson process of mean `rate`
    per second, admitted under a 120 GB budget. Latency is submit -> result
    in the caller's buffer (host clock), so it includes the uploads of the
    sources and points and the download of the heights."""
    from oceanlib_b200 import workloads as W
    from oceanlib_b200.serve import OceanServer

    oceans, field = W.serving_sessions(256)
    srv = OceanServer(hbm_budget=120e9)
    sids = [srv.open_session(o, field) for o in oceans]
    pts = W.serving_points(sets=16)
    frames = [0] * 256

    paths = W.DiscPaths(256)

    def run(duration, seed, paced=True):
        times, sess, upd = W.poisson_arrivals(256, rate, duration, seed=seed)
        script = _serve_script(paths, sess, upd, pts, frames)
        srv.reset_stats()
        wall = _serve_run(srv, sids, script, times if paced else None)
        return wall, len(script), srv.stats()

    run(1.0, 1)  # warm-up: admission, t = 0 frames, staging growth
    wall, n, st = run(seconds, 2)
    import numpy as np

    _, lat, _ = srv.latency_samples()
    p999 = float(np.quantile(lat, 0.999)) if len(lat) else 0.0
    slow = int((lat > 10.0).sum())
    cap_wall, cap_n, cap = run(seconds / 2, 3, paced=False)
    out = {
        "workload": "256 sessions (ocean N from {128,256,512} by PCG32(5,0); 512^2 iWave field, 64 m, "
                    "P=6, 32 continuous disc sources on random-walk paths), Poisson arrivals, "
                    "50% updates / 50% 4096-point height queries",
        "offered_rps": n / seconds,
        "achieved_rps": st["requests_completed"] / wall,
        "latency_p50_ms": st["latency_p50_ms"],
        "latency_p99_ms": st["latency_p99_ms"],
        "latency_p999_ms": p999,
        "latency_max_ms": st["latency_max_ms"],
        "requests_over_10ms": slow,
        "update_p50_ms": st["update_p50_ms"], "update_p99_ms": st["update_p99_ms"],
        "query_p50_ms": st["query_p50_ms"], "query_p99_ms": st["query_p99_ms"],
        "updates_per_s": st["updates_completed"] / wall,
        "query_points_per_s": st["query_points_completed"] / wall,
        "batches": st["batches"], "mean_batch_requests": st["mean_batch_requests"],
        "gpu_busy_fraction": st["gpu_busy_ms"] / (1000.0 * wall),
        "kernel_launches": st["kernel_launches"],
        "sessions_active": st["sessions_active"], "bytes_in_use": st["bytes_in_use"],
        "hbm_budget": st["hbm_budget"], "failed": st["requests_failed"],
        "dispatch_max_ms": st["dispatch_max_ms"], "staging_growths": st["staging_growths"],
        "capacity_closed_loop_rps": cap["requests_completed"] / cap_wall,
        "capacity_p99_ms": cap["latency_p99_ms"],
        "capacity_mean_batch_requests": cap["mean_batch_requests"],
    }
    srv.close()
    # The same sessions and arrivals with every ocean in the tensor-core form.
    from oceanlib_b200 import abi

    srv = OceanServer(hbm_budget=120e9, form=abi.OCEAN_FFT_TENSOR)
    sids = [srv.open_session(o, field) for o in oceans]
    run(1.0, 1)
    wall, n, st = run(seconds, 2)
    out["tensor_core_form"] = {"offered_rps": n / seconds, "achieved_rps": st["requests_completed"] / wall,
                               "latency_p50_ms": st["latency_p50_ms"], "latency_p99_ms": st["latency_p99_ms"],
                               "update_p99_ms": st["update_p99_ms"], "query_p99_ms": st["query_p99_ms"],
                               "gpu_busy_fraction": st["gpu_busy_ms"] / (1000.0 * wall),
                               "failed": st["requests_failed"]}
    srv.close()
    return out


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch

    torch.cuda.set_device(local)
    if args.extra is not None:
        fn = {"bench_update_512": lambda: bench_plain_update(torch), "cascade": lambda: bench_cascade(torch),
              "iwave": bench_iwave, "ensemble": lambda: bench_ensemble(torch), "serving": bench_serving,
              "large_sizes": lambda: bench_large_sizes(torch)}[args.extra]
        print(json.dumps({"extra": args.extra, "result": fn()}))
        return
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    import oceanlib_b200 as ob
    from oceanlib_b200 import workloads as W

    B = args.batch
    descs = [W.foam_patch_512(seed=s) for s in rank_seeds(rank, B)]
    from oceanlib_b200 import abi

    batch = ob.OceanBatch(descs, foam=W.foam_desc(), chunk=args.chunk,
                          form={"exact": abi.OCEAN_FFT_EXACT, "fast": abi.OCEAN_FFT_FAST,
                                "tensor": abi.OCEAN_FFT_TENSOR, "precise": abi.OCEAN_FFT_PRECISE}[args.form],
                          schedule=abi.OCEAN_SCHEDULE_CHUNKED if args.schedule == "chunked"
                          else abi.OCEAN_SCHEDULE_PERSISTENT)
    # An explicit stream: the library launches on it and the CUDA events
    # below are recorded on it, so they bracket exactly the frame kernels.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    assert sh != 0
    dt = W.FOAM_DT
    frame = 0

    def step():
        nonlocal frame
        frame += 1
        batch.update([frame * dt], foam_dt=dt, stream=sh)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()

    # ---- device-timed region ----
    batch.set_profiling(True)
    batch.read_profile()  # reset
    launches0 = batch.launch_count
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    clocks = ClockSampler(smi_id(local))
    clocks.start()
    time.sleep(0.4)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    evs[0].record(stream)
    for i in range(args.steps):
        step()
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    step_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    total_ms = evs[0].elapsed_time(evs[-1])
    prof = batch.read_profile()
    batch.set_profiling(False)
    launches = batch.launch_count - launches0

    if world > 1:
        total_ms = max_over_ranks(total_ms, torch.distributed, "cuda")
    updates = B * args.steps * world
    value = updates / (total_ms / 1000.0)

    # ---- end to end through the C ABI with pinned host buffers ----
    pinned = [torch.empty((B, CELLS, 4), dtype=torch.float32, pin_memory=True) for _ in range(3)]
    pinned.append(torch.empty((B, CELLS), dtype=torch.float32, pin_memory=True))
    disp, nrm, vel, foam = (t.numpy() for t in pinned)
    e2e_steps = max(3, args.steps // 3)
    for _ in range(2):
        frame += 1
        batch.update_host([frame * dt], dt, disp, nrm, vel, foam)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        frame += 1
        batch.update_host([frame * dt], dt, disp, nrm, vel, foam)
    e2e_s = time.perf_counter() - t0
    if world > 1:
        e2e_s = max_over_ranks(e2e_s, torch.distributed, "cuda")
    e2e_value = B * e2e_steps * world / e2e_s
    d2h = B * CELLS * (3 * 16 + 4)
    h2d = 8  # one absolute time per frame (double)

    # ---- the same, narrowed to RGBA16F on the device (the viewer's upload format) ----
    half = [torch.empty((B, CELLS, 4), dtype=torch.int16, pin_memory=True) for _ in range(3)]
    hd, hn, hv = (t.numpy().view(np.uint16) for t in half)
    for _ in range(2):
        frame += 1
        batch.update_host_rgba16([frame * dt], dt, hd, hn, hv)
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        frame += 1
        batch.update_host_rgba16([frame * dt], dt, hd, hn, hv)
    h_s = time.perf_counter() - t0
    if world > 1:
        h_s = max_over_ranks(h_s, torch.distributed, "cuda")
    e2e_half = {"value": B * e2e_steps * world / h_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": B * CELLS * 3 * 8,
                "api": "ocean_batch_update_host_rgba16 (RGBA16F packed on the device, foam in the alpha)"}

    # ---- the tensor-core and precise forms on the same workload, beside the
    # FP32 form (both within 2e-6 of FP64 on every channel) ----
    def other_form(form, kernel):
        ob_ = ob.OceanBatch(descs, foam=W.foam_desc(), form=form)
        fr = 0

        def step():
            nonlocal fr
            fr += 1
            ob_.update([fr * dt], foam_dt=dt, stream=sh)

        for _ in range(max(3, args.warmup)):
            step()
        torch.cuda.synchronize()
        steps = max(5, args.steps // 3)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        if world > 1:
            torch.distributed.barrier()
        launches0 = ob_.launch_count
        ev[0].record(stream)
        for _ in range(steps):
            step()
        ev[1].record(stream)
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1])
        if world > 1:
            ms = max_over_ranks(ms, torch.distributed, "cuda")
        out = {"value": B * steps * world / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms / steps,
               "steps": steps, "gpu_launches": int(ob_.launch_count - launches0), "kernel": kernel}
        ob_.close()
        return out

    tc = None
    if args.form != "tensor":
        tc = other_form(abi.OCEAN_FFT_TENSOR,
                        "frame_kernel, tensor form (tcgen05 four-step DFT, exact FP16 digit-slice GEMMs)")
    precise = None
    if args.form != "precise":
        precise = other_form(abi.OCEAN_FFT_PRECISE,
                             "frame_kernel, precise form (radix-2 stage blocks in FP64, FP32 between them)")

    if rank == 0:
        peak, peak_kind = measured_peaks()
        frame_achieved = ALG_BYTES_PER_CELL * CELLS * (value / world) / 1e9
        traffic = profile_traffic()
        if prof["frame_launches"] > 0:
            # Persistent schedule: one frame kernel per step does all the work.
            launch_ms = prof["frame_ms"] / prof["frame_launches"]
            oceans_per_launch = B * args.steps / prof["frame_launches"]
            alg = ALG_BYTES_PER_CELL * CELLS * oceans_per_launch
            achieved = alg / (launch_ms / 1000.0) / 1e9
            roof = {"bound": "hbm", "kernel": "frame_kernel (persistent: evolve + row FFT, "
                                              "column FFT + finalize + foam)",
                    "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "peak_kind": peak_kind, "alg_bytes_per_launch": alg, "avg_launch_ms": launch_ms,
                    "traffic": None if traffic is None else traffic.get("frame_bytes_per_launch"),
                    "frame": {"achieved": frame_achieved, "frac": frame_achieved / peak,
                              "alg_bytes_per_update": ALG_BYTES_PER_CELL * CELLS}}
            # The unit that bounds this kernel, from the committed ncu capture of
            # the same kernel and workload (HBM is not it).
            if traffic is not None and "binding_unit" in traffic:
                roof["binding_unit"] = traffic["binding_unit"]
        else:
            col_launch_ms = prof["col_ms"] / max(1, prof["col_launches"])
            row_launch_ms = prof["row_ms"] / max(1, prof["row_launches"])
            oceans_per_launch = B * args.steps / max(1, prof["col_launches"])
            col_alg = COL_ALG_BYTES_PER_CELL * CELLS * oceans_per_launch
            row_alg = ROW_ALG_BYTES_PER_CELL * CELLS * oceans_per_launch
            col_achieved = col_alg / (col_launch_ms / 1000.0) / 1e9
            tot = max(1e-9, prof["row_ms"] + prof["col_ms"])
            roof = {"bound": "hbm", "kernel": "col_pass (column FFT + finalize + foam)",
                    "achieved": col_achieved, "peak": peak, "unit": "GB/s",
                    "frac": col_achieved / peak, "peak_kind": peak_kind,
                    "alg_bytes_per_launch": col_alg, "avg_launch_ms": col_launch_ms,
                    "traffic": None if traffic is None else traffic.get("col_bytes_per_launch"),
                    "row_pass": {"avg_launch_ms": row_launch_ms, "alg_bytes_per_launch": row_alg,
                                 "achieved": row_alg / (row_launch_ms / 1000.0) / 1e9},
                    "frame": {"achieved": frame_achieved, "frac": frame_achieved / peak,
                              "alg_bytes_per_update": ALG_BYTES_PER_CELL * CELLS},
                    "share": {"row": prof["row_ms"] / tot, "col": prof["col_ms"] / tot}}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "foam_patch_512 (N=512, L=250 m, U=22 m/s, choppiness 1.5, "
                                   "velocity + persistent foam, dt=1/60 s)",
                       "oceans_per_gpu": B, "grid": N, "fft_form": args.form,
                       "schedule": args.schedule,
                       "oceans_per_launch": int(round(oceans_per_launch)),
                       "l2": f"inputs larger than L2 (per-step working set "
                             f"{B * CELLS * 72 / 2**30:.2f} GiB > 126 MB)",
                       "parallelism": f"replicas x{world}"},
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)),
                           "p99": float(np.percentile(step_ms, 99))},
            "roofline": roof,
            "gpu_launches": int(launches),
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "api": "ocean_batch_update_host (pinned host buffers)",
                    # device -> host bytes per second over the end-to-end steps: the
                    # PCIe link's rate, which bounds this figure (the frame itself
                    # takes a few per cent of each step)
                    "d2h_gbs_per_gpu": d2h * e2e_steps / e2e_s / 1e9,
                    "rgba16": e2e_half},
        }
        if tc is not None:
            tc["vs_plain_fp32"] = tc["value"] / value
            line["tensor_core_form"] = tc
        if precise is not None:
            precise["vs_plain_fp32"] = precise["value"] / value
            line["precise_form"] = precise
        if not args.no_extra and world == 1:
            extra = {}
            plain_cpu = 0.0 if args.no_cpu_baseline else 4.0
            for name, fn in (("bench_update_512", lambda: bench_plain_update(torch, cpu_seconds=plain_cpu)),
                             ("cascade", lambda: bench_cascade(torch)), ("iwave", bench_iwave),
                             ("ensemble", lambda: bench_ensemble(torch)), ("serving", bench_serving),
                             ("large_sizes", lambda: bench_large_sizes(torch))):
                try:
                    extra[name] = fn()
                except Exception as e:  # report, do not lose the headline line
                    extra[name] = {"error": str(e)}
            if not args.no_cpu_baseline:
                for name, fn in (("cascade", bench_cascade_reference), ("iwave", bench_iwave_reference),
                                 ("large_sizes", bench_large_reference)):
                    try:
                        extra[name]["reference_cpu"] = fn()
                    except Exception as e:
                        extra[name]["reference_cpu"] = {"error": str(e)}
            line["extra"] = extra
            srv = extra.get("serving", {})
            if "latency_p99_ms" in srv:
                line["p99_ms"] = {"value": srv["latency_p99_ms"], "p50": srv["latency_p50_ms"],
                                  "what": "serving loop request -> result in host memory, "
                                          f"{srv['offered_rps']:.0f} requests/s offered over 256 sessions"}
        if not args.no_cpu_baseline and world == 1:
            try:
                import oracle as O

                rate, cores, frames = reference_rate(args.cpu_seconds)
                rate1, _, frames1 = reference_rate(min(args.cpu_seconds, 4.0), threads=1)
                line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                                        "sample": f"{frames} sequential frames of one 512^2 ocean "
                                                  f"(reference Ocean + FoamField, its thread pool "
                                                  f"over {cores} hardware threads)",
                                        "cpu_model": cpu_model(),
                                        "simd_level": O.ref().oref_c_simd_level().decode(),
                                        "single_thread": {"value": rate1, "unit": UNIT, "cores": 1,
                                                          "sample": f"{frames1} sequential frames, "
                                                                    "thread_count = 1"}}
            except Exception as e:  # the checker is optional on a box without it
                line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": None, "kind": "reference",
                                        "sample": f"unavailable: {e}"}
        print(json.dumps(line))
    batch.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
