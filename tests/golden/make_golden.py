"""Regenerates the golden fixtures in this folder from the REFERENCE library
(oracle/_ref/libocean_ref.so, compiled from the reference's own sources by
oracle/Makefile). Run here, where the reference sources exist:

    python tests/golden/make_golden.py           # every fixture
    python tests/golden/make_golden.py hashes    # only the named ones

Outputs
  ref_small.npz    full tables and frame outputs for small grids (N <= 64)
  ref_hashes.json  sha256 of the reference's output bytes at full sizes,
                   so GPU tests can check bit-exactness at N = 128 ... 4096
                   without storing the arrays
  ref_queries.npz  reference sample_at results for seeded query points
  ref_cascade.npz  reference CascadeStack::sample_at results (3 levels)
  ref_pack.json    sha256 of the viewer's RGBA16F pack over seeded bit patterns
  ref_foam.json    FoamField::foam_at / coverage / set_desc / clear on the foam patch
  ref_foam_long.json  the foam patch's FoamField over 1000 frames at 60 Hz:
                   sha256 of the foam plane, coverage and plane statistics
                   at the checkpoint frames
  abi_layout.json  offsets/sizes of the reference's C structs (include/ocean/ocean.h)
"""
from __future__ import annotations

import hashlib
import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle as O  # noqa: E402
from oceanlib_b200.abi import OceanDescC  # noqa: E402
from tests.workloads import (SMALL_CASES, HASH_CASES, FOAM_CASE, QUERY_CASE, CASCADE_CASE,  # noqa: E402
                             FOAM_QUERY_FRAMES, FOAM_RETUNE, FOAM_LONG_CASE, FOAM_LONG_CHECKPOINTS,
                             desc_to_json, query_points, cascade_points, pack_patterns)

HERE = Path(__file__).resolve().parent


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def small() -> None:
    arrays = {}
    meta = []
    for i, (desc, times) in enumerate(SMALL_CASES):
        arrays[f"c{i}_tables"] = O.ref_tables(desc)
        ro = O.RefOcean(desc)
        for j, t in enumerate(times):
            ro.update(t)
            d, n, v = ro.buffers()
            arrays[f"c{i}_t{j}_disp"] = d
            arrays[f"c{i}_t{j}_normal"] = n
            if v is not None:
                arrays[f"c{i}_t{j}_vel"] = v
        meta.append({"desc": desc_to_json(desc), "times": list(times)})
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(HERE / "ref_small.npz", **arrays)


def hashes() -> None:
    out = {"cases": []}
    for desc, times in HASH_CASES:
        tables = O.ref_tables(desc)
        h0 = np.stack([tables[0], tables[1]], axis=1)  # interleaved complex
        entry = {"desc": desc_to_json(desc), "h0": sha(h0), "frames": []}
        ro = O.RefOcean(desc)
        for t in times:
            ro.update(t)
            d, n, v = ro.buffers()
            fr = {"t": t, "disp": sha(d), "normal": sha(n)}
            if v is not None:
                fr["vel"] = sha(v)
            entry["frames"].append(fr)
        out["cases"].append(entry)
    # Persistent foam: the reference FoamField after each of `frames` frames.
    desc, foam, frames, dt = FOAM_CASE
    ro = O.RefOcean(desc)
    rf = O.RefFoam(ro, foam)
    foam_hashes = []
    for k in range(frames):
        ro.update((k + 1) * dt)
        rf.update(dt)
        foam_hashes.append(sha(rf.data()))
    out["foam"] = {"desc": desc_to_json(desc), "frames": frames, "dt": dt,
                   "hashes": foam_hashes, "coverage_last": float(rf.data().mean())}
    (HERE / "ref_hashes.json").write_text(json.dumps(out, indent=1))


def queries() -> None:
    desc, t, count = QUERY_CASE
    ro = O.RefOcean(desc)
    ro.update(t)
    xz = query_points(desc, count)
    res = ro.sample_many(xz)
    np.savez_compressed(HERE / "ref_queries.npz", xz=xz, out=res)


def cascades() -> None:
    import ctypes as C

    levels, t, count = CASCADE_CASE
    arr = (OceanDescC * len(levels))(*[O.c_desc_bytes(d) for d in levels])
    st = C.c_int(-1)
    h = O.ref().oref_cascade_create(arr, len(levels), C.byref(st))
    assert h, st.value
    O.ref().oref_cascade_update(h, t)
    xz = cascade_points(count)
    out = np.empty((count, 10), np.float32)
    O.ref().oref_cascade_sample_many(h, xz.ctypes.data, count, out.ctypes.data)
    O.ref().oref_cascade_destroy(h)
    np.savez_compressed(HERE / "ref_cascade.npz", xz=xz, out=out)


def interaction() -> None:
    from oracle import iwave as OI
    from tests.workloads import interaction_script, run_interaction

    desc, script, frames, dt = interaction_script()
    r = OI.RefInteraction(desc)
    fields = []
    run_interaction(r, script, frames, dt, lambda f, fld: fields.append(fld.field()))
    rng = np.random.default_rng(9)
    xz = rng.uniform(-4.0, 40.0, size=(2048, 2)).astype(np.float32)
    samples = r.sample_many(xz)
    taps, stats = OI.ref_taps(desc.kernel_radius, float(np.float32(desc.extent) / np.float32(desc.size)),
                              desc.depth)
    np.savez_compressed(HERE / "ref_interaction.npz", fields=np.stack(fields), xz=xz, samples=samples,
                        taps=taps, stats=stats, fixed_dt=np.float32(r.fixed_dt),
                        dt_limit=np.float32(r.dt_limit), dispersion_error=np.float32(r.dispersion_error),
                        energy=np.float64(r.energy()))


def abi_layout() -> None:
    src = r"""
#include <stddef.h>
#include <stdio.h>
#include "ocean/ocean.h"
#define OFF(T, f) printf("\"%s.%s\": %zu,\n", #T, #f, offsetof(T, f))
int main(void) {
  printf("{\n");
  printf("\"sizeof.ocean_desc\": %zu,\n", sizeof(ocean_desc));
  printf("\"sizeof.ocean_spectrum_desc\": %zu,\n", sizeof(ocean_spectrum_desc));
  printf("\"sizeof.ocean_buffers\": %zu,\n", sizeof(ocean_buffers));
  printf("\"sizeof.ocean_surface\": %zu,\n", sizeof(ocean_surface));
  printf("\"sizeof.ocean_surface_ex\": %zu,\n", sizeof(ocean_surface_ex));
  OFF(ocean_desc, struct_size); OFF(ocean_desc, size); OFF(ocean_desc, patch_length);
  OFF(ocean_desc, spectrum); OFF(ocean_desc, choppiness); OFF(ocean_desc, foam_threshold);
  OFF(ocean_desc, seed); OFF(ocean_desc, parallel_for); OFF(ocean_desc, parallel_for_user);
  OFF(ocean_desc, thread_count); OFF(ocean_desc, water_depth); OFF(ocean_desc, compute_velocity);
  OFF(ocean_buffers, displacement); OFF(ocean_buffers, normal); OFF(ocean_buffers, size);
  OFF(ocean_buffers, patch_length);
  printf("\"end\": 0\n}\n");
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as td:
        c = Path(td) / "layout.c"
        c.write_text(src)
        exe = Path(td) / "layout"
        subprocess.run(["gcc", "-I", str(O.REF_SRC / "include"), str(c), "-o", str(exe)], check=True)
        res = subprocess.run([str(exe)], check=True, capture_output=True, text=True)
    layout = json.loads(res.stdout)
    layout.pop("end")
    (HERE / "abi_layout.json").write_text(json.dumps(layout, indent=1))


def pack() -> None:
    """sha256 of the reference viewer's RGBA16F pack (examples/viewer/half.hpp)
    over the bit patterns of workloads.pack_patterns, without and with the
    separate alpha plane."""
    src, alpha = pack_patterns()
    out = {"texels": int(src.shape[0]), "plain": sha(O.ref_pack_rgba16(src)),
           "alpha": sha(O.ref_pack_rgba16(src, alpha))}
    (HERE / "ref_pack.json").write_text(json.dumps(out, indent=1))


def foam_queries() -> None:
    desc, foam, _, dt = FOAM_CASE
    first, second = FOAM_QUERY_FRAMES
    ro = O.RefOcean(desc)
    rf = O.RefFoam(ro, foam)
    for k in range(first):
        ro.update((k + 1) * dt)
        rf.update(dt)
    xz = query_points(desc, 4096)
    out = {"desc": desc_to_json(desc), "dt": dt, "frames": [first, second],
           "at": sha(rf.foam_at_many(xz)), "coverage": rf.coverage(), "field": sha(rf.data())}
    rf.set_desc(FOAM_RETUNE)
    retuned = []
    for k in range(first, first + second):
        ro.update((k + 1) * dt)
        rf.update(dt)
        retuned.append({"field": sha(rf.data()), "substeps": rf.last_substeps})
    out["retuned"] = retuned
    out["coverage_retuned"] = rf.coverage()
    rf.clear()
    out["coverage_cleared"] = rf.coverage()
    ro.update((first + second + 1) * dt)
    rf.update(dt)
    out["after_clear"] = sha(rf.data())
    (HERE / "ref_foam.json").write_text(json.dumps(out, indent=1))


def foam_long() -> None:
    desc, foam, frames, dt = FOAM_LONG_CASE
    ro = O.RefOcean(desc)
    rf = O.RefFoam(ro, foam)
    checks = {}
    for k in range(1, frames + 1):
        ro.update(k * dt)
        rf.update(dt)
        if k in FOAM_LONG_CHECKPOINTS:
            f = rf.data()
            checks[str(k)] = {"sha": sha(f), "coverage": rf.coverage(), "max": float(f.max()),
                              "nonzero": int(np.count_nonzero(f)), "substeps": rf.last_substeps}
    out = {"desc": desc_to_json(desc), "frames": frames, "dt": dt, "checkpoints": checks}
    (HERE / "ref_foam_long.json").write_text(json.dumps(out, indent=1))


PARTS = {"foam_long": foam_long, "small": small, "hashes": hashes, "queries": queries, "cascades": cascades,
         "interaction": interaction, "pack": pack, "abi_layout": abi_layout, "foam_queries": foam_queries}


def main() -> None:
    if not O.ref_available():
        raise SystemExit("the reference library could not be built (reference sources absent)")
    O.ref().oref_c_force_simd_level(None)
    names = sys.argv[1:] or list(PARTS)
    unknown = [n for n in names if n not in PARTS]
    if unknown:
        raise SystemExit(f"unknown fixture(s) {unknown}; choose from {list(PARTS)}")
    for name in names:
        PARTS[name]()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
