"""Builds the native API checks in this folder against include/ and
libocean_b200.so (test infrastructure):

    ocean_api_check   C++20 program over include/ocean/*.hpp
    c_header_check    C99 program over include/ocean/ocean.h (-pedantic -Werror)

Outputs go to _build/native/ (git-ignored). Returns the executables' paths.
"""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = ROOT / "_build" / "native"
LIBDIR = ROOT / "oceanlib_b200"


def build() -> dict:
    OUT.mkdir(parents=True, exist_ok=True)
    link = [f"-L{LIBDIR}", "-locean_b200", f"-Wl,-rpath,{LIBDIR}"]
    cxx = shutil.which("g++") or "g++"
    cc = shutil.which("gcc") or "gcc"
    jobs = {
        "ocean_api_check": [cxx, "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}",
                            str(HERE / "ocean_api_check.cpp"), *link, "-o", str(OUT / "ocean_api_check")],
        "c_header_check": [cc, "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}",
                           str(HERE / "c_header_check.c"), *link, "-o", str(OUT / "c_header_check")],
    }
    out = {}
    for name, cmd in jobs.items():
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"{name} failed to build:\n{res.stdout}\n{res.stderr}")
        out[name] = OUT / name
    return out
