"""Build recipe for the B200 shared library and the command-line drop-ins.

    python ice_crystal_phase_b200/build.py      (or __graft_entry__.build())

Produces, in-tree (git-ignored, shipped with the repository snapshot):
    ice_crystal_phase_b200/libicp_b200.so        C ABI of include/icp_b200.h (sm_100a)
    ice_crystal_phase_b200/bin/ice_generate_phase   hex drop-in CLI (C++ host over the C ABI)
    ice_crystal_phase_b200/bin/rainbow_generate     drop drop-in CLI
    ice_crystal_phase_b200/bin/ice_precompute_atlas deterministic atlas precompute drop-in CLI

Every CUDA translation unit is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a).  The FP32 trace unit keeps FMA contraction;
the FP64 trace, CDF and ABI units are built with -fmad=false so their binary64 arithmetic
rounds operation by operation.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
APPS = PKG / "apps"
OUT = PKG / "_build"
LIB = PKG / "libicp_b200.so"
BIN = PKG / "bin"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "--Werror", "cross-execution-space-call", *ARCH, "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-I", str(ROOT / "include"), "-I", str(CSRC), "-I", str(HOST)]

UNITS = {
    "icp_hex_f32.cu": ["-fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "icp_hex_f64.cu": ["-fmad=false"],
    "icp_drop_f32.cu": ["-fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "icp_drop_f64.cu": ["-fmad=false"],
    "icp_cdf.cu": ["-fmad=false"],
    "icp_capi.cu": ["-fmad=false"],
    "icp_capi_drop.cu": ["-fmad=false"],
    "icp_drop_device.cu": ["-fmad=false"],
    "icp_capi_batch.cu": ["-fmad=false"],
    "icp_mlp_gemm.cu": [],
    "icp_mlp.cu": [],
    "icp_capi_mlp.cu": ["-fmad=false"],
    "icp_cdf_static.cu": ["-fmad=false"],
    "icp_atlas.cu": ["-fmad=false"],
    "icp_rainbow.cu": ["-fmad=false"],
    "icp_optics.cu": ["-fmad=false"],
    "icp_patches.cu": ["-fmad=false"],
    "icp_query.cu": ["-fmad=false"],
    "icp_lattice.cu": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"],
}

HOST_SOURCES = ["icp_record_io.cpp"]
APP_SOURCES = {"ice_generate_phase": "ice_generate_phase.cpp", "rainbow_generate": "rainbow_generate.cpp",
               "ice_precompute_atlas": "ice_precompute_atlas.cpp"}


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def _headers() -> list[Path]:
    return [*CSRC.glob("*.cuh"), *CSRC.glob("*.h"), *HOST.glob("*.hpp"), ROOT / "include" / "icp_b200.h"]


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ... {cmd[-1]}")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build_library(verbose: bool = False, ptxas_info: bool = False) -> Path:
    OUT.mkdir(exist_ok=True)
    hdrs = _headers()
    objs = []
    for unit, flags in UNITS.items():
        src = CSRC / unit
        if not src.exists():
            continue
        obj = OUT / (unit + ".o")
        if _newer(obj, [src, *hdrs]) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            _run([NVCC, *COMMON, *flags, *extra, "-c", str(src), "-o", str(obj)], verbose or ptxas_info)
        objs.append(obj)
    if _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcuda"], verbose)
    return LIB


def build_apps(verbose: bool = False) -> list[Path]:
    BIN.mkdir(exist_ok=True)
    built = []
    for name, src in APP_SOURCES.items():
        s = APPS / src
        if not s.exists():
            continue
        exe = BIN / name
        host = [HOST / h for h in HOST_SOURCES if (HOST / h).exists()]
        if _newer(exe, [s, LIB, *host, *_headers()]):
            _run(["g++", "-std=c++20", "-O2", "-ffp-contract=off", "-fno-fast-math", "-I", str(ROOT / "include"),
                  "-I", str(HOST), str(s), *map(str, host), "-L", str(PKG), "-licp_b200", "-Wl,-rpath,$ORIGIN/..",
                  "-o", str(exe)], verbose)
        built.append(exe)
    return built


def build(verbose: bool = False) -> Path:
    lib = build_library(verbose)
    build_apps(verbose)
    return lib


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    if "--ptxas" in sys.argv:
        build_library(ptxas_info=True)
    print(LIB)
