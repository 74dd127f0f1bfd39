"""Build recipe of the B200 phase-field library (sm_100a) and its C++ front end.

Outputs (in-tree, git-ignored, shipped with the working copy):
  general-simulator_b200/libgsb200.so   CUDA kernels + C ABI (include/gs_capi.h)
  general-simulator_b200/libgsb200_bc.so  the same with the kernels' index asserts (-DGS_BOUNDS_CHECK)
  general-simulator_b200/gsi            script interpreter (the reference's front end)
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-Xptxas", "-warn-spills"]
CU_SOURCES = ["gs_capi.cu", "gs_k_zy.cu", "gs_k_zy_f32.cu", "gs_k_zy_f64.cu", "gs_k_x.cu", "gs_k_x33.cu",
              "gs_k_x55.cu", "gs_k_x86.cu", "gs_k_x99.cu", "gs_k_xt.cu", "gs_k_xp10.cu", "gs_k_xp2.cu", "gs_k_xp18.cu",
              "gs_k_precip.cu", "gs_k_mart.cu", "gs_k_mart_f32.cu", "gs_k_mart_f64.cu",
              "gs_k_adj_f32.cu", "gs_k_adj_f64.cu", "gs_plain.cu", "gs_cores.cu", "gs_k_padj.cu", "gs_k_xtma.cu", "gs_noise.cu", "gs_cufft.cu", "gs_bounds.cu"]
LIB = os.path.join(HERE, "libgsb200.so")
LIB_BC = os.path.join(HERE, "libgsb200_bc.so")


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return hs + [os.path.join(ROOT, "include", "gs_capi.h")]


def build_lib(jobs: int = 8, verbose: bool = False, bounds_check: bool = False) -> str:
    """libgsb200.so, or with bounds_check the bounds-check build libgsb200_bc.so
    (index asserts in every pass kernel, GS_EBOUNDS from the step entries)."""
    bdir = BUILD + ("_bc" if bounds_check else "")
    lib = LIB_BC if bounds_check else LIB
    extra = ["-DGS_BOUNDS_CHECK"] if bounds_check else []
    os.makedirs(bdir, exist_ok=True)
    hdrs = _headers()
    objs = []
    todo = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(bdir, src.replace(".cu", ".o"))
        objs.append(o)
        if _stale(o, [s] + hdrs):
            todo.append([NVCC, *ARCH, *NVFLAGS, *extra, "-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for f in [ex.submit(_run, c) for c in todo]:
            f.result()
    if todo or _stale(lib, objs):
        _run([NVCC, *ARCH, "-shared", "-o", lib, *objs, "-lcufft", "-Xlinker",
              "-rpath=/usr/local/cuda/lib64"])
    return lib


HOST_SOURCES = ["gs_script.cpp", "gs_driver.cpp", "gs_plugins.cpp", "gs_main.cpp"]
GSI = os.path.join(HERE, "gsi")


def build_frontend() -> str:
    """The script interpreter (C++17), linked against libgsb200.so."""
    srcs = [os.path.join(HOST, f) for f in HOST_SOURCES]
    deps = srcs + [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".h")] + [LIB]
    if _stale(GSI, deps):
        _run(["g++", "-O2", "-std=c++17", "-Wall", "-pthread", "-o", GSI, *srcs, "-L" + HERE, "-lgsb200",
              "-Wl,-rpath,$ORIGIN"])
    return GSI


def build_oracle() -> str:
    _run(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    return os.path.join(ROOT, "oracle", "liboracle.so")


def build_reference() -> str | None:
    """The reference's own gsi in oracle/_ref/ (test infrastructure: it
    generated the committed fixtures under tests/golden/).  Built only where
    the reference tree is present and the binary is missing; a failure is
    reported, not raised, since nothing at run time needs it."""
    out = os.path.join(ROOT, "oracle", "_ref", "gsi")
    if os.path.exists(out):
        return out
    ref = os.environ.get("REF", "/root/reference")  # where the reference tree sits in the build container
    if not os.path.isdir(os.path.join(ref, "src")):
        return None
    r = subprocess.run(["bash", os.path.join(ROOT, "oracle", "build_ref.sh")], capture_output=True, text=True,
                       env={**os.environ, "REF": ref})
    if r.returncode != 0:
        print("reference build skipped:", (r.stdout + r.stderr).strip().splitlines()[-1:], file=sys.stderr)
        return None
    return out


def build_all(jobs: int = 8) -> None:
    build_lib(jobs)
    build_lib(jobs, bounds_check=True)
    build_frontend()
    build_oracle()
    build_reference()


if __name__ == "__main__":
    build_all()
    print("built", LIB)
