"""Builds the native libraries in-tree.

  ae-engine_b200/_build/libae_mpm.so      the CUDA library behind include/ae_mpm.h (sm_100a)
  ae-engine_b200/_build/test_host_mirror  tests/cpp/test_host_mirror.cpp: the reference's unit
                                          tests through the C++ mirror of its API (host/ae_mpm_host.hpp)
  oracle/_build/libae_mpm_oracle.so       the CPU oracle (test infrastructure only)

nvcc cross-compiles for sm_100a without a GPU, so this runs on CPU-only machines too.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
ORACLE = os.path.join(ROOT, "oracle")
ORACLE_BUILD = os.path.join(ORACLE, "_build")

LIB = os.path.join(BUILD, "libae_mpm.so")
HOST_TEST = os.path.join(BUILD, "test_host_mirror")
ORACLE_LIB = os.path.join(ORACLE_BUILD, "libae_mpm_oracle.so")

CU_SOURCES = ["radix_sort.cu", "mpm_world.cu", "ae_mpm_api.cu", "ae_mpm_server.cu", "ae_mpm_noalloc.cu", "ae_mpm_lod.cu",
              "ae_mpm_ck.cu"]
# per-source flags: the CK-MPM kernels round every operation separately, as the reference's f32
# arithmetic does (no fused multiply-add)
SOURCE_FLAGS = {"ae_mpm_ck.cu": ["--fmad=false"],
                # the drop-in's host copies to and from pinned staging run on an OpenMP team
                "ae_mpm_api.cu": ["-Xcompiler", "-fopenmp"]}
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA library cannot be built")


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed (%d): %s\n%s" % (r.returncode, " ".join(cmd), r.stdout))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h", ".hpp"))]
    hs.append(os.path.join(ROOT, "include", "ae_mpm.h"))
    return hs


def build_cuda(force: bool = False) -> str:
    os.makedirs(os.path.join(BUILD, "obj"), exist_ok=True)
    nvcc = _nvcc()
    hdrs = _headers()
    objs, jobs = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, "obj", src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            jobs.append([nvcc] + NVCC_FLAGS + SOURCE_FLAGS.get(src, []) + ["-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(_run, jobs))
    if force or jobs or _stale(LIB, objs):
        _run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "static",
              "-o", LIB] + objs + ["-lgomp", "-lpthread"])
    return LIB


def build_host_test(force: bool = False) -> str:
    src = os.path.join(ROOT, "tests", "cpp", "test_host_mirror.cpp")
    hdrs = [os.path.join(HERE, "host", h) for h in ("ae_mpm_host.hpp", "ae_ck_mpm_host.hpp")]
    deps = [src] + hdrs + [os.path.join(ROOT, "include", "ae_mpm.h"), LIB]
    if force or _stale(HOST_TEST, deps):
        _run(["g++", "-O2", "-std=c++17", "-o", HOST_TEST, src, "-I" + os.path.join(ROOT, "include"),
              "-I" + os.path.join(HERE, "host"), "-L" + BUILD, "-lae_mpm", "-Wl,-rpath,$ORIGIN", "-lpthread"])
    return HOST_TEST


def build_oracle(force: bool = False) -> str:
    os.makedirs(ORACLE_BUILD, exist_ok=True)
    srcs = [os.path.join(ORACLE, f) for f in ("mpm_oracle.cpp", "lod_oracle.cpp", "ck_oracle.cpp")]
    if force or _stale(ORACLE_LIB, srcs + [os.path.join(ROOT, "include", "ae_mpm.h")]):
        # x86-64-v3 so the binary also runs on the GPU hosts' CPUs; no FMA contraction, as in Rust
        _run(["g++", "-O3", "-std=c++17", "-march=x86-64-v3", "-ffp-contract=off", "-fPIC", "-shared", "-o", ORACLE_LIB]
             + srcs + ["-lpthread"])
    return ORACLE_LIB


def build_all(force: bool = False) -> None:
    build_oracle(force)
    build_cuda(force)
    build_host_test(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", LIB, HOST_TEST, ORACLE_LIB)
