"""Build recipe for the native libraries (in-tree, sm_100a).

``build()`` compiles
  * ``lib/libtm_b200.so`` -- the CUDA search core behind the C ABI in
    include/tm_b200.h (nvcc cross-compiles without a GPU);
  * ``lib/libtm_host.so`` -- the C++ host preparation (whitening, template
    spectrum, projection filter, search grid, MRC I/O) with C entry points;
  * ``lib/match_template`` -- the match_template program (C++ host over the
    C ABI, linked against libtm_b200.so with an $ORIGIN rpath);
  * ``lib/match_template_merge`` -- the master side of a distributed run
    (merges worker result arrays; host only);
  * ``lib/refine_template`` -- the refine_template program (C++ host over the
    C ABI's batched TemplateScore).
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_DIR = os.path.join(PKG, "lib")
CSRC = os.path.join(PKG, "csrc")
CORE_LIB = os.path.join(LIB_DIR, "libtm_b200.so")
HOST_DIR = os.path.join(PKG, "host")
HOST_LIB = os.path.join(LIB_DIR, "libtm_host.so")
CLI = os.path.join(LIB_DIR, "match_template")
MERGE_CLI = os.path.join(LIB_DIR, "match_template_merge")
REFINE_CLI = os.path.join(LIB_DIR, "refine_template")
HOST_COMMON = ["host_fft.cpp", "mrc.cpp", "prep.cpp", "peaks.cpp", "montage.cpp", "result_array.cpp", "refine.cpp"]
CXX_FLAGS = ["-std=c++17", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-Wall", "-Wno-unused-parameter",
             "-I" + os.path.join(ROOT, "include"), "-I" + HOST_DIR]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--extended-lambda",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-shared",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))] + [os.path.join(ROOT, "include", "tm_b200.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_core(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    if force or _stale(CORE_LIB, _sources()):
        cmd = [_nvcc(), *NVCC_FLAGS, "-o", CORE_LIB, os.path.join(CSRC, "tm_capi.cu"), os.path.join(CSRC, "tm_noalloc.cu"),
               os.path.join(CSRC, "tm_refine.cu"), os.path.join(CSRC, "tm_proposal.cu")]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return CORE_LIB


def _cxx():
    # the system g++ carries libgomp; some images put a compiler without it first on PATH
    for cand in (os.environ.get("TM_CXX"), "/usr/bin/g++", os.environ.get("CXX"), "g++"):
        if cand and (not os.path.isabs(cand) or os.path.exists(cand)):
            return cand
    return "g++"


def _host_deps():
    return [os.path.join(HOST_DIR, f) for f in sorted(os.listdir(HOST_DIR))] + [os.path.join(ROOT, "include", "tm_b200.h")]


def build_host(force: bool = False, verbose: bool = False) -> None:
    os.makedirs(LIB_DIR, exist_ok=True)
    common = [os.path.join(HOST_DIR, f) for f in HOST_COMMON]
    if force or _stale(HOST_LIB, _host_deps()):
        cmd = [_cxx(), *CXX_FLAGS, "-shared", "-fvisibility=hidden", "-o", HOST_LIB,
               *common, os.path.join(HOST_DIR, "host_capi.cpp")]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    if force or _stale(CLI, _host_deps() + [CORE_LIB]):
        cmd = [_cxx(), *CXX_FLAGS, "-o", CLI, *common,
               os.path.join(HOST_DIR, "template_matching_core.cpp"), os.path.join(HOST_DIR, "match_template_main.cpp"),
               "-L" + LIB_DIR, "-ltm_b200", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    if force or _stale(REFINE_CLI, _host_deps() + [CORE_LIB]):
        cmd = [_cxx(), *CXX_FLAGS, "-pthread", "-o", REFINE_CLI, *common, os.path.join(HOST_DIR, "refine_template_main.cpp"),
               "-L" + LIB_DIR, "-ltm_b200", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    if force or _stale(MERGE_CLI, _host_deps()):
        cmd = [_cxx(), *CXX_FLAGS, "-o", MERGE_CLI, *common, os.path.join(HOST_DIR, "match_template_merge.cpp")]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False) -> None:
    build_core(force=force, verbose=verbose)
    build_host(force=force, verbose=verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
