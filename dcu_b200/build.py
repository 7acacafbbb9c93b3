"""Build recipe of libdcu_spai.so (CUDA sm_100a + host C++) and the
spai_multi_dcu and spai_single_dcu command-line drivers, in-tree under
dcu_b200/lib/.

nvcc compiles every kernel file for sm_100a only
(-gencode arch=compute_100a,code=sm_100a); the host C++ (drop-in API,
MatrixMarket reader, CLI) is compiled by the system g++.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(ROOT, "_build", "obj")
INCLUDE = os.path.join(ROOT, "include")
LIBNAME = os.path.join(LIBDIR, "libdcu_spai.so")
CLINAME = os.path.join(LIBDIR, "spai_multi_dcu")
CLI_SINGLE = os.path.join(LIBDIR, "spai_single_dcu")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["runtime.cu", "sparse_format.cu", "spai_build.cu", "bicgstab.cu", "batched.cu", "capi.cu"]
CXX_SOURCES = ["host_api.cpp", "mtx_io.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    for dp, _, fs in os.walk(INCLUDE):
        hs += [os.path.join(dp, f) for f in fs if f.endswith(".h")]
    return hs


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile (incrementally) and return the path of libdcu_spai.so."""
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    hdrs = _headers()
    jobs = []
    objs = []
    for f in CU_SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJDIR, f + ".o")
        objs.append(obj)
        if force or ptxas_info or _stale(obj, [src] + hdrs):
            cmd = [NVCC, "-ccbin", HOST_CXX, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    for f in CXX_SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJDIR, f + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            jobs.append([HOST_CXX, "-O2", "-std=c++17", "-fPIC", "-Wall", "-I", INCLUDE,
                         "-I", os.path.join(CUDA_HOME, "include"), "-c", src, "-o", obj])
    outs = []
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        for out in ex.map(_run, jobs):
            outs.append(out)
    if verbose or ptxas_info:
        print("\n".join(o for o in outs if o))
    if force or jobs or _stale(LIBNAME, objs):
        _run([NVCC, "-ccbin", HOST_CXX, *ARCH, "-shared", "-o", LIBNAME, *objs, "-Xlinker", "-z,defs",
              "-lpthread"])
    for src_name, exe in (("cli.cpp", CLINAME), ("cli_single.cpp", CLI_SINGLE)):
        cli_src = os.path.join(CSRC, src_name)
        if force or _stale(exe, [cli_src, LIBNAME] + hdrs):
            _run([HOST_CXX, "-O2", "-std=c++17", "-Wall", "-I", INCLUDE, "-I", os.path.join(CUDA_HOME, "include"),
                  cli_src, "-o", exe, "-L", LIBDIR, "-ldcu_spai", "-Wl,-rpath,$ORIGIN",
                  "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart"])
    return LIBNAME


def clean() -> None:
    shutil.rmtree(os.path.join(ROOT, "_build"), ignore_errors=True)
    shutil.rmtree(LIBDIR, ignore_errors=True)


if __name__ == "__main__":
    import sys

    print(build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv))
