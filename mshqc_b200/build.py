"""Build recipe for libmshqc_cuda.so (sm_100a) and the pybind11 module.

    python -m mshqc_b200.build            # builds into mshqc_b200/lib/

The shared library is built in-tree so that it travels with the repository
snapshot; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libmshqc_cuda.so")

CUDA_SOURCES = ["cd_abi.cu", "cd_mp2.cu", "cd_omp2.cu", "cd_vectors.cu", "cd_decompose.cu", "cd_noalloc.cu",
                "cd_t2.cu"]
# host-only C++ (the AO integral engine), compiled by g++ with OpenMP
HOST_SOURCES = ["ao_integrals.cc"]
HOST_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-fopenmp", "-march=x86-64-v3"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-Xptxas", "-warn-spills",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_compiler_flags():
    # nvcc drives the system g++; make sure it links the shared libstdc++ (a
    # static copy inside a library that Python loads next to the system one
    # breaks iostreams)
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
    return ["-ccbin", gxx]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_cuda(verbose: bool = False, force: bool = False, extra_flags=()) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "mshqc_cd.h"))
    deps.append(os.path.join(ROOT, "include", "mshqc_ao.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in CUDA_SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        _run([nvcc(), *_host_compiler_flags(), *NVCC_FLAGS, *extra_flags, "-c",
              os.path.join(CSRC, src), "-o", obj], verbose)
        objs.append(obj)
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
    for src in HOST_SOURCES:
        obj = os.path.join(objdir, src.replace(".cc", ".o"))
        _run([gxx, *HOST_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj], verbose)
        objs.append(obj)
    tmp = LIB + ".tmp"
    _run([nvcc(), *_host_compiler_flags(), "-gencode", "arch=compute_100a,code=sm_100a",
          "-shared", "-Xcompiler", "-fPIC", "-o", tmp, *objs, "-cudart", "static", "-lgomp"], verbose)
    os.replace(tmp, LIB)
    return LIB


CPP_DIR = os.path.join(HERE, "cpp")
CPP_SOURCES = ["mshqc_b200.cc", "bindings.cc"]


def module_path() -> str:
    return os.path.join(HERE, "_mshqc" + sysconfig.get_config_var("EXT_SUFFIX"))


def build_module(verbose: bool = False, force: bool = False) -> str:
    """The pybind11 module mshqc_b200._mshqc (the C++ mirror classes), linked
    against libmshqc_cuda.so next to it (rpath $ORIGIN/lib)."""
    import pybind11
    target = module_path()
    deps = [os.path.join(CPP_DIR, f) for f in os.listdir(CPP_DIR)] + [LIB,
                                                                      os.path.join(ROOT, "include", "mshqc_cd.h")]
    if not force and not _stale(target, deps):
        return target
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
    cmd = [gxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
           "-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"],
           *[os.path.join(CPP_DIR, f) for f in CPP_SOURCES],
           "-L", LIBDIR, "-lmshqc_cuda", "-Wl,-rpath,$ORIGIN/lib", "-o", target + ".tmp"]
    _run(cmd, verbose)
    os.replace(target + ".tmp", target)
    return target


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    force = "--force" in argv
    lib = build_cuda(verbose=True, force=force)
    print("built", lib)
    mod = build_module(verbose=True, force=force)
    print("built", mod)


if __name__ == "__main__":
    main()
