"""Builds the native library libftlm_gpu.so in-tree (sm_100a) with nvcc/g++.

    python -m ftlm_extended_hubbard_b200.build [--force]

Sources live in ftlm_extended_hubbard_b200/csrc; objects go to ftlm_extended_hubbard_b200/_build
(git-ignored).  Rebuilds only what changed (mtime of the sources and headers).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libftlm_gpu.so")
DROPIN_LIB = os.path.join(HERE, "libftlm_dropin.so")
DROPIN_SRC = os.path.join(HERE, "cpp", "dropin.cpp")
DROPIN_INC = os.path.join(HERE, "cpp", "include")
PYMOD_SRC = os.path.join(HERE, "python", "bindings.cpp")
PYMOD_DIR = os.path.join(HERE, "python", "ftlm")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC"]
CU_SOURCES = ["hv.cu", "lanczos.cu", "quad.cu", "capi.cu", "capi_batched.cu", "capi_grad.cu", "capi_orbit.cu", "noalloc.cu", "batched.cu", "orbit.cu", "grad.cu", "chains.cu", "symeig.cu"]
CXX_SOURCES = ["plan.cpp", "tridiag.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    return os.environ.get("CXX") or shutil.which("g++") or "g++"


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    hs.append(os.path.join(ROOT, "include", "ftlm_gpu.h"))
    return hs


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc, cxx = _nvcc(), _cxx()
    hdrs = _headers()
    jobs, objs = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            jobs.append([nvcc, *NVCC_FLAGS, "-I", CSRC, "-I", os.path.join(ROOT, "include"), "-c", s, "-o", o])
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            jobs.append([cxx, *CXX_FLAGS, "-I", CSRC, "-c", s, "-o", o])
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            list(ex.map(_run, jobs))
    if force or jobs or _stale(LIB, objs):
        _run([nvcc, "-shared", *ARCH, "-o", LIB, *objs, "-lcudart"])
    # C++ drop-in of the reference API (namespace ftlm), host code over the C ABI
    dhdrs = [os.path.join(DROPIN_INC, "ftlm", f) for f in os.listdir(os.path.join(DROPIN_INC, "ftlm"))]
    if force or _stale(DROPIN_LIB, [DROPIN_SRC, LIB, os.path.join(ROOT, "include", "ftlm_gpu.h")] + dhdrs):
        _run([cxx, *CXX_FLAGS, "-shared", "-I", DROPIN_INC, "-I", os.path.join(ROOT, "include"), DROPIN_SRC, "-o",
              DROPIN_LIB, "-L", HERE, "-lftlm_gpu", "-Wl,-rpath,$ORIGIN"])
    build_pymodule(force)
    if verbose:
        print(LIB)
    return LIB


def pymodule_path() -> str:
    import sysconfig
    return os.path.join(PYMOD_DIR, "_ftlm_core" + sysconfig.get_config_var("EXT_SUFFIX"))


def build_pymodule(force: bool = False) -> str:
    """The reference's pybind11 module _ftlm_core (python/ftlm/), compiled against torch's headers
    (torch's own pybind11, its C++ ABI flag) and linked to libftlm_gpu.so + libftlm_dropin.so."""
    import sysconfig

    import torch
    from torch.utils import cpp_extension as ce
    out = pymodule_path()
    deps = [PYMOD_SRC, LIB, DROPIN_LIB, os.path.join(ROOT, "include", "ftlm_gpu.h")]
    if not force and not _stale(out, deps):
        return out
    incs = ce.include_paths() + [os.path.join(_cuda_home(), "include"), sysconfig.get_paths()["include"], DROPIN_INC,
                                 os.path.join(ROOT, "include")]
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cmd = [_cxx(), "-O2", "-std=c++17", "-fPIC", "-shared", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           "-DTORCH_EXTENSION_NAME=_ftlm_core", "-DTORCH_API_INCLUDE_EXTENSION_H", "-fvisibility=hidden"]
    for i in incs:
        cmd += ["-isystem" if "torch" in i or "python" in i else "-I", i]
    cmd += [PYMOD_SRC, "-o", out]
    for lp in ce.library_paths():
        cmd += ["-L", lp, f"-Wl,-rpath,{lp}"]
    cmd += ["-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_python", "-L", HERE, "-lftlm_dropin",
            "-lftlm_gpu", "-Wl,-rpath,$ORIGIN/../.."]
    _run(cmd)
    return out


def _cuda_home() -> str:
    return os.path.dirname(os.path.dirname(_nvcc()))


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
