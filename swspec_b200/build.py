"""Build the in-tree native libraries.

  swspec_b200/libswsgpu.so   : CUDA kernels + C ABI (include/swsgpu.h), sm_100a
  swspec_b200/libswshost.so  : C++ host (TaskCoreCUDA, dispatcher, INI, sinks)
  swspec_b200/swspectrometer_gpu : command-line front end over libswshost

nvcc cross-compiles for sm_100a without a GPU, so this runs anywhere the
CUDA toolkit is installed.  Objects go to swspec_b200/_build/.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
BUILD = os.path.join(PKG, "_build")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CUDA_HOME = os.path.dirname(os.path.dirname(os.path.realpath(NVCC)))

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
           "-diag-suppress", "20281"] + ARCH

CU_SOURCES = ["engine.cu", "unpack.cu", "pcal.cu", "plans.cu", "bigfft.cu", "noalloc.cu", "pcallib.cu"]
HOST_SOURCES = ["settings.cpp", "iniparser.cpp", "buffer.cpp", "filesource.cpp", "filesink.cpp",
                "taskcore_cuda.cpp", "dispatcher.cpp"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _headers(d: str) -> list[str]:
    return [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".cuh", ".h", ".hpp"))]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")


def build_cuda(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(PKG, "libswsgpu.so")
    hdrs = _headers(CSRC) + [os.path.join(ROOT, "include", "swsgpu.h")]
    srcs = [s for s in CU_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    jobs = []
    objs = []
    for s in srcs:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s.replace(".cu", ".o"))
        objs.append(obj)
        if _newer(obj, [src] + hdrs):
            jobs.append([NVCC] + NVFLAGS + ["-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        list(ex.map(_run, jobs))
    if jobs or _newer(out, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", out] + objs + ["-lcudart"])
    return out


def build_probe() -> str:
    """The benchmark's FP32 FMA peak probe (fp32_probe.cu beside bench.py;
    not part of the library or its C ABI)."""
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(ROOT, "libfp32probe.so")
    src = os.path.join(ROOT, "fp32_probe.cu")
    if os.path.exists(src) and _newer(out, [src]):
        _run([NVCC] + NVFLAGS + ["-shared", "-o", out, src])
    return out


def build_host() -> str:
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(PKG, "libswshost.so")
    exe = os.path.join(PKG, "swspectrometer_gpu")
    if not os.path.isdir(HOST):
        return out
    hdrs = _headers(HOST) + [os.path.join(ROOT, "include", "swsgpu.h")]
    srcs = [os.path.join(HOST, s) for s in HOST_SOURCES if os.path.exists(os.path.join(HOST, s))]
    cxx = shutil.which("g++") or "g++"
    flags = ["-std=c++17", "-O2", "-fPIC", "-Wall", "-I", os.path.join(ROOT, "include")]
    if _newer(out, srcs + hdrs):
        _run([cxx] + flags + ["-shared", "-o", out] + srcs +
             ["-L", PKG, "-lswsgpu", "-Wl,-rpath,$ORIGIN", "-lpthread"])
    main = os.path.join(HOST, "main.cpp")
    if os.path.exists(main) and _newer(exe, [main, out] + hdrs):
        _run([cxx] + flags + ["-o", exe, main, "-L", PKG, "-lswshost", "-lswsgpu",
                              "-Wl,-rpath,$ORIGIN", "-lpthread"])
    return out


def build_refcore() -> None:
    """The reference's own spectrometer program with TaskCoreCUDA as its core
    (swspec_b200/refcore/Makefile); built only where the reference sources
    are present, the result travels with the repository snapshot."""
    subprocess.run(["make", "-s", "-C", os.path.join(PKG, "refcore")], check=True)


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


def build_all() -> None:
    build_cuda()
    build_probe()
    build_host()
    build_refcore()
    build_oracle()


if __name__ == "__main__":
    build_all()
    print("built", os.path.join(PKG, "libswsgpu.so"))
