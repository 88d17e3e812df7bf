"""Build the CUDA engine (sm_100a) into hawassi_c_b200/lib/libhawassi_b200.so.

    python -m hawassi_c_b200.build [--force] [--ptxas]

Each slice-size instantiation of the kernels is its own translation unit, so
the objects compile in parallel; the host set-up is plain C++.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(LIBDIR, "libhawassi_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["hw_engine.cu", "hw_setup.cpp", "hw_inst_256.cu", "hw_inst_512.cu", "hw_inst_1024.cu",
           "hw_inst_2048.cu", "hw_noalloc.cu", "hw_mlp.cu", "hw2d_engine.cu", "hw_kin.cu", "hw_influx.cu", "hw_peak.cu",
           "hw2d_influx.cu"]
HEADERS = ["hw_fft.cuh", "hw_device.cuh", "hw_rhs.cuh", "hw_stepper.cuh", "hw_breaking.cuh",
           "hw_kernels.cuh", "hw_kernels.h", "hw_setup.hpp", "hw_rhs_fast.cuh", "hw2d.cuh", "hw2d_var.cuh", "hw2d_brk.cuh", "hw2d_wall.cuh", "hw2d_out.cuh", "hw2d_hs3.cuh", "hw_output.cuh", "hw_kin.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC"]


def _deps():
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "hawassi_b200.h"))
    deps.append(os.path.abspath(__file__))
    return deps


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in _deps() if os.path.exists(p))


def _compile(src, extra, verbose):
    obj = os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")
    cmd = [NVCC, *NVCC_FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stdout + r.stderr


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, extra, verbose), SOURCES))
    if verbose:
        for _, log in results:
            if log.strip():
                print(log)
    objs = [o for o, _ in results]
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB + ".tmp", *objs]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
