"""In-tree build of libhtfeti_b200.so (CUDA for sm_100a + C++ host code).

    python hfls_b200/build.py          # incremental (runs without importing the package)
    python hfls_b200/build.py --clean

CUDA sources are compiled by nvcc with -gencode arch=compute_100a,code=sm_100a;
host sources by g++ without FMA contraction, so host-side sums match the
oracle bit for bit.  Objects go to hfls_b200/_build/, the library to
hfls_b200/libhtfeti_b200.so.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libhtfeti_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

CU_SOURCES = ["device/setup_kernels.cu", "device/pcpg_kernels.cu", "device/engine.cu", "device/noalloc.cu",
              "device/tc_gemm.cu", "device/pcpg_multi.cu", "device/engine_batch.cu", "device/coarse.cu",
              "device/autotune.cu", "device/kernel_fix.cu", "device/frontend.cu"]
CPP_SOURCES = ["host/mesh.cpp", "host/problem.cpp", "host/vtk.cpp", "host/dump.cpp", "capi.cpp", "server.cpp",
               "cxx/surface.cpp"]
HEADERS = ["device/device.cuh", "device/engine.hpp", "host/problem.hpp"]

INC = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC,-fopenmp,-O2", "--expt-relaxed-constexpr"] + INC
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-I" + os.path.join(CUDA, "include")] + INC


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "htfeti.h")]
    deps += [os.path.join(ROOT, "include", "hfls", h) for h in os.listdir(os.path.join(ROOT, "include", "hfls"))]
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    jobs = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s.replace("/", "_") + ".o")
        objs.append(obj)
        if _stale(obj, src):
            flags = NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_info else [])
            jobs.append([NVCC] + flags + ["-c", "-o", obj, src])
    cxx = shutil.which("g++") or "g++"
    for s in CPP_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s.replace("/", "_") + ".o")
        objs.append(obj)
        if _stale(obj, src):
            jobs.append([cxx] + CXX_FLAGS + ["-c", "-o", obj, src])
    procs = [(j, subprocess.Popen(j, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)) for j in jobs]
    failed = False
    for j, p in procs:
        out, errs = p.communicate()
        if verbose or p.returncode != 0 or (ptxas_info and "nvcc" in j[0]):
            sys.stderr.write(out + errs)
        if p.returncode != 0:
            failed = True
            sys.stderr.write("FAILED: " + " ".join(j) + "\n")
    if failed:
        raise RuntimeError("compilation failed")
    if jobs or not os.path.exists(LIB):
        _run([cxx, "-shared", "-o", LIB] + objs +
             ["-L" + os.path.join(CUDA, "lib64"), "-lcudart", "-lgomp",
              "-Wl,-rpath," + os.path.join(CUDA, "lib64")])
    return LIB


if __name__ == "__main__":
    if "--clean" in sys.argv:
        shutil.rmtree(BUILD, ignore_errors=True)
        if os.path.exists(LIB):
            os.remove(LIB)
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
