"""Build the in-tree C-ABI library fesom-c_b200/libfesomc_gpu.so for sm_100a.

Host C++ (mesh builder, orchestration helpers) is compiled with g++, CUDA
sources with nvcc for compute_100a/sm_100a.  FMA contraction is off in both so
the FP64 path follows the reference's operation order (bit-for-bit parity
with the CPU oracle, which is built the same way).

The FP32-form objects (the second compilation of the kernel sources, which
holds only fesomc::f32 kernels) are held to an error budget against the FP64
path instead of to bit parity, so they are compiled for speed: FMA
contraction, FP32 division and square root to within 2 ulp instead of
correctly rounded, FP32 subnormals flushed to zero.  These flags act on
every operation of those objects, the FP64 elevation family of the form
included (contraction only: FP64 division and square root stay correctly
rounded whatever the flags).  The results are still deterministic, and two
runs of the form that differ only in launch shapes, storage order, packing
or decomposition give the same bits.
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

from .abi import LIB_PATH, REPO_DIR, ROOT_DIR

CSRC = os.path.join(ROOT_DIR, "csrc")
INC = os.path.join(REPO_DIR, "include")
OBJ_DIR = os.path.join(ROOT_DIR, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
DUAL_PRECISION = ("k_baroclinic.cu", "k_barotropic.cu", "k_tracer.cu", "k_mixing.cu", "k_closure.cu")
FP64_FLAGS = ["--fmad=false"]
FP32_FORM_FLAGS = ["--fmad=true", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"]


def _nvcc():
    for c in (os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"), shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    return (glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True)
            + glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
            + glob.glob(os.path.join(CSRC, "**", "*.inc"), recursive=True)
            + glob.glob(os.path.join(INC, "*.h")))


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build_library(verbose=False, ptxas_v=False):
    os.makedirs(OBJ_DIR, exist_ok=True)
    # this file holds the compile flags: a change to them rebuilds every object
    hdrs = _headers() + [os.path.abspath(__file__)]
    jobs, objs = [], []
    for src in sorted(glob.glob(os.path.join(CSRC, "**", "*.cpp"), recursive=True)):
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs):
            jobs.append([_cxx(), "-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-fno-fast-math",
                         "-Wall", "-I", INC, "-I", CSRC, "-c", src, "-o", obj])
    nvcc = _nvcc()
    for src in sorted(glob.glob(os.path.join(CSRC, "**", "*.cu"), recursive=True)):
        # kernel sources with level fields are compiled once per arithmetic
        # precision (fesomc::f64 and fesomc::f32)
        variants = [("", "0")]
        if os.path.basename(src) in DUAL_PRECISION:
            variants.append((".f32", "1"))
        for suffix, fp32 in variants:
            obj = os.path.join(OBJ_DIR, os.path.basename(src) + suffix + ".o")
            objs.append(obj)
            if _stale(obj, [src] + hdrs) or ptxas_v:
                cmd = [nvcc] + ARCH + ["-lineinfo", "-O3"] + (FP32_FORM_FLAGS if fp32 == "1" else FP64_FLAGS) + [
                    "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", _cxx(), "-DFESOMC_FP32=" + fp32, "-I", INC,
                    "-I", CSRC, "-c", src, "-o", obj]
                if ptxas_v:
                    cmd += ["-Xptxas", "-v"]
                jobs.append(cmd)
    logs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            logs = list(ex.map(_compile, jobs))
    if jobs or not os.path.exists(LIB_PATH):
        # static CUDA runtime: the library does not depend on the runtime
        # that other packages in the process (e.g. torch) bring along
        link = [nvcc] + ARCH + ["-shared", "--cudart", "static", "-ccbin", _cxx(), "-o", LIB_PATH] + objs
        _compile(link)
    if verbose:
        for log in logs:
            if log.strip():
                print(log)
    return LIB_PATH


def build_oracle():
    oracle_dir = os.path.join(REPO_DIR, "oracle")
    r = subprocess.run(["make", "-C", oracle_dir], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return os.path.join(oracle_dir, "_build", "liboracle.so")


if __name__ == "__main__":
    print(build_library(verbose=True, ptxas_v="-v" in sys.argv))
