"""Build the in-tree shared libraries.

* ``fdd3260_b200/libmimica_gpu.so`` -- the sm_100a CUDA library behind
  ``include/mimica_gpu.h`` (nvcc, -gencode arch=compute_100a,code=sm_100a).
  The FP64 kernels are compiled with ``-fmad=false`` so that their arithmetic is
  the reference's operation for operation (no contraction into FMA).
* ``oracle/libmimica_oracle.so`` -- the CPU restatement used as the checker by
  the tests (gcc, -O2 -fno-fast-math -ffp-contract=off), plus an OpenMP build
  ``oracle/libmimica_oracle_omp.so`` used as the timed CPU baseline.
* ``oracle/_ref/libkissref.so`` -- only when MIMICA_REFERENCE_TREE names a
  reference tree: the reference's own KISS FFT header compiled from where it
  lies (see ``oracle/build_ref.sh``).

Run ``python -m fdd3260_b200.build`` (or ``python fdd3260_b200/build.py``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libmimica_gpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# (source, extra flags)
SOURCES = [
    ("k_scalar.cu", ["-fmad=false"]),
    ("k_scalar_mixed.cu", ["-use_fast_math"]),
    ("k_momentum.cu", ["-fmad=false"]),
    ("k_momentum_mixed.cu", []),
    ("k_pressure.cu", ["-fmad=false"]),
    ("capi.cu", []),
    ("noalloc.cu", ["-fmad=false"]),
    ("k_adjoint.cu", ["-fmad=false"]),
    ("k_sgs.cu", ["-fmad=false", "-Xcompiler", "-ffp-contract=off"]),
    ("k_check.cu", ["-fmad=false"]),
    ("k_momadj.cu", ["-fmad=false"]),
    ("k_traj.cu", ["-fmad=false"]),
    ("k_acoustic.cu", ["-fmad=false"]),
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"command failed: {' '.join(cmd)}")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_cuda(verbose: bool = False, ptxas_verbose: bool = False) -> str:
    nvcc = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(INCLUDE, "mimica_gpu.h"))
    objs = []
    for src, extra in SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(obj)
        if _stale(obj, [path] + headers) or ptxas_verbose:
            cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-I", INCLUDE, "-I", CSRC, *extra, "-c", path, "-o", obj]
            if ptxas_verbose:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd, verbose or ptxas_verbose)
    if _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"], verbose)
    return LIB


ORACLE_DIR = os.path.join(ROOT, "oracle")


def build_oracle(verbose: bool = False) -> str:
    src = os.path.join(ORACLE_DIR, "mimica_oracle.c")
    hdr = os.path.join(ORACLE_DIR, "mimica_oracle.h")
    out = os.path.join(ORACLE_DIR, "libmimica_oracle.so")
    if _stale(out, [src, hdr]):
        _run(["gcc", "-O2", "-fno-fast-math", "-ffp-contract=off", "-fPIC", "-shared", "-o", out, src, "-lm"], verbose)
    out_omp = os.path.join(ORACLE_DIR, "libmimica_oracle_omp.so")
    if _stale(out_omp, [src, hdr]):
        # the timed CPU baseline: OpenMP, the table-driven FFT and a heap that keeps freed fields (MO_FAST_FFT); built here and run on
        # another host, so the instruction set is a portable x86-64-v3 (AVX2), not this host's
        _run(["gcc", "-O3", "-march=x86-64-v3", "-fno-fast-math", "-ffp-contract=off", "-fopenmp", "-DMO_FAST_FFT", "-fPIC",
              "-shared", "-o", out_omp, src, "-lm"], verbose)
    return out


def build_reference_kiss(verbose: bool = False) -> str | None:
    """Compile the reference's KISS FFT (checker only) when a reference tree is named by
    the MIMICA_REFERENCE_TREE environment variable and holds its sources."""
    script = os.path.join(ORACLE_DIR, "build_ref.sh")
    target = os.path.join(ORACLE_DIR, "_ref", "libkissref.so")
    tree = os.environ.get("MIMICA_REFERENCE_TREE", "")
    if tree and os.path.isdir(os.path.join(tree, "src", "fftmpi", "src")) and os.path.exists(script):
        if _stale(target, [script, os.path.join(ORACLE_DIR, "ref_kiss_shim.cpp")]):
            _run(["bash", script, tree], verbose)
    return target if os.path.exists(target) else None


def build_all(verbose: bool = False) -> None:
    build_cuda(verbose)
    build_oracle(verbose)
    build_reference_kiss(verbose)


if __name__ == "__main__":
    v = "-v" in sys.argv
    if "--ptxas" in sys.argv:
        build_cuda(verbose=True, ptxas_verbose=True)
    else:
        build_all(verbose=v)
    print("built", LIB)
