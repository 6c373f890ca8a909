"""Build the in-tree native libraries with nvcc / gcc (no JIT cache).

* ``lib/libqzb200.so``  -- CUDA kernels + C ABI (include/qz_b200.h), sm_100a only,
  built with -fmad=false so FP64 expressions round like the reference's
  x86-64 code (products and sums are never contracted).
* ``lib/libqz_dropin.so`` -- the reference-symbol shim (include/qz_dropin.h):
  exports grid_density, potential, ... and resolves the reference's globals
  from the host program at first call.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

CUDA_SOURCES = ["qz_capi.cu", "qz_particles.cu", "qz_poisson.cu", "qz_sort.cu", "qz_amr.cu",
                "qz_noalloc.cu", "qz_observe.cu",
                "qz_ensemble.cu", "qz_adjoint.cu", "qz_snapshot.cu", "qz_testhooks.cu",
                "qz_node_mg.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "-I", os.path.join(ROOT, "include")]


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]) + " ...")


def build_cuda(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    out = os.path.join(LIBDIR, "libqzb200.so")
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES]
    deps = srcs + [os.path.join(CSRC, "qz_internal.cuh"), os.path.join(CSRC, "qz_amr_dev.cuh"),
                   os.path.join(ROOT, "include", "qz_b200.h")]
    if not force and not _newer(out, deps):
        return out
    objs = []
    for s in srcs:
        o = os.path.join(LIBDIR, os.path.basename(s).replace(".cu", ".o"))
        cmd = [NVCC, *ARCH, *NVCC_FLAGS, "-c", s, "-o", o]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
        _run(cmd)
        objs.append(o)
    _run([NVCC, *ARCH, "-shared", "-o", out, *objs, "-lcudart_static", "-Xcompiler", "-fPIC"])
    for o in objs:
        os.remove(o)
    return out


def build_dropin(force: bool = False) -> str:
    out = os.path.join(LIBDIR, "libqz_dropin.so")
    src = os.path.join(CSRC, "qz_dropin.c")
    deps = [src, os.path.join(ROOT, "include", "qz_dropin.h"), os.path.join(ROOT, "include", "qz_b200.h")]
    if not force and not _newer(out, deps + [os.path.join(LIBDIR, "libqzb200.so")]):
        return out
    _run(["gcc", "-O2", "-fPIC", "-shared", "-Wall", "-I", os.path.join(ROOT, "include"), src,
          "-o", out, "-L", LIBDIR, "-lqzb200", "-Wl,-rpath,$ORIGIN", "-ldl"])
    return out


def build_all(force: bool = False) -> None:
    build_cuda(force)
    build_dropin(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", LIBDIR)
