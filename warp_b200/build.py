"""Builds libwarp_b200.so in-tree with nvcc for sm_100a (no GPU needed).

    python -m warp_b200.build

The FP64 field and particle kernels are compiled with --fmad=false so their
rounding follows the reference's expression order (bit-identical to the
oracle for identical inputs).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libwarp_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["wg_api.cu", "wg_mg.cu", "wg_particles.cu", "wg_conductors.cpp", "wg_unet.cu"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


FMAD_CONTRACT = {"wg_unet.cu"}


def _obj(src):
    return os.path.join(CSRC, "_build", os.path.splitext(src)[0] + ".o")


def build(verbose=False, force=False):
    os.makedirs(os.path.join(CSRC, "_build"), exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "warp_b200.h"))
    newest_dep = max(os.path.getmtime(d) for d in deps)
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = _obj(src)
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), newest_dep):
            continue
        # --fmad=false keeps every FP64 expression in the reference's operand
        # order, without fused multiply-adds, so the FP64 paths match the
        # oracle bit for bit. The convolutions of the learned guess have no
        # such reference and keep contraction.
        fmad = "--fmad=true" if src in FMAD_CONTRACT else "--fmad=false"
        cmd = [nvcc(), "-c", path, "-o", obj, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", fmad,
               "-lineinfo"] + ARCH
        if src.endswith(".cpp"):
            cmd += ["-x", "cu"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
