"""Builds oracle/_ref/libjuicer_ref.so: the reference's own CUDA render kernels,
compiled for sm_100a straight from the read-only reference tree, plus ref_shim.cu.

Test infrastructure only (GPU parity tests). Nothing is copied out of the reference:
nvcc reads the sources where they lie; only the built library lands in oracle/_ref/
(git-ignored, shipped to the GPU box with the snapshot).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF = os.environ.get("FJ_REFERENCE_ROOT", "/root/reference")
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libjuicer_ref.so")
TUS = ["src/Cuda/Scan/JuicerCudaScanPipeline.cu", "src/Cuda/Film/JuicerCudaFilmPipeline.cu",
       "src/Cuda/Film/JuicerCudaScatterHalation.cu", "src/Cuda/Film/JuicerCudaHighlightBoost.cu",
       "src/Cuda/JuicerCudaAutoExposure.cu"]


def main() -> int:
    if not os.path.isdir(REF):
        print("reference tree absent; keeping any prebuilt", LIB)
        return 0
    os.makedirs(OUT, exist_ok=True)
    srcs = [os.path.join(REF, t) for t in TUS] + [os.path.join(HERE, "ref_shim.cu")]
    newest = max(os.path.getmtime(s) for s in srcs)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return 0
    inc = ["-I", os.path.join(REF, "src"), "-I", os.path.join(REF, "third_party"), "-I", os.path.join(REF, "native")]
    objs = []
    procs = []
    for s in srcs:
        obj = os.path.join(OUT, os.path.basename(s) + ".o")
        extra = ["-I", os.path.join(REPO, "include")] if s.endswith("ref_shim.cu") else []
        cmd = ["nvcc", "-std=c++20", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-Xcompiler", "-fPIC",
               *inc, *extra, "-c", s, "-o", obj]
        procs.append(subprocess.Popen(cmd))
        objs.append(obj)
    if any(p.wait() != 0 for p in procs):
        return 1
    return subprocess.call(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs,
                            "-cudart=static"])


FFT_LIB = os.path.join(OUT, "libjuicer_ref_fft.so")
FFT_TUS = ["src/Cuda/Diffusion/JuicerCudaDiffusion.cu", "src/DiffusionExecution.cpp", "src/Cuda/JuicerCudaFailure.cpp",
           "src/DiffusionHostBehavior.cpp"]


def build_fft() -> int:
    """oracle/_ref/libjuicer_ref_fft.so: the reference's cuFFT camera diffusion with its
    execution planner, driven by ref_fft_shim.cu, linked against the toolkit's cuFFT."""
    srcs = [os.path.join(REF, t) for t in FFT_TUS] + [os.path.join(HERE, "ref_fft_shim.cu")]
    newest = max(os.path.getmtime(s) for s in srcs)
    if os.path.exists(FFT_LIB) and os.path.getmtime(FFT_LIB) >= newest:
        return 0
    inc = ["-I", os.path.join(REF, "src"), "-I", os.path.join(REF, "third_party"), "-I", os.path.join(REF, "native")]
    objs, procs = [], []
    for s in srcs:
        obj = os.path.join(OUT, "fft_" + os.path.basename(s) + ".o")
        lang = ["-x", "cu"] if s.endswith(".cpp") else []
        cmd = ["nvcc", "-std=c++20", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-Xcompiler", "-fPIC",
               *lang, *inc, "-c", s, "-o", obj]
        procs.append(subprocess.Popen(cmd))
        objs.append(obj)
    if any(p.wait() != 0 for p in procs):
        return 1
    return subprocess.call(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", FFT_LIB, *objs,
                            "-lcufft", "-cudart=static"])


if __name__ == "__main__":
    rc = main()
    if rc == 0 and os.path.isdir(REF):
        rc = build_fft()
    sys.exit(rc)
