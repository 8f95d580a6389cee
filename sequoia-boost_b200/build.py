"""In-tree build of libsb_gpu.so (sm_100a) with nvcc.

Every CUDA source is compiled for `sm_100a` only, with `-fmad=false` so that
no multiply-add is contracted: the FP64 split scan and the f32 leaf / margin
arithmetic then round exactly as the CPU oracle (and the reference) round.
The TreeSHAP file is the exception (`-fmad=true`): its results are checked
within 1e-4, and contracting its f64 multiply-adds halves their instructions.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsb_gpu.so")
SOURCES = ["sb_core.cu", "sb_bin.cu", "sb_hist.cu", "sb_grow.cu", "sb_predict.cu", "sb_shap.cu", "sb_static.cu",
           "sb_serve.cu", "sb_jobs.cu", "sb_eval.cu", "sb_approx.cu"]
# per-source flags that replace the defaults above
SOURCE_FLAGS = {"sb_shap.cu": {"-fmad=false": "-fmad=true"}}
HEADERS = ["sb_internal.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
    "-Xptxas", "-warn-spills",
]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, extra_flags=()):
    os.makedirs(BUILD, exist_ok=True)
    inc = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(HERE, "..", "include", "sb_gpu.h"),
        os.path.join(HERE, "..", "include", "sb_sampling.h")]
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if _newer(o, [s] + inc + [os.path.abspath(__file__)]):
            flags = [SOURCE_FLAGS.get(src, {}).get(f, f) for f in FLAGS]
            cmd = [NVCC, *flags, *extra_flags, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if _newer(LIB, objs):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", LIB,
               "-lcudart", "-lpthread", "-Xlinker", "--no-undefined"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra_flags=sys.argv[1:])
