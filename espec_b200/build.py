"""Build libespecgpu.so in-tree with nvcc for sm_100a.

    python -m espec_b200.build          # or espec_b200.build.build()

The library has no torch dependency: plain CUDA runtime + C-ABI.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libespecgpu.so")
SOURCES = ["spo1d.cu", "capi.cu", "spo1d_inst_f32_pow2.cu", "spo1d_inst_f32_r3.cu",
           "spo1d_inst_f64_pow2.cu", "spo1d_inst_f64_r3.cu", "spo1d_persist.cu", "spo1d_any.cu", "spo_tc.cu", "spo1d_static.cu", "sod1d_inst.cu",
           "diag1d.cu", "dropin.cu", "sil.cu",
           "spectrum.cu", "potential.cu", "eig.cu", "mlp.cu", "mlp_tc.cu",
           "spond.cu", "deck.cpp", "pulse.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# per-file flags: the analytic potentials follow the reference's arithmetic
# (no fused multiply-add), so that they match it to the last bit of exp/cos
FILE_FLAGS = {"potential.cu": ["-fmad=false"]}


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "espec_gpu.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.isfile(d))


def build(force=False, verbose=False):
    """Compile each translation unit in parallel, then link the shared library."""
    if not force and not needs_build():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
    if verbose:
        common.append("-Xptxas=-v")
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        cmd = common + FILE_FLAGS.get(src, []) + ["-c", os.path.join(CSRC, src), "-o", obj]
        procs.append((src, subprocess.Popen(cmd)))
    bad = [src for src, pr in procs if pr.wait() != 0]
    if bad:
        raise RuntimeError("nvcc failed for " + ", ".join(bad))
    subprocess.check_call([nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart"])
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
