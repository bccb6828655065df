"""Build libalfa.so in-tree for sm_100a with nvcc (no JIT cache, no torch
extension machinery: the library is a plain C-ABI shared object)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libalfa.so")
# the engine, compiled once per storage precision (alfa_prec.cuh): FP64 into
# alfa::f64, FP32 (-DALFA_BUILD_FP32) into alfa::f32
ENGINE = ["alfa_line.cu", "alfa_spectral.cu", "alfa_physics.cu", "alfa_step.cu", "alfa_tc.cu"]
# the C-ABI, the no-allocation entry and the learned-coefficient network (FP64)
ONCE = ["alfa_capi.cu", "alfa_noalloc.cu", "alfa_mlp.cu"]
SOURCES = ENGINE + ONCE
HEADERS = ["alfa_prec.cuh", "alfa_fft.cuh", "alfa_fft_ct.cuh", "alfa_internal.cuh",
           "alfa_physics.cuh", "alfa_tile.cuh", "alfa_mlp.cuh", "alfa_step.cuh", "alfa_iface.cuh"]
# translation units: (source, extra flags, object suffix)
UNITS = ([(s, [], "") for s in ENGINE] + [(s, ["-DALFA_BUILD_FP32"], "_f32") for s in ENGINE] +
         [(s, [], "") for s in ONCE])

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-Xptxas", "-O3",
]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "alfa.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compile every CUDA source into jax_alfa_b200/libalfa.so."""
    if not force and not _stale():
        return LIB
    objs, procs = [], []
    for src, extra, suffix in UNITS:  # translation units compile concurrently
        obj = os.path.join(CSRC, src.replace(".cu", suffix + ".o"))
        cmd = [nvcc(), *NVCC_FLAGS, *extra, "-I", os.path.join(ROOT, "include"), "-I", CSRC,
               "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((src + suffix, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                            stderr=subprocess.PIPE, text=True)))
        objs.append(obj)
    failed = []
    for src, pr in procs:
        _, err = pr.communicate()
        if pr.returncode != 0:
            failed.append(f"nvcc failed on {src}:\n{err}")
        elif verbose:
            sys.stderr.write(err)
    if failed:
        raise RuntimeError("\n".join(failed))
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs,
           "-o", LIB, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
