"""Build libalfa.so in-tree for sm_100a with nvcc (no JIT cache, no torch
extension machinery: the library is a plain C-ABI shared object)."""
import os
import subprocess
import sys
import time

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


OBJ_DIR = os.path.join(ROOT, "_build")


def _deps(src, obj):
    """The files an object was compiled from: nvcc's dependency list of its
    last compile (obj.d), else the source and every header of the library."""
    try:
        with open(obj + ".d") as f:
            text = f.read().replace("\\\n", " ")
        files = [t for t in text.split(":", 1)[1].split() if os.path.exists(t)]
        if files:
            return files
    except (OSError, IndexError):
        pass
    return ([os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS]
            + [os.path.join(ROOT, "include", "alfa.h")])


def _unit_stale(src, obj, cmd):
    """An object is rebuilt when it is missing, was compiled with another
    recorded command line, or is older than a file it was compiled from."""
    if not os.path.exists(obj):
        return True
    try:
        with open(obj + ".cmd") as f:
            if f.read() != " ".join(cmd):
                return True
    except OSError:  # compiled before command lines were recorded
        pass
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in _deps(src, obj))


def build(force=False, verbose=False):
    """Compile every CUDA source into jax_alfa_b200/libalfa.so (objects kept
    in _build/ so that an edit recompiles only the units it touches)."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    objs, procs = [], []
    for src, extra, suffix in UNITS:  # translation units compile concurrently
        obj = os.path.join(OBJ_DIR, src.replace(".cu", suffix + ".o"))
        objs.append(obj)
        cmd = [nvcc(), *NVCC_FLAGS, *extra, "-I", os.path.join(ROOT, "include"), "-I", CSRC,
               "-c", os.path.join(CSRC, src), "-o", obj]
        if not force and not _unit_stale(src, obj, cmd):
            continue
        with open(obj + ".cmd", "w") as f:
            f.write(" ".join(cmd))
        cmd += ["-MD", "-MF", obj + ".d"]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((src + suffix, obj, time.time(),
                      subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                       text=True)))
    failed = []
    for src, obj, t0, pr in procs:
        _, err = pr.communicate()
        if pr.returncode != 0:
            failed.append(f"nvcc failed on {src}:\n{err}")
            continue
        # the object describes the sources as they were when its compile
        # started: an edit made meanwhile leaves it stale
        os.utime(obj, (t0, t0))
        if verbose:
            sys.stderr.write(err)
    if failed:
        raise RuntimeError("\n".join(failed))
    if not procs and os.path.exists(LIB) and all(
            os.path.getmtime(o) <= os.path.getmtime(LIB) for o in objs):
        return LIB  # every object current and already linked
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs,
           "-o", LIB, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv or "--all" in sys.argv, verbose="-v" in sys.argv))
