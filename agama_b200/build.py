"""Build recipe for the engine's native library (in-tree, so the .so travels with the repo).

    python -m agama_b200.build          # or agama_b200.build.build()

Compiles every source under agama_b200/csrc with nvcc for sm_100a only into
agama_b200/_lib/libagama_b200.so.  Objects are cached in agama_b200/_lib/obj and rebuilt when a
source or any header changed.
"""
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUTDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(OUTDIR, "obj")
LIBNAME = os.path.join(OUTDIR, "libagama_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]
CUDA_FLAGS = ARCH + ["-Xptxas", "-O3", "--expt-relaxed-constexpr", "--extended-lambda"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _compile(src, newest_header, verbose):
    obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), newest_header):
        return obj
    cmd = [NVCC, "-c", src, "-o", obj] + COMMON
    if src.endswith(".cu"):
        cmd += CUDA_FLAGS
    else:
        # host construction code: FMA contraction on, as in the reference's own -march builds,
        # so that the spline tables come out identical to the reference's
        cmd += ["-x", "c++", "-Xcompiler", "-march=x86-64-v3"] + ARCH
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
    if verbose and r.stderr.strip():
        print(r.stderr, flush=True)
    return obj


def build(verbose=False, force=False):
    os.makedirs(OBJDIR, exist_ok=True)
    if force:
        for f in glob.glob(os.path.join(OBJDIR, "*.o")):
            os.remove(f)
    newest_header = max([os.path.getmtime(h) for h in _headers()] + [os.path.getmtime(__file__)])
    srcs = _sources()
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, newest_header, verbose), srcs))
    if os.path.exists(LIBNAME) and os.path.getmtime(LIBNAME) >= max(os.path.getmtime(o) for o in objs):
        return LIBNAME
    cmd = [NVCC, "-shared", "-o", LIBNAME] + objs + ARCH + ["-lcudart", "-lcuda"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    return LIBNAME


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
