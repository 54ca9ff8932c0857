"""Build ``deconlib_b200/libdecon_b200.so`` from the CUDA sources (sm_100a).

    python deconlib_b200/csrc/build.py [--verbose-ptxas]

One ``nvcc`` per translation unit (parallel), then one link.  The library is
built in-tree so it travels with the source snapshot; nothing is installed.
"""

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
OBJ = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(PKG, "libdecon_b200.so")
SOURCES = ["capi.cu", "conv.cu", "reduce.cu", "ops.cu", "solvers.cu", "noalloc.cu", "batch.cu", "psf.cu", "nlcg.cu", "pdhg_run.cu", "pupil.cu",
           "xstatic_r2c.cu", "xstatic_c2r.cu", "xstatic_col.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _compile(src, ptxas_v):
    obj = os.path.join(OBJ, src.replace(".cu", ".o"))
    path = os.path.join(HERE, src)
    deps = [path] + [os.path.join(HERE, h) for h in os.listdir(HERE) if h.endswith(".cuh")]
    deps.append(os.path.join(ROOT, "include", "decon_b200.h"))
    if os.path.exists(obj) and not ptxas_v and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj, ""
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
           "--expt-relaxed-constexpr", "-c", path, "-o", obj]
    if ptxas_v:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose_ptxas=False, quiet=True):
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas), SOURCES))
    objs = [o for o, _ in results]
    if verbose_ptxas:
        for _, log in results:
            print(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    if not quiet:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    try:
        build(a.verbose_ptxas, quiet=False)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
