"""Build libmagic_b200.so in-tree with nvcc for sm_100a.

    python -m magic_b200.csrc.build        (or call build())

Each .cu file is compiled separately (parallel) and linked into
magic_b200/libmagic_b200.so, a plain C-ABI shared library (include/magic_b200.h).
"""

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
OUT = os.path.join(PKG, "libmagic_b200.so")
BUILD = os.path.join(ROOT, "_build")

SOURCES = ["api.cu", "tables.cu", "legendre_f64.cu", "fourier.cu", "nonlinear.cu",
           "split_tables.cu", "legendre_split.cu", "nl_split.cu", "split_transforms.cu",
           "nl_anel_split.cu", "radial_td.cu",
           "implicit.cu", "energy.cu", "ozaki.cu", "batch.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-I", os.path.join(ROOT, "include"),
]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _compile(src, verbose):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    cmd = [_nvcc(), *NVCC_FLAGS, "-c", os.path.join(HERE, src), "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
    return obj, r.stderr


def build(verbose=False, force=False):
    """Compile (if any source is newer than the library) and return its path."""
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    hdrs = [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith(".cuh")]
    hdrs.append(os.path.join(ROOT, "include", "magic_b200.h"))
    if not force and os.path.exists(OUT):
        t = os.path.getmtime(OUT)
        if all(os.path.getmtime(s) <= t for s in srcs + hdrs + [os.path.abspath(__file__)]):
            return OUT
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, len(SOURCES))) as ex:
        res = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if verbose:
        for _, log in res:
            sys.stderr.write(log)
    tmp = OUT + ".tmp"
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
           *[o for o, _ in res], "-o", tmp, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
