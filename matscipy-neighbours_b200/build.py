"""Build the engine's shared library in-tree for sm_100a.

    python matscipy-neighbours_b200/build.py [--force]

Compiles csrc/*.cu with nvcc (``-gencode arch=compute_100a,code=sm_100a``),
links ``matscipy_neighbours/libnbl_b200.so`` next to the Python package, and
skips the work when the library is newer than every source.  Host code is
compiled without floating-point contraction: the grid planning must produce
the same doubles as the reference's CPU core.
"""

import argparse
import concurrent.futures
import os
import pathlib
import shutil
import subprocess
import sys

PKG_ROOT = pathlib.Path(__file__).resolve().parent
REPO = PKG_ROOT.parent
CSRC = PKG_ROOT / "csrc"
INCLUDE = REPO / "include"
OUT = PKG_ROOT / "matscipy_neighbours" / "libnbl_b200.so"
BUILD_DIR = PKG_ROOT / "_build"

SOURCES = ["nbl_api.cu", "nbl_build.cu", "nbl_sort.cu", "nbl_noalloc.cu",
           "nbl_batch.cu", "nbl_backward.cu", "nbl_csr.cu", "nbl_verlet.cu",
           "nbl_trav_count32.cu", "nbl_trav_count64.cu", "nbl_trav_fill32.cu",
           "nbl_trav_fill64.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", f"-I{INCLUDE}", f"-I{CSRC}",
         "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
         "--expt-relaxed-constexpr"]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build")
    return exe


def _sources():
    return [CSRC / s for s in SOURCES if (CSRC / s).exists()]


def _deps():
    return list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + \
        list(CSRC.glob("*.hh")) + list(INCLUDE.glob("*.h")) + [pathlib.Path(__file__)]


def up_to_date():
    if not OUT.exists():
        return False
    t = OUT.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in _deps())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return OUT
    BUILD_DIR.mkdir(exist_ok=True)
    exe = nvcc()

    def compile_one(src):
        obj = BUILD_DIR / (src.stem + ".o")
        cmd = [exe, *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        return obj

    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, _sources()))
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [exe, *ARCH, "-shared", "-o", str(tmp), *map(str, objs)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
    sys.exit(0)
