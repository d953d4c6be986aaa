"""Build the engine's shared library in-tree for sm_100a.

    python matscipy-neighbours_b200/build.py [--force] [--checked]

Compiles csrc/*.cu with nvcc (``-gencode arch=compute_100a,code=sm_100a``),
links ``matscipy_neighbours/libnbl_b200.so`` next to the Python package, and
skips the work when the library is newer than every source.  Host code is
compiled without floating-point contraction: the grid planning must produce
the same doubles as the reference's CPU core.

``--checked`` builds ``libnbl_b200_checked.so`` instead: the same engine with
``-DNBL_CHECKED=1``, whose pair passes also test every cell slice, candidate,
hit-word and output-slot index and report a failed test as
NBL_ERROR_INTERNAL.  The Python package loads it when the environment sets
``MATSCIPY_NEIGHBOURS_CHECKED=1``.
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
OUT_CHECKED = PKG_ROOT / "matscipy_neighbours" / "libnbl_b200_checked.so"
BUILD_DIR = PKG_ROOT / "_build"

SOURCES = ["nbl_api.cu", "nbl_build.cu", "nbl_sort.cu", "nbl_noalloc.cu",
           "nbl_batch.cu", "nbl_backward.cu", "nbl_csr.cu", "nbl_verlet.cu",
           "nbl_trav_count32.cu", "nbl_trav_count32r.cu", "nbl_trav_count64.cu",
           "nbl_trav_fill32.cu", "nbl_trav_fill32r.cu", "nbl_trav_fill64.cu",
           "nbl_small.cu", "nbl_trav_atoms.cu"]

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


def up_to_date(checked=False):
    out = OUT_CHECKED if checked else OUT
    if not out.exists():
        return False
    t = out.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in _deps())


def build(force=False, verbose=False, checked=False):
    out = OUT_CHECKED if checked else OUT
    if not force and up_to_date(checked):
        return out
    bdir = BUILD_DIR / "checked" if checked else BUILD_DIR
    bdir.mkdir(parents=True, exist_ok=True)
    exe = nvcc()
    extra = ["-DNBL_CHECKED=1"] if checked else []

    def compile_one(src):
        obj = bdir / (src.stem + ".o")
        cmd = [exe, *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        return obj

    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, _sources()))
    tmp = out.with_suffix(".so.tmp")
    cmd = [exe, *ARCH, "-shared", "-o", str(tmp), *map(str, objs)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--checked", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, checked=a.checked))
    sys.exit(0)
