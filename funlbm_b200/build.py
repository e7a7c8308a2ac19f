"""Build ``liblbm_b200.so`` in-tree with nvcc for sm_100a.

    python -m funlbm_b200.build            # rebuild when a source is newer
    python -m funlbm_b200.build --force
    python -m funlbm_b200.build --checked  # the bounds-checked library

Each ``csrc/*.cu`` translation unit is compiled to an object in
``funlbm_b200/_build/`` (in parallel; ``lbm_step_inst.cu`` once per velocity
set and storage type) and linked into
``funlbm_b200/liblbm_b200.so`` with the CUDA runtime linked statically, so the
library only needs the driver at run time.  ``--checked`` builds the same
sources with -DLBM_BOUNDS_CHECK into ``funlbm_b200/liblbm_b200_checked.so``
(objects in ``funlbm_b200/_build_checked/``): every kernel verifies its index
invariants and counts violations instead of making the access; the package
loads it when FUNLBM_B200_CHECKED=1.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "liblbm_b200.so")
BUILD_CHECKED = os.path.join(PKG, "_build_checked")
LIB_CHECKED = os.path.join(PKG, "liblbm_b200_checked.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: no implicit multiply-add contraction; the kernels spell every
# fused multiply-add out, so all launch shapes produce the same bits
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "-I" + os.path.join(ROOT, "include")]


def _nvcc():
    exe = shutil.which("nvcc")
    if exe is None:
        cand = "/usr/local/cuda/bin/nvcc"
        if os.path.exists(cand):
            return cand
        raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build liblbm_b200.so")
    return exe


INSTANCED = "lbm_step_inst.cu"   # compiled once per (velocity set, storage)
INSTANCES = [(q, st) for q in (13, 15, 19, 27) for st in (0, 1, 2, 3)]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _units(build_dir=BUILD):
    """(source, object, extra flags) of every translation unit."""
    units = []
    for src in _sources():
        base = os.path.basename(src)[:-3]
        if os.path.basename(src) == INSTANCED:
            for q, st in INSTANCES:
                units.append((src, os.path.join(build_dir, "%s_q%d_s%d.o" % (base, q, st)),
                              ["-DLBM_Q=%d" % q, "-DLBM_S=%d" % st]))
        else:
            units.append((src, os.path.join(build_dir, base + ".o"), []))
    return units


def _deps():
    return _sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [
        os.path.join(ROOT, "include", "funlbm_b200.h"), os.path.abspath(__file__)]


def needs_build(lib=LIB):
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    return any(os.path.getmtime(p) > t for p in _deps())


def build(force=False, verbose=False, extra_flags=(), checked=False):
    """Compile and link the library (checked: the bounds-checked one);
    returns its path."""
    lib, build_dir = (LIB_CHECKED, BUILD_CHECKED) if checked else (LIB, BUILD)
    if checked:
        extra_flags = tuple(extra_flags) + ("-DLBM_BOUNDS_CHECK",)
    if not force and not needs_build(lib):
        return lib
    nvcc = _nvcc()
    os.makedirs(build_dir, exist_ok=True)
    units = _units(build_dir)
    objs = [u[1] for u in units]

    def compile_one(unit):
        src, obj, defs = unit
        cmd = [nvcc, *ARCH, *FLAGS, *extra_flags, *defs, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed on %s:\n%s%s" % (src, r.stdout, r.stderr))
        return obj

    # largest units first so the parallel build ends evenly
    order = sorted(units, key=lambda u: 0 if u[2] else 1)
    with cf.ThreadPoolExecutor(max_workers=min(len(units), os.cpu_count() or 4)) as ex:
        list(ex.map(compile_one, order))
    tmp = lib + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    os.replace(tmp, lib)
    return lib


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--checked", action="store_true",
                    help="build the bounds-checked library instead")
    args = ap.parse_args(argv)
    path = build(force=args.force, verbose=args.verbose, checked=args.checked)
    print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
