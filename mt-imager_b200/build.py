"""Builds libmtb.so (the sm_100a kernels and the C ABI) in-tree.

    python mt-imager_b200/build.py [--force] [--verbose] [--checked]

Every translation unit in csrc/ is compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) and linked against the CUDA
toolkit's cuFFT.  Objects go to csrc/_build/, the library to
mt-imager_b200/libmtb.so.  ``--checked`` builds the bounds-checked variant
instead (-DMTB_CHECKED: the gridders check every table tap and grid cell
they touch and record an index out of range in a status word instead of
faulting; see mtb_bounds_status in include/mtb.h): objects in
csrc/_build_checked/, library mt-imager_b200/libmtb_checked.so, loaded by
the Python binding when MTB_LIBRARY=checked.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(CSRC, "_build")
LIB = os.path.join(HERE, "libmtb.so")
OBJ_CHECKED = os.path.join(CSRC, "_build_checked")
LIB_CHECKED = os.path.join(HERE, "libmtb_checked.so")
INCLUDE = os.path.join(ROOT, "include")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc") if os.path.exists(os.path.join(CUDA, "bin", "nvcc")) else shutil.which("nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I", INCLUDE, "-I", CSRC]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose, obj_dir=OBJ, defines=()):
    obj = os.path.join(obj_dir, os.path.basename(src)[:-3] + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, *defines, "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    if NVCC is None:
        raise RuntimeError("nvcc not found")
    obj_dir, lib = (OBJ_CHECKED, LIB_CHECKED) if checked else (OBJ, LIB)
    defines = ("-DMTB_CHECKED",) if checked else ()
    os.makedirs(obj_dir, exist_ok=True)
    srcs = _sources()
    hdrs = _headers()
    todo = [s for s in srcs if force or verbose or
            _stale(os.path.join(obj_dir, os.path.basename(s)[:-3] + ".o"), [s, *hdrs])]
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(todo)))) as ex:
        for obj, err in ex.map(lambda s: _compile(s, verbose, obj_dir, defines), todo):
            if verbose and err:
                sys.stderr.write(err)
    objs = [os.path.join(obj_dir, os.path.basename(s)[:-3] + ".o") for s in srcs]
    if force or todo or _stale(lib, objs):
        tmp = lib + ".tmp%d" % os.getpid()
        cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-L", os.path.join(CUDA, "lib64"), "-lcufft",
               "-Xlinker", "-rpath," + os.path.join(CUDA, "lib64")]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
        os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv, checked="--checked" in sys.argv))
