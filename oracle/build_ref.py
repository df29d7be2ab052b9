"""TEST INFRASTRUCTURE, NOT PRODUCT CODE.

Builds oracle/_ref/libmtref.so: mt-imager's own operator sources, compiled
unchanged from where they lie in the reference tree for sm_100a against the
GAFW stand-in headers in oracle/ref_stubs/, linked with oracle/ref_harness.cu.
Nothing is copied out of the reference tree; the only outputs are the object
files and the library under oracle/_ref/ (git-ignored).  The library is used
to make the golden fixtures under tests/golden/ (tests/golden/make_golden.py)
and is never loaded by the product.

    python oracle/build_ref.py --reference DIR      (or MTB_REFERENCE_DIR=DIR)

The reference tree's location comes from the argument or the environment
variable only; without either, nothing is built.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
ENV_REF = "MTB_REFERENCE_DIR"

# (directory inside the reference's code/ tree, source file)
SOURCES = [
    ("mt-imager/lib/operators", "WProjPreProcessUVW.cu"),
    ("mt-imager/lib/operators", "CreateindexAndReorder.cu"),
    ("mt-imager/lib/operators", "CreateBlockIndex.cu"),
    ("mt-imager/lib/operators", "NotSameSupportManipulate.cu"),
    ("mt-imager/lib/operators", "CreateCompressionPlan.cu"),
    ("mt-imager/lib/operators", "CompressVisibilties.cu"),
    ("mt-imager/lib/operators", "ConvolutionGridder.cu"),
    ("mt-imager/lib/operators", "CasaGridSF.cu"),
    ("mt-imager/lib/operators", "WProjPreFFTconvFunc.cu"),
    ("mt-imager/lib/operators", "ConvFunctionSupportFind.cu"),
    ("mt-imager/lib/operators", "ConvFunctionReOrganize.cu"),
    ("mt-imager/lib/operators", "SumConvolutionFunctions.cu"),
    ("mt-imager/lib/operators", "PreIFFTUVCorrection.cu"),
    ("mt-imager/lib/operators", "PostIFFTStokesConverter.cu"),
    ("mt-imager/lib/operators", "SincCorrector.cu"),
    ("gafw/Implimentation/StandardOperators", "AccumulatedSum.cu"),
    ("gafw/Implimentation/StandardOperators", "ValueChangeDetect.cu"),
    ("gafw/Implimentation/StandardOperators", "ZeroToCentre2DShift.cu"),
    ("gafw/Implimentation/StandardOperators", "SingleMultiply.cu"),
]
INCLUDE_DIRS = ["mt-imager/lib/operators", "gafw/Implimentation/StandardOperators"]
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(reference: str | None = None, verbose: bool = False) -> str | None:
    """Builds the library from the reference tree at `reference` (default: the
    MTB_REFERENCE_DIR environment variable); returns None when no tree is
    given or found."""
    reference = reference or os.environ.get(ENV_REF)
    if not reference:
        return None
    code = os.path.join(reference, "code")
    if not os.path.isdir(code):
        return None
    os.makedirs(OUT, exist_ok=True)
    # stand-in headers first, so "GPUafw.h" and friends resolve to them
    inc = ["-I" + os.path.join(HERE, "ref_stubs")] + ["-I" + os.path.join(code, d) for d in INCLUDE_DIRS]
    # -maxrregcount=64: the reference was written for sm_20/sm_30, whose
    # 63-register limit every 1024-thread launch of its operators relies on
    flags = [ARCH, "-O2", "-std=c++17", "-maxrregcount=64", "-Xcompiler", "-fPIC", "-w", "-x", "cu"]
    jobs = [(os.path.join(code, d, f), os.path.join(OUT, f + ".o")) for d, f in SOURCES]
    jobs.append((os.path.join(HERE, "ref_harness.cu"), os.path.join(OUT, "ref_harness.o")))

    def compile_one(job):
        src, obj = job
        if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _stub_mtime()):
            return obj
        cmd = [nvcc()] + flags + inc + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed on %s:\n%s" % (src, r.stderr[-4000:]))
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, jobs))
    lib = os.path.join(OUT, "libmtref.so")
    cmd = [nvcc(), ARCH, "-shared", "-o", lib] + objs + ["-lcufft"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stderr[-4000:])
    if verbose:
        print(lib)
    return lib


def _stub_mtime():
    d = os.path.join(HERE, "ref_stubs")
    return max([os.path.getmtime(os.path.join(d, f)) for f in os.listdir(d)] +
               [os.path.getmtime(os.path.join(HERE, "ref_harness.cu"))])


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="the reference tree (default: $%s)" % ENV_REF)
    a = ap.parse_args()
    out = build(a.reference, verbose=True)
    if out is None:
        sys.exit("no reference tree: pass --reference DIR or set %s" % ENV_REF)
