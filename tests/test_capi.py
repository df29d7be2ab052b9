"""The C ABI library builds for sm_100a, loads, and exports every entry point
include/*.h declares (no GPU needed, no compute calls)."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(mtb_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("mtb_wkernel_query", "mtb_wkernel_build", "mtb_grid", "mtb_grid_workspace_size",
              "mtb_preprocess_uvw", "mtb_finalize", "mtb_finalize_workspace_size", "mtb_status_string",
              "mtb_version", "mtb_release_caches"):
        assert n in names


def test_library_exports_every_declared_symbol(mtblib):
    for n in sorted(declared_symbols()):
        assert hasattr(mtblib, n), n
    assert mtblib.mtb_version() >= 100
    assert mtblib.mtb_status_string(0) == b"ok"
    assert b"workspace" in mtblib.mtb_status_string(3)


def test_build_targets_sm100a_only():
    import importlib.util
    spec = importlib.util.spec_from_file_location("mtb_build", os.path.join(ROOT, "mt-imager_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    assert mod.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_python_binding_matches_header():
    from mtb import _lib
    assert set(_lib.EXPORTS) == declared_symbols()
    # struct layouts the binding passes by pointer
    assert ctypes.sizeof(_lib.WKernelParams) == 48
    assert ctypes.sizeof(_lib.GridStats) == 32
