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


def test_cmake_target_matches_build_script(tmp_path):
    """mt-imager_b200/CMakeLists.txt (the target a CMake host project adds)
    configures, compiles every csrc/*.cu that build.py compiles, and targets
    sm_100a only.  Configure step only: no compilation."""
    import shutil
    import subprocess
    import pytest
    cmake = shutil.which("cmake")
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    if cmake is None or not os.path.exists(nvcc):
        pytest.skip("cmake or nvcc not available")
    r = subprocess.run([cmake, "-S", os.path.join(ROOT, "mt-imager_b200"), "-B", str(tmp_path),
                        "-DCMAKE_CUDA_COMPILER=" + nvcc], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    flags = open(tmp_path / "CMakeFiles" / "mtb.dir" / "flags.make").read()
    assert "arch=compute_100a,code=[sm_100a]" in flags
    assert not re.search(r"sm_(?!100a)\d+", flags)
    build_make = open(tmp_path / "CMakeFiles" / "mtb.dir" / "build.make").read()
    compiled = set(re.findall(r"csrc/(\w+)\.cu\.o:", build_make))
    sources = {os.path.basename(s)[:-3] for s in glob.glob(os.path.join(ROOT, "mt-imager_b200", "csrc", "*.cu"))}
    assert compiled == sources


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    """No CPU fallback: without libmtb.so the binding raises instead of
    returning a stand-in."""
    import pytest
    from mtb import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="libmtb.so not found"):
        _lib.load(str(tmp_path / "libmtb.so"))


def test_c_program_uses_the_abi(tmp_path, mtblib):
    """tests/cpp/host_abi.c, plain C99 built with gcc against include/ and
    libmtb.so, calls the host-side entry points (ingest order, column gather,
    status strings, parameter refusals) without Python or a GPU."""
    import shutil
    import subprocess
    import pytest
    cc = os.environ.get("CC", "gcc")
    if shutil.which(cc) is None:
        pytest.skip("no C compiler")
    lib = os.path.join(ROOT, "mt-imager_b200")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    exe = tmp_path / "host_abi"
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-O2",
                    os.path.join(ROOT, "tests", "cpp", "host_abi.c"), "-o", str(exe),
                    "-I", os.path.join(ROOT, "include"), "-L", lib, "-lmtb", "-Wl,-rpath," + lib,
                    "-Wl,-rpath," + os.path.join(cuda, "lib64")], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"


def test_cpp_host_classes_compile():
    """include/mtb.hpp (the C++ classes over the C ABI) and the C++ programs
    that use them compile with g++ -std=c++17 on a machine without a GPU;
    running the programs is a GPU test."""
    import shutil
    import subprocess
    import pytest
    cxx = os.environ.get("CXX", "g++")
    if shutil.which(cxx) is None:
        pytest.skip("no C++ compiler")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    for prog in ("image_one.cpp", "lsrk_one.cpp"):
        r = subprocess.run([cxx, "-std=c++17", "-Wall", "-Werror", "-fsyntax-only",
                            os.path.join(ROOT, "tests", "cpp", prog),
                            "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include")],
                           capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, (prog, r.stderr)
