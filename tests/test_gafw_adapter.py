"""The GAFW operator adapter (mt-imager_b200/gafw_adapter/): the four operators
compiled against the GAFW interface (oracle/ref_stubs/GPUafw.h mirrors
GPUArrayOperator.h:27-43, GPUSubmissionData.h:27-47 and ArrayDimensions.h) and
linked to libmtb.so on a machine without a GPU; on the GPU,
tests/cpp/gafw_adapter.cpp drives them through validate / submitToGPU as GAFW's
engine does and compares every output with the direct C-ABI call.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "mt-imager_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _compile(out, mtblib_dir):
    cxx = os.environ.get("CXX", "g++")
    if shutil.which(cxx) is None:
        pytest.skip("no C++ compiler")
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Werror",
           os.path.join(ROOT, "tests", "cpp", "gafw_adapter.cpp"),
           os.path.join(PKG, "gafw_adapter", "mtb_gafw_operators.cpp"),
           "-I", os.path.join(ROOT, "oracle", "ref_stubs"), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(PKG, "gafw_adapter"), "-I", os.path.join(CUDA, "include"),
           "-L", mtblib_dir, "-lmtb", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           "-Wl,-rpath," + mtblib_dir, "-Wl,-rpath," + os.path.join(CUDA, "lib64"), "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr


def test_adapter_compiles_and_links(tmp_path, mtblib):
    """The operators and their driver compile with -Wall -Werror against the
    GAFW interface and link against libmtb.so (no GPU needed)."""
    _compile(tmp_path / "gafw_adapter", PKG)
    assert (tmp_path / "gafw_adapter").exists()


def test_adapter_scratch_fits_an_int():
    """validate() refuses scratch above INT_MAX: GAFW passes the size to
    submitToGPU as an int (GPUSubmissionData.h:42)."""
    src = open(os.path.join(PKG, "gafw_adapter", "mtb_gafw_operators.cpp")).read()
    assert "kMaxScratch = (size_t)INT_MAX" in src
    for op in ("PreProcessUVW", "mtb::GridChunk", "mtb::ImageFinalizer", "mtb::WProjectionConvFunction"):
        assert f'"{op}: ' in src or f'"{op}' in src
    assert src.count("> kMaxScratch") == 4


@pytest.mark.gpu
def test_adapter_matches_direct_calls(tmp_path, mtblib):
    """validate + submitToGPU of each operator, with engine-allocated outputs
    and an int scratch size, equals the direct mtb_* call: the kernel tables,
    PreProcessUVW's seven outputs, the normaliser and statistics bit for bit;
    the grid of two accumulated chunks to 2e-6 of its peak (FP32 atomics in
    the per-call delta grid); the finalised image bit for bit."""
    from mtb import synth
    exe = tmp_path / "gafw_adapter"
    _compile(exe, PKG)
    obs, setup = synth.small_config(seed=21, n_ant=10, ntimes=60, nx=128, wplanes=8, sampling=4)
    P = 4
    R = obs.nrec
    d = tmp_path / "case"
    d.mkdir()
    with open(d / "params.txt", "w") as f:
        f.write(f"{setup.nx} {setup.ny} {setup.dl!r} {setup.wplanes} {setup.sampling} {R} {P}\n")
    np.ascontiguousarray(obs.uvw, np.float32).tofile(d / "uvw.f32")
    np.ascontiguousarray(obs.freq_over_c(0), np.float32).tofile(d / "freq.f32")
    np.ascontiguousarray(obs.vis[0][:, :P], np.complex64).tofile(d / "vis.c64")
    np.ascontiguousarray(obs.weights[0][:, :P], np.float32).tofile(d / "weights.f32")
    np.ascontiguousarray(obs.flags[0][:, :P], np.int32).tofile(d / "flags.i32")
    r = subprocess.run([str(exe), str(d)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "all match"
