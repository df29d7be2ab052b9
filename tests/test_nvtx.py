"""NVTX ranges: every entry point that enqueues device work pushes a range
named after itself on entry and pops it on return (also on an early error
return), so profilers can attribute its kernels to it.  Checked on the CPU
with an NVTX injection probe (tests/cpp/nvtx_probe.c) that logs the pushes;
the calls here are refused on the host before any device work."""
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")

CALLS = r'''
import sys
sys.path.insert(0, sys.argv[1])
from mtb import _lib as L
lib = L.load()
N = None
assert lib.mtb_grid(N, N, N, N, N, N, N, N, N, N, 0, N, N, N, N, N, 0, N) == L.MTB_ERR_NULL
assert lib.mtb_grid_batch(N, 0, N, 0, N) != 0
assert lib.mtb_preprocess_uvw(N, N, N, N, N, N, N, N, 0, N, N, N, N, N, N, N, N, 0, N) == L.MTB_ERR_NULL
assert lib.mtb_finalize(N, N, N, N, N, N, 0, N) == L.MTB_ERR_NULL
assert lib.mtb_wkernel_build(N, N, 0, N, 0, N, N, N, N, N) == L.MTB_ERR_NULL
assert lib.mtb_taper_kernel_build(0, 0, N, 0, N, N, N, N, N) != 0
assert lib.mtb_grid_autotune(N, 0, N, 0, N, N, N) == L.MTB_ERR_NULL
print("calls done")
'''

NAMES = ["mtb_grid", "mtb_grid_batch", "mtb_preprocess_uvw", "mtb_finalize", "mtb_wkernel_build",
         "mtb_taper_kernel_build", "mtb_grid_autotune"]


def test_entry_points_push_nvtx_ranges(tmp_path, mtblib):
    cc = os.environ.get("CC", "gcc")
    if shutil.which(cc) is None:
        pytest.skip("no C compiler")
    probe = tmp_path / "nvtx_probe.so"
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-shared", "-fPIC",
                    "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "nvtx_probe.c"),
                    "-o", str(probe)], check=True)
    log = tmp_path / "nvtx.log"
    env = dict(os.environ, NVTX_INJECTION64_PATH=str(probe), MTB_NVTX_LOG=str(log))
    r = subprocess.run([sys.executable, "-c", CALLS, os.path.join(ROOT, "mt-imager_b200")], env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "calls done" in r.stdout, r.stdout + r.stderr
    lines = log.read_text().split("\n")
    pushed = [l[5:] for l in lines if l.startswith("push ")]
    assert pushed == NAMES, pushed
    assert sum(1 for l in lines if l == "pop") == len(NAMES)
