"""The bounds-checked build (libmtb_checked.so, build.py --checked,
-DMTB_CHECKED): the gridders check every kernel-table tap and grid cell they
touch before the access and record an index out of range in a status word
(mtb_bounds_status) instead of faulting.  On the CPU: both libraries export
the whole ABI and say which build they are.  On the GPU: images through the
checked build, with every gridder, match the FP64 oracle and leave the status
word at 0."""
import ctypes
import importlib.util
import os
import subprocess
import sys

import pytest

from mtb import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "mt-imager_b200")


@pytest.fixture(scope="module")
def checked_lib():
    spec = importlib.util.spec_from_file_location("mtb_build", os.path.join(PKG, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(checked=True)


def run_checked(code):
    env = dict(os.environ, MTB_LIBRARY="checked")
    return subprocess.run([sys.executable, "-c", code, PKG, ROOT], env=env, capture_output=True, text=True,
                          timeout=900)


def test_plain_library_is_unchecked(mtblib):
    checked, word = ctypes.c_int(-1), ctypes.c_uint(7)
    assert mtblib.mtb_bounds_status(ctypes.byref(checked), ctypes.byref(word)) == L.MTB_OK
    assert checked.value == 0 and word.value == 0
    assert mtblib.mtb_bounds_status(None, ctypes.byref(word)) == L.MTB_ERR_NULL


def test_checked_library_exports_the_abi(checked_lib):
    assert checked_lib.endswith("libmtb_checked.so") and os.path.exists(checked_lib)
    r = run_checked(r'''
import ctypes, sys
sys.path.insert(0, sys.argv[1])
from mtb import _lib as L
lib = L.load()
assert L.LIB_PATH.endswith("libmtb_checked.so")
for name in L.EXPORTS:
    getattr(lib, name)
c, w = ctypes.c_int(-1), ctypes.c_uint(0)
rc = lib.mtb_bounds_status(ctypes.byref(c), ctypes.byref(w))
import torch
if torch.cuda.is_available():
    assert rc == L.MTB_OK and c.value == 1, (rc, c.value)
else:
    assert rc == L.MTB_ERR_CUDA, rc       # the status word lives on the device
print("exports ok")
''')
    assert r.returncode == 0 and "exports ok" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_checked_build_images_match_oracle(checked_lib):
    r = run_checked(r'''
import ctypes, sys
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[2])
import numpy as np, torch
from mtb import synth, _lib as L
from mtb.imager import WProjectionImager, grid_batch
from oracle import oracle as O
lib = L.load()
assert L.LIB_PATH.endswith("libmtb_checked.so")
obs, setup = synth.small_config(seed=31, n_ant=10, ntimes=60, nx=128, cell_arcsec=20, wplanes=8, sampling=4,
                                flag_frac=0.1)
ref, _, _ = O.image_channel(obs, 0, setup)
peak = np.abs(ref[0]).max()
def image(**kw):
    im = WProjectionImager(setup.nx, setup.ny, setup.dl, wplanes=setup.wplanes, sampling=setup.sampling, **kw)
    im.build_kernels()
    im.grid_chunk(obs.uvw, obs.freq_over_c(0), obs.vis[0], obs.weights[0], obs.flags[0])
    return im.finalize().cpu().numpy()
for kw in (dict(gridder=3), dict(gridder=5), dict(gridder=7), dict(gridder=8), dict(merge=1),
           dict(gridder=7, support_bucket=3), dict(gridder=7, exact_delta=True)):
    img = image(**kw)
    err = max(np.sqrt(np.mean((img[p] - ref[p]) ** 2)) / peak for p in range(4))
    assert err <= 1e-5, (kw, err)
im = WProjectionImager(setup.nx, setup.ny, setup.dl, wplanes=setup.wplanes, sampling=setup.sampling)
dev = torch.device("cuda")
t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)
grid_batch([(im, t(obs.uvw, torch.float32), t(obs.freq_over_c(0), torch.float32), t(obs.vis[0], torch.complex64),
             t(obs.weights[0], torch.float32), t(obs.flags[0], torch.int32))])
img = im.finalize().cpu().numpy()
assert np.sqrt(np.mean((img[0] - ref[0]) ** 2)) / peak <= 1e-5
torch.cuda.synchronize()
c, w = ctypes.c_int(0), ctypes.c_uint(99)
assert lib.mtb_bounds_status(ctypes.byref(c), ctypes.byref(w)) == L.MTB_OK
assert c.value == 1 and w.value == 0, (c.value, w.value)
print("checked ok")
''')
    assert r.returncode == 0 and "checked ok" in r.stdout, r.stdout + r.stderr
