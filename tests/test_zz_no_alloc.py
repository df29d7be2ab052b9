"""mtb_preprocess_uvw_noalloc (fixed device scratch, no workspace) against
mtb_preprocess_uvw (caller workspace) on the same inputs.

The entry point serves callers that must not allocate device memory: code
running inside an allocator or memory-pool callback (where cudaMalloc would
re-enter the allocator), a framework that partitions the device up front and
hands plugins only the buffers it owns, a plugin whose host forbids
allocation.  Its scratch is a fixed array in the library's device image, so
it allocates nothing and refuses chunks above its stated capacity.

The file name sorts last so the fixed scratch is exercised after every other
test has used the library; two different chunks run back to back so a value
left in the scratch by the first call would show up in the second.
"""
import ctypes

import numpy as np
import pytest
import torch

from mtb import _lib as L
from mtb.imager import _ptr, _stream

from test_gpu_parity import imager_for, preprocess_gpu, wide_case

pytestmark = pytest.mark.gpu

KEYS = ("loc", "convidx", "togrid", "compress", "support", "imgmult")
CONVSUM_TOL = 1e-6


def preprocess_noalloc(im, obs, npol=4):
    k = im.build_kernels()
    R = obs.nrec
    dev = im.device
    gp = im.grid_params(False)
    uvw = torch.from_numpy(obs.uvw).to(dev)
    freq = torch.from_numpy(obs.freq_over_c(0)).to(dev)
    wts = torch.from_numpy(np.ascontiguousarray(obs.weights[0][:, :npol])).to(dev)
    flg = torch.from_numpy(np.ascontiguousarray(obs.flags[0][:, :npol])).to(dev)
    # outputs start as garbage: the entry point must write every element
    out = dict(loc=torch.full((R, 4), -7, dtype=torch.int32, device=dev),
               convidx=torch.full((R,), -7, dtype=torch.int32, device=dev),
               togrid=torch.full((R,), -7, dtype=torch.int32, device=dev),
               compress=torch.full((R,), -7, dtype=torch.int32, device=dev),
               support=torch.full((R,), -7, dtype=torch.int32, device=dev),
               imgmult=torch.full((R,), 7.0, dtype=torch.float32, device=dev),
               convsum=torch.full((npol, R), 7.0, dtype=torch.float32, device=dev))
    L.check(im.lib.mtb_preprocess_uvw_noalloc(
        ctypes.byref(gp), _ptr(k.d_conv_info), k.conv_info.ctypes.data_as(ctypes.c_void_p), _ptr(k.conv_sums),
        _ptr(uvw), _ptr(freq), _ptr(wts), _ptr(flg), R, _ptr(out["loc"]), _ptr(out["convidx"]), _ptr(out["togrid"]),
        _ptr(out["compress"]), _ptr(out["support"]), _ptr(out["imgmult"]), _ptr(out["convsum"]), _stream()),
        "mtb_preprocess_uvw_noalloc")
    torch.cuda.synchronize()
    return {kk: v.cpu().numpy() for kk, v in out.items()}


def test_noalloc_matches_workspace_entry_point_twice():
    cases = [wide_case(seed=5), wide_case(nx=320, cell=150, s=3, seed=9)]
    for obs, setup in cases:
        im = imager_for(setup)
        ref = preprocess_gpu(im, obs)
        got = preprocess_noalloc(im, obs)
        for key in KEYS:
            assert np.array_equal(got[key], ref[key]), key
        assert np.abs(got["convsum"] - ref["convsum"]).max() <= CONVSUM_TOL * np.abs(ref["convsum"]).max()
        assert ref["togrid"].sum() > 0 and ref["compress"].sum() > 0


def test_noalloc_refuses_more_than_capacity():
    obs, setup = wide_case()
    im = imager_for(setup)
    k = im.build_kernels()
    gp = im.grid_params(False)
    cap = im.lib.mtb_preprocess_uvw_noalloc_capacity()
    assert cap == 1 << 20
    dummy = torch.zeros(16, dtype=torch.int32, device=im.device)
    d = _ptr(dummy)
    rc = im.lib.mtb_preprocess_uvw_noalloc(ctypes.byref(gp), d, k.conv_info.ctypes.data_as(ctypes.c_void_p), d, d,
                                           d, d, d, cap + 1, d, d, d, d, d, d, d, _stream())
    assert rc == L.MTB_ERR_TOO_LARGE
    assert b"capacity" in im.lib.mtb_status_string(rc)


def test_noalloc_matches_oracle(oracle):
    """The no-alloc entry point against the FP64 oracle directly: the six
    integer outputs bit for bit, ConvSums·weight to 1e-6 of its peak."""
    obs, setup = wide_case(nx=320, cell=150, s=3, seed=11)
    geo = oracle.geometry_for(setup)
    kern = oracle.wkernels(geo)
    im = imager_for(setup)
    got = preprocess_noalloc(im, obs)
    pre = oracle.preprocess(obs.uvw, obs.freq_over_c(0), obs.weights[0], obs.flags[0], geo, kern)
    for key in KEYS:
        assert np.array_equal(got[key], pre[key]), key
    assert np.abs(got["convsum"] - pre["convsum"]).max() <= CONVSUM_TOL * np.abs(pre["convsum"]).max()
