"""Golden fixtures produced by mt-imager itself (tests/golden/make_golden.py:
the reference's own operator sources compiled for sm_100a and run through the
WImager operator graph, WImager.cpp:167-234).

CPU tests pin the FP64 oracle to them; GPU tests check the sm_100a path
against them through the C ABI.  Tolerances: the seven PreProcessUVW outputs
bit-exact (the reference computes them in FP32 and the oracle and the product
in FP64; the fixtures contain no record whose decision falls on an FP32
rounding boundary); the grid within 2e-6 of its peak (the reference
accumulates in FP32 with atomics in an unspecified order).
"""
import ctypes
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "grid_*.npz")))
GRID_TOL = 2e-6
PRE_KEYS = [("loc", "gridding_data"), ("convidx", "conv_index"), ("togrid", "to_grid"),
            ("compress", "to_compress"), ("support", "support"), ("imgmult", "take_conjugate")]


def load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def geometry(O, c):
    return O.kernel_geometry(int(c["nx"]), int(c["ny"]), float(c["dl"]), float(c["dl"]), int(c["wplanes"]),
                             int(c["sampling"]), int(c["trial_support"]), 0, float(c["w_max"]))


def chunks(c):
    R = c["freq"].size
    b = np.linspace(0, R, int(c["chunks"]) + 1).astype(int)
    return list(zip(b[:-1], b[1:]))


def sl(x, a, b):
    return np.ascontiguousarray(x[..., a:b]) if x.ndim == 2 and x.shape[0] == 3 else np.ascontiguousarray(x[a:b])


def test_fixtures_present():
    assert len(FIXTURES) >= 3


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p))
def test_oracle_matches_reference(oracle, path):
    c = load(path)
    geo = geometry(oracle, c)
    assert geo["w_inc"] == pytest.approx(float(c["w_inc"]), rel=1e-12)
    kern = dict(table=c["table"].astype(np.complex128), conv_info=c["conv_info"],
                conv_sums=c["conv_sums"].astype(np.float64))
    g = n = None
    for k, (a, b) in enumerate(chunks(c)):
        g, n, pre = oracle.grid_chunk(sl(c["uvw"], a, b), sl(c["freq"], a, b), sl(c["vis"], a, b),
                                      sl(c["weights"], a, b), sl(c["flags"], a, b), geo, kern, g, n)
        for mine, ref in PRE_KEYS:
            assert np.array_equal(pre[mine], c["ref_%s_%d" % (ref, k)]), (mine, k)
        cs = c["ref_conv_sum_%d" % k]
        assert np.array_equal(pre["convsum"].astype(np.float32), cs)
        assert pre["togrid"].sum() > 0 and pre["compress"].sum() > 0
    rg = c["ref_grid"].astype(np.complex128)
    assert np.abs(g - rg).max() <= GRID_TOL * np.abs(rg).max()


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p))
def test_gpu_matches_reference(path):
    import torch
    from mtb import _lib as L
    from mtb.imager import WProjectionImager, KernelTable, _ptr, _stream

    c = load(path)
    P, nx, ny = int(c["npol"]), int(c["nx"]), int(c["ny"])
    dev = torch.device("cuda")
    im = WProjectionImager(nx, ny, float(c["dl"]), wplanes=int(c["wplanes"]), sampling=int(c["sampling"]),
                           npol=P, trial_support=int(c["trial_support"]), w_max=float(c["w_max"]))
    info = L.WKernelInfo()
    L.check(im.lib.mtb_wkernel_query(ctypes.byref(im.params), ctypes.byref(info)), "mtb_wkernel_query")
    # grid with the fixture's own kernel table (the reference gridded with it)
    im.kernels = KernelTable(table=torch.from_numpy(c["table"]).to(dev),
                             conv_info=np.ascontiguousarray(c["conv_info"]),
                             d_conv_info=torch.from_numpy(np.ascontiguousarray(c["conv_info"])).to(dev),
                             conv_sums=torch.from_numpy(c["conv_sums"]).to(dev), info=info, params=im.params)
    for k, (a, b) in enumerate(chunks(c)):
        R = int(b - a)
        args = [torch.from_numpy(sl(c[key], a, b)).to(dev) for key in ("uvw", "freq", "weights", "flags")]
        out = dict(loc=torch.empty((R, 4), dtype=torch.int32, device=dev),
                   convidx=torch.empty(R, dtype=torch.int32, device=dev),
                   togrid=torch.empty(R, dtype=torch.int32, device=dev),
                   compress=torch.empty(R, dtype=torch.int32, device=dev),
                   support=torch.empty(R, dtype=torch.int32, device=dev),
                   imgmult=torch.empty(R, dtype=torch.float32, device=dev),
                   convsum=torch.empty((P, R), dtype=torch.float32, device=dev))
        gp = im.grid_params(False)
        ws, nbytes = im._workspace(R, gp)
        kt = im.kernels
        L.check(im.lib.mtb_preprocess_uvw(ctypes.byref(gp), _ptr(kt.d_conv_info),
                                          kt.conv_info.ctypes.data_as(ctypes.c_void_p), _ptr(kt.conv_sums),
                                          *[_ptr(t) for t in args], R, *[_ptr(out[key]) for key in out],
                                          _ptr(ws), nbytes, _stream()), "mtb_preprocess_uvw")
        torch.cuda.synchronize()
        for mine, ref in PRE_KEYS:
            assert np.array_equal(out[mine].cpu().numpy(), c["ref_%s_%d" % (ref, k)]), (mine, k)
        assert np.array_equal(out["convsum"].cpu().numpy(), c["ref_conv_sum_%d" % k])
        im.grid_chunk(sl(c["uvw"], a, b), sl(c["freq"], a, b), sl(c["vis"], a, b), sl(c["weights"], a, b),
                      sl(c["flags"], a, b))
    torch.cuda.synchronize()
    g = im.grid_sum().cpu().numpy().astype(np.complex128)
    rg = c["ref_grid"].astype(np.complex128)
    assert np.abs(g - rg).max() <= GRID_TOL * np.abs(rg).max()


# ---------------------------------------------------------------- images --
IMAGES = sorted(glob.glob(os.path.join(HERE, "golden", "image_*.npz")))
# The reference finalises in FP32 (cuFFT C2C, float corrections); the taper
# correction divides by grdsf^2, which amplifies FP32 rounding towards the
# image edges.  Inside the central half (correction < 4x) the images agree to
# FP32 rounding; over the whole image to the reference's own FP32 error.
IMAGE_CENTRE_RMS = 1e-6
IMAGE_CENTRE_MAX = 2e-6
IMAGE_FULL_RMS = 2e-5


def image_case(path):
    name = os.path.basename(path)[len("image_"):-len(".npz")]
    return load(os.path.join(HERE, "golden", "grid_%s.npz" % name)), load(path)


def check_image(mine, ref):
    n = ref.shape[1]
    q = n // 4
    peak = np.abs(ref[0]).max()
    d = mine.astype(np.float64) - ref
    assert np.sqrt(np.mean(d[:, q:-q, q:-q] ** 2)) <= IMAGE_CENTRE_RMS * peak
    assert np.abs(d[:, q:-q, q:-q]).max() <= IMAGE_CENTRE_MAX * peak
    assert np.sqrt(np.mean(d ** 2)) <= IMAGE_FULL_RMS * peak


def test_image_fixtures_present():
    assert len(IMAGES) >= 3


@pytest.mark.parametrize("path", IMAGES, ids=lambda p: os.path.basename(p))
def test_oracle_finalize_matches_reference(oracle, path):
    c, im = image_case(path)
    geo = geometry(oracle, c)
    pol = "circular" if int(im["pol_type"]) == 1 else "linear"
    mine = oracle.finalize(c["ref_grid"].astype(np.complex128), im["normalizer"].astype(np.float64), geo, pol)
    check_image(mine, im["ref_image"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", IMAGES, ids=lambda p: os.path.basename(p))
def test_gpu_finalize_matches_reference(path):
    import torch
    from mtb import _lib as L
    from mtb.imager import WProjectionImager

    c, im = image_case(path)
    P = int(c["npol"])
    pol = L.MTB_POL_CIRCULAR if int(im["pol_type"]) == 1 else L.MTB_POL_LINEAR
    w = WProjectionImager(int(c["nx"]), int(c["ny"]), float(c["dl"]), wplanes=int(c["wplanes"]),
                          sampling=int(c["sampling"]), npol=P, pol_type=pol, compensated=False)
    w.grid.copy_(torch.from_numpy(c["ref_grid"]))
    w.normalizer.copy_(torch.from_numpy(im["normalizer"]))
    img = w.finalize().cpu().numpy()
    torch.cuda.synchronize()
    check_image(img, im["ref_image"])


# --------------------------------------------------------------- w-kernels --
WKERNELS = sorted(glob.glob(os.path.join(HERE, "golden", "wkernels_*.npz")))
# The reference builds the kernels in FP32 (float w, float w-screen phase,
# cuFFT C2C); supports and the table layout must agree exactly, values to the
# convolution-function bound.
KERNEL_TOL = 1e-6
CONV_SUM_RTOL = 1e-5


def test_wkernel_fixtures_present():
    assert len(WKERNELS) >= 2


@pytest.mark.parametrize("path", WKERNELS, ids=lambda p: os.path.basename(p))
def test_oracle_wkernels_match_reference(oracle, path):
    z = load(path)
    nx, dl = int(z["nx"]), float(z["dl"])
    geo = oracle.kernel_geometry(nx, nx, dl, dl, int(z["wplanes"]), int(z["sampling"]))
    k = oracle.wkernels(geo)
    assert np.array_equal(k["conv_info"], z["ref_conv_info"])
    assert np.abs(k["table"] - z["ref_table"].astype(np.complex128)).max() <= KERNEL_TOL
    assert np.abs(k["conv_sums"] - z["ref_conv_sums"]).max() <= CONV_SUM_RTOL * np.abs(z["ref_conv_sums"]).max()
    assert k["divisor"].real == pytest.approx(float(z["ref_divisor"][0]), rel=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("path", WKERNELS, ids=lambda p: os.path.basename(p))
def test_gpu_wkernels_match_reference(path):
    from mtb.imager import build_wkernels, wkernel_params

    z = load(path)
    nx, dl = int(z["nx"]), float(z["dl"])
    k = build_wkernels(wkernel_params(nx, nx, dl, dl, int(z["wplanes"]), int(z["sampling"])))
    assert np.array_equal(k.conv_info, z["ref_conv_info"])
    t = k.table.cpu().numpy().astype(np.complex128)
    assert np.abs(t - z["ref_table"]).max() <= KERNEL_TOL
    cs = k.conv_sums.cpu().numpy()
    assert np.abs(cs - z["ref_conv_sums"]).max() <= CONV_SUM_RTOL * np.abs(z["ref_conv_sums"]).max()
