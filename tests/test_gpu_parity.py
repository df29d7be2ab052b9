"""Parity of the sm_100a path (through the C ABI) with the FP64 oracle.

Tolerances (from the imaging path's accuracy contract): convolution functions
within 1e-6 absolute of the oracle (the w=0 kernel is normalised to 1 at its
centre); images within 1e-5 RMS relative to the image peak; integer decisions
of the preprocessing (w-plane, corner, oversampling offset, conv index,
compression, statistics) bit-exact.
"""
import ctypes

import numpy as np
import pytest
import torch

from mtb import synth
from mtb import _lib as L
from mtb.imager import WProjectionImager, _ptr, _stream

pytestmark = pytest.mark.gpu

KERNEL_TOL = 1e-6
IMAGE_RMS_TOL = 1e-5
GRID_TOL = 2e-6


def imager_for(setup, npol=4, **kw):
    return WProjectionImager(setup.nx, setup.ny, setup.dl, wplanes=setup.wplanes, sampling=setup.sampling,
                             npol=npol, trial_support=setup.trial_support, max_support=setup.max_support,
                             w_max=setup.w_max, **kw)


def partial_flags(obs, seed=0, frac=0.05):
    rng = np.random.default_rng(seed)
    for f in obs.flags:
        m = rng.random(f.shape) < frac
        f[m] = 1


def wide_case(nx=256, cell=200, s=4, rad=150, nw=16, seed=5):
    obs, setup = synth.small_config(seed=seed, n_ant=12, ntimes=60, nx=nx, cell_arcsec=cell, wplanes=nw,
                                    sampling=s, radius_m=rad, dec_deg=-88, flag_frac=0.1)
    setup.w_max = float(np.abs(obs.uvw[2] * obs.freq_over_c(0)).max())
    partial_flags(obs)
    return obs, setup


@pytest.fixture(scope="module")
def cfg1(oracle):
    obs, setup = synth.config1(seed=1)
    partial_flags(obs, seed=1)
    geo = oracle.geometry_for(setup)
    kern = oracle.wkernels(geo)
    img, g, n = oracle.image_channel(obs, 0, setup, kern, geo)
    return obs, setup, geo, kern, img, g, n


def run_gpu(obs, setup, npol=4, chunks=1, **kw):
    im = imager_for(setup, npol=npol, **kw)
    im.build_kernels()
    R = obs.nrec
    f = obs.freq_over_c(0)
    bounds = np.linspace(0, R, chunks + 1).astype(int)
    for a, b in zip(bounds[:-1], bounds[1:]):
        im.grid_chunk(obs.uvw[:, a:b], f[a:b], obs.vis[0][a:b, :npol], obs.weights[0][a:b, :npol],
                      obs.flags[0][a:b, :npol])
    img = im.finalize()
    torch.cuda.synchronize()
    return im, img.cpu().numpy()


def rel_rms(a, b):
    return np.sqrt(np.mean((a - b) ** 2)) / np.abs(b).max()


def test_kernel_table_parity(cfg1):
    obs, setup, geo, kern, *_ = cfg1
    im = imager_for(setup)
    k = im.build_kernels()
    assert np.array_equal(k.conv_info, kern["conv_info"])
    t = k.table.cpu().numpy()
    assert t.size == kern["table"].size
    assert np.abs(t - kern["table"]).max() <= KERNEL_TOL
    cs = k.conv_sums.cpu().numpy()
    assert np.abs(cs - kern["conv_sums"]).max() <= KERNEL_TOL * np.abs(kern["conv_sums"]).max()
    assert k.info.trial_support == geo["trial_support"] and k.info.T == geo["T"]
    assert k.info.w_sq_increment == pytest.approx(geo["w_inc"], rel=1e-15)


def preprocess_gpu(im, obs, npol=4):
    k = im.build_kernels()
    R = obs.nrec
    dev = im.device
    gp = im.grid_params(False)
    ws, nbytes = im._workspace(R, gp)
    uvw = torch.from_numpy(obs.uvw).to(dev)
    freq = torch.from_numpy(obs.freq_over_c(0)).to(dev)
    wts = torch.from_numpy(np.ascontiguousarray(obs.weights[0][:, :npol])).to(dev)
    flg = torch.from_numpy(np.ascontiguousarray(obs.flags[0][:, :npol])).to(dev)
    out = dict(loc=torch.empty((R, 4), dtype=torch.int32, device=dev),
               convidx=torch.empty(R, dtype=torch.int32, device=dev),
               togrid=torch.empty(R, dtype=torch.int32, device=dev),
               compress=torch.empty(R, dtype=torch.int32, device=dev),
               support=torch.empty(R, dtype=torch.int32, device=dev),
               imgmult=torch.empty(R, dtype=torch.float32, device=dev),
               convsum=torch.empty((npol, R), dtype=torch.float32, device=dev))
    L.check(im.lib.mtb_preprocess_uvw(ctypes.byref(gp), _ptr(k.d_conv_info), k.conv_info.ctypes.data_as(ctypes.c_void_p),
                                      _ptr(k.conv_sums), _ptr(uvw), _ptr(freq), _ptr(wts), _ptr(flg), R,
                                      _ptr(out["loc"]), _ptr(out["convidx"]), _ptr(out["togrid"]),
                                      _ptr(out["compress"]), _ptr(out["support"]), _ptr(out["imgmult"]),
                                      _ptr(out["convsum"]), _ptr(ws), nbytes, _stream()), "mtb_preprocess_uvw")
    torch.cuda.synchronize()
    return {kk: v.cpu().numpy() for kk, v in out.items()}


@pytest.mark.parametrize("case", ["cfg1", "wide"])
def test_preprocess_bit_exact(cfg1, oracle, case):
    if case == "cfg1":
        obs, setup, geo, kern, *_ = cfg1
    else:
        obs, setup = wide_case()
        geo = oracle.geometry_for(setup)
        kern = oracle.wkernels(geo)
    im = imager_for(setup)
    g = preprocess_gpu(im, obs)
    pre = oracle.preprocess(obs.uvw, obs.freq_over_c(0), obs.weights[0], obs.flags[0], geo, kern)
    for key in ("loc", "convidx", "togrid", "compress", "support", "imgmult"):
        assert np.array_equal(g[key], pre[key]), key
    assert np.abs(g["convsum"] - pre["convsum"]).max() <= 1e-6 * np.abs(pre["convsum"]).max()
    assert pre["togrid"].sum() > 0 and pre["compress"].sum() > 0


def test_config1_image_parity(cfg1):
    obs, setup, geo, kern, img_o, grid_o, norm_o = cfg1
    im, img = run_gpu(obs, setup)
    g = im.grid_sum().cpu().numpy()
    assert np.abs(g - grid_o).max() <= GRID_TOL * np.abs(grid_o).max()
    n = im.normalizer.cpu().numpy()
    assert np.allclose(n, norm_o, rtol=1e-6)
    # every Stokes plane, RMS relative to the Stokes I peak
    peak = np.abs(img_o[0]).max()
    for p in range(4):
        assert np.sqrt(np.mean((img[p] - img_o[p]) ** 2)) <= IMAGE_RMS_TOL * peak
    from oracle import oracle as O
    st = O.stats(O.preprocess(obs.uvw, obs.freq_over_c(0), obs.weights[0], obs.flags[0], geo, kern))
    assert im.statistics() == st


def test_chunked_equals_single(cfg1):
    obs, setup, *_ = cfg1
    a, ia = run_gpu(obs, setup, chunks=1)
    b, ib = run_gpu(obs, setup, chunks=5)
    ga, gb = a.grid_sum().cpu().numpy(), b.grid_sum().cpu().numpy()
    assert np.abs(ga - gb).max() <= GRID_TOL * np.abs(ga).max()
    assert rel_rms(ib[0], ia[0]) <= IMAGE_RMS_TOL
    # duplicates cannot be merged across a chunk boundary, so only the split
    # between gridded and compressed records may move, never their sum
    sa, sb = a.statistics(), b.statistics()
    assert sa["gridded_records"] + sa["compressed_records"] == sb["gridded_records"] + sb["compressed_records"]


# 37-record work items multiply the flushes per cell; the FP32 delta grid's
# rounding then nears the image bound, so that tuning runs with the FP64 delta
@pytest.mark.parametrize("tuning", [dict(tile=16), dict(tile=64), dict(support_bucket=3),
                                    dict(max_chunk=37, exact_delta=True),
                                    dict(merge=1), dict(merge=2), dict(merge=1, tile=16),
                                    dict(exact_delta=True),
                                    dict(gridder_threads=512), dict(gridder_threads=512, tile=16, max_chunk=256),
                                    dict(gridder=5), dict(gridder=5, tile=64),
                                    dict(gridder=7), dict(gridder=7, tile=64), dict(gridder=7, tile=16),
                                    dict(gridder=7, support_bucket=3), dict(gridder=7, exact_delta=True),
                                    dict(gridder=7, max_chunk=37, exact_delta=True),
                                    dict(gridder=8), dict(gridder=8, tile=16), dict(gridder=8, support_bucket=3),
                                    dict(gridder=8, exact_delta=True), dict(gridder=8, max_chunk=37, exact_delta=True)])
def test_tuning_does_not_change_result(cfg1, tuning):
    obs, setup, geo, kern, img_o, grid_o, norm_o = cfg1
    im, img = run_gpu(obs, setup, **tuning)
    g = im.grid_sum().cpu().numpy()
    assert np.abs(g - grid_o).max() <= GRID_TOL * np.abs(grid_o).max()
    assert rel_rms(img[0], img_o[0]) <= IMAGE_RMS_TOL


@pytest.mark.parametrize("kw", [dict(), dict(tile=64), dict(nx=320, s=3), dict(merge=1), dict(gridder=5),
                                dict(gridder=7), dict(nx=320, s=3, gridder=7), dict(gridder=8),
                                dict(nx=320, s=3, gridder=8),
                                ])
def test_large_supports(oracle, kw):
    """Supports up to 55 (and 105 with odd sampling): the direct gridders
    (block-staged, rolling-items, streaming with 4 and 8 slots per lane; one
    and several record streams), the shared-memory window variant, and
    support bands split across blocks."""
    tile = kw.pop("tile", 0)
    merge = kw.pop("merge", 0)
    gridder = kw.pop("gridder", 0)
    obs, setup = wide_case(**kw)
    geo = oracle.geometry_for(setup)
    kern = oracle.wkernels(geo)
    img_o, grid_o, norm_o = oracle.image_channel(obs, 0, setup, kern, geo)
    im, img = run_gpu(obs, setup, tile=tile, merge=merge, gridder=gridder)
    assert np.array_equal(im.kernels.conv_info, kern["conv_info"])
    assert np.abs(im.kernels.table.cpu().numpy() - kern["table"]).max() <= KERNEL_TOL
    g = im.grid_sum().cpu().numpy()
    assert np.abs(g - grid_o).max() <= GRID_TOL * np.abs(grid_o).max()
    assert rel_rms(img[0], img_o[0]) <= IMAGE_RMS_TOL


@pytest.mark.parametrize("npol", [1, 2])
def test_fewer_polarisations(oracle, npol):
    obs, setup = synth.small_config(seed=9, n_ant=10, ntimes=80, nx=128, flag_frac=0.1)
    obs.vis[0] = np.ascontiguousarray(obs.vis[0][:, :npol])
    obs.weights[0] = np.ascontiguousarray(obs.weights[0][:, :npol])
    obs.flags[0] = np.ascontiguousarray(obs.flags[0][:, :npol])
    img_o, grid_o, norm_o = oracle.image_channel(obs, 0, setup)
    im, img = run_gpu(obs, setup, npol=npol)
    g = im.grid_sum().cpu().numpy()
    assert np.abs(g - grid_o).max() <= GRID_TOL * np.abs(grid_o).max()
    assert rel_rms(img[0], img_o[0]) <= IMAGE_RMS_TOL


def test_circular_stokes(oracle):
    obs, setup = synth.small_config(seed=4, n_ant=10, ntimes=60, nx=96)
    geo = oracle.geometry_for(setup)
    _, grid_o, norm_o = oracle.image_channel(obs, 0, setup)
    img_o = oracle.finalize(grid_o, norm_o, geo, pol_type="circular")
    _, img = run_gpu(obs, setup, pol_type=L.MTB_POL_CIRCULAR)
    for p in range(4):
        assert np.sqrt(np.mean((img[p] - img_o[p]) ** 2)) <= IMAGE_RMS_TOL * np.abs(img_o[0]).max()


def test_empty_and_fully_rejected_chunks(oracle):
    obs, setup = synth.small_config(seed=2, n_ant=8, ntimes=40, nx=64)
    im = imager_for(setup)
    im.build_kernels()
    z = np.zeros((0, 4))
    im.grid_chunk(np.zeros((3, 0), np.float32), np.zeros(0, np.float32), z.astype(np.complex64),
                  z.astype(np.float32), z.astype(np.int32))
    R = obs.nrec
    im.grid_chunk(obs.uvw, obs.freq_over_c(0), obs.vis[0], obs.weights[0], np.ones((R, 4), np.int32))
    far = obs.uvw * 1e3
    im.grid_chunk(far, obs.freq_over_c(0), obs.vis[0], obs.weights[0], obs.flags[0])
    bad = obs.uvw.copy()
    bad[:, ::2] = np.nan
    bad[:, 1::2] = np.inf
    im.grid_chunk(bad, obs.freq_over_c(0), obs.vis[0], obs.weights[0], obs.flags[0])
    torch.cuda.synchronize()
    assert not im.grid.abs().sum().item()
    assert not im.normalizer.abs().sum().item()
    assert im.statistics()["gridded_records"] == 0


def test_compensated_merge_tracks_fp64(cfg1):
    """Accumulated over many chunks, the two-float grid stays at least as close
    to the FP64 grid as plain FP32 accumulation (within one chunk both
    accumulate identically, so only the cross-chunk merge can differ; the
    slack covers the unspecified order of the FP32 reductions)."""
    obs, setup, geo, kern, img_o, grid_o, norm_o = cfg1
    a, _ = run_gpu(obs, setup, chunks=16, compensated=True)
    b, _ = run_gpu(obs, setup, chunks=16, compensated=False)
    ea = np.sqrt(np.mean(np.abs(a.grid_sum().cpu().numpy() - grid_o) ** 2))
    eb = np.sqrt(np.mean(np.abs(b.grid.cpu().numpy() - grid_o) ** 2))
    assert ea <= eb * 1.02
    assert np.abs(a.grid_sum().cpu().numpy() - grid_o).max() <= GRID_TOL * np.abs(grid_o).max()


def test_status_codes(oracle):
    obs, setup = synth.small_config(seed=2, n_ant=6, ntimes=10, nx=64)
    with pytest.raises(L.MtbError) as e:
        WProjectionImager(64, 64, setup.dl, wplanes=4, sampling=4, trial_support=32).build_kernels()
    assert e.value.status == 1
    im = imager_for(setup)
    with pytest.raises(ValueError):
        im.grid_chunk(obs.uvw[:, :5], obs.freq_over_c(0)[:4], obs.vis[0][:4], obs.weights[0][:4], obs.flags[0][:4])
    lib = L.load()
    gp = im.grid_params(True)
    gp.npol = 3
    n = ctypes.c_size_t(0)
    ci = im.build_kernels().conv_info.ctypes.data_as(ctypes.c_void_p)
    assert lib.mtb_grid_workspace_size(ctypes.byref(gp), ci, 10, ctypes.byref(n)) == 2
    im2 = imager_for(setup)
    k = im2.build_kernels()
    gp = im2.grid_params(True)
    ws = torch.empty(16, dtype=torch.uint8, device="cuda")
    R = obs.nrec
    st = lib.mtb_grid(ctypes.byref(gp), _ptr(k.table), _ptr(k.d_conv_info), k.conv_info.ctypes.data_as(ctypes.c_void_p),
                      _ptr(k.conv_sums), _ptr(torch.zeros((3, R), device="cuda")), _ptr(torch.zeros(R, device="cuda")),
                      _ptr(torch.zeros((R, 4), dtype=torch.complex64, device="cuda")),
                      _ptr(torch.zeros((R, 4), device="cuda")), _ptr(torch.zeros((R, 4), dtype=torch.int32, device="cuda")),
                      R, _ptr(im2.grid), None, _ptr(im2.normalizer), None, _ptr(ws), 16, _stream())
    assert st == 3   # workspace too small


@pytest.mark.parametrize("ny,gridder", [(96, 0), (160, 0), (160, 8), (96, 3)])
def test_rectangular_image_parity(oracle, ny, gridder):
    """nx != ny (ConfigurationManager.cpp:170-202 sizes the axes
    independently): Δv = 1/(Δm·ny), rows of the grid and image indexed by ny
    and columns by nx in the preprocessing, the gridders, the inverse FFT, the
    Stokes conversion and the taper and sinc corrections.  Grid and every
    Stokes plane against the FP64 oracle, statistics exact."""
    import dataclasses
    obs, setup = synth.small_config(seed=3, n_ant=10, ntimes=60, nx=128, cell_arcsec=20, flag_frac=0.1)
    setup = dataclasses.replace(setup, ny=ny)
    geo = oracle.geometry_for(setup)
    kern = oracle.wkernels(geo)
    img_o, grid_o, norm_o = oracle.image_channel(obs, 0, setup, kern, geo)
    im, img = run_gpu(obs, setup, gridder=gridder)
    assert img.shape == img_o.shape == (4, ny, 128)
    g = im.grid_sum().cpu().numpy()
    assert g.shape == grid_o.shape
    assert np.abs(g - grid_o).max() <= GRID_TOL * np.abs(grid_o).max()
    peak = np.abs(img_o[0]).max()
    for p in range(4):
        assert np.sqrt(np.mean((img[p] - img_o[p]) ** 2)) <= IMAGE_RMS_TOL * peak, p
    st = oracle.stats(oracle.preprocess(obs.uvw, obs.freq_over_c(0), obs.weights[0], obs.flags[0], geo, kern))
    assert im.statistics() == st
