"""Known-answer tests that pin the FP64 oracle (CPU only).

mt-imager ships no tests or golden vectors, so the oracle is pinned by
properties the reference's method must have: DC normalisation of the w=0
kernel (WProjectionConvFunction.cpp:208-219), the preprocessing decisions of
WProjPreProcessUVW.cu on hand-built records, the direct FP64 DFT, chunk
invariance and the conjugation of w<0 records.
"""
import math

import numpy as np
import pytest

from mtb import synth


def small_geo(O, nx=64, cell=20.0, nw=8, s=4, **kw):
    dl = cell * synth.ARCSEC
    return O.kernel_geometry(nx, nx, dl, dl, nw, s, **kw)


def test_grdsf_shape(oracle):
    g = oracle.lib().orc_grdsf
    assert abs(g(0.0) - 1.0) < 1e-6
    vals = [g(x / 20) for x in range(21)]
    assert all(a >= b for a, b in zip(vals, vals[1:]))   # monotone fall-off to the edge
    t = oracle.taper_lm(33)
    assert np.allclose(t, t[::-1, :]) and np.allclose(t, t.T)


def test_kernel_geometry_reference_rules(oracle):
    geo = small_geo(oracle, nx=256, cell=2.0, nw=32, s=8)
    assert geo["trial_support"] == 33          # 256/8 = 32 forced odd
    assert geo["support_cap"] == 31
    assert geo["T"] == 9                        # even sampling -> s+1 offsets
    assert math.isclose(geo["w_max"], 0.25 / (2.0 * synth.ARCSEC))
    assert math.isclose(geo["w_inc"], geo["w_max"] / 31 ** 2)
    assert oracle.kernel_geometry(64, 64, 1e-4, 1e-4, 4, 3)["T"] == 3


@pytest.mark.parametrize("s", [3, 4, 8])
def test_w0_kernel_dc_is_one(oracle, s):
    geo = small_geo(oracle, s=s)
    k = oracle.wkernels(geo)
    S0 = int(k["conv_info"][0, 0])
    T = geo["T"]
    c = k["table"][: T * T * S0 * S0].reshape(T, T, S0, S0)
    centre = c[s // 2, s // 2, S0 // 2, S0 // 2]
    assert abs(centre - 1.0) < 1e-12
    # supports are odd, within the cap, and the table is laid out contiguously
    sup = k["supports"]
    assert np.all(sup % 2 == 1) and np.all(sup <= geo["support_cap"])
    offs = np.concatenate([[0], np.cumsum(T * T * sup.astype(np.int64) ** 2)[:-1]])
    assert np.array_equal(k["conv_info"][:, 1], offs)
    assert k["table"].size == int((T * T * sup.astype(np.int64) ** 2).sum())
    # ConvSums are the real-part sums of each sub-kernel
    sub = k["table"][offs[-1]:].reshape(T * T, -1)
    assert np.allclose(k["conv_sums"][-1], sub.real.sum(axis=1))


def _one_record(oracle, geo, kern, u, v, w, flags=(0, 0, 0, 0), freq=None):
    lam = 0.2
    f = np.float32(1.0 / lam) if freq is None else np.float32(freq)
    uvw = np.array([[u * lam], [v * lam], [w * lam]], np.float32)
    return oracle.preprocess(uvw, np.array([f], np.float32), np.ones((1, 4), np.float32),
                             np.array([flags], np.int32), geo, kern)


def test_preprocess_known_answers(oracle):
    geo = small_geo(oracle)
    kern = oracle.wkernels(geo)
    S0 = int(kern["conv_info"][0, 0])
    n2 = geo["nx"] // 2
    # u = v = w = 0: centre cell, centre offset, plane 0
    p = _one_record(oracle, geo, kern, 0.0, 0.0, 0.0)
    assert p["togrid"][0] == 1 and p["plane"][0] == 0 and p["support"][0] == S0
    assert p["offx"][0] == geo["sampling"] // 2 and p["offy"][0] == geo["sampling"] // 2
    assert p["loc"][0, 0] == n2 - S0 // 2
    assert p["loc"][0, 1] == (n2 - S0 // 2) * geo["nx"] + n2 - S0 // 2
    assert p["imgmult"][0] == 1.0
    # w < 0: u, v negated and imaginary multiplier -1
    du = geo["du"]
    p1 = _one_record(oracle, geo, kern, 3.25 * du, -2.0 * du, -10.0)
    p2 = _one_record(oracle, geo, kern, -3.25 * du, 2.0 * du, 10.0)
    assert p1["imgmult"][0] == -1.0 and p2["imgmult"][0] == 1.0
    for key in ("loc", "convidx", "support", "plane", "offx", "offy"):
        assert np.array_equal(p1[key], p2[key])
    # fractional position maps to the oversampling offset round((loc-pos)*s)+s/2
    p = _one_record(oracle, geo, kern, 3.25 * du, 0.0, 0.0)
    assert p["offx"][0] == int(round((3 - 3.25) * geo["sampling"])) + geo["sampling"] // 2
    # all pols flagged -> not gridded; partial flag -> gridded, that pol's convsum 0
    assert _one_record(oracle, geo, kern, 0, 0, 0, flags=(1, 1, 1, 1))["togrid"][0] == 0
    p = _one_record(oracle, geo, kern, 0, 0, 0, flags=(0, 1, 0, 0))
    assert p["togrid"][0] == 1 and p["convsum"][1, 0] == 0.0 and p["convsum"][0, 0] > 0
    # outside the grid -> rejected, all outputs zero
    p = _one_record(oracle, geo, kern, (n2 - 1) * du, 0.0, 0.0)
    assert p["togrid"][0] == 0 and p["support"][0] == 0 and not p["loc"].any()
    # non-finite coordinates are rejected
    p = _one_record(oracle, geo, kern, float("nan"), 0.0, 0.0)
    assert p["togrid"][0] == 0


def test_compression_semantics(oracle):
    geo = small_geo(oracle)
    kern = oracle.wkernels(geo)
    lam = 0.2
    du = geo["du"]
    us = [1.0, 1.0, 1.0, 5.0, 5.0, -80.0, 5.0]      # record 5 is outside the grid
    R = len(us)
    uvw = np.zeros((3, R), np.float32)
    uvw[0] = np.array(us) * du * lam
    freq = np.full(R, 1.0 / lam, np.float32)
    flags = np.zeros((R, 4), np.int32)
    pre = oracle.preprocess(uvw, freq, np.ones((R, 4), np.float32), flags, geo, kern)
    assert list(pre["compress"]) == [0, 1, 1, 0, 1, 0, 0]
    assert list(pre["togrid"]) == [1, 0, 0, 1, 0, 0, 1]
    vis = (np.arange(R * 4).reshape(R, 4) + 1j).astype(np.complex64)
    cv = oracle.compress_vis(pre, vis, np.ones((R, 4), np.float32), flags)
    assert np.allclose(cv[0], vis[0] + vis[1] + vis[2])
    assert np.allclose(cv[3], vis[3] + vis[4])
    assert np.allclose(cv[6], vis[6])
    st = oracle.stats(pre)
    assert st["gridded_records"] == 3 and st["compressed_records"] == 3


def test_point_source_at_centre_matches_dft(oracle):
    obs, setup = synth.small_config(seed=3, n_ant=10, ntimes=60, nx=128, cell_arcsec=20, flag_frac=0.0)
    src = np.array([[0.0, 0.0, 1.0, 0.0, 0.0, 0.0]])
    obs.vis[0] = synth.predict_vis(obs.uvw.astype(np.float64), obs.freqs_hz[0], src).astype(np.complex64)
    img, _, _ = oracle.image_channel(obs, 0, setup)
    d = oracle.dft_image(obs, 0, setup)
    c = (127 - 64, 64)
    assert abs(d[0][c] - 1.0) < 1e-9
    assert abs(img[0][c] - 1.0) < 5e-3          # method error of the reference's kernels
    assert np.unravel_index(np.argmax(img[0]), img[0].shape) == c
    assert np.sqrt(np.mean((img[0] - d[0]) ** 2)) < 0.02


def test_w_projection_corrects_w_term(oracle):
    """With many w-planes the off-axis source is imaged closer to the DFT than
    with one plane (no w correction)."""
    errs = []
    for nw in (1, 16):
        obs, setup = synth.small_config(seed=5, n_ant=12, ntimes=80, nx=128, cell_arcsec=120, wplanes=nw,
                                        radius_m=80, flag_frac=0.0, dec_deg=-80)
        setup.w_max = float(np.abs(obs.uvw[2] * obs.freq_over_c(0)).max())
        dl = setup.dl
        src = np.array([[30 * dl, -25 * dl, 1.0, 0, 0, 0]])
        obs.vis[0] = synth.predict_vis(obs.uvw.astype(np.float64), obs.freqs_hz[0], src).astype(np.complex64)
        img, _, _ = oracle.image_channel(obs, 0, setup)
        d = oracle.dft_image(obs, 0, setup)
        errs.append(np.sqrt(np.mean((img[0] - d[0]) ** 2)))
        if nw > 1:
            assert np.unravel_index(np.argmax(img[0]), img[0].shape) == (127 - (64 - 25), 64 + 30)
    assert errs[1] < 0.8 * errs[0]


def test_chunk_invariance(oracle):
    obs, setup = synth.small_config(seed=7, n_ant=8, ntimes=50, nx=64, flag_frac=0.2)
    a, ga, na = oracle.image_channel(obs, 0, setup)
    b, gb, nb = oracle.image_channel(obs, 0, setup, chunk=97)
    # chunk boundaries can only split duplicate runs; the grid is linear in records
    assert np.allclose(na, nb, rtol=1e-12)
    assert np.abs(ga - gb).max() <= 1e-9 * np.abs(ga).max()
    assert np.abs(a - b).max() <= 1e-9 * np.abs(a).max()


def test_hermitian_mirror_grids_identically(oracle):
    """A visibility measured on (u, v, w) equals the conjugate of the one on
    (-u, -v, -w).  PreProcessUVW folds every w<0 record onto -uvw with its
    imaginary part negated (WProjPreProcessUVW.cu:160-175), so a chunk and
    its mirror (uvw negated, visibilities conjugated) must give the same
    decisions, the same grid and the same normaliser, bit for bit."""
    obs, setup = synth.small_config(seed=11, n_ant=8, ntimes=40, nx=64, wplanes=4, flag_frac=0.2)
    keep = obs.uvw[2] != 0                     # w = 0 exactly is not folded (w < 0 is false for -0)
    uvw = np.ascontiguousarray(obs.uvw[:, keep])
    f = obs.freq_over_c(0)[keep]
    vis, wts, flg = obs.vis[0][keep], obs.weights[0][keep], obs.flags[0][keep]
    geo = oracle.geometry_for(setup)
    kern = oracle.wkernels(geo)
    g1, n1, p1 = oracle.grid_chunk(uvw, f, vis, wts, flg, geo, kern)
    g2, n2, p2 = oracle.grid_chunk(-uvw, f, np.conj(vis), wts, flg, geo, kern)
    assert p1["togrid"].sum() > 0 and (p1["imgmult"] == -1).any() and (p1["imgmult"] == 1).any()
    for key in ("loc", "convidx", "togrid", "compress", "support", "plane", "offx", "offy"):
        assert np.array_equal(p1[key], p2[key]), key
    used = (p1["togrid"] | p1["compress"]) == 1      # a rejected record's multiplier is not used
    assert np.array_equal(p1["imgmult"][used], -p2["imgmult"][used])
    assert np.array_equal(n1, n2)
    assert np.array_equal(g1, g2)


def test_odd_and_even_sampling_layout(oracle):
    for s in (3, 5, 4):
        geo = small_geo(oracle, s=s, nw=2)
        k = oracle.wkernels(geo)
        T = geo["T"]
        assert T == (s if s % 2 else s + 1)
        # every record offset maps inside the table
        obs, setup = synth.small_config(seed=2, n_ant=6, ntimes=30, nx=64, wplanes=2, sampling=s)
        pre = oracle.preprocess(obs.uvw, obs.freq_over_c(0), obs.weights[0], obs.flags[0], geo, k)
        g = pre["togrid"] == 1
        assert np.all(pre["offx"][g] < T) and np.all(pre["offy"][g] < T) and np.all(pre["offx"][g] >= 0)
        end = pre["convidx"][g] + pre["support"][g] ** 2
        assert np.all(end <= k["table"].size)


@pytest.mark.parametrize("ny", [96, 160])
def test_rectangular_image_places_source(oracle, ny):
    """image.nx and image.ny are independent (ConfigurationManager.cpp:170-202):
    Δv = 1/(Δm·ny), the taper correction of each axis uses its own size and
    the Stokes rows are flipped over ny.  An off-centre point source lands on
    the pixel the FP64 DFT puts it on."""
    import dataclasses
    obs, setup = synth.small_config(seed=3, n_ant=10, ntimes=60, nx=128, cell_arcsec=20, flag_frac=0.0)
    setup = dataclasses.replace(setup, ny=ny)
    dl = setup.dl
    src = np.array([[12 * dl, -7 * dl, 1.0, 0.0, 0.0, 0.0]])
    obs.vis[0] = synth.predict_vis(obs.uvw.astype(np.float64), obs.freqs_hz[0], src).astype(np.complex64)
    img, _, _ = oracle.image_channel(obs, 0, setup)
    d = oracle.dft_image(obs, 0, setup)
    assert img.shape == d.shape == (4, ny, 128)
    pk = (ny - 1 - (ny // 2 - 7), 64 + 12)
    assert np.unravel_index(np.argmax(d[0]), d[0].shape) == pk
    assert np.unravel_index(np.argmax(img[0]), img[0].shape) == pk
    assert abs(img[0][pk] - d[0][pk]) < 0.05        # method error of the reference's kernels
    assert np.sqrt(np.mean((img[0] - d[0]) ** 2)) < 0.02


@pytest.mark.parametrize("nx,cell,nw,s,st,ms", [(4096, 2.4, 128, 8, 67, 65), (512, 6.0, 16, 3, 0, 0)])
def test_kernel_table_symmetries(oracle, nx, cell, nw, s, st, ms):
    """Size-independent properties of the kernel tables, the first case at the
    mid-size geometry (4096^2, 128 w-planes, oversampling 8, trial support 67).
    The taper x w-screen depends on l^2 + m^2 only (WProjPreFFTconvFunc.cu:
    34-105), so every plane's oversampled kernel is unchanged by uv -> -uv and
    by u <-> v; supports are odd, within the cap and grow with |w|; the w = 0
    plane has DC 1; ConvSums are the sub-kernels' real sums."""
    dl = cell * synth.ARCSEC
    geo = oracle.kernel_geometry(nx, nx, dl, dl, nw, s, st, ms)
    k = oracle.wkernels(geo)
    T = geo["T"]
    sup = k["supports"]
    assert np.all(sup % 2 == 1) and np.all(sup <= geo["support_cap"]) and np.all(np.diff(sup) >= 0)
    assert sup[-1] > sup[0]
    for pl in range(nw):
        S, o = int(sup[pl]), int(k["conv_info"][pl, 1])
        c = k["table"][o:o + T * T * S * S].reshape(T, T, S, S)
        pk = np.abs(c).max()
        assert np.abs(c - c[::-1, ::-1, ::-1, ::-1]).max() <= 1e-13 * pk
        assert np.abs(c - c.transpose(1, 0, 3, 2)).max() <= 1e-13 * pk
        assert np.allclose(k["conv_sums"][pl], c.real.reshape(T * T, -1).sum(axis=1), rtol=0, atol=1e-12)
    S0 = int(sup[0])
    c0 = k["table"][:T * T * S0 * S0].reshape(T, T, S0, S0)
    assert abs(c0[s // 2, s // 2, S0 // 2, S0 // 2] - 1.0) < 1e-12
    # w = 0: the transform of a real, even taper is real
    assert np.abs(c0.imag).max() <= 1e-12 * np.abs(c0).max()


def test_w_negative_cross_hands_are_not_exchanged(oracle):
    """The reference conjugates a w<0 record polarisation by polarisation
    (imaginary part x -1, common.hcu:80-104, after WProjPreProcessUVW.cu:
    170-175) without exchanging XY and YX.  For a real sky conj(XY(u)) is
    YX(-u), so such a record adds its Stokes V with the opposite sign (I, Q
    and U are symmetric in the cross hands).  The oracle, and the path it
    pins, keep this: V at a polarised source is V * (N+ - N-) / N of the
    gridded records, and it is recovered in full when every record has w >= 0."""
    obs, setup = synth.small_config(seed=3, n_ant=10, ntimes=60, nx=128, cell_arcsec=20, flag_frac=0.0)
    dl = setup.dl
    I, Q, U, V = 1.0, 0.3, -0.2, 0.1
    src = np.array([[12 * dl, -7 * dl, I, Q, U, V]])
    obs.vis[0] = synth.predict_vis(obs.uvw.astype(np.float64), obs.freqs_hz[0], src).astype(np.complex64)
    geo = oracle.geometry_for(setup)
    kern = oracle.wkernels(geo)
    pk = (127 - (64 - 7), 64 + 12)
    img, _, _ = oracle.image_channel(obs, 0, setup, kern, geo)
    d = oracle.dft_image(obs, 0, setup, geo, kern)
    for p, want in enumerate((I, Q, U)):
        assert abs(d[p][pk] - want) < 2e-3
        assert abs(img[p][pk] - want * img[0][pk] / I) < 2e-3
    pre = oracle.preprocess(obs.uvw, obs.freq_over_c(0), obs.weights[0], obs.flags[0], geo, kern)
    w = obs.uvw[2][(pre["togrid"] | pre["compress"]) == 1]
    frac = ((w >= 0).sum() - (w < 0).sum()) / w.size
    assert 0.0 < frac < 0.5
    assert abs(d[3][pk] - V * frac * d[0][pk]) < 1e-4
    assert abs(img[3][pk] - V * frac * img[0][pk]) < 1e-4
    # the same source seen by the records with w >= 0 only: V in full
    keep = obs.uvw[2] >= 0
    obs.uvw = np.ascontiguousarray(obs.uvw[:, keep])
    for name in ("vis", "weights", "flags"):
        getattr(obs, name)[0] = np.ascontiguousarray(getattr(obs, name)[0][keep])
    d = oracle.dft_image(obs, 0, setup, geo, kern)
    assert abs(d[3][pk] - V * d[0][pk]) < 2e-3


def test_circular_feeds_against_the_dft(oracle):
    """Circular feeds (StokesConverter, PostIFFTStokesConverter.cu:72-90):
    RR = I + V, LL = I - V, RL = Q - iU, LR = Q + iU, the convention under which
    the converter's U = (Im LR - Im RL) / 2 is +U.  I, Q and V of a polarised
    source come out in full; U, carried by the cross hands, is scaled by
    (N+ - N-) / N like V with linear feeds (w<0 records are conjugated without
    exchanging RL and LR)."""
    obs, setup = synth.small_config(seed=3, n_ant=10, ntimes=60, nx=128, cell_arcsec=20, flag_frac=0.0)
    dl = setup.dl
    I, Q, U, V = 1.0, 0.3, -0.2, 0.1
    l, m = 12 * dl, -7 * dl
    f = obs.freqs_hz[0] / synth.C_LIGHT
    u, v, w = obs.uvw.astype(np.float64) * f
    ph = np.exp(-2j * np.pi * (u * l + v * m + w * (math.sqrt(1 - l * l - m * m) - 1.0)))
    obs.vis[0] = np.stack([(I + V) * ph, (Q - 1j * U) * ph, (Q + 1j * U) * ph, (I - V) * ph], axis=1).astype(np.complex64)
    geo = oracle.geometry_for(setup)
    kern = oracle.wkernels(geo)
    pk = (127 - (64 - 7), 64 + 12)
    img, _, _ = oracle.image_channel(obs, 0, setup, kern, geo, pol_type="circular")
    d = oracle.dft_image(obs, 0, setup, geo, kern, pol_type="circular")
    pre = oracle.preprocess(obs.uvw, obs.freq_over_c(0), obs.weights[0], obs.flags[0], geo, kern)
    ws = obs.uvw[2][(pre["togrid"] | pre["compress"]) == 1]
    frac = ((ws >= 0).sum() - (ws < 0).sum()) / ws.size
    for p, want in ((0, I), (1, Q), (3, V)):
        assert abs(d[p][pk] - want) < 2e-3
        assert abs(img[p][pk] - want * img[0][pk] / I) < 2e-3
    assert abs(d[2][pk] - U * frac * d[0][pk]) < 1e-4
    assert abs(img[2][pk] - U * frac * img[0][pk]) < 1e-4
    for p in range(4):
        assert np.sqrt(np.mean((img[p] - d[p]) ** 2)) < 0.02


def test_image_is_invariant_to_a_weight_scale(oracle):
    """The grid and the normaliser (sum of ConvSums x weight, WImager.cpp:
    196-197) both scale with the weights, so multiplying every weight by a
    constant leaves the normalised image unchanged; per-record weights do
    change it."""
    obs, setup = synth.small_config(seed=17, n_ant=8, ntimes=40, nx=64, flag_frac=0.1)
    a, ga, na = oracle.image_channel(obs, 0, setup)
    obs2 = synth.Observation(**{**obs.__dict__, "weights": [obs.weights[0] * np.float32(2.5)]})
    b, gb, nb = oracle.image_channel(obs2, 0, setup)
    assert np.allclose(nb, 2.5 * na, rtol=1e-12)
    assert np.abs(gb - 2.5 * ga).max() <= 1e-12 * np.abs(gb).max()
    assert np.abs(b - a).max() <= 1e-10 * np.abs(a).max()     # FP64 rounding through the FFT and corrections
    rng = np.random.default_rng(0)
    obs3 = synth.Observation(**{**obs.__dict__, "weights": [(obs.weights[0] *
                                                            rng.uniform(0.5, 2.0, obs.weights[0].shape)
                                                            ).astype(np.float32)]})
    c, _, _ = oracle.image_channel(obs3, 0, setup)
    assert np.abs(c - a).max() > 1e-6 * np.abs(a).max()
