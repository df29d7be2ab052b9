"""mode=normal (taper-only kernel, OnlyTaperConvFunction.cpp:29-99) and PSF
imaging (psf=true, VisibilityForPSFStorageManager.cpp:65-77): oracle
properties on the CPU, the sm_100a path against the oracle on the GPU."""
import glob
import os

import numpy as np
import pytest

from mtb import synth

HERE = os.path.dirname(os.path.abspath(__file__))
TAPERS = sorted(glob.glob(os.path.join(HERE, "golden", "taper_*.npz")))
KERNEL_TOL = 1e-6
IMAGE_RMS_TOL = 1e-5


@pytest.mark.parametrize("S,s", [(7, 8), (7, 3), (9, 4)])
def test_oracle_taper_kernel_properties(oracle, S, s):
    k = oracle.taper_kernels(S, s)
    T = s if s % 2 else s + 1
    t = k["table"].reshape(T, T, S, S)
    assert np.all(t.imag == 0)
    # the zero-offset sub-kernel peaks at its centre with grdsf(0)^2
    c = t[s // 2, s // 2]
    assert np.unravel_index(np.argmax(c.real), c.shape) == (S // 2, S // 2)
    assert abs(c[S // 2, S // 2].real - oracle.lib().orc_grdsf(0.0) ** 2) < 1e-12
    # separable and symmetric under reversal of the oversampling offset
    assert np.allclose(t[s // 2, s // 2], t[s // 2, s // 2].T)
    assert np.allclose(k["conv_sums"][0], t.real.reshape(T * T, -1).sum(axis=1))


@pytest.mark.parametrize("path", TAPERS, ids=lambda p: os.path.basename(p))
def test_oracle_taper_matches_reference(oracle, path):
    z = np.load(path)
    k = oracle.taper_kernels(int(z["support"]), int(z["sampling"]))
    assert np.abs(k["table"] - z["ref_table"].astype(np.complex128)).max() <= KERNEL_TOL
    assert np.abs(k["conv_sums"] - z["ref_conv_sums"]).max() <= 1e-5 * np.abs(z["ref_conv_sums"]).max()


@pytest.mark.gpu
@pytest.mark.parametrize("S,s", [(7, 8), (7, 3), (9, 4)])
def test_gpu_taper_kernel_matches_oracle(oracle, S, s):
    from mtb.imager import build_taper_kernels
    k = build_taper_kernels(64, 64, 1e-4, 1e-4, S, s)
    o = oracle.taper_kernels(S, s)
    assert np.array_equal(k.conv_info, o["conv_info"])
    assert np.abs(k.table.cpu().numpy() - o["table"]).max() <= KERNEL_TOL
    assert np.abs(k.conv_sums.cpu().numpy() - o["conv_sums"]).max() <= 1e-6 * np.abs(o["conv_sums"]).max()


def _normal_setup(oracle, setup, S=7):
    geo = oracle.kernel_geometry(setup.nx, setup.ny, setup.dl, setup.dl, 1, setup.sampling)
    return geo, oracle.taper_kernels(S, setup.sampling)


@pytest.mark.gpu
def test_normal_mode_image_matches_oracle(oracle):
    from mtb.imager import WProjectionImager
    obs, setup = synth.small_config(seed=51, n_ant=12, ntimes=60, nx=128, cell_arcsec=20, flag_frac=0.1)
    setup.wplanes = 1
    geo, kern = _normal_setup(oracle, setup)
    img_o, grid_o, _ = oracle.image_channel(obs, 0, setup, kern, geo)
    im = WProjectionImager(setup.nx, setup.ny, setup.dl, sampling=setup.sampling, mode="normal", taper_support=7)
    im.grid_chunk(obs.uvw, obs.freq_over_c(0), obs.vis[0], obs.weights[0], obs.flags[0])
    img = im.finalize().cpu().numpy()
    g = im.grid_sum().cpu().numpy()
    assert np.abs(g - grid_o).max() <= 2e-6 * np.abs(grid_o).max()
    peak = np.abs(img_o[0]).max()
    for p in range(4):
        assert np.sqrt(np.mean((img[p] - img_o[p]) ** 2)) <= IMAGE_RMS_TOL * peak


@pytest.mark.gpu
def test_psf_image_matches_oracle(oracle):
    from mtb.imager import WProjectionImager
    obs, setup = synth.small_config(seed=52, n_ant=12, ntimes=60, nx=128, cell_arcsec=20, flag_frac=0.1)
    ones = np.ones_like(obs.vis[0])
    obs_psf = synth.Observation(**{**obs.__dict__, "vis": [ones]})
    img_o, _, _ = oracle.image_channel(obs_psf, 0, setup)
    im = WProjectionImager(setup.nx, setup.ny, setup.dl, wplanes=setup.wplanes, sampling=setup.sampling, psf=True)
    # the visibilities are ignored: pass noise to make sure
    noise = (np.random.default_rng(0).standard_normal(obs.vis[0].shape) * 5).astype(np.complex64)
    im.grid_chunk(obs.uvw, obs.freq_over_c(0), noise, obs.weights[0], obs.flags[0])
    img = im.finalize().cpu().numpy()
    c = (setup.ny - 1 - setup.ny // 2, setup.nx // 2)
    assert abs(img[0][c] - 1.0) < 1e-3                 # normalised PSF peaks at 1 in the centre
    assert np.sqrt(np.mean((img[0] - img_o[0]) ** 2)) <= IMAGE_RMS_TOL * np.abs(img_o[0]).max()


def test_oracle_psf_known_answer(oracle):
    """psf=true grids every visibility as 1 + 0i (VisibilityForPSFStorageManager.cpp:
    65-77): the normalised PSF peaks at 1 at the phase centre, and the FP64 DFT
    of the same records agrees with it (CPU)."""
    obs, setup = synth.small_config(seed=52, n_ant=12, ntimes=60, nx=128, cell_arcsec=20, flag_frac=0.1)
    obs_psf = synth.Observation(**{**obs.__dict__, "vis": [np.ones_like(obs.vis[0])]})
    img, _, _ = oracle.image_channel(obs_psf, 0, setup)
    d = oracle.dft_image(obs_psf, 0, setup)
    c = (setup.ny - 1 - setup.ny // 2, setup.nx // 2)
    assert abs(d[0][c] - 1.0) < 1e-12
    assert abs(img[0][c] - 1.0) < 1e-3
    assert np.unravel_index(np.argmax(img[0]), img[0].shape) == c
    assert np.sqrt(np.mean((img[0] - d[0]) ** 2)) < 0.02
