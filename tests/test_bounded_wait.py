"""A gridder wait that runs out ends the call cleanly and is reported.

The rolling-items gridder (gridder = 5) hands work items between warps with
mbarriers; every wait gives up after a bound (about a second by default) and
sets the call's error flag, after which every thread leaves once its own
copies have landed.  The bound comes from MTB_GRIDDER_WAIT_CYCLES when set
(read at every call): at 0 cycles the waits for the first item run out while
warp 0 is still staging it.  The call then reports MTB_ERR_KERNEL (with
MTB_CHECK_GRIDDER=1) or leaves a NaN normaliser, so the image cannot pass for a
valid one; with the bound restored, the next call on the same stream grids the
same records exactly as before.  Nothing faults, traps or hangs."""
import numpy as np
import pytest
import torch

from mtb import synth
from mtb import _lib as L
from mtb.imager import WProjectionImager

pytestmark = pytest.mark.gpu


def _imager(setup):
    return WProjectionImager(setup.nx, setup.ny, setup.dl, wplanes=setup.wplanes, sampling=setup.sampling,
                             gridder=5, exact_delta=True)


def _grid(im, obs):
    im.grid_chunk(obs.uvw, obs.freq_over_c(0), obs.vis[0], obs.weights[0], obs.flags[0])
    torch.cuda.synchronize()


def test_expired_wait_is_reported_and_the_next_call_succeeds(monkeypatch):
    obs, setup = synth.small_config(seed=41, n_ant=20, ntimes=120, nx=256, cell_arcsec=10.0, wplanes=8,
                                    sampling=4, flag_frac=0.1)
    ref = _imager(setup)
    _grid(ref, obs)
    g_ref = ref.grid_sum().cpu().numpy()
    n_ref = ref.normalizer.cpu().numpy()
    assert np.isfinite(n_ref).all()

    monkeypatch.setenv("MTB_GRIDDER_WAIT_CYCLES", "0")
    bad = _imager(setup)
    status = L.MTB_OK
    try:
        _grid(bad, obs)
    except L.MtbError as e:
        status = e.status
    torch.cuda.synchronize()
    if status == L.MTB_OK:
        assert np.isnan(bad.normalizer.cpu().numpy()).all()
    else:
        assert status == L.MTB_ERR_KERNEL

    monkeypatch.delenv("MTB_GRIDDER_WAIT_CYCLES")
    good = _imager(setup)
    _grid(good, obs)
    g = good.grid_sum().cpu().numpy()
    assert np.array_equal(good.normalizer.cpu().numpy(), n_ref)
    assert np.abs(g - g_ref).max() <= 1e-6 * np.abs(g_ref).max()
    assert good.statistics() == ref.statistics()
