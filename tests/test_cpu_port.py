"""The timed CPU baseline (oracle/cpu_port.c, the FP32 OpenMP transcription
of the reference's per-chunk gridding that `bench.py --impl reference` and
the cpu_baseline leg run) against the FP64 oracle, on the CPU.

A baseline that gridded something else would make its samples/s
meaningless, so its record statistics must equal the oracle's exactly and
its grid and normaliser must agree to FP32 rounding (the reference grids in
FP32: ConvolutionGridder.cu:130-181).
"""
import numpy as np
import pytest

from mtb import synth

GRID_TOL = 2e-6      # max |port - oracle| / max |oracle| over the complex grid (FP32 sums of <= 2e3 taps)
NORM_TOL = 1e-6


def _port_chunk(O, obs, geo, kern, npol, threads=None):
    PT = O.port()
    if threads:
        PT.port_set_threads(threads)
    R = obs.nrec
    grid = np.zeros((geo["ny"], geo["nx"], npol), np.complex64)
    norm = np.zeros(npol, np.float32)
    st = np.zeros(4, np.int64)
    uvw = np.ascontiguousarray(obs.uvw, np.float32)
    freq = np.ascontiguousarray(obs.freq_over_c(0), np.float32)
    vis = np.ascontiguousarray(obs.vis[0][:, :npol], np.complex64)
    wts = np.ascontiguousarray(obs.weights[0][:, :npol], np.float32)
    flg = np.ascontiguousarray(obs.flags[0][:, :npol], np.int32)
    table = np.ascontiguousarray(kern["table"], np.complex64)
    sums = np.ascontiguousarray(kern["conv_sums"], np.float32)
    rc = PT.port_grid_chunk(R, npol, O._p(uvw), O._p(freq), O._p(vis), O._p(wts), O._p(flg), geo["wplanes"],
                            geo["w_inc"], O._p(kern["conv_info"]), O._p(sums), O._p(table), geo["sampling"],
                            geo["ny"], geo["nx"], geo["du"], geo["dv"], O._p(grid), O._p(norm), O._p(st))
    assert rc == 0
    return grid, norm, st


@pytest.mark.parametrize("npol,sampling,wplanes,seed,ny", [(4, 4, 8, 4, 128), (4, 3, 4, 6, 128), (2, 8, 8, 8, 128),
                                                         (1, 4, 2, 9, 128), (4, 4, 8, 10, 96)])
def test_port_matches_oracle(oracle, npol, sampling, wplanes, seed, ny):
    import dataclasses
    obs, setup = synth.small_config(seed=seed, n_ant=10, ntimes=60, nx=128, cell_arcsec=20, wplanes=wplanes,
                                    sampling=sampling, flag_frac=0.2)
    setup = dataclasses.replace(setup, ny=ny)
    geo = oracle.geometry_for(setup)
    kern = oracle.wkernels(geo)
    g, n, pre = oracle.grid_chunk(obs.uvw, obs.freq_over_c(0), obs.vis[0][:, :npol], obs.weights[0][:, :npol],
                                  obs.flags[0][:, :npol], geo, kern)
    st = oracle.stats(pre)
    grid, norm, pst = _port_chunk(oracle, obs, geo, kern, npol)
    assert st["gridded_records"] > 0 and st["compressed_records"] > 0
    assert list(pst) == [st["gridded_records"], st["compressed_records"], st["gridded_points"],
                         st["compressed_points"]]
    assert np.abs(grid - g).max() <= GRID_TOL * np.abs(g).max()
    assert np.abs(norm - n).max() <= NORM_TOL * np.abs(n).max()


def test_port_result_does_not_depend_on_threads(oracle):
    """The port splits grid rows over threads (no two threads write a cell),
    so its grid is the same for any thread count."""
    obs, setup = synth.small_config(seed=12, n_ant=10, ntimes=60, nx=128, cell_arcsec=20, wplanes=8, sampling=4,
                                    flag_frac=0.1)
    geo = oracle.geometry_for(setup)
    kern = oracle.wkernels(geo)
    PT = oracle.port()
    full = PT.port_threads()
    try:
        g1, n1, s1 = _port_chunk(oracle, obs, geo, kern, 4, threads=1)
        g3, n3, s3 = _port_chunk(oracle, obs, geo, kern, 4, threads=3)
    finally:
        PT.port_set_threads(full)
    assert np.array_equal(s1, s3)
    assert np.array_equal(g1, g3)
    assert np.allclose(n1, n3, rtol=1e-6)


def test_port_empty_and_fully_flagged_chunks(oracle):
    obs, setup = synth.small_config(seed=13, n_ant=6, ntimes=20, nx=64, wplanes=4, sampling=4, flag_frac=0.0)
    geo = oracle.geometry_for(setup)
    kern = oracle.wkernels(geo)
    obs.flags[0][:] = 1
    grid, norm, st = _port_chunk(oracle, obs, geo, kern, 4)
    assert not st.any() and not grid.any() and not norm.any()
    empty = synth.Observation(**{**obs.__dict__, "uvw": np.zeros((3, 0), np.float32),
                                 "vis": [obs.vis[0][:0]], "weights": [obs.weights[0][:0]],
                                 "flags": [obs.flags[0][:0]]})
    grid, norm, st = _port_chunk(oracle, empty, geo, kern, 4)
    assert not st.any() and not grid.any() and not norm.any()
