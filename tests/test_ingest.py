"""Visibility ingest: the baseline-major record order (mtb_sort_index)
against the oracle's restatement of SortIndex.cpp:46-87, the threaded row
gathers (mtb_gather_rows) against numpy indexing, and a record file written
time-major with autocorrelations read back into exactly the synthetic
observation's baseline-major records.  Host code; the last test images the
file on the GPU."""
import numpy as np
import pytest

from mtb import _lib as L
from mtb import ingest, synth


@pytest.mark.parametrize("seed,n_ant,R", [(1, 5, 200), (2, 27, 20000), (3, 64, 150000), (4, 2, 7)])
def test_sort_index_matches_oracle(oracle, seed, n_ant, R):
    rng = np.random.default_rng(seed)
    a1 = rng.integers(0, n_ant, R)
    a2 = rng.integers(0, n_ant, R)
    got = ingest.sort_index(a1, a2, n_ant)
    ref = oracle.sort_index(a1, a2, n_ant)
    assert got.dtype == np.int32 and np.array_equal(got, ref)
    assert got.size == int((a1 != a2).sum())


def test_sort_index_edges(oracle):
    assert ingest.sort_index(np.zeros(0), np.zeros(0), 3).size == 0
    assert ingest.sort_index([1, 2, 2], [1, 2, 2], 3).size == 0          # autocorrelations only
    with pytest.raises(L.MtbError):
        ingest.sort_index([0, 3], [1, 1], 3)                               # antenna id out of range
    with pytest.raises(L.MtbError):
        ingest.sort_index([0], [1], 0)


def test_gather_rows_matches_numpy():
    rng = np.random.default_rng(5)
    R = 300000
    idx = rng.permutation(R)[: R // 2].astype(np.int32)
    data = (rng.standard_normal((R, 3, 4)) + 1j * rng.standard_normal((R, 3, 4))).astype(np.complex64)
    for c in range(3):
        got = ingest.gather_rows(data, idx, offset_bytes=c * 32, row_bytes=32)
        assert np.array_equal(got, data[idx, c, :])
    uvw = rng.standard_normal((R, 3))
    for c in range(3):
        assert np.array_equal(ingest.gather_rows(uvw, idx, offset_bytes=8 * c, row_bytes=8).ravel(), uvw[idx, c])
    w = rng.random((R, 4)).astype(np.float32)
    assert np.array_equal(ingest.gather_rows(w, idx, threads=3), w[idx])
    f = (rng.random((R, 2, 4)) < 0.3).astype(np.uint8)
    assert np.array_equal(ingest.gather_rows(f, idx, offset_bytes=4, row_bytes=4), f[idx, 1, :])


def observation():
    return synth.make_observation(n_ant=9, radius_m=800.0, freqs_hz=(1.40e9, 1.42e9), hours=0.5, dt_s=60.0,
                                  nsrc=4, fov_rad=128 * 20 * synth.ARCSEC, noise=0.0, flag_frac=0.1, seed=11)


def test_record_file_round_trip(tmp_path):
    obs = observation()
    path = tmp_path / "obs.npz"
    ingest.write_record_file(path, obs)
    rf = ingest.RecordFile(path)
    assert rf.nrec == obs.nrec and rf.nchan == 2 and rf.npol == 4
    assert rf.antenna1.size == obs.nrec + obs.ntimes * obs.meta["n_ant"]   # autocorrelations on file
    assert np.array_equal(rf.uvw(), obs.uvw)
    for c in range(2):
        freq, vis, wts, flags = rf.channel(c)
        assert np.array_equal(vis, obs.vis[c])
        assert np.array_equal(flags, obs.flags[c].astype(np.uint8))
        assert np.array_equal(wts, obs.weights[c])
        assert np.array_equal(freq, obs.freq_over_c(c))
    n = sum(ch[2].shape[0] for ch in rf.chunks(1, 100))
    assert n == obs.nrec


@pytest.mark.gpu
def test_record_file_images_like_the_observation(tmp_path):
    from mtb.imager import WProjectionImager
    obs = observation()
    setup = synth.ImagingSetup(nx=128, ny=128, cell_arcsec=20.0, wplanes=8, sampling=4)
    path = tmp_path / "obs.npz"
    ingest.write_record_file(path, obs)
    rf = ingest.RecordFile(path)

    def imager():
        return WProjectionImager(setup.nx, setup.ny, setup.dl, wplanes=setup.wplanes, sampling=setup.sampling,
                                 exact_delta=True)
    a = imager()
    a.grid_chunk(obs.uvw, obs.freq_over_c(1), obs.vis[1], obs.weights[1], obs.flags[1])
    ia = a.finalize().cpu().numpy()
    peak = np.abs(ia[0]).max()
    # the file's records in one chunk: the same inputs in the same order
    b = imager()
    for chunk in rf.chunks(1, rf.nrec):
        b.grid_chunk(*chunk)
    ib = b.finalize().cpu().numpy()
    assert a.statistics() == b.statistics()
    assert np.abs(ia - ib).max() <= 1e-6 * peak
    # in 97-record chunks (duplicates do not merge across chunks, other sums):
    # the image bound
    c = imager()
    for chunk in rf.chunks(1, 97):
        c.grid_chunk(*chunk)
    ic = c.finalize().cpu().numpy()
    sa, sc = a.statistics(), c.statistics()
    assert sa["gridded_records"] + sa["compressed_records"] == sc["gridded_records"] + sc["compressed_records"]
    assert np.sqrt(np.mean((ia - ic) ** 2)) <= 1e-5 * peak
