"""Visibility ingest: a MeasurementSet-like record file in, the path's sorted,
per-channel host arrays out.

mt-imager reads a MeasurementSet with casacore (VisibilityManager,
``code/mt-imager/lib/components/VisibilityManager/``), sorts its rows
baseline-major (SortIndex.cpp:46-87), and copies every column in that order
into chunks (SortedStorage.h:205-246), the UVW column transposed to [3][R].
casacore is not available here, so the file format is NPZ holding the same
main-table columns:

* ``antenna1``, ``antenna2``  int [R]
* ``uvw``                     float64 [R][3] metres (the MS UVW column)
* ``data``                    complex64 [R][nchan][npol]
* ``weight``                  float32 [R][npol]
* ``flag``                    bool [R][nchan][npol]
* ``chan_freq``               float64 [nchan] Hz
* ``n_antennas``              int (optional; max antenna id + 1 otherwise)
* ``time``                    float64 [R] MJD seconds (optional; the MS TIME column)
* ``site_itrf``               float64 [3] observatory ITRF metres (optional)
* ``phase_dir``               float64 [2] phase centre RA, Dec J2000 radians (optional)

Rows may be in any order (a MeasurementSet is usually time-major);
autocorrelations are dropped.  The sort and the column gathers run in the
library (mtb_sort_index, mtb_gather_rows: host code, threads, no GPU).
``RecordFile.channel`` takes the frequencies as given (nu/c of a record is
chan_freq / c); ``RecordFile.lsrk_freq_over_c`` converts them from TOPO to
LSRK per record on the GPU (mtb.lsrk, FrequencyConverter's part) when the
file holds the time, site and phase-centre columns.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L

C_LIGHT = 299792458.0


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def sort_index(antenna1, antenna2, n_antennas):
    """Baseline-major record order (mtb_sort_index): int32 [R_kept]."""
    lib = L.load()
    a1 = np.ascontiguousarray(antenna1, np.int32)
    a2 = np.ascontiguousarray(antenna2, np.int32)
    if a1.shape != a2.shape or a1.ndim != 1:
        raise ValueError("antenna1 and antenna2 must be 1-D of the same length")
    idx = np.empty(max(1, a1.size), np.int32)
    n = ctypes.c_int(0)
    L.check(lib.mtb_sort_index(_ptr(a1), _ptr(a2), int(a1.size), int(n_antennas), _ptr(idx), ctypes.byref(n)),
            "mtb_sort_index")
    return idx[:n.value].copy()


def gather_rows(column, index, offset_bytes=0, row_bytes=None, dtype=None, threads=0):
    """out[k] = row_bytes bytes of column's row index[k] starting at offset_bytes
    (mtb_gather_rows).  column: C-contiguous numpy array, rows on axis 0."""
    lib = L.load()
    col = np.ascontiguousarray(column)
    stride = col.strides[0] if col.ndim > 1 else col.itemsize
    row_bytes = stride - offset_bytes if row_bytes is None else row_bytes
    dtype = col.dtype if dtype is None else np.dtype(dtype)
    if row_bytes % dtype.itemsize:
        raise ValueError("row_bytes is not a whole number of %s" % dtype)
    idx = np.ascontiguousarray(index, np.int32)
    out = np.empty((idx.size, row_bytes // dtype.itemsize), dtype)
    L.check(lib.mtb_gather_rows(_ptr(col), stride, offset_bytes, row_bytes, _ptr(idx), int(idx.size), _ptr(out),
                                int(threads)), "mtb_gather_rows")
    return out


class RecordFile:
    """A record file sorted baseline-major, read out channel by channel in the
    layouts mtb_grid takes (uvw float32 [3][R], nu/c float32 [R], vis
    complex64 [R][P], weights float32 [R][P], flags uint8 [R][P])."""

    def __init__(self, path):
        z = np.load(path)
        self.antenna1 = np.ascontiguousarray(z["antenna1"], np.int32)
        self.antenna2 = np.ascontiguousarray(z["antenna2"], np.int32)
        self.n_antennas = int(z["n_antennas"]) if "n_antennas" in z else int(
            max(self.antenna1.max(initial=-1), self.antenna2.max(initial=-1)) + 1)
        self._uvw = np.ascontiguousarray(z["uvw"], np.float64)
        self._data = np.ascontiguousarray(z["data"], np.complex64)
        self._weight = np.ascontiguousarray(z["weight"], np.float32)
        self._flag = np.ascontiguousarray(z["flag"], np.uint8)
        self.chan_freq = np.asarray(z["chan_freq"], np.float64)
        R = self.antenna1.size
        if self._uvw.shape != (R, 3) or self._data.ndim != 3 or self._data.shape[0] != R:
            raise ValueError("uvw must be [R][3] and data [R][nchan][npol]")
        self.nchan, self.npol = self._data.shape[1], self._data.shape[2]
        if self._flag.shape != self._data.shape or self._weight.shape != (R, self.npol):
            raise ValueError("flag must match data, weight must be [R][npol]")
        if self.chan_freq.shape != (self.nchan,):
            raise ValueError("chan_freq must be [nchan]")
        self.time = np.ascontiguousarray(z["time"], np.float64) if "time" in z else None
        self.site_itrf = np.asarray(z["site_itrf"], np.float64) if "site_itrf" in z else None
        self.phase_dir = np.asarray(z["phase_dir"], np.float64) if "phase_dir" in z else None
        if self.time is not None and self.time.shape != (R,):
            raise ValueError("time must be [R]")
        self.index = sort_index(self.antenna1, self.antenna2, self.n_antennas)
        self.nrec = int(self.index.size)
        self._uvw_sorted = None
        self._weights_sorted = None

    def uvw(self):
        """float32 [3][R] metres in record order (transposed like the
        reference's UVW storage)."""
        if self._uvw_sorted is None:
            rows = [gather_rows(self._uvw, self.index, offset_bytes=8 * c, row_bytes=8).ravel() for c in range(3)]
            self._uvw_sorted = np.stack(rows).astype(np.float32)
        return self._uvw_sorted

    def weights(self):
        if self._weights_sorted is None:
            self._weights_sorted = gather_rows(self._weight, self.index)
        return self._weights_sorted

    def channel(self, chan):
        """(freq, vis, weights, flags) of one channel in record order."""
        if not 0 <= chan < self.nchan:
            raise IndexError("channel %d of %d" % (chan, self.nchan))
        P = self.npol
        vis = gather_rows(self._data, self.index, offset_bytes=chan * P * 8, row_bytes=P * 8)
        flags = gather_rows(self._flag, self.index, offset_bytes=chan * P, row_bytes=P)
        freq = np.full(self.nrec, self.chan_freq[chan] / C_LIGHT, np.float32)
        return freq, vis, self.weights(), flags

    def lsrk_freq_over_c(self, device="cuda", stream=None, **kw):
        """float32 device tensor [nchan][nrec]: every channel's nu/c converted
        from TOPO to LSRK per record, in record order (FrequencyConverter:
        the conversion runs over the rows in file order, where equal
        consecutive times share one evaluation, and the result is taken in
        the sort index's order)."""
        if self.time is None or self.site_itrf is None or self.phase_dir is None:
            raise ValueError("the record file has no time, site_itrf or phase_dir column")
        from .lsrk import lsrk_freq_over_c
        return lsrk_freq_over_c(self.time, self.chan_freq, self.site_itrf, self.phase_dir[0], self.phase_dir[1],
                                index=self.index, device=device, stream=stream, **kw)

    def chunks(self, chan, chunk_records):
        """(uvw, freq, vis, weights, flags) of one channel in record chunks."""
        uvw = self.uvw()
        freq, vis, wts, flags = self.channel(chan)
        for a in range(0, self.nrec, chunk_records):
            b = min(self.nrec, a + chunk_records)
            yield (np.ascontiguousarray(uvw[:, a:b]), freq[a:b], vis[a:b], wts[a:b], flags[a:b])


def write_record_file(path, obs, autocorrelations=True, time_s=None, site_itrf=None, phase_dir=None):
    """Write a synthetic observation (mtb.synth, baseline-major) as a record
    file in time-major row order, the usual MeasurementSet order, with an
    autocorrelation row per antenna and time (dropped again on ingest).
    ``time_s`` (MJD seconds per time sample), ``site_itrf`` and ``phase_dir``
    add the columns the TOPO -> LSRK conversion needs."""
    from .synth import baseline_order
    n_ant = obs.meta["n_ant"]
    pairs = baseline_order(n_ant)
    nbl, nt = len(pairs), obs.ntimes
    nchan = len(obs.freqs_hz)
    P = obs.vis[0].shape[1]
    # obs records are [baseline][time]; time-major rows: [time][baseline]
    order = np.arange(nbl * nt).reshape(nbl, nt).T.ravel()
    a1 = np.repeat(np.array([[p[0] for p in pairs]]), nt, axis=0).ravel()
    a2 = np.repeat(np.array([[p[1] for p in pairs]]), nt, axis=0).ravel()
    uvw = obs.uvw.T[order].astype(np.float64)
    data = np.stack([obs.vis[c][order] for c in range(nchan)], axis=1)
    flag = np.stack([obs.flags[c][order] for c in range(nchan)], axis=1).astype(bool)
    weight = obs.weights[0][order]
    if autocorrelations:
        # one autocorrelation row per antenna before each time's cross rows
        ta1 = np.tile(np.arange(n_ant), nt)
        rows_t = nbl + n_ant
        na1 = np.empty(nt * rows_t, np.int32)
        na2 = np.empty_like(na1)
        nuvw = np.zeros((nt * rows_t, 3))
        ndata = np.ones((nt * rows_t, nchan, P), np.complex64)
        nflag = np.zeros((nt * rows_t, nchan, P), bool)
        nweight = np.ones((nt * rows_t, P), np.float32)
        cross = np.ones(nt * rows_t, bool)
        for t in range(nt):
            cross[t * rows_t:t * rows_t + n_ant] = False
        na1[~cross], na2[~cross] = ta1, ta1
        na1[cross], na2[cross] = a1, a2
        nuvw[cross], ndata[cross], nflag[cross], nweight[cross] = uvw, data, flag, weight
        a1, a2, uvw, data, flag, weight = na1, na2, nuvw, ndata, nflag, nweight
    extra = {}
    if time_s is not None:
        time_s = np.asarray(time_s, np.float64)
        if time_s.shape != (nt,):
            raise ValueError("time_s needs one time per time sample")
        extra["time"] = np.repeat(time_s, a1.size // nt)
    if site_itrf is not None:
        extra["site_itrf"] = np.asarray(site_itrf, np.float64)
    if phase_dir is not None:
        extra["phase_dir"] = np.asarray(phase_dir, np.float64)
    np.savez(path, antenna1=a1, antenna2=a2, uvw=uvw, data=data, weight=weight, flag=flag,
             chan_freq=np.asarray(obs.freqs_hz, np.float64), n_antennas=n_ant, **extra)
