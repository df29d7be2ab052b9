"""TOPO -> LSRK channel frequencies per record (nu/c), on the GPU.

Plays the part of mt-imager's FrequencyConverter
(``code/mt-imager/lib/components/VisibilityManager/FrequencyConverter.cpp``):
its inputs are the MeasurementSet TIME column, the TOPO channel frequencies,
the observatory position and the phase centre
(``MSVisibilityDataSetAsync.cpp:169``), and its output per channel is the
float32 nu/c column PreProcessUVW takes, in the ingest's record order (the
reference sorts each channel's store by the sort index,
``FrequencyConverter.cpp:155-165``).  The computation is
``mtb_lsrk_freq_over_c`` in libmtb.so.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L
from .imager import _dev, _ptr, _require_cuda, _stream

# TT - UTC from 2017-01-01 (37 leap seconds + 32.184 s)
TT_MINUS_UTC = 69.184


def lsrk_freq_over_c(time_s, chan_hz, site_itrf, ra, dec, index=None, tt_minus_time=TT_MINUS_UTC,
                     ut1_minus_time=0.0, device="cuda", stream=None, out=None, workspace=None):
    """float32 tensor [nchan][n] on `device`: nu_LSRK / c per channel and record.

    time_s     MJD seconds per row (MeasurementSet TIME), [nrows]
    chan_hz    TOPO channel frequencies (Hz), [nchan]
    site_itrf  observatory ITRF position (m), 3 values
    ra, dec    phase centre, J2000 radians
    index      rows in output order (e.g. ``RecordFile.index``), or None for
               every row in its own order
    out        optional float32 device tensor [nchan][n] to write into
    workspace  optional uint8 device tensor of at least
               ``lsrk_workspace_bytes(nrows)`` bytes (reused between calls on
               one stream)
    """
    _require_cuda(device)
    lib = L.load()
    t = _dev(np.asarray(time_s, np.float64) if not isinstance(time_s, torch.Tensor) else time_s, torch.float64,
             device)
    ch = _dev(np.asarray(chan_hz, np.float64) if not isinstance(chan_hz, torch.Tensor) else chan_hz,
              torch.float64, device)
    idx = None if index is None else _dev(np.asarray(index, np.int32) if not isinstance(index, torch.Tensor)
                                          else index, torch.int32, device)
    nrows, nchan = int(t.numel()), int(ch.numel())
    n = nrows if idx is None else int(idx.numel())
    p = L.LsrkParams()
    site = np.asarray(site_itrf, np.float64).ravel()
    if site.size != 3:
        raise ValueError("site_itrf needs 3 values")
    for k in range(3):
        p.site_itrf[k] = float(site[k])
    p.ra, p.dec = float(ra), float(dec)
    p.tt_minus_time, p.ut1_minus_time = float(tt_minus_time), float(ut1_minus_time)
    nbytes = lsrk_workspace_bytes(nrows)
    if workspace is None:
        workspace = torch.empty(max(1, nbytes), dtype=torch.uint8, device=device)
    elif workspace.numel() * workspace.element_size() < nbytes or not workspace.is_cuda:
        raise ValueError("workspace needs %d device bytes" % nbytes)
    if out is None:
        out = torch.empty((nchan, n), dtype=torch.float32, device=device)
    elif (tuple(out.shape) != (nchan, n) or out.dtype != torch.float32 or not out.is_contiguous()
          or not out.is_cuda):
        raise ValueError("out must be a contiguous float32 device tensor [%d][%d]" % (nchan, n))
    ws = workspace
    L.check(lib.mtb_lsrk_freq_over_c(ctypes.byref(p), _ptr(t), nrows, _ptr(ch), nchan, _ptr(idx), n, _ptr(out),
                                     _ptr(ws), ws.numel() * ws.element_size(), _stream(stream)),
            "mtb_lsrk_freq_over_c")
    return out


def lsrk_workspace_bytes(nrows):
    """Device workspace bytes of one conversion over nrows rows."""
    nbytes = ctypes.c_size_t(0)
    L.check(L.load().mtb_lsrk_workspace_size(int(nrows), ctypes.byref(nbytes)), "mtb_lsrk_workspace_size")
    return nbytes.value
