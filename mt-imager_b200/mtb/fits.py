"""FITS output of Stokes image cubes through mtb_fits_* (include/mtb_fits.h),
the file layout mt-imager's ImageManager writes
(code/mt-imager/lib/components/ImageManager.cpp:59-236)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L

STOKES_CODES = {"I": 1, "Q": 2, "U": 3, "V": 4}


class FitsCube:
    """Open cube; write channels (float32 [P][ny][nx]) in any order, then close()."""

    def __init__(self, path, nx, ny, freqs_hz, l_increment, m_increment=None, stokes="IQUV", ra_deg=0.0,
                 dec_deg=-30.0, telescope=None, observer=None, obs_mjd=0.0):
        self.lib = L.load()
        self._freqs = np.ascontiguousarray(freqs_hz, np.float64)
        self._stokes = np.array([STOKES_CODES[c] for c in stokes], np.int32)
        m_increment = l_increment if m_increment is None else m_increment
        self._tel = telescope.encode() if telescope else None
        self._obs = observer.encode() if observer else None
        h = L.FitsHeader(nx, ny, len(self._stokes), len(self._freqs), float(l_increment), float(m_increment),
                         float(ra_deg), float(dec_deg), self._freqs.ctypes.data_as(ctypes.c_void_p),
                         self._stokes.ctypes.data_as(ctypes.c_void_p), self._tel, self._obs, float(obs_mjd))
        self.shape = (len(self._stokes), ny, nx)
        self._h = ctypes.c_void_p()
        L.check(self.lib.mtb_fits_create(str(path).encode(), ctypes.byref(h), ctypes.byref(self._h)),
                "mtb_fits_create")

    def write(self, chan, image):
        a = np.ascontiguousarray(image, np.float32)
        if a.shape != self.shape:
            raise ValueError("channel image must be %s" % (self.shape,))
        L.check(self.lib.mtb_fits_write_channel(self._h, int(chan), a.ctypes.data_as(ctypes.c_void_p)),
                "mtb_fits_write_channel")

    def close(self):
        if self._h:
            L.check(self.lib.mtb_fits_close(self._h), "mtb_fits_close")
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
