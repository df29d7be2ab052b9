"""Python access to the imaging request engine (include/mtb_engine.h).

``Engine`` accepts imaging requests of any geometry while others run: each is
admitted when a worker slot is free and its device memory fits in the HBM
budget, runs on its own CUDA stream, and shares the cached w-kernel table of
its geometry.  Inputs are host numpy arrays in the layouts of mtb.h; they are
kept referenced until the request is waited for.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _lib as L


@dataclasses.dataclass
class Result:
    image: np.ndarray
    status: int
    kernel_cache_hit: bool
    queue_ms: float
    service_ms: float
    latency_ms: float
    stats: dict


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class Engine:
    def __init__(self, slots=4, hbm_budget_bytes=0, kernel_cache_bytes=0, chunk_records=0, host_threads=0):
        self.lib = L.load()
        cfg = L.EngineConfig(slots, hbm_budget_bytes, kernel_cache_bytes, chunk_records, host_threads)
        self._h = ctypes.c_void_p()
        L.check(self.lib.mtb_engine_create(ctypes.byref(cfg), ctypes.byref(self._h)), "mtb_engine_create")
        self._pending = {}

    def _request(self, nx, ny, l_increment, m_increment, wplanes, sampling, uvw, freq, vis, weights, flags,
                 trial_support=0, max_support=0, w_max=0.0, pol_type=L.MTB_POL_LINEAR, compensated=True,
                 exact_delta=False):
        uvw = np.asarray(uvw)
        # a [3][R] slice of a longer float32 uvw array is passed as it is, with its row stride
        row_stride = 0
        if (uvw.dtype == np.float32 and uvw.ndim == 2 and uvw.strides[1] == 4 and uvw.strides[0] % 4 == 0
                and uvw.strides[0] >= 4 * uvw.shape[1]):
            row_stride = uvw.strides[0] // 4
        else:
            uvw = _c(uvw, np.float32)
        freq = _c(freq, np.float32)
        vis = _c(vis, np.complex64)
        weights = _c(weights, np.float32)
        byte_flags = np.asarray(flags).dtype in (np.uint8, np.bool_)
        flags = _c(flags, np.uint8 if byte_flags else np.int32)
        R = int(freq.size)
        P = int(vis.shape[1]) if vis.ndim == 2 else 1
        if uvw.shape != (3, R) or vis.shape != (R, P) or weights.shape != (R, P) or flags.shape != (R, P):
            raise ValueError("record arrays must be uvw [3][R], vis/weights/flags [R][P]")
        image = np.empty((P, ny, nx), np.float32)
        g = L.WKernelParams(nx, ny, float(l_increment), float(m_increment), wplanes, sampling, trial_support,
                            max_support, float(w_max))
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        req = L.ImageRequest(g, P, pol_type, int(bool(compensated)), R, ptr(uvw), ptr(freq), ptr(vis),
                             ptr(weights), ptr(flags), ptr(image), int(bool(exact_delta)), row_stride,
                             int(byte_flags))
        return req, (uvw, freq, vis, weights, flags, image)

    def request_bytes(self, *args, **kw) -> int:
        req, _ = self._request(*args, **kw)
        n = ctypes.c_size_t(0)
        L.check(self.lib.mtb_engine_request_bytes(self._h, ctypes.byref(req), ctypes.byref(n)),
                "mtb_engine_request_bytes")
        return n.value

    def submit(self, nx, ny, l_increment, m_increment, wplanes, sampling, uvw, freq, vis, weights, flags,
               **kw) -> int:
        """Queue one image; returns a ticket for wait()."""
        req, keep = self._request(nx, ny, l_increment, m_increment, wplanes, sampling, uvw, freq, vis, weights,
                                  flags, **kw)
        t = ctypes.c_longlong(0)
        L.check(self.lib.mtb_engine_submit(self._h, ctypes.byref(req), ctypes.byref(t)), "mtb_engine_submit")
        self._pending[t.value] = keep
        return t.value

    def cancel(self, ticket: int) -> None:
        """Cancel a request: dropped if still queued, stopped at its next chunk
        boundary if running; wait() then returns status MTB_ERR_CANCELLED (a
        request that had completed keeps its result).  The host arrays stay
        referenced until wait()."""
        L.check(self.lib.mtb_engine_cancel(self._h, ticket), "mtb_engine_cancel")

    def wait(self, ticket: int) -> Result:
        res = L.ImageResult()
        L.check(self.lib.mtb_engine_wait(self._h, ticket, ctypes.byref(res)), "mtb_engine_wait")
        keep = self._pending.pop(ticket)
        s = res.stats
        return Result(image=keep[5], status=res.status, kernel_cache_hit=bool(res.kernel_cache_hit),
                      queue_ms=res.queue_ms, service_ms=res.service_ms, latency_ms=res.latency_ms,
                      stats=dict(gridded_records=s.gridded_records, compressed_records=s.compressed_records,
                                 gridded_points=s.gridded_points, compressed_points=s.compressed_points))

    def close(self):
        if self._h:
            self.lib.mtb_engine_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._pending.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
