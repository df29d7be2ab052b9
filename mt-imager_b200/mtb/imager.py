"""Host API of the W-projection imaging path over the C ABI.

``WProjectionImager`` plays the part of mt-imager's three imaging modules on
one GPU: WProjectionConvFunction (kernel table), WImager (per-chunk gridding
into an accumulating grid and normaliser) and ImageFinalizer (Stokes cube),
as wired by ``code/mt-imager/app/mtimager.cpp:138-199``.  Device memory and
streams come from PyTorch; every computation is a call into libmtb.so.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import torch

from . import _lib as L


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _dev(x, dtype, device):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(x)).to(device=device, dtype=dtype)


def _require_cuda(device):
    if torch.device(device).type != "cuda":
        raise ValueError("the library runs on a CUDA device (no CPU fallback); got %s" % device)


def _on_device(t, device):
    """t lives on `device` (a device without an index means the current one)."""
    if t.device.type != device.type:
        return False
    if device.type != "cuda":
        return True
    want = device.index if device.index is not None else torch.cuda.current_device()
    return t.device.index == want


def _is_byte_flags(flags):
    dt = getattr(flags, "dtype", None)
    return dt in (np.uint8, np.bool_, torch.uint8, torch.bool)


def _flags_u8(flags, R, P):
    """mtb_grid_params.flags_u8 for a device flag tensor: int32 [R][P] -> 0,
    uint8 [R][P] -> 1, uint8 [ceil(R*P/8)] bit-packed (pack_flags) -> 2."""
    if flags.dtype == torch.uint8:
        if flags.dim() == 1 and flags.numel() == (R * P + 7) // 8 and flags.numel() != R * P:
            return 2
        if flags.numel() != R * P:
            raise ValueError("uint8 flags must be [R][P] bytes or ceil(R*P/8) packed bytes")
        return 1
    if flags.dtype == torch.int32:
        return 0
    raise TypeError("flags must be int32 or uint8 on the device")


def pack_flags(flags):
    """One bit per flag (mtb_grid_params.flags_u8 = 2): flags [R][P] (any
    dtype; non-zero = flagged) -> uint8 [ceil(R*P/8)], flag i = r*P + p in bit
    i % 8 of byte i / 8.  A torch tensor stays on its device; numpy gives numpy."""
    if isinstance(flags, torch.Tensor):
        bits = (flags.reshape(-1) != 0).to(torch.uint8)
        pad = (-bits.numel()) % 8
        if pad:
            bits = torch.cat([bits, bits.new_zeros(pad)])
        w = torch.tensor([1, 2, 4, 8, 16, 32, 64, 128], dtype=torch.uint8, device=bits.device)
        return (bits.view(-1, 8) * w).sum(dim=1, dtype=torch.uint8).contiguous()
    return np.packbits(np.asarray(flags).reshape(-1) != 0, bitorder="little")


@dataclasses.dataclass
class KernelTable:
    """AmalgamatedConvFunction, convInfo and ConvSums
    (WProjectionConvFunction.cpp:297-301)."""
    table: torch.Tensor          # complex64 [elems]
    conv_info: np.ndarray        # int32 [wplanes][2] (host)
    d_conv_info: torch.Tensor    # int32 [wplanes][2]
    conv_sums: torch.Tensor      # float32 [wplanes][T*T]
    info: L.WKernelInfo
    params: L.WKernelParams

    @property
    def supports(self):
        return self.conv_info[:, 0].copy()


def wkernel_params(nx, ny, l_increment, m_increment, wplanes, sampling, trial_support=0, max_support=0,
                   w_max=0.0) -> L.WKernelParams:
    return L.WKernelParams(nx, ny, float(l_increment), float(m_increment), wplanes, sampling, trial_support,
                           max_support, float(w_max))


def build_taper_kernels(nx, ny, l_increment, m_increment, support=7, sampling=8, device="cuda",
                        stream=None) -> KernelTable:
    """mode=normal: the taper-only kernel table (one plane, no w-term) of
    OnlyTaperConvFunction.cpp:29-99 through mtb_taper_kernel_build."""
    _require_cuda(device)
    lib = L.load()
    T = sampling if sampling % 2 else sampling + 1
    n = T * T * support * support
    table = torch.empty(n, dtype=torch.complex64, device=device)
    d_ci = torch.empty((1, 2), dtype=torch.int32, device=device)
    h_ci = np.zeros((1, 2), np.int32)
    sums = torch.empty((1, T * T), dtype=torch.float32, device=device)
    got = ctypes.c_size_t(0)
    L.check(lib.mtb_taper_kernel_build(support, sampling, _ptr(table), n, _ptr(d_ci),
                                       h_ci.ctypes.data_as(ctypes.c_void_p), _ptr(sums), ctypes.byref(got),
                                       _stream(stream)), "mtb_taper_kernel_build")
    params = wkernel_params(nx, ny, l_increment, m_increment, 1, sampling)
    info = L.WKernelInfo()
    info.trial_support = support
    info.support_cap = support
    info.T = T
    info.w_sq_increment = 1.0        # one plane (WProjectionConvFunction.cpp:110)
    info.total_l, info.total_m = l_increment * nx, m_increment * ny
    info.u_increment, info.v_increment = 1.0 / (l_increment * nx), 1.0 / (m_increment * ny)
    info.table_capacity = n
    return KernelTable(table=table, conv_info=h_ci, d_conv_info=d_ci, conv_sums=sums, info=info, params=params)


def query_wkernels(params: L.WKernelParams) -> L.WKernelInfo:
    lib = L.load()
    info = L.WKernelInfo()
    L.check(lib.mtb_wkernel_query(ctypes.byref(params), ctypes.byref(info)), "mtb_wkernel_query")
    return info


def build_wkernels(params: L.WKernelParams, device="cuda", stream=None) -> KernelTable:
    _require_cuda(device)
    lib = L.load()
    info = query_wkernels(params)
    ws = torch.empty(max(1, info.workspace_bytes), dtype=torch.uint8, device=device)
    table = torch.empty(max(1, info.table_capacity), dtype=torch.complex64, device=device)
    nw = params.wplanes
    d_ci = torch.empty((nw, 2), dtype=torch.int32, device=device)
    h_ci = np.zeros((nw, 2), np.int32)
    sums = torch.empty((nw, info.T * info.T), dtype=torch.float32, device=device)
    n = ctypes.c_size_t(0)
    L.check(lib.mtb_wkernel_build(ctypes.byref(params), _ptr(ws), info.workspace_bytes, _ptr(table),
                                  info.table_capacity, _ptr(d_ci), h_ci.ctypes.data_as(ctypes.c_void_p),
                                  _ptr(sums), ctypes.byref(n), _stream(stream)), "mtb_wkernel_build")
    del ws
    return KernelTable(table=table[: n.value].clone(), conv_info=h_ci, d_conv_info=d_ci, conv_sums=sums,
                       info=info, params=params)


class WProjectionImager:
    """One image (one channel) on one GPU: kernel table, resident grid and
    normaliser, chunked gridding and finalisation."""

    def __init__(self, nx, ny, l_increment, m_increment=None, wplanes=32, sampling=8, npol=4,
                 trial_support=0, max_support=0, w_max=0.0, pol_type=L.MTB_POL_LINEAR, compensated=True,
                 tile=0, support_bucket=0, max_chunk=0, merge=0, device="cuda",
                 kernels: KernelTable | None = None, psf=False, mode="wproj", taper_support=7,
                 exact_delta=False, gridder_threads=0, gridder=0):
        """mode "wproj" (W-projection kernels) or "normal" (taper-only kernel of
        support taper_support at oversampling `sampling`, one plane); psf
        grids every visibility as 1 + 0i (mt-imager's psf=true)."""
        self.lib = L.load()
        self.device = torch.device(device)
        _require_cuda(self.device)
        self.nx, self.ny, self.npol = nx, ny, npol
        m_increment = l_increment if m_increment is None else m_increment
        if mode not in ("wproj", "normal"):
            raise ValueError("mode must be 'wproj' or 'normal'")
        self.mode, self.psf, self.taper_support = mode, bool(psf), taper_support
        self.exact_delta = bool(exact_delta)
        if mode == "normal":
            wplanes = 1
        self.params = wkernel_params(nx, ny, l_increment, m_increment, wplanes, sampling, trial_support,
                                     max_support, w_max)
        self.kernels = kernels
        self.compensated = compensated
        self.pol_type = pol_type
        self.tuning = dict(tile=tile, support_bucket=support_bucket, max_chunk=max_chunk, merge=merge,
                           gridder_threads=gridder_threads, gridder=gridder)
        self.grid = torch.zeros((ny, nx, npol), dtype=torch.complex64, device=self.device)
        self.grid_lo = torch.zeros_like(self.grid) if compensated else None
        self.normalizer = torch.zeros(npol, dtype=torch.float32, device=self.device)
        self.stats = torch.zeros(4, dtype=torch.int64, device=self.device)
        self._ws = None
        self._fin_ws = None
        # optional (start, end) torch.cuda.Event pair recorded around the
        # gridder kernels of every mtb_grid call
        self.gridder_events = None
        self._fresh = True

    # -- WProjectionConvFunction
    def build_kernels(self, stream=None) -> KernelTable:
        if self.kernels is None:
            if self.mode == "normal":
                p = self.params
                self.kernels = build_taper_kernels(p.nx, p.ny, p.l_increment, p.m_increment, self.taper_support,
                                                   p.sampling, self.device, stream)
            else:
                self.kernels = build_wkernels(self.params, self.device, stream)
        return self.kernels

    def grid_params(self, initialize: bool) -> L.GridParams:
        k = self.build_kernels()
        gp = L.GridParams(self.nx, self.ny, self.npol, self.params.sampling, self.params.wplanes,
                          k.info.u_increment, k.info.v_increment, k.info.w_sq_increment, int(initialize),
                          self.tuning["tile"], self.tuning["support_bucket"], self.tuning["max_chunk"],
                          self.tuning["merge"])
        gp.psf = int(self.psf)
        gp.exact_delta = int(self.exact_delta)
        gp.no_grid_lo = 0 if self.compensated else 1
        gp.gridder_threads = self.tuning["gridder_threads"]
        gp.gridder = self.tuning["gridder"]
        if self.gridder_events is not None:
            gp.gridder_start_event = self.gridder_events[0].cuda_event
            gp.gridder_end_event = self.gridder_events[1].cuda_event
        return gp

    def _workspace(self, nrec, gp):
        need = ctypes.c_size_t(0)
        ci = self.build_kernels().conv_info
        L.check(self.lib.mtb_grid_workspace_size(ctypes.byref(gp), ci.ctypes.data_as(ctypes.c_void_p), nrec,
                                                 ctypes.byref(need)),
                "mtb_grid_workspace_size")
        if self._ws is None or self._ws.numel() < need.value:
            self._ws = torch.empty(max(1, need.value), dtype=torch.uint8, device=self.device)
        return self._ws, need.value

    def reset(self):
        self._fresh = True

    # -- WImager
    def grid_chunk(self, uvw, freq, vis, weights, flags, stream=None):
        """Grid one chunk: uvw [3][R] float32 metres, freq [R] nu/c, vis [R][P]
        complex64, weights [R][P] float32, flags [R][P] int32, or uint8 / bool
        (one byte per flag, mtb_grid_params.flags_u8) -- numpy or torch."""
        dev = self.device
        uvw = _dev(uvw, torch.float32, dev)
        freq = _dev(freq, torch.float32, dev)
        vis = _dev(vis, torch.complex64, dev)
        weights = _dev(weights, torch.float32, dev)
        flags = _dev(flags, torch.uint8 if _is_byte_flags(flags) else torch.int32, dev)
        R = int(freq.numel())
        if vis.shape != (R, self.npol) or weights.shape != (R, self.npol) or flags.shape != (R, self.npol):
            raise ValueError("record arrays must be [R][npol]")
        if uvw.shape != (3, R):
            raise ValueError("uvw must be [3][R]")
        return self.grid_device(uvw, freq, vis, weights, flags, stream)

    def grid_device(self, uvw, freq, vis, weights, flags, stream=None):
        """One chunk from tensors already on the imager's device (layouts of
        grid_chunk); anything else is refused before a kernel sees it."""
        for name, t in (("uvw", uvw), ("freq", freq), ("vis", vis), ("weights", weights), ("flags", flags)):
            if not (isinstance(t, torch.Tensor) and _on_device(t, self.device) and t.is_contiguous()):
                raise ValueError("%s must be a contiguous tensor on %s" % (name, self.device))
        k = self.build_kernels()
        R = int(freq.numel())
        gp = self.grid_params(self._fresh)
        gp.flags_u8 = _flags_u8(flags, R, self.npol)
        ws, nbytes = self._workspace(R, gp)
        st = L.check(self.lib.mtb_grid(ctypes.byref(gp), _ptr(k.table), _ptr(k.d_conv_info),
                                       k.conv_info.ctypes.data_as(ctypes.c_void_p), _ptr(k.conv_sums),
                                       _ptr(uvw), _ptr(freq), _ptr(vis), _ptr(weights), _ptr(flags), R,
                                       _ptr(self.grid), _ptr(self.grid_lo), _ptr(self.normalizer),
                                       _ptr(self.stats), _ptr(ws), nbytes, _stream(stream)), "mtb_grid")
        self._fresh = False
        return st

    # -- ImageFinalizer
    def finalize(self, out=None, stream=None):
        fp = L.FinalizeParams(self.nx, self.ny, self.npol, self.params.sampling, self.pol_type)
        need = ctypes.c_size_t(0)
        L.check(self.lib.mtb_finalize_workspace_size(ctypes.byref(fp), ctypes.byref(need)),
                "mtb_finalize_workspace_size")
        if self._fin_ws is None or self._fin_ws.numel() < need.value:
            self._fin_ws = torch.empty(max(1, need.value), dtype=torch.uint8, device=self.device)
        if out is None:
            out = torch.empty((self.npol, self.ny, self.nx), dtype=torch.float32, device=self.device)
        L.check(self.lib.mtb_finalize(ctypes.byref(fp), _ptr(self.grid), _ptr(self.grid_lo), _ptr(self.normalizer),
                                      _ptr(out), _ptr(self._fin_ws), need.value, _stream(stream)), "mtb_finalize")
        return out

    def grid_sum(self):
        """Grid value the finaliser uses (hi + compensation term)."""
        g = self.grid.clone()
        if self.grid_lo is not None:
            g += self.grid_lo
        return g

    def statistics(self):
        s = self.stats.cpu().numpy()
        return dict(gridded_records=int(s[0]), compressed_records=int(s[1]), gridded_points=int(s[2]),
                    compressed_points=int(s[3]))


def _batch_jobs(entries):
    jobs = (L.GridJob * len(entries))()
    keep = []
    for j, (im, uvw, freq, vis, weights, flags) in enumerate(entries):
        for name, t in (("uvw", uvw), ("freq", freq), ("vis", vis), ("weights", weights), ("flags", flags)):
            if not (isinstance(t, torch.Tensor) and _on_device(t, im.device) and t.is_contiguous()):
                raise ValueError("image %d: %s must be a contiguous tensor on %s" % (j, name, im.device))
        k = im.build_kernels()
        gp = im.grid_params(im._fresh)
        J = jobs[j]
        gp.flags_u8 = _flags_u8(flags, int(freq.numel()), im.npol)
        J.params = gp
        J.d_table, J.d_conv_info = _ptr(k.table), _ptr(k.d_conv_info)
        J.h_conv_info = k.conv_info.ctypes.data_as(ctypes.c_void_p)
        J.d_conv_sums = _ptr(k.conv_sums)
        J.d_uvw, J.d_freq, J.d_vis = _ptr(uvw), _ptr(freq), _ptr(vis)
        J.d_weights, J.d_flags = _ptr(weights), _ptr(flags)
        J.nrecords = int(freq.numel())
        J.d_grid, J.d_grid_lo = _ptr(im.grid), _ptr(im.grid_lo)
        J.d_normalizer, J.d_stats = _ptr(im.normalizer), _ptr(im.stats)
        keep.append(k)
    return jobs, keep


def grid_batch(entries, workspace=None, stream=None):
    """Grid one chunk into each of several images with one persistent gridder
    launch (mtb_grid_batch).  entries: (WProjectionImager, uvw, freq, vis,
    weights, flags) with device tensors in the layouts of grid_device; every
    imager must have the same npol, gridder_threads and gridder.  Returns the workspace
    tensor so a caller can pass it back (or keep it alive across a CUDA graph
    replay)."""
    if not entries:
        return workspace
    lib = L.load()
    jobs, keep = _batch_jobs(entries)
    need = ctypes.c_size_t(0)
    L.check(lib.mtb_grid_batch_workspace_size(jobs, len(entries), ctypes.byref(need)),
            "mtb_grid_batch_workspace_size")
    if workspace is None or workspace.numel() < need.value:
        workspace = torch.empty(max(1, need.value), dtype=torch.uint8, device=entries[0][0].device)
    L.check(lib.mtb_grid_batch(jobs, len(entries), _ptr(workspace), need.value, _stream(stream)),
            "mtb_grid_batch")
    for im, *_ in entries:
        im._fresh = False
    return workspace


TUNING_KEYS = ("tile", "support_bucket", "max_chunk", "gridder_threads", "gridder")


def autotune(entries, workspace=None, stream=None):
    """Choose the gridder knobs (tile, support_bucket, max_chunk,
    gridder_threads, gridder) for a batch by timing every candidate on this chunk
    (mtb_grid_autotune).  entries as for grid_batch; every imager must start a
    fresh image.  The chosen knobs are set on every imager (later chunks use
    them) and its grid holds this chunk gridded with them.  Returns (best,
    candidates, workspace): dicts with the knobs and the measured ms."""
    if not entries:
        raise ValueError("no images to tune")
    if not all(im._fresh for im, *_ in entries):
        raise ValueError("autotune needs fresh images (reset() first)")
    lib = L.load()
    jobs, keep = _batch_jobs(entries)
    need = ctypes.c_size_t(0)
    L.check(lib.mtb_grid_autotune_workspace_size(jobs, len(entries), ctypes.byref(need)),
            "mtb_grid_autotune_workspace_size")
    if workspace is None or workspace.numel() < need.value:
        workspace = torch.empty(max(1, need.value), dtype=torch.uint8, device=entries[0][0].device)
    best = L.GridTuning()
    cands = (L.GridTuning * lib.mtb_grid_autotune_candidate_count())()
    L.check(lib.mtb_grid_autotune(jobs, len(entries), _ptr(workspace), need.value, _stream(stream),
                                  ctypes.byref(best), cands), "mtb_grid_autotune")
    as_dict = lambda t: dict({k: getattr(t, k) for k in TUNING_KEYS}, ms=t.ms)  # noqa: E731
    for im, *_ in entries:
        im.tuning.update({k: getattr(best, k) for k in TUNING_KEYS})
        im._fresh = False
    return as_dict(best), [as_dict(c) for c in cands], workspace
