"""ctypes binding of libmtb.so (the C ABI declared in include/mtb.h).

The library is the product: there is no Python or CPU implementation of any
kernel behind this module.  If libmtb.so is missing the import of the compute
entry points fails loudly.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
# MTB_LIBRARY=checked selects the bounds-checked build (build.py --checked)
LIB_PATH = os.path.join(PKG, "libmtb_checked.so" if os.environ.get("MTB_LIBRARY") == "checked" else "libmtb.so")

# status codes (include/mtb.h)
MTB_OK = 0
MTB_ERR_BAD_PARAM = 1
MTB_ERR_BAD_SHAPE = 2
MTB_ERR_WORKSPACE = 3
MTB_ERR_CAPACITY = 4
MTB_ERR_CUDA = 5
MTB_ERR_CUFFT = 6
MTB_ERR_KERNEL = 7
MTB_ERR_NULL = 8
MTB_ERR_TOO_LARGE = 9
MTB_ERR_CANCELLED = 10
MTB_POL_LINEAR = 0
MTB_POL_CIRCULAR = 1

# every entry point include/mtb.h declares
EXPORTS = (
    "mtb_wkernel_query", "mtb_wkernel_build", "mtb_grid_workspace_size", "mtb_grid", "mtb_preprocess_uvw",
    "mtb_preprocess_uvw_noalloc", "mtb_preprocess_uvw_noalloc_capacity",
    "mtb_finalize_workspace_size", "mtb_finalize", "mtb_finalize_planes_bytes", "mtb_grid_delta_bytes",
    "mtb_status_string", "mtb_version",
    "mtb_release_caches", "mtb_kernel_launch_count", "mtb_calibrate_fp32",
    "mtb_taper_kernel_build", "mtb_grid_batch_workspace_size", "mtb_grid_batch",
    "mtb_grid_autotune_workspace_size", "mtb_grid_autotune", "mtb_grid_autotune_candidate_count", "mtb_sort_index", "mtb_gather_rows", "mtb_fits_create", "mtb_fits_write_channel", "mtb_fits_close",
    "mtb_engine_create", "mtb_engine_submit", "mtb_engine_wait", "mtb_engine_cancel", "mtb_engine_request_bytes",
    "mtb_engine_destroy", "mtb_bounds_status", "mtb_lsrk_workspace_size", "mtb_lsrk_freq_over_c",
)


class MtbError(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        msg = _lib.mtb_status_string(status).decode() if _lib is not None else str(status)
        super().__init__("%s failed: %s (status %d)" % (where, msg, status))


class WKernelParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("l_increment", ctypes.c_double),
                ("m_increment", ctypes.c_double), ("wplanes", ctypes.c_int), ("sampling", ctypes.c_int),
                ("trial_support", ctypes.c_int), ("max_support", ctypes.c_int), ("w_max", ctypes.c_double)]


class LsrkParams(ctypes.Structure):
    _fields_ = [("site_itrf", ctypes.c_double * 3), ("ra", ctypes.c_double), ("dec", ctypes.c_double),
                ("tt_minus_time", ctypes.c_double), ("ut1_minus_time", ctypes.c_double)]


class WKernelInfo(ctypes.Structure):
    _fields_ = [("trial_support", ctypes.c_int), ("planesize", ctypes.c_int), ("support_cap", ctypes.c_int),
                ("T", ctypes.c_int), ("w_max", ctypes.c_double), ("w_sq_increment", ctypes.c_double),
                ("total_l", ctypes.c_double), ("total_m", ctypes.c_double), ("u_increment", ctypes.c_double),
                ("v_increment", ctypes.c_double), ("table_capacity", ctypes.c_size_t),
                ("workspace_bytes", ctypes.c_size_t)]


class GridParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("npol", ctypes.c_int), ("sampling", ctypes.c_int),
                ("wplanes", ctypes.c_int), ("u_increment", ctypes.c_double), ("v_increment", ctypes.c_double),
                ("w_sq_increment", ctypes.c_double), ("initialize_output", ctypes.c_int), ("tile", ctypes.c_int),
                ("support_bucket", ctypes.c_int), ("max_chunk", ctypes.c_int), ("merge", ctypes.c_int),
                ("gridder_start_event", ctypes.c_void_p), ("gridder_end_event", ctypes.c_void_p),
                ("bulk_min_support", ctypes.c_int), ("psf", ctypes.c_int), ("exact_delta", ctypes.c_int),
                ("gridder_threads", ctypes.c_int), ("gridder", ctypes.c_int), ("flags_u8", ctypes.c_int),
                ("no_grid_lo", ctypes.c_int), ("external_delta", ctypes.c_int), ("d_delta", ctypes.c_void_p)]


class GridStats(ctypes.Structure):
    _fields_ = [("gridded_records", ctypes.c_ulonglong), ("compressed_records", ctypes.c_ulonglong),
                ("gridded_points", ctypes.c_ulonglong), ("compressed_points", ctypes.c_ulonglong)]


class FinalizeParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("npol", ctypes.c_int), ("sampling", ctypes.c_int),
                ("pol_type", ctypes.c_int), ("external_planes", ctypes.c_int), ("d_planes", ctypes.c_void_p)]


class GridJob(ctypes.Structure):
    _fields_ = [("params", GridParams), ("d_table", ctypes.c_void_p), ("d_conv_info", ctypes.c_void_p),
                ("h_conv_info", ctypes.c_void_p), ("d_conv_sums", ctypes.c_void_p), ("d_uvw", ctypes.c_void_p),
                ("d_freq", ctypes.c_void_p), ("d_vis", ctypes.c_void_p), ("d_weights", ctypes.c_void_p),
                ("d_flags", ctypes.c_void_p), ("nrecords", ctypes.c_int), ("d_grid", ctypes.c_void_p),
                ("d_grid_lo", ctypes.c_void_p), ("d_normalizer", ctypes.c_void_p), ("d_stats", ctypes.c_void_p)]


class FitsHeader(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nstokes", ctypes.c_int), ("nchan", ctypes.c_int),
                ("l_increment", ctypes.c_double), ("m_increment", ctypes.c_double), ("ra_deg", ctypes.c_double),
                ("dec_deg", ctypes.c_double), ("freqs_hz", ctypes.c_void_p), ("stokes", ctypes.c_void_p),
                ("telescope", ctypes.c_char_p), ("observer", ctypes.c_char_p), ("obs_mjd", ctypes.c_double)]


class GridTuning(ctypes.Structure):
    _fields_ = [("tile", ctypes.c_int), ("support_bucket", ctypes.c_int), ("max_chunk", ctypes.c_int),
                ("gridder_threads", ctypes.c_int), ("gridder", ctypes.c_int), ("ms", ctypes.c_float)]


class EngineConfig(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_size_t),
                ("kernel_cache_bytes", ctypes.c_size_t), ("chunk_records", ctypes.c_int),
                ("host_threads", ctypes.c_int)]


class ImageRequest(ctypes.Structure):
    _fields_ = [("geometry", WKernelParams), ("npol", ctypes.c_int), ("pol_type", ctypes.c_int),
                ("compensated", ctypes.c_int), ("nrecords", ctypes.c_int), ("uvw", ctypes.c_void_p),
                ("freq", ctypes.c_void_p), ("vis", ctypes.c_void_p), ("weights", ctypes.c_void_p),
                ("flags", ctypes.c_void_p), ("image", ctypes.c_void_p), ("exact_delta", ctypes.c_int),
                ("uvw_row_stride", ctypes.c_longlong), ("flags_u8", ctypes.c_int)]


class ImageResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("kernel_cache_hit", ctypes.c_int), ("queue_ms", ctypes.c_double),
                ("service_ms", ctypes.c_double), ("latency_ms", ctypes.c_double), ("stats", GridStats)]


_lib = None


def load(path: str = LIB_PATH):
    """Load libmtb.so and declare the prototypes.  Raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("%s not found: build it with python mt-imager_b200/build.py%s"
                           % (path, " --checked" if path.endswith("_checked.so") else ""))
    L = ctypes.CDLL(path)
    p, i, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
    L.mtb_wkernel_query.argtypes = [ctypes.POINTER(WKernelParams), ctypes.POINTER(WKernelInfo)]
    L.mtb_wkernel_build.argtypes = [ctypes.POINTER(WKernelParams), p, sz, p, sz, p, p, p,
                                    ctypes.POINTER(sz), p]
    L.mtb_grid_workspace_size.argtypes = [ctypes.POINTER(GridParams), p, i, ctypes.POINTER(sz)]
    L.mtb_grid.argtypes = [ctypes.POINTER(GridParams), p, p, p, p, p, p, p, p, p, i, p, p, p, p, p, sz, p]
    L.mtb_preprocess_uvw.argtypes = [ctypes.POINTER(GridParams), p, p, p, p, p, p, p, i] + [p] * 8 + [sz, p]
    L.mtb_preprocess_uvw_noalloc.argtypes = [ctypes.POINTER(GridParams), p, p, p, p, p, p, p, i] + [p] * 7 + [p]
    L.mtb_preprocess_uvw_noalloc_capacity.argtypes = []
    L.mtb_taper_kernel_build.argtypes = [i, i, p, sz, p, p, p, ctypes.POINTER(sz), p]
    L.mtb_finalize_workspace_size.argtypes = [ctypes.POINTER(FinalizeParams), ctypes.POINTER(sz)]
    L.mtb_finalize.argtypes = [ctypes.POINTER(FinalizeParams), p, p, p, p, p, sz, p]
    L.mtb_finalize_planes_bytes.argtypes = [ctypes.POINTER(FinalizeParams), ctypes.POINTER(sz)]
    L.mtb_grid_delta_bytes.argtypes = [ctypes.POINTER(GridParams), ctypes.POINTER(sz)]
    for name in EXPORTS:
        getattr(L, name).restype = i
    L.mtb_status_string.restype = ctypes.c_char_p
    L.mtb_status_string.argtypes = [i]
    L.mtb_version.argtypes = []
    L.mtb_release_caches.restype = None
    L.mtb_release_caches.argtypes = []
    L.mtb_kernel_launch_count.restype = ctypes.c_ulonglong
    L.mtb_kernel_launch_count.argtypes = []
    L.mtb_calibrate_fp32.argtypes = [ctypes.POINTER(ctypes.c_double), p]
    L.mtb_grid_batch_workspace_size.argtypes = [ctypes.POINTER(GridJob), i, ctypes.POINTER(sz)]
    L.mtb_grid_batch.argtypes = [ctypes.POINTER(GridJob), i, p, sz, p]
    L.mtb_sort_index.argtypes = [p, p, i, i, p, ctypes.POINTER(i)]
    L.mtb_gather_rows.argtypes = [p, sz, sz, sz, p, i, p, i]
    L.mtb_grid_autotune_workspace_size.argtypes = [ctypes.POINTER(GridJob), i, ctypes.POINTER(sz)]
    L.mtb_grid_autotune_candidate_count.argtypes = []
    L.mtb_grid_autotune.argtypes = [ctypes.POINTER(GridJob), i, p, sz, p, ctypes.POINTER(GridTuning),
                                    ctypes.POINTER(GridTuning)]
    L.mtb_fits_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(FitsHeader), ctypes.POINTER(p)]
    L.mtb_fits_write_channel.argtypes = [p, i, p]
    L.mtb_fits_close.argtypes = [p]
    L.mtb_engine_create.argtypes = [ctypes.POINTER(EngineConfig), ctypes.POINTER(p)]
    L.mtb_engine_submit.argtypes = [p, ctypes.POINTER(ImageRequest), ctypes.POINTER(ctypes.c_longlong)]
    L.mtb_engine_wait.argtypes = [p, ctypes.c_longlong, ctypes.POINTER(ImageResult)]
    L.mtb_engine_cancel.argtypes = [p, ctypes.c_longlong]
    L.mtb_bounds_status.argtypes = [ctypes.POINTER(i), ctypes.POINTER(ctypes.c_uint)]
    L.mtb_engine_request_bytes.argtypes = [p, ctypes.POINTER(ImageRequest), ctypes.POINTER(sz)]
    L.mtb_engine_destroy.argtypes = [p]
    L.mtb_lsrk_workspace_size.argtypes = [i, ctypes.POINTER(sz)]
    L.mtb_lsrk_freq_over_c.argtypes = [ctypes.POINTER(LsrkParams), p, i, p, i, p, i, p, p, sz, p]
    _lib = L
    return L


def check(status: int, where: str):
    if status != MTB_OK:
        raise MtbError(status, where)
