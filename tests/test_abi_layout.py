"""Every struct the Python binding passes across the C ABI has the size and
field offsets the C headers give it (a C program compiled with gcc against
include/*.h prints them), and host-side parameter checks refuse bad input
before any CUDA call.  No GPU."""
import ctypes
import os
import subprocess

import pytest

from mtb import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "mtb_wkernel_params": L.WKernelParams,
    "mtb_wkernel_info": L.WKernelInfo,
    "mtb_grid_params": L.GridParams,
    "mtb_grid_stats": L.GridStats,
    "mtb_finalize_params": L.FinalizeParams,
    "mtb_grid_job": L.GridJob,
    "mtb_grid_tuning": L.GridTuning,
    "mtb_fits_header": L.FitsHeader,
    "mtb_engine_config": L.EngineConfig,
    "mtb_image_request": L.ImageRequest,
    "mtb_image_result": L.ImageResult,
}


@pytest.fixture(scope="module")
def c_layouts(tmp_path_factory):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "mtb.h"', '#include "mtb_engine.h"',
             '#include "mtb_fits.h"', 'int main(void) {']
    for cname, py in STRUCTS.items():
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for f, _ in py._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, f, cname, f))
    lines += ['return 0;', '}']
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines))
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        a, b, v = line.split()
        out[(a, b)] = int(v)
    return out


@pytest.mark.parametrize("cname", sorted(STRUCTS))
def test_struct_matches_header(c_layouts, cname):
    py = STRUCTS[cname]
    assert ctypes.sizeof(py) == c_layouts[(cname, "size")], cname
    for f, _ in py._fields_:
        assert getattr(py, f).offset == c_layouts[(cname, f)], (cname, f)


def test_autotune_refuses_images_that_are_not_fresh(mtblib):
    jobs = (L.GridJob * 1)()
    jobs[0].params.initialize_output = 0
    best = L.GridTuning()
    rc = mtblib.mtb_grid_autotune(jobs, 1, None, 0, None, ctypes.byref(best), None)
    assert rc == L.MTB_ERR_BAD_PARAM
    assert mtblib.mtb_grid_autotune(jobs, 0, None, 0, None, ctypes.byref(best), None) == L.MTB_ERR_BAD_SHAPE
    n = ctypes.c_size_t(0)
    assert mtblib.mtb_grid_autotune_workspace_size(jobs, 65, ctypes.byref(n)) == L.MTB_ERR_BAD_SHAPE


def test_batch_refuses_mixed_gridder_block_sizes(mtblib):
    jobs = (L.GridJob * 2)()
    info = (ctypes.c_int * 2)(7, 0)
    for j, thr in enumerate((256, 512)):
        p = jobs[j].params
        p.nx = p.ny = 64
        p.npol, p.sampling, p.wplanes = 4, 4, 1
        p.u_increment = p.v_increment = p.w_sq_increment = 1.0
        p.gridder_threads = thr
        jobs[j].h_conv_info = ctypes.cast(info, ctypes.c_void_p)
    n = ctypes.c_size_t(0)
    assert mtblib.mtb_grid_batch_workspace_size(jobs, 2, ctypes.byref(n)) == L.MTB_ERR_BAD_PARAM
    jobs[1].params.gridder_threads = 300
    assert mtblib.mtb_grid_batch_workspace_size(jobs, 2, ctypes.byref(n)) == L.MTB_ERR_BAD_PARAM


def test_status_codes_match_header():
    import re
    src = open(os.path.join(ROOT, "include", "mtb.h")).read()
    codes = {m.group(1): int(m.group(2)) for m in re.finditer(r"\b(MTB_(?:OK|ERR_\w+))\s*=\s*(\d+)", src)}
    assert len(codes) == 11
    for name, v in codes.items():
        assert getattr(L, name) == v, name


@pytest.mark.parametrize("support,tile,status", [(255, 0, L.MTB_OK), (257, 0, L.MTB_ERR_KERNEL),
                                                 (16, 0, L.MTB_ERR_KERNEL), (7, 2, L.MTB_ERR_BAD_PARAM)])
def test_plan_limits(mtblib, support, tile, status):
    """The direct gridders lay one support-box column per thread of a block:
    supports are odd and at most 255; tiles at least 4 cells.  Refused on the
    host, before any device work."""
    p = L.GridParams()
    p.nx = p.ny = 1024
    p.npol, p.sampling, p.wplanes = 4, 4, 1
    p.u_increment = p.v_increment = p.w_sq_increment = 1.0
    p.tile = tile
    info = (ctypes.c_int * 2)(support, 0)
    n = ctypes.c_size_t(0)
    rc = mtblib.mtb_grid_workspace_size(ctypes.byref(p), ctypes.cast(info, ctypes.c_void_p), 1000, ctypes.byref(n))
    if status == L.MTB_OK and rc != L.MTB_OK:
        pytest.skip("workspace query needs the device on this host (status %d)" % rc)
    assert rc == status


def test_imager_refuses_a_cpu_device():
    from mtb.imager import WProjectionImager
    with pytest.raises(ValueError):
        WProjectionImager(64, 64, 1e-4, device="cpu")


def test_kernel_builders_refuse_a_cpu_device():
    from mtb.imager import build_taper_kernels, build_wkernels, wkernel_params
    with pytest.raises(ValueError):
        build_wkernels(wkernel_params(64, 64, 1e-4, 1e-4, 4, 4), device="cpu")
    with pytest.raises(ValueError):
        build_taper_kernels(64, 64, 1e-4, 1e-4, device="cpu")


def test_entry_points_report_a_missing_device():
    """Without a CUDA device the entry points that need one return
    MTB_ERR_CUDA (no host fallback, no crash), and the engine calls refuse
    null handles before touching the device."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib = L.load()
    h = ctypes.c_void_p(123)
    assert lib.mtb_engine_create(None, ctypes.byref(h)) == L.MTB_ERR_CUDA
    assert h.value is None                      # no engine handed out on failure
    t = ctypes.c_double(-1.0)
    assert lib.mtb_calibrate_fp32(ctypes.byref(t), None) == L.MTB_ERR_CUDA
    # the w-kernel query sizes the cuFFT work area, which needs the device
    p = L.WKernelParams(nx=256, ny=256, l_increment=1e-5, m_increment=1e-5, wplanes=32, sampling=8)
    assert lib.mtb_wkernel_query(ctypes.byref(p), ctypes.byref(L.WKernelInfo())) == L.MTB_ERR_CUDA
    assert lib.mtb_status_string(L.MTB_ERR_CUDA)
    ticket = ctypes.c_longlong()
    req = L.ImageRequest()
    assert lib.mtb_engine_submit(None, ctypes.byref(req), ctypes.byref(ticket)) == L.MTB_ERR_NULL
    assert lib.mtb_engine_wait(None, 1, ctypes.byref(L.ImageResult())) == L.MTB_ERR_NULL
    assert lib.mtb_engine_destroy(None) == L.MTB_ERR_NULL


def _valid_grid_params():
    p = L.GridParams()
    p.nx = p.ny = 1024
    p.npol, p.sampling, p.wplanes = 4, 4, 1
    p.u_increment = p.v_increment = p.w_sq_increment = 1.0
    return p


@pytest.mark.parametrize("field,value,status", [
    ("nx", 65536, L.MTB_ERR_BAD_SHAPE),        # with ny = 65536: 2^32 cells, above the 2^31-cell limit
    ("npol", 3, L.MTB_ERR_BAD_SHAPE),
    ("nx", 1, L.MTB_ERR_BAD_PARAM),
    ("sampling", 0, L.MTB_ERR_BAD_PARAM),
    ("wplanes", 0, L.MTB_ERR_BAD_PARAM),
    ("u_increment", 0.0, L.MTB_ERR_BAD_PARAM),
    ("w_sq_increment", float("nan"), L.MTB_ERR_BAD_PARAM),
    ("merge", 3, L.MTB_ERR_BAD_PARAM),
    ("gridder_threads", 384, L.MTB_ERR_BAD_PARAM),
    ("gridder", 4, L.MTB_ERR_BAD_PARAM),
    ("gridder", 9, L.MTB_ERR_BAD_PARAM),
    ("bulk_min_support", 17, L.MTB_ERR_BAD_PARAM),   # reserved: the bulk-copy gridder was removed
    ("max_chunk", -1, L.MTB_ERR_BAD_PARAM),
])
def test_grid_parameter_refusals(mtblib, field, value, status):
    """Out-of-range gridding parameters are refused on the host with the
    status the reference's ValidationException cases map to, before any
    device work (so without a GPU too)."""
    p = _valid_grid_params()
    if field == "nx" and value == 65536:
        p.ny = 65536                            # 2^32 cells
    setattr(p, field, value)
    info = (ctypes.c_int * 2)(7, 0)
    n = ctypes.c_size_t(0)
    rc = mtblib.mtb_grid_workspace_size(ctypes.byref(p), ctypes.cast(info, ctypes.c_void_p), 1000, ctypes.byref(n))
    assert rc == status


def test_grid_refuses_negative_records_and_rolling_512(mtblib):
    info = (ctypes.c_int * 2)(7, 0)
    n = ctypes.c_size_t(0)
    p = _valid_grid_params()
    assert mtblib.mtb_grid_workspace_size(ctypes.byref(p), ctypes.cast(info, ctypes.c_void_p), -1,
                                          ctypes.byref(n)) == L.MTB_ERR_BAD_SHAPE
    for g in (5, 7, 8):                       # the rolling and streaming gridders take no block size
        p.gridder, p.gridder_threads = g, 512
        assert mtblib.mtb_grid_workspace_size(ctypes.byref(p), ctypes.cast(info, ctypes.c_void_p), 10,
                                              ctypes.byref(n)) == L.MTB_ERR_BAD_PARAM
    assert mtblib.mtb_grid_workspace_size(None, ctypes.cast(info, ctypes.c_void_p), 10,
                                          ctypes.byref(n)) == L.MTB_ERR_NULL


@pytest.mark.parametrize("nx,ny,npol,s,pol,status", [
    (1024, 1024, 3, 8, 0, L.MTB_ERR_BAD_SHAPE),
    (1, 1024, 4, 8, 0, L.MTB_ERR_BAD_PARAM),
    (1024, 1024, 4, 0, 0, L.MTB_ERR_BAD_PARAM),
    (1024, 1024, 4, 8, 2, L.MTB_ERR_BAD_PARAM),      # neither linear nor circular feeds
    (65536, 65536, 4, 8, 0, L.MTB_ERR_BAD_SHAPE),    # 2^32 cells
])
def test_finalize_parameter_refusals(mtblib, nx, ny, npol, s, pol, status):
    p = L.FinalizeParams(nx=nx, ny=ny, npol=npol, sampling=s, pol_type=pol)
    n = ctypes.c_size_t(0)
    assert mtblib.mtb_finalize_workspace_size(ctypes.byref(p), ctypes.byref(n)) == status
    assert mtblib.mtb_finalize(ctypes.byref(p), None, None, None, None, None, 0, None) == status


@pytest.mark.parametrize("kw,status", [
    (dict(trial_support=32), L.MTB_ERR_BAD_PARAM),            # supports are odd (WProjPreFFTconvFunc.cpp:77)
    (dict(nx=1), L.MTB_ERR_BAD_PARAM),
    (dict(l_increment=0.0), L.MTB_ERR_BAD_PARAM),
    (dict(wplanes=0), L.MTB_ERR_BAD_PARAM),
    (dict(nx=4, ny=4), L.MTB_ERR_BAD_PARAM),                  # trial support 4/8 -> 1: no kernel
    (dict(trial_support=6001), L.MTB_ERR_BAD_SHAPE),          # (S_t * s)^2 screen above 2^31 elements
])
def test_wkernel_parameter_refusals(mtblib, kw, status):
    """The w-kernel parameters are checked on the host before the cuFFT plan
    (and so before any device is needed)."""
    base = dict(nx=256, ny=256, l_increment=1e-5, m_increment=1e-5, wplanes=32, sampling=8)
    base.update(kw)
    p = L.WKernelParams(**base)
    assert mtblib.mtb_wkernel_query(ctypes.byref(p), ctypes.byref(L.WKernelInfo())) == status


def _ws(mtblib, p, records=1000):
    info = (ctypes.c_int * 2)(7, 0)
    n = ctypes.c_size_t(0)
    assert mtblib.mtb_grid_workspace_size(ctypes.byref(p), ctypes.cast(info, ctypes.c_void_p), records,
                                          ctypes.byref(n)) == L.MTB_OK
    return n.value


def test_workspace_delta_grid_by_mode(mtblib):
    """The per-call delta grid is sized by the accumulation mode: none for
    calls without grid_lo (no_grid_lo) or with the shared-memory tile merge,
    8 bytes per cell and polarisation for the FP32 delta, 16 for the FP64 one
    (exact_delta, or work items shorter than 128 records, which always use it)."""
    cells = 1024 * 1024 * 4
    base = _valid_grid_params()
    p = L.GridParams.from_buffer_copy(base)
    p.no_grid_lo = 1
    none = _ws(mtblib, p)
    fp32 = _ws(mtblib, base)
    p = L.GridParams.from_buffer_copy(base)
    p.exact_delta = 1
    fp64 = _ws(mtblib, p)
    p = L.GridParams.from_buffer_copy(base)
    p.max_chunk = 64
    short = _ws(mtblib, p)
    p = L.GridParams.from_buffer_copy(base)
    p.merge = 1
    window = _ws(mtblib, p)
    assert abs((fp32 - none) - 8 * cells) < 512
    assert abs((fp64 - none) - 16 * cells) < 512
    assert abs((short - none) - 16 * cells) < 512      # short items use the FP64 delta
    assert abs(window - none) < 512
    p = L.GridParams.from_buffer_copy(base)
    p.max_chunk = 128
    assert abs(_ws(mtblib, p) - fp32) < 512             # at the safe length the FP32 delta stays
