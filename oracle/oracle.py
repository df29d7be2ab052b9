"""TEST INFRASTRUCTURE, NOT PRODUCT CODE.

FP64 restatement of mt-imager's W-projection imaging path (the checker).
Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline/reference
legs import this module; the product library in mt-imager_b200/ never does.

The per-element work lives in ``wproj_oracle.c`` (compiled here with gcc,
``-ffp-contract=off``); the FFTs are numpy's pocketfft in complex128.  Each
function names the reference step it restates (paths relative to the
reference project's ``code/`` directory).

Parity anchors: the reference ships no tests, fixtures or golden vectors.
This restatement is pinned (tests/test_golden.py) against outputs of
mt-imager's own operator code -- its sources compiled unchanged by
oracle/build_ref.py and run on a GPU by tests/golden/make_golden.py -- and by
the known-answer tests in tests/test_oracle.py (w=0 kernel DC = 1, point
sources imaged where the direct FP64 DFT puts them, chunk invariance,
Hermitian conjugation of w<0 records).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
SRC = os.path.join(HERE, "wproj_oracle.c")
PORT_SRC = os.path.join(HERE, "cpu_port.c")

# ConvFunctionSupportFind takes (1e-3f)^2 (WPlaneConvFunctionCalculator.cpp:61,
# ConvFunctionSupportFind.cu:99)
TAKE_AS_ZERO2 = float(np.float32(1e-3)) ** 2

_lib = None
_port = None


def _compile(src, out, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    if os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    tmp = out + ".tmp%d" % os.getpid()
    cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-o", tmp, src, "-lm", *extra]
    subprocess.check_call(cmd)
    os.replace(tmp, out)
    return out


def _port_path():
    """The CPU port is built with -march=native, so its file name carries a
    digest of this host's CPU model and flags: a copy built on another CPU
    (whose instructions this one may lack) is never loaded; it is rebuilt."""
    import hashlib
    key = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("model name", "flags")):
                    key += line
                if line.startswith("flags"):
                    break
    except OSError:
        pass
    tag = hashlib.sha1(key.encode()).hexdigest()[:12] if key else "generic"
    return os.path.join(BUILD, "libcpu_port-%s.so" % tag)


def build():
    """Compile the oracle (and the FP32 CPU port) shared libraries."""
    _compile(SRC, os.path.join(BUILD, "liboracle_wproj.so"))
    if os.path.exists(PORT_SRC):
        _compile(PORT_SRC, _port_path(), extra=("-O3", "-march=native"))


def lib():
    global _lib
    if _lib is None:
        path = _compile(SRC, os.path.join(BUILD, "liboracle_wproj.so"))
        L = ctypes.CDLL(path)
        d, i, p = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        L.orc_grdsf.restype = d
        L.orc_grdsf.argtypes = [d]
        L.orc_taper_lm.argtypes = [i, i, p]
        L.orc_gridsf_uv.argtypes = [i, i, p]
        L.orc_wscreen.argtypes = [p, i, i, d, d, d, i, p]
        L.orc_zero_to_centre.argtypes = [p, p, i, i]
        L.orc_support_find.restype = i
        L.orc_support_find.argtypes = [p, i, i, d]
        L.orc_reorganize.argtypes = [p, i, i, i, p]
        L.orc_conv_sums.argtypes = [p, p, i, i, p]
        L.orc_preprocess.argtypes = [i, i, p, p, p, p, i, d, p, p, i, i, i, d, d] + [p] * 10
        L.orc_compress_vis.argtypes = [i, i, p, p, p, p, p, p, p]
        L.orc_grid.argtypes = [i, i, p, p, p, p, p, p, i, i, p]
        L.orc_dft.argtypes = [i, i, p, p, p, i, i, d, d, p]
        L.orc_origin_to_corner.restype = i
        L.orc_origin_to_corner.argtypes = [i, i]
        L.orc_origin_to_centre.restype = i
        L.orc_origin_to_centre.argtypes = [i, i]
        _lib = L
    return _lib


def port():
    """FP32 OpenMP transcription of the reference's gridding (cpu_port.c),
    the CPU baseline bench.py times."""
    global _port
    if _port is None:
        path = _compile(PORT_SRC, _port_path(), extra=("-O3", "-march=native"))
        P = ctypes.CDLL(path)
        i, p, f = ctypes.c_int, ctypes.c_void_p, ctypes.c_float
        P.port_threads.restype = i
        P.port_set_threads.restype = None
        P.port_set_threads.argtypes = [i]
        # every core this process may run on, whatever OMP_NUM_THREADS says
        P.port_set_threads(len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count())
        P.port_grid_chunk.restype = i
        P.port_grid_chunk.argtypes = [i, i, p, p, p, p, p, i, f, p, p, p, i, i, i, f, f, p, p, p]
        _port = P
    return _port


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# ------------------------------------------------------------ parameters --
def kernel_geometry(nx, ny, dl, dm, wplanes, sampling, trial_support=0, max_support=0, w_max=0.0):
    """Scalars of WProjectionConvFunction (WProjectionConvFunction.cpp:105-112,
    194-198) and ConfigurationManager (ConfigurationManager.cpp:173-202).
    trial_support / max_support / w_max of 0 select the reference's rules."""
    img_min = min(nx, ny)
    if trial_support <= 0:
        st = img_min // sampling
        if st % 2 == 0:
            st += 1
    else:
        st = int(trial_support)
        if st % 2 == 0:
            raise ValueError("trial support must be odd")
    cap = st - 2
    if max_support > 0:
        cap = min(cap, int(max_support))
    wmax = 0.25 / dl if w_max <= 0 else float(w_max)
    w_inc = 1.0 if wplanes == 1 else wmax / float((wplanes - 1) * (wplanes - 1))
    T = sampling if sampling % 2 else sampling + 1
    return dict(trial_support=st, planesize=st * sampling, support_cap=cap, w_max=wmax,
                w_inc=w_inc, total_l=dl * nx, total_m=dm * ny, T=T, sampling=sampling,
                wplanes=wplanes, du=1.0 / (dl * nx), dv=1.0 / (dm * ny), nx=nx, ny=ny)


def geometry_for(setup):
    return kernel_geometry(setup.nx, setup.ny, setup.dl, setup.dl, setup.wplanes, setup.sampling,
                           setup.trial_support, setup.max_support, setup.w_max)


# ------------------------------------------------------- w-kernel tables --
def taper_lm(n):
    out = np.empty((n, n), np.float64)
    lib().orc_taper_lm(n, n, _p(out))
    return out


def wscreen(taper, st, s, total_l, total_m, w, leavedge=0):
    ps = st * s
    out = np.empty((ps, ps), np.complex128)
    lib().orc_wscreen(_p(np.ascontiguousarray(taper)), st, s, total_l, total_m, float(w), leavedge, _p(out))
    return out


def zero_to_centre(a):
    out = np.empty_like(a)
    lib().orc_zero_to_centre(_p(np.ascontiguousarray(a)), _p(out), a.shape[0], a.shape[1])
    return out


def wkernels(geo):
    """All w-plane kernels: WProjectionConvFunction::calculate
    (WProjectionConvFunction.cpp:186-291) driving WPlaneConvFunctionCalculator
    (WPlaneConvFunctionCalculator.cpp:40-67: taper -> WProjPreFFTConvFunc ->
    multiFFT2D FORWARD -> ZeroToCentre2DShift -> SingleMultiply ->
    ConvFunctionSupportFind) and ConvFunctionReOrganize / ArraysToVector /
    SumConvolutionFunctions.  Returns dict(table complex128 1-D, conv_info
    int32 [nw][2], conv_sums float64 [nw][T*T], multiplier, supports)."""
    st, s, nw, T = geo["trial_support"], geo["sampling"], geo["wplanes"], geo["T"]
    ps = st * s
    taper = taper_lm(st)
    # DC divisor from the unshifted FFT of the w=0 screen (WPlaneConvFunctionCalculator.cpp:128-142)
    f0 = np.fft.fft2(wscreen(taper, st, s, geo["total_l"], geo["total_m"], 0.0))
    divisor = f0[0, 0]
    if divisor.imag > 1e-3:
        raise ValueError("w=0 kernel origin has a non-zero imaginary part")
    mult = 1.0 / divisor.real
    tables, info, sups = [], np.zeros((nw, 2), np.int32), []
    offset = 0
    for k in range(nw):
        w = k * k * geo["w_inc"]
        f = np.fft.fft2(wscreen(taper, st, s, geo["total_l"], geo["total_m"], w))
        c = np.ascontiguousarray(zero_to_centre(f) * mult)
        sup = lib().orc_support_find(_p(c), ps, s, TAKE_AS_ZERO2)
        sup = min(sup, geo["support_cap"])
        if sup < 1:
            raise ValueError("w-plane %d has no kernel support" % k)
        out = np.empty(T * T * sup * sup, np.complex128)
        lib().orc_reorganize(_p(c), ps, sup, s, _p(out))
        tables.append(out)
        info[k] = (sup, offset)
        sups.append(sup)
        offset += out.size
    table = np.concatenate(tables)
    sums = np.empty((nw, T * T), np.float64)
    lib().orc_conv_sums(_p(table), _p(info), nw, T, _p(sums))
    return dict(table=table, conv_info=info, conv_sums=sums, multiplier=mult, supports=np.array(sups),
                divisor=divisor)


def taper_kernels(support, sampling):
    """mode=normal kernel table (OnlyTaperConvFunction.cpp:29-99): the uv
    gridding function of CasaGridSF.cu:107-149 -- per axis (1 - nu^2) grdsf(nu),
    nu = d / (3 s) for offsets d < 3 s from the centre of a (S s [+1 for even
    s])^2 array -- cut by ConvFunctionReOrganize.cu:30-71 into one plane of
    [oy][ox][sy][sx] sub-kernels, with SumConvolutionFunctions.cu:29-56 sums."""
    S, s = int(support), int(sampling)
    T = s if s % 2 else s + 1
    dim = S * s + (0 if s % 2 else 1)
    zero_at = 3 * s
    g = lib().orc_grdsf

    def f(d):
        d = abs(d)
        if d >= zero_at:
            return 0.0
        nu = d / zero_at
        return (1.0 - nu * nu) * g(nu)

    axis = np.array([f(i - dim // 2) for i in range(dim)])
    full = np.outer(axis, axis)
    cb = dim // 2 - ((S // 2) * s + s // 2)
    table = np.zeros((T, T, S, S), np.complex128)
    for oy in range(T):
        for ox in range(T):
            rows = np.arange(S) * s + oy + cb
            cols = np.arange(S) * s + ox + cb
            table[oy, ox] = full[np.ix_(rows, cols)]
    table = table.reshape(-1)
    sums = table.real.reshape(T * T, S * S).sum(axis=1)[None, :]
    return dict(table=table, conv_info=np.array([[S, 0]], np.int32), conv_sums=sums, supports=np.array([S]))


# ------------------------------------------------------------ preprocess --
def preprocess(uvw, freq, weights, flags, geo, kern):
    """PreProcessUVW (WProjPreProcessUVW.cu:112-324) in FP64."""
    uvw = np.ascontiguousarray(uvw, np.float32)
    freq = np.ascontiguousarray(freq, np.float32)
    weights = np.ascontiguousarray(weights, np.float32)
    flags = np.ascontiguousarray(flags, np.int32)
    R, P = weights.shape
    o = dict(loc=np.zeros((R, 4), np.int32), convidx=np.zeros(R, np.int32), togrid=np.zeros(R, np.int32),
             compress=np.zeros(R, np.int32), support=np.zeros(R, np.int32), plane=np.zeros(R, np.int32),
             offx=np.zeros(R, np.int32), offy=np.zeros(R, np.int32), imgmult=np.zeros(R, np.float32),
             convsum=np.zeros((P, R), np.float64))
    if R == 0:
        return o
    lib().orc_preprocess(R, P, _p(uvw), _p(freq), _p(weights), _p(flags), geo["wplanes"], geo["w_inc"],
                         _p(kern["conv_info"]), _p(np.ascontiguousarray(kern["conv_sums"])), geo["sampling"],
                         geo["ny"], geo["nx"], geo["du"], geo["dv"],
                         _p(o["loc"]), _p(o["convidx"]), _p(o["togrid"]), _p(o["compress"]), _p(o["support"]),
                         _p(o["plane"]), _p(o["offx"]), _p(o["offy"]), _p(o["imgmult"]), _p(o["convsum"]))
    return o


def compress_vis(pre, vis, weights, flags):
    vis = np.ascontiguousarray(vis, np.complex64)
    R, P = weights.shape
    out = np.zeros((R, P), np.complex128)
    if R:
        lib().orc_compress_vis(R, P, _p(pre["togrid"]), _p(pre["compress"]), _p(vis),
                               _p(np.ascontiguousarray(weights, np.float32)),
                               _p(np.ascontiguousarray(flags, np.int32)), _p(pre["imgmult"]), _p(out))
    return out


def grid(pre, cvis, kern, geo, out=None):
    """ConvolutionGridder (ConvolutionGridder.cu:130-181, 394-442) in FP64.
    Accumulates into ``out`` (complex128 [ny][nx][P]) when given."""
    R, P = cvis.shape
    ny, nx = geo["ny"], geo["nx"]
    if out is None:
        out = np.zeros((ny, nx, P), np.complex128)
    if R:
        lib().orc_grid(R, P, _p(pre["togrid"]), _p(pre["loc"]), _p(pre["convidx"]), _p(pre["support"]),
                       _p(np.ascontiguousarray(cvis)), _p(kern["table"]), ny, nx, _p(out))
    return out


def grid_chunk(uvw, freq, vis, weights, flags, geo, kern, grid_acc=None, norm_acc=None):
    """One WImager chunk: preprocess, normaliser sum (WImager.cpp:196-197),
    compression and gridding.  Returns (grid, norm, pre)."""
    pre = preprocess(uvw, freq, weights, flags, geo, kern)
    cv = compress_vis(pre, vis, weights, flags)
    g = grid(pre, cv, kern, geo, grid_acc)
    n = pre["convsum"].sum(axis=1)
    if norm_acc is not None:
        n = n + norm_acc
    return g, n, pre


def stats(pre):
    """Statistics the reference reduces per chunk (WImager.cpp:173-176)."""
    s2 = pre["support"].astype(np.int64) ** 2
    return dict(gridded_records=int(pre["togrid"].sum()), compressed_records=int(pre["compress"].sum()),
                gridded_points=int((pre["togrid"] * s2).sum()), compressed_points=int((pre["compress"] * s2).sum()))


# ----------------------------------------------------------------- ingest --
def sort_index(antenna1, antenna2, n_antennas):
    """Baseline-major record order of the visibility ingest
    (code/mt-imager/lib/components/VisibilityManager/SortIndex.cpp:46-87):
    autocorrelations dropped, rows grouped by nA*nA - a1*nA - a2 - 1
    ascending, original order kept inside a baseline (a stable sort)."""
    a1 = np.asarray(antenna1, np.int64)
    a2 = np.asarray(antenna2, np.int64)
    keep = np.flatnonzero(a1 != a2)
    key = n_antennas * n_antennas - a1[keep] * n_antennas - a2[keep] - 1
    return keep[np.argsort(key, kind="stable")].astype(np.int32)


# --------------------------------------------------------------- finalize --
def _idx(fn, n):
    return np.array([fn(i, n) for i in range(n)], np.int64)


def finalize(grid_vup, norm, geo, pol_type="linear"):
    """ImageFinalizer (ImageFinalizer.cpp:31-44): PreIFFTUVCorrection
    (PreIFFTUVCorrection.cu:28-90), IFFT2D INVERSE unnormalised
    (IFFT2D.cpp:104-111), ZeroToCentre2DShift, StokesConverter
    (PostIFFTStokesConverter.cu:42-180), casagridsf taper correction
    (CasaGridSF.cu:174-199) and SincCorrector (SincCorrector.cu:29-58).
    grid_vup complex [ny][nx][P] -> float64 [P][ny][nx]."""
    L = lib()
    ny, nx, P = grid_vup.shape
    oc_y = _idx(L.orc_origin_to_corner, ny)
    oc_x = _idx(L.orc_origin_to_corner, nx)
    pre = np.empty((P, ny, nx), np.complex128)
    pre[:, oc_y[:, None], oc_x[None, :]] = np.transpose(grid_vup, (2, 0, 1))
    img = np.fft.ifft2(pre, axes=(1, 2)) * (ny * nx)
    ce_y = _idx(L.orc_origin_to_centre, ny)
    ce_x = _idx(L.orc_origin_to_centre, nx)
    sh = np.empty_like(img)
    sh[:, ce_y[:, None], ce_x[None, :]] = img
    return stokes_and_corrections(sh, norm, geo, pol_type)


def stokes_and_corrections(sh, norm, geo, pol_type="linear"):
    """From the shifted complex polarisation images [P][ny][nx] to the
    corrected Stokes cube [P][ny][nx]."""
    P, ny, nx = sh.shape
    n = np.asarray(norm, np.float64)
    re = sh.real / n[:, None, None]
    im = sh.imag / n[:, None, None]
    st = np.empty((P, ny, nx), np.float64)
    if P == 4 and pol_type == "linear":
        st[0] = (re[0] + re[3]) * 0.5
        st[1] = (re[0] - re[3]) * 0.5
        st[2] = (re[1] + re[2]) * 0.5
        st[3] = (im[1] - im[2]) * 0.5
    elif P == 4:
        st[0] = (re[0] + re[3]) * 0.5
        st[1] = (re[1] + re[2]) * 0.5
        st[2] = (im[2] - im[1]) * 0.5
        st[3] = (re[0] - re[3]) * 0.5
    elif P == 2:
        st[0] = (re[0] + re[1]) * 0.5
        st[1] = (re[0] - re[1]) * 0.5
    else:
        st[0] = re[0]
    st = st[:, ::-1, :]  # output row = ny-1-y (FITS m axis)
    g = lib().orc_grdsf
    fy = np.array([g(abs((j - ny // 2) / (ny // 2))) for j in range(ny)])
    fx = np.array([g(abs((i - nx // 2) / (nx // 2))) for i in range(nx)])
    st = st / (fy[None, :, None] * fx[None, None, :])
    s = geo["sampling"]

    def invsinc(i, n):
        x = (i - n // 2) / (n * s)
        return 1.0 if x == 0.0 else math.pi * x / math.sin(math.pi * x)
    sy = np.array([invsinc(j, ny) for j in range(ny)])
    sx = np.array([invsinc(i, nx) for i in range(nx)])
    return st * (sy[None, :, None] * sx[None, None, :])


# -------------------------------------------------------------- pipelines --
def image_channel(obs, chan, setup, kern=None, geo=None, chunk=None, pol_type="linear"):
    """Full W-projection image of one channel (optionally in record chunks)."""
    geo = geo or geometry_for(setup)
    kern = kern or wkernels(geo)
    R = obs.nrec
    chunk = chunk or R
    g, n = None, None
    freq = obs.freq_over_c(chan)
    for a in range(0, R, chunk):
        b = min(R, a + chunk)
        g, n, _ = grid_chunk(obs.uvw[:, a:b], freq[a:b], obs.vis[chan][a:b], obs.weights[chan][a:b],
                             obs.flags[chan][a:b], geo, kern, g, n)
    return finalize(g, n, geo, pol_type), g, n


def dft_image(obs, chan, setup, geo=None, kern=None, pol_type="linear"):
    """FP64 direct-DFT Stokes image of exactly the records the W-projection
    path grids, normalised by the gridded weight sum and flipped like the
    reference's Stokes output (no taper or sinc correction applies).
    pol_type "linear" or "circular" (PostIFFTStokesConverter.cu:42-90)."""
    geo = geo or geometry_for(setup)
    kern = kern or wkernels(geo)
    freq = obs.freq_over_c(chan)
    pre = preprocess(obs.uvw, freq, obs.weights[chan], obs.flags[chan], geo, kern)
    cv = compress_vis(pre, obs.vis[chan], obs.weights[chan], obs.flags[chan])
    R, P = cv.shape
    uvw_l = (obs.uvw.astype(np.float64) * freq.astype(np.float64)[None, :]).copy()
    out = np.empty((P, geo["ny"], geo["nx"]), np.complex128)
    use = pre["togrid"].astype(np.int32)
    lib().orc_dft(R, P, _p(uvw_l), _p(cv), _p(use), geo["nx"], geo["ny"], setup.dl, setup.dl, _p(out))
    wts = obs.weights[chan].astype(np.float64) * (1.0 - obs.flags[chan].astype(np.float64))
    gridded = (pre["togrid"] + pre["compress"]) > 0
    wsum = wts[gridded].sum(axis=0)
    re, im = out.real / wsum[:, None, None], out.imag / wsum[:, None, None]
    st = np.empty((P, geo["ny"], geo["nx"]))
    if P == 4 and pol_type == "linear":
        st[0] = (re[0] + re[3]) * 0.5
        st[1] = (re[0] - re[3]) * 0.5
        st[2] = (re[1] + re[2]) * 0.5
        st[3] = (im[1] - im[2]) * 0.5
    elif P == 4:
        st[0] = (re[0] + re[3]) * 0.5
        st[1] = (re[1] + re[2]) * 0.5
        st[2] = (im[2] - im[1]) * 0.5
        st[3] = (re[0] - re[3]) * 0.5
    else:
        st[:] = re
    return st[:, ::-1, :]
