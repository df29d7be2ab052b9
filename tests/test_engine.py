"""The C++ host layer: the request engine (include/mtb_engine.h) and the
header-only classes of include/mtb.hpp, against the FP64 oracle and against
the single-image path.

A request's image must be the same alone and in a mix of concurrent requests
of other geometries (with the same chunking); with compensated gridding the
per-call FP64 delta grid makes the result independent of the order of the
reductions, so the bound is tight.
"""
import os
import subprocess

import numpy as np
import pytest

from mtb import synth
from mtb import _lib as L

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
IMAGE_RMS_TOL = 1e-5
MIX_TOL = 1e-6


def case(seed, nx, npol, s=4, nw=8, ntimes=60, cell=20.0):
    obs, setup = synth.small_config(seed=seed, n_ant=10, ntimes=ntimes, nx=nx, cell_arcsec=cell, wplanes=nw,
                                    sampling=s, flag_frac=0.1)
    P = npol
    return dict(nx=nx, ny=nx, l_increment=setup.dl, m_increment=setup.dl, wplanes=nw, sampling=s,
                uvw=obs.uvw, freq=obs.freq_over_c(0), vis=obs.vis[0][:, :P], weights=obs.weights[0][:, :P],
                flags=obs.flags[0][:, :P]), obs, setup


def submit(e, c, **kw):
    return e.submit(c["nx"], c["ny"], c["l_increment"], c["m_increment"], c["wplanes"], c["sampling"], c["uvw"],
                    c["freq"], c["vis"], c["weights"], c["flags"], **kw)


def test_engine_image_matches_oracle(oracle):
    from mtb.engine import Engine
    c, obs, setup = case(31, 128, 4)
    with Engine(slots=2) as e:
        r = e.wait(submit(e, c))
    assert r.status == 0
    img_o, _, _ = oracle.image_channel(obs, 0, setup)
    peak = np.abs(img_o[0]).max()
    for p in range(4):
        assert np.sqrt(np.mean((r.image[p] - img_o[p]) ** 2)) <= IMAGE_RMS_TOL * peak
    st = oracle.stats(oracle.preprocess(obs.uvw, obs.freq_over_c(0), obs.weights[0], obs.flags[0],
                                        oracle.geometry_for(setup), oracle.wkernels(oracle.geometry_for(setup))))
    assert r.stats["gridded_records"] == st["gridded_records"]


def test_alone_equals_in_mix():
    from mtb.engine import Engine
    cases = [case(41, 128, 4)[0], case(42, 96, 2, s=3, nw=6)[0], case(43, 64, 1, nw=4)[0], case(44, 128, 4)[0]]
    # exact_delta: order-independent accumulation, so alone and mixed agree to rounding of the merge
    kws = [dict(exact_delta=True), dict(pol_type=L.MTB_POL_CIRCULAR, exact_delta=True), dict(exact_delta=True),
           dict(exact_delta=True)]
    alone = []
    with Engine(slots=1, chunk_records=1500) as e:
        for c, kw in zip(cases, kws):
            r = e.wait(submit(e, c, **kw))
            assert r.status == 0
            alone.append(r.image.copy())
    with Engine(slots=3, chunk_records=1500) as e:
        tickets = [submit(e, c, **kw) for c, kw in zip(cases, kws)] + [submit(e, cases[0], **kws[0])]
        mixed = [e.wait(t) for t in tickets]
    for a, m in zip(alone + [alone[0]], mixed):
        assert m.status == 0
        peak = np.abs(a[0]).max()
        assert np.abs(m.image - a).max() <= MIX_TOL * peak
    # the repeated geometry found its w-kernels in the cache
    assert mixed[-1].kernel_cache_hit or mixed[0].kernel_cache_hit


def test_host_copy_threads_and_uvw_slices():
    """The host copy pool's width does not change an image, and a request
    imaging a slice of a longer uvw array (uvw_row_stride) equals one given a
    contiguous copy; images large enough to come back in several pieces."""
    from mtb.engine import Engine
    c = case(46, 2048, 4, nw=4, ntimes=30, cell=10.0)[0]
    R = c["freq"].size
    longer = np.zeros((3, R + 1000), np.float32)
    longer[:, 500:500 + R] = c["uvw"]
    sliced = dict(c, uvw=longer[:, 500:500 + R])
    assert sliced["uvw"].strides[0] == 4 * (R + 1000)
    imgs = []
    for threads, cc in ((1, c), (6, c), (6, sliced)):
        with Engine(slots=1, host_threads=threads, chunk_records=700) as e:
            r = e.wait(submit(e, cc, exact_delta=True, trial_support=33, max_support=31))
            assert r.status == 0
            imgs.append(r.image.copy())
    peak = np.abs(imgs[0][0]).max()
    assert peak > 0
    for im in imgs[1:]:
        assert np.abs(im - imgs[0]).max() <= MIX_TOL * peak


def test_empty_request_and_capacity():
    from mtb.engine import Engine
    c = case(45, 64, 4, nw=4)[0]
    empty = {k: (v[..., :0] if k == "uvw" else v[:0]) if k in ("uvw", "freq", "vis", "weights", "flags") else v
             for k, v in c.items()}
    with Engine(slots=1, hbm_budget_bytes=(6 << 30), kernel_cache_bytes=(1 << 30), chunk_records=4096) as e:
        r = e.wait(submit(e, empty))
        assert r.status == 0 and r.stats["gridded_records"] == 0
        big = dict(c, nx=16384, ny=16384)
        with pytest.raises(L.MtbError) as err:
            submit(e, big)
        assert err.value.status == L.MTB_ERR_CAPACITY


def test_cpp_host_api(tmp_path):
    """tests/cpp/image_one.cpp images a chunk through mtb::KernelTable and
    mtb::Imager; its image equals the Python path's."""
    from mtb.imager import WProjectionImager
    cxx = os.environ.get("CXX", "g++")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    exe = tmp_path / "image_one"
    lib = os.path.join(ROOT, "mt-imager_b200")
    subprocess.run([cxx, "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "image_one.cpp"), "-o", str(exe),
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"), "-L", lib, "-lmtb",
                    "-L", os.path.join(cuda, "lib64"), "-lcudart", "-Wl,-rpath," + lib,
                    "-Wl,-rpath," + os.path.join(cuda, "lib64")], check=True)
    c, obs, setup = case(46, 128, 4)
    R, P = c["freq"].size, 4
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        np.array([128, 128, P, 8, 4, 0, 1, R], np.int32).tofile(f)
        np.array([setup.dl], np.float64).tofile(f)
        for a, t in ((c["uvw"], np.float32), (c["freq"], np.float32), (c["vis"], np.complex64),
                     (c["weights"], np.float32), (c["flags"], np.int32)):
            np.ascontiguousarray(a, t).tofile(f)
    out = tmp_path / "out.bin"
    subprocess.run([str(exe), str(inp), str(out)], check=True)
    raw = np.fromfile(out, np.uint8)
    img = raw[: 4 * P * 128 * 128].view(np.float32).reshape(P, 128, 128)
    im = WProjectionImager(128, 128, setup.dl, wplanes=8, sampling=4, exact_delta=True)
    im.build_kernels()
    im.grid_chunk(c["uvw"], c["freq"], c["vis"], c["weights"], c["flags"])
    ref = im.finalize().cpu().numpy()
    assert np.abs(img - ref).max() <= MIX_TOL * np.abs(ref[0]).max()


def test_cancel_queued_and_running_requests():
    """mtb_engine_cancel: with one slot, a long request (many small chunks)
    and two queued ones.  The queued request cancelled before admission is
    dropped (no service time); the long one, cancelled while it is admitted
    or queued, ends with MTB_ERR_CANCELLED; the untouched request still images
    as it does alone.  A request that completed keeps its result, and an
    unknown ticket is refused."""
    import time
    from mtb.engine import Engine
    big = case(47, 128, 4, ntimes=600)[0]
    small = case(48, 64, 4, nw=4)[0]
    with Engine(slots=1, chunk_records=256) as e:
        t1 = submit(e, big, exact_delta=True)
        t2 = submit(e, small, exact_delta=True)
        t3 = submit(e, small, exact_delta=True)
        e.cancel(t2)
        e.cancel(t1)                          # just admitted (building its kernels) or still queued
        r1, r2, r3 = e.wait(t1), e.wait(t2), e.wait(t3)
        assert r2.status == L.MTB_ERR_CANCELLED and r2.service_ms == 0.0
        assert r1.status == L.MTB_ERR_CANCELLED
        assert r3.status == 0 and r3.stats["gridded_records"] > 0
        t4 = submit(e, small, exact_delta=True)
        r4 = e.wait(t4)
        assert r4.status == 0
        assert np.abs(r3.image - r4.image).max() <= MIX_TOL * np.abs(r4.image[0]).max()
        t5 = submit(e, small, exact_delta=True)
        time.sleep(2.0)                       # long done: cancelling it changes nothing
        e.cancel(t5)
        r5 = e.wait(t5)
        assert r5.status == 0 and np.array_equal(r5.image, r4.image)
        with pytest.raises(L.MtbError) as err:
            e.cancel(t5)                      # already waited for
        assert err.value.status == L.MTB_ERR_BAD_PARAM
