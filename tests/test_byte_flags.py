"""Flags given as one byte per flag (mtb_grid_params.flags_u8,
mtb_image_request.flags_u8) or one bit per flag (flags_u8 = 2, mtb_grid and
mtb_grid_batch) grid exactly like the reference's int32 flags:
through mtb_grid, mtb_preprocess_uvw, mtb_grid_batch (the two formats mixed in
one batch) and the request engine.  The preprocessing outputs are compared
bit for bit; images to 1e-6 of the peak (with the FP64 per-call delta grid
only the order of the FP64 reductions can differ between runs)."""
import ctypes

import numpy as np
import pytest
import torch

from mtb import synth
from mtb import _lib as L
from mtb.engine import Engine
from mtb.imager import WProjectionImager, _ptr, _stream, grid_batch

pytestmark = pytest.mark.gpu
TOL = 1e-6


def same(a, b):
    return np.abs(a - b).max() <= TOL * np.abs(b[0]).max()


def case(seed=31, nx=128):
    obs, setup = synth.small_config(seed=seed, n_ant=12, ntimes=60, nx=nx, cell_arcsec=20.0, wplanes=8,
                                    sampling=4, flag_frac=0.2)
    fl = obs.flags[0].copy()
    rng = np.random.default_rng(seed)
    fl[rng.random(fl.shape) < 0.05] = 1          # some single-polarisation flags too
    obs.flags[0] = fl
    return obs, setup


def imager(setup):
    return WProjectionImager(setup.nx, setup.ny, setup.dl, wplanes=setup.wplanes, sampling=setup.sampling,
                             exact_delta=True)


def image(obs, setup, flags):
    im = imager(setup)
    im.grid_chunk(obs.uvw, obs.freq_over_c(0), obs.vis[0], obs.weights[0], flags)
    return im.finalize().cpu().numpy(), im.statistics(), im


def test_mtb_grid_byte_flags_equal_int32():
    obs, setup = case()
    a, sa, _ = image(obs, setup, obs.flags[0].astype(np.int32))
    b, sb, _ = image(obs, setup, obs.flags[0].astype(np.uint8))
    c, sc, _ = image(obs, setup, obs.flags[0].astype(bool))
    assert sa == sb == sc
    assert same(b, a) and same(c, a)


def test_any_nonzero_flag_is_flagged():
    """The flag contract is 0 = keep, any other value = flagged: flags of 2
    (int32) and 0xFF (a bool column written as bytes) grid exactly like 1.  The
    reference weights by 1 - flag, which agrees for 0 / 1 and would give a
    negative weight for other values."""
    obs, setup = case(seed=33)
    fl = obs.flags[0].astype(np.int32)
    a, sa, _ = image(obs, setup, fl)
    b, sb, _ = image(obs, setup, fl * 2)
    c, sc, _ = image(obs, setup, (fl * 255).astype(np.uint8))
    assert sa == sb == sc
    assert same(b, a) and same(c, a)


def test_preprocess_byte_flags_bit_exact():
    obs, setup = case(seed=32)
    im = imager(setup)
    k = im.build_kernels()
    R = obs.nrec
    dev = im.device
    outs = []
    for dt in (torch.int32, torch.uint8):
        gp = im.grid_params(False)
        gp.flags_u8 = int(dt == torch.uint8)
        ws, nbytes = im._workspace(R, gp)
        uvw = torch.from_numpy(obs.uvw).to(dev)
        freq = torch.from_numpy(obs.freq_over_c(0)).to(dev)
        wts = torch.from_numpy(obs.weights[0]).to(dev)
        flg = torch.from_numpy(obs.flags[0]).to(dev, dt)
        o = dict(loc=torch.empty((R, 4), dtype=torch.int32, device=dev),
                 convidx=torch.empty(R, dtype=torch.int32, device=dev),
                 togrid=torch.empty(R, dtype=torch.int32, device=dev),
                 compress=torch.empty(R, dtype=torch.int32, device=dev),
                 support=torch.empty(R, dtype=torch.int32, device=dev),
                 imgmult=torch.empty(R, dtype=torch.float32, device=dev),
                 convsum=torch.empty((4, R), dtype=torch.float32, device=dev))
        L.check(im.lib.mtb_preprocess_uvw(ctypes.byref(gp), _ptr(k.d_conv_info),
                                          k.conv_info.ctypes.data_as(ctypes.c_void_p), _ptr(k.conv_sums), _ptr(uvw),
                                          _ptr(freq), _ptr(wts), _ptr(flg), R, _ptr(o["loc"]), _ptr(o["convidx"]),
                                          _ptr(o["togrid"]), _ptr(o["compress"]), _ptr(o["support"]),
                                          _ptr(o["imgmult"]), _ptr(o["convsum"]), _ptr(ws), nbytes, _stream()),
                "mtb_preprocess_uvw")
        torch.cuda.synchronize()
        outs.append({kk: v.cpu().numpy() for kk, v in o.items()})
    for kk in outs[0]:
        assert np.array_equal(outs[0][kk], outs[1][kk]), kk


def test_batch_mixes_flag_formats():
    cs = [case(seed=33), case(seed=34, nx=96)]
    single = [image(obs, setup, obs.flags[0])[0] for obs, setup in cs]
    dev = torch.device("cuda")
    entries = []
    for i, (obs, setup) in enumerate(cs):
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
        entries.append((imager(setup), t(obs.uvw, torch.float32), t(obs.freq_over_c(0), torch.float32),
                        t(obs.vis[0], torch.complex64), t(obs.weights[0], torch.float32),
                        t(obs.flags[0], torch.uint8 if i == 0 else torch.int32)))
    grid_batch(entries)
    for (im, *_), img1 in zip(entries, single):
        assert same(im.finalize().cpu().numpy(), img1)


def test_packed_bit_flags_equal_bytes():
    """One bit per flag (flags_u8 = 2, mtb.imager.pack_flags) grids exactly
    like one byte per flag, through mtb_grid on an odd record count (the last
    byte half used) and through mtb_grid_batch beside byte flags."""
    from mtb.imager import pack_flags
    dev = torch.device("cuda")
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
    obs, setup = case(seed=36)
    R = obs.nrec - 1                                 # R * P / 8 not whole
    args = (obs.uvw[:, :R], obs.freq_over_c(0)[:R], obs.vis[0][:R], obs.weights[0][:R])
    fl = obs.flags[0][:R].astype(np.uint8)
    ref = imager(setup)
    ref.grid_chunk(*args, fl)
    a = ref.finalize().cpu().numpy()
    im = imager(setup)
    bits = pack_flags(t(fl, torch.uint8))
    assert bits.numel() == (R * 4 + 7) // 8
    im.grid_device(t(args[0], torch.float32), t(args[1], torch.float32), t(args[2], torch.complex64),
                   t(args[3], torch.float32), bits)
    assert im.statistics() == ref.statistics()
    assert same(im.finalize().cpu().numpy(), a)
    cs = [case(seed=37), case(seed=38, nx=96)]
    single = [image(o, st, o.flags[0])[0] for o, st in cs]
    entries = []
    for i, (o, st) in enumerate(cs):
        f = t(o.flags[0], torch.uint8)
        entries.append((imager(st), t(o.uvw, torch.float32), t(o.freq_over_c(0), torch.float32),
                        t(o.vis[0], torch.complex64), t(o.weights[0], torch.float32), pack_flags(f) if i else f))
    grid_batch(entries)
    for (im2, *_), img1 in zip(entries, single):
        assert same(im2.finalize().cpu().numpy(), img1)


def test_engine_byte_flags_equal_int32():
    obs, setup = case(seed=35)
    res = []
    with Engine(slots=2) as eng:
        for fl in (obs.flags[0].astype(np.int32), obs.flags[0].astype(np.uint8)):
            t = eng.submit(setup.nx, setup.ny, setup.dl, setup.dl, setup.wplanes, setup.sampling, obs.uvw,
                           obs.freq_over_c(0), obs.vis[0], obs.weights[0], fl, exact_delta=True)
            r = eng.wait(t)
            assert r.status == 0
            res.append((r.image.copy(), r.stats))
    assert res[0][1] == res[1][1]
    assert same(res[1][0], res[0][0])
