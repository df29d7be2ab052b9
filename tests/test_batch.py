"""mtb_grid_batch: several images -- different geometries, kernel tables and
record counts, one of them empty -- gridded with one persistent launch must
equal mtb_grid image by image; the batch and the finaliser replay correctly
from a captured CUDA graph.  With the FP64 per-call delta grid the result is
order-independent, so the bound is tight."""
import numpy as np
import pytest
import torch

from mtb import synth
from mtb.imager import TUNING_KEYS, WProjectionImager, autotune, grid_batch

pytestmark = pytest.mark.gpu
TOL = 1e-6


def cases():
    out = []
    for seed, nx, s, nw, ntimes in ((61, 128, 4, 8, 60), (62, 96, 3, 6, 50), (63, 160, 8, 12, 40),
                                   (64, 64, 4, 4, 0)):
        obs, setup = synth.small_config(seed=seed, n_ant=10, ntimes=max(ntimes, 1), nx=nx, cell_arcsec=20.0,
                                        wplanes=nw, sampling=s, flag_frac=0.1)
        R = obs.nrec if ntimes else 0
        dev = torch.device("cuda")
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
        out.append((setup, t(obs.uvw[:, :R], torch.float32), t(obs.freq_over_c(0)[:R], torch.float32),
                    t(obs.vis[0][:R], torch.complex64), t(obs.weights[0][:R], torch.float32),
                    t(obs.flags[0][:R], torch.int32)))
    return out


def imager(setup):
    # FP64 per-call delta grid: the result does not depend on the order of the reductions
    return WProjectionImager(setup.nx, setup.ny, setup.dl, wplanes=setup.wplanes, sampling=setup.sampling,
                             exact_delta=True)


def test_batch_equals_single():
    cs = cases()
    single = []
    for setup, *arrs in cs:
        im = imager(setup)
        if arrs[1].numel():
            im.grid_device(*arrs)
        else:
            im.grid_chunk(np.zeros((3, 0), np.float32), np.zeros(0, np.float32), np.zeros((0, 4), np.complex64),
                          np.zeros((0, 4), np.float32), np.zeros((0, 4), np.int32))
        single.append((im.finalize().cpu().numpy(), im.statistics()))
    ims = [imager(setup) for setup, *_ in cs]
    grid_batch([(im, *arrs) for im, (setup, *arrs) in zip(ims, cs)])
    for im, (img1, st1) in zip(ims, single):
        assert im.statistics() == st1
        if st1["gridded_records"] == 0:
            # an empty image: zero grid and normaliser (its image is 0/0)
            assert not im.grid.abs().max().item() and not im.normalizer.abs().max().item()
            continue
        img = im.finalize().cpu().numpy()
        assert np.abs(img - img1).max() <= TOL * np.abs(img1[0]).max()


def test_batch_and_finalize_replay_from_cuda_graph():
    cs = cases()[:3]
    ims = [imager(setup) for setup, *_ in cs]
    for im in ims:
        im.build_kernels()
    eager = [imager(setup) for setup, *_ in cs]
    grid_batch([(im, *arrs) for im, (setup, *arrs) in zip(eager, cs)])
    ref = [im.finalize().cpu().numpy() for im in eager]
    ws = grid_batch([(im, *arrs) for im, (setup, *arrs) in zip(ims, cs)])   # warm-up, sizes the workspace
    outs = [torch.empty((4, s.ny, s.nx), dtype=torch.float32, device="cuda") for s, *_ in cs]
    for im, o in zip(ims, outs):
        im.finalize(out=o)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for im in ims:
            im.reset()
        grid_batch([(im, *arrs) for im, (setup, *arrs) in zip(ims, cs)], workspace=ws)
        for im, o in zip(ims, outs):
            im.finalize(out=o)
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        for o, r in zip(outs, ref):
            assert np.abs(o.cpu().numpy() - r).max() <= TOL * np.abs(r[0]).max()
    del g


def test_autotune_grids_with_the_chosen_knobs():
    """The autotuner times every candidate, applies the fastest to every
    imager, and leaves the chunk gridded with it: equal to image-by-image
    gridding with those knobs.  (Different knobs split the records
    differently over FP32 register sums, so results of different knobs agree
    only to the FP32 tolerance of the parity tests.)"""
    cs = cases()[:3]
    ims = [imager(setup) for setup, *_ in cs]
    best, cands, ws = autotune([(im, *arrs) for im, (setup, *arrs) in zip(ims, cs)])
    assert len(cands) == 54 and all(c["ms"] > 0 for c in cands)
    assert best["ms"] == min(c["ms"] for c in cands)
    assert {c["tile"] for c in cands} == {16, 32, 64} and {c["gridder_threads"] for c in cands} == {256, 512}
    assert {c["gridder"] for c in cands} == {3, 5, 7, 8}
    knobs = {k: best[k] for k in TUNING_KEYS}
    single = []
    for setup, *arrs in cs:
        im = imager(setup)
        im.tuning.update(knobs)
        im.grid_device(*arrs)
        single.append((im.finalize().cpu().numpy(), im.statistics()))
    for im, (img1, st1) in zip(ims, single):
        assert {k: im.tuning[k] for k in TUNING_KEYS} == knobs
        assert im.statistics() == st1
        img = im.finalize().cpu().numpy()
        assert np.abs(img - img1).max() <= TOL * np.abs(img1[0]).max()
    # later chunks use the chosen knobs
    for im in ims:
        im.reset()
    grid_batch([(im, *arrs) for im, (setup, *arrs) in zip(ims, cs)], workspace=ws)
    for im, (img1, _) in zip(ims, single):
        img = im.finalize().cpu().numpy()
        assert np.abs(img - img1).max() <= TOL * np.abs(img1[0]).max()


def test_autotune_needs_fresh_images():
    setup, *arrs = cases()[0]
    im = imager(setup)
    im.grid_device(*arrs)
    with pytest.raises(ValueError):
        autotune([(im, *arrs)])


def test_batch_images_match_oracle(oracle):
    """Images gridded together by one batched launch, each against the FP64
    oracle: every Stokes plane within 1e-5 RMS of its Stokes I peak, and the
    record statistics exact (the batched path is otherwise only checked
    against mtb_grid)."""
    setups = []
    for seed, nx, s, nw in ((71, 128, 4, 8), (72, 96, 3, 6), (73, 160, 8, 12)):
        obs, setup = synth.small_config(seed=seed, n_ant=10, ntimes=60, nx=nx, cell_arcsec=20.0, wplanes=nw,
                                        sampling=s, flag_frac=0.1)
        setups.append((obs, setup))
    dev = torch.device("cuda")
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
    ims = [imager(setup) for _, setup in setups]
    grid_batch([(im, t(obs.uvw, torch.float32), t(obs.freq_over_c(0), torch.float32),
                 t(obs.vis[0], torch.complex64), t(obs.weights[0], torch.float32), t(obs.flags[0], torch.int32))
                for im, (obs, setup) in zip(ims, setups)])
    for im, (obs, setup) in zip(ims, setups):
        img = im.finalize().cpu().numpy()
        img_o, _, _ = oracle.image_channel(obs, 0, setup)
        peak = np.abs(img_o[0]).max()
        for p in range(4):
            assert np.sqrt(np.mean((img[p] - img_o[p]) ** 2)) <= 1e-5 * peak, p
        geo = oracle.geometry_for(setup)
        st = oracle.stats(oracle.preprocess(obs.uvw, obs.freq_over_c(0), obs.weights[0], obs.flags[0], geo,
                                            oracle.wkernels(geo)))
        assert im.statistics() == st
