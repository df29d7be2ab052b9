#!/usr/bin/env python
"""Benchmark of the W-projection imaging path: vis·pol samples gridded per second.

Workload (default, one GPU): the mid-size plain W-projection configuration --
64 antennas within 4 km, 16 channels over 1.3-1.5 GHz, an 8 h track at 2 s
(2016 baselines x 14,400 integrations = 29,030,400 records per channel,
4.64e8 visibilities), 4 complex64 polarisations, 200 power-law point sources,
25 % of records flagged, 4096 x 4096 image, 128 w-planes, oversampling 8,
supports 7-65.  Synthetic, seeded data stand in for a MeasurementSet.

One step images every channel: mtb_grid (preprocess, bin, tile gridder) into a
fresh grid, then mtb_finalize (IFFT, Stokes, corrections).  The w-kernel table
is built once and shared (the reference also builds it once per run).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mtb|reference]
                    [--channels C] [--hours H] [--config mid|small]

Under torchrun each rank runs an independent replica (the path has no
cross-GPU exchange); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "mt-imager_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "vis·pol samples/s gridded; p50/p99 image latency vs plain GPU path at ≤1e-5 RMS"
C_LIGHT = 299792458.0
ARCSEC = math.pi / (180.0 * 3600.0)


# ------------------------------------------------------------ replicas ----
def host_available_bytes():
    """Host memory available now (bytes)."""
    try:
        import psutil
        return psutil.virtual_memory().available
    except Exception:
        return os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")


def max_over_ranks(ms, world, dist, torch, device):
    """The slowest rank's time, returned on every rank (an all-reduce MAX;
    every rank takes this step in the same order)."""
    if world <= 1:
        return float(ms)
    tt = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def job_throughput(samples_per_rank_step, world, ms_per_step):
    """Whole-job samples/s: every replica grids the same work per step."""
    return samples_per_rank_step * world / (ms_per_step * 1e-3)


# ------------------------------------------------------------- workload ----
def workload_spec(args):
    if args.config == "small":
        return dict(name="small", n_ant=27, radius=1000.0, f_lo=1.4e9, f_hi=1.4e9, nchan=1, hours=1.0, dt=10.0,
                    nsrc=10, powerlaw=None, flux=(0.1, 1.0), flag=0.0, nx=256, cell_arcsec=2.0, wplanes=32,
                    sampling=8, trial_support=0, max_support=0, lat=-30.0, dec=-45.0)
    return dict(name="mid", n_ant=64, radius=4000.0, f_lo=1.3e9, f_hi=1.5e9, nchan=args.channels,
                hours=args.hours, dt=2.0, nsrc=200, powerlaw=-1.5, flux=(1e-3, 1.0), flag=0.25, nx=4096,
                cell_arcsec=None, wplanes=128, sampling=8, trial_support=67, max_support=65, lat=-30.0,
                dec=-45.0)


def make_uvw(spec, device, torch, rng, nbl_limit=None, nt_limit=None):
    from mtb import synth
    enu = synth.antenna_layout(spec["n_ant"], spec["radius"], rng)
    pairs = synth.baseline_order(spec["n_ant"])
    if nbl_limit:
        pairs = pairs[:nbl_limit]
    nt = int(round(spec["hours"] * 3600.0 / spec["dt"]))
    if nt_limit:
        nt = min(nt, nt_limit)
    lat, dec = math.radians(spec["lat"]), math.radians(spec["dec"])
    a1 = torch.tensor([p[0] for p in pairs], device=device)
    a2 = torch.tensor([p[1] for p in pairs], device=device)
    e = torch.tensor(enu, dtype=torch.float64, device=device)
    d = e[a2] - e[a1]
    lx = (-d[:, 1] * math.sin(lat) + d[:, 2] * math.cos(lat))[:, None]
    ly = d[:, 0][:, None]
    lz = (d[:, 1] * math.cos(lat) + d[:, 2] * math.sin(lat))[:, None]
    ha = ((torch.arange(nt, device=device, dtype=torch.float64) - (nt - 1) / 2.0) * spec["dt"]
          * (2 * math.pi / 86164.0905))[None, :]
    sh, ch = torch.sin(ha), torch.cos(ha)
    uvw = torch.empty((3, len(pairs), nt), dtype=torch.float32, device=device)
    uvw[0] = (sh * lx + ch * ly).float()
    uvw[1] = (-math.sin(dec) * ch * lx + math.sin(dec) * sh * ly + math.cos(dec) * lz).float()
    uvw[2] = (math.cos(dec) * ch * lx - math.cos(dec) * sh * ly + math.sin(dec) * lz).float()
    return uvw.reshape(3, -1).contiguous(), len(pairs), nt


def channel_freqs(spec):
    if spec["nchan"] == 1:
        return np.array([spec["f_lo"]])
    return np.linspace(spec["f_lo"], spec["f_hi"], spec["nchan"])


def cell_for(spec, uvw_max_m, torch):
    """Largest cell with max|u|/du + 65/2 < N/2 at the highest frequency."""
    if spec["cell_arcsec"]:
        return spec["cell_arcsec"] * ARCSEC
    n = spec["nx"]
    uv_max = uvw_max_m * spec["f_hi"] / C_LIGHT
    du = uv_max / (n / 2 - (spec["max_support"] / 2 + 1))
    return 1.0 / (n * du)


def make_vis(uvw, freq_hz, sources, torch, generator):
    """Point-source visibilities complex64 [R][4] (XX, XY, YX, YY)."""
    R = uvw.shape[1]
    k = 2 * math.pi * freq_hz / C_LIGHT
    out = torch.zeros((R, 4), dtype=torch.complex64, device=uvw.device)
    for l, m, si, sq, su, sv in sources:
        n1 = math.sqrt(1 - l * l - m * m) - 1
        ph = (uvw[0] * l + uvw[1] * m + uvw[2] * n1) * (-k)
        e = torch.polar(torch.ones_like(ph), ph)
        out[:, 0] += (si + sq) * e
        out[:, 1] += complex(su, sv) * e
        out[:, 2] += complex(su, -sv) * e
        out[:, 3] += (si - sq) * e
    return out


def sources_for(spec, fov, rng):
    from mtb import synth
    return synth.random_sources(spec["nsrc"], fov, rng, flux=spec["flux"], powerlaw=spec["powerlaw"])


# ----------------------------------------------------------------- clocks --
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, log_dir=None):
        """Samples nvidia-smi every 200 ms into log_dir/clocks_rank<i>.csv, or
        into a temporary file when log_dir is None."""
        self.proc = None
        self.gpu = gpu_index
        self.keep = bool(log_dir)
        if log_dir:
            self.path = os.path.join(log_dir, "clocks_rank%d.csv" % gpu_index)
        else:
            import tempfile
            fd, self.path = tempfile.mkstemp(prefix="mtb_clocks_", suffix=".csv")
            os.close(fd)

    def start(self):
        try:
            if os.path.dirname(self.path):
                os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nme, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nme)
        if not self.keep:
            os.remove(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------- reference arm --
def run_reference(args, rank, world):
    """The reference's gridding semantics on the host cores: the FP32 OpenMP
    transcription (oracle/cpu_port.c), each step a bounded sample of the same
    workload (one channel, a block of baselines over the full track)."""
    if rank != 0:
        return
    import torch
    from oracle import oracle as O
    spec = workload_spec(args)
    rng = np.random.default_rng(2)
    nt_full = int(round(spec["hours"] * 3600.0 / spec["dt"]))
    nbl = max(1, cpu_sample_records(args, spec, nt_full) // nt_full) if spec["name"] == "mid" else None
    uvw, _, _ = make_uvw(spec, "cpu", torch, rng, nbl_limit=nbl)
    full, _, _ = make_uvw(spec, "cpu", torch, np.random.default_rng(2), nbl_limit=None, nt_limit=8)
    dl = cell_for(spec, float(full[:2].abs().max()), torch)
    freqs = channel_freqs(spec)
    f = freqs[len(freqs) // 2]
    gen = torch.Generator().manual_seed(3)
    srcs = sources_for(spec, spec["nx"] * dl, rng)
    vis = make_vis(uvw.double(), f, srcs, torch, gen).numpy()
    R = uvw.shape[1]
    flags = (torch.rand(R, generator=gen) < spec["flag"]).int()[:, None].repeat(1, 4).numpy()
    weights = np.ones((R, 4), np.float32)
    freq = np.full(R, f / C_LIGHT, np.float32)
    geo = O.kernel_geometry(spec["nx"], spec["nx"], dl, dl, spec["wplanes"], spec["sampling"],
                            spec["trial_support"], spec["max_support"])
    kern = O.wkernels(geo)
    table = kern["table"].astype(np.complex64)
    sums = kern["conv_sums"].astype(np.float32)
    P = O.port()
    cores = P.port_threads()
    grid = np.zeros((spec["nx"], spec["nx"], 4), np.complex64)
    norm = np.zeros(4, np.float32)
    uvw_np = uvw.numpy()

    def step():
        grid[:] = 0
        st = np.zeros(4, np.int64)
        P.port_grid_chunk(R, 4, O._p(uvw_np), O._p(freq), O._p(vis), O._p(weights), O._p(flags),
                          spec["wplanes"], geo["w_inc"], O._p(kern["conv_info"]), O._p(sums), O._p(table),
                          spec["sampling"], spec["nx"], spec["nx"], geo["du"], geo["dv"], O._p(grid),
                          O._p(norm), O._p(st))
        return int(st[0] + st[1]) * 4
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    samples = 0
    for _ in range(args.steps):
        samples += step()
    dt = time.perf_counter() - t0
    v = samples / dt
    nbl_all = spec["n_ant"] * (spec["n_ant"] - 1) // 2
    sample = "%d records of one %s channel (%d of %d baselines, full track), FP32 OpenMP port" % (
        R, spec["name"], min(nbl or nbl_all, nbl_all), nbl_all)
    line = {"metric": METRIC, "value": v, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference", "config": {"workload": workload_name(spec), "sample": sample},
            "cpu_baseline": {"value": v, "unit": "samples/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_ref_gpu:
        line["reference_gpu"] = reference_gpu(spec, geo, table, sums, kern["conv_info"], uvw_np, freq, vis,
                                              weights, flags, samples // max(1, args.steps), torch)
    print(json.dumps(line), flush=True)


# bytes per gridder launch, one 8 h mid-size channel (ncu: profiles/k_grid7_pairs_mid4096_8h_dram.md
# for the default tap-pair shape, profiles/k_grid7_mid4096_8h_dram.md for gridder 7)
GRIDDER_TRAFFIC = {8: 5.017e9, 7: 5.018e9}
REF_CHUNK = 1000000   # records per WImager chunk: mt-imager's default `records` (mtimager.properties:47-48)


def reference_gpu(spec, geo, table, sums, conv_info, uvw, freq, vis, weights, flags, samples, torch):
    """mt-imager's own gridding operators on this GPU: the reference's
    PreProcessUVW ... ConvolutionGridder sources rebuilt unchanged for sm_100a
    (oracle/_ref/libmtref.so, oracle/ref_harness.cu), run over the same sample
    in chunks of the reference's default 1,000,000 records, each chunk through
    the operator graph of one WImager chunk.  Reported: samples/s over the
    ConvolutionGridder kernels' own events, and over the whole graph (each
    operator's span; the harness synchronises between operators)."""
    path = os.path.join(ROOT, "oracle", "_ref", "libmtref.so")
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/libmtref.so not built (needs the reference sources)"}
    lib = ctypes.CDLL(path)
    lib.mtref_grid_chunk.restype = ctypes.c_int
    lib.mtref_last_chunk_ms.restype = ctypes.c_int
    n = spec["nx"]
    R = uvw.shape[1]
    table = np.ascontiguousarray(table, np.complex64)
    sums = np.ascontiguousarray(sums, np.float32)
    ci = np.ascontiguousarray(conv_info, np.int32)
    grid = np.zeros((n, n, 4), np.complex64)
    err = ctypes.create_string_buffer(512)
    nul = ctypes.c_void_p(None)
    bounds = [(a, min(R, a + REF_CHUNK)) for a in range(0, R, REF_CHUNK)]
    if len(bounds) > 1 and bounds[-1][1] - bounds[-1][0] < 2048:
        bounds[-2:] = [(bounds[-2][0], R)]

    def chunk(a, b, first):
        u = np.ascontiguousarray(uvw[:, a:b])
        parts = [np.ascontiguousarray(x[a:b]) for x in (freq, vis, weights, flags)]
        rc = lib.mtref_grid_chunk(n, n, 4, spec["sampling"], spec["wplanes"], ctypes.c_float(geo["du"]),
                                  ctypes.c_float(geo["dv"]), ctypes.c_float(geo["w_inc"]), _ptr(table),
                                  int(table.size), _ptr(ci), _ptr(sums), _ptr(u), *[_ptr(x) for x in parts],
                                  int(b - a), 1 if first else 0, _ptr(grid), nul, nul, nul, nul, nul, nul, nul,
                                  err, 512)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        g, c = ctypes.c_float(0), ctypes.c_float(0)
        lib.mtref_last_chunk_ms(ctypes.byref(g), ctypes.byref(c))
        return g.value, c.value
    try:
        chunk(*bounds[0], True)                       # module load and first-launch costs
        g_ms = c_ms = 0.0
        for i, (a, b) in enumerate(bounds):
            g, c = chunk(a, b, i == 0)
            g_ms += g
            c_ms += c
    except RuntimeError as e:
        return {"unavailable": "reference operators refused this sample: %s" % e}
    return {"value": samples / (c_ms * 1e-3), "unit": "samples/s",
            "gridder_value": samples / (g_ms * 1e-3), "gridder_ms": g_ms, "graph_ms": c_ms,
            "chunks": len(bounds), "chunk_records": REF_CHUNK, "device": torch.cuda.get_device_name(0),
            "kind": "reference operators rebuilt for sm_100a (oracle/_ref), run one at a time",
            "sample": "the cpu_baseline sample (%d records) in chunks of %d records" % (R, REF_CHUNK)}


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def workload_name(spec):
    if spec["name"] == "small":
        return ("plain small W-projection image: 27 antennas / 1 km, 1 channel at 1.4 GHz, 1 h at 10 s "
                "(126,360 records), 4 pol, 256^2 at 2 arcsec, 32 w-planes, oversampling 8")
    return ("mid-size plain GPU path: 64 antennas / 4 km, %d channels over 1.3-1.5 GHz, %.3g h at 2 s, 4 pol, "
            "200 power-law sources, 25%% flagged, 4096^2, 128 w-planes, oversampling 8, support 7-65"
            % (spec["nchan"], spec["hours"]))


# ------------------------------------------------------------------ main ----
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mtb", choices=["mtb", "reference"])
    ap.add_argument("--config", default="mid", choices=["mid", "small", "serve", "cube"])
    ap.add_argument("--channels", type=int, default=16)
    ap.add_argument("--hours", type=float, default=8.0)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--e2e-slots", type=int, default=2, help="device buffer sets the e2e leg's channel copies rotate over")
    ap.add_argument("--streams", type=int, default=1, help="CUDA streams the channels of a step alternate over")
    ap.add_argument("--cpu-records", type=int, default=0, help="records for the CPU baseline sample")
    ap.add_argument("--ref-baselines", type=int, default=560)
    ap.add_argument("--tile", type=int, default=0)
    ap.add_argument("--support-bucket", type=int, default=0)
    ap.add_argument("--max-chunk", type=int, default=0)
    ap.add_argument("--merge", type=int, default=0)
    ap.add_argument("--gridder", type=int, default=0, help="mtb_grid_params.gridder (0: the library default)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the request-stream measurement")
    ap.add_argument("--no-oracle", action="store_true", help="skip the FP64 oracle check of the first channel")
    ap.add_argument("--no-cube", action="store_true", help="skip the batched-cubes measurement")
    ap.add_argument("--no-lsrk", action="store_true", help="skip the TOPO->LSRK frequency measurement")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="reference arm: skip timing the reference's own gridding operators on the GPU")
    ap.add_argument("--cube-images", type=int, default=64)
    ap.add_argument("--cube-min-hours", type=float, default=1.0)
    ap.add_argument("--cube-max-hours", type=float, default=8.0)
    ap.add_argument("--cube-chunk", type=float, default=1 << 22, help="records per image per batched call")
    ap.add_argument("--serve-requests", type=int, default=500)
    ap.add_argument("--serve-rate", type=float, default=20.0, help="Poisson arrival rate, requests per second")
    ap.add_argument("--serve-min-records", type=float, default=1e5)
    ap.add_argument("--serve-max-records", type=float, default=5e7)
    ap.add_argument("--serve-slots", type=int, default=8)
    ap.add_argument("--clock-log", default=None,
                    help="directory that keeps the nvidia-smi clock samples of the timed region")
    ap.add_argument("--profile-range", action="store_true",
                    help="bracket the timed steps with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    args = ap.parse_args()

    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: relaunch under torch.distributed.run
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
               "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
        os.execv(sys.executable, cmd)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    from mtb import _lib as L
    from mtb.imager import WProjectionImager, build_wkernels, pack_flags, wkernel_params

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.config == "cube":
        if rank == 0:
            cb = run_cube(args, torch, dev)
            print(json.dumps({"metric": METRIC, "value": cb["batched_cuda_graph"]["samples_per_s"],
                              "unit": "samples/s", "n_gpus": 1, "higher_is_better": True, "impl": "mtb-batch",
                              "data": "synthetic", "config": {"workload": "batched cubes: %d channel images, "
                                                                          "%.3g-%.3g h tracks, 1024^2/2048^2, 64 "
                                                                          "w-planes" % (args.cube_images,
                                                                                       args.cube_min_hours,
                                                                                       args.cube_max_hours)},
                              "cube": cb}), flush=True)
        return
    if args.config == "serve":
        if rank == 0:
            sv = run_serve(args, torch, dev)
            print(json.dumps({"metric": METRIC, "value": sv["engine"]["samples_per_s"], "unit": "samples/s",
                              "n_gpus": 1, "higher_is_better": True, "impl": "mtb-engine", "data": "synthetic",
                              "config": {"workload": "request stream: %d requests, Poisson %.3g/s, images "
                                                     "512^2-4096^2, records %.3g-%.3g log-uniform"
                                                     % (args.serve_requests, args.serve_rate,
                                                        args.serve_min_records, args.serve_max_records)},
                              "latency_ms": {"p50": sv["engine"]["p50_ms"], "p99": sv["engine"]["p99_ms"]},
                              "serving": sv}), flush=True)
        return
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    spec = workload_spec(args)
    lib = L.load()

    # ---- data (seeded; every replica images the same cube)
    t_gen = time.perf_counter()
    rng = np.random.default_rng(2)
    uvw, nbl, nt = make_uvw(spec, dev, torch, rng)
    R = uvw.shape[1]
    dl = cell_for(spec, float(uvw[:2].abs().max()), torch)
    fov = spec["nx"] * dl
    srcs = sources_for(spec, fov, rng)
    freqs = channel_freqs(spec)
    gen = torch.Generator(device=dev).manual_seed(7 + rank)
    chans = []
    # one weights array for every channel: mt-imager reads the MS WEIGHT column
    # (per row and polarisation) and hands the same array to each channel
    # (MSVisibilityDataSetAsync.cpp:262-271)
    weights = torch.ones((R, 4), dtype=torch.float32, device=dev)
    # nu/c of every record and channel comes from the TIME column (MS row
    # order: row = t * nbl + b, 2 s apart) through the TOPO -> LSRK conversion
    # (mtb_lsrk_freq_over_c), taken in the baseline-major record order
    # (record k = b * nt + t) -- once per step, on the device
    mscol = lsrk_inputs(torch, dev, spec, nbl, nt, freqs)
    packed = []
    nu = torch.empty((len(freqs), R), dtype=torch.float32, device=dev)
    mscol["run"](mscol["time"], mscol["index"], nu)
    for c, f in enumerate(freqs):
        vis = make_vis(uvw, f, srcs, torch, gen)
        # one byte per flag (mtb_grid_params.flags_u8 = 1) for the checks and
        # samples outside the timed region; the timed step and the e2e leg
        # take the same flags packed one bit per flag (flags_u8 = 2)
        flags = (torch.rand(R, device=dev, generator=gen) < spec["flag"]).to(torch.uint8)[:, None].repeat(1, 4).contiguous()
        chans.append((nu[c], vis, weights, flags))
        packed.append(pack_flags(flags))
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen

    # ---- w-kernels (once) and one imager per channel
    n = spec["nx"]
    kp = wkernel_params(n, n, dl, dl, spec["wplanes"], spec["sampling"], spec["trial_support"],
                        spec["max_support"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    kern = build_wkernels(kp, dev)
    torch.cuda.synchronize()
    wk_ms = (time.perf_counter() - t0) * 1e3
    imagers = [WProjectionImager(n, n, dl, wplanes=spec["wplanes"], sampling=spec["sampling"],
                                 trial_support=spec["trial_support"], max_support=spec["max_support"],
                                 kernels=kern, device=dev, tile=args.tile, support_bucket=args.support_bucket,
                                 max_chunk=args.max_chunk, merge=args.merge, gridder=args.gridder) for _ in freqs]
    images = [torch.empty((4, n, n), dtype=torch.float32, device=dev) for _ in freqs]
    gev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in freqs]
    for im, ev in zip(imagers, gev):
        for e in ev:          # torch creates the CUDA event on first record
            e.record()
        im.gridder_events = ev
    torch.cuda.synchronize()
    lat_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in freqs]

    # the channels of a step alternate over args.streams CUDA streams, so one
    # channel's finalisation overlaps the next channel's binning
    main_stream = torch.cuda.current_stream(dev)
    streams = [main_stream] + [torch.cuda.Stream(device=dev) for _ in range(max(1, args.streams) - 1)]

    def step(record_latency=True):
        mscol["run"](mscol["time"], mscol["index"], nu)
        begin = torch.cuda.Event()
        begin.record(main_stream)
        for st in streams[1:]:
            st.wait_event(begin)
        for c, (im, (freq, vis, weights, _), flags) in enumerate(zip(imagers, chans, packed)):
            st = streams[c % len(streams)]
            with torch.cuda.stream(st):
                if record_latency:
                    lat_ev[c][0].record(st)
                im.reset()
                im.grid_device(uvw, freq, vis, weights, flags)
                im.finalize(out=images[c])
                if record_latency:
                    lat_ev[c][1].record(st)
        for st in streams[1:]:
            done = torch.cuda.Event()
            done.record(st)
            main_stream.wait_event(done)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    stats = [im.statistics() for im in imagers]
    samples_per_step = sum((s["gridded_records"] + s["compressed_records"]) * 4 for s in stats)
    flops_per_step = sum(8.0 * 4 * s["gridded_points"] for s in stats)

    clocks = ClockSampler(local, args.clock_log)
    launches0 = lib.mtb_kernel_launch_count()
    lat, gms = [], []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    if args.profile_range:
        torch.cuda.profiler.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record()
    for _ in range(args.steps):
        step()
        torch.cuda.synchronize()
        lat += [a.elapsed_time(b) for a, b in lat_ev]
        gms.append(sum(a.elapsed_time(b) for a, b in gev))
    t_end.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    if args.profile_range:
        torch.cuda.profiler.stop()
    clk = clocks.stop()
    launches = (lib.mtb_kernel_launch_count() - launches0) // max(1, args.steps)
    ms = max_over_ranks(t_start.elapsed_time(t_end), world, dist, torch, dev)
    ms_per_step = ms / args.steps
    value = job_throughput(samples_per_step, world, ms_per_step)

    # ---- roofline of the gridder (FP32 FMA pipe; peak measured on this GPU)
    peak = ctypes.c_double(0)
    L.check(lib.mtb_calibrate_fp32(ctypes.byref(peak), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
            "mtb_calibrate_fp32")
    gridder_ms = float(np.mean(gms))
    achieved = flops_per_step / (gridder_ms * 1e-3) / 1e12
    # DRAM bytes of one gridder launch over one channel of this workload (8 h,
    # 4096^2), measured with ncu (dram__bytes_read.sum + dram__bytes_write.sum,
    # one pass; GRIDDER_TRAFFIC); other workloads and gridders were not captured
    gridder = args.gridder or 8
    traffic = (GRIDDER_TRAFFIC.get(gridder) if (spec["name"] == "mid" and spec["hours"] == 8.0 and R == 29030400)
               else None)
    props = torch.cuda.get_device_properties(dev)
    spec_peak = props.multi_processor_count * 128 * 2 * 1.965e9 / 1e12
    roof = {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
            "frac": achieved / peak.value if peak.value else None, "traffic": traffic,
            "traffic_unit": "bytes per gridder launch (one channel), ncu dram__bytes_read+write",
            "kernel": "k_grid7 (gridder %d: job segments + the streaming gridder of one mtb_grid call, "
                      "span timed by events)" % gridder if gridder in (7, 8) else "gridder %d" % gridder,
            "peak_source": "measured: mtb_calibrate_fp32 (packed f32x2 FMA chains, this GPU)",
            "peak_spec": spec_peak, "frac_of_spec": achieved / spec_peak,
            "peak_spec_source": "SMs x 128 FP32 lanes x 2 flop x 1965 MHz (clocks.max.sm)"}

    # ---- end to end: host buffers, H2D per channel overlapped with compute
    e2e = None
    if not args.no_e2e:
        # every rank pins a host copy of its inputs and images; with several
        # ranks on one host that can exceed its memory: all ranks skip the leg
        # (the same decision on every rank) when the node's share is too small
        unique = {id(t): t for ch in chans for t in ch}       # the shared weights count once
        pinned = uvw.numel() * 4 + sum(t.numel() * t.element_size() for t in unique.values()) + \
            sum(im.numel() * 4 for im in images)
        local_ranks = int(os.environ.get("LOCAL_WORLD_SIZE", str(world)))
        fits = pinned * local_ranks <= 0.6 * host_available_bytes()
        if world > 1:
            flag = torch.tensor([1 if fits else 0], device=dev)
            dist.all_reduce(flag, op=dist.ReduceOp.MIN)
            fits = bool(flag.item())
        if fits:
            e2e = run_e2e(args, torch, dev, uvw, chans, imagers, images, samples_per_step, world, dist, mscol,
                          packed)
        else:
            e2e = {"value": None, "skipped": "pinned host copies of %d ranks (%.0f GB) exceed 60 %% of the host's "
                                          "available memory" % (local_ranks, pinned * local_ranks / 1e9)}

    # ---- the first channel's image against the FP64 oracle (rank 0, one GPU)
    oracle = None
    if rank == 0 and world == 1 and not args.no_oracle:
        oracle = oracle_check(spec, dl, uvw, chans[0], images[0], kern)

    # ---- CPU baseline (rank 0, one GPU)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args, spec, uvw, chans, kern, dl, torch, nt)

    # ---- this gridder on the sample and chunking of the reference arm's GPU leg
    same = None
    if rank == 0 and world == 1 and not args.no_cpu:
        same = reference_sample_gpu(args, spec, uvw, chans, kern, dl, torch, nt, dev)

    # ---- TOPO -> LSRK frequencies of the workload's records (rank 0, one GPU)
    lsrk = None
    if rank == 0 and world == 1 and not args.no_lsrk:
        lsrk = run_lsrk(torch, dev, nt, nbl, freqs)

    # ---- batched cubes and the request stream (rank 0, one GPU): the other
    # two configurations of the workload, measured after the main line
    cube, serve = None, None
    if rank == 0 and world == 1 and (not args.no_cube or not args.no_serve):
        chans.clear()
        imagers.clear()
        images.clear()
        del uvw, weights
        torch.cuda.empty_cache()
        if not args.no_cube:
            cube = run_cube(args, torch, dev)
            torch.cuda.empty_cache()
        if not args.no_serve:
            serve = run_serve(args, torch, dev)

    if rank == 0:
        sup = kern.supports
        line = {
            "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 coordinates and w-phase)",
            "data": "synthetic (seeded earth-rotation tracks, point-source sky; one weights array shared by the "
                    "channels, as the MS WEIGHT column; nu/c of every record and channel converted TOPO -> LSRK "
                    "from the TIME column on the device every step)",
            "config": {"workload": workload_name(spec), "records_per_channel": R, "channels": len(freqs),
                       "image": n, "cell_arcsec": dl / ARCSEC, "wplanes": spec["wplanes"],
                       "sampling": spec["sampling"], "supports": [int(sup.min()), int(sup.max())],
                       "samples_per_step": samples_per_step, "l2": "inputs larger than L2 (1.6 GB per channel)",
                       "flags": "bit-packed, uint8 [R*4/8] (flags_u8 = 2)", "streams": args.streams,
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "images_per_s": len(freqs) * world / (ms_per_step * 1e-3),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "roofline": roof, "gpu_launches": int(launches), "wkernel_ms": wk_ms,
            "gridder_ms_per_step": gridder_ms, "datagen_s": t_gen,
        }
        if e2e:
            line["e2e"] = e2e
        if cpu:
            line["cpu_baseline"] = cpu
        if same:
            line["reference_sample_gpu"] = same
        if clk:
            line["clocks"] = clk
        if oracle:
            line["oracle_check"] = oracle
        if cube:
            line["cube"] = cube
        if lsrk:
            line["lsrk"] = lsrk
        if serve:
            line["serving"] = serve
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_e2e(args, torch, dev, uvw_d, chans, imagers, images, samples_per_step, world, dist, mscol, packed):
    """Same metric through the public API from pinned host buffers: per step
    the H2D copy of every channel's records (and of the arrays the channels
    share: uvw, the weights, the TIME column and the record order) and the
    D2H of every image are inside the timed region; nu/c of every channel is
    computed on the device from the TIME column (mtb_lsrk_freq_over_c), as
    the MeasurementSet holds no per-record frequency column.  H2D copies run on a side stream,
    double-buffered against the compute of the previous channel; each image's
    D2H runs on a third stream once it is finalised.  Steps follow each other
    without a device drain (a streaming imager): events guard every buffer
    reuse, and the timed region ends after the last image is on the host."""
    def pinned(t):
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        h.copy_(t)
        return h

    shared_w = all(ch[2] is chans[0][2] for ch in chans)
    host_uvw = pinned(uvw_d)
    host_w = pinned(chans[0][2]) if shared_w else None
    host_time, host_index = pinned(mscol["time"]), pinned(mscol["index"])
    time_bufs = [torch.empty_like(mscol["time"]) for _ in range(2)]
    index_bufs = [torch.empty_like(mscol["index"]) for _ in range(2)]
    nu_bufs = [torch.empty((len(chans), uvw_d.shape[1]), dtype=torch.float32, device=dev) for _ in range(2)]
    # per channel: vis, bit-packed flags (and weights when the channels do not share them)
    host = [[pinned(t) for t in ((v, fl) if shared_w else (v, w, fl))]
            for (f, v, w, _), fl in zip(chans, packed)]
    out_host = [torch.empty(im.shape, dtype=im.dtype, pin_memory=True) for im in images]
    nslots = max(2, args.e2e_slots)
    bufs = [[torch.empty(t.shape, dtype=t.dtype, device=dev) for t in host[0]] for _ in range(nslots)]
    uvw_bufs = [torch.empty_like(uvw_d) for _ in range(2)]
    w_bufs = [torch.empty_like(chans[0][2]) for _ in range(2)] if shared_w else None
    copy = torch.cuda.Stream(device=dev)
    back = torch.cuda.Stream(device=dev)
    comp = torch.cuda.current_stream(dev)
    h2d = host_uvw.numel() * 4 + (host_w.numel() * 4 if shared_w else 0) + host_time.numel() * 8 + \
        host_index.numel() * 4 + sum(sum(t.numel() * t.element_size() for t in hc) for hc in host)
    d2h = sum(o.numel() * 4 for o in out_host)
    ref_image = images[-1].clone()          # the device path's image of the last channel
    # events: buffer pair free (last gridding that read it done), uvw buffer
    # free, image c read back
    state = dict(seq=0, free=[None] * nslots, uvw_free=[None, None], back=[None] * len(host), shared={})

    def record(stream):
        e = torch.cuda.Event()
        e.record(stream)
        return e

    def shared_pairs(p):
        pairs = [(time_bufs[p], host_time), (index_bufs[p], host_index), (uvw_bufs[p], host_uvw)]
        return pairs + ([(w_bufs[p], host_w)] if shared_w else [])

    def shared_copy(n, part=0, parts=1):
        """H2D of step n's shared arrays (TIME, record order, uvw, weights)
        into the buffers of its parity once step n - 2 has released them,
        whole or as slice `part` of `parts` of every array."""
        p = n % 2
        with torch.cuda.stream(copy):
            if part == 0 and state["uvw_free"][p] is not None:
                copy.wait_event(state["uvw_free"][p])
            for dst, src in shared_pairs(p):
                d, h = dst.view(-1), src.view(-1)
                a, b = d.numel() * part // parts, d.numel() * (part + 1) // parts
                d[a:b].copy_(h[a:b], non_blocking=True)
            if part == parts - 1:
                state["shared"][n] = record(copy)

    def step(n, prefetch_next):
        """Step n; with prefetch_next, step n + 1's shared arrays follow this
        step's channel copies on the copy stream in slices (one after each
        channel from the second on), so that no whole-array copy stands
        between one step's last channel and the next step's first."""
        p = n % 2
        ub = uvw_bufs[p]
        wb = w_bufs[p] if shared_w else None
        tb, ib, nub = time_bufs[p], index_bufs[p], nu_bufs[p]
        nch = len(host)
        if n not in state["shared"]:
            shared_copy(n)
        comp.wait_event(state["shared"].pop(n))
        mscol["run"](tb, ib, nub)
        for c, hc in enumerate(host):
            k = state["seq"] % nslots
            state["seq"] += 1
            b = bufs[k]
            with torch.cuda.stream(copy):
                if state["free"][k] is not None:
                    copy.wait_event(state["free"][k])
                for dst, src in zip(b, hc):
                    dst.copy_(src, non_blocking=True)
                ready = record(copy)
            if prefetch_next and (nch == 1 or c >= 1):
                shared_copy(n + 1, 0 if nch == 1 else c - 1, 1 if nch == 1 else nch - 1)
            comp.wait_event(ready)
            im = imagers[c]
            im.reset()
            if shared_w:
                im.grid_device(ub, nub[c], b[0], wb, b[1])
            else:
                im.grid_device(ub, nub[c], *b)
            state["free"][k] = record(comp)
            if state["back"][c] is not None:
                comp.wait_event(state["back"][c])      # images[c] of the last step is on the host
            im.finalize(out=images[c])
            back.wait_event(record(comp))
            with torch.cuda.stream(back):
                out_host[c].copy_(images[c], non_blocking=True)
                state["back"][c] = record(back)
        state["uvw_free"][p] = record(comp)

    # the host link's own rate, outside the timed region: pinned H2D copies of
    # one channel's visibilities alone on the copy stream
    vis_h, vis_d = host[0][0], bufs[0][0]
    with torch.cuda.stream(copy):
        vis_d.copy_(vis_h, non_blocking=True)
        l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0.record(copy)
        for _ in range(3):
            vis_d.copy_(vis_h, non_blocking=True)
        l1.record(copy)
    torch.cuda.synchronize()
    link_gbs = 3 * vis_h.numel() * vis_h.element_size() / (l0.elapsed_time(l1) * 1e-3) / 1e9

    # steady streaming: every step queues the next step's shared arrays behind
    # its channel copies, so the timed region holds K sets of them (those of
    # steps 2..K+1; step 1's came with the warm-up step), every copy ending
    # inside it
    step(0, True)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    K = args.e2e_steps
    for n in range(1, K + 1):
        step(n, True)
    for e in state["back"]:
        comp.wait_event(e)
    comp.wait_event(state["shared"].pop(K + 1))
    b.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(a.elapsed_time(b) / args.e2e_steps, world, dist, torch, dev)
    # the image that came back to the host equals the device path's (to the
    # rounding of the FP32 reductions)
    ref = ref_image.cpu().numpy()
    got = out_host[-1].numpy()
    check = float(np.sqrt(np.mean((got - ref) ** 2)) / max(float(np.abs(ref[0]).max()), 1e-30))
    if not check <= 1e-5:
        raise RuntimeError("e2e image differs from the device path: rms/peak %g" % check)
    return {"value": job_throughput(samples_per_step, world, ms), "unit": "samples/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": ms, "image_check_rms": check,
            "h2d_gbs": h2d / (ms * 1e-3) / 1e9, "h2d_link_gbs": link_gbs,
            "h2d_link_note": "h2d_link_gbs: pinned copies of one channel's visibilities alone, before the timed region"}


# ---------------------------------------------------------------- serving --
SERVE_WPLANES = {512: 32, 1024: 64, 2048: 96, 4096: 128}


def make_request_pool(torch, dev, rng, records):
    """Host record arrays the serving requests take slices of (views, no
    copies): the 64-antenna 8 h, 2 s track repeated over channels between 1.3
    and 1.5 GHz until it holds `records` records (records stay baseline-major
    within a channel), 4 pol visibilities of a 3-source sky per channel, 10 %
    of records flagged."""
    from mtb import synth
    spec = workload_spec(argparse.Namespace(config="mid", channels=1, hours=8.0))
    uvw1, _, _ = make_uvw(spec, dev, torch, rng)
    R1 = uvw1.shape[1]
    nch = max(1, -(-int(records) // R1))
    Rp = nch * R1
    freqs = np.linspace(1.3e9, 1.5e9, nch) if nch > 1 else np.array([1.4e9])
    uv_max = float(uvw1[:2].abs().max())
    gen = torch.Generator(device=dev).manual_seed(11)
    pool = dict(uvw=np.empty((3, Rp), np.float32), freq=np.empty(Rp, np.float32),
                vis=np.empty((Rp, 4), np.complex64), weights=np.ones((Rp, 4), np.float32),
                flags=np.empty((Rp, 4), np.uint8), uv_max=uv_max)
    u1 = uvw1.cpu().numpy()
    srcs = synth.random_sources(3, 4096 * cell_for(dict(spec, nx=4096, f_hi=1.5e9), uv_max, torch), rng,
                                flux=(0.1, 1.0))
    for c, f in enumerate(freqs):
        sl = slice(c * R1, (c + 1) * R1)
        pool["uvw"][:, sl] = u1
        pool["freq"][sl] = f / C_LIGHT
        pool["vis"][sl] = make_vis(uvw1, f, srcs, torch, gen).cpu().numpy()
        pool["flags"][sl] = ((torch.rand(R1, device=dev, generator=gen) < 0.1).to(torch.uint8)[:, None].repeat(1, 4)
                             .cpu().numpy())
    return pool


def make_requests(args, torch, dev, rng):
    """A stream of imaging requests in the shape of the serving configuration:
    image size uniform over {512, 1024, 2048, 4096}^2, record counts
    log-uniform in [serve_min_records, serve_max_records], each a contiguous
    slice of the request pool (synthetic 64-antenna tracks, 4 pol, point-source
    sky, 10 % flagged), w-planes 32-128 by image size, Poisson arrivals at
    serve_rate per second."""
    spec = workload_spec(argparse.Namespace(config="mid", channels=1, hours=8.0))
    pool = make_request_pool(torch, dev, rng, args.serve_max_records)
    Rp = pool["freq"].size
    reqs = []
    t = 0.0
    for k in range(args.serve_requests):
        n = int(rng.choice([512, 1024, 2048, 4096]))
        R = int(math.exp(rng.uniform(math.log(args.serve_min_records), math.log(args.serve_max_records))))
        R = min(R, Rp)
        s0 = int(rng.integers(0, Rp - R + 1))
        dl = cell_for(dict(spec, nx=n, f_hi=1.5e9), pool["uv_max"], torch)
        t += float(rng.exponential(1.0 / args.serve_rate))
        sl = slice(s0, s0 + R)
        reqs.append(dict(nx=n, dl=dl, wplanes=SERVE_WPLANES[n], arrival=t, uvw=pool["uvw"][:, sl],
                         freq=pool["freq"][sl], vis=pool["vis"][sl], weights=pool["weights"][sl],
                         flags=pool["flags"][sl]))
    return reqs


def run_cube(args, torch, dev):
    """Batched cubes: independent channel images with uneven record counts
    (64-antenna tracks of U(cube_min_hours, cube_max_hours) at 2 s, flagging
    U(0, 60 %)), image size 1024^2 or 2048^2 per image, 64 w-planes, supports
    up to 49, inputs resident in HBM.  Every image's records are gridded in
    chunks of cube_chunk records: (a) image by image with mtb_grid, (b) chunk
    by chunk for all images at once with mtb_grid_batch (one persistent
    gridder launch per chunk index), with default knobs and then with the
    knobs the autotuner picks on the cube's first chunks, (c) the tuned chunk
    sequence replayed from one captured CUDA graph.  Samples/s of the gridding
    of every image."""
    from mtb.imager import WProjectionImager, autotune, build_wkernels, grid_batch, wkernel_params
    rng = np.random.default_rng(4)
    spec = workload_spec(argparse.Namespace(config="mid", channels=1, hours=8.0))
    pool, nbl, nt = make_uvw(spec, dev, torch, rng)
    uv_max = float(pool[:2].abs().max())
    gen = torch.Generator(device=dev).manual_seed(13)
    chunk = int(args.cube_chunk)
    ones = torch.ones((min(chunk, nbl * nt), 4), dtype=torch.float32, device=dev)   # shared weights
    kern = {}
    images = []      # (imager, [chunk arrays])
    for k in range(args.cube_images):
        n = int(rng.choice([1024, 2048]))
        hours = float(rng.uniform(args.cube_min_hours, args.cube_max_hours))
        ntk = max(1, min(nt, int(hours * 1800)))
        # the first ntk integrations of every baseline (records stay baseline-major)
        sel = pool.reshape(3, nbl, nt)[:, :, :ntk].reshape(3, -1)
        R = sel.shape[1]
        dl = cell_for(dict(spec, nx=n, max_support=49), uv_max, torch)
        if n not in kern:
            kern[n] = build_wkernels(wkernel_params(n, n, dl, dl, 64, 8, 51, 49), dev)
        f = float(rng.uniform(1.3e9, 1.5e9))
        srcs = sources_for(dict(spec, nsrc=20), n * dl, rng)
        frac = float(rng.uniform(0.0, 0.6))
        im = WProjectionImager(n, n, dl, wplanes=64, sampling=8, trial_support=51, max_support=49, kernels=kern[n],
                               device=dev)
        chunks = []
        for a0 in range(0, R, chunk):
            b0 = min(R, a0 + chunk)
            u = sel[:, a0:b0].contiguous()
            chunks.append((u, torch.full((b0 - a0,), f / C_LIGHT, dtype=torch.float32, device=dev),
                           make_vis(u, f, srcs, torch, gen), ones[:b0 - a0],
                           (torch.rand(b0 - a0, device=dev, generator=gen) < frac).to(torch.uint8)[:, None].repeat(1, 4)
                           .contiguous()))
        images.append((im, chunks))
    del pool
    torch.cuda.synchronize()
    nchunks = max(len(c) for _, c in images)

    def single():
        for im, chunks in images:
            im.reset()
            for arrs in chunks:
                im.grid_device(*arrs)
            im._ws = None    # one workspace at a time (the allocator reuses it)

    ws = [None]

    def batched():
        for im, _ in images:
            im.reset()
        for c in range(nchunks):
            ws[0] = grid_batch([(im, *chunks[c]) for im, chunks in images if c < len(chunks)], workspace=ws[0])

    def timed(fn, reps=3):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    ms_single = timed(single)
    stats = [im.statistics() for im, _ in images]
    samples = sum((s["gridded_records"] + s["compressed_records"]) * 4 for s in stats)
    torch.cuda.empty_cache()
    ms_default = timed(batched)
    # autotune the batch's knobs on the cube's first chunks, then time the tuned batch
    for im, _ in images:
        im.reset()
    ws[0] = None              # the autotuner sizes its own (largest-candidate) workspace
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    best, cands, ws[0] = autotune([(im, *chunks[0]) for im, chunks in images])
    tune_s = time.perf_counter() - t0
    ms_batch = timed(batched)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        batched()
    ms_graph = timed(graph.replay)
    del graph
    recs = [sum(a[1].numel() for a in chunks) for _, chunks in images]
    return {"images": len(images), "records": {"min": int(min(recs)), "max": int(max(recs)), "total": int(sum(recs))},
            "image_sizes": sorted({im.nx for im, _ in images}), "chunk_records": chunk, "chunk_calls": nchunks,
            "samples_per_image_set": int(samples),
            "per_image_launches": {"ms": ms_single, "samples_per_s": samples / (ms_single * 1e-3)},
            "one_batched_launch_default_knobs": {"ms": ms_default, "samples_per_s": samples / (ms_default * 1e-3)},
            "autotune": {"best": best, "seconds": tune_s,
                         "fastest_candidates": sorted(cands, key=lambda c: c["ms"])[:4]},
            "one_batched_launch": {"ms": ms_batch, "samples_per_s": samples / (ms_batch * 1e-3),
                                   "knobs": "autotuned"},
            "batched_cuda_graph": {"ms": ms_graph, "samples_per_s": samples / (ms_graph * 1e-3)}}


def run_serve(args, torch, dev):
    """The request stream through (a) the engine (continuous batching,
    w-kernel cache, overlapping slots) with real-time Poisson arrivals, and
    (b) the plain path, one request at a time in arrival order, each building
    its w-kernels as the reference does per run.  Reports p50/p99 latency
    (arrival to image on the host) and samples/s over the stream for both."""
    import queue
    import threading
    from mtb.engine import Engine
    from mtb.imager import WProjectionImager
    rng = np.random.default_rng(5)
    t_gen = time.perf_counter()
    reqs = make_requests(args, torch, dev, rng)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    common = dict(sampling=8, trial_support=67, max_support=65)
    # warm-up (untimed, both paths): the smallest request of every image size
    warm = []
    for n in sorted({r["nx"] for r in reqs}):
        warm.append(min((r for r in reqs if r["nx"] == n), key=lambda r: r["freq"].size))

    kcache = {}

    def plain(r, cached=False):
        """One request alone: w-kernels built for it (as the reference does
        per run) or, cached=True, taken from a per-geometry cache."""
        key = (r["nx"], r["dl"], r["wplanes"])
        im = WProjectionImager(r["nx"], r["nx"], r["dl"], wplanes=r["wplanes"], device=dev,
                               kernels=kcache.get(key) if cached else None, **common)
        k = im.build_kernels()
        if cached:
            kcache[key] = k
        R = r["freq"].size
        for a in range(0, R, 1 << 22):
            b = min(R, a + (1 << 22))
            im.grid_chunk(r["uvw"][:, a:b], r["freq"][a:b], r["vis"][a:b], r["weights"][a:b], r["flags"][a:b])
        im.finalize().cpu().numpy()
        st = im.statistics()
        return (st["gridded_records"] + st["compressed_records"]) * 4

    for r in warm:
        plain(r)
    torch.cuda.synchronize()

    # (b) plain path: service times measured back to back, then FIFO queueing
    def plain_stream(cached):
        service, samples = [], 0
        for r in reqs:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            samples += plain(r, cached)
            service.append(time.perf_counter() - t0)
        done, lat = 0.0, []
        for r, sv in zip(reqs, service):
            start = max(r["arrival"], done)
            done = start + sv
            lat.append((done - r["arrival"]) * 1e3)
        return service, samples, lat, done - reqs[0]["arrival"]

    service, samples_plain, lat_plain, span_plain = plain_stream(False)
    for r in warm:                # the cache starts with the warm-up geometries, as the engine's does
        plain(r, True)
    service_c, samples_c, lat_c, span_c = plain_stream(True)

    # (a) engine, real-time arrivals; a waiter thread collects results as they
    # finish (images dropped) while this thread submits
    def submit(eng, r):
        return eng.submit(r["nx"], r["nx"], r["dl"], r["dl"], r["wplanes"], 8, r["uvw"], r["freq"], r["vis"],
                          r["weights"], r["flags"], trial_support=67, max_support=65)

    results, queue_service = [], []
    # the plain path's device memory goes back to the driver: the engine sizes
    # its HBM budget from the free memory when it starts
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    with Engine(slots=args.serve_slots) as eng:
        # every slot runs one request of every image size (slot buffers grow
        # to the largest geometry; w-kernels and FFT plans built)
        for r in warm:
            for t in [submit(eng, r) for _ in range(args.serve_slots)]:
                eng.wait(t)
        tickets = queue.Queue()

        def waiter():
            for sub, tk in iter(tickets.get, None):
                res = eng.wait(tk)
                results.append((sub, res.status, res.latency_ms, res.kernel_cache_hit,
                                res.stats["gridded_records"] + res.stats["compressed_records"]))
                queue_service.append((res.queue_ms, res.service_ms))

        th = threading.Thread(target=waiter)
        th.start()
        t_base = time.perf_counter()
        for r in reqs:
            now = time.perf_counter() - t_base
            if r["arrival"] > now:
                time.sleep(r["arrival"] - now)
            sub = time.perf_counter() - t_base
            tickets.put((sub, submit(eng, r)))
        tickets.put(None)
        th.join()
        # saturation: every request queued at once (the engine's capacity; the
        # plain path's is its total service time)
        burst = []
        tickets = queue.Queue()

        def burst_waiter():
            for tk in iter(tickets.get, None):
                res = eng.wait(tk)
                burst.append((res.status, res.stats["gridded_records"] + res.stats["compressed_records"]))

        th = threading.Thread(target=burst_waiter)
        th.start()
        t0 = time.perf_counter()
        for r in reqs:
            tickets.put(submit(eng, r))
        tickets.put(None)
        th.join()
        burst_s = time.perf_counter() - t0
    bad = [st for _, st, _, _, _ in results if st != 0] + [st for st, _ in burst if st != 0]
    if bad:
        raise RuntimeError("engine request failed: status %d" % bad[0])
    samples_eng = sum(4 * n for *_, n in results)
    lat_eng = [lat for _, _, lat, _, _ in results]
    end = max(sub + lat * 1e-3 for sub, _, lat, _, _ in results)
    span_eng = end - min(sub for sub, *_ in results)
    hits = sum(h for _, _, _, h, _ in results)
    recs = [r["freq"].size for r in reqs]
    return {
        "requests": len(reqs), "arrival_rate_per_s": args.serve_rate, "slots": args.serve_slots,
        "image_sizes": [512, 1024, 2048, 4096],
        "warm_up": "untimed requests of every image size through each path (engine: one per slot and size, so "
                   "w-kernels are cached and every slot's buffers are grown; plain path: one per size, allocator "
                   "and FFT plans warm, w-kernels rebuilt per request)",
        "records": {"min": int(min(recs)), "max": int(max(recs)), "total": int(sum(recs)),
                    "range": [args.serve_min_records, args.serve_max_records]},
        "engine": {"samples_per_s": samples_eng / span_eng, "p50_ms": float(np.percentile(lat_eng, 50)),
                   "p99_ms": float(np.percentile(lat_eng, 99)), "makespan_s": span_eng, "kernel_cache_hits": hits,
                   "mean_queue_ms": float(np.mean([q for q, _ in queue_service])),
                   "mean_service_ms": float(np.mean([v for _, v in queue_service])),
                   "max_service_ms": float(np.max([v for _, v in queue_service]))},
        "plain": {"samples_per_s": samples_plain / span_plain, "p50_ms": float(np.percentile(lat_plain, 50)),
                  "p99_ms": float(np.percentile(lat_plain, 99)), "makespan_s": span_plain,
                  "mean_service_ms": float(np.mean(service)) * 1e3,
                  "w_kernels": "built for every request (as the reference does per run)"},
        "plain_cached_kernels": {"samples_per_s": samples_c / span_c, "p50_ms": float(np.percentile(lat_c, 50)),
                                 "p99_ms": float(np.percentile(lat_c, 99)), "makespan_s": span_c,
                                 "mean_service_ms": float(np.mean(service_c)) * 1e3,
                                 "w_kernels": "cached per geometry (isolates the engine's overlap from its cache)"},
        "speedup_samples_per_s": (samples_eng / span_eng) / (samples_plain / span_plain),
        "speedup_vs_cached_plain": (samples_eng / span_eng) / (samples_c / span_c),
        "saturation": {"engine_samples_per_s": sum(4 * n for _, n in burst) / burst_s, "engine_makespan_s": burst_s,
                       "plain_samples_per_s": samples_plain / float(np.sum(service)),
                       "plain_cached_samples_per_s": samples_c / float(np.sum(service_c)),
                       "speedup": (sum(4 * n for _, n in burst) / burst_s) / (samples_plain / float(np.sum(service))),
                       "speedup_vs_cached_plain": (sum(4 * n for _, n in burst) / burst_s) /
                                                  (samples_c / float(np.sum(service_c))),
                       "note": "all requests queued at once; plain = total samples / summed service times"},
        "datagen_s": t_gen,
    }


LSRK_SITE = (5109360.133, 2006852.586, -3238948.127)   # ITRF metres of a site at latitude -30.7 deg
LSRK_T0 = 60389.0 * 86400.0                              # MJD seconds of the first time sample


def lsrk_inputs(torch, dev, spec, nbl, nt, freqs):
    """The TIME column of the workload's rows in MeasurementSet order (row =
    t * nbl + b, spec["dt"] apart), the record order that takes them to the
    baseline-major records (record b * nt + t is row t * nbl + b), the
    channel frequencies, and a call that writes nu/c [nchan][R] from them on
    the current stream with a reused workspace."""
    from mtb.lsrk import lsrk_freq_over_c, lsrk_workspace_bytes
    times = LSRK_T0 + spec["dt"] * torch.arange(nt, dtype=torch.float64, device=dev)
    time_rows = times.repeat_interleave(nbl)
    index = torch.arange(nt * nbl, device=dev, dtype=torch.int32).view(nt, nbl).t().contiguous().view(-1)
    chan = torch.tensor(np.asarray(freqs, np.float64), device=dev)
    ws = torch.empty(lsrk_workspace_bytes(nt * nbl), dtype=torch.uint8, device=dev)
    ra, dec = 1.2, math.radians(spec["dec"])

    def run(time_s, idx, out):
        return lsrk_freq_over_c(time_s, chan, LSRK_SITE, ra, dec, index=idx, device=dev, out=out, workspace=ws)
    return {"time": time_rows, "index": index, "run": run}


def run_lsrk(torch, dev, nt, nbl, freqs, reps=5):
    """mtb_lsrk_freq_over_c on the workload's rows: a MeasurementSet-order
    TIME column (nt times x nbl baselines, 2 s apart), every channel, taken
    in the baseline-major record order; CUDA events around each call on its
    stream, outside the timed region.  Algorithmic bytes per call: the time
    column (8 B per row), the index (4 B per record) and nu/c (4 B per record
    and channel); the peak is MEASURED_PEAKS.json's copy bandwidth when the
    file is there.  The oracle checks the records of 24 spread-out times."""
    from mtb.lsrk import lsrk_freq_over_c
    from oracle import lsrk_oracle as O
    site, ra, dec = (5109360.133, 2006852.586, -3238948.127), 2.1, -0.7
    t0 = 60389.0 * 86400.0
    times = t0 + 2.0 * np.arange(nt)
    t_rows = torch.from_numpy(times).to(dev).repeat_interleave(nbl)            # row = t * nbl + b
    index = torch.arange(nt * nbl, device=dev, dtype=torch.int32).view(nt, nbl).t().contiguous().view(-1)
    chan = np.asarray(freqs, np.float64)
    st = torch.cuda.current_stream()
    out = lsrk_freq_over_c(t_rows, chan, site, ra, dec, index=index)        # warm-up: plan, caches
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for a, b in ev:
        a.record(st)
        out = lsrk_freq_over_c(t_rows, chan, site, ra, dec, index=index)
        b.record(st)
    torch.cuda.synchronize()
    ms = sorted(a.elapsed_time(b) for a, b in ev)[reps // 2]
    rows = nt * nbl
    nbytes = 8 * rows + 4 * rows + 4 * rows * len(chan)
    pick = np.linspace(0, nt - 1, 24).astype(int)
    got = out.view(len(chan), nbl, nt)[:, 0, pick].cpu().numpy()               # baseline 0 at the picked times
    ref = O.lsrk_freq_over_c(times[pick], chan, site, ra, dec)
    ulps = int(np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64)).max())
    same = bool((out.view(len(chan), nbl, nt) == out.view(len(chan), nbl, nt)[:, :1, :]).all())
    peak, src = None, None
    pk = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        with open(pk) as fh:
            peak, src = json.load(fh).get("hbm_gbs"), "MEASURED_PEAKS.json hbm_gbs (copy)"
    gbs = nbytes / (ms * 1e-3) / 1e9
    del out, t_rows, index
    torch.cuda.empty_cache()
    return {"rows": rows, "channels": len(chan), "ms": ms, "algorithmic_bytes": nbytes, "achieved_gbs": gbs,
            "peak_gbs": peak, "frac": gbs / peak if peak else None, "peak_source": src,
            "oracle_max_ulps": ulps, "every_baseline_same_per_time": same,
            "kernels": "k_lsrk_heads (FP64 velocity per distinct time) + CUB max-scan + k_lsrk_write"}


def oracle_check(spec, dl, uvw_d, chan, image_d, kern):
    """The image of one full channel against the FP64 W-projection oracle
    (oracle/, on the host cores), outside the timed region: the RMS error of
    every Stokes plane relative to the Stokes I peak (bound 1e-5), and the
    kernel table's largest deviation (bound 1e-6)."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    n = spec["nx"]
    geo = O.kernel_geometry(n, n, dl, dl, spec["wplanes"], spec["sampling"], spec["trial_support"],
                            spec["max_support"])
    ko = O.wkernels(geo)
    if not np.array_equal(ko["conv_info"], kern.conv_info):
        return {"error": "kernel supports differ from the oracle's"}
    tab_err = float(np.abs(kern.table.cpu().numpy() - ko["table"]).max())
    freq, vis, weights, flags = chan
    g, nrm, _ = O.grid_chunk(uvw_d.cpu().numpy(), freq.cpu().numpy(), vis.cpu().numpy(), weights.cpu().numpy(),
                             flags.cpu().numpy().astype(np.int32), geo, ko)
    img_o = O.finalize(g, nrm, geo)
    img = image_d.cpu().numpy()
    peak = float(np.abs(img_o[0]).max())
    err = {s: float(np.sqrt(np.mean((img[p] - img_o[p]) ** 2)) / peak) for p, s in enumerate("IQUV")}
    return {"image_rms_vs_oracle": err, "bound": 1e-5, "kernel_table_max_abs_err": tab_err, "kernel_bound": 1e-6,
            "records": int(uvw_d.shape[1]), "oracle_s": time.perf_counter() - t0,
            "oracle": "FP64 W-projection restatement (oracle/wproj_oracle.c + numpy FFT), host cores"}


def reference_sample_gpu(args, spec, uvw_d, chans, kern, dl, torch, nt, dev):
    """mtb_grid on the records the reference arm's GPU leg grids (the CPU
    sample: the first baselines of the middle channel over the full track) in
    chunks of the reference's default 1,000,000 records, timed with CUDA
    events: samples/s over the gridder kernels' span and over whole mtb_grid
    calls, with a plain FP32 grid as the reference accumulates (the
    like-for-like comparison with that leg's reference operators), and over
    whole calls with the default two-float grid, whose per-call merge of the
    delta grid (4096^2 x 4 pol) weighs on 1,000,000-record chunks."""
    from mtb.imager import WProjectionImager
    n_rec = min(uvw_d.shape[1], cpu_sample_records(args, spec, nt))
    freq, vis, weights, flags = chans[len(chans) // 2]
    n = spec["nx"]
    bounds = list(range(0, n_rec, REF_CHUNK)) + [n_rec]
    chunks = [(uvw_d[:, a:b].contiguous(), freq[a:b].contiguous(), vis[a:b].contiguous(),
               weights[a:b].contiguous(), flags[a:b].contiguous()) for a, b in zip(bounds[:-1], bounds[1:])]

    def run(compensated):
        im = WProjectionImager(n, n, dl, wplanes=spec["wplanes"], sampling=spec["sampling"],
                               trial_support=spec["trial_support"], max_support=spec["max_support"], kernels=kern,
                               gridder=args.gridder, compensated=compensated)
        gev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        for e in gev:         # torch creates the CUDA event on first record
            e.record()
        im.gridder_events = gev

        def once():
            im.reset()
            g_ms, c_ms = 0.0, 0.0
            for c in chunks:
                c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                c0.record()
                im.grid_device(*c)
                c1.record()
                torch.cuda.synchronize()
                g_ms += gev[0].elapsed_time(gev[1])
                c_ms += c0.elapsed_time(c1)
            return g_ms, c_ms
        once()                                # workspace and plans
        g_ms, c_ms = once()
        st = im.statistics()
        return (st["gridded_records"] + st["compressed_records"]) * 4, g_ms, c_ms
    samples, g_ms, c_ms = run(False)
    _, _, cc_ms = run(True)
    return {"value": samples / (c_ms * 1e-3), "unit": "samples/s", "gridder_value": samples / (g_ms * 1e-3),
            "gridder_ms": g_ms, "calls_ms": c_ms, "grid": "plain FP32 (as the reference accumulates)",
            "compensated_value": samples / (cc_ms * 1e-3), "compensated_calls_ms": cc_ms,
            "records": int(n_rec), "chunk_records": REF_CHUNK,
            "sample": "the cpu_baseline sample in chunks of %d records: the records and chunking of the "
                      "reference arm's reference_gpu leg" % REF_CHUNK}


def cpu_sample_records(args, spec, nt):
    """Records of the CPU sample, the same for this line's cpu_baseline and the
    --impl reference arm: the first args.ref_baselines baselines of one channel
    over the full track (records are baseline-major), or --cpu-records."""
    if args.cpu_records:
        return int(args.cpu_records)
    nbl_all = spec["n_ant"] * (spec["n_ant"] - 1) // 2
    return min(args.ref_baselines, nbl_all) * nt if spec["name"] == "mid" else nbl_all * nt


def cpu_baseline(args, spec, uvw_d, chans, kern, dl, torch, nt, min_seconds=12.0, max_passes=40):
    """FP32 OpenMP port of the reference's gridding on the host cores, on a
    bounded sample (cpu_sample_records) of one channel, gridded repeatedly
    until about min_seconds of CPU time have been spent."""
    from oracle import oracle as O
    R = uvw_d.shape[1]
    n_rec = min(R, cpu_sample_records(args, spec, nt))
    freq, vis, weights, flags = chans[len(chans) // 2]
    u = np.ascontiguousarray(uvw_d[:, :n_rec].cpu().numpy())
    fq = np.ascontiguousarray(freq[:n_rec].cpu().numpy())
    vs = np.ascontiguousarray(vis[:n_rec].cpu().numpy())
    wt = np.ascontiguousarray(weights[:n_rec].cpu().numpy())
    fl = np.ascontiguousarray(flags[:n_rec].cpu().numpy(), dtype=np.int32)
    table = kern.table.cpu().numpy()
    sums = kern.conv_sums.cpu().numpy()
    ci = kern.conv_info
    n = spec["nx"]
    P = O.port()
    grid = np.zeros((n, n, 4), np.complex64)
    norm = np.zeros(4, np.float32)
    samples, passes, dt = 0, 0, 0.0
    while passes < max_passes and (passes == 0 or dt < min_seconds):
        st = np.zeros(4, np.int64)
        t0 = time.perf_counter()
        P.port_grid_chunk(n_rec, 4, O._p(u), O._p(fq), O._p(vs), O._p(wt), O._p(fl), spec["wplanes"],
                          kern.info.w_sq_increment, O._p(ci), O._p(sums), O._p(table), spec["sampling"], n, n,
                          kern.info.u_increment, kern.info.v_increment, O._p(grid), O._p(norm), O._p(st))
        dt += time.perf_counter() - t0
        samples += int(st[0] + st[1]) * 4
        passes += 1
    nbl_all = spec["n_ant"] * (spec["n_ant"] - 1) // 2
    return {"value": samples / dt, "unit": "samples/s", "cores": P.port_threads(), "kind": "port",
            "sample": "%d records of one %s channel (%d of %d baselines, full track), %d passes (%d samples "
                      "gridded in %.1f s), FP32 OpenMP port"
                      % (n_rec, spec["name"], n_rec // max(1, nt), nbl_all, passes, samples, dt)}


if __name__ == "__main__":
    main()
