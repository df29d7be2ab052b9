"""Generate the golden fixtures in this directory from mt-imager itself.

TEST INFRASTRUCTURE.  Runs mt-imager's own operator code (built by
oracle/build_ref.py from the reference sources into oracle/_ref/libmtref.so;
needs a GPU) on seeded synthetic chunks and stores inputs and outputs as
compressed .npz files:

  grid_<case>.npz   one or more WImager chunks (WImager.cpp:167-234):
                    inputs (uvw, nu/c, vis, weights, flags), the kernel table
                    they are gridded with (the FP64 oracle's, rounded to
                    complex64, with its convInfo and ConvSums), the seven
                    PreProcessUVW outputs of every chunk and the accumulated
                    grid from ConvolutionGridder.
  image_<case>.npz  ImageFinalizer (ImageFinalizer.cpp:31-44) applied to that
                    grid with the normaliser sum of the chunks' ConvSums.
  wkernels_<g>.npz  WProjectionConvFunction (WProjectionConvFunction.cpp:
                    186-291): kernel table, convInfo, ConvSums and the w=0
                    divisor for a geometry.
  taper_<g>.npz     mode=normal kernel (OnlyTaperConvFunction.cpp:29-99):
                    table and ConvSums for a support and oversampling.

    python tests/golden/make_golden.py [--out DIR]
"""
from __future__ import annotations

import argparse
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "mt-imager_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

from mtb import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

# name: (observation and geometry, number of chunks, npol)
CASES = {
    # 45 baselines x 120 integrations, even oversampling, supports 7-9, two chunks
    "even_s4": dict(obs=dict(seed=11, n_ant=10, ntimes=120, nx=128, cell_arcsec=60.0, wplanes=8, sampling=4,
                             radius_m=300.0, flag_frac=0.1, dec_deg=-80.0, nsrc=4), chunks=2, npol=4),
    # odd oversampling, two polarisations
    "odd_s3_p2": dict(obs=dict(seed=12, n_ant=10, ntimes=120, nx=96, cell_arcsec=80.0, wplanes=6, sampling=3,
                               radius_m=300.0, flag_frac=0.1, dec_deg=-85.0, nsrc=3), chunks=1, npol=2),
    # wide field: supports 9-27, both of the reference's gridder kernels (S < 16 and S > 16)
    "wide_s4": dict(obs=dict(seed=13, n_ant=12, ntimes=80, nx=128, cell_arcsec=400.0, wplanes=8, sampling=4,
                             radius_m=150.0, flag_frac=0.1, dec_deg=-88.0, nsrc=3), chunks=1, npol=1,
                    w_max_from_data=True),
}


# name: (nx, cell arcsec, w-planes, oversampling); w_max by the reference's rule
KERNEL_GEOMETRIES = {
    "cap_s4": (128, 2000.0, 6, 4),     # supports 7-31, the last planes at the S_t - 2 cap
    "odd_s3": (96, 1500.0, 6, 3),      # odd oversampling, supports 7-23
}
# name: (support, oversampling) of mode=normal kernels
TAPER_KERNELS = {"s7_o8": (7, 8), "s7_o3": (7, 3), "s9_o4": (9, 4)}
# polarisation type of each grid case's image (0 linear, 1 circular)
IMAGE_POL_TYPE = {"even_s4": 0, "odd_s3_p2": 1, "wide_s4": 0}


def partial_flags(flags, rng, frac=0.05):
    m = rng.random(flags.shape) < frac
    flags[m] = 1


def make_case(name, spec):
    obs, setup = synth.small_config(**spec["obs"])
    if spec.get("w_max_from_data"):
        setup.w_max = float(np.abs(obs.uvw[2] * obs.freq_over_c(0)).max())
    P = spec["npol"]
    rng = np.random.default_rng(100 + spec["obs"]["seed"])
    flags = np.ascontiguousarray(obs.flags[0][:, :P]).copy()
    if P == 2:
        # the reference's 2-pol ConvSum reads pol 0's flag for pol 1
        # (WProjPreProcessUVW.cu:94): keep both pols' flags equal
        m = rng.random(flags.shape[0]) < 0.05
        flags[m, :] = 1
    else:
        partial_flags(flags, rng)
    geo = O.geometry_for(setup)
    kern = O.wkernels(geo)
    return dict(uvw=np.ascontiguousarray(obs.uvw, np.float32),
                freq=np.ascontiguousarray(obs.freq_over_c(0), np.float32),
                vis=np.ascontiguousarray(obs.vis[0][:, :P], np.complex64),
                weights=np.ascontiguousarray(obs.weights[0][:, :P], np.float32),
                flags=np.ascontiguousarray(flags, np.int32),
                table=kern["table"].astype(np.complex64), conv_info=kern["conv_info"].astype(np.int32),
                conv_sums=kern["conv_sums"].astype(np.float32),
                nx=setup.nx, ny=setup.ny, npol=P, sampling=setup.sampling, wplanes=setup.wplanes,
                dl=setup.dl, trial_support=geo["trial_support"], support_cap=geo["support_cap"],
                w_max=geo["w_max"], w_inc=geo["w_inc"], du=geo["du"], dv=geo["dv"], chunks=spec["chunks"])


def run_reference(lib, c):
    R = c["freq"].size
    P = c["npol"]
    bounds = np.linspace(0, R, c["chunks"] + 1).astype(int)
    grid = np.zeros((c["ny"], c["nx"], P), np.complex64)
    out = {}
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    for k, (a, b) in enumerate(zip(bounds[:-1], bounds[1:])):
        n = int(b - a)
        uvw = np.ascontiguousarray(c["uvw"][:, a:b])
        sl = lambda x: np.ascontiguousarray(x[a:b])  # noqa: E731
        pre = dict(gridding_data=np.zeros((n, 4), np.int32), conv_index=np.zeros(n, np.int32),
                   to_grid=np.zeros(n, np.int32), to_compress=np.zeros(n, np.int32),
                   support=np.zeros(n, np.int32), take_conjugate=np.zeros(n, np.float32),
                   conv_sum=np.zeros((P, n), np.float32))
        err = ctypes.create_string_buffer(512)
        rc = lib.mtref_grid_chunk(c["nx"], c["ny"], P, c["sampling"], c["wplanes"], ctypes.c_float(c["du"]),
                                  ctypes.c_float(c["dv"]), ctypes.c_float(c["w_inc"]), p(c["table"]),
                                  c["table"].size, p(c["conv_info"]), p(c["conv_sums"]), p(uvw),
                                  p(sl(c["freq"])), p(sl(c["vis"])), p(sl(c["weights"])), p(sl(c["flags"])), n,
                                  int(k == 0), p(grid), p(pre["gridding_data"]), p(pre["conv_index"]),
                                  p(pre["to_grid"]), p(pre["to_compress"]), p(pre["support"]),
                                  p(pre["take_conjugate"]), p(pre["conv_sum"]), err, 512)
        if rc:
            raise RuntimeError("reference chunk %d failed: %s" % (k, err.value.decode()))
        for key, v in pre.items():
            out["ref_%s_%d" % (key, k)] = v
    out["ref_grid"] = grid
    return out


def run_wkernels(lib, nx, cell, nw, s):
    dl = cell * synth.ARCSEC
    cap = 4_000_000
    table = np.zeros(cap, np.complex64)
    info = np.zeros((nw, 2), np.int32)
    T = s if s % 2 else s + 1
    sums = np.zeros((nw, T * T), np.float32)
    n = ctypes.c_int(0)
    div = np.zeros(2, np.float32)
    err = ctypes.create_string_buffer(512)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    rc = lib.mtref_wkernels(nx, nx, ctypes.c_double(dl), ctypes.c_double(dl), nw, s, p(table), cap, p(info),
                            p(sums), ctypes.byref(n), p(div), err, 512)
    if rc:
        raise RuntimeError("reference w-kernels failed: " + err.value.decode())
    return dict(nx=nx, dl=dl, wplanes=nw, sampling=s, ref_table=table[: n.value].copy(), ref_conv_info=info,
                ref_conv_sums=sums, ref_divisor=div)


def run_finalize(lib, c, ref, pol_type):
    P = int(c["npol"])
    norm = np.zeros(P, np.float64)
    for k in range(int(c["chunks"])):
        norm += ref["ref_conv_sum_%d" % k].astype(np.float64).sum(axis=1)
    norm = norm.astype(np.float32)
    img = np.zeros((P, int(c["ny"]), int(c["nx"])), np.float32)
    err = ctypes.create_string_buffer(512)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    grid = np.ascontiguousarray(ref["ref_grid"])
    rc = lib.mtref_finalize(int(c["nx"]), int(c["ny"]), P, int(c["sampling"]), pol_type, p(grid), p(norm), p(img),
                            err, 512)
    if rc:
        raise RuntimeError("reference finalize failed: " + err.value.decode())
    return dict(pol_type=pol_type, normalizer=norm, ref_image=img)


def run_taper(lib, support, sampling):
    T = sampling if sampling % 2 else sampling + 1
    table = np.zeros(T * T * support * support, np.complex64)
    sums = np.zeros((1, T * T), np.float32)
    err = ctypes.create_string_buffer(512)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    rc = lib.mtref_taper_kernel(support, sampling, p(table), p(sums), err, 512)
    if rc:
        raise RuntimeError("reference taper kernel failed: " + err.value.decode())
    return dict(support=support, sampling=sampling, ref_table=table, ref_conv_sums=sums)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--lib", default=os.path.join(ROOT, "oracle", "_ref", "libmtref.so"))
    ap.add_argument("--only", default="", help="comma-separated fixture kinds to make (grid,wkernels,taper)")
    a = ap.parse_args()
    only = set(a.only.split(",")) if a.only else {"grid", "wkernels", "taper"}
    lib = ctypes.CDLL(a.lib)
    for f in (lib.mtref_grid_chunk, lib.mtref_wkernels, lib.mtref_finalize, lib.mtref_taper_kernel):
        f.restype = ctypes.c_int
    O.build()
    os.makedirs(a.out, exist_ok=True)
    for name, spec in (CASES.items() if "grid" in only else []):
        c = make_case(name, spec)
        ref = run_reference(lib, c)
        path = os.path.join(a.out, "grid_%s.npz" % name)
        np.savez_compressed(path, **c, **ref)
        print("%s: %d records, %d chunks, grid peak %.4g, %d bytes" % (
            name, c["freq"].size, c["chunks"], np.abs(ref["ref_grid"]).max(), os.path.getsize(path)))
        img = run_finalize(lib, c, ref, IMAGE_POL_TYPE[name])
        path = os.path.join(a.out, "image_%s.npz" % name)
        np.savez_compressed(path, **img)
        print("  image peak %.4g, %d bytes" % (np.abs(img["ref_image"]).max(), os.path.getsize(path)))
    for name, (sup, smp) in (TAPER_KERNELS.items() if "taper" in only else []):
        k = run_taper(lib, sup, smp)
        path = os.path.join(a.out, "taper_%s.npz" % name)
        np.savez_compressed(path, **k)
        print("%s: %d elements, %d bytes" % (name, k["ref_table"].size, os.path.getsize(path)))
    for name, g in (KERNEL_GEOMETRIES.items() if "wkernels" in only else []):
        k = run_wkernels(lib, *g)
        path = os.path.join(a.out, "wkernels_%s.npz" % name)
        np.savez_compressed(path, **k)
        print("%s: supports %s, %d elements, divisor %s, %d bytes" % (
            name, k["ref_conv_info"][:, 0].tolist(), k["ref_table"].size, k["ref_divisor"].tolist(),
            os.path.getsize(path)))


if __name__ == "__main__":
    main()
