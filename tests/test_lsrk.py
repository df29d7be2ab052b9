"""TOPO -> LSRK frequencies per record (mtb_lsrk_freq_over_c), the part of
mt-imager's FrequencyConverter (FrequencyConverter.cpp:112-140).

The oracle (oracle/lsrk_oracle.py) is held to known answers on the CPU: the
J2000 direction of the standard solar motion (18h03m50.2s +30d00m16.8s),
the Earth's barycentric velocity at J2000.0 as the JPL DE405 ephemeris gives
it (-0.017202, -0.002904, -0.001259 au/day), the annual range of the Earth's
speed (29.29-30.29 km/s), the diurnal speed of a site on the equator
(465.1 m/s), and the Earth's velocity from the Astronomical Almanac's
low-precision Sun formula, a second published method.  casacore's own
conversion cannot run here, so parity with the reference is unpinned beyond
these answers.  The GPU tests compare the
device path with the oracle: nu/c in float32 equal to the oracle's or one
unit in the last place away (FP64 sin/cos of the two libraries differ in
their last bits, which moves a rounding only next to a tie)."""
import ctypes

import numpy as np
import pytest

from mtb import _lib as L
from oracle import lsrk_oracle as O

MEERKAT = (5109360.133, 2006852.586, -3238948.127)   # an ITRF site (m), latitude -30.7 deg
MJD_2024_03_20 = 60389.0 * 86400.0


def _ulps(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


# ------------------------------------------------------------- oracle, CPU
def test_apex_of_solar_motion_in_j2000():
    a = O.lsr_apex_j2000()
    ra = np.degrees(np.arctan2(a[1], a[0])) % 360.0
    dec = np.degrees(np.arcsin(a[2]))
    assert abs(ra - (18 + 3 / 60 + 50.2 / 3600) * 15) < 1.0 / 3600 * 15
    assert abs(dec - (30 + 16.8 / 3600)) < 1.0 / 3600


def test_earth_velocity_at_j2000_matches_de405():
    v = O.earth_velocity(O.J2000) / O.AU * O.DAY      # au/day
    assert np.allclose(v, [-0.017202, -0.002904, -0.001259], atol=1e-5)   # 17 m/s


def test_earth_velocity_agrees_with_the_almanac_sun():
    """A second, independent published formula: the Astronomical Almanac's
    low-precision geocentric Sun (mean longitude and anomaly, two-term
    equation of centre, of-date equator), differentiated and precessed to
    J2000, gives the Earth's velocity within 40 m/s and 0.08 deg of the
    oracle's over 30 years; it leaves out the Earth's monthly motion about the
    Earth-Moon barycentre and the Sun's motion about the barycentre (each up
    to ~13 m/s), which the oracle carries."""
    def sun(jd):
        n = jd - 2451545.0
        g = np.radians(357.528 + 0.9856003 * n)
        lam = np.radians(280.460 + 0.9856474 * n + 1.915 * np.sin(g) + 0.020 * np.sin(2 * g))
        r = 1.00014 - 0.01671 * np.cos(g) - 0.00014 * np.cos(2 * g)
        eps = np.radians(23.439 - 0.0000004 * n)
        return np.array([r * np.cos(lam), r * np.cos(eps) * np.sin(lam), r * np.sin(eps) * np.sin(lam)])
    for d in np.arange(0.0, 30 * 365.25, 41.7):
        jd = O.J2000 + d
        v1 = O.earth_velocity(jd)
        v2 = -(sun(jd + 0.01) - sun(jd - 0.01)) / 0.02 * O.AU / O.DAY
        v2 = O.precession_matrix(O.J2000, jd).T @ v2
        assert abs(np.linalg.norm(v1) - np.linalg.norm(v2)) < 40.0
        cosang = v1 @ v2 / (np.linalg.norm(v1) * np.linalg.norm(v2))
        assert np.degrees(np.arccos(min(1.0, cosang))) < 0.08


def test_earth_speed_annual_range():
    s = np.array([np.linalg.norm(O.earth_velocity(O.J2000 + 9000 + d)) for d in range(0, 366, 3)]) / 1e3
    assert 29.2 < s.min() < 29.35 and 30.25 < s.max() < 30.35


def test_diurnal_speed():
    assert abs(np.linalg.norm(O.diurnal_velocity(O.J2000, O.J2000, [6378137.0, 0, 0])) - 465.10) < 0.02
    assert np.linalg.norm(O.diurnal_velocity(O.J2000, O.J2000, [0, 0, 6356752.0])) < 1e-9


def test_factor_is_a_doppler_shift_of_the_observer_velocity():
    t = MJD_2024_03_20 + 3600.0
    v = O.observer_velocity(t, MEERKAT)
    n = v / np.linalg.norm(v)
    ra, dec = np.arctan2(n[1], n[0]), np.arcsin(n[2])
    beta = np.linalg.norm(v) / O.C
    # moving straight at the source: nu_LSRK = nu_TOPO * sqrt((1 - b) / (1 + b))
    assert np.isclose(O.doppler_factor(t, MEERKAT, ra, dec), np.sqrt((1 - beta) / (1 + beta)), rtol=1e-14)
    assert np.isclose(O.doppler_factor(t, MEERKAT, ra + np.pi, -dec), np.sqrt((1 + beta) / (1 - beta)), rtol=1e-14)


def test_time_scale_offsets():
    """tt_minus_time and ut1_minus_time only move the epoch: shifting the
    record time and both offsets against each other changes nothing; one
    second of UT1 turns the site by 7.3e-5 rad, a few cm/s of its velocity."""
    t = MJD_2024_03_20 + 1234.5
    a = O.doppler_factor(t, MEERKAT, 1.0, 0.2, tt_minus_time=69.184, ut1_minus_time=0.3)
    b = O.doppler_factor(t + 10.0, MEERKAT, 1.0, 0.2, tt_minus_time=59.184, ut1_minus_time=-9.7)
    assert abs(a - b) < 1e-15
    c = O.doppler_factor(t, MEERKAT, 1.0, 0.2, tt_minus_time=69.184, ut1_minus_time=1.3)
    assert 1e-13 < abs(c - a) < 1e-9


def test_oracle_evaluates_once_per_run_of_equal_times():
    t = np.repeat(MJD_2024_03_20 + 10.0 * np.arange(4), 3)
    out = O.lsrk_freq_over_c(t, [1.4e9], MEERKAT, 1.0, -0.5)
    assert out.shape == (1, 12) and out.dtype == np.float32
    assert np.all(out[0].reshape(4, 3) == out[0].reshape(4, 3)[:, :1])
    perm = np.array([11, 0, 5])
    assert np.array_equal(O.lsrk_freq_over_c(t, [1.4e9], MEERKAT, 1.0, -0.5, index=perm)[0], out[0, perm])


# ------------------------------------------------------- C ABI, no GPU work
def test_refusals_before_any_launch():
    lib = L.load()
    p = L.LsrkParams()
    p.site_itrf[0], p.site_itrf[1], p.site_itrf[2] = MEERKAT
    n = ctypes.c_size_t(0)
    assert lib.mtb_lsrk_workspace_size(-1, ctypes.byref(n)) == L.MTB_ERR_BAD_PARAM
    assert lib.mtb_lsrk_workspace_size(10, None) == L.MTB_ERR_NULL
    f = lib.mtb_lsrk_freq_over_c
    z = ctypes.c_void_p(0)
    assert f(None, z, 1, z, 1, z, 1, z, z, 0, z) == L.MTB_ERR_NULL
    assert f(ctypes.byref(p), z, -1, z, 1, z, 1, z, z, 0, z) == L.MTB_ERR_BAD_PARAM
    assert f(ctypes.byref(p), z, 4, z, 1, z, 3, z, z, 0, z) == L.MTB_ERR_BAD_PARAM   # no index: n == nrows
    assert f(ctypes.byref(p), z, 0, z, 1, ctypes.c_void_p(8), 3, z, z, 0, z) == L.MTB_ERR_BAD_PARAM
    assert f(ctypes.byref(p), z, 4, z, 0, z, 4, z, z, 0, z) == L.MTB_OK              # nothing to write
    assert f(ctypes.byref(p), z, 4, z, 2, z, 0, z, z, 0, z) == L.MTB_OK              # no records
    p.dec = float("nan")
    assert f(ctypes.byref(p), z, 4, z, 1, z, 4, z, z, 0, z) == L.MTB_ERR_BAD_PARAM
    p.dec = 0.0
    assert f(ctypes.byref(p), z, 4, z, 1, z, 4, z, z, 0, z) == L.MTB_ERR_NULL        # device pointers missing


def test_record_file_carries_the_conversion_columns(tmp_path):
    from mtb import ingest, synth
    obs, _ = synth.small_config(seed=3, n_ant=5, ntimes=6, nx=64)
    times = MJD_2024_03_20 + 8.0 * np.arange(obs.ntimes)
    path = str(tmp_path / "rec.npz")
    ingest.write_record_file(path, obs, time_s=times, site_itrf=MEERKAT, phase_dir=(1.2, -0.6))
    rf = ingest.RecordFile(path)
    assert rf.time.shape == rf.antenna1.shape and np.allclose(rf.site_itrf, MEERKAT)
    # records are baseline-major: each baseline walks the time samples in order
    assert np.array_equal(rf.time[rf.index].reshape(-1, obs.ntimes)[0], times)
    with pytest.raises(ValueError):
        rf.lsrk_freq_over_c(device="cpu")          # the library runs on a CUDA device only


# ---------------------------------------------------------------- GPU parity
def _gpu(time_s, chan, ra, dec, index=None, **kw):
    from mtb.lsrk import lsrk_freq_over_c
    return lsrk_freq_over_c(time_s, chan, MEERKAT, ra, dec, index=index, **kw).cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1])
def test_gpu_matches_oracle_time_major_rows(seed):
    rng = np.random.default_rng(seed)
    nt, nbl = 90, 37
    times = MJD_2024_03_20 + rng.uniform(-4e8, 4e8) + 4.0 * np.arange(nt)
    t = np.repeat(times, nbl)                              # MeasurementSet order: rows of one time together
    chan = 1.3e9 + 0.2e9 * rng.random(5)
    ra, dec = rng.uniform(0, 2 * np.pi), rng.uniform(-1.4, 1.4)
    index = rng.permutation(t.size)[: t.size - 11].astype(np.int32)
    got = _gpu(t, chan, ra, dec, index=index)
    ref = O.lsrk_freq_over_c(t, chan, MEERKAT, ra, dec, index=index)
    u = _ulps(got, ref)
    assert u.max() <= 1 and (u == 0).mean() > 0.99, (u.max(), (u == 0).mean())
    # the conversion moved the frequencies by the observer's velocity (< 60 km/s)
    topo = (chan[:, None] / O.C).astype(np.float32)
    assert np.all(np.abs(got / topo - 1.0) < 2e-4) and np.any(got != topo)


@pytest.mark.gpu
def test_gpu_every_row_its_own_time_over_decades():
    rng = np.random.default_rng(7)
    t = np.sort((51544.5 + rng.uniform(0, 40 * 365.25, 700)) * 86400.0)[rng.permutation(700)]
    chan = np.array([0.35e9, 1.42e9, 8.4e9])
    got = _gpu(t, chan, 4.0, 0.3, tt_minus_time=32.184 + 37, ut1_minus_time=-0.2)
    ref = O.lsrk_freq_over_c(t, chan, MEERKAT, 4.0, 0.3, tt_minus_time=32.184 + 37, ut1_minus_time=-0.2)
    assert _ulps(got, ref).max() <= 1


@pytest.mark.gpu
def test_gpu_ragged_and_out_of_range_rows():
    t = np.array([MJD_2024_03_20])
    one = _gpu(t, [1.4e9], 0.5, 0.1)
    assert one.shape == (1, 1) and _ulps(one, O.lsrk_freq_over_c(t, [1.4e9], MEERKAT, 0.5, 0.1)).max() <= 1
    bad = _gpu(np.repeat(t, 4), [1.4e9, 1.5e9], 0.5, 0.1, index=np.array([2, -1, 4, 0], np.int32))
    assert np.isnan(bad[:, 1]).all() and np.isnan(bad[:, 2]).all()
    assert np.array_equal(bad[:, 0], bad[:, 3]) and np.isfinite(bad[:, 0]).all()
    assert _gpu(t, [1.4e9], 0.5, 0.1, index=np.zeros(0, np.int32)).shape == (1, 0)


@pytest.mark.gpu
def test_gpu_full_track_size_against_the_oracle_per_time():
    """A full 8 h track at 2 s in MeasurementSet order (14,400 times x 2016
    baselines = 29,030,400 rows), 16 channels: every record carries its
    time's factor, checked against the oracle at every distinct time."""
    import torch
    nt, nbl = 14400, 2016
    times = MJD_2024_03_20 + 2.0 * np.arange(nt)
    t = torch.from_numpy(times).cuda().repeat_interleave(nbl)
    chan = np.linspace(1.3e9, 1.5e9, 16)
    from mtb.lsrk import lsrk_freq_over_c
    out = lsrk_freq_over_c(t, chan, MEERKAT, 2.1, -0.7)
    assert out.shape == (16, nt * nbl)
    per_time = out.view(16, nt, nbl)
    assert bool((per_time == per_time[:, :, :1]).all())
    pick = np.linspace(0, nt - 1, 60).astype(int)
    ref = O.lsrk_freq_over_c(times[pick], chan, MEERKAT, 2.1, -0.7)
    assert _ulps(per_time[:, pick, 0].cpu().numpy(), ref).max() <= 1
    del out, per_time, t
    torch.cuda.empty_cache()


@pytest.mark.gpu
def test_record_file_lsrk_frequencies_follow_the_record_order(tmp_path):
    from mtb import ingest, synth
    obs, _ = synth.small_config(seed=4, n_ant=6, ntimes=9, nx=64)
    times = MJD_2024_03_20 + 30.0 * np.arange(obs.ntimes)
    path = str(tmp_path / "rec.npz")
    ingest.write_record_file(path, obs, time_s=times, site_itrf=MEERKAT, phase_dir=(0.3, 0.9))
    rf = ingest.RecordFile(path)
    got = rf.lsrk_freq_over_c().cpu().numpy()
    ref = O.lsrk_freq_over_c(rf.time, rf.chan_freq, MEERKAT, 0.3, 0.9, index=rf.index)
    assert got.shape == (rf.nchan, rf.nrec) and _ulps(got, ref).max() <= 1


@pytest.mark.gpu
def test_cpp_frequency_converter(tmp_path):
    """tests/cpp/lsrk_one.cpp converts through mtb::FrequencyConverter
    (include/mtb.hpp); its nu/c equals the oracle's to 1 ulp."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cxx = os.environ.get("CXX", "g++")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    lib = os.path.join(root, "mt-imager_b200")
    exe = tmp_path / "lsrk_one"
    subprocess.run([cxx, "-std=c++17", "-O2", os.path.join(root, "tests", "cpp", "lsrk_one.cpp"), "-o", str(exe),
                    "-I", os.path.join(root, "include"), "-I", os.path.join(cuda, "include"), "-L", lib, "-lmtb",
                    "-L", os.path.join(cuda, "lib64"), "-lcudart", "-Wl,-rpath," + lib,
                    "-Wl,-rpath," + os.path.join(cuda, "lib64")], check=True)
    rng = np.random.default_rng(12)
    t = np.repeat(MJD_2024_03_20 + 6.0 * np.arange(40), 9)
    chan = np.array([1.31e9, 1.42e9, 1.49e9])
    index = rng.permutation(t.size).astype(np.int32)
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        np.array([t.size, chan.size, index.size, 1], np.int32).tofile(f)
        np.array(list(MEERKAT) + [0.7, -0.9, 69.184, 0.1], np.float64).tofile(f)
        t.astype(np.float64).tofile(f)
        chan.tofile(f)
        index.tofile(f)
    out = tmp_path / "out.bin"
    subprocess.run([str(exe), str(inp), str(out)], check=True)
    got = np.fromfile(out, np.float32).reshape(chan.size, index.size)
    ref = O.lsrk_freq_over_c(t, chan, MEERKAT, 0.7, -0.9, 69.184, 0.1, index=index)
    assert _ulps(got, ref).max() <= 1
