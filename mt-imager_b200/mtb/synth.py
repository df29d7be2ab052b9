"""Seeded synthetic interferometer observations in mt-imager's record layout.

No MeasurementSet reader exists on this path (casacore is absent), so every
test, the smoke run and the benchmark feed the imager with observations made
here.  The layout is exactly what mt-imager's WImager module receives per
chunk and channel (``code/mt-imager/lib/components/WImager.cpp:157-161``,
``code/mt-imager/lib/components/VisibilityManager/VisibilityManager.cpp:168-225``):

* ``uvw``      float32 [3][R]  u, v, w rows in metres (row-planar)
* ``freq``     float32 [R]     nu/c per record (1/metres)
* ``vis``      complex64 [R][P] pol-interleaved (XX, XY, YX, YY)
* ``weights``  float32 [R][P]
* ``flags``    int32 [R][P]    1 = flagged

Records are ordered baseline-major with time order kept inside a baseline and
autocorrelations dropped, following the sort key
``nA*nA - a1*nA - a2 - 1`` ascending of
``code/mt-imager/lib/components/VisibilityManager/SortIndex.cpp:46-87``.

Sky model convention: V = sum_k S_k exp(-2 pi i (u l_k + v m_k + w (n_k - 1))),
which the reference's +phase w-screen and inverse FFT image back onto (l_k, m_k).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

C_LIGHT = 299792458.0
ARCSEC = math.pi / (180.0 * 3600.0)


@dataclasses.dataclass
class Observation:
    uvw: np.ndarray          # float32 [3][R] metres (shared by all channels)
    freqs_hz: np.ndarray     # float64 [nchan]
    vis: list                # per channel complex64 [R][P]
    weights: list            # per channel float32 [R][P]
    flags: list              # per channel int32 [R][P]
    nbaselines: int
    ntimes: int
    meta: dict

    @property
    def nrec(self) -> int:
        return self.uvw.shape[1]

    def freq_over_c(self, chan: int) -> np.ndarray:
        """nu/c per record for one channel (float32 [R]), the reference's
        'MyLSRKFrequencies' input (FrequencyConverter.cpp:133)."""
        return np.full(self.nrec, self.freqs_hz[chan] / C_LIGHT, dtype=np.float32)


@dataclasses.dataclass
class ImagingSetup:
    """Image and kernel parameters, the keys of mt-imager's property file
    (``code/mt-imager/conf/mtimager.properties:17-67``)."""
    nx: int
    ny: int
    cell_arcsec: float
    wplanes: int
    sampling: int
    trial_support: int = 0      # 0 -> reference rule min(nx,ny)/sampling forced odd
    max_support: int = 0        # 0 -> reference cap trial_support-2
    w_max: float = 0.0          # 0 -> reference rule 0.25/dl

    @property
    def dl(self) -> float:
        return self.cell_arcsec * ARCSEC


def antenna_layout(n_ant: int, radius_m: float, rng: np.random.Generator) -> np.ndarray:
    """ENU positions (metres) uniform inside a disk, up = 0."""
    r = radius_m * np.sqrt(rng.random(n_ant))
    th = 2 * np.pi * rng.random(n_ant)
    return np.stack([r * np.cos(th), r * np.sin(th), np.zeros(n_ant)], axis=1)


def baseline_order(n_ant: int):
    """Antenna pairs (a1 < a2) in the reference's sorted order."""
    pairs = [(a1, a2) for a1 in range(n_ant) for a2 in range(a1 + 1, n_ant)]
    pairs.sort(key=lambda p: n_ant * n_ant - p[0] * n_ant - p[1] - 1)
    return pairs


def track_uvw(enu: np.ndarray, lat_deg: float, dec_deg: float, ha_rad: np.ndarray) -> np.ndarray:
    """uvw (metres) for every baseline (reference order) x hour angle.
    Returns float64 [3][nbl*nt], baseline-major."""
    lat = math.radians(lat_deg)
    dec = math.radians(dec_deg)
    pairs = baseline_order(enu.shape[0])
    a1 = np.array([p[0] for p in pairs])
    a2 = np.array([p[1] for p in pairs])
    d = enu[a2] - enu[a1]                      # [nbl][3] east, north, up
    e, n, up = d[:, 0], d[:, 1], d[:, 2]
    lx = -n * math.sin(lat) + up * math.cos(lat)
    ly = e
    lz = n * math.cos(lat) + up * math.sin(lat)
    sh, ch = np.sin(ha_rad)[None, :], np.cos(ha_rad)[None, :]
    lx, ly, lz = lx[:, None], ly[:, None], lz[:, None]
    u = sh * lx + ch * ly
    v = -math.sin(dec) * ch * lx + math.sin(dec) * sh * ly + math.cos(dec) * lz
    w = math.cos(dec) * ch * lx - math.cos(dec) * sh * ly + math.sin(dec) * lz
    return np.stack([u.ravel(), v.ravel(), w.ravel()])


def random_sources(nsrc, fov_rad, rng, flux=(0.1, 1.0), powerlaw=None, pol_frac=0.1):
    """Point sources uniform in the field: rows (l, m, I, Q, U, V)."""
    half = 0.45 * fov_rad
    l = rng.uniform(-half, half, nsrc)
    m = rng.uniform(-half, half, nsrc)
    if powerlaw is None:
        i = rng.uniform(flux[0], flux[1], nsrc)
    else:
        # N(>S) ~ S^index between flux[0] and flux[1]
        a = powerlaw
        u = rng.random(nsrc)
        lo, hi = flux[0] ** a, flux[1] ** a
        i = (lo + u * (hi - lo)) ** (1.0 / a)
    q = pol_frac * i * rng.uniform(-1, 1, nsrc)
    uu = pol_frac * i * rng.uniform(-1, 1, nsrc)
    vv = 0.5 * pol_frac * i * rng.uniform(-1, 1, nsrc)
    return np.stack([l, m, i, q, uu, vv], axis=1)


def predict_vis(uvw_m: np.ndarray, freq_hz: float, sources: np.ndarray) -> np.ndarray:
    """Linear-feed visibilities complex64 [R][4] of point sources (float64 math)."""
    lam_inv = freq_hz / C_LIGHT
    u, v, w = (uvw_m * lam_inv)
    out = np.zeros((uvw_m.shape[1], 4), dtype=np.complex128)
    for l, m, si, sq, su, sv in sources:
        n = math.sqrt(1.0 - l * l - m * m)
        ph = np.exp(-2j * np.pi * (u * l + v * m + w * (n - 1.0)))
        out[:, 0] += (si + sq) * ph
        out[:, 1] += (su + 1j * sv) * ph
        out[:, 2] += (su - 1j * sv) * ph
        out[:, 3] += (si - sq) * ph
    return out


def make_observation(n_ant=27, radius_m=1000.0, freqs_hz=(1.4e9,), hours=1.0, dt_s=10.0,
                     lat_deg=-30.0, dec_deg=-45.0, nsrc=10, fov_rad=256 * 2 * ARCSEC,
                     noise=0.01, flag_frac=0.0, seed=0, powerlaw=None, flux=(0.1, 1.0),
                     ntimes=None, predict=True, pol_frac=0.1):
    """Earth-rotation-synthesis observation.  ``ntimes`` overrides hours/dt."""
    rng = np.random.default_rng(seed)
    enu = antenna_layout(n_ant, radius_m, rng)
    nt = int(round(hours * 3600.0 / dt_s)) if ntimes is None else int(ntimes)
    ha = (np.arange(nt) - (nt - 1) / 2.0) * dt_s * (2 * np.pi / 86164.0905)
    uvw = track_uvw(enu, lat_deg, dec_deg, ha)
    nbl = n_ant * (n_ant - 1) // 2
    srcs = random_sources(nsrc, fov_rad, rng, flux=flux, powerlaw=powerlaw, pol_frac=pol_frac)
    R = uvw.shape[1]
    vis, wts, flg = [], [], []
    for f in freqs_hz:
        if predict:
            v = predict_vis(uvw, f, srcs)
        else:
            v = np.zeros((R, 4), np.complex128)
        if noise > 0:
            v = v + noise * (rng.standard_normal((R, 4)) + 1j * rng.standard_normal((R, 4)))
        vis.append(v.astype(np.complex64))
        wts.append(np.ones((R, 4), np.float32))
        fl = np.zeros((R, 4), np.int32)
        if flag_frac > 0:
            fl[rng.random(R) < flag_frac, :] = 1
        flg.append(fl)
    meta = dict(n_ant=n_ant, radius_m=radius_m, lat_deg=lat_deg, dec_deg=dec_deg,
                hours=nt * dt_s / 3600.0, dt_s=dt_s, nsrc=nsrc, seed=seed, sources=srcs)
    return Observation(uvw=uvw.astype(np.float32), freqs_hz=np.asarray(freqs_hz, np.float64),
                       vis=vis, weights=wts, flags=flg, nbaselines=nbl, ntimes=nt, meta=meta)


# ---------------------------------------------------------------- presets --
def config1(seed=1, predict=True):
    """Plain small W-projection image: 27 antennas / 1 km, 1 channel at
    1.4 GHz, 1 h at 10 s (351 x 360 = 126,360 records), 10 point sources,
    noise 0.01 Jy, 256x256 at 2 arcsec, 32 w-planes, oversampling 8."""
    setup = ImagingSetup(nx=256, ny=256, cell_arcsec=2.0, wplanes=32, sampling=8)
    obs = make_observation(n_ant=27, radius_m=1000.0, freqs_hz=(1.4e9,), hours=1.0, dt_s=10.0,
                           nsrc=10, fov_rad=256 * 2 * ARCSEC, noise=0.01, seed=seed, predict=predict)
    return obs, setup


def small_config(seed=0, n_ant=8, ntimes=40, nx=64, cell_arcsec=20.0, wplanes=8, sampling=4,
                 radius_m=1000.0, freq=1.4e9, flag_frac=0.1, dec_deg=-60.0, nsrc=3,
                 max_support=0, trial_support=0):
    """A case the FP64 oracle and the direct DFT finish in well under a second."""
    setup = ImagingSetup(nx=nx, ny=nx, cell_arcsec=cell_arcsec, wplanes=wplanes, sampling=sampling,
                         max_support=max_support, trial_support=trial_support)
    obs = make_observation(n_ant=n_ant, radius_m=radius_m, freqs_hz=(freq,), ntimes=ntimes,
                           dt_s=60.0, nsrc=nsrc, fov_rad=nx * cell_arcsec * ARCSEC, noise=0.0,
                           flag_frac=flag_frac, seed=seed, dec_deg=dec_deg)
    return obs, setup


def config3(seed=3, full=True, torch=None):
    """Precision stress, wide field: 64 antennas within 10 km, 1 channel at
    725 MHz (|u| up to ~48 klambda fits the 8192^2 grid at 1.5 arcsec, and
    |w| reaches ~5e4 lambda), 12 h at 4 s (2016 x 10,800 = 21,772,800
    records), 20 point sources out to the field edge, 256 w-planes,
    oversampling 8, support <= 129 (trial support 131), w_max = max |w|.
    full=False keeps the field, the array extent and the kernels' support
    range with 12 antennas, 12 h at 120 s (66 x 360 = 23,760 records) and 64
    w-planes: a case the FP64 oracle finishes in about a minute.
    Visibilities are predicted on the device when `torch` is given."""
    freq = 725e6
    nx, cell = 8192, 1.5
    obs = make_observation(n_ant=64 if full else 12, radius_m=10000.0, freqs_hz=(freq,), hours=12.0,
                           dt_s=4.0 if full else 120.0, dec_deg=-45.0, nsrc=20, fov_rad=nx * cell * ARCSEC,
                           noise=0.0, seed=seed, predict=torch is None)
    if torch is not None:
        obs.vis[0] = predict_vis_torch(torch.from_numpy(obs.uvw).cuda(), freq, obs.meta["sources"],
                                       torch).cpu().numpy()
    w_max = float(np.abs(obs.uvw[2].astype(np.float64)).max() * freq / C_LIGHT)
    setup = ImagingSetup(nx=nx, ny=nx, cell_arcsec=cell, wplanes=256 if full else 64, sampling=8,
                         trial_support=131, max_support=129, w_max=w_max)
    return obs, setup


def predict_vis_torch(uvw_m, freq_hz: float, sources: np.ndarray, torch):
    """predict_vis on the device: uvw_m a float32 torch tensor [3][R] (metres),
    float64 phases, complex64 [R][4] out (linear feeds)."""
    lam_inv = freq_hz / C_LIGHT
    u, v, w = (uvw_m.double() * lam_inv)
    out = torch.zeros((uvw_m.shape[1], 4), dtype=torch.complex128, device=uvw_m.device)
    for l, m, si, sq, su, sv in sources:
        n = math.sqrt(1.0 - l * l - m * m)
        ph = torch.exp(-2j * math.pi * (u * l + v * m + w * (n - 1.0)))
        out[:, 0] += (si + sq) * ph
        out[:, 1] += complex(su, sv) * ph
        out[:, 2] += complex(su, -sv) * ph
        out[:, 3] += (si - sq) * ph
    return out.to(torch.complex64)


def config2_channel(seed=2, full=True, torch=None):
    """One channel (1.4 GHz) of the mid-size configuration: 64 antennas within
    4 km, 8 h at 2 s (2016 x 14,400 = 29,030,400 records), 200 power-law
    sources (index -1.5, 1 mJy-1 Jy), 25 % of records flagged, 4096^2 at the
    largest cell with max|u|/du + 65/2 < N/2 at 1.5 GHz, 128 w-planes,
    oversampling 8, supports 7-65 (trial support 67).  Visibilities are
    predicted on the device when `torch` is given.  full=False: 16 antennas,
    8 h at 60 s (120 x 480 = 57,600 records)."""
    rng = np.random.default_rng(seed)
    n_ant = 64 if full else 16
    enu = antenna_layout(n_ant, 4000.0, rng)
    dt = 2.0 if full else 60.0
    nt = int(round(8.0 * 3600.0 / dt))
    ha = (np.arange(nt) - (nt - 1) / 2.0) * dt * (2 * np.pi / 86164.0905)
    uvw = track_uvw(enu, -30.0, -45.0, ha).astype(np.float32)
    R = uvw.shape[1]
    n = 4096
    uv_max = float(np.abs(uvw[:2]).max()) * 1.5e9 / C_LIGHT
    du = uv_max / (n / 2 - (65 / 2 + 1))
    dl = 1.0 / (n * du)
    srcs = random_sources(200, n * dl, rng, flux=(1e-3, 1.0), powerlaw=-1.5)
    f = 1.4e9
    if torch is not None:
        vis = predict_vis_torch(torch.from_numpy(uvw).cuda(), f, srcs, torch).cpu().numpy()
    else:
        vis = predict_vis(uvw, f, srcs).astype(np.complex64)
    fl = np.zeros((R, 4), np.int32)
    fl[rng.random(R) < 0.25, :] = 1
    obs = Observation(uvw=uvw, freqs_hz=np.array([f]), vis=[vis], weights=[np.ones((R, 4), np.float32)],
                      flags=[fl], nbaselines=n_ant * (n_ant - 1) // 2, ntimes=nt,
                      meta=dict(n_ant=n_ant, sources=srcs))
    setup = ImagingSetup(nx=n, ny=n, cell_arcsec=dl / ARCSEC, wplanes=128, sampling=8, trial_support=67,
                         max_support=65)
    return obs, setup

