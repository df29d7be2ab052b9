"""TEST INFRASTRUCTURE, NOT PRODUCT CODE.

FP64 numpy restatement of the TOPO -> LSRK frequency conversion of
mt-imager's FrequencyConverter (code/mt-imager/lib/components/
VisibilityManager/FrequencyConverter.cpp:112-140): for every record whose
time differs from the previous record's, the channel frequencies are
converted from the topocentric frame to the kinematic local standard of rest
and stored as (float)(nu_LSRK / c) (c = 299792458, FrequencyConverter.cpp:116).
Only tests/ import this module.

The reference asks casacore's MFrequency::Convert for the conversion, and
casacore is not available here, so this restatement and the device code
follow the same published formulas (each named where it is used) and the
oracle's own method is held to known answers in tests/test_lsrk.py: the
standard solar-motion apex in J2000, the Earth's barycentric velocity at
J2000.0, the diurnal speed of a site on the equator, and the annual range of
the Earth's speed.  Parity with casacore itself is unpinned: the expected
agreement is the accuracy of the mean elements (a few m/s, ~1e-8 of the
frequency; float32 nu/c resolves 6e-8).

Rotations are composed here from elementary rotation matrices, and the
Keplerian state is solved in numpy, so that the device code's expanded
matrices are checked against a second writing of them.
"""
from __future__ import annotations

import numpy as np

C = 299792458.0
AU = 149597870700.0
DAY = 86400.0
J2000 = 2451545.0
B1900 = 2415020.3135
ARCSEC = np.pi / 180.0 / 3600.0
DEG = np.pi / 180.0
OBLIQUITY = 84381.448 * ARCSEC           # IAU 1976 obliquity of J2000
HALF_STEP_DAYS = 0.01                    # central-difference half step
LSR_SPEED = 20000.0                      # m/s towards 18h +30 deg (B1900)
MOON_FRACTION = 0.0123000371 / 1.0123000371

# JPL approximate-position Keplerian elements (Standish), table 1 (1800-2050),
# J2000 ecliptic: a, e, I, L, long. perihelion, long. node and rates per century
ELEMENTS = {
    "emb": ((1.00000261, 0.01671123, -0.00001531, 100.46457166, 102.93768193, 0.0),
            (0.00000562, -0.00004392, -0.01294668, 35999.37244981, 0.32327364, 0.0)),
    "jupiter": ((5.20288700, 0.04838624, 1.30439695, 34.39644051, 14.72847983, 100.47390909),
                (-0.00011607, -0.00013253, -0.00183714, 3034.74612775, 0.21252668, 0.20469106)),
    "saturn": ((9.53667594, 0.05386179, 2.48599187, 49.95424423, 92.59887831, 113.66242448),
               (-0.00125060, -0.00050991, 0.00193609, 1222.49362201, -0.41897216, -0.28867794)),
    "uranus": ((19.18916464, 0.04725744, 0.77263783, 313.23810451, 170.95427630, 74.01692503),
               (-0.00196176, -0.00004397, -0.00242939, 428.48202785, 0.40805281, 0.04240589)),
    "neptune": ((30.06992276, 0.00859048, 1.77004347, -55.12002969, 44.96476227, 131.78422574),
                (0.00026291, 0.00005105, 0.00035372, 218.45945325, -0.32241464, -0.00508664)),
}
SUN_OVER_MASS = {"emb": 328900.56, "jupiter": 1047.3486, "saturn": 3497.898, "uranus": 22902.98,
                 "neptune": 19412.24}


def rot1(a):
    """Frame rotation about x by angle a (vector components in the new frame)."""
    c, s = np.cos(a), np.sin(a)
    return np.array([[1, 0, 0], [0, c, s], [0, -s, c]])


def rot2(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, 0, -s], [0, 1, 0], [s, 0, c]])


def rot3(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, s, 0], [-s, c, 0], [0, 0, 1]])


ECL_TO_EQ = rot1(-OBLIQUITY)


def precession_matrix(jd0, jd1):
    """IAU 1976 precession (Lieske et al. 1977) from the mean equator and
    equinox of jd0 to those of jd1: R3(-z) R2(theta) R3(-zeta)."""
    T = (jd0 - J2000) / 36525.0
    t = (jd1 - jd0) / 36525.0
    c1 = 2306.2181 + 1.39656 * T - 0.000139 * T * T
    zeta = (c1 * t + (0.30188 - 0.000344 * T) * t * t + 0.017998 * t ** 3) * ARCSEC
    z = (c1 * t + (1.09468 + 0.000066 * T) * t * t + 0.018203 * t ** 3) * ARCSEC
    theta = ((2004.3109 - 0.85330 * T - 0.000217 * T * T) * t - (0.42665 + 0.000217 * T) * t * t
             - 0.041833 * t ** 3) * ARCSEC
    return rot3(-z) @ rot2(theta) @ rot3(-zeta)


def kepler_position(name, T):
    """Heliocentric J2000 equatorial position (au) from the mean elements."""
    v, r = ELEMENTS[name]
    a, e, inc, L, wbar, node = (v[k] + r[k] * T for k in range(6))
    M = np.mod(L - wbar, 360.0)
    M = np.where(M > 180.0, M - 360.0, M) * DEG
    E = M + e * np.sin(M)
    for _ in range(8):
        E = E - (E - e * np.sin(E) - M) / (1.0 - e * np.cos(E))
    xp = a * (np.cos(E) - e)
    yp = a * np.sqrt(1.0 - e * e) * np.sin(E)
    orb = np.array([xp, yp, 0.0])
    # orbit plane -> ecliptic: R3(-node) R1(-I) R3(-omega)
    ecl = rot3(-node * DEG) @ rot1(-inc * DEG) @ rot3(-(wbar - node) * DEG) @ orb
    return ECL_TO_EQ @ ecl


def moon_position(T):
    """Geocentric J2000 equatorial position of the Moon (au): leading terms of
    Meeus, Astronomical Algorithms ch. 47, ecliptic of date brought to J2000
    by the general precession in longitude."""
    Lp = 218.3164477 + 481267.88123421 * T - 0.0015786 * T * T
    D = (297.8501921 + 445267.1114034 * T - 0.0018819 * T * T) * DEG
    Ms = (357.5291092 + 35999.0502909 * T - 0.0001536 * T * T) * DEG
    Mm = (134.9633964 + 477198.8675055 * T + 0.0087414 * T * T) * DEG
    F = (93.2720950 + 483202.0175233 * T - 0.0036539 * T * T) * DEG
    lon_terms = [(6.288774, Mm), (1.274027, 2 * D - Mm), (0.658314, 2 * D), (0.213618, 2 * Mm),
                 (-0.185116, Ms), (-0.114332, 2 * F), (0.058793, 2 * D - 2 * Mm), (0.057066, 2 * D - Ms - Mm),
                 (0.053322, 2 * D + Mm), (0.045758, 2 * D - Ms)]
    lat_terms = [(5.128122, F), (0.280602, Mm + F), (0.277693, Mm - F), (0.173237, 2 * D - F),
                 (0.055413, 2 * D - Mm + F), (0.046271, 2 * D - Mm - F)]
    dist_terms = [(-20905.355, Mm), (-3699.111, 2 * D - Mm), (-2955.968, 2 * D), (-569.925, 2 * Mm),
                  (48.888, Ms), (246.158, 2 * D - 2 * Mm), (-152.138, 2 * D - Ms - Mm), (-170.733, 2 * D + Mm),
                  (-204.586, 2 * D - Ms)]
    lon = Lp + sum(c * np.sin(x) for c, x in lon_terms)
    lat = sum(c * np.sin(x) for c, x in lat_terms)
    dist = 385000.56 + sum(c * np.cos(x) for c, x in dist_terms)
    lam = (lon - (5029.0966 * T + 1.11113 * T * T) / 3600.0) * DEG
    bet = lat * DEG
    r = dist * 1000.0 / AU
    return ECL_TO_EQ @ np.array([r * np.cos(bet) * np.cos(lam), r * np.cos(bet) * np.sin(lam), r * np.sin(bet)])


def earth_position(T):
    """Barycentric J2000 equatorial position of the Earth (au)."""
    helio = {k: kepler_position(k, T) for k in ELEMENTS}
    masses = {k: 1.0 / SUN_OVER_MASS[k] for k in ELEMENTS}
    sun = -sum(masses[k] * helio[k] for k in ELEMENTS) / (1.0 + sum(masses.values()))
    return helio["emb"] + sun - MOON_FRACTION * moon_position(T)


def earth_velocity(jd_tt):
    """Barycentric J2000 equatorial velocity of the Earth, m/s."""
    T = (jd_tt - J2000) / 36525.0
    h = HALF_STEP_DAYS / 36525.0
    return (earth_position(T + h) - earth_position(T - h)) * AU / (2.0 * HALF_STEP_DAYS * DAY)


def lsr_apex_j2000():
    """Unit vector of the solar motion (18h, +30 deg, B1900) in J2000."""
    a0, d0 = 270.0 * DEG, 30.0 * DEG
    return precession_matrix(B1900, J2000) @ np.array([np.cos(d0) * np.cos(a0), np.cos(d0) * np.sin(a0), np.sin(d0)])


def diurnal_velocity(jd_ut1, jd_tt, site_itrf):
    """Velocity of the site from the Earth's rotation, J2000 equatorial, m/s:
    GMST of IAU 1982 (Meeus eq. 12.4) about the mean pole of date."""
    du = jd_ut1 - J2000
    Tu = du / 36525.0
    gmst = np.mod(280.46061837 + 360.98564736629 * du + 0.000387933 * Tu * Tu - Tu ** 3 / 38710000.0, 360.0) * DEG
    omega = 360.98564736629 * DEG / DAY
    r = rot3(-gmst) @ np.asarray(site_itrf, float)
    v_date = np.cross(np.array([0.0, 0.0, omega]), r)
    return precession_matrix(J2000, jd_tt).T @ v_date


def observer_velocity(time_s, site_itrf, tt_minus_time=69.184, ut1_minus_time=0.0):
    """Velocity of the observer with respect to the kinematic LSR (m/s, J2000)."""
    jd_tt = 2400000.5 + (time_s + tt_minus_time) / DAY
    jd_ut1 = 2400000.5 + (time_s + ut1_minus_time) / DAY
    return earth_velocity(jd_tt) + diurnal_velocity(jd_ut1, jd_tt, site_itrf) + LSR_SPEED * lsr_apex_j2000()


def doppler_factor(time_s, site_itrf, ra, dec, tt_minus_time=69.184, ut1_minus_time=0.0):
    """nu_LSRK / nu_TOPO: one boost with the observer's velocity."""
    v = observer_velocity(time_s, site_itrf, tt_minus_time, ut1_minus_time)
    n = np.array([np.cos(dec) * np.cos(ra), np.cos(dec) * np.sin(ra), np.sin(dec)])
    bn = v @ n / C
    b2 = v @ v / (C * C)
    return np.sqrt(1.0 - b2) / (1.0 + bn)


def lsrk_freq_over_c(time_s, chan_hz, site_itrf, ra, dec, tt_minus_time=69.184, ut1_minus_time=0.0, index=None):
    """float32 [nchan][n]: nu_LSRK / c per channel and record, the factor
    evaluated once per run of equal consecutive times
    (FrequencyConverter.cpp:117-137), then records taken in `index` order."""
    time_s = np.asarray(time_s, np.float64)
    chan_hz = np.asarray(chan_hz, np.float64)
    f = np.empty(time_s.size)
    last_t, last_f = None, None
    for r, t in enumerate(time_s):
        if last_t is None or not (t == last_t):
            last_t, last_f = t, doppler_factor(t, site_itrf, ra, dec, tt_minus_time, ut1_minus_time)
        f[r] = last_f
    rows = np.arange(time_s.size) if index is None else np.asarray(index)
    out = np.empty((chan_hz.size, rows.size), np.float32)
    for c in range(chan_hz.size):
        out[c] = (chan_hz[c] * f[rows] / C).astype(np.float32)
    return out
