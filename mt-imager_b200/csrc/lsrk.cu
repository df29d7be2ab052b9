// TOPO -> LSRK channel frequencies per record, as nu/c (include/mtb.h,
// mtb_lsrk_freq_over_c).  Replaces mt-imager's FrequencyConverter
// (code/mt-imager/lib/components/VisibilityManager/FrequencyConverter.cpp:112-140),
// which asks casacore's MFrequency::Convert(TOPO -> LSRK) for every distinct
// record time and stores (float)(nu_LSRK / c) per record and channel.
//
// casacore and its measures data are not available, so the observer's
// velocity with respect to the kinematic local standard of rest is built
// here, in FP64, from published formulas:
//   - Earth rotation: GMST of IAU 1982 (Meeus, Astronomical Algorithms,
//     eq. 12.4) turns the ITRF site position into the mean equator and
//     equinox of date; velocity = Omega x r.  Polar motion and nutation are
//     left out (< 0.1 m/s).
//   - Precession J2000 <-> date and B1900 -> J2000: IAU 1976 angles
//     zeta, z, theta (Lieske et al. 1977) with their epoch-dependent terms.
//   - The Earth-Moon barycentre and the giant planets: the JPL Keplerian
//     elements and rates for 1800-2050 (Standish, "Keplerian Elements for
//     Approximate Positions of the Major Planets", table 1), J2000 ecliptic,
//     obliquity 84381.448".  The Sun's motion about the barycentre is
//     -sum(m_p v_p) / M over Jupiter, Saturn, Uranus, Neptune and the EMB.
//   - The Earth about the EMB: the Moon's geocentric position from the
//     leading terms of Meeus ch. 47 (ELP-2000/82), scaled by m_Moon / (m_E + m_M).
//   - The Sun with respect to the LSRK: 20 km/s towards RA 18h, Dec +30 deg
//     (B1900), the kinematic LSR definition.
// Velocities are central differences of positions 0.01 day apart.  The
// frequency is Doppler-shifted by one boost with the summed velocity:
// nu_LSRK = nu_TOPO * sqrt(1 - beta^2) / (1 + beta . n), n the J2000 unit
// vector of the phase centre.  Time arguments: TT (= TDB within 2 ms) for
// the ephemerides, UT1 for the Earth's rotation.
//
// On the device: a record whose time differs from the previous record's (a
// "head", the reference's `time_storage[recordNo] != last_time` test)
// evaluates the velocity once; an inclusive max-scan hands every record its
// head; a last kernel writes nu/c per channel in the caller's record order.
#include <algorithm>
#include <cmath>

#include <cub/cub.cuh>

#include "mtb_internal.cuh"

namespace mtb {
namespace lsrk {

constexpr double kPi = 3.14159265358979323846;
constexpr double kDeg = kPi / 180.0;
constexpr double kArcsec = kDeg / 3600.0;
constexpr double kC = 299792458.0;             // m/s, the reference's c
constexpr double kAU = 149597870700.0;         // m
constexpr double kDay = 86400.0;               // s
constexpr double kJ2000 = 2451545.0;           // JD of J2000.0
constexpr double kB1900 = 2415020.3135;        // JD of B1900.0
constexpr double kObliquity = 84381.448 * kArcsec;
constexpr double kHalfStepDays = 0.01;         // central-difference half step
constexpr double kLsrSpeed = 20000.0;          // m/s
constexpr double kMoonFraction = 0.0123000371 / 1.0123000371;   // m_Moon / (m_Earth + m_Moon)

// Standish table 1: a (au), e, I, L, long. perihelion, long. node (deg) and
// their rates per Julian century.
struct Elements {
    double v[6], r[6];
};
__constant__ Elements kBodies[5] = {
    // Earth-Moon barycentre
    {{1.00000261, 0.01671123, -0.00001531, 100.46457166, 102.93768193, 0.0},
     {0.00000562, -0.00004392, -0.01294668, 35999.37244981, 0.32327364, 0.0}},
    // Jupiter
    {{5.20288700, 0.04838624, 1.30439695, 34.39644051, 14.72847983, 100.47390909},
     {-0.00011607, -0.00013253, -0.00183714, 3034.74612775, 0.21252668, 0.20469106}},
    // Saturn
    {{9.53667594, 0.05386179, 2.48599187, 49.95424423, 92.59887831, 113.66242448},
     {-0.00125060, -0.00050991, 0.00193609, 1222.49362201, -0.41897216, -0.28867794}},
    // Uranus
    {{19.18916464, 0.04725744, 0.77263783, 313.23810451, 170.95427630, 74.01692503},
     {-0.00196176, -0.00004397, -0.00242939, 428.48202785, 0.40805281, 0.04240589}},
    // Neptune
    {{30.06992276, 0.00859048, 1.77004347, -55.12002969, 44.96476227, 131.78422574},
     {0.00026291, 0.00005105, 0.00035372, 218.45945325, -0.32241464, -0.00508664}},
};
// Sun / body mass ratios (IAU): EMB, Jupiter, Saturn, Uranus, Neptune
__constant__ double kSunOverMass[5] = {328900.56, 1047.3486, 3497.898, 22902.98, 19412.24};

struct V3 {
    double x, y, z;
};
__device__ __forceinline__ V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// J2000 ecliptic -> J2000 equator
__device__ __forceinline__ V3 ecl_to_eq(V3 e) {
    const double ce = cos(kObliquity), se = sin(kObliquity);
    return {e.x, ce * e.y - se * e.z, se * e.y + ce * e.z};
}

// Heliocentric J2000 equatorial position (au) of body b, T centuries TT from J2000.
__device__ V3 kepler_position(int b, double T) {
    const Elements &el = kBodies[b];
    const double a = el.v[0] + el.r[0] * T, e = el.v[1] + el.r[1] * T;
    const double I = (el.v[2] + el.r[2] * T) * kDeg, L = el.v[3] + el.r[3] * T;
    const double wbar = el.v[4] + el.r[4] * T, node = el.v[5] + el.r[5] * T;
    const double w = (wbar - node) * kDeg, O = node * kDeg;
    double M = fmod(L - wbar, 360.0);
    M = (M > 180.0 ? M - 360.0 : (M < -180.0 ? M + 360.0 : M)) * kDeg;
    double E = M + e * sin(M);
#pragma unroll 1
    for (int it = 0; it < 8; it++) E -= (E - e * sin(E) - M) / (1.0 - e * cos(E));
    const double xp = a * (cos(E) - e), yp = a * sqrt(1.0 - e * e) * sin(E);
    const double cw = cos(w), sw = sin(w), cO = cos(O), sO = sin(O), cI = cos(I), sI = sin(I);
    const V3 ecl = {(cw * cO - sw * sO * cI) * xp + (-sw * cO - cw * sO * cI) * yp,
                    (cw * sO + sw * cO * cI) * xp + (-sw * sO + cw * cO * cI) * yp, sw * sI * xp + cw * sI * yp};
    return ecl_to_eq(ecl);
}

// Geocentric J2000 equatorial position of the Moon (au), leading terms of
// Meeus ch. 47; the ecliptic of date is brought to J2000 by the general
// precession in longitude.
__device__ V3 moon_position(double T) {
    const double Lp = 218.3164477 + 481267.88123421 * T - 0.0015786 * T * T;
    const double D = (297.8501921 + 445267.1114034 * T - 0.0018819 * T * T) * kDeg;
    const double Ms = (357.5291092 + 35999.0502909 * T - 0.0001536 * T * T) * kDeg;
    const double Mm = (134.9633964 + 477198.8675055 * T + 0.0087414 * T * T) * kDeg;
    const double F = (93.2720950 + 483202.0175233 * T - 0.0036539 * T * T) * kDeg;
    const double lon = Lp + 6.288774 * sin(Mm) + 1.274027 * sin(2 * D - Mm) + 0.658314 * sin(2 * D) +
                       0.213618 * sin(2 * Mm) - 0.185116 * sin(Ms) - 0.114332 * sin(2 * F) +
                       0.058793 * sin(2 * D - 2 * Mm) + 0.057066 * sin(2 * D - Ms - Mm) + 0.053322 * sin(2 * D + Mm) +
                       0.045758 * sin(2 * D - Ms);
    const double lat = 5.128122 * sin(F) + 0.280602 * sin(Mm + F) + 0.277693 * sin(Mm - F) +
                       0.173237 * sin(2 * D - F) + 0.055413 * sin(2 * D - Mm + F) + 0.046271 * sin(2 * D - Mm - F);
    const double dist_km = 385000.56 - 20905.355 * cos(Mm) - 3699.111 * cos(2 * D - Mm) - 2955.968 * cos(2 * D) -
                           569.925 * cos(2 * Mm) + 48.888 * cos(Ms) + 246.158 * cos(2 * D - 2 * Mm) -
                           152.138 * cos(2 * D - Ms - Mm) - 170.733 * cos(2 * D + Mm) - 204.586 * cos(2 * D - Ms);
    const double lam = (lon - (5029.0966 * T + 1.11113 * T * T) / 3600.0) * kDeg, bet = lat * kDeg;
    const double r = dist_km * 1000.0 / kAU;
    return ecl_to_eq({r * cos(bet) * cos(lam), r * cos(bet) * sin(lam), r * sin(bet)});
}

// IAU 1976 precession matrix from epoch jd0 to epoch jd1 (rows: x, y, z of
// the target frame in the source frame's coordinates).
__device__ void precession(double jd0, double jd1, double m[3][3]) {
    const double T = (jd0 - kJ2000) / 36525.0, t = (jd1 - jd0) / 36525.0;
    const double c1 = 2306.2181 + 1.39656 * T - 0.000139 * T * T;
    const double zeta = (c1 * t + (0.30188 - 0.000344 * T) * t * t + 0.017998 * t * t * t) * kArcsec;
    const double z = (c1 * t + (1.09468 + 0.000066 * T) * t * t + 0.018203 * t * t * t) * kArcsec;
    const double th = ((2004.3109 - 0.85330 * T - 0.000217 * T * T) * t - (0.42665 + 0.000217 * T) * t * t -
                       0.041833 * t * t * t) * kArcsec;
    const double cz = cos(zeta), sz = sin(zeta), cZ = cos(z), sZ = sin(z), ct = cos(th), st = sin(th);
    m[0][0] = cZ * ct * cz - sZ * sz;
    m[0][1] = -cZ * ct * sz - sZ * cz;
    m[0][2] = -cZ * st;
    m[1][0] = sZ * ct * cz + cZ * sz;
    m[1][1] = -sZ * ct * sz + cZ * cz;
    m[1][2] = -sZ * st;
    m[2][0] = st * cz;
    m[2][1] = -st * sz;
    m[2][2] = ct;
}

__device__ __forceinline__ V3 mul(const double m[3][3], V3 v) {
    return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
            m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
}
__device__ __forceinline__ V3 mul_t(const double m[3][3], V3 v) {
    return {m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z, m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
            m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z};
}

// Sun / body mass of the barycentre's bodies, summed once: 1 + sum(m_b / M_sun)
__device__ __forceinline__ double total_mass() {
    double m = 1.0;
#pragma unroll
    for (int b = 0; b < 5; b++) m += 1.0 / kSunOverMass[b];
    return m;
}

// One warp per distinct time: the terms of the observer's velocity (m/s,
// J2000 equator) are spread over lanes and summed by shuffles.
//   lanes 0..9:   body b = lane / 2 at T + h (even lane) or T - h (odd): its
//                 heliocentric position times its weight in the Earth's
//                 barycentric position (EMB: 1 - m/M, the others: -m/M, the
//                 Sun's barycentric offset), +-1/(2h) for the central difference
//   lanes 10, 11: the Moon at T + h, T - h, weight -m_Moon / (m_E + m_M)
//   lane 12:      the site's rotation velocity (GMST, precession date -> J2000)
//   lane 13:      the solar motion, 20 km/s towards the B1900 apex
// Lane 0 turns the sum into nu_LSRK / nu_TOPO for the phase centre.
__device__ double warp_doppler_factor(const mtb_lsrk_params &p, double time_s, int lane, V3 &v) {
    const double jd_tt = 2400000.5 + (time_s + p.tt_minus_time) / kDay;
    const double T = (jd_tt - kJ2000) / 36525.0;
    const double h = kHalfStepDays / 36525.0;
    const double dscale = kAU / (2.0 * kHalfStepDays * kDay);   // au per 2h -> m/s
    v = {0.0, 0.0, 0.0};
    if (lane < 10) {
        const int b = lane >> 1;
        const double sgn = (lane & 1) ? -1.0 : 1.0;
        const double w = (b == 0 ? 1.0 : 0.0) - 1.0 / (kSunOverMass[b] * total_mass());
        v = scale(kepler_position(b, T + sgn * h), sgn * w * dscale);
    } else if (lane < 12) {
        const double sgn = lane == 10 ? 1.0 : -1.0;
        v = scale(moon_position(T + sgn * h), -sgn * kMoonFraction * dscale);
    } else if (lane == 12) {
        const double jd_ut1 = 2400000.5 + (time_s + p.ut1_minus_time) / kDay;
        const double du = jd_ut1 - kJ2000, Tu = du / 36525.0;
        double gmst =
            fmod(280.46061837 + 360.98564736629 * du + 0.000387933 * Tu * Tu - Tu * Tu * Tu / 38710000.0, 360.0);
        gmst *= kDeg;
        const double omega = 360.98564736629 * kDeg / kDay;
        const double cg = cos(gmst), sg = sin(gmst);
        const V3 r = {cg * p.site_itrf[0] - sg * p.site_itrf[1], sg * p.site_itrf[0] + cg * p.site_itrf[1],
                      p.site_itrf[2]};
        double P[3][3];
        precession(kJ2000, jd_tt, P);
        v = mul_t(P, {-omega * r.y, omega * r.x, 0.0});
    } else if (lane == 13) {
        double Q[3][3];
        precession(kB1900, kJ2000, Q);
        const double a0 = 270.0 * kDeg, d0 = 30.0 * kDeg;
        v = scale(mul(Q, {cos(d0) * cos(a0), cos(d0) * sin(a0), sin(d0)}), kLsrSpeed);
    }
    // butterfly sum: lane pairs first, so each body's central difference is
    // formed before the bodies are added
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        v.x += __shfl_xor_sync(0xFFFFFFFFu, v.x, o);
        v.y += __shfl_xor_sync(0xFFFFFFFFu, v.y, o);
        v.z += __shfl_xor_sync(0xFFFFFFFFu, v.z, o);
    }
    const V3 n = {cos(p.dec) * cos(p.ra), cos(p.dec) * sin(p.ra), sin(p.dec)};
    const double bn = dot(v, n) / kC, b2 = dot(v, v) / (kC * kC);
    return sqrt(1.0 - b2) / (1.0 + bn);
}

__device__ __forceinline__ bool is_head(const double *__restrict__ time_s, int r) {
    return r == 0 || !(time_s[r] == time_s[r - 1]);   // the reference's last_time test
}

// flags: 1 where a row starts a run of equal times (a head)
__global__ void k_lsrk_flags(const double *__restrict__ time_s, int nrows, int *__restrict__ flags) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nrows) flags[r] = is_head(time_s, r) ? 1 : 0;
}

// rank = inclusive count of heads: the head of row r is heads[rank[r] - 1]
__global__ void k_lsrk_heads(const double *__restrict__ time_s, int nrows, const int *__restrict__ rank,
                             int *__restrict__ heads, int *__restrict__ nheads) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    if (is_head(time_s, r)) heads[rank[r] - 1] = r;
    if (r == nrows - 1) *nheads = rank[r];
}

// one warp per head (grid-stride over the device-side head count)
__global__ void k_lsrk_eval(mtb_lsrk_params p, const double *__restrict__ time_s, const int *__restrict__ heads,
                            const int *__restrict__ nheads, double *__restrict__ factor) {
    const int lane = threadIdx.x & 31;
    const int nw = gridDim.x * (blockDim.x >> 5);
    const int nh = *nheads;
    for (int h = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); h < nh; h += nw) {
        V3 v;
        const double f = warp_doppler_factor(p, time_s[heads[h]], lane, v);
        if (lane == 0) factor[h] = f;
    }
}

// x / c rounded to nearest: the product with the rounded reciprocal and one
// residual correction (Brisebarre, Muller and Raina, "Accelerating correctly
// rounded floating-point division when the divisor is known in advance",
// IEEE Trans. Computers 53(8), 2004); the residual x - q0 c is exact under FMA
__device__ __forceinline__ double div_c(double x) {
    constexpr double inv = 1.0 / kC;
    const double q0 = x * inv;
    const double e = fma(-q0, kC, x);
    return fma(e, inv, q0);
}

// out[c][k] = (float)(chan_hz[c] * factor / c) for row = index[k] (k itself
// without an index); a row outside [0, nrows) gives NaN.  VEC: 4 consecutive
// records per thread, one 16-byte store per channel (n a multiple of 4 and
// out 16-byte aligned); the four rows' gathers are independent loads in
// flight together.  Streaming stores: the output is not read again here.
__device__ __forceinline__ float lsrk_value(const double *__restrict__ chan_hz, int c, double f, bool ok) {
    return ok ? (float)div_c(chan_hz[c] * f) : __int_as_float(0x7fc00000);
}

template <bool VEC>
__global__ void k_lsrk_write(const double *__restrict__ chan_hz, int nchan, const int *__restrict__ index, int n,
                             int nrows, const int *__restrict__ rank, const double *__restrict__ factor,
                             float *__restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if constexpr (VEC) {
        const int k0 = 4 * t;
        if (k0 >= n) return;
        int row[4];
        bool ok[4];
        double f[4];
        if (index) {
            const int4 r4 = *reinterpret_cast<const int4 *>(index + k0);
            row[0] = r4.x, row[1] = r4.y, row[2] = r4.z, row[3] = r4.w;
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) row[j] = k0 + j;
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            ok[j] = row[j] >= 0 && row[j] < nrows;
            f[j] = ok[j] ? factor[rank[row[j]] - 1] : 0.0;
        }
        for (int c = 0; c < nchan; c++) {
            const float4 v = make_float4(lsrk_value(chan_hz, c, f[0], ok[0]), lsrk_value(chan_hz, c, f[1], ok[1]),
                                         lsrk_value(chan_hz, c, f[2], ok[2]), lsrk_value(chan_hz, c, f[3], ok[3]));
            __stcs(reinterpret_cast<float4 *>(out + (size_t)c * n + k0), v);
        }
    } else {
        const int k = t;
        if (k >= n) return;
        const int row = index ? index[k] : k;
        const bool ok = row >= 0 && row < nrows;
        const double f = ok ? factor[rank[row] - 1] : 0.0;
        for (int c = 0; c < nchan; c++) __stcs(out + (size_t)c * n + k, lsrk_value(chan_hz, c, f, ok));
    }
}

struct Carve {
    int *flags;     // 1 at head rows
    int *rank;      // inclusive count of heads
    int *heads;     // head rows in order
    int *nheads;    // head count (device)
    double *factor; // nu_LSRK / nu_TOPO per head
    void *cub;
    size_t cub_bytes;
};

static int carve(int nrows, void *ws, size_t ws_bytes, Carve &c, size_t *total) {
    size_t cub_bytes = 0;
    MTB_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, cub_bytes, (int *)nullptr, (int *)nullptr, nrows));
    Arena a(ws, ws_bytes);
    c.flags = a.take<int>((size_t)nrows);
    c.rank = a.take<int>((size_t)nrows);
    c.heads = a.take<int>((size_t)nrows);
    c.nheads = a.take<int>(1);
    c.factor = a.take<double>((size_t)nrows);
    c.cub = a.take<char>(cub_bytes);
    c.cub_bytes = cub_bytes;
    if (total) *total = a.used;
    return (ws && !a.ok()) ? MTB_ERR_WORKSPACE : MTB_OK;
}

}  // namespace lsrk
}  // namespace mtb

extern "C" int mtb_lsrk_workspace_size(int nrows, size_t *bytes) {
    if (!bytes) return MTB_ERR_NULL;
    if (nrows < 0) return MTB_ERR_BAD_PARAM;
    mtb::lsrk::Carve c;
    return mtb::lsrk::carve(nrows > 0 ? nrows : 1, nullptr, 0, c, bytes);
}

extern "C" int mtb_lsrk_freq_over_c(const mtb_lsrk_params *params, const double *time_s, int nrows,
                                    const double *chan_hz, int nchan, const int *index, int n, float *out,
                                    void *workspace, size_t workspace_bytes, mtb_stream_t stream) {
    using namespace mtb::lsrk;
    MTB_RANGE("mtb_lsrk_freq_over_c");
    if (!params) return MTB_ERR_NULL;
    if (nrows < 0 || nchan < 0 || n < 0) return MTB_ERR_BAD_PARAM;
    if (!index && n != nrows && n > 0) return MTB_ERR_BAD_PARAM;
    const mtb_lsrk_params p = *params;
    if (!std::isfinite(p.ra) || !std::isfinite(p.dec) || !std::isfinite(p.tt_minus_time) ||
        !std::isfinite(p.ut1_minus_time) || !std::isfinite(p.site_itrf[0]) || !std::isfinite(p.site_itrf[1]) ||
        !std::isfinite(p.site_itrf[2]))
        return MTB_ERR_BAD_PARAM;
    if (n == 0 || nchan == 0) return MTB_OK;
    if (nrows == 0) return MTB_ERR_BAD_PARAM;   // records to write but no rows to read
    if (!time_s || !chan_hz || !out || !workspace) return MTB_ERR_NULL;
    Carve c;
    MTB_TRY(carve(nrows, workspace, workspace_bytes, c, nullptr));
    cudaStream_t st = (cudaStream_t)stream;
    const int T = 256;
    const int rb = (nrows + T - 1) / T;
    k_lsrk_flags<<<rb, T, 0, st>>>(time_s, nrows, c.flags);
    MTB_LAUNCHED();
    MTB_CUDA_TRY(cub::DeviceScan::InclusiveSum(c.cub, c.cub_bytes, c.flags, c.rank, nrows, st));
    k_lsrk_heads<<<rb, T, 0, st>>>(time_s, nrows, c.rank, c.heads, c.nheads);
    MTB_LAUNCHED();
    int dev = 0, sms = 148;
    MTB_CUDA_TRY(cudaGetDevice(&dev));
    MTB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int eval_blocks = std::min((nrows + 3) / 4, sms * 16);   // 4 warps per block, one head per warp
    k_lsrk_eval<<<eval_blocks, 128, 0, st>>>(p, time_s, c.heads, c.nheads, c.factor);
    MTB_LAUNCHED();
    // 16-byte rows: n a multiple of 4, out and index 16-byte aligned
    const bool vec = n % 4 == 0 && ((uintptr_t)out & 15) == 0 && ((uintptr_t)index & 15) == 0;
    if (vec)
        k_lsrk_write<true><<<(n / 4 + T - 1) / T, T, 0, st>>>(chan_hz, nchan, index, n, nrows, c.rank, c.factor, out);
    else
        k_lsrk_write<false><<<(n + T - 1) / T, T, 0, st>>>(chan_hz, nchan, index, n, nrows, c.rank, c.factor, out);
    MTB_LAUNCHED();
    return MTB_OK;
}
