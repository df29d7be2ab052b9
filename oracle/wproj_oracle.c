/*
 * wproj_oracle.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * FP64 CPU restatement of mt-imager's W-projection imaging path, used only by
 * tests/, __graft_entry__.smoke() and the cpu_baseline / reference legs of
 * bench.py as the checker.  Nothing in mt-imager_b200/ links, loads or calls
 * this file.  Each function names the reference file:line it restates (paths
 * relative to the reference project's code/ directory).
 *
 * Precision: every quantity the reference computes in float is computed here
 * in double, in the same operation order, with FP contraction disabled
 * (-ffp-contract=off), so the integer decisions (w-plane, grid corner,
 * oversampling offset) agree bit for bit with the CUDA path, which evaluates
 * the same expressions with explicitly rounded FP64 intrinsics.
 *
 * Complex arrays are interleaved (re, im) doubles unless stated otherwise.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ taper */
/* Schwab's rational approximation of the M=6, alpha=1 prolate spheroidal
 * function: mt-imager/lib/operators/CasaGridSF.cu:41-85 (coefficients are the
 * published casacore/Schwab values). */
double orc_grdsf(double nu)
{
    static const double P[2][5] = {
        {8.203343e-2, -3.644705e-1, 6.278660e-1, -5.335581e-1, 2.312756e-1},
        {4.028559e-3, -3.697768e-2, 1.021332e-1, -1.201436e-1, 6.412774e-2}};
    static const double Q[2][3] = {{1.0, 8.212018e-1, 2.078043e-1},
                                   {1.0, 9.599102e-1, 2.918724e-1}};
    int part = (nu < 0.75) ? 0 : 1;
    double nuend2 = part ? 1.0 : 0.5625;
    double d = nu * nu - nuend2;
    double top = P[part][0], bot = Q[part][0], dk = 1.0;
    for (int k = 1; k < 5; k++) { dk *= d; top += P[part][k] * dk; }
    dk = 1.0;
    for (int k = 1; k < 3; k++) { dk *= d; bot += Q[part][k] * dk; }
    return (bot != 0.0) ? top / bot : 0.0;
}

/* Image-plane taper on an ny x nx lm grid: CasaGridSF.cu:151-173
 * (casacore_gridsf_correction_generate; nu = |j - n/2| / (n/2), integer n/2). */
void orc_taper_lm(int ny, int nx, double *out)
{
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            double nuy = fabs((double)(j - ny / 2) / (double)(ny / 2));
            double nux = fabs((double)(i - nx / 2) / (double)(nx / 2));
            out[(size_t)j * nx + i] = orc_grdsf(nuy) * orc_grdsf(nux);
        }
}

/* uv-plane spheroidal kernel for mode=normal: CasaGridSF.cu:107-149,
 * size from CasaGridSF.cpp:89-92.  out: real [size][size]. */
void orc_gridsf_uv(int size, int sampling, double *out)
{
    int first_zero = 3 * sampling;
    for (int j = 0; j < size; j++)
        for (int i = 0; i < size; i++) {
            int ii = abs(i - size / 2), jj = abs(j - size / 2);
            double v = 0.0;
            if (ii < first_zero && jj < first_zero) {
                double ni = (double)ii / (double)first_zero, nj = (double)jj / (double)first_zero;
                v = (1 - ni * ni) * orc_grdsf(ni) * (1 - nj * nj) * orc_grdsf(nj);
            }
            out[(size_t)j * size + i] = v;
        }
}

/* mt-imager/lib/operators/common.hcu:107-136 */
static int origin_to_corner(int loc, int dim)
{
    if (dim % 2) return (loc < dim / 2) ? loc + dim / 2 + 1 : loc - dim / 2;
    return (loc < dim / 2) ? loc + dim / 2 : loc - dim / 2;
}
static int origin_to_centre(int loc, int dim)
{
    if (dim % 2) return (loc <= dim / 2) ? loc + dim / 2 : loc - dim / 2 - 1;
    return (loc < dim / 2) ? loc + dim / 2 : loc - dim / 2;
}
int orc_origin_to_corner(int loc, int dim) { return origin_to_corner(loc, dim); }
int orc_origin_to_centre(int loc, int dim) { return origin_to_centre(loc, dim); }

/* w-screen times taper, zero padded to (St*s)^2 and written origin-to-corner:
 * mt-imager/lib/operators/WProjPreFFTconvFunc.cu:34-105, increments from
 * :130-131 (total_l / support).  out: complex [St*s][St*s]. */
void orc_wscreen(const double *taper, int St, int s, double total_l, double total_m,
                 double w, int leavedge, double *out)
{
    int ps = St * s;
    double linc = total_l / (double)St, minc = total_m / (double)St;
    for (int y = 0; y < ps; y++)
        for (int x = 0; x < ps; x++) {
            int cx = x - ps / 2, cy = y - ps / 2;
            double re = 0.0, im = 0.0;
            if (!(cy < -St / 2 || cy > (St / 2 - leavedge) || cx < -St / 2 || cx > (St / 2 - leavedge))) {
                double two_w = 2.0 * w;
                double m = minc * (double)cy; double msq = m * m;
                double l = linc * (double)cx; double lsq = l * l;
                double rsq = lsq + msq;
                double t = taper[(size_t)(cy + St / 2) * St + (cx + St / 2)];
                if (rsq < 1.0) {
                    double phase = two_w * (sqrt(1.0 - rsq) - 1.0);
                    /* cospi/sinpi(phase) */
                    re = cos(M_PI * phase) * t;
                    im = sin(M_PI * phase) * t;
                } else {
                    re = t;
                    im = 0.0;
                }
            }
            size_t pos = (size_t)origin_to_corner(y, ps) * ps + origin_to_corner(x, ps);
            out[2 * pos] = re;
            out[2 * pos + 1] = im;
        }
}

/* fftshift of a complex plane: std ZeroToCentre2DShift.cu:67-91 */
void orc_zero_to_centre(const double *in, double *out, int ny, int nx)
{
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
            size_t src = (size_t)y * nx + x;
            size_t dst = (size_t)origin_to_centre(y, ny) * nx + origin_to_centre(x, nx);
            out[2 * dst] = in[2 * src];
            out[2 * dst + 1] = in[2 * src + 1];
        }
}

/* Support of a centred, normalised kernel plane: ConvFunctionSupportFind.cu:28-77.
 * The last location (scanning the centre row and the centre column outwards
 * from the centre) whose |C|^2 exceeds takezero2 sets
 * support = ((loc - dim/2 + (s+1)/2) / s) * 2 + 1, or 0 if none. */
int orc_support_find(const double *c, int dim, int s, double takezero2)
{
    int last = -1;
    for (int loc = dim / 2; loc < dim; loc++) {
        size_t prow = (size_t)(dim / 2) * dim + loc;   /* threadIdx.y == 0 */
        size_t pcol = (size_t)loc * dim + dim / 2;     /* threadIdx.y == 1 */
        double m0 = c[2 * prow] * c[2 * prow] + c[2 * prow + 1] * c[2 * prow + 1];
        double m1 = c[2 * pcol] * c[2 * pcol] + c[2 * pcol + 1] * c[2 * pcol + 1];
        if (m0 > takezero2 || m1 > takezero2) last = loc;
    }
    if (last < 0) return 0;
    return ((last - dim / 2 + (s + 1) / 2) / s) * 2 + 1;
}

/* Cut-out and reorder into [oy][ox][sy][sx] sub-kernels:
 * ConvFunctionReOrganize.cu:30-71 (odd and even sampling; T = s or s+1).
 * out: complex [T*T*S*S]. */
void orc_reorganize(const double *c, int dim, int S, int s, double *out)
{
    int T = (s % 2) ? s : s + 1;
    int cb = dim / 2 - ((S / 2) * s + s / 2);
    for (int oy = 0; oy < T; oy++)
        for (int ox = 0; ox < T; ox++)
            for (int py = 0; py < S; py++)
                for (int px = 0; px < S; px++) {
                    size_t o = ((size_t)(oy * T + ox) * S + py) * S + px;
                    size_t i = (size_t)(py * s + oy + cb) * dim + (px * s + ox + cb);
                    out[2 * o] = c[2 * i];
                    out[2 * o + 1] = c[2 * i + 1];
                }
}

/* Per-(plane, offset) sum of the real part: SumConvolutionFunctions.cu:29-56.
 * conv_info: int [nw][2] {support, offset (complex elements)}. out: [nw][T*T]. */
void orc_conv_sums(const double *table, const int *conv_info, int nw, int T, double *out)
{
    for (int k = 0; k < nw; k++) {
        int S = conv_info[2 * k], base = conv_info[2 * k + 1];
        for (int o = 0; o < T * T; o++) {
            double v = 0.0;
            size_t b = (size_t)base + (size_t)o * S * S;
            for (int i = 0; i < S * S; i++) v += table[2 * (b + i)];
            out[(size_t)k * T * T + o] = v;
        }
    }
}

/* ----------------------------------------------------------- preprocess */
/* Per-record gridding decisions: WProjPreProcessUVW.cu:112-286 (block part)
 * and :287-324 (compression across block boundaries), here over the whole
 * record stream at once, FP64 coordinates.
 *   uvw   float [3][R] metres       freq  float [R] nu/c
 *   weights float [R][P]            flags int [R][P]
 *   conv_info int [nw][2]           conv_sums double [nw][T*T]
 * Outputs (all [R] unless noted):
 *   loc int [R][4] = {cx, cy*nu+cx, -(cx % S), -(cy % S)}  (zero if not gridded)
 *   convidx, togrid (after compression), compress, support, plane, offx, offy
 *   imgmult float (+1 / -1), convsum double [P][R]. */
void orc_preprocess(int R, int P, const float *uvw, const float *freq, const float *weights,
                    const int *flags, int nw, double w_inc, const int *conv_info,
                    const double *conv_sums, int s, int nv, int nu, double du, double dv,
                    int *loc, int *convidx, int *togrid, int *compress, int *support,
                    int *plane, int *offx, int *offy, float *imgmult, double *convsum)
{
    int T = (s % 2) ? s : s + 1;
    for (int r = 0; r < R; r++) {
        int grid = 0;
        for (int p = 0; p < P; p++) if (flags[(size_t)r * P + p] == 0) grid = 1;
        int l4[4] = {0, 0, 0, 0}, ci = 0, S = 0, k = 0, ox = 0, oy = 0;
        float im = 1.0f;
        double cs = 0.0;
        if (grid) {
            double u = uvw[r], v = uvw[(size_t)R + r], w = uvw[2 * (size_t)R + r], f = freq[r];
            if (w < 0.0) { u = -u; v = -v; im = -1.0f; }
            double wp = round(sqrt(fabs((w * f) / w_inc)));
            /* non-finite input is rejected (the reference's float->int
             * conversion is undefined there) */
            if (!(wp == wp)) wp = 0.0;
            k = (wp > (double)(nw - 1)) ? nw - 1 : (int)wp;
            S = conv_info[2 * k];
            ci = conv_info[2 * k + 1];
            double pos_v = ((v * f) / dv) + (double)(nv / 2);
            double pos_u = ((u * f) / du) + (double)(nu / 2);
            double lx = round(pos_u), ly = round(pos_v);
            /* range test in double before any conversion to int */
            double cxd = lx - (double)(S / 2), cyd = ly - (double)(S / 2);
            if (!(cyd >= 0.0) || cyd > (double)((nv - 1) - S) || !(cxd >= 0.0) || cxd > (double)(nu - 1 - S)) {
                grid = 0;
            } else {
                int cx = (int)cxd, cy = (int)cyd;
                ox = (int)round((lx - pos_u) * (double)s) + s / 2;
                oy = (int)round((ly - pos_v) * (double)s) + s / 2;
                if (s % 2) {
                    if (ox < 0) ox = 0;
                    if (oy < 0) oy = 0;
                    if (ox == s) ox--;
                    if (oy == s) oy--;
                }
                cs = conv_sums[(size_t)k * T * T + oy * T + ox];
                ci += oy * S * S * T + ox * S * S;
                l4[0] = cx; l4[1] = cy * nu + cx; l4[2] = -(cx % S); l4[3] = -(cy % S);
            }
        }
        if (!grid) { S = 0; ci = 0; l4[0] = l4[1] = l4[2] = l4[3] = 0; cs = 0.0; k = 0; ox = oy = 0; }
        memcpy(loc + 4 * (size_t)r, l4, sizeof l4);
        convidx[r] = ci; togrid[r] = grid; support[r] = S; imgmult[r] = im;
        plane[r] = k; offx[r] = ox; offy[r] = oy;
        for (int p = 0; p < P; p++) {
            double wt = weights[(size_t)r * P + p];
            double fl = (double)flags[(size_t)r * P + p];
            convsum[(size_t)p * R + r] = cs * wt * (1.0 - fl);
        }
    }
    /* consecutive duplicates (same corner row-index and conv index) compress
     * into the previous record; the previous record's stored values are used
     * whether or not it was gridded (WProjPreProcessUVW.cu:265-284, 316) */
    compress[0] = 0;
    for (int r = R - 1; r >= 1; r--) {
        int c = 0;
        if (togrid[r] && convidx[r] == convidx[r - 1] && loc[4 * (size_t)r + 1] == loc[4 * (size_t)(r - 1) + 1]) c = 1;
        compress[r] = c;
    }
    for (int r = 1; r < R; r++) if (compress[r]) togrid[r] = 0;
}

/* Weighted, conjugation-corrected visibility of every gridded record summed
 * over the run of records compressed into it: CreateCompressionPlan.cu:32-67
 * and CompressVisibilties.cu:41-74 with common.hcu:94-104.
 *   vis float [R][2P]  ->  out double [R][2P] (rows of non-gridded records = 0) */
void orc_compress_vis(int R, int P, const int *togrid, const int *compress, const float *vis,
                      const float *weights, const int *flags, const float *imgmult, double *out)
{
    memset(out, 0, sizeof(double) * (size_t)R * 2 * P);
    for (int g = 0; g < R; g++) {
        if (!togrid[g]) continue;
        int e = g;
        while (e + 1 < R && compress[e + 1]) e++;
        for (int r = g; r <= e; r++)
            for (int p = 0; p < P; p++) {
                double wt = weights[(size_t)r * P + p] * (1.0 - (double)flags[(size_t)r * P + p]);
                out[(size_t)g * 2 * P + 2 * p] += (double)vis[(size_t)r * 2 * P + 2 * p] * wt;
                out[(size_t)g * 2 * P + 2 * p + 1] += (double)vis[(size_t)r * 2 * P + 2 * p + 1] * wt * (double)imgmult[r];
            }
    }
}

/* Convolutional gridding: ConvolutionGridder.cu:130-181 (complex multiply,
 * no conjugate of C) and :394-442 (cell = corner + (sx, sy), tap = sy*S + sx).
 * Row bands are split across OpenMP threads so no two threads touch a cell.
 *   cvis double [R][2P] (from orc_compress_vis), table complex double,
 *   grid complex double [nv][nu][P] (accumulated). */
void orc_grid(int R, int P, const int *togrid, const int *loc, const int *convidx,
              const int *support, const double *cvis, const double *table, int nv, int nu,
              double *grid)
{
#pragma omp parallel
    {
        int nt = 1, t = 0;
#ifdef _OPENMP
        nt = omp_get_num_threads();
        t = omp_get_thread_num();
#endif
        int y0 = (int)((long)nv * t / nt), y1 = (int)((long)nv * (t + 1) / nt);
        for (int r = 0; r < R; r++) {
            if (!togrid[r]) continue;
            int S = support[r], cx = loc[4 * (size_t)r];
            int cy = (loc[4 * (size_t)r + 1] - cx) / nu;
            if (cy + S <= y0 || cy >= y1) continue;
            const double *V = cvis + (size_t)r * 2 * P;
            for (int sy = 0; sy < S; sy++) {
                int y = cy + sy;
                if (y < y0 || y >= y1) continue;
                for (int sx = 0; sx < S; sx++) {
                    size_t ti = (size_t)convidx[r] + (size_t)sy * S + sx;
                    double cr = table[2 * ti], cim = table[2 * ti + 1];
                    double *g = grid + ((size_t)y * nu + (cx + sx)) * 2 * P;
                    for (int p = 0; p < P; p++) {
                        double vr = V[2 * p], vi = V[2 * p + 1];
                        g[2 * p] += vr * cr - vi * cim;
                        g[2 * p + 1] += vi * cr + vr * cim;
                    }
                }
            }
        }
    }
}

/* Direct FP64 DFT of the same weighted records the gridder sees, giving the
 * dirty polarisation images before Stokes conversion:
 *   out[p][y][x] = sum_r V'_rp exp(+2 pi i (u l + v m + w (n - 1)))
 * with l = (x - nx/2) dl, m = (y - ny/2) dm and (u, v, w, V') the
 * reference's conjugated record for w < 0 (WProjPreProcessUVW.cu:170-175).
 *   uvw_lambda double [3][R], cvis double [R][2P]  -> out complex [P][ny][nx] */
void orc_dft(int R, int P, const double *uvw_lambda, const double *cvis, const int *use,
             int nx, int ny, double dl, double dm, double *out)
{
    const double *U = uvw_lambda, *Vv = uvw_lambda + R, *W = uvw_lambda + 2 * (size_t)R;
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < ny; y++) {
        double m = (double)(y - ny / 2) * dm;
        for (int x = 0; x < nx; x++) {
            double l = (double)(x - nx / 2) * dl;
            double n1 = sqrt(1.0 - l * l - m * m) - 1.0;
            double acc[8] = {0};
            for (int r = 0; r < R; r++) {
                if (!use[r]) continue;
                double u = U[r], v = Vv[r], w = W[r];
                if (w < 0.0) { u = -u; v = -v; w = -w; }
                double ph = 2.0 * M_PI * (u * l + v * m + w * n1);
                double c = cos(ph), sn = sin(ph);
                for (int p = 0; p < P; p++) {
                    double vr = cvis[(size_t)r * 2 * P + 2 * p], vi = cvis[(size_t)r * 2 * P + 2 * p + 1];
                    acc[2 * p] += vr * c - vi * sn;
                    acc[2 * p + 1] += vr * sn + vi * c;
                }
            }
            for (int p = 0; p < P; p++) {
                size_t o = ((size_t)p * ny + y) * nx + x;
                out[2 * o] = acc[2 * p];
                out[2 * o + 1] = acc[2 * p + 1];
            }
        }
    }
}
