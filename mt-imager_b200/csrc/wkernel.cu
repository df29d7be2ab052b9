// W-projection kernel generation for sm_100a.
//
// Replaces the reference's serial host loop over w-planes
// (code/mt-imager/lib/components/ConvolutionFunctionsGenerator/
// WProjectionConvFunction.cpp:186-291), which runs taper -> screen -> FFT ->
// shift -> scale -> support find for one plane at a time and reads the support
// back to the host twice per plane.  Here all planes go through each step as
// one batch: one screen launch, one batched cuFFT Z2Z, one support launch, one
// host read-back of all supports, one cut-out launch and one sum launch.  The
// w-phase and the FFT are FP64; the table is stored as float2 (the reference's
// complex_float AmalgamatedConvFunction).
#include <cmath>
#include <vector>

#include "fft_plans.cuh"
#include "mtb_internal.cuh"

namespace mtb {

// (1e-3f)^2: ConvFunctionSupportFind's threshold
// (WPlaneConvFunctionCalculator.cpp:61, ConvFunctionSupportFind.cu:99)
static const double kTakeAsZero2 = (double)1e-3f * (double)1e-3f;
static const size_t kPlaneBatchBytes = (size_t)4 << 30;

struct WGeom {
    int St, s, ps, nw, T, cap;
    double w_inc, total_l, total_m, w_max;
};

static int wgeom(const mtb_wkernel_params *p, WGeom *g) {
    if (!p) return MTB_ERR_NULL;
    if (p->nx < 2 || p->ny < 2 || p->wplanes < 1 || p->sampling < 1) return MTB_ERR_BAD_PARAM;
    if (!(p->l_increment > 0.0) || !(p->m_increment > 0.0)) return MTB_ERR_BAD_PARAM;
    int img_min = p->nx < p->ny ? p->nx : p->ny;
    int St = p->trial_support;
    if (St <= 0) {
        St = img_min / p->sampling;           // WProjectionConvFunction.cpp:196-197
        if (St % 2 == 0) St++;
    } else if (St % 2 == 0) {
        return MTB_ERR_BAD_PARAM;             // support is expected to be odd (WProjPreFFTconvFunc.cpp:77)
    }
    if (St < 3) return MTB_ERR_BAD_PARAM;
    g->St = St;
    g->s = p->sampling;
    g->ps = St * p->sampling;
    g->nw = p->wplanes;
    g->T = oversample_T(p->sampling);
    g->cap = St - 2;                          // WProjectionConvFunction.cpp:248-249
    if (p->max_support > 0 && p->max_support < g->cap) g->cap = p->max_support;
    g->w_max = (p->w_max > 0.0) ? p->w_max : 0.25 / p->l_increment;   // :105
    g->w_inc = (p->wplanes == 1) ? 1.0 : g->w_max / (double)((p->wplanes - 1) * (p->wplanes - 1));  // :111-112
    g->total_l = p->l_increment * (double)p->nx;
    g->total_m = p->m_increment * (double)p->ny;
    if ((size_t)g->ps * g->ps > ((size_t)1 << 31)) return MTB_ERR_BAD_SHAPE;
    return MTB_OK;
}

static int plane_batch(const WGeom &g) {
    size_t per = (size_t)g.ps * g.ps * sizeof(double2);
    size_t nb = kPlaneBatchBytes / per;
    if (nb < 1) nb = 1;
    if (nb > (size_t)g.nw) nb = g.nw;
    return (int)nb;
}

// workspace layout (carved in this order)
struct WSpace {
    double2 *divisor;
    int *supports;
    int *conv_info;
    double2 *planes;
    void *fftwork;
    size_t fftbytes;
};

static int carve(const WGeom &g, int nb, void *ws, size_t bytes, WSpace *w, size_t *need) {
    cufftHandle h;
    size_t fw = 0;
    MTB_TRY(fft_plan(CUFFT_Z2Z, g.ps, g.ps, nb, &h, &fw));
    Arena a(ws, bytes);
    w->divisor = a.take<double2>(1);
    w->supports = a.take<int>(g.nw);
    w->conv_info = a.take<int>(2 * (size_t)g.nw);
    w->planes = a.take<double2>((size_t)nb * g.ps * g.ps);
    w->fftwork = a.take<char>(fw ? fw : 1);
    w->fftbytes = fw;
    if (need) *need = a.used;
    return MTB_OK;
}

// ---------------------------------------------------------------- kernels --
// Taper x w-screen, zero padded and written origin-to-corner, for planes
// [k0, k0+nb): WProjPreFFTconvFunc.cu:34-105 with the taper of
// CasaGridSF.cu:151-173 evaluated in place (nu = |c| / (St/2)).  FP64.
__global__ void k_wscreen(double2 *planes, int nb, int k0, int St, int ps, double linc,
                          double minc, double w_inc) {
    const size_t per = (size_t)ps * ps;
    const size_t total = per * nb;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        int b = (int)(i / per);
        int rem = (int)(i - (size_t)b * per);
        int y = rem / ps, x = rem - y * ps;
        int cx = x - ps / 2, cy = y - ps / 2;
        double re = 0.0, im = 0.0;
        if (!(cy < -St / 2 || cy > St / 2 || cx < -St / 2 || cx > St / 2)) {
            int k = k0 + b;
            double w = (double)k * (double)k * w_inc;
            double half = (double)(St / 2);
            double t = grdsf(fabs((double)cy / half)) * grdsf(fabs((double)cx / half));
            double m = __dmul_rn(minc, (double)cy);
            double l = __dmul_rn(linc, (double)cx);
            double rsq = __dadd_rn(__dmul_rn(l, l), __dmul_rn(m, m));
            if (rsq < 1.0) {
                double phase = __dmul_rn(2.0 * w, __dadd_rn(sqrt(1.0 - rsq), -1.0));
                double sn, cs;
                sincospi(phase, &sn, &cs);
                re = cs * t;
                im = sn * t;
            } else {
                re = t;
            }
        }
        size_t o = (size_t)b * per + (size_t)origin_to_corner(y, ps) * ps + origin_to_corner(x, ps);
        planes[o] = make_double2(re, im);
    }
}

__global__ void k_copy_divisor(const double2 *plane0, double2 *divisor) { *divisor = plane0[0]; }

// ConvFunctionSupportFind.cu:28-77 on the unshifted FFT output: the centred
// (fftshifted, ZeroToCentre2DShift.cu:67-91) location c reads unshifted index
// centre_to_origin(c).  One block per plane; the largest c >= ps/2 on the
// centre row or column whose normalised |C|^2 exceeds (1e-3)^2 sets the support.
__global__ void k_support_find(const double2 *planes, int k0, int ps, int s, const double2 *divisor,
                               int cap, int *supports) {
    __shared__ int last;
    if (threadIdx.x == 0) last = -1;
    __syncthreads();
    const double2 *pl = planes + (size_t)blockIdx.x * ps * ps;
    const double mult = 1.0 / divisor->x;
    const int oc = centre_to_origin(ps / 2, ps);
    for (int c = ps / 2 + threadIdx.x; c < ps; c += blockDim.x) {
        int oi = centre_to_origin(c, ps);
        double2 a = pl[(size_t)oc * ps + oi];      // centre row
        double2 b = pl[(size_t)oi * ps + oc];      // centre column
        double ar = __dmul_rn(a.x, mult), ai = __dmul_rn(a.y, mult);
        double br = __dmul_rn(b.x, mult), bi = __dmul_rn(b.y, mult);
        double ma = __dadd_rn(__dmul_rn(ar, ar), __dmul_rn(ai, ai));
        double mb = __dadd_rn(__dmul_rn(br, br), __dmul_rn(bi, bi));
        if (ma > kTakeAsZero2 || mb > kTakeAsZero2) atomicMax(&last, c);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int sup = 0;
        if (last > -1) sup = ((last - ps / 2 + (s + 1) / 2) / s) * 2 + 1;
        if (sup > cap) sup = cap;
        supports[k0 + blockIdx.x] = sup;
    }
}

// ConvFunctionReOrganize.cu:30-71: cut out S*T per axis around the centre and
// reorder to [oy][ox][sy][sx] (T = s for odd, s+1 for even sampling), scaled
// by 1/DC(w=0) (SingleMultiply), into the concatenated table (ArraysToVector).
__global__ void k_reorganize(const double2 *planes, int nb, int k0, int ps, int s, int T,
                             const int *conv_info, const double2 *divisor, float2 *table) {
    const double mult = 1.0 / divisor->x;
    for (int b = blockIdx.y; b < nb; b += gridDim.y) {
        int k = k0 + b;
        int S = conv_info[2 * k], base = conv_info[2 * k + 1];
        int cb = ps / 2 - ((S / 2) * s + s / 2);
        size_t n = (size_t)T * T * S * S;
        const double2 *pl = planes + (size_t)b * ps * ps;
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
             i += (size_t)gridDim.x * blockDim.x) {
            int px = (int)(i % S);
            size_t r = i / S;
            int py = (int)(r % S);
            r /= S;
            int ox = (int)(r % T), oy = (int)(r / T);
            int yc = py * s + oy + cb, xc = px * s + ox + cb;
            double2 v = pl[(size_t)centre_to_origin(yc, ps) * ps + centre_to_origin(xc, ps)];
            table[(size_t)base + i] = make_float2((float)(v.x * mult), (float)(v.y * mult));
        }
    }
}

// SumConvolutionFunctions.cu:29-56: sum of the real part of each sub-kernel,
// one warp per (plane, offset), FP64 accumulation.
__global__ void k_conv_sums(const float2 *table, const int *conv_info, int nw, int T, float *sums) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int total = nw * T * T;
    if (warp >= total) return;
    int k = warp / (T * T), o = warp - k * T * T;
    int S = conv_info[2 * k];
    size_t b = (size_t)conv_info[2 * k + 1] + (size_t)o * S * S;
    double v = 0.0;
    for (int i = lane; i < S * S; i += 32) v += (double)table[b + i].x;
    for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) sums[warp] = (float)v;
}

static int launch_screen_fft(const WGeom &g, const WSpace &w, int k0, int nb, cudaStream_t st) {
    size_t total = (size_t)nb * g.ps * g.ps;
    int blocks = (int)((total + 255) / 256);
    int cap = sm_count() * 16;
    if (blocks > cap) blocks = cap;
    k_wscreen<<<blocks, 256, 0, st>>>(w.planes, nb, k0, g.St, g.ps, g.total_l / (double)g.St,
                                      g.total_m / (double)g.St, g.w_inc);
    MTB_LAUNCHED();
    return fft_exec(CUFFT_Z2Z, g.ps, g.ps, nb, w.planes, w.planes, CUFFT_FORWARD, w.fftwork,
                    w.fftbytes, st);
}

}  // namespace mtb

using namespace mtb;

extern "C" int mtb_wkernel_query(const mtb_wkernel_params *p, mtb_wkernel_info *info) {
    if (!info) return MTB_ERR_NULL;
    WGeom g;
    MTB_TRY(wgeom(p, &g));
    int nb = plane_batch(g);
    WSpace w;
    size_t need = 0;
    MTB_TRY(carve(g, nb, nullptr, 0, &w, &need));
    info->trial_support = g.St;
    info->planesize = g.ps;
    info->support_cap = g.cap;
    info->T = g.T;
    info->w_max = g.w_max;
    info->w_sq_increment = g.w_inc;
    info->total_l = g.total_l;
    info->total_m = g.total_m;
    info->u_increment = 1.0 / g.total_l;
    info->v_increment = 1.0 / g.total_m;
    info->table_capacity = (size_t)g.nw * g.T * g.T * (size_t)g.cap * g.cap;
    info->workspace_bytes = need;
    return MTB_OK;
}

extern "C" int mtb_wkernel_build(const mtb_wkernel_params *p, void *d_workspace, size_t workspace_bytes,
                                 void *d_table, size_t table_capacity, int *d_conv_info, int *h_conv_info,
                                 float *d_conv_sums, size_t *table_elems, mtb_stream_t stream) {
    MTB_RANGE("mtb_wkernel_build");
    if (!d_workspace || !d_table || !h_conv_info || !d_conv_sums) return MTB_ERR_NULL;
    cudaStream_t st = (cudaStream_t)stream;
    WGeom g;
    MTB_TRY(wgeom(p, &g));
    int nb = plane_batch(g);
    WSpace w;
    size_t need = 0;
    MTB_TRY(carve(g, nb, d_workspace, workspace_bytes, &w, &need));
    if (need > workspace_bytes) return MTB_ERR_WORKSPACE;

    // pass 1: screens, FFTs and supports of every plane (plane 0 is w = 0 and
    // supplies the DC divisor, WPlaneConvFunctionCalculator.cpp:128-142)
    for (int k0 = 0; k0 < g.nw; k0 += nb) {
        int n = (g.nw - k0 < nb) ? g.nw - k0 : nb;
        MTB_TRY(launch_screen_fft(g, w, k0, n, st));
        if (k0 == 0) {
            k_copy_divisor<<<1, 1, 0, st>>>(w.planes, w.divisor);
            MTB_LAUNCHED();
        }
        k_support_find<<<n, 256, 0, st>>>(w.planes, k0, g.ps, g.s, w.divisor, g.cap, w.supports);
        MTB_LAUNCHED();
    }
    std::vector<int> sup(g.nw);
    double2 div;
    MTB_CUDA_TRY(cudaMemcpyAsync(sup.data(), w.supports, sizeof(int) * g.nw, cudaMemcpyDeviceToHost, st));
    MTB_CUDA_TRY(cudaMemcpyAsync(&div, w.divisor, sizeof(double2), cudaMemcpyDeviceToHost, st));
    MTB_CUDA_TRY(cudaStreamSynchronize(st));
    // WProjectionConvFunction.cpp:213-218
    if (div.y > 1e-3 || !(div.x != 0.0)) return MTB_ERR_KERNEL;
    size_t off = 0;
    for (int k = 0; k < g.nw; k++) {
        if (sup[k] < 1) return MTB_ERR_KERNEL;
        h_conv_info[2 * k] = sup[k];
        if (off > (size_t)0x7fffffff) return MTB_ERR_CAPACITY;
        h_conv_info[2 * k + 1] = (int)off;              // WProjectionConvFunction.cpp:253-265
        off += (size_t)g.T * g.T * sup[k] * sup[k];
    }
    if (off > table_capacity) return MTB_ERR_CAPACITY;
    if (table_elems) *table_elems = off;
    int *ci = d_conv_info ? d_conv_info : w.conv_info;
    MTB_CUDA_TRY(cudaMemcpyAsync(ci, h_conv_info, sizeof(int) * 2 * g.nw, cudaMemcpyHostToDevice, st));
    if (ci != w.conv_info)
        MTB_CUDA_TRY(cudaMemcpyAsync(w.conv_info, ci, sizeof(int) * 2 * g.nw, cudaMemcpyDeviceToDevice, st));

    // pass 2: cut-out and reorder.  When every plane fit one batch the FFT
    // output of pass 1 is still resident; otherwise each batch is recomputed.
    for (int k0 = 0; k0 < g.nw; k0 += nb) {
        int n = (g.nw - k0 < nb) ? g.nw - k0 : nb;
        if (nb < g.nw) MTB_TRY(launch_screen_fft(g, w, k0, n, st));
        dim3 grid(64, n < 65535 ? n : 65535);
        k_reorganize<<<grid, 256, 0, st>>>(w.planes, n, k0, g.ps, g.s, g.T, w.conv_info, w.divisor,
                                           (float2 *)d_table);
        MTB_LAUNCHED();
    }
    int warps = g.nw * g.T * g.T;
    k_conv_sums<<<(warps * 32 + 255) / 256, 256, 0, st>>>((const float2 *)d_table, w.conv_info, g.nw, g.T,
                                                         d_conv_sums);
    MTB_LAUNCHED();
    // the host copy of conv_info is read by the caller right away; make sure the
    // H2D above has consumed it before returning
    MTB_CUDA_TRY(cudaStreamSynchronize(st));
    return MTB_OK;
}

// ----------------------------------------------------- taper-only kernel --
// mode=normal (OnlyTaperConvFunction.cpp:29-99): the uv-plane gridding
// function of CasaGridSF.cu:107-149 -- per axis (1 - nu^2) grdsf(nu) with
// nu = d / (3 s) for offsets d < 3 s from the centre of a (S s [+1 for even s])^2
// array, zero beyond -- cut into the [oy][ox][sy][sx] table of one plane by the
// same rule as ConvFunctionReOrganize.cu:30-71, with its ConvSums.  Small
// enough to evaluate on the host in FP64.
extern "C" int mtb_taper_kernel_build(int support, int sampling, void *d_table, size_t table_capacity,
                                      int *d_conv_info, int *h_conv_info, float *d_conv_sums, size_t *table_elems,
                                      mtb_stream_t stream) {
    MTB_RANGE("mtb_taper_kernel_build");
    using namespace mtb;
    if (!d_table || !h_conv_info || !d_conv_sums || !table_elems) return MTB_ERR_NULL;
    if (support < 1 || support % 2 == 0 || support > 255 || sampling < 1 || sampling > 64) return MTB_ERR_BAD_PARAM;
    const int S = support, s = sampling, T = oversample_T(s);
    const int dim = S * s + ((s & 1) ? 0 : 1);
    const size_t n = (size_t)T * T * S * S;
    if (table_capacity < n) return MTB_ERR_CAPACITY;
    const int zero_at = 3 * s;
    auto g = [&](int d) {
        d = d < 0 ? -d : d;
        if (d >= zero_at) return 0.0;
        const double nu = (double)d / (double)zero_at;
        return (1.0 - nu * nu) * grdsf(nu);
    };
    const int cb = dim / 2 - ((S / 2) * s + s / 2);
    std::vector<float2> tab(n);
    std::vector<float> sums((size_t)T * T);
    for (int oy = 0; oy < T; oy++)
        for (int ox = 0; ox < T; ox++) {
            double sum = 0.0;
            for (int py = 0; py < S; py++)
                for (int px = 0; px < S; px++) {
                    const int yc = py * s + oy + cb, xc = px * s + ox + cb;
                    const double v = g(yc - dim / 2) * g(xc - dim / 2);
                    const size_t i = (((size_t)oy * T + ox) * S + py) * S + px;
                    tab[i] = make_float2((float)v, 0.0f);
                    sum += (double)(float)v;
                }
            sums[(size_t)oy * T + ox] = (float)sum;
        }
    cudaStream_t st = (cudaStream_t)stream;
    h_conv_info[0] = S;
    h_conv_info[1] = 0;
    MTB_CUDA_TRY(cudaMemcpyAsync(d_table, tab.data(), n * sizeof(float2), cudaMemcpyHostToDevice, st));
    MTB_CUDA_TRY(cudaMemcpyAsync(d_conv_sums, sums.data(), sums.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    if (d_conv_info) MTB_CUDA_TRY(cudaMemcpyAsync(d_conv_info, h_conv_info, 2 * sizeof(int), cudaMemcpyHostToDevice, st));
    // the host staging vectors go out of scope on return
    MTB_CUDA_TRY(cudaStreamSynchronize(st));
    *table_elems = n;
    return MTB_OK;
}
