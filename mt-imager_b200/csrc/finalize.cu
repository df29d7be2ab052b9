// Image finalisation for sm_100a: ImageFinalizer
// (code/mt-imager/lib/components/ImageFinalizer.cpp:31-44).
//
//   k_pre_ifft     PreIFFTUVCorrection (PreIFFTUVCorrection.cu:28-90): grid
//                  [v][u][pol] -> planes [pol][v][u] with the origin moved to
//                  the corner.  The two-float grid (hi + lo) becomes one FP64
//                  value, exactly.
//   cuFFT Z2Z      IFFT2D INVERSE, unnormalised (IFFT2D.cpp:86-111), all
//                  polarisation planes in one batched plan on the caller's
//                  stream.  FP64: the taper correction below divides by
//                  grdsf(nu)^2, about 1.6e-5 at the image corners, so a float
//                  FFT's rounding would be amplified ~6e4x there.
//   k_stokes       ZeroToCentre2DShift + StokesConverter (PostIFFTStokesConverter.cu:
//                  42-180, including the m-axis flip of :172) + casagridsf taper
//                  correction (CasaGridSF.cu:174-199) + SincCorrector
//                  (SincCorrector.cu:29-58) fused into one pass in FP64; the
//                  two corrections are separable and come from per-axis factor
//                  tables.  Output float (the reference's FinalImage type).
#include "fft_plans.cuh"
#include "mtb_internal.cuh"

namespace mtb {

__global__ void k_pre_ifft(const float2 *__restrict__ grid, const float2 *__restrict__ lo, double2 *__restrict__ out,
                           int nx, int ny, int P) {
    const size_t plane = (size_t)nx * ny;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < plane * P;
         i += (size_t)gridDim.x * blockDim.x) {
        // i enumerates input cells in [y][x][p] order: coalesced reads
        int p = (int)(i % P);
        size_t c = i / P;
        int y = (int)(c / nx), x = (int)(c - (size_t)y * nx);
        float2 h = grid[i];
        double2 v = make_double2((double)h.x, (double)h.y);
        if (lo) {
            float2 e = lo[i];
            v.x += (double)e.x;
            v.y += (double)e.y;
        }
        out[(size_t)p * plane + (size_t)origin_to_corner(y, ny) * nx + origin_to_corner(x, nx)] = v;
    }
}

// f[j] = invsinc((j - n/2)/(n*s)) / grdsf(|j - n/2| / (n/2)) per axis
__global__ void k_axis_factors(double *fx, int nx, double *fy, int ny, int s) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = (i < nx) ? nx : ny;
    double *f = (i < nx) ? fx : fy;
    int j = (i < nx) ? i : i - nx;
    if (i >= nx + ny) return;
    double nu = fabs((double)(j - n / 2) / (double)(n / 2));
    double x = (double)(j - n / 2) / ((double)n * (double)s);
    double inv = (x == 0.0) ? 1.0 : (M_PI * x) / sin(M_PI * x);
    f[j] = inv / grdsf(nu);
}

// One output pixel (all Stokes planes) per thread.  Output row j holds the
// shifted row ny-1-j; shifted (y, x) reads unshifted (centre_to_origin(y),
// centre_to_origin(x)) of the FFT output.
template <int P, int CIRC>
__global__ void k_stokes(const double2 *__restrict__ img, const float *__restrict__ norm,
                         const double *__restrict__ fx, const double *__restrict__ fy, float *__restrict__ out,
                         int nx, int ny) {
    const size_t plane = (size_t)nx * ny;
    double nrm[P];
#pragma unroll
    for (int p = 0; p < P; p++) nrm[p] = (double)norm[p];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < plane; i += (size_t)gridDim.x * blockDim.x) {
        int j = (int)(i / nx), x = (int)(i - (size_t)j * nx);
        int y = ny - 1 - j;
        size_t src = (size_t)centre_to_origin(y, ny) * nx + centre_to_origin(x, nx);
        double2 d[P];
#pragma unroll
        for (int p = 0; p < P; p++) {
            d[p] = img[(size_t)p * plane + src];
            d[p].x /= nrm[p];
            d[p].y /= nrm[p];
        }
        double st[P];
        if (P == 4 && !CIRC) {
            st[0] = (d[0].x + d[3].x) * 0.5;
            st[1] = (d[0].x - d[3].x) * 0.5;
            st[2] = (d[1].x + d[2].x) * 0.5;
            st[3] = (d[1].y - d[2].y) * 0.5;
        } else if (P == 4) {
            st[0] = (d[0].x + d[3].x) * 0.5;
            st[1] = (d[1].x + d[2].x) * 0.5;
            st[2] = (d[2].y - d[1].y) * 0.5;
            st[3] = (d[0].x - d[3].x) * 0.5;
        } else if (P == 2) {
            st[0] = (d[0].x + d[1].x) * 0.5;
            st[P - 1] = (d[0].x - d[1].x) * 0.5;
        } else {
            st[0] = d[0].x;
        }
        double f = fy[j] * fx[x];
#pragma unroll
        for (int p = 0; p < P; p++) out[(size_t)p * plane + i] = (float)(st[p] * f);
    }
}

struct FSpace {
    double2 *planes;
    double *fx, *fy;
    void *work;
    size_t work_bytes;
};

// The FP64 planes come from the workspace, or are the caller's (external_planes).
static int carve_fin(const mtb_finalize_params *p, void *ws, size_t bytes, FSpace *f, size_t *need) {
    cufftHandle h;
    size_t fw = 0;
    MTB_TRY(fft_plan(CUFFT_Z2Z, p->ny, p->nx, p->npol, &h, &fw));
    Arena A(ws, bytes);
    if (p->external_planes) f->planes = (double2 *)p->d_planes;
    else f->planes = A.take<double2>((size_t)p->nx * p->ny * p->npol);
    f->fx = A.take<double>(p->nx);
    f->fy = A.take<double>(p->ny);
    f->work = A.take<char>(fw ? fw : 1);
    f->work_bytes = fw;
    *need = A.used;
    return MTB_OK;
}

static int check_fin(const mtb_finalize_params *p) {
    if (!p) return MTB_ERR_NULL;
    if (p->npol != 1 && p->npol != 2 && p->npol != 4) return MTB_ERR_BAD_SHAPE;
    if (p->nx < 2 || p->ny < 2 || p->sampling < 1) return MTB_ERR_BAD_PARAM;
    if (p->pol_type != MTB_POL_LINEAR && p->pol_type != MTB_POL_CIRCULAR) return MTB_ERR_BAD_PARAM;
    if ((size_t)p->nx * p->ny > ((size_t)1 << 31)) return MTB_ERR_BAD_SHAPE;
    return MTB_OK;
}

}  // namespace mtb

using namespace mtb;

extern "C" int mtb_finalize_workspace_size(const mtb_finalize_params *p, size_t *bytes) {
    if (!bytes) return MTB_ERR_NULL;
    MTB_TRY(check_fin(p));
    FSpace f;
    return carve_fin(p, nullptr, 0, &f, bytes);
}

extern "C" int mtb_finalize_planes_bytes(const mtb_finalize_params *p, size_t *bytes) {
    if (!bytes) return MTB_ERR_NULL;
    MTB_TRY(check_fin(p));
    *bytes = (size_t)p->nx * p->ny * p->npol * sizeof(double2);
    return MTB_OK;
}

extern "C" int mtb_finalize(const mtb_finalize_params *p, const void *d_grid, const void *d_grid_lo,
                            const float *d_normalizer, float *d_image, void *d_workspace, size_t workspace_bytes,
                            mtb_stream_t stream) {
    MTB_RANGE("mtb_finalize");
    MTB_TRY(check_fin(p));
    if (!d_grid || !d_normalizer || !d_image || !d_workspace) return MTB_ERR_NULL;
    if (p->external_planes && !p->d_planes) return MTB_ERR_NULL;
    if (p->external_planes && (uintptr_t)p->d_planes % 256) return MTB_ERR_BAD_PARAM;
    cudaStream_t st = (cudaStream_t)stream;
    FSpace f;
    size_t need = 0;
    MTB_TRY(carve_fin(p, d_workspace, workspace_bytes, &f, &need));
    if (need > workspace_bytes) return MTB_ERR_WORKSPACE;
    const int nx = p->nx, ny = p->ny, P = p->npol;
    size_t cells = (size_t)nx * ny * P;
    int blocks = (int)std::min<size_t>((cells + 255) / 256, (size_t)sm_count() * 16);
    k_pre_ifft<<<blocks, 256, 0, st>>>((const float2 *)d_grid, (const float2 *)d_grid_lo, f.planes, nx, ny, P);
    MTB_LAUNCHED();
    MTB_TRY(fft_exec(CUFFT_Z2Z, ny, nx, P, f.planes, f.planes, CUFFT_INVERSE, f.work, f.work_bytes, st));
    k_axis_factors<<<(nx + ny + 255) / 256, 256, 0, st>>>(f.fx, nx, f.fy, ny, p->sampling);
    MTB_LAUNCHED();
    size_t px = (size_t)nx * ny;
    blocks = (int)std::min<size_t>((px + 255) / 256, (size_t)sm_count() * 16);
    bool circ = p->pol_type == MTB_POL_CIRCULAR;
    if (P == 4) {
        if (circ) k_stokes<4, 1><<<blocks, 256, 0, st>>>(f.planes, d_normalizer, f.fx, f.fy, d_image, nx, ny);
        else k_stokes<4, 0><<<blocks, 256, 0, st>>>(f.planes, d_normalizer, f.fx, f.fy, d_image, nx, ny);
    } else if (P == 2) {
        k_stokes<2, 0><<<blocks, 256, 0, st>>>(f.planes, d_normalizer, f.fx, f.fy, d_image, nx, ny);
    } else {
        k_stokes<1, 0><<<blocks, 256, 0, st>>>(f.planes, d_normalizer, f.fx, f.fy, d_image, nx, ny);
    }
    MTB_LAUNCHED();
    return MTB_OK;
}
