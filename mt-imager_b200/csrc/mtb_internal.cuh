// Internal helpers shared by the sm_100a kernels of the W-projection path.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <cstddef>
#include <cstdint>
#include "mtb.h"

namespace mtb {

// NVTX range over one entry point's host scope, named after the entry point:
// profilers attribute the kernels it launches to it (ncu --nvtx
// --nvtx-include "mtb_grid/").  Header-only NVTX: with no tool attached a
// push and a pop cost a few nanoseconds.
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};
#define MTB_RANGE(name) ::mtb::Range mtb_range_scope_(name)

#define MTB_CUDA_TRY(expr)                                   \
    do {                                                     \
        cudaError_t _e = (expr);                             \
        if (_e != cudaSuccess) return MTB_ERR_CUDA;          \
    } while (0)

// every launch of this library's own kernels goes through here so the
// process-wide launch count stays exact
void count_launch();
#define MTB_LAUNCHED()                                       \
    do {                                                     \
        ::mtb::count_launch();                               \
        cudaError_t _e = cudaGetLastError();                 \
        if (_e != cudaSuccess) return MTB_ERR_CUDA;          \
    } while (0)

#define MTB_TRY(expr)                                        \
    do {                                                     \
        int _s = (expr);                                     \
        if (_s != MTB_OK) return _s;                         \
    } while (0)

// Bump allocator over a caller-owned workspace.  Every carve is 256-byte
// aligned so any vector or TMA access into it is aligned.
struct Arena {
    char *base;
    size_t size;
    size_t used;
    explicit Arena(void *b = nullptr, size_t s = 0) : base((char *)b), size(s), used(0) {}
    template <class T>
    T *take(size_t n) {
        size_t off = (used + 255) & ~(size_t)255;
        used = off + n * sizeof(T);
        if (!base) return nullptr;          // sizing pass
        if (used > size) return nullptr;
        return (T *)(base + off);
    }
    bool ok() const { return used <= size; }
};

// OriginToCorner1D / OriginToCentre1D (mt-imager/lib/operators/common.hcu:107-136)
__host__ __device__ inline int origin_to_corner(int loc, int dim) {
    if (dim & 1) return (loc < dim / 2) ? loc + dim / 2 + 1 : loc - dim / 2;
    return (loc < dim / 2) ? loc + dim / 2 : loc - dim / 2;
}
__host__ __device__ inline int origin_to_centre(int loc, int dim) {
    if (dim & 1) return (loc <= dim / 2) ? loc + dim / 2 : loc - dim / 2 - 1;
    return (loc < dim / 2) ? loc + dim / 2 : loc - dim / 2;
}
// inverse of origin_to_centre: the unshifted index that lands on `c`
__host__ __device__ inline int centre_to_origin(int c, int dim) {
    if (dim & 1) return (c >= dim / 2) ? c - dim / 2 : c + dim / 2 + 1;
    return (c >= dim / 2) ? c - dim / 2 : c + dim / 2;
}

// Schwab's rational approximation of the M=6, alpha=1 spheroidal function
// (casacore grdsf; mt-imager/lib/operators/CasaGridSF.cu:41-85), in FP64.
__host__ __device__ inline double grdsf(double nu) {
    const double P0[5] = {8.203343e-2, -3.644705e-1, 6.278660e-1, -5.335581e-1, 2.312756e-1};
    const double P1[5] = {4.028559e-3, -3.697768e-2, 1.021332e-1, -1.201436e-1, 6.412774e-2};
    const double Q0[3] = {1.0, 8.212018e-1, 2.078043e-1};
    const double Q1[3] = {1.0, 9.599102e-1, 2.918724e-1};
    const bool part = !(nu < 0.75);
    const double *P = part ? P1 : P0;
    const double *Q = part ? Q1 : Q0;
    double d = nu * nu - (part ? 1.0 : 0.5625);
    double top = P[0], bot = Q[0], dk = 1.0;
    for (int k = 1; k < 5; k++) { dk *= d; top += P[k] * dk; }
    dk = 1.0;
    for (int k = 1; k < 3; k++) { dk *= d; bot += Q[k] * dk; }
    return (bot != 0.0) ? top / bot : 0.0;
}

inline int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

inline int oversample_T(int s) { return (s & 1) ? s : s + 1; }

}  // namespace mtb
