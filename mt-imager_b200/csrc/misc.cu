// Status strings, version and cache release of the C ABI.
#include "fft_plans.cuh"
#include "mtb_internal.cuh"

extern "C" const char *mtb_status_string(int status) {
    switch (status) {
        case MTB_OK: return "ok";
        case MTB_ERR_BAD_PARAM: return "invalid parameter";
        case MTB_ERR_BAD_SHAPE: return "unsupported array shape or polarisation count";
        case MTB_ERR_WORKSPACE: return "workspace too small";
        case MTB_ERR_CAPACITY: return "output buffer too small";
        case MTB_ERR_CUDA: return "CUDA error";
        case MTB_ERR_CUFFT: return "cuFFT error";
        case MTB_ERR_KERNEL: return "w-kernel generation failed (origin not real or no support)";
        case MTB_ERR_NULL: return "required pointer is NULL";
        default: return "unknown status";
    }
}

extern "C" int mtb_version(void) { return 100; }

extern "C" void mtb_release_caches(void) { mtb::fft_release_all(); }
