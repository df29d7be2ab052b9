// cuFFT plan cache.  The reference builds and destroys a plan on every
// submit and runs it on stream 0 behind two stream synchronisations
// (code/gafw/Implimentation/StandardOperators/MultiFFT2D.cpp:86-115,
// IFFT2D.cpp:86-115).  Here a plan is made once per (device, type, shape,
// batch) with auto-allocation off; every execution binds the caller's
// workspace as the work area and runs on the caller's stream.
#include "fft_plans.cuh"

#include <map>
#include <mutex>
#include <tuple>

namespace mtb {

namespace {
struct Entry {
    cufftHandle plan;
    size_t work;
};
std::mutex g_mu;
std::map<std::tuple<int, int, int, int, int>, Entry> g_plans;
}  // namespace

int fft_plan(cufftType type, int ny, int nx, int batch, cufftHandle *plan, size_t *work) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MTB_ERR_CUDA;
    auto key = std::make_tuple(dev, (int)type, ny, nx, batch);
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_plans.find(key);
    if (it != g_plans.end()) {
        *plan = it->second.plan;
        *work = it->second.work;
        return MTB_OK;
    }
    cufftHandle h;
    if (cufftCreate(&h) != CUFFT_SUCCESS) return MTB_ERR_CUFFT;
    if (cufftSetAutoAllocation(h, 0) != CUFFT_SUCCESS) { cufftDestroy(h); return MTB_ERR_CUFFT; }
    int n[2] = {ny, nx};
    size_t ws = 0;
    if (cufftMakePlanMany(h, 2, n, nullptr, 1, ny * nx, nullptr, 1, ny * nx, type, batch, &ws) != CUFFT_SUCCESS) {
        cufftDestroy(h);
        return MTB_ERR_CUFFT;
    }
    g_plans[key] = Entry{h, ws};
    *plan = h;
    *work = ws;
    return MTB_OK;
}

int fft_exec(cufftType type, int ny, int nx, int batch, void *in, void *out, int direction,
             void *work, size_t work_bytes, cudaStream_t stream) {
    cufftHandle h;
    size_t need = 0;
    int st = fft_plan(type, ny, nx, batch, &h, &need);
    if (st != MTB_OK) return st;
    if (need > work_bytes) return MTB_ERR_WORKSPACE;
    // a cached plan is shared; binding stream and work area and executing
    // happen under the lock so two host threads cannot interleave them
    std::lock_guard<std::mutex> lk(g_mu);
    if (cufftSetStream(h, stream) != CUFFT_SUCCESS) return MTB_ERR_CUFFT;
    if (need && cufftSetWorkArea(h, work) != CUFFT_SUCCESS) return MTB_ERR_CUFFT;
    cufftResult r;
    if (type == CUFFT_Z2Z)
        r = cufftExecZ2Z(h, (cufftDoubleComplex *)in, (cufftDoubleComplex *)out, direction);
    else
        r = cufftExecC2C(h, (cufftComplex *)in, (cufftComplex *)out, direction);
    return (r == CUFFT_SUCCESS) ? MTB_OK : MTB_ERR_CUFFT;
}

void fft_release_all() {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto &kv : g_plans) cufftDestroy(kv.second.plan);
    g_plans.clear();
}

}  // namespace mtb
