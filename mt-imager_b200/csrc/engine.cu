// Imaging request engine: continuous batching of W-projection images on one
// GPU (include/mtb_engine.h).  Host C++ over the C ABI through the classes of
// include/mtb.hpp; no kernels of its own.
//
// Worker threads, one per slot, each drive one CUDA stream.  A worker takes
// the oldest queued request once the request's device memory fits in the
// budget left by the requests in flight, looks its w-kernels up in the shared
// cache (building them on its own stream on a miss), streams the records
// through pinned double-buffered staging in chunks of chunk_records, grids
// every chunk with mtb_grid, finalises with mtb_finalize and copies the image
// to the request's host buffer.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <exception>
#include <future>
#include <list>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "mtb.hpp"
#include "mtb_engine.h"

namespace mtb {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Bytes of one record's inputs for P polarisations (uvw, nu/c, vis, weights, flags).
size_t record_bytes(int P) { return 3 * 4 + 4 + (size_t)P * (8 + 4 + 4); }

struct Job {
    long long ticket = 0;
    mtb_image_request req{};
    size_t bytes = 0;
    Clock::time_point t_submit, t_admit, t_done;
    bool done = false;
    mtb_image_result res{};
};

// w-kernel tables by geometry, least recently used evicted beyond `cap` bytes.
// A table in use by a request stays alive (shared_ptr) after eviction.
class KernelCache {
public:
    explicit KernelCache(size_t cap) : cap_(cap) {}

    std::shared_ptr<KernelTable> get(const mtb_wkernel_params &p, cudaStream_t st, bool *hit) {
        std::shared_ptr<Entry> e;
        bool builder = false;
        {
            std::lock_guard<std::mutex> lk(m_);
            for (auto it = lru_.begin(); it != lru_.end(); ++it)
                if ((*it)->g == Geometry{p}) {
                    e = *it;
                    lru_.splice(lru_.begin(), lru_, it);
                    break;
                }
            if (!e) {
                e = std::make_shared<Entry>();
                e->g = Geometry{p};
                e->f = e->prom.get_future().share();
                lru_.push_front(e);
                builder = true;
            }
        }
        *hit = !builder;
        if (builder) {
            try {
                std::shared_ptr<KernelTable> k = KernelTable::build(p, st);
                cuda_check(cudaStreamSynchronize(st), "kernel build");
                // the table outlives this worker's use of it: free it on the
                // default stream, not on the stream of whichever slot built it
                k->release_on(0);
                e->prom.set_value(k);
                std::lock_guard<std::mutex> lk(m_);
                e->bytes = k->bytes();
                used_ += e->bytes;
                while (used_ > cap_ && lru_.size() > 1) {
                    used_ -= lru_.back()->bytes;
                    lru_.pop_back();
                }
            } catch (...) {
                e->prom.set_exception(std::current_exception());
                std::lock_guard<std::mutex> lk(m_);
                lru_.remove(e);
            }
        }
        return e->f.get();
    }

private:
    struct Entry {
        Geometry g{};
        std::promise<std::shared_ptr<KernelTable>> prom;
        std::shared_future<std::shared_ptr<KernelTable>> f;
        size_t bytes = 0;
    };
    std::mutex m_;
    std::list<std::shared_ptr<Entry>> lru_;
    size_t cap_, used_ = 0;
};

}  // namespace
}  // namespace mtb

struct mtb_engine {
    mtb_engine_config cfg{};
    int device = 0;
    size_t budget = 0, in_use = 0;
    std::mutex m;
    std::condition_variable cv;
    std::deque<mtb::Job *> queue;
    std::unordered_map<long long, mtb::Job *> jobs;
    long long next_ticket = 1;
    bool stop = false;
    std::unique_ptr<mtb::KernelCache> cache;
    std::vector<std::thread> workers;

    void worker(int slot);
    void run(mtb::Job *j, cudaStream_t st, unsigned char *const pinned[2], unsigned char *const dstage[2],
             cudaEvent_t const ev[2], mtb::ImagerBuffers &bufs, mtb::DeviceArray<float> &img);
};

namespace {

// Admission estimate: the request's grid, compensation and delta grids, image,
// and an mtb_grid workspace for its largest chunk with every plane at the
// support cap (an upper bound before the kernel table exists).
int request_bytes(const mtb_engine_config &cfg, const mtb_image_request *r, size_t *out) {
    mtb_wkernel_info info;
    int s = mtb_wkernel_query(&r->geometry, &info);
    if (s != MTB_OK) return s;
    const size_t cells = (size_t)r->geometry.nx * r->geometry.ny * r->npol;
    std::vector<int> ci((size_t)r->geometry.wplanes * 2);
    for (int k = 0; k < r->geometry.wplanes; k++) {
        ci[2 * k] = info.support_cap;
        ci[2 * k + 1] = k * info.T * info.T * info.support_cap * info.support_cap;
    }
    mtb_grid_params gp;
    std::memset(&gp, 0, sizeof(gp));
    gp.nx = r->geometry.nx;
    gp.ny = r->geometry.ny;
    gp.npol = r->npol;
    gp.sampling = r->geometry.sampling;
    gp.wplanes = r->geometry.wplanes;
    gp.u_increment = info.u_increment;
    gp.v_increment = info.v_increment;
    gp.w_sq_increment = info.w_sq_increment;
    const int chunk = std::min(r->nrecords, cfg.chunk_records);
    size_t ws = 0;
    s = mtb_grid_workspace_size(&gp, ci.data(), chunk, &ws);
    if (s != MTB_OK) return s;
    mtb_finalize_params fp{r->geometry.nx, r->geometry.ny, r->npol, r->geometry.sampling, r->pol_type};
    size_t fin = 0;
    s = mtb_finalize_workspace_size(&fp, &fin);
    if (s != MTB_OK) return s;
    gp.exact_delta = r->exact_delta;
    *out = cells * 8 * (r->compensated ? 2 : 1) + cells * 4 + ws + fin + (1 << 20);
    return MTB_OK;
}

int check_request(const mtb_image_request *r) {
    if (!r) return MTB_ERR_NULL;
    if (r->npol != 1 && r->npol != 2 && r->npol != 4) return MTB_ERR_BAD_SHAPE;
    if (r->nrecords < 0) return MTB_ERR_BAD_SHAPE;
    if (!r->image) return MTB_ERR_NULL;
    if (r->nrecords > 0 && (!r->uvw || !r->freq || !r->vis || !r->weights || !r->flags)) return MTB_ERR_NULL;
    if (r->pol_type != MTB_POL_LINEAR && r->pol_type != MTB_POL_CIRCULAR) return MTB_ERR_BAD_PARAM;
    return MTB_OK;
}

}  // namespace

void mtb_engine::worker(int slot) {
    (void)slot;
    cudaSetDevice(device);
    cudaStream_t st = nullptr;
    unsigned char *pinned[2] = {nullptr, nullptr}, *dstage[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    const size_t sbytes = (size_t)cfg.chunk_records * mtb::record_bytes(4);
    bool ok = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
    for (int b = 0; b < 2 && ok; b++) {
        ok = cudaMallocHost((void **)&pinned[b], sbytes) == cudaSuccess &&
             cudaMalloc((void **)&dstage[b], sbytes) == cudaSuccess &&
             cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming) == cudaSuccess;
    }
    {
    // device buffers of this slot, reused (grow-only) by every request it runs
    mtb::ImagerBuffers bufs;
    mtb::DeviceArray<float> img;
    for (;;) {
        mtb::Job *j = nullptr;
        {
            std::unique_lock<std::mutex> lk(m);
            cv.wait(lk, [&] { return (stop && queue.empty()) || (!queue.empty() && queue.front()->bytes + in_use <= budget); });
            if (queue.empty()) break;
            j = queue.front();
            queue.pop_front();
            in_use += j->bytes;
            j->t_admit = mtb::Clock::now();
        }
        if (ok) {
            run(j, st, pinned, dstage, ev, bufs, img);
        } else {
            j->res.status = MTB_ERR_CUDA;
        }
        {
            std::lock_guard<std::mutex> lk(m);
            in_use -= j->bytes;
            j->t_done = mtb::Clock::now();
            j->res.queue_ms = mtb::ms_between(j->t_submit, j->t_admit);
            j->res.service_ms = mtb::ms_between(j->t_admit, j->t_done);
            j->res.latency_ms = mtb::ms_between(j->t_submit, j->t_done);
            j->done = true;
        }
        cv.notify_all();
    }
    if (st) cudaStreamSynchronize(st);
    }   // slot buffers released on the slot's stream
    for (int b = 0; b < 2; b++) {
        if (pinned[b]) cudaFreeHost(pinned[b]);
        if (dstage[b]) cudaFree(dstage[b]);
        if (ev[b]) cudaEventDestroy(ev[b]);
    }
    if (st) cudaStreamDestroy(st);
}

void mtb_engine::run(mtb::Job *j, cudaStream_t st, unsigned char *const pinned[2], unsigned char *const dstage[2],
                     cudaEvent_t const ev[2], mtb::ImagerBuffers &bufs, mtb::DeviceArray<float> &img) {
    const mtb_image_request &r = j->req;
    const int P = r.npol, R = r.nrecords;
    try {
        bool hit = false;
        std::shared_ptr<mtb::KernelTable> k = cache->get(r.geometry, st, &hit);
        j->res.kernel_cache_hit = hit ? 1 : 0;
        mtb::Imager im(k, P, r.pol_type, r.compensated != 0, st, &bufs, r.exact_delta != 0);
        const int chunk = cfg.chunk_records;
        int b = 0;
        for (int c0 = 0; c0 < R; c0 += chunk, b ^= 1) {
            const int n = std::min(chunk, R - c0);
            // staging b is free once the copy issued from it two chunks ago is done
            mtb::cuda_check(cudaEventSynchronize(ev[b]), "staging");
            unsigned char *h = pinned[b];
            float *h_uvw = (float *)h;
            float *h_freq = h_uvw + 3 * (size_t)n;
            float2 *h_vis = (float2 *)(h_freq + n);
            float *h_wt = (float *)(h_vis + (size_t)n * P);
            int *h_fl = (int *)(h_wt + (size_t)n * P);
            for (int row = 0; row < 3; row++)
                std::memcpy(h_uvw + (size_t)row * n, r.uvw + (size_t)row * R + c0, (size_t)n * 4);
            std::memcpy(h_freq, r.freq + c0, (size_t)n * 4);
            std::memcpy(h_vis, (const float2 *)r.vis + (size_t)c0 * P, (size_t)n * P * 8);
            std::memcpy(h_wt, r.weights + (size_t)c0 * P, (size_t)n * P * 4);
            std::memcpy(h_fl, r.flags + (size_t)c0 * P, (size_t)n * P * 4);
            const size_t bytes = (size_t)n * mtb::record_bytes(P);
            unsigned char *d = dstage[b];
            mtb::cuda_check(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st), "H2D");
            mtb::cuda_check(cudaEventRecord(ev[b], st), "event");
            const size_t off_freq = 12 * (size_t)n, off_vis = off_freq + 4 * (size_t)n;
            const size_t off_wt = off_vis + 8 * (size_t)n * P, off_fl = off_wt + 4 * (size_t)n * P;
            im.grid((const float *)d, (const float *)(d + off_freq), d + off_vis, (const float *)(d + off_wt),
                    (const int *)(d + off_fl), n);
        }
        if (R == 0) im.grid(nullptr, nullptr, nullptr, nullptr, nullptr, 0);
        const size_t npix = (size_t)P * r.geometry.nx * r.geometry.ny;
        mtb::ImagerBuffers::ensure(img, npix, st);
        im.finalize(img.data());
        mtb::cuda_check(cudaMemcpyAsync(r.image, img.data(), npix * sizeof(float), cudaMemcpyDeviceToHost, st),
                        "D2H");
        j->res.stats = im.stats();   // synchronises the stream
        j->res.status = MTB_OK;
    } catch (const mtb::Error &e) {
        j->res.status = e.status;
        cudaStreamSynchronize(st);
    } catch (const std::exception &) {
        j->res.status = MTB_ERR_CUDA;
        cudaStreamSynchronize(st);
    }
}

extern "C" int mtb_engine_create(const mtb_engine_config *cfg, mtb_engine **engine) {
    if (!engine) return MTB_ERR_NULL;
    *engine = nullptr;
    std::unique_ptr<mtb_engine> e(new mtb_engine());
    if (cfg) e->cfg = *cfg;
    if (e->cfg.slots <= 0) e->cfg.slots = 4;
    if (e->cfg.chunk_records <= 0) e->cfg.chunk_records = 1 << 22;
    if (e->cfg.kernel_cache_bytes == 0) e->cfg.kernel_cache_bytes = (size_t)4 << 30;
    if (e->cfg.slots > 64) return MTB_ERR_BAD_PARAM;
    if (cudaGetDevice(&e->device) != cudaSuccess) return MTB_ERR_CUDA;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return MTB_ERR_CUDA;
    const size_t staging = (size_t)e->cfg.slots * 2 * (size_t)e->cfg.chunk_records * mtb::record_bytes(4);
    size_t budget = e->cfg.hbm_budget_bytes ? e->cfg.hbm_budget_bytes : free_b / 10 * 7;
    if (budget <= staging + e->cfg.kernel_cache_bytes) return MTB_ERR_CAPACITY;
    e->budget = budget - staging - e->cfg.kernel_cache_bytes;
    // keep memory freed by finished requests in the device's stream-ordered
    // pool instead of returning it to the driver at every synchronisation, so
    // the next request's cudaMallocAsync is served from the pool
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, e->device) == cudaSuccess) {
        uint64_t keep = (uint64_t)budget;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    e->cache.reset(new mtb::KernelCache(e->cfg.kernel_cache_bytes));
    for (int s = 0; s < e->cfg.slots; s++) e->workers.emplace_back(&mtb_engine::worker, e.get(), s);
    *engine = e.release();
    return MTB_OK;
}

extern "C" int mtb_engine_request_bytes(const mtb_engine *engine, const mtb_image_request *req, size_t *bytes) {
    if (!engine || !bytes) return MTB_ERR_NULL;
    int s = check_request(req);
    if (s != MTB_OK) return s;
    return request_bytes(engine->cfg, req, bytes);
}

extern "C" int mtb_engine_submit(mtb_engine *engine, const mtb_image_request *req, long long *ticket) {
    if (!engine || !ticket) return MTB_ERR_NULL;
    int s = check_request(req);
    if (s != MTB_OK) return s;
    size_t bytes = 0;
    s = request_bytes(engine->cfg, req, &bytes);
    if (s != MTB_OK) return s;
    if (bytes > engine->budget) return MTB_ERR_CAPACITY;
    mtb::Job *j = new mtb::Job();
    j->req = *req;
    j->bytes = bytes;
    j->t_submit = mtb::Clock::now();
    {
        std::lock_guard<std::mutex> lk(engine->m);
        if (engine->stop) {
            delete j;
            return MTB_ERR_BAD_PARAM;
        }
        j->ticket = engine->next_ticket++;
        engine->jobs[j->ticket] = j;
        engine->queue.push_back(j);
        *ticket = j->ticket;
    }
    engine->cv.notify_all();
    return MTB_OK;
}

extern "C" int mtb_engine_wait(mtb_engine *engine, long long ticket, mtb_image_result *result) {
    if (!engine || !result) return MTB_ERR_NULL;
    std::unique_lock<std::mutex> lk(engine->m);
    auto it = engine->jobs.find(ticket);
    if (it == engine->jobs.end()) return MTB_ERR_BAD_PARAM;
    mtb::Job *j = it->second;
    engine->cv.wait(lk, [&] { return j->done; });
    *result = j->res;
    engine->jobs.erase(it);
    delete j;
    return MTB_OK;
}

extern "C" int mtb_engine_destroy(mtb_engine *engine) {
    if (!engine) return MTB_ERR_NULL;
    {
        std::lock_guard<std::mutex> lk(engine->m);
        engine->stop = true;
    }
    engine->cv.notify_all();
    for (auto &t : engine->workers) t.join();
    for (auto &kv : engine->jobs) delete kv.second;
    engine->cache.reset();
    delete engine;
    return MTB_OK;
}
