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
//
// Host copies between the caller's (pageable) arrays and pinned memory run on
// a pool of host threads: one thread copies a few GB/s, more so into pages
// touched for the first time, while DMA from pinned memory runs at tens of
// GB/s.  Inputs are copied array by array, each array's H2D issued as soon as
// it is staged; the image comes back in pieces through two pinned buffers,
// each piece copied out while the next one is in flight.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
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
#include "mtb_internal.cuh"

namespace mtb {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Bytes of one record's inputs for P polarisations (uvw, nu/c, vis, weights, flags).
size_t record_bytes(int P) { return 3 * 4 + 4 + (size_t)P * (8 + 4 + 4); }

// Host threads that split large memcpys.  copy() returns when every piece is
// done; the calling thread copies one piece itself.
class CopyPool {
public:
    explicit CopyPool(int threads) {
        for (int i = 0; i < threads; i++) th_.emplace_back([this] { loop(); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
    }
    void copy(void *dst, const void *src, size_t bytes) {
        const size_t min_piece = (size_t)1 << 20;
        size_t pieces = std::min((size_t)th_.size() + 1, (bytes + min_piece - 1) / min_piece);
        if (pieces <= 1) {
            std::memcpy(dst, src, bytes);
            return;
        }
        const size_t step = (bytes / pieces + 63) & ~(size_t)63;
        Batch b;
        b.left = 0;
        {
            std::lock_guard<std::mutex> lk(m_);
            for (size_t off = step; off < bytes; off += step) {
                tasks_.push_back(Task{(char *)dst + off, (const char *)src + off, std::min(step, bytes - off), &b});
                b.left++;
            }
        }
        cv_.notify_all();
        std::memcpy(dst, src, std::min(step, bytes));
        std::unique_lock<std::mutex> lk(b.m);
        b.cv.wait(lk, [&] { return b.left == 0; });
    }

private:
    struct Batch {
        std::mutex m;
        std::condition_variable cv;
        int left;
    };
    struct Task {
        char *dst;
        const char *src;
        size_t n;
        Batch *b;
    };
    void loop() {
        for (;;) {
            Task t;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return stop_ || !tasks_.empty(); });
                if (tasks_.empty()) return;
                t = tasks_.front();
                tasks_.pop_front();
            }
            std::memcpy(t.dst, t.src, t.n);
            std::lock_guard<std::mutex> lk(t.b->m);
            if (--t.b->left == 0) t.b->cv.notify_all();
        }
    }
    std::vector<std::thread> th_;
    std::mutex m_;
    std::condition_variable cv_;
    std::deque<Task> tasks_;
    bool stop_ = false;
};

struct Job {
    long long ticket = 0;
    mtb_image_request req{};
    size_t bytes = 0;
    Clock::time_point t_submit, t_admit, t_done;
    bool done = false;
    std::atomic<bool> cancel{false};    // set by mtb_engine_cancel, read between chunks
    mtb_image_result res{};
};

// A running request's cancellation, seen at a chunk boundary.
struct Cancelled {};

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
                // count the table only while its entry is still listed, and
                // evict from the cold end only finished tables other than this
                // one: an entry another worker is still building holds no bytes
                // yet, and dropping it would let its bytes be added later for
                // an entry that is no longer in the list (never subtracted)
                if (std::find(lru_.begin(), lru_.end(), e) != lru_.end()) {
                    e->bytes = k->bytes();
                    used_ += e->bytes;
                }
                for (auto it = lru_.end(); used_ > cap_ && it != lru_.begin();) {
                    --it;
                    if (*it == e || (*it)->bytes == 0) continue;
                    used_ -= (*it)->bytes;
                    it = lru_.erase(it);
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
    std::unique_ptr<mtb::CopyPool> copier;
    std::vector<std::thread> workers;

    // per-slot resources of a worker thread
    struct Slot {
        cudaStream_t st = nullptr;
        unsigned char *pinned[2] = {nullptr, nullptr};   // input staging (chunk)
        unsigned char *dstage[2] = {nullptr, nullptr};
        cudaEvent_t ev[2] = {nullptr, nullptr};
        float *out[2] = {nullptr, nullptr};              // image pieces on the way back
        cudaEvent_t out_ev[2] = {nullptr, nullptr};
        mtb::ImagerBuffers bufs;
        mtb::DeviceArray<float> img;
    };
    static constexpr size_t kOutPiece = (size_t)8 << 20; // floats per image piece (32 MiB)

    void worker(int slot);
    void run(mtb::Job *j, Slot &sl);
};

namespace {

// Admission estimate: the request's grid, compensation and delta grids, image,
// and an mtb_grid workspace for its largest chunk with every plane at the
// largest support the gridders take (an upper bound before the kernel table
// exists).
int request_bytes(const mtb_engine_config &cfg, const mtb_image_request *r, size_t *out) {
    mtb_wkernel_info info;
    int s = mtb_wkernel_query(&r->geometry, &info);
    if (s != MTB_OK) return s;
    const size_t cells = (size_t)r->geometry.nx * r->geometry.ny * r->npol;
    // every plane at the largest support the gridders take (odd, at most 255)
    int S = std::min(info.support_cap, 255);
    if (S % 2 == 0) S--;
    if (S < 1) S = 1;
    std::vector<int> ci((size_t)r->geometry.wplanes * 2, 0);   // table offsets do not size the workspace
    for (int k = 0; k < r->geometry.wplanes; k++) ci[2 * k] = S;
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
    gp.exact_delta = r->exact_delta;
    gp.no_grid_lo = r->compensated ? 0 : 1;   // plain requests reserve no delta grid
    const int chunk = std::min(r->nrecords, cfg.chunk_records);
    size_t ws = 0;
    s = mtb_grid_workspace_size(&gp, ci.data(), chunk, &ws);
    if (s != MTB_OK) return s;
    mtb_finalize_params fp{r->geometry.nx, r->geometry.ny, r->npol, r->geometry.sampling, r->pol_type};
    size_t fin = 0;
    s = mtb_finalize_workspace_size(&fp, &fin);
    if (s != MTB_OK) return s;
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
    if (r->uvw_row_stride != 0 && r->uvw_row_stride < r->nrecords) return MTB_ERR_BAD_SHAPE;
    if (r->flags_u8 != 0 && r->flags_u8 != 1) return MTB_ERR_BAD_PARAM;   // whole bytes: chunks start anywhere
    return MTB_OK;
}

}  // namespace

void mtb_engine::worker(int slot) {
    (void)slot;
    cudaSetDevice(device);
    const size_t sbytes = (size_t)cfg.chunk_records * mtb::record_bytes(4);
    Slot sl;
    bool ok = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking) == cudaSuccess;
    for (int b = 0; b < 2 && ok; b++) {
        ok = cudaMallocHost((void **)&sl.pinned[b], sbytes) == cudaSuccess &&
             cudaMalloc((void **)&sl.dstage[b], sbytes) == cudaSuccess &&
             cudaEventCreateWithFlags(&sl.ev[b], cudaEventDisableTiming) == cudaSuccess &&
             cudaMallocHost((void **)&sl.out[b], kOutPiece * sizeof(float)) == cudaSuccess &&
             cudaEventCreateWithFlags(&sl.out_ev[b], cudaEventDisableTiming) == cudaSuccess;
    }
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
            run(j, sl);
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
    if (sl.st) cudaStreamSynchronize(sl.st);
    // slot buffers are released on the slot's stream before it is destroyed
    sl.bufs = mtb::ImagerBuffers();
    sl.img = mtb::DeviceArray<float>();
    if (sl.st) cudaStreamSynchronize(sl.st);
    for (int b = 0; b < 2; b++) {
        if (sl.pinned[b]) cudaFreeHost(sl.pinned[b]);
        if (sl.dstage[b]) cudaFree(sl.dstage[b]);
        if (sl.ev[b]) cudaEventDestroy(sl.ev[b]);
        if (sl.out[b]) cudaFreeHost(sl.out[b]);
        if (sl.out_ev[b]) cudaEventDestroy(sl.out_ev[b]);
    }
    if (sl.st) cudaStreamDestroy(sl.st);
}

void mtb_engine::run(mtb::Job *j, Slot &sl) {
    MTB_RANGE("mtb_engine_request");
    const mtb_image_request &r = j->req;
    const int P = r.npol, R = r.nrecords;
    cudaStream_t st = sl.st;
    try {
        bool hit = false;
        std::shared_ptr<mtb::KernelTable> k = cache->get(r.geometry, st, &hit);
        j->res.kernel_cache_hit = hit ? 1 : 0;
        mtb::Imager im(k, P, r.pol_type, r.compensated != 0, st, &sl.bufs, r.exact_delta != 0, r.flags_u8 != 0);
        const size_t flag_bytes = r.flags_u8 ? 1 : 4;
        const int chunk = cfg.chunk_records;
        int b = 0;
        for (int c0 = 0; c0 < R; c0 += chunk, b ^= 1) {
            if (j->cancel.load()) throw mtb::Cancelled();
            const int n = std::min(chunk, R - c0);
            // staging b is free once the copy issued from it two chunks ago is done
            mtb::cuda_check(cudaEventSynchronize(sl.ev[b]), "staging");
            unsigned char *h = sl.pinned[b], *d = sl.dstage[b];
            const size_t off_freq = 12 * (size_t)n, off_vis = off_freq + 4 * (size_t)n;
            const size_t off_wt = off_vis + 8 * (size_t)n * P, off_fl = off_wt + 4 * (size_t)n * P;
            // one array (or uvw row) at a time: its H2D runs while the next is staged
            auto stage = [&](size_t off, const void *src, size_t bytes) {
                copier->copy(h + off, src, bytes);
                mtb::cuda_check(cudaMemcpyAsync(d + off, h + off, bytes, cudaMemcpyHostToDevice, st), "H2D");
            };
            const size_t us = r.uvw_row_stride ? (size_t)r.uvw_row_stride : (size_t)R;
            for (int row = 0; row < 3; row++) stage((size_t)row * n * 4, r.uvw + row * us + c0, (size_t)n * 4);
            stage(off_freq, r.freq + c0, (size_t)n * 4);
            stage(off_vis, (const float2 *)r.vis + (size_t)c0 * P, (size_t)n * P * 8);
            stage(off_wt, r.weights + (size_t)c0 * P, (size_t)n * P * 4);
            stage(off_fl, (const unsigned char *)r.flags + (size_t)c0 * P * flag_bytes, (size_t)n * P * flag_bytes);
            mtb::cuda_check(cudaEventRecord(sl.ev[b], st), "event");
            im.grid((const float *)d, (const float *)(d + off_freq), d + off_vis, (const float *)(d + off_wt),
                    (const int *)(d + off_fl), n);
        }
        if (R == 0) im.grid(nullptr, nullptr, nullptr, nullptr, nullptr, 0);
        if (j->cancel.load()) throw mtb::Cancelled();
        const size_t npix = (size_t)P * r.geometry.nx * r.geometry.ny;
        mtb::ImagerBuffers::ensure(sl.img, npix, st);
        im.finalize(sl.img.data());
        // image pieces: D2H of piece q + 2 goes out once piece q has left pinned buffer q % 2
        const size_t npiece = (npix + kOutPiece - 1) / kOutPiece;
        auto d2h = [&](size_t q) {
            const size_t o = q * kOutPiece, n = std::min(kOutPiece, npix - o);
            mtb::cuda_check(cudaMemcpyAsync(sl.out[q & 1], sl.img.data() + o, n * sizeof(float),
                                            cudaMemcpyDeviceToHost, st),
                            "D2H");
            mtb::cuda_check(cudaEventRecord(sl.out_ev[q & 1], st), "event");
        };
        for (size_t q = 0; q < npiece && q < 2; q++) d2h(q);
        for (size_t q = 0; q < npiece; q++) {
            mtb::cuda_check(cudaEventSynchronize(sl.out_ev[q & 1]), "D2H");
            const size_t o = q * kOutPiece, n = std::min(kOutPiece, npix - o);
            copier->copy(r.image + o, sl.out[q & 1], n * sizeof(float));
            if (q + 2 < npiece) d2h(q + 2);
        }
        j->res.stats = im.stats();   // synchronises the stream
        j->res.status = MTB_OK;
    } catch (const mtb::Cancelled &) {
        j->res.status = MTB_ERR_CANCELLED;
        cudaStreamSynchronize(st);    // the chunks already enqueued finish before the slot is reused
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
    if (e->cfg.host_threads <= 0) {
        const int hw = (int)std::thread::hardware_concurrency();
        e->cfg.host_threads = std::max(1, std::min(8, hw > 0 ? hw / 2 : 1));
    }
    e->copier.reset(new mtb::CopyPool(e->cfg.host_threads - 1));
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

extern "C" int mtb_engine_cancel(mtb_engine *engine, long long ticket) {
    if (!engine) return MTB_ERR_NULL;
    {
        std::lock_guard<std::mutex> lk(engine->m);
        auto it = engine->jobs.find(ticket);
        if (it == engine->jobs.end()) return MTB_ERR_BAD_PARAM;
        mtb::Job *j = it->second;
        if (j->done) return MTB_OK;
        j->cancel.store(true);
        auto q = std::find(engine->queue.begin(), engine->queue.end(), j);
        if (q == engine->queue.end()) return MTB_OK;    // running: its worker stops at a chunk boundary
        engine->queue.erase(q);
        j->t_admit = j->t_done = mtb::Clock::now();
        j->res.status = MTB_ERR_CANCELLED;
        j->res.queue_ms = j->res.latency_ms = mtb::ms_between(j->t_submit, j->t_done);
        j->res.service_ms = 0.0;
        j->done = true;
    }
    engine->cv.notify_all();    // waiters of this ticket, and workers whose queue head changed
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
    engine->copier.reset();
    delete engine;
    return MTB_OK;
}
