/*
 * mtb.hpp -- C++ host API over the C ABI of mtb.h.
 *
 * The classes mirror mt-imager's imaging modules on one GPU stream:
 *   mtb::KernelTable   WProjectionConvFunction (the w-kernel table, convInfo and
 *                      ConvSums of one imaging geometry;
 *                      code/mt-imager/lib/components/ConvolutionFunctionsGenerator/
 *                      WProjectionConvFunction.cpp:186-291)
 *   mtb::Imager        WImager + ImageFinalizer: a resident grid (two-float when
 *                      compensated) and normaliser that chunks are gridded into,
 *                      then the Stokes image (WImager.cpp:167-290,
 *                      ImageFinalizer.cpp:31-65)
 *   mtb::FrequencyConverter
 *                      FrequencyConverter: nu/c per record and channel converted
 *                      TOPO -> LSRK from the TIME column
 *                      (VisibilityManager/FrequencyConverter.cpp:112-140)
 * Unlike the C ABI, these classes own their device memory: allocations are
 * stream-ordered (cudaMallocAsync / cudaFreeAsync on the object's stream), and
 * every call only enqueues work on that stream.  Errors throw mtb::Error.
 *
 * Header-only; link with libmtb.so and the CUDA runtime.
 */
#ifndef MTB_HPP
#define MTB_HPP

#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "mtb.h"

namespace mtb {

class Error : public std::runtime_error {
public:
    Error(int status, const std::string &where)
        : std::runtime_error(where + ": " + mtb_status_string(status)), status(status) {}
    int status;
};

inline void check(int status, const char *where) {
    if (status != MTB_OK) throw Error(status, where);
}
inline void cuda_check(cudaError_t e, const char *where) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e));
}

// Stream-ordered device array (move-only).
template <class T>
class DeviceArray {
public:
    DeviceArray() = default;
    DeviceArray(size_t n, cudaStream_t s) : n_(n), s_(s) {
        if (n) cuda_check(cudaMallocAsync((void **)&p_, n * sizeof(T), s), "cudaMallocAsync");
    }
    DeviceArray(const DeviceArray &) = delete;
    DeviceArray &operator=(const DeviceArray &) = delete;
    DeviceArray(DeviceArray &&o) noexcept { swap(o); }
    DeviceArray &operator=(DeviceArray &&o) noexcept {
        DeviceArray t(std::move(o));
        swap(t);
        return *this;
    }
    ~DeviceArray() {
        if (p_) cudaFreeAsync(p_, s_);
    }
    T *data() const { return p_; }
    size_t size() const { return n_; }
    // stream the memory is released on
    void release_on(cudaStream_t s) { s_ = s; }
    size_t bytes() const { return n_ * sizeof(T); }

private:
    void swap(DeviceArray &o) noexcept {
        std::swap(p_, o.p_);
        std::swap(n_, o.n_);
        std::swap(s_, o.s_);
    }
    T *p_ = nullptr;
    size_t n_ = 0;
    cudaStream_t s_ = 0;
};

// Imaging geometry: the parameters the w-kernel table depends on.
struct Geometry {
    mtb_wkernel_params p;
    bool operator==(const Geometry &o) const { return std::memcmp(&p, &o.p, sizeof(p)) == 0; }
};

class KernelTable {
public:
    // Builds every w-plane kernel on `stream` (synchronises it once).
    static std::shared_ptr<KernelTable> build(const mtb_wkernel_params &params, cudaStream_t stream) {
        std::shared_ptr<KernelTable> k(new KernelTable());
        k->params = params;
        check(mtb_wkernel_query(&params, &k->info), "mtb_wkernel_query");
        DeviceArray<unsigned char> ws(k->info.workspace_bytes ? k->info.workspace_bytes : 1, stream);
        DeviceArray<float2> full(k->info.table_capacity ? k->info.table_capacity : 1, stream);
        k->conv_info = DeviceArray<int>((size_t)params.wplanes * 2, stream);
        k->h_conv_info.assign((size_t)params.wplanes * 2, 0);
        k->conv_sums = DeviceArray<float>((size_t)params.wplanes * k->info.T * k->info.T, stream);
        size_t n = 0;
        check(mtb_wkernel_build(&params, ws.data(), k->info.workspace_bytes, full.data(), k->info.table_capacity,
                                k->conv_info.data(), k->h_conv_info.data(), k->conv_sums.data(), &n,
                                (mtb_stream_t)stream),
              "mtb_wkernel_build");
        k->elems = n;
        k->table = DeviceArray<float2>(n ? n : 1, stream);
        cuda_check(cudaMemcpyAsync(k->table.data(), full.data(), n * sizeof(float2), cudaMemcpyDeviceToDevice,
                                   stream),
                   "table copy");
        return k;
    }
    size_t bytes() const { return table.bytes() + conv_info.bytes() + conv_sums.bytes(); }
    void release_on(cudaStream_t s) {
        table.release_on(s);
        conv_info.release_on(s);
        conv_sums.release_on(s);
    }

    mtb_wkernel_params params{};
    mtb_wkernel_info info{};
    DeviceArray<float2> table;
    DeviceArray<int> conv_info;
    std::vector<int> h_conv_info;
    DeviceArray<float> conv_sums;
    size_t elems = 0;

private:
    KernelTable() = default;
};

// Device buffers an Imager works in.  Grow-only: a Buffers object kept across
// images (one per stream in a server) is reused without new allocations once
// it has seen the largest image.
struct ImagerBuffers {
    DeviceArray<float2> grid, lo;
    DeviceArray<float> norm;
    DeviceArray<mtb_grid_stats> stats;
    DeviceArray<unsigned char> ws, fin;

    template <class T>
    static void ensure(DeviceArray<T> &a, size_t n, cudaStream_t s) {
        if (a.size() < n) a = DeviceArray<T>(n, s);
    }
};

class Imager {
public:
    // buffers: kept by the caller and reused across images, or nullptr to let
    // the imager own its own
    // flags_u8: grid() receives one byte per flag instead of int32
    Imager(std::shared_ptr<const KernelTable> k, int npol, int pol_type, bool compensated, cudaStream_t stream,
           ImagerBuffers *buffers = nullptr, bool exact_delta = false, bool flags_u8 = false)
        : k_(std::move(k)), npol_(npol), pol_type_(pol_type), compensated_(compensated), exact_delta_(exact_delta),
          flags_u8_(flags_u8), s_(stream) {
        if (!buffers) {
            own_.reset(new ImagerBuffers());
            buffers = own_.get();
        }
        b_ = buffers;
        const size_t cells = (size_t)k_->params.nx * k_->params.ny * npol;
        ImagerBuffers::ensure(b_->grid, cells, s_);
        if (compensated) ImagerBuffers::ensure(b_->lo, cells, s_);
        ImagerBuffers::ensure(b_->norm, (size_t)npol, s_);
        ImagerBuffers::ensure(b_->stats, 1, s_);
        reset();
    }
    const KernelTable &kernels() const { return *k_; }
    int npol() const { return npol_; }
    cudaStream_t stream() const { return s_; }

    // The next grid() call starts a new image (zero grid, normaliser, statistics).
    void reset() { fresh_ = true; }

    mtb_grid_params grid_params() const {
        mtb_grid_params gp;
        std::memset(&gp, 0, sizeof(gp));
        gp.nx = k_->params.nx;
        gp.ny = k_->params.ny;
        gp.npol = npol_;
        gp.sampling = k_->params.sampling;
        gp.wplanes = k_->params.wplanes;
        gp.u_increment = k_->info.u_increment;
        gp.v_increment = k_->info.v_increment;
        gp.w_sq_increment = k_->info.w_sq_increment;
        gp.initialize_output = fresh_ ? 1 : 0;
        gp.exact_delta = exact_delta_ ? 1 : 0;
        gp.flags_u8 = flags_u8_ ? 1 : 0;
        gp.no_grid_lo = compensated_ ? 0 : 1;
        return gp;
    }

    // Device bytes a grid() call over `records` records needs as workspace.
    size_t workspace_bytes(int records) const {
        mtb_grid_params gp = grid_params();
        size_t b = 0;
        check(mtb_grid_workspace_size(&gp, k_->h_conv_info.data(), records, &b), "mtb_grid_workspace_size");
        return b;
    }

    // One WImager chunk from device arrays (layouts of mtb.h; flags int32, or
    // bytes passed cast to int * when the imager was made with flags_u8).
    void grid(const float *uvw, const float *freq, const void *vis, const float *weights, const int *flags,
              int records) {
        mtb_grid_params gp = grid_params();
        ImagerBuffers::ensure(b_->ws, workspace_bytes(records), s_);
        check(mtb_grid(&gp, k_->table.data(), k_->conv_info.data(), k_->h_conv_info.data(), k_->conv_sums.data(),
                       uvw, freq, vis, weights, flags, records, b_->grid.data(),
                       compensated_ ? b_->lo.data() : nullptr, b_->norm.data(), b_->stats.data(), b_->ws.data(),
                       b_->ws.bytes(), (mtb_stream_t)s_),
              "mtb_grid");
        fresh_ = false;
    }

    // Stokes image [npol][ny][nx] into device memory.
    void finalize(float *image) {
        mtb_finalize_params fp;
        fp.nx = k_->params.nx;
        fp.ny = k_->params.ny;
        fp.npol = npol_;
        fp.sampling = k_->params.sampling;
        fp.pol_type = pol_type_;
        size_t need = 0;
        check(mtb_finalize_workspace_size(&fp, &need), "mtb_finalize_workspace_size");
        ImagerBuffers::ensure(b_->fin, need, s_);
        check(mtb_finalize(&fp, b_->grid.data(), compensated_ ? b_->lo.data() : nullptr, b_->norm.data(), image,
                           b_->fin.data(), b_->fin.bytes(), (mtb_stream_t)s_),
              "mtb_finalize");
    }

    // Statistics of the image so far (synchronises the stream).
    mtb_grid_stats stats() const {
        mtb_grid_stats h;
        cuda_check(cudaMemcpyAsync(&h, b_->stats.data(), sizeof(h), cudaMemcpyDeviceToHost, s_), "stats");
        cuda_check(cudaStreamSynchronize(s_), "stats sync");
        return h;
    }

private:
    std::shared_ptr<const KernelTable> k_;
    int npol_, pol_type_;
    bool compensated_, exact_delta_, flags_u8_;
    cudaStream_t s_;
    bool fresh_ = true;
    std::unique_ptr<ImagerBuffers> own_;
    ImagerBuffers *b_ = nullptr;
};

// TOPO -> LSRK nu/c of every record and channel from the MeasurementSet TIME
// column (mtb_lsrk_freq_over_c).  The workspace grows to the largest row count
// seen and is reused; every call only enqueues work on the stream.
class FrequencyConverter {
public:
    FrequencyConverter(const mtb_lsrk_params &params, cudaStream_t stream) : p_(params), s_(stream) {}

    // time: device double [nrows] (MJD seconds, row order); chan_hz: device
    // double [nchan]; index: device int [n] record order (nullptr: n == nrows);
    // out: device float [nchan][n]
    void convert(const double *time, int nrows, const double *chan_hz, int nchan, const int *index, int n,
                 float *out) {
        size_t need = 0;
        check(mtb_lsrk_workspace_size(nrows, &need), "mtb_lsrk_workspace_size");
        if (ws_.size() < need) ws_ = DeviceArray<unsigned char>(need, s_);
        check(mtb_lsrk_freq_over_c(&p_, time, nrows, chan_hz, nchan, index, n, out, ws_.data(), ws_.bytes(),
                                   (mtb_stream_t)s_),
              "mtb_lsrk_freq_over_c");
    }
    const mtb_lsrk_params &params() const { return p_; }

private:
    mtb_lsrk_params p_;
    cudaStream_t s_;
    DeviceArray<unsigned char> ws_;
};

}  // namespace mtb

#endif  // MTB_HPP
