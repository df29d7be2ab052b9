// Visibility preprocessing, binning and tile gridding for sm_100a.
//
// One mtb_grid call is one WImager chunk (code/mt-imager/lib/components/
// WImager.cpp:167-234).  The reference runs ~14 operators per chunk:
// PreProcessUVW, four statistics reductions, the normaliser sum, three
// exclusive scans with compaction / run detection to build a plan of <=440
// record runs of equal support, duplicate compression, and the Romein gridder
// that flushes every cell change with float atomics into the global grid
// (ConvolutionGridder.cu:325-444).
//
// Here:
//   k_preprocess   one pass over the records in FP64: w-plane, grid corner,
//                  oversampling offset, conv index, normaliser sums (FP64)
//                  (WProjPreProcessUVW.cu:112-286 semantics).
//   k_compress     duplicate detection exactly as the reference decides it
//                  (WProjPreProcessUVW.cu:265-324), statistics, and the bin key
//                  (support bucket, tile row, tile column) of every gridded record.
//   CUB            stable radix sort of the keys (original order kept inside a
//                  bin, so consecutive records of a baseline stay consecutive),
//                  run-length encoding and a scan to cut bins into work items.
//   k_gather       weighted, conjugation-corrected visibility of each gridded
//                  record summed over its compressed duplicates
//                  (CompressVisibilties.cu:41-74), stored in bin order together
//                  with the record's gridder layout.
//   k_pad_expand   row-padded copy of the kernel table (rows of S + 1 taps,
//                  16-byte aligned), every tap in {re,re,im,im} form.
//   k_grid5        default gridder: persistent blocks take work items (up to 256
//                  records of one bin) from a queue; one warp stages the item
//                  two ahead into the second of two shared-memory buffers
//                  (mbarrier hand-offs), so threads never wait at a block
//                  barrier.  The jobs of an item are those of k_grid3.
//   k_grid3        the same jobs with block-wide staging of one item at a time
//                  (items of up to 512 records; gridder = 3).  Threads own support-box
//                  positions (Romein's assignment: cell x belongs to the slot
//                  with a == x mod M), accumulate V * C in registers with packed
//                  f32x2 FMAs while their cell is unchanged, and flush a cell
//                  when it changes -- no global atomic per sample.  Each item's
//                  (support-box unit, record stream) jobs are balanced over
//                  the block's threads.  Kernel taps are fetched a few records
//                  ahead into a per-thread shared-memory ring with cp.async.
//   k_grid         shared-memory tile-window variant (merge = 1).
//   k_merge_delta  compensated mode: flushes go to a delta grid of the call
//                  (plain reductions; FP32, or FP64 with exact_delta), merged
//                  afterwards into the two-float grid (hi, lo).
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "mtb_internal.cuh"

namespace mtb {

static const unsigned kNoKey = 0xFFFFFFFFu;
static const int kMaxBuckets = 128;
static const int kStage = 64;          // records staged in shared memory per pass
static const int kDefaultTile = 32;
static const int kDefaultChunk = 2048;
static const size_t kWindowSmemLimit = 200 * 1024;

struct BucketTable {
    int n;                       // number of buckets in use
    int half;                    // odd supports per bucket
    int M[kMaxBuckets];          // modulus (largest support) of each bucket, 0 = empty
    int tile[kMaxBuckets];       // grid tile edge used for the bucket's keys
    // A record's sort key packs {bucket, tile row, tile column} into the low
    // xbits + ybits + bbits bits, bucket most significant; the bit counts
    // hold the largest tile column, tile row and bucket number + 1, so the
    // kNoKey sentinel (all ones) sorts after every record when the sort
    // covers only those bits.
    int xbits, ybits, bbits;
};

__device__ __forceinline__ int bucket_of(int S, int half) { return (S - 1) / (2 * half); }

// ------------------------------------------------------------- preprocess --
// Flag readers: flag i = r * P + p of the caller's array is set (flagged).
// FlagArray: one int (the reference's layout) or one byte per flag;
// FlagBits: one bit per flag, bit i % 8 of byte i / 8 (mtb_grid_params.flags_u8 = 2)
template <typename F>
struct FlagArray {
    const F *f;
    __device__ __forceinline__ bool operator()(size_t i) const { return __ldg(f + i) != 0; }
};
struct FlagBits {
    const unsigned char *f;
    __device__ __forceinline__ bool operator()(size_t i) const { return (__ldg(f + (i >> 3)) >> (i & 7)) & 1u; }
};

template <int P, typename FR>
__global__ void k_preprocess(int R, const float *__restrict__ uvw, const float *__restrict__ freq,
                             const float *__restrict__ weights, const FR flags,
                             const int *__restrict__ conv_info, const float *__restrict__ conv_sums,
                             int nw, double w_inc, int s, int T, int nx, int ny, double du, double dv,
                             int4 *__restrict__ pos, int *__restrict__ meta, double *__restrict__ norm_acc,
                             float *__restrict__ convsum_out) {
    double nsum[P];
#pragma unroll
    for (int p = 0; p < P; p++) nsum[p] = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
        int fl[P];
        float wt[P];
        bool grid = false;
#pragma unroll
        for (int p = 0; p < P; p++) {
            // any non-zero flag is a flagged sample; the reference weights by
            // 1 - flag (WProjPreProcessUVW.cu:84-106), which agrees for 0 / 1
            fl[p] = flags((size_t)r * P + p) ? 1 : 0;
            wt[p] = weights[(size_t)r * P + p];
            if (fl[p] == 0) grid = true;
        }
        int4 out = make_int4(0, 0, 0, 0);
        int m = 0;
        double cs = 0.0;
        if (grid) {
            double u = (double)uvw[r], v = (double)uvw[(size_t)R + r], w = (double)uvw[2 * (size_t)R + r];
            double f = (double)freq[r];
            // TakeConjugateIndicator is set before the bounds test, so a
            // rejected w < 0 record still reports -1 (WProjPreProcessUVW.cu:170-175)
            if (w < 0.0) { u = -u; v = -v; m = 2; }
            // WProjPreProcessUVW.cu:181-182
            double wp = round(sqrt(fabs(__ddiv_rn(__dmul_rn(w, f), w_inc))));
            if (!(wp == wp)) wp = 0.0;
            int k = (wp > (double)(nw - 1)) ? nw - 1 : (int)wp;
            int S = conv_info[2 * k];
            int ci = conv_info[2 * k + 1];
            // WProjPreProcessUVW.cu:188-199
            double pos_v = __dadd_rn(__ddiv_rn(__dmul_rn(v, f), dv), (double)(ny / 2));
            double pos_u = __dadd_rn(__ddiv_rn(__dmul_rn(u, f), du), (double)(nx / 2));
            double lx = round(pos_u), ly = round(pos_v);
            double cxd = lx - (double)(S / 2), cyd = ly - (double)(S / 2);
            if (!(cyd >= 0.0) || cyd > (double)((ny - 1) - S) || !(cxd >= 0.0) || cxd > (double)(nx - 1 - S)) {
                grid = false;
            } else {
                int cx = (int)cxd, cy = (int)cyd;
                // WProjPreProcessUVW.cu:206-239
                int ox = (int)round(__dmul_rn(__dadd_rn(lx, -pos_u), (double)s)) + s / 2;
                int oy = (int)round(__dmul_rn(__dadd_rn(ly, -pos_v), (double)s)) + s / 2;
                if (s & 1) {
                    ox = ox < 0 ? 0 : (ox == s ? s - 1 : ox);
                    oy = oy < 0 ? 0 : (oy == s ? s - 1 : oy);
                }
                cs = (double)conv_sums[(size_t)k * T * T + oy * T + ox];
                ci += oy * S * S * T + ox * S * S;
                out = make_int4(cx, cy, ci, S);
                m |= 1;
            }
        }
        pos[r] = out;
        meta[r] = m;
#pragma unroll
        for (int p = 0; p < P; p++) {
            double c = grid ? cs * (double)wt[p] * (1.0 - (double)fl[p]) : 0.0;
            nsum[p] += c;
            if (convsum_out) convsum_out[(size_t)p * R + r] = (float)c;
        }
    }
    // normaliser: NormalizerCalculate = Sum over records (WImager.cpp:196-197)
#pragma unroll
    for (int p = 0; p < P; p++) {
        double v = nsum[p];
        for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        __shared__ double red[P][32];
        if ((threadIdx.x & 31) == 0) red[p][threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x < 32) {
            double t = (threadIdx.x < (blockDim.x >> 5)) ? red[p][threadIdx.x] : 0.0;
            for (int off = 16; off; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
            if (threadIdx.x == 0 && t != 0.0) atomicAdd(&norm_acc[p], t);
        }
        __syncthreads();
    }
}

// Duplicate compression (a record whose corner row-index and conv index equal
// the previous record's stored values is merged into it; a non-gridded
// previous record stores zeros: WProjPreProcessUVW.cu:243-284, 316), the four
// record statistics, and the bin key of every record left to grid.
__global__ void k_compress(int R, int nx, const int4 *__restrict__ pos, int *__restrict__ meta,
                           unsigned *__restrict__ keys, int *__restrict__ iota, BucketTable bt,
                           unsigned long long *__restrict__ stats) {
    unsigned long long st[4] = {0, 0, 0, 0};
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
        int m = meta[r];
        int4 q = pos[r];
        bool comp = false;
        if ((m & 1) && r > 0) {
            int4 pq = pos[r - 1];   // zeros when the previous record is not gridded
            comp = (q.z == pq.z) && (q.y * nx + q.x == pq.y * nx + pq.x);
        }
        unsigned key = kNoKey;
        unsigned long long s2 = (unsigned long long)q.w * (unsigned long long)q.w;
        if (comp) {
            meta[r] = m | 4;
            st[1] += 1;
            st[3] += s2;
        } else if (m & 1) {
            int b = bucket_of(q.w, bt.half);
            int t = bt.tile[b];
            key = ((unsigned)b << (bt.xbits + bt.ybits)) | ((unsigned)(q.y / t) << bt.xbits) | (unsigned)(q.x / t);
            st[0] += 1;
            st[2] += s2;
        }
        keys[r] = key;
        iota[r] = r;
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        unsigned long long v = st[i];
        for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&stats[i], v);
    }
}

// Per bin-run: number of work items (bins of the kNoKey run give none).
__global__ void k_chunk_counts(const unsigned *__restrict__ ukeys, const int *__restrict__ counts,
                               const int *__restrict__ num_runs, int cap, int chunk, int *__restrict__ nchunks) {
    int n = *num_runs;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) {
        int c = 0;
        if (i < n && ukeys[i] != kNoKey) c = (counts[i] + chunk - 1) / chunk;
        nchunks[i] = c;
    }
}

// Work items: {first record (bin order), record count, bin key}, the key
// widened from the packed sort key to bucket << 24 | tile row << 12 | tile
// column, the layout the gridders decode.
__global__ void k_make_items(const unsigned *__restrict__ ukeys, const int *__restrict__ counts,
                             const int *__restrict__ run_start, const int *__restrict__ item_start,
                             const int *__restrict__ nchunks, const int *__restrict__ num_runs, int chunk,
                             int xbits, int ybits, int4 *__restrict__ items) {
    int n = *num_runs;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int c = nchunks[i];
        int base = item_start[i], s0 = run_start[i], cnt = counts[i];
        const unsigned k = ukeys[i];
        const unsigned key = ((k >> (xbits + ybits)) << 24) | (((k >> xbits) & ((1u << ybits) - 1u)) << 12) |
                             (k & ((1u << xbits) - 1u));
        for (int j = 0; j < c; j++) {
            int a = s0 + j * chunk;
            int len = min(chunk, s0 + cnt - a);
            items[base + j] = make_int4(a, len, (int)key, 0);
        }
    }
}

// Per bucket [begin, end) of the item list and the total item count.
__global__ void k_bucket_bounds(const int4 *__restrict__ items, const int *__restrict__ item_start,
                                const int *__restrict__ nchunks, const int *__restrict__ num_runs,
                                int *__restrict__ bounds, int nb, int *__restrict__ n_items) {
    int nr = *num_runs;
    int total = nr > 0 ? item_start[nr - 1] + nchunks[nr - 1] : 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) *n_items = total;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        int b = (int)((unsigned)items[i].z >> 24);
        int bp = i > 0 ? (int)((unsigned)items[i - 1].z >> 24) : -1;
        int bn = i + 1 < total ? (int)((unsigned)items[i + 1].z >> 24) : -1;
        if (b != bp) bounds[2 * b] = i;
        if (b != bn) bounds[2 * b + 1] = i + 1;
    }
}

// Gridded records in bin order with the weighted, conjugation-corrected
// visibility summed over the run of records compressed into it
// (CreateCompressionPlan.cu:32-67, CompressVisibilties.cu:41-74,
// common.hcu:94-104).  Two layouts:
//   DIRECT = false  {cx, cy, conv index, support} and float2 [P] (window gridder)
//   DIRECT = true   {cy*nx+cx, rxm | rym << 16, padded table index, support}
//                   with rxm = (-cx) mod M, rym = (-cy) mod M for the record's
//                   bucket modulus M, and per pol {re, im, -im, re} (direct
//                   gridders)
// Index of a record's sub-kernel in the row-padded table (rows of S + 1
// taps; see k_pad_expand) from its conv index in the reference layout.
__device__ __forceinline__ int padded_index(int ci, int S, const int *__restrict__ conv_info,
                                            const int *__restrict__ pbase, int nw) {
    int lo = 0, hi = nw - 1;             // last plane whose first element is <= ci
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&conv_info[2 * mid + 1]) <= ci) lo = mid;
        else hi = mid - 1;
    }
    const int sub = (ci - __ldg(&conv_info[2 * lo + 1])) / (S * S);
    return __ldg(&pbase[lo]) + sub * S * (S + 1);
}

template <int P, bool DIRECT, typename FR>
__global__ void k_gather(int R, const unsigned *__restrict__ skeys, const int *__restrict__ sidx,
                         const int4 *__restrict__ pos, const int *__restrict__ meta,
                         const float2 *__restrict__ vis, const float *__restrict__ weights,
                         const FR flags, int4 *__restrict__ wpos, void *__restrict__ wvis,
                         BucketTable bt, int nx, const int *__restrict__ conv_info, const int *__restrict__ pbase,
                         int nw, int psf, int vpairs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < R; i += gridDim.x * blockDim.x) {
        if (skeys[i] == kNoKey) continue;
        int g = sidx[i];
        float2 acc[P];
#pragma unroll
        for (int p = 0; p < P; p++) acc[p] = make_float2(0.f, 0.f);
        int r = g;
        do {
            int m = meta[r];
            float im = (m & 2) ? -1.0f : 1.0f;
#pragma unroll
            for (int p = 0; p < P; p++) {
                const float2 v = psf ? make_float2(1.0f, 0.0f) : vis[(size_t)r * P + p];
                float wgt = weights[(size_t)r * P + p];
                float keep = flags((size_t)r * P + p) ? 0.0f : 1.0f;
                acc[p].x += v.x * wgt * keep;
                acc[p].y += v.y * wgt * keep * im;
            }
            r++;
        } while (r < R && (meta[r] & 4));
        const int4 q = pos[g];
        if (DIRECT) {
            const int M = bt.M[bucket_of(q.w, bt.half)];
            const int rxm = (M - q.x % M) % M, rym = (M - q.y % M) % M;
            wpos[i] = make_int4(q.y * nx + q.x, rxm | (rym << 16), padded_index(q.z, q.w, conv_info, pbase, nw),
                                q.w);
            // {re, im, -im, re}: two packed FMAs per expanded tap; vpairs (the
            // tap-pair gridder): {re, re, im, im}
            float4 *o = (float4 *)wvis + (size_t)i * P;
#pragma unroll
            for (int p = 0; p < P; p++)
                o[p] = vpairs ? make_float4(acc[p].x, acc[p].x, acc[p].y, acc[p].y)
                              : make_float4(acc[p].x, acc[p].y, -acc[p].y, acc[p].x);
        } else {
            wpos[i] = q;
            float2 *o = (float2 *)wvis + (size_t)i * P;
#pragma unroll
            for (int p = 0; p < P; p++) o[p] = acc[p];
        }
    }
}

// err (may be null): the gridder's error flag; when set, the normaliser
// becomes NaN so the image of a gridding that did not complete cannot pass
// for a valid one.
__global__ void k_finish(int P, const double *__restrict__ norm_acc, float *__restrict__ normalizer,
                         const unsigned long long *__restrict__ st, mtb_grid_stats *__restrict__ out,
                         const int *__restrict__ err) {
    int t = threadIdx.x;
    if (t < P) normalizer[t] = (err && *err) ? __int_as_float(0x7fc00000) : normalizer[t] + (float)norm_acc[t];
    if (out && t == 0) {
        out->gridded_records += st[0];
        out->compressed_records += st[1];
        out->gridded_points += st[2];
        out->compressed_points += st[3];
    }
}

// ------------------------------------------------------- checked build --
// Built with -DMTB_CHECKED (libmtb_checked.so, build.py --checked): every
// data-dependent index of the gridders -- the kernel-table taps each slot
// reads and the grid cell each flush adds to -- is checked before use; an
// index out of range is skipped and the first such site is recorded in a
// device status word (mtb_bounds_status) instead of faulting.  Other indices
// of the path are loop-bounded by construction.  The unchecked build
// compiles the checks away.
enum BoundsSite : unsigned {
    kSiteTapStreaming = 1,   // k_grid7: tap read outside the padded table
    kSiteTapStaged = 2,      // k_grid3 / k_grid5: tap read outside the padded table
    kSiteFlush = 3,          // direct gridders: flush outside the grid
    kSiteTapWindow = 4,      // k_grid: tap read outside the table
    kSiteCellWindow = 5      // k_grid: flush outside the tile window or the grid
};
#ifdef MTB_CHECKED
__device__ unsigned g_bounds_word;
__device__ __forceinline__ bool in_bounds(long long i, long long n, unsigned site) {
    if (i >= 0 && i < n) return true;
    atomicCAS(&g_bounds_word, 0u, site);
    return false;
}
#else
__device__ __forceinline__ bool in_bounds(long long, long long, unsigned) { return true; }
#endif

// ---------------------------------------------------------------- gridder --
struct GridArgs {
    const int4 *items;
    const int *bounds;          // [bucket][2]
    int *counters;              // per bucket work counter
    const int4 *wpos;
    const float2 *wvis;
    const float2 *table;
    float *grid;                // float2 [ny][nx][P] as floats
    float *grid_lo;             // may be null
    int nx, ny;
    int bucket, M, rows, nbands, tile, W;
    int table_elems, cells;     // bounds of the checked build
};

// Two-float merge: hi += t with the rounding error of that add accumulated in lo.
__device__ __forceinline__ void merge4(float *hi, float *lo, float4 t) {
    if (lo) {
        float4 old = atomicAdd((float4 *)hi, t);
        float4 e;
        float s, bp;
        s = old.x + t.x; bp = s - old.x; e.x = (old.x - (s - bp)) + (t.x - bp);
        s = old.y + t.y; bp = s - old.y; e.y = (old.y - (s - bp)) + (t.y - bp);
        s = old.z + t.z; bp = s - old.z; e.z = (old.z - (s - bp)) + (t.z - bp);
        s = old.w + t.w; bp = s - old.w; e.w = (old.w - (s - bp)) + (t.w - bp);
        atomicAdd((float4 *)lo, e);
    } else {
        atomicAdd((float4 *)hi, t);
    }
}
__device__ __forceinline__ void merge2(float *hi, float *lo, float2 t) {
    if (lo) {
        float2 old = atomicAdd((float2 *)hi, t);
        float2 e;
        float s, bp;
        s = old.x + t.x; bp = s - old.x; e.x = (old.x - (s - bp)) + (t.x - bp);
        s = old.y + t.y; bp = s - old.y; e.y = (old.y - (s - bp)) + (t.y - bp);
        atomicAdd((float2 *)lo, e);
    } else {
        atomicAdd((float2 *)hi, t);
    }
}

template <int P>
__device__ __forceinline__ void merge_cell(float *hi, float *lo, const float *v) {
    if (P == 1) {
        merge2(hi, lo, make_float2(v[0], v[1]));
    } else {
#pragma unroll
        for (int q = 0; q < 2 * P; q += 4) merge4(hi + q, lo ? lo + q : nullptr, make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]));
    }
}

// WINDOW: cell flushes go to the shared-memory window of the work item's
// tile, merged into the grid at the end of the item.  !WINDOW (supports too
// large for a window): flushes go straight to the grid.
template <int P, int KMAX, bool WINDOW>
__global__ void __launch_bounds__(KMAX >= 8 ? 576 : 1024) k_grid(GridArgs a) {
    extern __shared__ float4 smem4[];
    const int M = a.M, rows = a.rows, W = a.W;
    const int nthreads = M * rows;
    const int t = threadIdx.x;
    float *win = (float *)smem4;
    // padded to 16 bytes so the staging area after it stays int4-aligned
    const size_t win_floats = WINDOW ? (((size_t)W * W * 2 * P + 3) & ~(size_t)3) : 0;
    int4 *s_rec = (int4 *)(win + win_floats);                 // {base, (rxm | rym<<16), conv, S}
    float *s_vis = (float *)(s_rec + kStage);                  // [kStage][2P]
    __shared__ int s_item;

    const int ta = t % M, tr = t / M;
    const bool live = t < nthreads;
    const int stride = WINDOW ? W : a.nx;

    if (WINDOW) {
        for (size_t i = t; i < (size_t)W * W * 2 * P; i += blockDim.x) win[i] = 0.f;
    }
    const int begin = a.bounds[2 * a.bucket], end = a.bounds[2 * a.bucket + 1];
    const int nvirt = (end - begin) * a.nbands;

    for (;;) {
        __syncthreads();
        if (t == 0) s_item = atomicAdd(&a.counters[a.bucket], 1);
        __syncthreads();
        const int v = s_item;
        if (v >= nvirt) break;
        const int item = begin + v / a.nbands, band = v % a.nbands;
        const int4 it = a.items[item];
        const unsigned key = (unsigned)it.z;
        const int wx0 = (int)(key & 0xFFFu) * a.tile, wy0 = (int)((key >> 12) & 0xFFFu) * a.tile;
        const int b0 = band * rows * KMAX + tr;               // first slot row of this thread

        float acc[KMAX][2 * P];
        int last[KMAX];
#pragma unroll
        for (int j = 0; j < KMAX; j++) {
            last[j] = -1;
#pragma unroll
            for (int c = 0; c < 2 * P; c++) acc[j][c] = 0.f;
        }

        for (int r0 = 0; r0 < it.y; r0 += kStage) {
            const int nrec = min(kStage, it.y - r0);
            __syncthreads();
            for (int i = t; i < nrec; i += blockDim.x) {
                int4 p = a.wpos[it.x + r0 + i];
                int rx = p.x - wx0, ry = p.y - wy0;
                int rxm = (M - rx % M) % M, rym = (M - ry % M) % M;
                int base = WINDOW ? ry * W + rx : (p.y * a.nx + p.x);
                s_rec[i] = make_int4(base, rxm | (rym << 16), p.z, p.w);
            }
            for (int i = t; i < nrec * P; i += blockDim.x) {
                float2 vv = a.wvis[(size_t)(it.x + r0) * P + i];
                s_vis[2 * i] = vv.x;
                s_vis[2 * i + 1] = vv.y;
            }
            __syncthreads();
            if (!live) continue;
            for (int i = 0; i < nrec; i++) {
                const int4 rec = s_rec[i];
                const int S = rec.w;
                int sx = ta + (rec.y & 0xFFFF);
                if (sx >= M) sx -= M;
                if (sx >= S) continue;
                int sy = b0 + (rec.y >> 16);
                if (sy >= M) sy -= M;
                float vr[P], vi[P];
#pragma unroll
                for (int p = 0; p < P; p++) {
                    vr[p] = s_vis[i * 2 * P + 2 * p];
                    vi[p] = s_vis[i * 2 * P + 2 * p + 1];
                }
                const int cbase = rec.x + sx, tbase = rec.z + sx;
#pragma unroll
                for (int j = 0; j < KMAX; j++) {
                    const int b = b0 + j * rows;
                    if (b < M && sy < S && in_bounds(tbase + sy * S, a.table_elems, kSiteTapWindow) &&
                        in_bounds(cbase + sy * stride, WINDOW ? W * W : a.cells, kSiteCellWindow)) {
                        const int cell = cbase + sy * stride;
                        const float2 cw = __ldg(&a.table[tbase + sy * S]);
                        if (cell != last[j]) {
                            if (last[j] >= 0) {
                                if (WINDOW) {
                                    float *wc = win + (size_t)last[j] * 2 * P;
#pragma unroll
                                    for (int c = 0; c < 2 * P; c++) wc[c] += acc[j][c];
                                } else {
                                    merge_cell<P>(a.grid + (size_t)last[j] * 2 * P,
                                                  a.grid_lo ? a.grid_lo + (size_t)last[j] * 2 * P : nullptr, acc[j]);
                                }
                            }
                            last[j] = cell;
#pragma unroll
                            for (int c = 0; c < 2 * P; c++) acc[j][c] = 0.f;
                        }
                        // ConvolutionGridder.cu:153-181: to += vis * wt (no conjugate)
#pragma unroll
                        for (int p = 0; p < P; p++) {
                            acc[j][2 * p] += vr[p] * cw.x;
                            acc[j][2 * p + 1] += vi[p] * cw.x;
                            acc[j][2 * p] -= vi[p] * cw.y;
                            acc[j][2 * p + 1] += vr[p] * cw.y;
                        }
                    }
                    sy += rows;
                    if (sy >= M) sy -= M;
                }
            }
        }
        // register flush
        if (live) {
#pragma unroll
            for (int j = 0; j < KMAX; j++) {
                if (last[j] >= 0) {
                    if (WINDOW) {
                        float *wc = win + (size_t)last[j] * 2 * P;
#pragma unroll
                        for (int c = 0; c < 2 * P; c++) wc[c] += acc[j][c];
                    } else {
                        merge_cell<P>(a.grid + (size_t)last[j] * 2 * P,
                                      a.grid_lo ? a.grid_lo + (size_t)last[j] * 2 * P : nullptr, acc[j]);
                    }
                }
            }
        }
        if (WINDOW) {
            __syncthreads();
            // one merge of the tile window into the grid; cells left at zero are skipped
            for (int c = t; c < W * W; c += blockDim.x) {
                float *wc = win + (size_t)c * 2 * P;
                float vals[2 * P];
                bool nz = false;
#pragma unroll
                for (int q = 0; q < 2 * P; q++) {
                    vals[q] = wc[q];
                    nz |= (vals[q] != 0.f);
                    wc[q] = 0.f;
                }
                if (!nz) continue;
                int y = wy0 + c / W, x = wx0 + c % W;
                if (y >= a.ny || x >= a.nx) continue;
                size_t g = ((size_t)y * a.nx + x) * 2 * P;
                merge_cell<P>(a.grid + g, a.grid_lo ? a.grid_lo + g : nullptr, vals);
            }
        }
    }
}

// ------------------------------------------------------- direct gridder --
// One persistent launch for every support bucket.  A block takes a work item
// (up to max_chunk records of one (support bucket, tile) bin, original record
// order) and splits it into (support-box unit, record stream) jobs over its
// threads.  A unit is one column of the M x M support box and every G-th row
// of it; for a record with corner (cx, cy) a slot (a, b) touches cell
// (cx + sx, cy + sy), sx = (a - cx) mod M, sy = (b - cy) mod M (Romein's
// assignment: a slot keeps its cell while the record moves less than a cell,
// and no two slots of a unit share a cell).  Each slot accumulates V * C for
// all polarisations in registers with packed f32x2 FMAs and merges into the
// grid (vector reductions) only when its cell changes and at the end of a job.
static const int kG3Threads = 256;          // default block size (threads per work item)
static const int kG3Chunk = 512;            // records of one work item, staged at once
static const int kG3Depth = 4;              // records of kernel values fetched ahead
static const int kG3KS = 4;                 // support-box slots per thread

// One image of a k_grid3 launch: its records and visibilities in gridder
// layout, its expanded padded kernel table, its grid (or FP64 delta grid in
// compensated mode) and the modulus of each of its support buckets.
struct GridJobDesc {
    const int4 *wpos;
    const float4 *wvis4;
    const float4 *table2;  // padded table, taps as {re, re, im, im}
    float *grid;
    double *dgrid;         // compensated mode: FP64 delta grid of this call, else null
    const int *M;          // [kMaxBuckets] bucket moduli (device)
    int nx;
    int uniform;           // 1: every record's support equals its bucket's modulus
    int table2_elems;      // entries of table2 (bounds of the checked build)
    int cells;             // nx * ny (bounds of the checked build)
};

static const int kMaxBatch = 64;   // images one batched launch grids

struct Grid2Args {
    const int4 *items;     // work items; item.w selects the image
    const int *n_items;
    int *counter;
    int njobs;
    long long wait_cycles; // bound of every mbarrier wait of k_grid5
    GridJobDesc jobs[kMaxBatch];
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Copies 16 bytes (bytes = 16), or writes 16 zero bytes and reads nothing
// (bytes = 0); gmem must be a mapped address either way.
__device__ __forceinline__ void cp_async16_zfill_n(unsigned smem_addr, const void *gmem, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr), "l"(gmem), "r"(bytes)
                 : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// One cell's flush: vector FP32 reductions into the grid, or, when dgrid is
// set (compensated mode), FP64 reductions into the call's delta grid.
template <int P>
__device__ __forceinline__ void flush_cell(float *grid, double *dgrid, int cell, int cells, const float *v) {
    if (!in_bounds(cell, cells, kSiteFlush)) return;
    const size_t g = (size_t)cell * 2 * P;
    if (dgrid) {
#pragma unroll
        for (int q = 0; q < 2 * P; q++)
            if (v[q] != 0.f) atomicAdd(dgrid + g + q, (double)v[q]);
    } else {
        merge_cell<P>(grid + g, nullptr, v);
    }
}

template <int P>
__device__ __forceinline__ void flush2(float *grid, double *dgrid, int cell, int cells, const float2 *acc) {
    float v[2 * P];
#pragma unroll
    for (int p = 0; p < P; p++) {
        v[2 * p] = acc[p].x;
        v[2 * p + 1] = acc[p].y;
    }
    flush_cell<P>(grid, dgrid, cell, cells, v);
}

// Work schedule of one item for modulus M (KS slots per thread, all in one
// support-box column so the column offset is computed once per record):
//   G = ceil(M / KS) row groups; a unit (column c, row group g) owns the rows
//   g + j*G of column c; U = M * G units cover the support box.
//   The item's N records are split into ns contiguous streams; a job is one
//   (stream, unit) pair, jobs are numbered unit-fastest (so the threads of a
//   warp share records) and thread t takes jobs t, t + T, t + 2T, ...
//   ns minimises rounds * (ceil(N / ns) + kSegCost), rounds = ceil(ns*U / T):
//   the slowest thread's time, each job paying a fixed cost for filling its
//   look-ahead and flushing its slots.  Streams keep at least kMinStreamRecords
//   records (each stream's flushes are extra FP32 reductions into the same
//   cells).  Every flush is an atomic merge, so streams may share cells.
static const int kSegCost = 4;          // per-job overhead in record times
static const int kMinStreamRecords = 4;

// ns in [1, min(N / kMinStreamRecords, 64)]; all lanes of a warp return the
// same value (warp-wide argmin, two candidates per lane).
__device__ __forceinline__ int pick_streams(int U, int N, int T) {
    const int lane = threadIdx.x & 31;
    const int cmax = N / kMinStreamRecords;
    unsigned best = 0xFFFFFFFFu;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int c = lane + 1 + 32 * h;
        if (c <= cmax) {
            const unsigned rounds = (unsigned)((c * U + T - 1) / T);
            const unsigned cost = rounds * (unsigned)((N + c - 1) / c + kSegCost);
            const unsigned key = (cost << 7) | (unsigned)c;
            best = key < best ? key : best;
        }
    }
    best = __reduce_min_sync(0xFFFFFFFFu, best);
    return best == 0xFFFFFFFFu ? 1 : (int)(best & 127u);
}

// Row-padded copy of the kernel table for the direct gridders: every
// sub-kernel row gets one zero tap (S + 1 taps, S odd), so each row and each
// sub-kernel starts on a 16-byte boundary and rows can be moved with bulk
// copies.  pbase[k] = first padded element of plane k; pbase[nw + k] = first
// row (of S taps) of plane k, pbase[2 nw] = every plane's rows.
__global__ void k_pad_bases(const int *__restrict__ conv_info, int nw, int T, int *__restrict__ pbase) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int b = 0, rows = 0;
        for (int k = 0; k < nw; k++) {
            pbase[k] = b;
            pbase[nw + k] = rows;
            const int S = conv_info[2 * k];
            b += T * T * S * (S + 1);
            rows += T * T * S;
        }
        pbase[2 * nw] = rows;
    }
}

// Row-padded, expanded table in one pass: each warp copies a contiguous range
// of kernel rows (S taps of one sub-kernel row each), so the plane is found
// once per warp and then followed across plane boundaries.  t2 gets every tap
// as {re, re, im, im} (one 128-bit load gives both packed operands of the
// f32x2 complex multiply-add) with a zero tap closing each row.
__global__ void k_pad_expand(const float2 *__restrict__ t, const int *__restrict__ conv_info,
                             const int *__restrict__ pbase, int nw, int rows, float4 *__restrict__ t2) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int per = (rows + nwarps - 1) / nwarps;
    const int r0 = warp * per, r1 = min(rows, r0 + per);
    if (r0 >= r1) return;
    const int *rbase = pbase + nw;
    int lo = 0, hi = nw - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&rbase[mid]) <= r0) lo = mid;
        else hi = mid - 1;
    }
    int k = lo;
    int S = __ldg(&conv_info[2 * k]), rb = __ldg(&rbase[k]), next = __ldg(&rbase[k + 1]);
    size_t cbase = (size_t)__ldg(&conv_info[2 * k + 1]), pb = (size_t)__ldg(&pbase[k]);
    for (int row = r0; row < r1; row++) {
        while (row >= next) {     // next plane (rbase[nw] is the total, so this ends)
            k++;
            S = __ldg(&conv_info[2 * k]);
            rb = next;
            next = __ldg(&rbase[k + 1]);
            cbase = (size_t)__ldg(&conv_info[2 * k + 1]);
            pb = (size_t)__ldg(&pbase[k]);
        }
        const int rel = row - rb;        // sub * S + y
        const int sub = rel / S, y = rel - sub * S;
        const size_t src = cbase + (size_t)rel * S;
        const size_t dst = pb + (size_t)sub * S * (S + 1) + (size_t)y * (S + 1);
        for (int x = lane; x <= S; x += 32) {
            const float2 c = x < S ? t[src + x] : make_float2(0.f, 0.f);
            t2[dst + x] = make_float4(c.x, c.x, c.y, c.y);
        }
    }
}

// The pair table of the tap-pair gridder, in k_pad_expand's layout (S + 1
// 16-byte entries per sub-kernel row): entry k < (S + 1) / 2 holds taps
// (2k, 2k + 1) and entry (S + 1) / 2 + k taps (2k + 1, 2k + 2), each {re, im};
// a tap index S stands for tap 0 (the neighbour of column S - 1 under Romein's
// wrap with one support per bucket), and the pair starting at column S is zero.
__global__ void k_pad_pairs(const float2 *__restrict__ t, const int *__restrict__ conv_info,
                            const int *__restrict__ pbase, int nw, int rows, float4 *__restrict__ t2) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int per = (rows + nwarps - 1) / nwarps;
    const int r0 = warp * per, r1 = min(rows, r0 + per);
    if (r0 >= r1) return;
    const int *rbase = pbase + nw;
    int lo = 0, hi = nw - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&rbase[mid]) <= r0) lo = mid;
        else hi = mid - 1;
    }
    int k = lo;
    int S = __ldg(&conv_info[2 * k]), rb = __ldg(&rbase[k]), next = __ldg(&rbase[k + 1]);
    size_t cbase = (size_t)__ldg(&conv_info[2 * k + 1]), pb = (size_t)__ldg(&pbase[k]);
    for (int row = r0; row < r1; row++) {
        while (row >= next) {     // next plane (rbase[nw] is the total, so this ends)
            k++;
            S = __ldg(&conv_info[2 * k]);
            rb = next;
            next = __ldg(&rbase[k + 1]);
            cbase = (size_t)__ldg(&conv_info[2 * k + 1]);
            pb = (size_t)__ldg(&pbase[k]);
        }
        const int rel = row - rb;        // sub * S + y
        const int sub = rel / S, y = rel - sub * S;
        const size_t src = cbase + (size_t)rel * S;
        const size_t dst = pb + (size_t)sub * S * (S + 1) + (size_t)y * (S + 1);
        const int half = (S + 1) >> 1;
        for (int x = lane; x <= S; x += 32) {
            const int c0 = x < half ? 2 * x : 2 * (x - half) + 1;    // first column of the pair
            float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
            if (c0 < S) {
                a = t[src + c0];
                b = t[src + (c0 + 1 < S ? c0 + 1 : 0)];
            }
            t2[dst + x] = make_float4(a.x, a.y, b.x, b.y);
        }
    }
}

// The jobs of one work item for this thread (the direct gridders k_grid3 and
// k_grid5): the item's records, visibilities and run ends are staged in
// shared memory.  Each thread fetches the kernel values of its slots
// kG3Depth records ahead into its own entries of a shared-memory ring
// (cp.async, completion tracked per thread with commit/wait groups, so no
// block barrier per record).  A slot outside a record's support box gets
// zeros in its ring entry, which keeps the accumulation loop free of
// per-slot branches.
// UNIFORM: every record's support equals the modulus M (one support per
// bucket), so no slot of a record's box falls outside it.
template <int P, int T, bool UNIFORM>
__device__ __forceinline__ void grid_item(const Grid2Args &a, const int4 it, const int4 *s_rec, const float4 *s_v,
                                          const unsigned short *s_runend, ulonglong2 *ring) {
    constexpr int KS = kG3KS, D = kG3Depth;
    const int t = threadIdx.x;
    const GridJobDesc &J = a.jobs[it.w];
    const ulonglong2 *tab = (const ulonglong2 *)J.table2;
    float *const ggrid = J.grid;
    double *const gdelta = J.dgrid;
    const int gnx = J.nx;
    const int N = it.y;
    const int M = J.M[(unsigned)it.z >> 24];
    const int G = (M + KS - 1) / KS;
    const int U = M * G;
    const int ns = pick_streams(U, N, T);
    const int njobs = ns * U;
    for (int job = t; job < njobs; job += T) {
        const int stream = job / U;
        const int u = job - stream * U;
        const int g = u / M;
        const int col = u - g * M;
        const int i0 = (N * stream) / ns;
        const int i1 = (N * (stream + 1)) / ns;
        // rows g + j*G that exist: j < nrow
        const int nrow = (M - g + G - 1) / G;
        if (i0 >= i1) continue;
        // Slot geometry depends only on the record's corner and support;
        // vbytes = 0 marks a slot outside the record's box.
        auto geometry = [&](const int4 &rec, int *cell, int *toff, int *vbytes) {
            const int S = rec.w;
            int sx = col + (rec.y & 0xFFFF);
            sx -= (sx >= M) ? M : 0;
            int sy = g + (rec.y >> 16);
            sy -= (sy >= M) ? M : 0;
            const bool xok = UNIFORM || sx < S;
#pragma unroll
            for (int j = 0; j < KS; j++) {
                const bool ok = xok && (j < nrow) && (UNIFORM || sy < S);
                cell[j] = ok ? rec.x + sy * gnx + sx : -1;
                toff[j] = ok ? sy * (S + 1) + sx : 0;
                vbytes[j] = ok ? 16 : 0;
                sy += G;
                sy -= (sy >= M) ? M : 0;
            }
        };
        // Look-ahead: the kernel values of record k go to ring slot k % D;
        // the geometry is recomputed when k enters a new run (k == pend).
        int pend = i0, toffL[KS], cellL[KS], vbL[KS];
        const unsigned ring_s = (unsigned)__cvta_generic_to_shared(ring) + t * 16;
        auto prefetch = [&](int k) {
            if (k == pend) {
                geometry(s_rec[k], cellL, toffL, vbL);
                const int e = s_runend[k];
                pend = e < i1 ? e : i1;
            }
            const int z = s_rec[k].z;
            const unsigned dst = ring_s + (unsigned)(k & (D - 1)) * (KS * T * 16);
            // slots outside the box get zeros (toff = 0 keeps the address valid)
#pragma unroll
            for (int j = 0; j < KS; j++) {
                const bool in = in_bounds((long long)z + toffL[j], J.table2_elems, kSiteTapStaged);
                cp_async16_zfill_n(dst + j * (T * 16), tab + (in ? z + toffL[j] : 0), in ? vbL[j] : 0);
            }
        };
#pragma unroll
        for (int d = 0; d < D; d++) {
            if (i0 + d < i1) prefetch(i0 + d);
            cp_async_commit();
        }
        int last[KS];
        float2 acc[KS][P];
#pragma unroll
        for (int j = 0; j < KS; j++) {
            last[j] = -1;
#pragma unroll
            for (int p = 0; p < P; p++) acc[j][p] = make_float2(0.f, 0.f);
        }
        // Runs of records with the same corner and support: the flushes sit
        // between runs, so the accumulators stay in place inside a run.
        int i = i0;
        while (i < i1) {
            {
                // corner or support changed: flush the slots whose cell changes
                int cellN[KS], toffN[KS], vN[KS];
                geometry(s_rec[i], cellN, toffN, vN);
#pragma unroll
                for (int j = 0; j < KS; j++) {
                    if (cellN[j] >= 0 && cellN[j] != last[j]) {
                        if (last[j] >= 0) flush2<P>(ggrid, gdelta, last[j], J.cells, acc[j]);
                        last[j] = cellN[j];
#pragma unroll
                        for (int p = 0; p < P; p++) acc[j][p] = make_float2(0.f, 0.f);
                    }
                }
            }
            const int e = s_runend[i];
            const int re = e < i1 ? e : i1;
            for (; i < re; ++i) {
                // the visibilities were staged before the item started: load
                // them ahead of the wait so their latency overlaps it
                float2 vp[P], wp[P];
                const float4 *vr = s_v + i * P;
#pragma unroll
                for (int p = 0; p < P; p++) {
                    const float4 q = vr[p];
                    vp[p] = make_float2(q.x, q.y);
                    wp[p] = make_float2(q.z, q.w);
                }
                cp_async_wait<D - 1>();     // this thread's copies for record i have landed
                const float4 *src = (const float4 *)(ring + ((i & (D - 1)) * KS * T + t));
#pragma unroll
                for (int j = 0; j < KS; j++) {
                    const float4 c = src[j * T];
                    const float2 cre = make_float2(c.x, c.y), cim = make_float2(c.z, c.w);
                    // ConvolutionGridder.cu:153-181: to += vis * wt (no conjugate)
#pragma unroll
                    for (int p = 0; p < P; p++) {
                        acc[j][p] = __ffma2_rn(cre, vp[p], acc[j][p]);
                        acc[j][p] = __ffma2_rn(cim, wp[p], acc[j][p]);
                    }
                }
                if (i + D < i1) prefetch(i + D);
                cp_async_commit();
            }
        }
        cp_async_wait<0>();
#pragma unroll
        for (int j = 0; j < KS; j++)
            if (last[j] >= 0) flush2<P>(ggrid, gdelta, last[j], J.cells, acc[j]);
    }
}

// Direct gridder with block-wide staging: the block takes a work item from
// the queue, copies its records (already in the gridder layout) and
// visibilities to shared memory with 16-byte cp.async, marks the runs, and
// every thread grids its jobs of the item.
template <int P, int T>
__global__ void __launch_bounds__(T, 512 / T) k_grid3(Grid2Args a) {
    extern __shared__ uint4 smem3[];
    int4 *s_rec = (int4 *)smem3;                                  // [kG3Chunk]
    float4 *s_v = (float4 *)(s_rec + kG3Chunk);                   // [kG3Chunk][P]
    ulonglong2 *ring = (ulonglong2 *)(s_v + kG3Chunk * P);        // [kG3Depth][kG3KS][T]
    __shared__ int s_item;
    __shared__ unsigned s_start[kG3Chunk / 32];    // bit k: record k starts a run
    __shared__ unsigned short s_runend[kG3Chunk];  // first record after k's run
    const int t = threadIdx.x;
    const int lane = t & 31;
    const int nitems = a.n_items[0];
    for (;;) {
        __syncthreads();
        if (t == 0) s_item = atomicAdd(a.counter, 1);
        __syncthreads();
        const int v = s_item;
        if (v >= nitems) break;
        const int4 it = a.items[v];
        const GridJobDesc &J = a.jobs[it.w];
        const int4 *grec = J.wpos;
        const float4 *gvis = J.wvis4;
        const int N = it.y;
        // stage the item's records (gridder layout, 16-byte pieces)
        for (int k = t; k < N; k += T) cp_async16(&s_rec[k], &grec[it.x + k]);
        for (int k = t; k < N * P; k += T) cp_async16(&s_v[k], &gvis[(size_t)it.x * P + k]);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        // Runs: maximal ranges of records with the same corner and support
        // (the slots' cells and table offsets within the sub-kernel are fixed
        // over a run).  s_runend[k] = first record after the run holding k.
        for (int k0 = 0; k0 < N; k0 += T) {
            const int k = k0 + t;
            bool start = false;
            if (k < N) {
                const int4 r = s_rec[k];
                start = (k == 0) || r.x != s_rec[k - 1].x || r.w != s_rec[k - 1].w;
            }
            const unsigned m = __ballot_sync(0xFFFFFFFFu, start);
            if (lane == 0) s_start[k >> 5] = m;
        }
        __syncthreads();
        const int nw = (N + 31) >> 5;
        for (int k = t; k < N; k += T) {
            int w = k >> 5;
            unsigned m = (k & 31) == 31 ? 0u : s_start[w] & (0xFFFFFFFFu << ((k & 31) + 1));
            while (m == 0 && ++w < nw) m = s_start[w];
            s_runend[k] = (unsigned short)(m == 0 ? N : (w << 5) + __ffs(m) - 1);
        }
        __syncthreads();
        if (J.uniform) grid_item<P, T, true>(a, it, s_rec, s_v, s_runend, ring);
        else grid_item<P, T, false>(a, it, s_rec, s_v, s_runend, ring);
    }
}

template <int P, int T>
static int launch_grid3_t(const Grid2Args &a, cudaStream_t st) {
    auto kern = k_grid3<P, T>;
    const size_t smem = (size_t)kG3Chunk * 16 * (1 + P) + (size_t)kG3Depth * kG3KS * T * 16;
    MTB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    MTB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, T, smem));
    if (per_sm < 1) return MTB_ERR_BAD_SHAPE;
    kern<<<per_sm * sm_count(), T, smem, st>>>(a);
    MTB_LAUNCHED();
    return MTB_OK;
}

// threads: gridder block size (0: default, 256 or 512)
template <int P>
static int launch_grid3(const Grid2Args &a, int threads, cudaStream_t st) {
    if (threads == 512) return launch_grid3_t<P, 512>(a, st);
    return launch_grid3_t<P, kG3Threads>(a, st);
}

// Bounded mbarrier waits of the rolling-items gridder: a wait gives up after
// this many SM clock cycles (about a second) unless the host sets another limit
// (MTB_GRIDDER_WAIT_CYCLES, read at every call: a test makes waits run out).
static const long long kWaitCycles = 1LL << 31;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the completion of the phase with the given parity: false
// when another thread gave up (abort_flag) or `limit` cycles passed.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, volatile int *abort_flag, long long limit) {
    if (mbar_try(bar, parity)) return true;
    const long long t0 = clock64();
    for (;;) {
        if (mbar_try(bar, parity)) return true;
        if (*abort_flag) return false;
        if (clock64() - t0 > limit) return false;
    }
}

// Rolling-items gridder: the jobs of k_grid3 without block barriers.  Two
// item buffers in shared memory; warp 0 refills a buffer with the item two
// ahead once every thread has left it ("empty" mbarrier, one arrival per
// thread) and publishes it ("full" mbarrier, one arrival per lane of warp 0),
// so a thread that finishes its jobs of one item starts on the next at once
// instead of waiting for the slowest thread at a block barrier.  Every wait
// is bounded by a clock deadline; a wait that runs out sets *err and the
// kernel returns.
static const int kG5Chunk = 256;   // records of one work item (one buffer)

template <int P, int CHUNK = kG5Chunk>
struct G5Layout {   // one item buffer of CHUNK records, byte offsets
    static constexpr int chunk = CHUNK;
    static constexpr size_t rec = 0;                                        // int4 [CHUNK]
    static constexpr size_t vis = rec + (size_t)CHUNK * 16;                 // float4 [CHUNK][P]
    static constexpr size_t runend = vis + (size_t)CHUNK * P * 16;          // ushort [CHUNK]
    static constexpr size_t start = runend + (size_t)CHUNK * 2;             // unsigned [CHUNK / 32]
    static constexpr size_t item = (start + (size_t)CHUNK / 8 + 15) & ~(size_t)15;   // int4 (y < 0: no more items)
    static constexpr size_t bytes = item + 16;
    static_assert(CHUNK % 32 == 0, "run starts are kept as 32-bit words");
    static_assert(rec % 16 == 0 && vis % 16 == 0 && item % 16 == 0 && bytes % 16 == 0,
                  "16-byte fields (cp.async targets, int4 loads) must stay 16-byte aligned");
};

// Warp 0 of a rolling-items block: the next item of the queue (or the end
// mark, item.y < 0) into item buffer B with its records, visibilities and run
// ends, then one arrival per lane on the buffer's "full" mbarrier.
template <int P, int CHUNK>
__device__ __forceinline__ void stage_item(const Grid2Args &a, unsigned char *B, unsigned full_bar, int nitems,
                                           int *err) {
    using LY = G5Layout<P, CHUNK>;
    const int lane = threadIdx.x & 31;
    int4 *s_rec = (int4 *)(B + LY::rec);
    float4 *s_v = (float4 *)(B + LY::vis);
    unsigned short *s_runend = (unsigned short *)(B + LY::runend);
    unsigned *s_start = (unsigned *)(B + LY::start);
    int v = 0;
    if (lane == 0) v = atomicAdd(a.counter, 1);
    v = __shfl_sync(0xFFFFFFFFu, v, 0);
    int4 it = make_int4(0, -1, 0, 0);
    if (v < nitems) it = a.items[v];
    if (it.y > CHUNK) {      // the plan caps items at CHUNK records
        if (lane == 0) atomicExch(err, 2);
        it.y = -1;
    }
    if (it.y >= 0) {
        const GridJobDesc &J = a.jobs[it.w];
        const int4 *grec = J.wpos;
        const float4 *gvis = J.wvis4;
        const int N = it.y;
        for (int k = lane; k < N; k += 32) cp_async16(&s_rec[k], &grec[it.x + k]);
        for (int k = lane; k < N * P; k += 32) cp_async16(&s_v[k], &gvis[(size_t)it.x * P + k]);
        cp_async_commit();
        cp_async_wait<0>();
        __syncwarp();
        for (int k0 = 0; k0 < N; k0 += 32) {      // run starts
            const int k = k0 + lane;
            bool st = false;
            if (k < N) {
                const int4 r = s_rec[k];
                st = (k == 0) || r.x != s_rec[k - 1].x || r.w != s_rec[k - 1].w;
            }
            const unsigned m = __ballot_sync(0xFFFFFFFFu, st);
            if (lane == 0) s_start[k0 >> 5] = m;
        }
        __syncwarp();
        const int nw = (N + 31) >> 5;
        for (int k = lane; k < N; k += 32) {      // run ends
            int w = k >> 5;
            unsigned m = (k & 31) == 31 ? 0u : s_start[w] & (0xFFFFFFFFu << ((k & 31) + 1));
            while (m == 0 && ++w < nw) m = s_start[w];
            s_runend[k] = (unsigned short)(m == 0 ? N : (w << 5) + __ffs(m) - 1);
        }
    }
    if (lane == 0) *(int4 *)(B + LY::item) = it;
    __syncwarp();
    mbar_arrive(full_bar);                    // every lane: its copies and stores are done
}

template <int P>
__global__ void __launch_bounds__(kG3Threads, 2) k_grid5(Grid2Args a, int *err) {
    constexpr int T = kG3Threads;
    using LY = G5Layout<P>;
    extern __shared__ uint4 smem5[];
    unsigned char *const base = (unsigned char *)smem5;
    ulonglong2 *const ring = (ulonglong2 *)(base + 2 * LY::bytes);      // [kG3Depth][kG3KS][T]
    __shared__ __align__(8) unsigned long long s_bars[4];                // full[2], empty[2]
    __shared__ volatile int s_abort;
    const int t = threadIdx.x, warp = t >> 5;
    const int nitems = a.n_items[0];
    const unsigned full0 = smem_u32(&s_bars[0]), empty0 = smem_u32(&s_bars[2]);
    if (t == 0) {
        mbar_init(full0, 32);
        mbar_init(full0 + 8, 32);
        mbar_init(empty0, T);
        mbar_init(empty0 + 8, T);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto fail = [&]() {
        s_abort = 1;
        atomicExch(err, 1);
    };

    if (warp == 0) {
        stage_item<P, LY::chunk>(a, base, full0, nitems, err);
        stage_item<P, LY::chunk>(a, base + LY::bytes, full0 + 8, nitems, err);
    }
    for (int k = 0;; k++) {
        const int b = k & 1;
        const unsigned ph = (unsigned)(k >> 1) & 1u;
        if (!mbar_wait(full0 + 8 * b, ph, &s_abort, a.wait_cycles)) {
            fail();
            break;
        }
        const unsigned char *B = base + b * LY::bytes;
        const int4 it = *(const int4 *)(B + LY::item);
        if (it.y < 0) break;
        if (a.jobs[it.w].uniform)
            grid_item<P, T, true>(a, it, (const int4 *)(B + LY::rec), (const float4 *)(B + LY::vis),
                                  (const unsigned short *)(B + LY::runend), ring);
        else
            grid_item<P, T, false>(a, it, (const int4 *)(B + LY::rec), (const float4 *)(B + LY::vis),
                                   (const unsigned short *)(B + LY::runend), ring);
        mbar_arrive(empty0 + 8 * b);
        if (warp == 0) {
            if (!mbar_wait(empty0 + 8 * b, ph, &s_abort, a.wait_cycles)) {
                fail();
                break;
            }
            stage_item<P, LY::chunk>(a, base + b * LY::bytes, full0 + 8 * b, nitems, err);   // item k + 2
        }
    }
}

// ---------------------------------------------------------------------------
// Per-warp streaming gridder (k_grid7).
//
// Every warp works on its own: it takes a job from one ticket counter, grids
// it and takes the next, with no barrier and no wait on another warp.  A job
// is one (work item, part) pair: the item's records (one bin: one support
// bucket of modulus M, at most kG7Chunk records) against one part of the
// item's M x M support box, 128 slots (4 per lane).  Lane l of part w owns
// the slots q = 128 w + 32 j + l (j < 4, q < M^2) at box position
// (a, b) = (q mod M, q / M); for a record with corner (cx, cy) slot (a, b)
// touches cell (cx + (a - cx) mod M, cy + (b - cy) mod M) (Romein's
// assignment), so a slot keeps its cell while the record moves by less than a
// cell and accumulates in registers until the cell changes.  The 32 lanes walk
// the same records in the same order, so every branch on records and runs is
// uniform across the warp.
//
// Pipeline of a job (distances in records; one cp.async group per record):
//   record i + 2D: lanes 0..P copy the record and its visibilities from
//                  global memory into the warp's record ring;
//   record i + D:  every lane copies its slots' taps (each {re, re, im, im},
//                  16 bytes: one shared-memory load feeds both packed FMAs of
//                  a tap and polarisation) into its entries of the tap ring
//                  (zero-fill for a slot outside the record's box);
//   record i:      two packed FMAs per tap and polarisation.
// A slot's cell and table offset change only between runs of records with
// the same corner and support (k_gather flags the first record of a run):
// the look-ahead computes the offsets when it reaches a run's first record and
// leaves the run's cells in a per-lane FIFO, where the accumulation side picks
// them up at the same record and flushes the slots whose cell changes.
//
// Jobs are ordered by segment (image, support bucket), largest support
// first, so the longest jobs are handed out first.
//
// Two shapes (G7Cfg).  Gridder 7: 4 slots per lane (128 per job), each tap
// copied on its own as {re, re, im, im}; 8-warp blocks, 2 per SM.  Gridder 8
// (tap pairs): the 4 slots of a lane are two pairs of neighbouring box
// columns (a, a + 1), whose taps sit side by side in a pair table, so one
// 16-byte copy fetches both (the per-lane tap copies are this kernel's
// measured limit: halving their number made it 21 % faster); the taps stay
// compact {re, im}, the visibilities come as {re, re, im, im} and each slot
// keeps two packed sums (re·{re, im}, im·{re, im} of the tap), combined at
// its flush; 4-warp blocks, 4 per SM (127 registers: the doubled sums fit
// without spilling).  The
// pair table (k_pad_pairs) holds, for every sub-kernel row, the pairs
// (tap 2k, tap 2k + 1) and (tap 2k + 1, tap 2k + 2), so a pair starting at
// any column is one aligned 16-byte entry; the pair at the last column holds
// tap 0 as its second tap, the neighbour of column S - 1 under Romein's wrap,
// which is why gridder 8 needs one support per bucket (the host uses gridder
// 7 otherwise).
template <int KS_, int D_, int WARPS_, int MINB_, bool PAIRS_>
struct G7Cfg {
    static constexpr bool PAIRS = PAIRS_;
    static constexpr int KS = KS_;                       // slots per lane
    static constexpr int D = D_;                         // taps fetched this many records ahead
    static constexpr int Warps = WARPS_;                 // warps per block
    static constexpr int Threads = 32 * WARPS_;
    static constexpr int MinBlocks = MINB_;              // blocks per SM the registers are capped for
    static constexpr int RR = 2 * D_ + 1 <= 8 ? 8 : 16;  // record-ring entries (records fetched 2D ahead)
    static constexpr int NF = PAIRS_ ? KS_ / 2 : KS_;     // tap copies per lane and record
    static constexpr int PartSlots = 32 * KS_;           // slots of one job
    static constexpr int TapStride = D_ * KS_ * 32;      // tap-ring / FIFO entries per warp
    static_assert(RR >= 2 * D_ + 1, "the record ring holds every record in flight");
    static_assert((D_ & (D_ - 1)) == 0, "ring indices are masked");
};
using G7Narrow = G7Cfg<4, 4, 8, 2, false>;   // gridder 7
using G7Pairs = G7Cfg<4, 4, 4, 4, true>;     // gridder 8, the default
static const int kG7Chunk = 512;       // records of one work item

// Jobs [job0, next.job0) are items [item0, item0 + n) x wu parts of modulus m.
struct G7Segment {
    int job0, item0, wu, m;
};

struct Grid7Args {
    const int4 *items;        // work items; item.w selects the image
    const G7Segment *segs;    // n_segs + 1 entries, the last holding the total job count
    const int *n_segs;
    int *counter;             // job tickets
    GridJobDesc jobs[kMaxBatch];
};

// Where the segments of a launch come from: per image, its bucket item ranges
// (k_bucket_bounds), its item count and its bucket moduli.
struct G7SegSrc {
    const int *bounds[kMaxBatch];
    const int *n_items[kMaxBatch];   // null: the image has no records
    const int *M[kMaxBatch];
};

// One block of kMaxBuckets threads: the segments of every image in image
// order (the order of the concatenated item list), buckets by descending
// modulus within an image.
// pairs: jobs hold 64 column pairs ((M + 1) / 2 per box row) instead of 128 slots.
__global__ void k_g7_segments(G7SegSrc src, int nimages, int pairs, G7Segment *__restrict__ segs,
                              int *__restrict__ n_segs) {
    using Scan = cub::BlockScan<int, kMaxBuckets>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ int s_nseg, s_job0, s_base;
    const int t = threadIdx.x;
    const int bb = kMaxBuckets - 1 - t;       // this thread's bucket
    if (t == 0) s_nseg = s_job0 = s_base = 0;
    __syncthreads();
    for (int j = 0; j < nimages; j++) {
        const int ni = src.n_items[j] ? *src.n_items[j] : 0;
        int cnt = 0, m = 0, lo = 0;
        if (ni > 0) {
            lo = src.bounds[j][2 * bb];
            cnt = src.bounds[j][2 * bb + 1] - lo;
            m = src.M[j][bb];
            if (m <= 0 || cnt <= 0) cnt = 0;
        }
        const int wu = cnt ? (pairs ? (((m + 1) >> 1) * m + 63) / 64 : (m * m + 127) / 128) : 0;
        int idx, njob, aggr_seg, aggr_job;
        Scan(tmp).ExclusiveSum(cnt ? 1 : 0, idx, aggr_seg);
        __syncthreads();
        Scan(tmp).ExclusiveSum(cnt * wu, njob, aggr_job);
        if (cnt) {
            G7Segment g;
            g.job0 = s_job0 + njob;
            g.item0 = s_base + lo;
            g.wu = wu;
            g.m = m;
            segs[s_nseg + idx] = g;
        }
        __syncthreads();
        if (t == 0) {
            s_nseg += aggr_seg;
            s_job0 += aggr_job;
            s_base += ni;
        }
        __syncthreads();
    }
    if (t == 0) {
        G7Segment g;
        g.job0 = s_job0;
        g.item0 = s_base;
        g.wu = 1;
        g.m = 0;
        segs[s_nseg] = g;
        *n_segs = s_nseg;
    }
}

__device__ __forceinline__ void cp_async16_s(unsigned smem_addr, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr), "l"(gmem) : "memory");
}

// Runs of the direct layout within each work item: the first record of every
// run (a record whose corner or support differs from the previous record of
// the item, and the item's first record) gets the run's length in bits 16-31
// of wpos.w (bits 0-15 hold the support).  One warp per item; items hold at
// most kG7Chunk records.
__global__ void k_mark_runs(const int4 *__restrict__ items, const int *__restrict__ n_items, int4 *__restrict__ wpos) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nit = *n_items;
    for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < nit; v += nwarps) {
        const int4 it = items[v];
        int4 *const w = wpos + it.x;
        const int N = it.y;
        int next = N;                              // first run start after the current group
        for (int g = ((N - 1) >> 5) << 5; g >= 0; g -= 32) {
            const int k = g + lane;
            bool st = false;
            int4 r = make_int4(0, 0, 0, 0);
            if (k < N) {
                r = w[k];
                st = k == 0;
                if (!st) {
                    const int4 q = w[k - 1];
                    st = q.x != r.x || (q.w & 0xFFFF) != (r.w & 0xFFFF);
                }
            }
            const unsigned m = __ballot_sync(0xFFFFFFFFu, st);
            const unsigned above = lane == 31 ? 0u : m & (0xFFFFFFFFu << (lane + 1));
            const int nxt = above ? g + __ffs(above) - 1 : next;
            __syncwarp();                          // every lane has read w[k - 1] before it is rewritten
            if (k < N) w[k].w = (r.w & 0xFFFF) | (st ? (nxt - k) << 16 : 0);
            if (m) next = g + __ffs(m) - 1;
        }
    }
}

// One job of this warp.  tring / fifo: this lane's first tap-ring and FIFO
// entry (entry (d, j) is (d * KS + j) * 32 entries further on); rring: the
// warp's record ring (entry e: the record, then its P visibilities).
// UNIFORM: every record's support equals the modulus M (one support per
// bucket), so a slot inside the box is inside every record's box.
// EXACT: flushes go to the FP64 delta grid, otherwise to the FP32 grid.
//
// The record loop is cut at run starts of both pipeline sides: the first
// record of a run on the accumulation side (flush the slots whose cell
// changes) and the record whose fetch opens a run on the look-ahead side (new
// table offsets).  Between those points the loop holds no branch and no
// conditional update of the accumulators.
template <class C, int P, bool UNIFORM, bool EXACT>
__device__ __forceinline__ void grid_job7(const GridJobDesc &J, const int first, const int N, const int M,
                                          const int part, float4 *tring, int *fifo, float4 *rring) {
    constexpr int KS = C::KS, D = C::D, RR = C::RR, E = 1 + P, NF = C::NF;
    constexpr bool PR = C::PAIRS;
    static_assert(!PR || UNIFORM, "tap pairs need one support per bucket");
    const int lane = threadIdx.x & 31;
    const float4 *const tab = J.table2;
    float *const ggrid = EXACT ? nullptr : J.grid;
    double *const gdelta = EXACT ? J.dgrid : nullptr;
    const int gnx = J.nx;
    const int MM = M * M;
    // box position (qa, qb) of every slot of this lane; qb = -1: no slot
    int qa[KS], qb[KS];
    int nb[NF];                  // bytes of each tap copy: 16, 8 (a pair's second column is off the box), 0
    if constexpr (PR) {
        // pair jp: box columns (2 pc, 2 pc + 1) of box row b, (M + 1) / 2 pairs per row
        const int PW = (M + 1) >> 1;
#pragma unroll
        for (int jp = 0; jp < NF; jp++) {
            const int pq = part * (32 * NF) + jp * 32 + lane;
            const int b = pq / PW;
            const int pc = pq - b * PW;
            const bool in = b < M, two = 2 * pc + 1 < M;
            qa[2 * jp] = 2 * pc;
            qb[2 * jp] = in ? b : -1;
            qa[2 * jp + 1] = 2 * pc + 1;
            qb[2 * jp + 1] = in && two ? b : -1;
            nb[jp] = in ? (two ? 16 : 8) : 0;
        }
    } else {
#pragma unroll
        for (int j = 0; j < KS; j++) {
            const int q = part * C::PartSlots + j * 32 + lane;
            const int b = q / M;
            qa[j] = q - b * M;
            qb[j] = q < MM ? b : -1;
            nb[j] = q < MM ? 16 : 0;
        }
    }
    // record ring: lane 0 copies the record, lanes 1..P its visibilities
    const int rflag = lane <= P ? 1 : 0;
    const char *const rsrc = lane == 0 ? (const char *)(J.wpos + first)
                                       : (const char *)(J.wvis4 + (size_t)first * P + (lane <= P ? lane - 1 : 0));
    const int rsh = lane == 0 ? 4 : (P == 4 ? 6 : (P == 2 ? 5 : 4));   // log2 of the bytes per record of the source
    const unsigned rdst = (unsigned)__cvta_generic_to_shared(rring) + (unsigned)lane * 16;
    auto rfetch = [&](int r) {
        asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %2, 0;\n @p cp.async.cg.shared.global [%0], [%1], 16;\n}" ::"r"(
                         rdst + (unsigned)((r & (RR - 1)) * E) * 16),
                     "l"(rsrc + ((size_t)r << rsh)), "r"(rflag)
                     : "memory");
    };
    auto rec = [&](int k) { return *(const int4 *)(rring + (k & (RR - 1)) * E); };
    // look-ahead: source of every tap copy for the run being fetched
    const float4 *src[NF];
    auto pgeom = [&](int k, const int4 r) {   // record k opens a run: geometry of its slots
        const int rxm = r.y & 0xFFFF, rym = r.y >> 16, S = r.w & 0xFFFF;
        int *const f = fifo + (k & (D - 1)) * KS * 32;
        if constexpr (PR) {
            // pair table row: (S + 1) / 2 pairs starting at even columns, then
            // (S + 1) / 2 starting at odd columns (S == M)
#pragma unroll
            for (int jp = 0; jp < NF; jp++) {
                int sx = qa[2 * jp] + rxm;
                sx -= (sx >= M) ? M : 0;
                int sy = qb[2 * jp] + rym;
                sy -= (sy >= M) ? M : 0;
                int sx1 = sx + 1;
                sx1 -= (sx1 >= M) ? M : 0;
                const bool ok = qb[2 * jp] >= 0;
                src[jp] = tab + (ok ? sy * (S + 1) + (sx & 1) * ((S + 1) >> 1) + (sx >> 1) : 0);
                f[2 * jp * 32] = ok ? r.x + sy * gnx + sx : -1;
                f[(2 * jp + 1) * 32] = qb[2 * jp + 1] >= 0 ? r.x + sy * gnx + sx1 : -1;
            }
            return;
        }
#pragma unroll
        for (int j = 0; j < KS; j++) {
            int sx = qa[j] + rxm;
            sx -= (sx >= M) ? M : 0;
            int sy = qb[j] + rym;
            sy -= (sy >= M) ? M : 0;
            const bool ok = qb[j] >= 0 && (UNIFORM || (sx < S && sy < S));
            src[j] = tab + (ok ? sy * (S + 1) + sx : 0);
            if (!UNIFORM) nb[j] = ok ? 16 : 0;
            f[j * 32] = ok ? r.x + sy * gnx + sx : -1;
        }
    };
    const unsigned tdst = (unsigned)__cvta_generic_to_shared(tring);
    auto tfetch = [&](int k, int z) {
        const unsigned d = tdst + (unsigned)((k & (D - 1)) * KS * 32) * 16;
#pragma unroll
        for (int j = 0; j < NF; j++) {
            const bool in = in_bounds((long long)(src[j] - tab) + z, J.table2_elems, kSiteTapStreaming);
            cp_async16_zfill_n(d + j * 32 * 16, in ? src[j] + z : tab, in ? nb[j] : 0);
        }
    };
    // prologue: records 0 .. 2D-1, then the taps of records 0 .. D-1
#pragma unroll 1
    for (int r = 0; r < 2 * D; r++) {
        if (r < N) rfetch(r);
        cp_async_commit();
    }
    cp_async_wait<D>();        // records 0 .. D-1 have landed (this lane's copies)
    __syncwarp();              // ... and every lane's
    int pend = 0;              // next record whose fetch opens a run
#pragma unroll 1
    for (int k = 0; k < D; k++) {
        if (k < N) {
            const int4 r = rec(k);
            if (k == pend) {
                pgeom(k, r);
                pend = k + max(1, r.w >> 16);
            }
            tfetch(k, r.z);
        }
        cp_async_commit();
    }
    int last[KS];
    float2 acc[KS][P];
    float2 accb[PR ? KS : 1][P];   // tap pairs: the sums of {re, im} of the tap times im of the visibility
#pragma unroll
    for (int j = 0; j < KS; j++) {
        last[j] = -1;
#pragma unroll
        for (int p = 0; p < P; p++) {
            acc[j][p] = make_float2(0.f, 0.f);
            if (PR) accb[PR ? j : 0][p] = make_float2(0.f, 0.f);
        }
    }
    // slot j's sums as {re, im} per polarisation, flushed to its last cell
    auto flush_slot = [&](int j) {
        if constexpr (PR) {
            float2 v[P];
#pragma unroll
            for (int p = 0; p < P; p++)
                v[p] = make_float2(acc[j][p].x - accb[j][p].y, accb[j][p].x + acc[j][p].y);
            flush2<P>(ggrid, gdelta, last[j], J.cells, v);
        } else {
            flush2<P>(ggrid, gdelta, last[j], J.cells, acc[j]);
        }
    };
    // One record: accumulate record i (two packed FMAs per tap and
    // polarisation; ConvolutionGridder.cu:153-181: to += vis * wt, no
    // conjugate); TAP: fetch the taps of record i + D; REC: refill the record
    // ring with record i + 2D.
    auto step = [&](const int i, auto TAP, auto REC) {
        cp_async_wait<D - 1>();     // taps of record i and record i + D have landed (this lane's copies)
        __syncwarp();               // ... and every lane's
        const float4 *ent = rring + (i & (RR - 1)) * E;
        float2 vp[P], wp[P];
#pragma unroll
        for (int p = 0; p < P; p++) {
            const float4 q = ent[1 + p];
            vp[p] = make_float2(q.x, q.y);
            wp[p] = make_float2(q.z, q.w);
        }
        const float4 *c4 = tring + (i & (D - 1)) * KS * 32;
        if constexpr (PR) {
            // visibilities {re, re, im, im}: vp = (re, re), wp = (im, im)
#pragma unroll
            for (int jp = 0; jp < NF; jp++) {
                const float4 c = c4[jp * 32];
                const float2 t0 = make_float2(c.x, c.y), t1 = make_float2(c.z, c.w);
#pragma unroll
                for (int p = 0; p < P; p++) {
                    acc[2 * jp][p] = __ffma2_rn(t0, vp[p], acc[2 * jp][p]);
                    accb[2 * jp][p] = __ffma2_rn(t0, wp[p], accb[2 * jp][p]);
                    acc[2 * jp + 1][p] = __ffma2_rn(t1, vp[p], acc[2 * jp + 1][p]);
                    accb[2 * jp + 1][p] = __ffma2_rn(t1, wp[p], accb[2 * jp + 1][p]);
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < KS; j++) {
                const float4 c = c4[j * 32];
                const float2 cre = make_float2(c.x, c.y), cim = make_float2(c.z, c.w);
#pragma unroll
                for (int p = 0; p < P; p++) {
                    acc[j][p] = __ffma2_rn(cre, vp[p], acc[j][p]);
                    acc[j][p] = __ffma2_rn(cim, wp[p], acc[j][p]);
                }
            }
        }
        if (decltype(TAP)::value) tfetch(i + D, rec(i + D).z);
        if (decltype(REC)::value) rfetch(i + 2 * D);
        cp_async_commit();
    };
    using T_ = std::true_type;
    using F_ = std::false_type;
    int i = 0, cend = 0;
    while (i < N) {
        cp_async_wait<D - 1>();     // taps of record i and record i + D have landed
        __syncwarp();
        if (i == cend) {
            // record i opens a run: flush the slots whose cell changes
            const int *f = fifo + (i & (D - 1)) * KS * 32;
            int cell[KS];
            bool chg = false;
#pragma unroll
            for (int j = 0; j < KS; j++) {
                cell[j] = f[j * 32];
                chg |= cell[j] >= 0 && cell[j] != last[j];
            }
            if (chg) {
#pragma unroll
                for (int j = 0; j < KS; j++)
                    if (cell[j] >= 0 && cell[j] != last[j] && last[j] >= 0) flush_slot(j);
            }
            // Reset of the flushed slots by a packed multiply with 0 (1 keeps
            // the sum), so the accumulators keep their registers through the
            // loop (an assignment under the branch above made the compiler
            // copy every accumulator once per record; a select instead of the
            // multiply measured 3.8 % slower).  It differs from an assignment
            // only for a non-finite sum, which has already gone to the grid,
            // where the inverse FFT spreads it over the whole image either
            // way.  Skipped, warp-uniformly, when no lane's cell changes (a
            // run that moves only across box rows the warp does not hold):
            // 1.5 % faster on the 8 h mid-size channel.
            if (__any_sync(0xFFFFFFFFu, chg)) {
#pragma unroll
                for (int j = 0; j < KS; j++) {
                    const bool c = cell[j] >= 0 && cell[j] != last[j];
                    const float kf = c ? 0.f : 1.f;
#pragma unroll
                    for (int p = 0; p < P; p++) {
                        acc[j][p] = __fmul2_rn(acc[j][p], make_float2(kf, kf));
                        if (PR) accb[PR ? j : 0][p] = __fmul2_rn(accb[PR ? j : 0][p], make_float2(kf, kf));
                    }
                    last[j] = c ? cell[j] : last[j];
                }
            }
            cend = i + max(1, rec(i).w >> 16);
        }
        if (i + D < N) {
            if (i + D == pend) {
                const int4 r = rec(i + D);
                pgeom(i + D, r);
                pend = i + D + max(1, r.w >> 16);
            }
            // records whose accumulation and look-ahead meet no run start
            int stop = cend < pend - D ? cend : pend - D;
            if (i + 2 * D < N) {
                stop = stop < N - 2 * D ? stop : N - 2 * D;
                #pragma unroll 1
                for (; i < stop; ++i) step(i, T_{}, T_{});
            } else {
                stop = stop < N - D ? stop : N - D;
                #pragma unroll 1
                for (; i < stop; ++i) step(i, T_{}, F_{});
            }
        } else {
            #pragma unroll 1
            for (; i < cend; ++i) step(i, F_{}, F_{});
        }
    }
    cp_async_wait<0>();
    __syncwarp();              // the rings are reused by the next job
#pragma unroll
    for (int j = 0; j < KS; j++)
        if (last[j] >= 0) flush_slot(j);
}

template <class C, int P, bool UNIFORM, bool EXACT>
__global__ void __launch_bounds__(C::Threads, C::MinBlocks) k_grid7(Grid7Args a) {
    constexpr int E = 1 + P, TS = C::TapStride;
    extern __shared__ float4 smem7[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float4 *const tring = smem7 + warp * TS + lane;                                  // [warp][D][KS][32]
    int *const fifo = (int *)(smem7 + C::Warps * TS) + warp * TS + lane;             // [warp][D][KS][32]
    float4 *const rring = smem7 + C::Warps * TS + C::Warps * TS / 4 + warp * C::RR * E;   // [warp][RR][E]
    const int nsegs = *a.n_segs;
    const int total = a.segs[nsegs].job0;
    int seg = 0;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(a.counter, 1);
        t = __shfl_sync(0xFFFFFFFFu, t, 0);
        if (t >= total) break;
        while (a.segs[seg + 1].job0 <= t) seg++;      // a warp's tickets only grow
        const G7Segment g = a.segs[seg];
        const int rel = t - g.job0;
        const int k = rel / g.wu;
        const int4 it = a.items[g.item0 + k];
        grid_job7<C, P, UNIFORM, EXACT>(a.jobs[it.w], it.x, it.y, g.m, rel - k * g.wu, tring, fifo, rring);
    }
}

template <class C, int P>
static size_t grid7_smem() {
    return (size_t)C::Warps * (C::TapStride * (sizeof(float4) + sizeof(int)) + C::RR * (1 + P) * sizeof(float4));
}

// UNIFORM kernel when every image of the launch has one support per bucket
// (always, for the tap-pair shape: the host chooses it only then)
template <class C, int P>
static int launch_grid7c(const Grid7Args &a, cudaStream_t st) {
    bool uniform = true;
    for (int j = 0; j < kMaxBatch && a.jobs[j].wpos; j++) uniform = uniform && a.jobs[j].uniform;
    const bool exact = a.jobs[0].dgrid != nullptr;
    void (*kern)(Grid7Args);
    if constexpr (C::PAIRS) {
        if (!uniform) return MTB_ERR_BAD_PARAM;
        kern = exact ? k_grid7<C, P, true, true> : k_grid7<C, P, true, false>;
    } else {
        kern = uniform ? (exact ? k_grid7<C, P, true, true> : k_grid7<C, P, true, false>)
                       : (exact ? k_grid7<C, P, false, true> : k_grid7<C, P, false, false>);
    }
    const size_t smem = grid7_smem<C, P>();
    MTB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    MTB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::Threads, smem));
    if (per_sm < 1) return MTB_ERR_BAD_SHAPE;
    kern<<<per_sm * sm_count(), C::Threads, smem, st>>>(a);
    MTB_LAUNCHED();
    return MTB_OK;
}

// pairs: the tap-pair shape (gridder 8, one support per bucket), else gridder 7
template <int P>
static int launch_grid7(const Grid7Args &a, bool pairs, cudaStream_t st) {
    return pairs ? launch_grid7c<G7Pairs, P>(a, st) : launch_grid7c<G7Narrow, P>(a, st);
}

template <int P>
static size_t grid5_smem() {
    return 2 * G5Layout<P>::bytes + (size_t)kG3Depth * kG3KS * kG3Threads * 16;
}

template <int P>
static int launch_grid5(const Grid2Args &a, int *err, cudaStream_t st) {
    auto kern = k_grid5<P>;
    const size_t smem = grid5_smem<P>();
    MTB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    MTB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kG3Threads, smem));
    if (per_sm < 1) return MTB_ERR_BAD_SHAPE;
    kern<<<per_sm * sm_count(), kG3Threads, smem, st>>>(a, err);
    MTB_LAUNCHED();
    return MTB_OK;
}

__global__ void k_set_moduli(BucketTable bt, int *__restrict__ M) {
    for (int b = threadIdx.x; b < kMaxBuckets; b += blockDim.x) M[b] = bt.M[b];
}

__global__ void k_merge_delta32(float4 *__restrict__ hi, float4 *__restrict__ lo, const float4 *__restrict__ delta,
                                size_t n4) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
        const float4 d = delta[i];
        if (d.x == 0.f && d.y == 0.f && d.z == 0.f && d.w == 0.f) continue;
        float4 h = hi[i], e = lo[i];
        float sx, bp;
        sx = h.x + d.x; bp = sx - h.x; e.x += (h.x - (sx - bp)) + (d.x - bp); h.x = sx;
        sx = h.y + d.y; bp = sx - h.y; e.y += (h.y - (sx - bp)) + (d.y - bp); h.y = sx;
        sx = h.z + d.z; bp = sx - h.z; e.z += (h.z - (sx - bp)) + (d.z - bp); h.z = sx;
        sx = h.w + d.w; bp = sx - h.w; e.w += (h.w - (sx - bp)) + (d.w - bp); h.w = sx;
        hi[i] = h;
        lo[i] = e;
    }
}

// the last complex value when the float count is not a multiple of 4 (npol 1)
__global__ void k_merge_delta32_tail(float2 *hi, float2 *lo, const float2 *delta, size_t i) {
    const float2 d = delta[i];
    float2 h = hi[i], e = lo[i];
    float sx, bp;
    sx = h.x + d.x; bp = sx - h.x; e.x += (h.x - (sx - bp)) + (d.x - bp); h.x = sx;
    sx = h.y + d.y; bp = sx - h.y; e.y += (h.y - (sx - bp)) + (d.y - bp); h.y = sx;
    hi[i] = h;
    lo[i] = e;
}

// FP64 delta grid (exact_delta = 1)
__global__ void k_merge_delta(float2 *__restrict__ hi, float2 *__restrict__ lo, const double2 *__restrict__ delta,
                              size_t n2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n2; i += (size_t)gridDim.x * blockDim.x) {
        const double2 d = delta[i];
        if (d.x == 0.0 && d.y == 0.0) continue;
        const float2 h = hi[i], e = lo[i];
        // (hi + lo) + delta in FP64, split back into a float pair
        const double tx = ((double)h.x + (double)e.x) + d.x, ty = ((double)h.y + (double)e.y) + d.y;
        const float hx = (float)tx, hy = (float)ty;
        hi[i] = make_float2(hx, hy);
        lo[i] = make_float2((float)(tx - (double)hx), (float)(ty - (double)hy));
    }
}

// ------------------------------------------------------------ host side --
struct GridPlan {
    BucketTable bt;
    int chunk;
    int ncap;        // record capacity of per-record arrays
    int table_rows;  // kernel rows (S taps each) of all planes: sum of T*T*S
};

struct GridSpace {
    int4 *pos;
    int *meta;
    unsigned *keys, *skeys;
    int *iota, *sidx;
    unsigned *ukeys;
    int *counts, *run_start, *nchunks, *item_start, *num_runs, *n_items;
    int4 *items;
    int *bounds, *counters;
    int4 *wpos;
    float2 *wvis;
    double *norm_acc;
    unsigned long long *stats;
    void *cub;
    size_t cub_bytes;
    float4 *table2;      // padded table with each tap as {re, re, im, im} (k_grid3)
    size_t table2_elems;
    int *pbase;          // first padded element, then first row, of every plane (k_pad_bases)
    int *moduli;         // bucket moduli of the plan (device copy)
    int *err;            // gridder pipeline error flag
    double *delta;       // this call's grid contribution (compensated mode; FP64 or FP32)
    G7Segment *segs;     // k_grid7 job segments (kMaxBuckets + 1)
    int *n_segs;
    int *counter7;       // k_grid7 job tickets
};

static size_t cub_bytes(int n) {
    size_t a = 0, b = 0, c = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, a, (unsigned *)nullptr, (unsigned *)nullptr, (int *)nullptr,
                                    (int *)nullptr, n);
    cub::DeviceRunLengthEncode::Encode(nullptr, b, (unsigned *)nullptr, (unsigned *)nullptr, (int *)nullptr,
                                       (int *)nullptr, n);
    cub::DeviceScan::ExclusiveSum(nullptr, c, (int *)nullptr, (int *)nullptr, n);
    return std::max(a, std::max(b, c));
}

// delta_bytes: bytes of the per-call delta grid (0: none)
static void carve_grid(Arena &A, int R, int P, int chunk, size_t table_elems, size_t delta_bytes, GridSpace *s,
                       int nw = 1) {
    size_t n = (size_t)(R > 0 ? R : 1);
    size_t nitems = n + n / (size_t)chunk + 2;
    s->pos = A.take<int4>(n);
    s->meta = A.take<int>(n);
    s->keys = A.take<unsigned>(n);
    s->skeys = A.take<unsigned>(n);
    s->iota = A.take<int>(n);
    s->sidx = A.take<int>(n);
    s->ukeys = A.take<unsigned>(n);
    s->counts = A.take<int>(n);
    s->run_start = A.take<int>(n);
    s->nchunks = A.take<int>(n);
    s->item_start = A.take<int>(n);
    s->num_runs = A.take<int>(1);
    s->n_items = A.take<int>(1);
    s->items = A.take<int4>(nitems);
    s->bounds = A.take<int>(2 * kMaxBuckets);
    s->counters = A.take<int>(kMaxBuckets);
    s->wpos = A.take<int4>(n);
    s->wvis = A.take<float2>(n * P * 2);   // float4 per pol for the direct gridder
    s->norm_acc = A.take<double>(4);
    s->stats = A.take<unsigned long long>(4);
    s->cub_bytes = cub_bytes((int)n);
    s->cub = A.take<char>(s->cub_bytes);
    s->table2 = A.take<float4>(table_elems ? table_elems : 1);
    s->table2_elems = table_elems;
    s->pbase = A.take<int>(2 * (nw > 0 ? nw : 1) + 1);
    s->moduli = A.take<int>(kMaxBuckets);
    s->err = A.take<int>(1);
    s->delta = A.take<double>(delta_bytes ? (delta_bytes + sizeof(double) - 1) / sizeof(double) : 1);
    s->segs = A.take<G7Segment>(kMaxBuckets + 1);
    s->n_segs = A.take<int>(1);
    s->counter7 = A.take<int>(1);
}

// float2 elements of the kernel table described by conv_info
static size_t table_elems_of(const mtb_grid_params *p, const int *h_conv_info) {
    size_t T = (size_t)oversample_T(p->sampling), n = 0;
    for (int k = 0; k < p->wplanes; k++) {
        size_t S = (size_t)(h_conv_info[2 * k] > 0 ? h_conv_info[2 * k] : 0);
        n = std::max(n, (size_t)(h_conv_info[2 * k + 1] > 0 ? h_conv_info[2 * k + 1] : 0) + T * T * S * S);
    }
    return n;
}

// float2 elements of the row-padded table (rows of S + 1 taps)
static size_t padded_elems_of(const mtb_grid_params *p, const int *h_conv_info) {
    size_t T = (size_t)oversample_T(p->sampling), n = 0;
    for (int k = 0; k < p->wplanes; k++) {
        size_t S = (size_t)(h_conv_info[2 * k] > 0 ? h_conv_info[2 * k] : 0);
        n += T * T * S * (S + 1);
    }
    return n;
}

// records per work item: the direct gridder stages a whole item in shared memory
// The direct gridder a call uses: gridder 0 selects the default, the
// rolling-items k_grid5, unless 512-thread blocks are asked for (k_grid3 only).
// A stream under CUDA-graph capture cannot be synchronised: the debug
// read-back of the gridder's error flag is skipped there.
static bool capturing(cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

// Wait bound of the rolling-items gridder's mbarrier waits: kWaitCycles, or
// the MTB_GRIDDER_WAIT_CYCLES environment variable (read at every call, so a
// test can make the waits run out and then restore the default).
static long long wait_cycles() {
    const char *e = std::getenv("MTB_GRIDDER_WAIT_CYCLES");
    if (!e || !e[0]) return kWaitCycles;
    const long long v = std::atoll(e);
    return v >= 0 ? v : kWaitCycles;
}

static int gridder_of(const mtb_grid_params *p) {
    if (p->gridder != 0) return p->gridder;
    if (p->gridder_threads == 512) return 3;
    return 8;
}

// The per-warp streaming gridders (k_grid7 in its two shapes).
static bool streaming(int which) { return which == 7 || which == 8; }

// The tap-pair shape runs when it is asked for and every record's support is
// its bucket's modulus (one support per bucket); otherwise gridder 7 does.
static bool pairs_of(const mtb_grid_params *p) {
    return p->merge != 1 && gridder_of(p) == 8 && p->support_bucket <= 1;
}

// Work items shorter than this many records multiply the flushes into each
// cell: with the FP32 per-call delta grid, 37-record items took the first
// configuration's image error to 1.2e-5 of its peak (above the 1e-5 bound),
// so shorter items always accumulate the call in the FP64 delta grid.
static const int kSafeChunk = 128;

// The call's delta grid is FP64: asked for (exact_delta), or forced by short items.
static bool exact_of(const mtb_grid_params *p) {
    return p->exact_delta != 0 || (p->max_chunk > 0 && p->max_chunk < kSafeChunk);
}

// Bytes of the per-call delta grid a call reserves per grid cell and
// polarisation: none when the calls pass no grid_lo (no_grid_lo) or merge in
// shared memory (merge = 1, which writes (grid, grid_lo) itself), 8 for the
// FP32 delta, 16 for the FP64 one.
static size_t delta_bytes_per_cell_pol(const mtb_grid_params *p) {
    if (p->no_grid_lo || p->merge == 1) return 0;
    return exact_of(p) ? 2 * sizeof(double) : 2 * sizeof(float);
}

// Bytes of the delta grid the call needs, and those its workspace holds (none
// when the caller passes its own: external_delta).
static size_t delta_bytes(const mtb_grid_params *p) {
    return (size_t)p->nx * p->ny * p->npol * delta_bytes_per_cell_pol(p);
}
static size_t workspace_delta_bytes(const mtb_grid_params *p) { return p->external_delta ? 0 : delta_bytes(p); }



static int effective_chunk(const mtb_grid_params *p) {
    int c = p->max_chunk > 0 ? p->max_chunk : kDefaultChunk;
    if (p->merge != 1 && c > kG3Chunk) c = kG3Chunk;
    if (p->merge != 1 && gridder_of(p) == 5 && c > kG5Chunk) c = kG5Chunk;
    if (p->merge != 1 && streaming(gridder_of(p)) && c > kG7Chunk) c = kG7Chunk;
    return c;
}

static int check_params(const mtb_grid_params *p) {
    if (!p) return MTB_ERR_NULL;
    if (p->npol != 1 && p->npol != 2 && p->npol != 4) return MTB_ERR_BAD_SHAPE;
    if (p->nx < 2 || p->ny < 2 || p->sampling < 1 || p->wplanes < 1) return MTB_ERR_BAD_PARAM;
    if ((size_t)p->nx * p->ny > ((size_t)1 << 31)) return MTB_ERR_BAD_SHAPE;
    if (!(p->u_increment > 0.0) || !(p->v_increment > 0.0) || !(p->w_sq_increment > 0.0)) return MTB_ERR_BAD_PARAM;
    if (p->tile < 0 || p->support_bucket < 0 || p->max_chunk < 0) return MTB_ERR_BAD_PARAM;
    if (p->merge < 0 || p->merge > 2) return MTB_ERR_BAD_PARAM;
    if (p->flags_u8 < 0 || p->flags_u8 > 2) return MTB_ERR_BAD_PARAM;
    if (p->bulk_min_support != 0) return MTB_ERR_BAD_PARAM;   // reserved (no bulk-copy gridder)
    if (p->gridder_threads != 0 && p->gridder_threads != 256 && p->gridder_threads != 512) return MTB_ERR_BAD_PARAM;
    if (p->gridder != 0 && p->gridder != 3 && p->gridder != 5 && !streaming(p->gridder)) return MTB_ERR_BAD_PARAM;
    if ((p->gridder == 5 || streaming(p->gridder)) && p->gridder_threads == 512) return MTB_ERR_BAD_PARAM;
    return MTB_OK;
}

static int make_plan(const mtb_grid_params *p, const int *h_conv_info, GridPlan *g) {
    int half = p->support_bucket > 0 ? p->support_bucket : 1;
    int tile = p->tile > 0 ? p->tile : kDefaultTile;
    g->chunk = effective_chunk(p);
    if (tile < 4 || p->nx / tile >= 4096 || p->ny / tile >= 4096) return MTB_ERR_BAD_PARAM;
    std::memset(&g->bt, 0, sizeof(g->bt));
    g->bt.half = half;
    const long long T = oversample_T(p->sampling);
    long long rows = 0;
    for (int k = 0; k < p->wplanes; k++) {
        int S = h_conv_info[2 * k];
        rows += T * T * S;
        // the direct gridders lay one support-box column per thread of a
        // 256-thread block: supports up to 255
        if (S < 1 || S % 2 == 0 || S > 255 || S >= p->nx || S >= p->ny) return MTB_ERR_KERNEL;
        int b = (S - 1) / (2 * half);
        if (b >= kMaxBuckets) return MTB_ERR_BAD_PARAM;
        g->bt.M[b] = std::max(g->bt.M[b], S);
        g->bt.n = std::max(g->bt.n, b + 1);
    }
    for (int b = 0; b < kMaxBuckets; b++) g->bt.tile[b] = tile;
    // bits that hold 0..v
    auto bits = [](int v) { int n = 0; while (n < 31 && (1 << n) <= v) n++; return n; };
    g->bt.xbits = bits((p->nx - 1) / tile);   // corners stay below nx - S, ny - S
    g->bt.ybits = bits((p->ny - 1) / tile);
    g->bt.bbits = bits(g->bt.n);              // bucket numbers stay below 2^bbits - 1
    if (rows > 0x7FFFFFFFLL) return MTB_ERR_BAD_SHAPE;
    g->table_rows = (int)rows;
    return MTB_OK;
}

struct Launch {
    int kmax, rows, nbands, threads;
    bool window;
    size_t smem;
};

static Launch launch_shape(int M, int P, int tile, int merge) {
    Launch L;
    if (M <= 16) L.kmax = 1;
    else if (M <= 32) L.kmax = 2;
    else L.kmax = 8;
    int rows = (M + L.kmax - 1) / L.kmax;
    int maxrows = std::max(1, (L.kmax == 8 ? 576 : 1024) / M);
    L.rows = std::min(rows, maxrows);
    L.nbands = (M + L.rows * L.kmax - 1) / (L.rows * L.kmax);
    L.threads = M * L.rows;
    size_t stage = kStage * (sizeof(int4) + 2 * P * sizeof(float));
    size_t W = (size_t)tile + M - 1;
    size_t wbytes = ((W * W * 2 * P + 3) & ~(size_t)3) * sizeof(float);
    L.window = (merge == 1) && (L.nbands == 1) && (wbytes + stage <= kWindowSmemLimit);
    L.smem = (L.window ? wbytes : 0) + stage;
    return L;
}

template <int P, int KMAX, bool WIN>
static int launch_one(const GridArgs &a, const Launch &L, cudaStream_t st) {
    auto kern = k_grid<P, KMAX, WIN>;
    if (L.smem > 48 * 1024)
        MTB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem));
    int per_sm = 0;
    MTB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, L.threads, L.smem));
    if (per_sm < 1) return MTB_ERR_BAD_SHAPE;
    int blocks = per_sm * sm_count();
    kern<<<blocks, L.threads, L.smem, st>>>(a);
    MTB_LAUNCHED();
    return MTB_OK;
}

template <int P>
static int launch_bucket(GridArgs a, const Launch &L, cudaStream_t st) {
    a.rows = L.rows;
    a.nbands = L.nbands;
    if (L.kmax == 1) return L.window ? launch_one<P, 1, true>(a, L, st) : launch_one<P, 1, false>(a, L, st);
    if (L.kmax == 2) return L.window ? launch_one<P, 2, true>(a, L, st) : launch_one<P, 2, false>(a, L, st);
    return L.window ? launch_one<P, 8, true>(a, L, st) : launch_one<P, 8, false>(a, L, st);
}

// MTB_CHECK_GRIDDER=1: every mtb_grid call synchronises its stream and reports
// a gridder pipeline timeout as MTB_ERR_KERNEL (a debugging aid; off by default).
static bool check_gridder() {
    static int v = -1;
    if (v < 0) {
        const char *e = std::getenv("MTB_CHECK_GRIDDER");
        v = (e && e[0] && e[0] != '0') ? 1 : 0;
    }
    return v == 1;
}

// k_preprocess / k_gather with the caller's flag layout: int32 (the
// reference's layout), bytes or bits (mtb_grid_params.flags_u8 = 0, 1, 2).
template <int P, typename FR>
static void launch_preprocess_fr(const mtb_grid_params *p, int blocks, cudaStream_t st, int R, const float *uvw,
                                 const float *freq, const float *weights, FR flags, const int *conv_info,
                                 const float *conv_sums, int T, int4 *pos, int *meta, double *norm_acc,
                                 float *convsum_out) {
    k_preprocess<P, FR><<<blocks, 256, 0, st>>>(R, uvw, freq, weights, flags, conv_info, conv_sums, p->wplanes,
                                                p->w_sq_increment, p->sampling, T, p->nx, p->ny, p->u_increment,
                                                p->v_increment, pos, meta, norm_acc, convsum_out);
}

template <int P>
static void launch_preprocess(const mtb_grid_params *p, int blocks, cudaStream_t st, int R, const float *uvw,
                              const float *freq, const float *weights, const int *flags, const int *conv_info,
                              const float *conv_sums, int T, int4 *pos, int *meta, double *norm_acc,
                              float *convsum_out) {
    const unsigned char *fb = (const unsigned char *)flags;
    if (p->flags_u8 == 2)
        launch_preprocess_fr<P>(p, blocks, st, R, uvw, freq, weights, FlagBits{fb}, conv_info, conv_sums, T, pos,
                                meta, norm_acc, convsum_out);
    else if (p->flags_u8)
        launch_preprocess_fr<P>(p, blocks, st, R, uvw, freq, weights, FlagArray<unsigned char>{fb}, conv_info,
                                conv_sums, T, pos, meta, norm_acc, convsum_out);
    else
        launch_preprocess_fr<P>(p, blocks, st, R, uvw, freq, weights, FlagArray<int>{flags}, conv_info, conv_sums, T,
                                pos, meta, norm_acc, convsum_out);
}

template <int P, bool DIRECT, typename FR>
static void launch_gather_fr(const mtb_grid_params *p, int blocks, cudaStream_t st, int R, const GridSpace &s,
                             const float2 *vis, const float *weights, FR flags, const GridPlan &plan,
                             const int *conv_info, const int *pbase, int nw, bool pairs) {
    k_gather<P, DIRECT, FR><<<blocks, 256, 0, st>>>(R, s.skeys, s.sidx, s.pos, s.meta, vis, weights, flags, s.wpos,
                                                    s.wvis, plan.bt, p->nx, conv_info, pbase, nw, p->psf,
                                                    pairs ? 1 : 0);
}

template <int P, bool DIRECT>
static void launch_gather(const mtb_grid_params *p, int blocks, cudaStream_t st, int R, const GridSpace &s,
                          const float2 *vis, const float *weights, const int *flags, const GridPlan &plan,
                          const int *conv_info, const int *pbase, int nw, bool pairs = false) {
    const unsigned char *fb = (const unsigned char *)flags;
    if (p->flags_u8 == 2)
        launch_gather_fr<P, DIRECT>(p, blocks, st, R, s, vis, weights, FlagBits{fb}, plan, conv_info, pbase, nw,
                                    pairs);
    else if (p->flags_u8)
        launch_gather_fr<P, DIRECT>(p, blocks, st, R, s, vis, weights, FlagArray<unsigned char>{fb}, plan, conv_info,
                                    pbase, nw, pairs);
    else
        launch_gather_fr<P, DIRECT>(p, blocks, st, R, s, vis, weights, FlagArray<int>{flags}, plan, conv_info, pbase,
                                    nw, pairs);
}

// Everything of one mtb_grid call before the gridder kernels: preprocessing,
// compression, binning into work items, the gathered records and
// visibilities, and (direct gridders) the padded and expanded kernel tables,
// the bucket moduli on the device and the zeroed delta grid.
template <int P>
static int prepare_grid(const mtb_grid_params *p, const GridPlan &plan, const float2 *table, size_t table_elems,
                        size_t padded, const int *conv_info, const float *conv_sums, const float *uvw,
                        const float *freq, const float2 *vis, const float *weights, const int *flags, int R,
                        bool compensated, GridSpace &s, cudaStream_t st, bool pairs) {
    const int T = oversample_T(p->sampling);
    const int sms = sm_count();
    MTB_CUDA_TRY(cudaMemsetAsync(s.norm_acc, 0, 4 * sizeof(double), st));
    MTB_CUDA_TRY(cudaMemsetAsync(s.stats, 0, 4 * sizeof(unsigned long long), st));
    MTB_CUDA_TRY(cudaMemsetAsync(s.bounds, 0, 2 * kMaxBuckets * sizeof(int), st));
    MTB_CUDA_TRY(cudaMemsetAsync(s.counters, 0, kMaxBuckets * sizeof(int), st));
    int blocks = std::min((R + 255) / 256, sms * 8);
    if (blocks < 1) blocks = 1;
    launch_preprocess<P>(p, blocks, st, R, uvw, freq, weights, flags, conv_info, conv_sums, T, s.pos, s.meta,
                         s.norm_acc, nullptr);
    MTB_LAUNCHED();
    k_compress<<<blocks, 256, 0, st>>>(R, p->nx, s.pos, s.meta, s.keys, s.iota, plan.bt, s.stats);
    MTB_LAUNCHED();
    // only the packed key's bits: 20 for a 4096² grid of 32² tiles and 32
    // buckets, three 8-bit digit passes instead of four
    const int end_bit = plan.bt.xbits + plan.bt.ybits + plan.bt.bbits;
    size_t cb = s.cub_bytes;
    MTB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(s.cub, cb, s.keys, s.skeys, s.iota, s.sidx, R, 0, end_bit, st));
    cb = s.cub_bytes;
    MTB_CUDA_TRY(cub::DeviceRunLengthEncode::Encode(s.cub, cb, s.skeys, s.ukeys, s.counts, s.num_runs, R, st));
    cb = s.cub_bytes;
    MTB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(s.cub, cb, s.counts, s.run_start, R, st));
    k_chunk_counts<<<blocks, 256, 0, st>>>(s.ukeys, s.counts, s.num_runs, R, plan.chunk, s.nchunks);
    MTB_LAUNCHED();
    cb = s.cub_bytes;
    MTB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(s.cub, cb, s.nchunks, s.item_start, R, st));
    k_make_items<<<blocks, 256, 0, st>>>(s.ukeys, s.counts, s.run_start, s.item_start, s.nchunks, s.num_runs,
                                         plan.chunk, plan.bt.xbits, plan.bt.ybits, s.items);
    MTB_LAUNCHED();
    k_bucket_bounds<<<blocks, 256, 0, st>>>(s.items, s.item_start, s.nchunks, s.num_runs, s.bounds, plan.bt.n,
                                            s.n_items);
    MTB_LAUNCHED();
    if (p->merge == 1) {
        launch_gather<P, false>(p, blocks, st, R, s, vis, weights, flags, plan, nullptr, nullptr, 0);
        MTB_LAUNCHED();
        return MTB_OK;
    }
    k_pad_bases<<<1, 1, 0, st>>>(conv_info, p->wplanes, T, s.pbase);
    MTB_LAUNCHED();
    launch_gather<P, true>(p, blocks, st, R, s, vis, weights, flags, plan, conv_info, s.pbase, p->wplanes, pairs);
    MTB_LAUNCHED();
    if (streaming(gridder_of(p))) {
        // one warp per work item; the item count is on the device: cover the
        // largest count this chunk can have and let the kernel read the rest
        const int wb = std::min((R / 8 + 7) / 8 + 1, sms * 16);
        k_mark_runs<<<wb, 256, 0, st>>>(s.items, s.n_items, s.wpos);
        MTB_LAUNCHED();
    }
    {
        // the expanded padded table the direct gridders read
        const int rows = plan.table_rows;
        const int pb = (int)std::min<size_t>(((size_t)rows + 7) / 8, (size_t)sms * 16);
        if (pairs)
            k_pad_pairs<<<pb > 0 ? pb : 1, 256, 0, st>>>(table, conv_info, s.pbase, p->wplanes, rows, s.table2);
        else
            k_pad_expand<<<pb > 0 ? pb : 1, 256, 0, st>>>(table, conv_info, s.pbase, p->wplanes, rows, s.table2);
        MTB_LAUNCHED();
        (void)table_elems;
        (void)padded;
    }
    k_set_moduli<<<1, 32, 0, st>>>(plan.bt, s.moduli);
    MTB_LAUNCHED();
    MTB_CUDA_TRY(cudaMemsetAsync(s.err, 0, sizeof(int), st));
    // compensated mode: the call's flushes go to a zeroed delta grid with
    // plain reductions (no returned values, so no stall at a flush) and one
    // pass merges it into the float pair (grid, grid_lo)
    if (compensated)
        MTB_CUDA_TRY(cudaMemsetAsync(s.delta, 0, delta_bytes(p), st));
    return MTB_OK;
}

template <int P>
static GridJobDesc job_desc(const mtb_grid_params *p, float *grid, bool compensated, const GridSpace &s) {
    GridJobDesc d;
    d.wpos = s.wpos;
    d.wvis4 = (const float4 *)s.wvis;
    d.table2 = s.table2;
    // compensated: flushes go to the call's delta grid, FP32 (vector
    // reductions, the default) or FP64 (exact_delta)
    d.grid = (compensated && !exact_of(p)) ? (float *)s.delta : grid;
    d.dgrid = (compensated && exact_of(p)) ? s.delta : nullptr;
    d.M = s.moduli;
    d.nx = p->nx;
    d.table2_elems = (int)s.table2_elems;
    d.cells = p->nx * p->ny;
    // one odd support per bucket: every record's support is its bucket's modulus
    d.uniform = p->support_bucket <= 1 ? 1 : 0;
    return d;
}

// After the gridder kernels: fold the delta grid into (grid, grid_lo) and
// add the call's normaliser sums and statistics.
template <int P>
static int finish_grid(const mtb_grid_params *p, float *grid, float *grid_lo, float *normalizer,
                       mtb_grid_stats *stats, GridSpace &s, const int *err, cudaStream_t st) {
    const int sms = sm_count();
    if (grid_lo) {
        const size_t n2 = (size_t)p->nx * p->ny * P;     // complex values
        if (exact_of(p)) {
            int mb = (int)std::min<size_t>((n2 + 255) / 256, (size_t)sms * 16);
            k_merge_delta<<<mb > 0 ? mb : 1, 256, 0, st>>>((float2 *)grid, (float2 *)grid_lo,
                                                         (const double2 *)s.delta, n2);
            MTB_LAUNCHED();
        } else {
            const size_t n4 = n2 / 2;
            int mb = (int)std::min<size_t>((n4 + 255) / 256, (size_t)sms * 16);
            k_merge_delta32<<<mb > 0 ? mb : 1, 256, 0, st>>>((float4 *)grid, (float4 *)grid_lo,
                                                           (const float4 *)s.delta, n4);
            MTB_LAUNCHED();
            if (n2 & 1) {
                k_merge_delta32_tail<<<1, 1, 0, st>>>((float2 *)grid, (float2 *)grid_lo, (const float2 *)s.delta,
                                                      n2 - 1);
                MTB_LAUNCHED();
            }
        }
    }
    k_finish<<<1, 32, 0, st>>>(P, s.norm_acc, normalizer, s.stats, stats, err);
    MTB_LAUNCHED();
    return MTB_OK;
}

template <int P>
static int run_grid(const mtb_grid_params *p, const GridPlan &plan, const float2 *table, size_t table_elems,
                    size_t padded, const int *conv_info, const float *conv_sums, const float *uvw,
                    const float *freq, const float2 *vis, const float *weights, const int *flags, int R,
                    float *grid, float *grid_lo, float *normalizer, mtb_grid_stats *stats, GridSpace &s,
                    cudaStream_t st) {
    const bool direct = p->merge != 1;
    const bool pairs = pairs_of(p);
    MTB_TRY(prepare_grid<P>(p, plan, table, table_elems, padded, conv_info, conv_sums, uvw, freq, vis, weights,
                            flags, R, direct && grid_lo != nullptr, s, st, pairs));
    if (p->gridder_start_event) MTB_CUDA_TRY(cudaEventRecord((cudaEvent_t)p->gridder_start_event, st));
    if (!direct) {
        GridArgs a;
        a.items = s.items;
        a.bounds = s.bounds;
        a.counters = s.counters;
        a.wpos = s.wpos;
        a.wvis = s.wvis;
        a.table = table;
        a.grid = grid;
        a.grid_lo = grid_lo;
        a.nx = p->nx;
        a.ny = p->ny;
        a.table_elems = (int)table_elems;
        a.cells = p->nx * p->ny;
        for (int b = 0; b < plan.bt.n; b++) {
            int M = plan.bt.M[b];
            if (M <= 0) continue;
            a.bucket = b;
            a.M = M;
            a.tile = plan.bt.tile[b];
            a.W = a.tile + M - 1;
            Launch L = launch_shape(M, P, a.tile, p->merge);
            MTB_TRY(launch_bucket<P>(a, L, st));
        }
        if (p->gridder_end_event) MTB_CUDA_TRY(cudaEventRecord((cudaEvent_t)p->gridder_end_event, st));
        k_finish<<<1, 32, 0, st>>>(P, s.norm_acc, normalizer, s.stats, stats, nullptr);
        MTB_LAUNCHED();
        return MTB_OK;
    }
    Grid2Args g2;
    g2.items = s.items;
    g2.n_items = s.n_items;
    g2.counter = s.counters;
    g2.njobs = 1;
    g2.wait_cycles = wait_cycles();
    g2.jobs[0] = job_desc<P>(p, grid, grid_lo != nullptr, s);
    const int which = gridder_of(p);
    const bool rolling = which == 5;
    if (streaming(which)) {
        G7SegSrc src;
        std::memset(&src, 0, sizeof(src));
        src.bounds[0] = s.bounds;
        src.n_items[0] = s.n_items;
        src.M[0] = s.moduli;
        k_g7_segments<<<1, kMaxBuckets, 0, st>>>(src, 1, pairs ? 1 : 0, s.segs, s.n_segs);
        MTB_LAUNCHED();
        MTB_CUDA_TRY(cudaMemsetAsync(s.counter7, 0, sizeof(int), st));
        Grid7Args g7;
        std::memset(&g7, 0, sizeof(g7));
        g7.items = s.items;
        g7.segs = s.segs;
        g7.n_segs = s.n_segs;
        g7.counter = s.counter7;
        g7.jobs[0] = g2.jobs[0];
        MTB_TRY(launch_grid7<P>(g7, pairs, st));
    } else if (which == 5) {
        MTB_TRY(launch_grid5<P>(g2, s.err, st));
    } else {
        MTB_TRY(launch_grid3<P>(g2, p->gridder_threads, st));
    }
    if (rolling && check_gridder() && !capturing(st)) {
        int e = 0;
        MTB_CUDA_TRY(cudaMemcpyAsync(&e, s.err, sizeof(int), cudaMemcpyDeviceToHost, st));
        MTB_CUDA_TRY(cudaStreamSynchronize(st));
        if (e) return MTB_ERR_KERNEL;
    }
    if (p->gridder_end_event) MTB_CUDA_TRY(cudaEventRecord((cudaEvent_t)p->gridder_end_event, st));
    return finish_grid<P>(p, grid, grid_lo, normalizer, stats, s, s.err, st);
}

// PreProcessUVW's seven outputs in the reference's layout
// (WProjPreProcessUVW.cpp:66-85): GriddingData int4 {cx, cy*nx+cx,
// -(cx%S), -(cy%S)}, conv index, ToGridIndicator (after compression),
// ToCompressIndicator, support, TakeConjugateIndicator (+1/-1).
__global__ void k_ref_outputs(int R, int nx, const int4 *__restrict__ pos, const int *__restrict__ meta,
                              int4 *__restrict__ gdata, int *__restrict__ convidx, int *__restrict__ togrid,
                              int *__restrict__ tocompress, int *__restrict__ support, float *__restrict__ imgmult) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
        int4 q = pos[r];
        int m = meta[r];
        bool g = (m & 1) != 0;
        gdata[r] = g ? make_int4(q.x, q.y * nx + q.x, -(q.x % q.w), -(q.y % q.w)) : make_int4(0, 0, 0, 0);
        convidx[r] = q.z;
        togrid[r] = (g && !(m & 4)) ? 1 : 0;
        tocompress[r] = (m & 4) ? 1 : 0;
        support[r] = q.w;
        imgmult[r] = (m & 2) ? -1.0f : 1.0f;
    }
}

}  // namespace mtb

using namespace mtb;

extern "C" int mtb_grid_workspace_size(const mtb_grid_params *p, const int *h_conv_info, int nrecords,
                                       size_t *bytes) {
    if (!bytes || !h_conv_info) return MTB_ERR_NULL;
    MTB_TRY(check_params(p));
    if (nrecords < 0) return MTB_ERR_BAD_SHAPE;
    GridPlan plan;   // refuses supports and tiles the gridders cannot take, as mtb_grid does
    MTB_TRY(make_plan(p, h_conv_info, &plan));
    int chunk = effective_chunk(p);
    Arena A;
    GridSpace s;
    carve_grid(A, nrecords, p->npol, chunk, padded_elems_of(p, h_conv_info), workspace_delta_bytes(p), &s,
               p->wplanes);
    *bytes = A.used;
    return MTB_OK;
}

extern "C" int mtb_bounds_status(int *checked, unsigned *word) {
    if (!checked || !word) return MTB_ERR_NULL;
#ifdef MTB_CHECKED
    *checked = 1;
    MTB_CUDA_TRY(cudaMemcpyFromSymbol(word, mtb::g_bounds_word, sizeof(unsigned)));
    const unsigned zero = 0;
    MTB_CUDA_TRY(cudaMemcpyToSymbol(mtb::g_bounds_word, &zero, sizeof(unsigned)));
#else
    *checked = 0;
    *word = 0;
#endif
    return MTB_OK;
}

extern "C" int mtb_grid_delta_bytes(const mtb_grid_params *p, size_t *bytes) {
    if (!bytes) return MTB_ERR_NULL;
    MTB_TRY(check_params(p));
    *bytes = delta_bytes(p);
    return MTB_OK;
}

extern "C" int mtb_grid(const mtb_grid_params *p, const void *d_table, const int *d_conv_info,
                        const int *h_conv_info, const float *d_conv_sums, const float *d_uvw,
                        const float *d_freq, const void *d_vis, const float *d_weights, const int *d_flags,
                        int nrecords, void *d_grid, void *d_grid_lo, float *d_normalizer,
                        mtb_grid_stats *d_stats, void *d_workspace, size_t workspace_bytes,
                        mtb_stream_t stream) {
    MTB_RANGE("mtb_grid");
    MTB_TRY(check_params(p));
    if (nrecords < 0) return MTB_ERR_BAD_SHAPE;
    if (!d_grid || !d_normalizer || !h_conv_info) return MTB_ERR_NULL;
    cudaStream_t st = (cudaStream_t)stream;
    GridPlan plan;
    MTB_TRY(make_plan(p, h_conv_info, &plan));
    const int P = p->npol;
    size_t gbytes = (size_t)p->nx * p->ny * P * sizeof(float2);
    if (p->initialize_output) {
        MTB_CUDA_TRY(cudaMemsetAsync(d_grid, 0, gbytes, st));
        if (d_grid_lo) MTB_CUDA_TRY(cudaMemsetAsync(d_grid_lo, 0, gbytes, st));
        MTB_CUDA_TRY(cudaMemsetAsync(d_normalizer, 0, P * sizeof(float), st));
        if (d_stats) MTB_CUDA_TRY(cudaMemsetAsync(d_stats, 0, sizeof(mtb_grid_stats), st));
    }
    if (nrecords == 0) return MTB_OK;
    if (!d_table || !d_conv_info || !d_conv_sums || !d_uvw || !d_freq || (!d_vis && !p->psf) || !d_weights ||
        !d_flags || !d_workspace)
        return MTB_ERR_NULL;
    if (d_grid_lo && p->no_grid_lo) return MTB_ERR_BAD_PARAM;   // its workspace holds no delta grid
    Arena A(d_workspace, workspace_bytes);
    GridSpace s;
    carve_grid(A, nrecords, P, plan.chunk, padded_elems_of(p, h_conv_info), workspace_delta_bytes(p), &s,
               p->wplanes);
    if (!A.ok()) return MTB_ERR_WORKSPACE;
    if (p->external_delta && delta_bytes(p)) {
        if (!p->d_delta) return MTB_ERR_NULL;
        if ((uintptr_t)p->d_delta % 256) return MTB_ERR_BAD_PARAM;
        s.delta = (double *)p->d_delta;
    }
    const float2 *tb = (const float2 *)d_table;
    const float2 *vis = (const float2 *)d_vis;
    float *g = (float *)d_grid, *lo = (float *)d_grid_lo;
    const size_t te = table_elems_of(p, h_conv_info), pe = padded_elems_of(p, h_conv_info);
    if (P == 1)
        return run_grid<1>(p, plan, tb, te, pe, d_conv_info, d_conv_sums, d_uvw, d_freq, vis, d_weights, d_flags,
                           nrecords, g, lo, d_normalizer, d_stats, s, st);
    if (P == 2)
        return run_grid<2>(p, plan, tb, te, pe, d_conv_info, d_conv_sums, d_uvw, d_freq, vis, d_weights, d_flags,
                           nrecords, g, lo, d_normalizer, d_stats, s, st);
    return run_grid<4>(p, plan, tb, te, pe, d_conv_info, d_conv_sums, d_uvw, d_freq, vis, d_weights, d_flags, nrecords,
                       g, lo, d_normalizer, d_stats, s, st);
}

// ---------------------------------------------------------- batched grid --
struct BatchQueues {
    const int4 *items[kMaxBatch];
    const int *n_items[kMaxBatch];   // null: the image has no records
};

// One queue of every image's work items, image index in item.w.
__global__ void k_concat_items(BatchQueues q, int njobs, int4 *__restrict__ out, int *__restrict__ n_total) {
    const int j = blockIdx.x;
    __shared__ int base, n;
    if (threadIdx.x == 0) {
        int b = 0;
        for (int i = 0; i < j; i++) b += q.n_items[i] ? *q.n_items[i] : 0;
        base = b;
        n = q.n_items[j] ? *q.n_items[j] : 0;
        if (j == njobs - 1) *n_total = b + n;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        int4 it = q.items[j][k];
        it.w = j;
        out[base + k] = it;
    }
}

static int check_batch(const mtb_grid_job *jobs, int njobs) {
    if (!jobs) return MTB_ERR_NULL;
    if (njobs < 1 || njobs > kMaxBatch) return MTB_ERR_BAD_SHAPE;
    for (int j = 0; j < njobs; j++) {
        MTB_TRY(check_params(&jobs[j].params));
        if (jobs[j].params.npol != jobs[0].params.npol) return MTB_ERR_BAD_SHAPE;
        if (jobs[j].params.gridder_threads != jobs[0].params.gridder_threads) return MTB_ERR_BAD_PARAM;
        if (jobs[j].params.gridder != jobs[0].params.gridder) return MTB_ERR_BAD_PARAM;
        if (jobs[j].params.external_delta) return MTB_ERR_BAD_PARAM;   // batches carve their delta grids
        if (jobs[j].nrecords < 0) return MTB_ERR_BAD_SHAPE;
        if (!jobs[j].h_conv_info) return MTB_ERR_NULL;
    }
    return MTB_OK;
}

static int batch_plans(const mtb_grid_job *jobs, int njobs, GridPlan *plans) {
    for (int j = 0; j < njobs; j++) {
        mtb_grid_params p = jobs[j].params;
        p.merge = 0;
        MTB_TRY(make_plan(&p, jobs[j].h_conv_info, &plans[j]));
    }
    return MTB_OK;
}

// every job's space, then the batch queue, its length and its counter
static void carve_batch(Arena &A, const mtb_grid_job *jobs, int njobs, const GridPlan *plans, GridSpace *spaces,
                        int4 **items, int **n_total, int **counter, G7Segment **segs) {
    size_t cap = 0;
    for (int j = 0; j < njobs; j++) {
        mtb_grid_params p = jobs[j].params;
        p.merge = 0;                      // the batch runs the direct gridders
        carve_grid(A, jobs[j].nrecords, p.npol, plans[j].chunk, padded_elems_of(&p, jobs[j].h_conv_info),
                   workspace_delta_bytes(&p), &spaces[j], p.wplanes);
        const size_t r = (size_t)(jobs[j].nrecords > 0 ? jobs[j].nrecords : 1);
        cap += r + r / (size_t)plans[j].chunk + 2;
    }
    *items = A.take<int4>(cap);
    *n_total = A.take<int>(1);
    *counter = A.take<int>(1);
    *segs = A.take<G7Segment>((size_t)njobs * kMaxBuckets + 1);
}

extern "C" int mtb_grid_batch_workspace_size(const mtb_grid_job *jobs, int njobs, size_t *bytes) {
    if (!bytes) return MTB_ERR_NULL;
    MTB_TRY(check_batch(jobs, njobs));
    GridPlan plans[kMaxBatch];
    MTB_TRY(batch_plans(jobs, njobs, plans));
    Arena A;
    GridSpace spaces[kMaxBatch];
    int4 *items;
    int *n_total, *counter;
    G7Segment *segs;
    carve_batch(A, jobs, njobs, plans, spaces, &items, &n_total, &counter, &segs);
    *bytes = A.used;
    return MTB_OK;
}

template <int P>
static int run_batch(const mtb_grid_job *jobs, int njobs, const GridPlan *plans, GridSpace *spaces, int4 *items,
                     int *n_total, int *counter, G7Segment *segs, cudaStream_t st) {
    BatchQueues q;
    Grid2Args g2;
    g2.njobs = njobs;
    g2.wait_cycles = wait_cycles();
    // tap pairs only when every image qualifies (the tables and visibility
    // layout of one launch are alike)
    bool pairs = true;
    for (int j = 0; j < njobs; j++) {
        mtb_grid_params pj = jobs[j].params;
        pj.merge = 0;
        pairs = pairs && pairs_of(&pj);
    }
    for (int j = 0; j < njobs; j++) {
        const mtb_grid_job &J = jobs[j];
        mtb_grid_params p = J.params;
        p.merge = 0;
        q.items[j] = spaces[j].items;
        q.n_items[j] = nullptr;
        g2.jobs[j] = job_desc<P>(&p, (float *)J.d_grid, J.d_grid_lo != nullptr, spaces[j]);
        if (J.nrecords == 0) continue;
        const size_t te = table_elems_of(&p, J.h_conv_info), pe = padded_elems_of(&p, J.h_conv_info);
        MTB_TRY(prepare_grid<P>(&p, plans[j], (const float2 *)J.d_table, te, pe, J.d_conv_info, J.d_conv_sums,
                                J.d_uvw, J.d_freq, (const float2 *)J.d_vis, J.d_weights, J.d_flags, J.nrecords,
                                J.d_grid_lo != nullptr, spaces[j], st, pairs));
        q.n_items[j] = spaces[j].n_items;
    }
    const mtb_grid_params &p0 = jobs[0].params;
    if (p0.gridder_start_event) MTB_CUDA_TRY(cudaEventRecord((cudaEvent_t)p0.gridder_start_event, st));
    k_concat_items<<<njobs, 256, 0, st>>>(q, njobs, items, n_total);
    MTB_LAUNCHED();
    MTB_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(int), st));
    g2.items = items;
    g2.n_items = n_total;
    g2.counter = counter;
    // the batch's gridder error flag (read by every image's k_finish)
    MTB_CUDA_TRY(cudaMemsetAsync(spaces[0].err, 0, sizeof(int), st));
    const int which = gridder_of(&p0);
    if (streaming(which)) {
        G7SegSrc src;
        std::memset(&src, 0, sizeof(src));
        for (int j = 0; j < njobs; j++) {
            src.bounds[j] = spaces[j].bounds;
            src.n_items[j] = jobs[j].nrecords > 0 ? spaces[j].n_items : nullptr;
            src.M[j] = spaces[j].moduli;
        }
        k_g7_segments<<<1, kMaxBuckets, 0, st>>>(src, njobs, pairs ? 1 : 0, segs, spaces[0].n_segs);
        MTB_LAUNCHED();
        MTB_CUDA_TRY(cudaMemsetAsync(spaces[0].counter7, 0, sizeof(int), st));
        Grid7Args g7;
        std::memset(&g7, 0, sizeof(g7));
        g7.items = items;
        g7.segs = segs;
        g7.n_segs = spaces[0].n_segs;
        g7.counter = spaces[0].counter7;
        for (int j = 0; j < njobs; j++) g7.jobs[j] = g2.jobs[j];
        MTB_TRY(launch_grid7<P>(g7, pairs, st));
    } else if (gridder_of(&p0) == 5) {
        MTB_TRY(launch_grid5<P>(g2, spaces[0].err, st));
        if (check_gridder() && !capturing(st)) {
            int e = 0;
            MTB_CUDA_TRY(cudaMemcpyAsync(&e, spaces[0].err, sizeof(int), cudaMemcpyDeviceToHost, st));
            MTB_CUDA_TRY(cudaStreamSynchronize(st));
            if (e) return MTB_ERR_KERNEL;
        }
    } else {
        MTB_TRY(launch_grid3<P>(g2, jobs[0].params.gridder_threads, st));
    }
    if (p0.gridder_end_event) MTB_CUDA_TRY(cudaEventRecord((cudaEvent_t)p0.gridder_end_event, st));
    for (int j = 0; j < njobs; j++) {
        const mtb_grid_job &J = jobs[j];
        if (J.nrecords == 0) continue;
        MTB_TRY(finish_grid<P>(&J.params, (float *)J.d_grid, (float *)J.d_grid_lo, J.d_normalizer, J.d_stats,
                               spaces[j], spaces[0].err, st));
    }
    return MTB_OK;
}

extern "C" int mtb_grid_batch(const mtb_grid_job *jobs, int njobs, void *d_workspace, size_t workspace_bytes,
                              mtb_stream_t stream) {
    MTB_RANGE("mtb_grid_batch");
    MTB_TRY(check_batch(jobs, njobs));
    cudaStream_t st = (cudaStream_t)stream;
    for (int j = 0; j < njobs; j++) {
        const mtb_grid_job &J = jobs[j];
        if (!J.d_grid || !J.d_normalizer) return MTB_ERR_NULL;
        if (J.nrecords > 0 && (!J.d_table || !J.d_conv_info || !J.d_conv_sums || !J.d_uvw || !J.d_freq ||
                               (!J.d_vis && !J.params.psf) || !J.d_weights || !J.d_flags))
            return MTB_ERR_NULL;
        if (J.d_grid_lo && J.params.no_grid_lo) return MTB_ERR_BAD_PARAM;
    }
    if (!d_workspace) return MTB_ERR_NULL;
    GridPlan plans[kMaxBatch];
    MTB_TRY(batch_plans(jobs, njobs, plans));
    Arena A(d_workspace, workspace_bytes);
    GridSpace spaces[kMaxBatch];
    int4 *items;
    int *n_total, *counter;
    G7Segment *segs;
    carve_batch(A, jobs, njobs, plans, spaces, &items, &n_total, &counter, &segs);
    if (!A.ok()) return MTB_ERR_WORKSPACE;
    for (int j = 0; j < njobs; j++) {
        const mtb_grid_job &J = jobs[j];
        const mtb_grid_params &p = J.params;
        if (!p.initialize_output) continue;
        const size_t gbytes = (size_t)p.nx * p.ny * p.npol * sizeof(float2);
        MTB_CUDA_TRY(cudaMemsetAsync(J.d_grid, 0, gbytes, st));
        if (J.d_grid_lo) MTB_CUDA_TRY(cudaMemsetAsync(J.d_grid_lo, 0, gbytes, st));
        MTB_CUDA_TRY(cudaMemsetAsync(J.d_normalizer, 0, p.npol * sizeof(float), st));
        if (J.d_stats) MTB_CUDA_TRY(cudaMemsetAsync(J.d_stats, 0, sizeof(mtb_grid_stats), st));
    }
    const int P = jobs[0].params.npol;
    if (P == 1) return run_batch<1>(jobs, njobs, plans, spaces, items, n_total, counter, segs, st);
    if (P == 2) return run_batch<2>(jobs, njobs, plans, spaces, items, n_total, counter, segs, st);
    return run_batch<4>(jobs, njobs, plans, spaces, items, n_total, counter, segs, st);
}

extern "C" int mtb_preprocess_uvw(const mtb_grid_params *p, const int *d_conv_info, const int *h_conv_info,
                                  const float *d_conv_sums, const float *d_uvw, const float *d_freq,
                                  const float *d_weights, const int *d_flags, int nrecords, int *d_gridding_data,
                                  int *d_conv_index, int *d_to_grid, int *d_to_compress, int *d_support,
                                  float *d_take_conjugate, float *d_conv_sum, void *d_workspace,
                                  size_t workspace_bytes, mtb_stream_t stream) {
    MTB_RANGE("mtb_preprocess_uvw");
    MTB_TRY(check_params(p));
    if (nrecords < 0) return MTB_ERR_BAD_SHAPE;
    if (nrecords == 0) return MTB_OK;
    if (!d_conv_info || !h_conv_info || !d_conv_sums || !d_uvw || !d_freq || !d_weights || !d_flags ||
        !d_gridding_data || !d_conv_index || !d_to_grid || !d_to_compress || !d_support || !d_take_conjugate ||
        !d_conv_sum || !d_workspace)
        return MTB_ERR_NULL;
    GridPlan plan;
    MTB_TRY(make_plan(p, h_conv_info, &plan));
    cudaStream_t st = (cudaStream_t)stream;
    Arena A(d_workspace, workspace_bytes);
    GridSpace s;
    carve_grid(A, nrecords, p->npol, plan.chunk, 0, 0, &s);
    if (!A.ok()) return MTB_ERR_WORKSPACE;
    const int R = nrecords, T = oversample_T(p->sampling);
    int blocks = std::min((R + 255) / 256, sm_count() * 8);
    MTB_CUDA_TRY(cudaMemsetAsync(s.norm_acc, 0, 4 * sizeof(double), st));
    MTB_CUDA_TRY(cudaMemsetAsync(s.stats, 0, 4 * sizeof(unsigned long long), st));
#define MTB_PRE(PP)                                                                                           \
    launch_preprocess<PP>(p, blocks, st, R, d_uvw, d_freq, d_weights, d_flags, d_conv_info, d_conv_sums, T,     \
                          s.pos, s.meta, s.norm_acc, d_conv_sum)
    if (p->npol == 1) MTB_PRE(1);
    else if (p->npol == 2) MTB_PRE(2);
    else MTB_PRE(4);
#undef MTB_PRE
    MTB_LAUNCHED();
    k_compress<<<blocks, 256, 0, st>>>(R, p->nx, s.pos, s.meta, s.keys, s.iota, plan.bt, s.stats);
    MTB_LAUNCHED();
    k_ref_outputs<<<blocks, 256, 0, st>>>(R, p->nx, s.pos, s.meta, (int4 *)d_gridding_data, d_conv_index,
                                          d_to_grid, d_to_compress, d_support, d_take_conjugate);
    MTB_LAUNCHED();
    return MTB_OK;
}

// ------------------------------------------------------ fixed-scratch path --
// Some callers cannot allocate device memory: code running where cudaMalloc
// is off limits (inside an allocator or memory-pool callback, a process whose
// device memory is pre-partitioned by a host framework, or a plugin that may
// only touch buffers its host hands it).  For them mtb_preprocess_uvw_noalloc
// runs the PreProcessUVW operator with its scratch in the fixed array below
// instead of a caller workspace.  The array is part of this library's device
// image, so every GPU that loads the library holds it until the process exits.
namespace mtb {
static const int kNoAllocMaxRecords = 1 << 20;
static const size_t kNoAllocPos = 0;
static const size_t kNoAllocMeta = kNoAllocPos + sizeof(int4) * (size_t)kNoAllocMaxRecords;
static const size_t kNoAllocKeys = kNoAllocMeta + sizeof(int) * (size_t)kNoAllocMaxRecords;
static const size_t kNoAllocIota = kNoAllocKeys + sizeof(unsigned) * (size_t)kNoAllocMaxRecords;
static const size_t kNoAllocNorm = kNoAllocIota + sizeof(int) * (size_t)kNoAllocMaxRecords;
static const size_t kNoAllocStats = kNoAllocNorm + sizeof(double) * 4;
static const size_t kNoAllocBytes = kNoAllocStats + sizeof(unsigned long long) * 4;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch on the current device, looked up once
// per device (host code must not use the symbol itself as an address).
static int noalloc_scratch(unsigned char **out) {
    static std::mutex mu;
    static unsigned char *addr[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MTB_ERR_CUDA;
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev]) {
        void *ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return MTB_ERR_CUDA;
        addr[dev] = (unsigned char *)ptr;
    }
    *out = addr[dev];
    return MTB_OK;
}
}  // namespace mtb

extern "C" int mtb_preprocess_uvw_noalloc_capacity(void) { return mtb::kNoAllocMaxRecords; }

extern "C" int mtb_preprocess_uvw_noalloc(const mtb_grid_params *p, const int *d_conv_info, const int *h_conv_info,
                                          const float *d_conv_sums, const float *d_uvw, const float *d_freq,
                                          const float *d_weights, const int *d_flags, int nrecords,
                                          int *d_gridding_data, int *d_conv_index, int *d_to_grid,
                                          int *d_to_compress, int *d_support, float *d_take_conjugate,
                                          float *d_conv_sum, mtb_stream_t stream) {
    MTB_RANGE("mtb_preprocess_uvw_noalloc");
    MTB_TRY(check_params(p));
    if (nrecords < 0) return MTB_ERR_BAD_SHAPE;
    if (nrecords > kNoAllocMaxRecords) return MTB_ERR_TOO_LARGE;
    if (nrecords == 0) return MTB_OK;
    if (!d_conv_info || !h_conv_info || !d_conv_sums || !d_uvw || !d_freq || !d_weights || !d_flags ||
        !d_gridding_data || !d_conv_index || !d_to_grid || !d_to_compress || !d_support || !d_take_conjugate ||
        !d_conv_sum)
        return MTB_ERR_NULL;
    GridPlan plan;
    MTB_TRY(make_plan(p, h_conv_info, &plan));
    unsigned char *base = nullptr;
    MTB_TRY(noalloc_scratch(&base));
    int4 *pos = (int4 *)(base + kNoAllocPos);
    int *meta = (int *)(base + kNoAllocMeta);
    unsigned *keys = (unsigned *)(base + kNoAllocKeys);
    int *iota = (int *)(base + kNoAllocIota);
    double *norm_acc = (double *)(base + kNoAllocNorm);
    unsigned long long *stats = (unsigned long long *)(base + kNoAllocStats);
    cudaStream_t st = (cudaStream_t)stream;
    const int R = nrecords, T = oversample_T(p->sampling);
    int blocks = std::min((R + 255) / 256, sm_count() * 8);
    // the accumulators keep the previous call's values: clear them
    MTB_CUDA_TRY(cudaMemsetAsync(norm_acc, 0, 4 * sizeof(double), st));
    MTB_CUDA_TRY(cudaMemsetAsync(stats, 0, 4 * sizeof(unsigned long long), st));
#define MTB_PRE(PP)                                                                                           \
    launch_preprocess<PP>(p, blocks, st, R, d_uvw, d_freq, d_weights, d_flags, d_conv_info, d_conv_sums, T,     \
                          pos, meta, norm_acc, d_conv_sum)
    if (p->npol == 1) MTB_PRE(1);
    else if (p->npol == 2) MTB_PRE(2);
    else MTB_PRE(4);
#undef MTB_PRE
    MTB_LAUNCHED();
    k_compress<<<blocks, 256, 0, st>>>(R, p->nx, pos, meta, keys, iota, plan.bt, stats);
    MTB_LAUNCHED();
    k_ref_outputs<<<blocks, 256, 0, st>>>(R, p->nx, pos, meta, (int4 *)d_gridding_data, d_conv_index, d_to_grid,
                                          d_to_compress, d_support, d_take_conjugate);
    MTB_LAUNCHED();
    return MTB_OK;
}
