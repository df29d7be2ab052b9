/*
 * mtb.h -- C ABI of the B200-native W-projection imaging path.
 *
 * Drop-in boundary for mt-imager's W-projection hot path.  mt-imager wires its
 * imaging dataflow out of GAFW operators (code/gafw/Implimentation/
 * GPUImplimentation/GPUArrayOperator.h:27-43): each operator validates its
 * inputs (validate(ValidationData&)) and enqueues work on the engine's stream
 * (submitToGPU(GPUSubmissionData&), GPUSubmissionData.h:27-47) with buffers the
 * engine owns.  The entry points below cover the three modules built out of
 * those operators, with the same ownership rules: the caller owns and
 * allocates every input, output and workspace buffer (device pointers), the
 * library only enqueues work on the caller's stream, and every call returns a
 * status code instead of throwing (0 = MTB_OK).
 *
 *   mtb_wkernel_*   WProjectionConvFunction::calculate
 *                   (code/mt-imager/lib/components/ConvolutionFunctionsGenerator/
 *                    WProjectionConvFunction.cpp:186-291) and its operators
 *                   casagridsf, WProjPreFFTConvFunc, multiFFT2D,
 *                   ZeroToCentre2DShift, SingleMultiply, ConvFunctionSupportFind,
 *                   ConvFunctionReOrganize, ArraysToVector, SumConvolutionFunctions.
 *   mtb_grid        one WImager chunk (code/mt-imager/lib/components/WImager.cpp:167-234):
 *                   PreProcessUVW, Sum / GriddedPointsCalculator statistics,
 *                   NormalizerCalculate, AccumulatedSum, CreateIndexAndReorder,
 *                   ValueChangeDetect, CreateBlockDataIndex, NotSameSupportManipulate,
 *                   CreateCompressionPlan, CompressVisibilities, ConvolutionGridder.
 *   mtb_finalize    ImageFinalizer (code/mt-imager/lib/components/ImageFinalizer.cpp:31-44):
 *                   PreIFFTUVCorrection, IFFT2D, ZeroToCentre2DShift, StokesConverter,
 *                   casagridsf (lmPlanePostCorrection), SincCorrector.
 *
 * Array layouts are mt-imager's (dimensions slowest first, ArrayDimensions.h:62-83):
 *   uvw        float   [3][R]        u, v, w rows in metres
 *   freq       float   [R]           nu / c per record
 *   vis        float2  [R][P]        pol-interleaved complex (XX, XY, YX, YY)
 *   weights    float   [R][P]
 *   flags      int     [R][P]        0 = keep, any other value = flagged (the reference
 *                                    weights by 1 - flag, the same for 0 / 1)
 *   table      float2  [sum_k T^2 S_k^2]  per plane [oy][ox][sy][sx], T = s (s odd) or s+1
 *   conv_info  int     [wplanes][2]  {support, first element of the plane in table}
 *   conv_sums  float   [wplanes][T*T]
 *   grid       float2  [ny][nx][P]   (v rows, u columns, pol fastest), accumulated
 *   normalizer float   [P]           accumulated
 *   image      float   [P][ny][nx]   Stokes planes, row 0 = top of the FITS image
 */
#ifndef MTB_H
#define MTB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* cudaStream_t without pulling in the CUDA headers */
typedef struct CUstream_st *mtb_stream_t;

/* Status codes; mirror the exception classes the reference throws
 * (ValidationException, CudaException, FFTException, ImagerException:
 * code/gafw/Implimentation/GPUImplimentation/GPUafw.h:28-33). */
enum {
    MTB_OK = 0,
    MTB_ERR_BAD_PARAM = 1,     /* ValidationException: a parameter is out of range   */
    MTB_ERR_BAD_SHAPE = 2,     /* ValidationException: sizes / pol count unsupported */
    MTB_ERR_WORKSPACE = 3,     /* workspace smaller than the query said              */
    MTB_ERR_CAPACITY = 4,      /* output buffer smaller than needed                  */
    MTB_ERR_CUDA = 5,          /* CudaException                                      */
    MTB_ERR_CUFFT = 6,         /* FFTException                                       */
    MTB_ERR_KERNEL = 7,        /* ImagerException: w=0 origin not real / no support  */
    MTB_ERR_NULL = 8,          /* a required pointer is NULL                         */
    MTB_ERR_TOO_LARGE = 9,     /* request exceeds a fixed-size entry point's capacity */
    MTB_ERR_CANCELLED = 10     /* an engine request cancelled before it completed    */
};

/* ------------------------------------------------------------ w-kernels -- */
typedef struct mtb_wkernel_params {
    int nx, ny;              /* image.nx, image.ny (pixels)                            */
    double l_increment;      /* image.lintervalsize in radians                         */
    double m_increment;      /* image.mintervalsize in radians                         */
    int wplanes;             /* wproj.wplanes                                          */
    int sampling;            /* wproj.convFunction.sampling                            */
    int trial_support;       /* 0: min(nx,ny)/sampling forced odd
                                (WProjectionConvFunction.cpp:194-198)                  */
    int max_support;         /* 0: trial_support-2 (WProjectionConvFunction.cpp:248)    */
    double w_max;            /* 0: 0.25/l_increment (WProjectionConvFunction.cpp:105)  */
} mtb_wkernel_params;

typedef struct mtb_wkernel_info {
    int trial_support;       /* odd S_t                                                */
    int planesize;           /* S_t * sampling                                         */
    int support_cap;         /* largest support a plane may get                        */
    int T;                   /* oversampling offsets per axis (s or s+1)               */
    double w_max;
    double w_sq_increment;   /* w_k = k^2 * w_sq_increment (WProjectionConvFunction.cpp:112,238) */
    double total_l, total_m; /* field size in radians (ConfigurationManager.cpp:190)   */
    double u_increment, v_increment; /* 1/(dl*nx), 1/(dm*ny) (ConfigurationManager.cpp:177-178) */
    size_t table_capacity;   /* float2 elements that always suffice for the table      */
    size_t workspace_bytes;  /* workspace mtb_wkernel_build needs                      */
} mtb_wkernel_info;

/* Derived scalars and buffer sizes; launches nothing and enqueues no stream
 * work, but needs the current device: the workspace size includes the work
 * area of the batched cuFFT plan, which is created here (and cached for
 * mtb_wkernel_build).  Without a device it returns MTB_ERR_CUDA.  Replaces the
 * parameter logic of WProjectionConvFunction's constructor
 * (WProjectionConvFunction.cpp:90-160). */
int mtb_wkernel_query(const mtb_wkernel_params *p, mtb_wkernel_info *info);

/* Builds every w-plane kernel in one pass (all planes batched through cuFFT Z2Z,
 * FP64 w-phase) into the reference's AmalgamatedConvFunction / convInfo /
 * ConvSums outputs.  Replaces WProjectionConvFunction::calculate
 * (WProjectionConvFunction.cpp:186-291).  Synchronises `stream` once, to bring
 * the per-plane supports to the host (the reference does so once per plane,
 * WPlaneConvFunctionCalculator.cpp:117-126).
 *   d_table       out float2 [table_capacity]
 *   d_conv_info   out int [wplanes][2] (device; may be NULL)
 *   h_conv_info   out int [wplanes][2] (host; required)
 *   d_conv_sums   out float [wplanes][T*T]
 *   table_elems   out: float2 elements written */
int mtb_wkernel_build(const mtb_wkernel_params *p, void *d_workspace, size_t workspace_bytes,
                      void *d_table, size_t table_capacity, int *d_conv_info, int *h_conv_info,
                      float *d_conv_sums, size_t *table_elems, mtb_stream_t stream);

/* The taper-only gridding kernel of mode=normal (OnlyTaperConvFunction.cpp:29-99):
 * the uv-plane prolate-spheroidal function of CasaGridSF.cu:107-149, per axis
 * (1 - nu^2) grdsf(nu) with nu = d / (3 sampling), evaluated in FP64, in the
 * table / convInfo / ConvSums format of mtb_wkernel_build with one plane
 * (grid with wplanes = 1 and w_sq_increment = 1).  Synchronises `stream`.
 *   d_table  out float2 [T*T*support*support]  (table_capacity at least that) */
int mtb_taper_kernel_build(int support, int sampling, void *d_table, size_t table_capacity, int *d_conv_info,
                           int *h_conv_info, float *d_conv_sums, size_t *table_elems, mtb_stream_t stream);

/* ------------------------------------------------------------- gridding -- */
typedef struct mtb_grid_params {
    int nx, ny;              /* uvImage.columns, uvImage.rows                          */
    int npol;                /* 1, 2 or 4                                              */
    int sampling;            /* ConvolutionFunction.sampling                           */
    int wplanes;
    double u_increment;      /* uvImage.u_increment                                    */
    double v_increment;      /* uvImage.v_increment                                    */
    double w_sq_increment;   /* ConvolutionFunction.wsquareincrement                   */
    int initialize_output;   /* zero grid, grid_lo and normalizer first (ConvolutionGridder.cu:496-502) */
    int tile;                /* 0: default; grid tile edge owned by one thread block   */
    int support_bucket;      /* 0: default; supports are grouped in buckets this wide  */
    int max_chunk;           /* 0: default; most records one block grids in one pass   */
    int merge;               /* 0: default; 1: cell flushes go to a shared-memory tile
                                window merged once per work item; 2: cell flushes merge
                                straight into the grid                                 */
    void *gridder_start_event; /* cudaEvent_t or NULL: recorded before the gridder kernels */
    void *gridder_end_event;   /* cudaEvent_t or NULL: recorded after them (the span of the
                                  ConvolutionGridder operator, like GPUSubmissionData's
                                  startEvent/endEvent, GPUSubmissionData.h:27-47)          */
    int bulk_min_support;      /* reserved, must be 0 (an earlier bulk-copy gridder, removed:
                                  it measured slower than the default)                     */
    int psf;                   /* 1: grid every visibility as 1 + 0i (the PSF; mt-imager's
                                  psf=true, VisibilityForPSFStorageManager.cpp:65-77);
                                  d_vis may then be NULL                                   */
    int exact_delta;           /* compensated mode (d_grid_lo set): 0 (default) the call's
                                  flushes accumulate in an FP32 delta grid merged into
                                  (grid, grid_lo) with TwoSum; 1 they accumulate in FP64
                                  (order-independent, about half the grid error, slower).
                                  Work items shorter than 128 records (max_chunk) always
                                  use the FP64 delta: their extra flushes would take the
                                  FP32 delta's rounding past the 1e-5 image bound           */
    int gridder_threads;       /* 0: 256; threads of a gridder block, which grids one work
                                  item at a time (256 or 512)                              */
    int gridder;               /* 0: default (8, or 3 with gridder_threads 512);
                                  3: k_grid3 (block-wide staging of each work item);
                                  5: k_grid5 (two item buffers refilled by one warp, no
                                  block barriers; items of at most 256 records);
                                  7: k_grid7 (every warp streams its own jobs -- one work
                                  item against 128 slots of its support box -- with no
                                  block barriers; items of at most 512 records);
                                  8: k_grid7 with tap pairs (a lane's slots are two pairs
                                  of neighbouring columns, each pair's taps fetched by one
                                  16-byte copy from a pair table; needs one support per
                                  bucket, else 7 runs).  A gridder that could not complete
                                  sets the normaliser to NaN                               */
    int flags_u8;              /* 0: d_flags is int32 [R][P] (the reference's layout); 1: it
                                  is one byte per flag, uint8 [R][P] (0 = keep, non-zero = flagged;
                                  a quarter of the bytes to move); 2: one bit per flag, flag
                                  i = r*P + p in bit i % 8 of byte i / 8 (ceil(R*P/8) bytes, 1 =
                                  flagged; a thirty-second of the bytes); 1 and 2 passed cast
                                  to int *; other values are refused                       */
    int no_grid_lo;            /* 0: the workspace holds the per-call delta grid compensated
                                  calls (d_grid_lo set) accumulate in: 8 bytes per cell and
                                  polarisation (FP32), 16 with exact_delta or with work
                                  items shorter than 128 records (max_chunk), which use the
                                  FP64 delta; 1: the calls pass d_grid_lo = NULL, the
                                  workspace holds no delta grid and mtb_grid refuses a
                                  d_grid_lo.  merge = 1 never needs one                   */
    int external_delta;        /* 1: the per-call delta grid is the caller's d_delta (of
                                  mtb_grid_delta_bytes bytes) and the workspace holds none:
                                  an engine that caps scratch buffers (GAFW's int buffer
                                  size) keeps it as a reusable array of its own           */
    void *d_delta;             /* with external_delta: the delta grid (device, 256-byte
                                  aligned); contents need not be kept between calls       */
} mtb_grid_params;

/* Bytes of the per-call delta grid a compensated call uses (0 when it needs
 * none: no_grid_lo or merge = 1); what d_delta must hold with external_delta. */
int mtb_grid_delta_bytes(const mtb_grid_params *p, size_t *bytes);

/* Status word of the bounds-checked build (libmtb_checked.so, built with
 * -DMTB_CHECKED by `build.py --checked`).  In that build the gridders check
 * every kernel-table tap they read and every grid cell they add to before the
 * access; an index out of range is skipped and the first one is recorded in a
 * device word instead of faulting.  *checked = 1 in that build, 0 otherwise
 * (and *word = 0).  *word: 0 = no index out of range since the last call;
 * 1 streaming gridder tap, 2 staged gridder tap, 3 direct-gridder flush,
 * 4 tile-window tap, 5 tile-window flush.  Reads and clears the word; call it
 * after synchronising the streams that ran the work (a copy from a device
 * symbol, ordered with the legacy default stream). */
int mtb_bounds_status(int *checked, unsigned *word);

typedef struct mtb_grid_stats {
    unsigned long long gridded_records;     /* Statistic:TotalGriddedRecords    (WImager.cpp:173) */
    unsigned long long compressed_records;  /* Statistic:TotalCompressedRecords (WImager.cpp:174) */
    unsigned long long gridded_points;      /* Statistic:TotalGriddedPoints     (WImager.cpp:175) */
    unsigned long long compressed_points;   /* Statistic:TotalCompressedPoints  (WImager.cpp:176) */
} mtb_grid_stats;

/* Workspace for one mtb_grid call over `nrecords` records with the kernel
 * table described by h_conv_info (host int [wplanes][2]). */
int mtb_grid_workspace_size(const mtb_grid_params *p, const int *h_conv_info, int nrecords, size_t *bytes);

/* Grids one chunk of records into the accumulating grid: one WImager::calculate
 * (WImager.cpp:271-290).  FP64 coordinates and oversampling offsets; records
 * binned by (support bucket, uv tile); FP32 sums in registers, each flushed
 * when its grid cell changes (merge = 0, the default), or into a shared-memory
 * tile window merged once per work item (merge = 1).  With d_grid_lo non-NULL
 * the call's flushes go to a delta grid that one pass merges into
 * d_grid + d_grid_lo with a TwoSum, carrying the running sum to about twice
 * FP32 precision (pass the same d_grid_lo to mtb_finalize).  d_stats (device
 * memory, may be NULL) accumulates the four record statistics.
 *   h_conv_info   host int [wplanes][2] as returned by mtb_wkernel_build */
int mtb_grid(const mtb_grid_params *p, const void *d_table, const int *d_conv_info,
             const int *h_conv_info, const float *d_conv_sums,
             const float *d_uvw, const float *d_freq, const void *d_vis, const float *d_weights,
             const int *d_flags, int nrecords,
             void *d_grid, void *d_grid_lo, float *d_normalizer, mtb_grid_stats *d_stats,
             void *d_workspace, size_t workspace_bytes, mtb_stream_t stream);

/* One image of a batched gridding launch. */
typedef struct mtb_grid_job {
    mtb_grid_params params;      /* per image; npol must be the same for every job of a batch;
                                    merge is ignored (the batch runs the
                                    per-thread direct gridder)                               */
    const void *d_table;         /* the image's kernel table, as for mtb_grid               */
    const int *d_conv_info;
    const int *h_conv_info;
    const float *d_conv_sums;
    const float *d_uvw, *d_freq; /* the image's chunk of records, as for mtb_grid           */
    const void *d_vis;
    const float *d_weights;
    const int *d_flags;
    int nrecords;
    void *d_grid;                /* accumulated outputs, as for mtb_grid                    */
    void *d_grid_lo;
    float *d_normalizer;
    mtb_grid_stats *d_stats;
} mtb_grid_job;

/* Workspace for mtb_grid_batch over these jobs. */
int mtb_grid_batch_workspace_size(const mtb_grid_job *jobs, int njobs, size_t *bytes);

/* ---------------------------------------------------------- ingest (host) */
/* Record order of mt-imager's visibility ingest (code/mt-imager/lib/
 * components/VisibilityManager/SortIndex.cpp:46-87): rows whose antenna1
 * equals antenna2 (autocorrelations) are dropped, the rest are grouped by
 * baseline number nA*nA - antenna1*nA - antenna2 - 1 ascending, and rows of
 * one baseline keep their original order -- consecutive records of a
 * baseline are what make the gridder's register accumulation and duplicate
 * compression effective.  Host memory, no GPU.
 *   index    out int [nrows] (the first *nsorted entries are written)
 *   nsorted  out rows kept
 * Antenna ids outside [0, nantennas) are refused with MTB_ERR_BAD_PARAM. */
int mtb_sort_index(const int *antenna1, const int *antenna2, int nrows, int nantennas, int *index, int *nsorted);

/* Applies a record order to one host column (SortedStorage.h:205-246):
 * out[k] = the row_bytes bytes at in + index[k]*in_stride + offset, for
 * k < n, split over host threads (threads 0: the hardware's, at most 16).
 * With in_stride/offset it also picks one channel out of a [row][chan][pol]
 * column or one coordinate out of a [row][3] uvw column. */
int mtb_gather_rows(const void *in, size_t in_stride, size_t offset, size_t row_bytes, const int *index, int n,
                    void *out, int threads);

/* ------------------------------------------------ LSRK frequencies (device) */
/* Observer and epoch of the TOPO -> LSRK conversion. */
typedef struct mtb_lsrk_params {
    double site_itrf[3];     /* observatory position, ITRF metres (what MeasTable::Observatory gives) */
    double ra, dec;          /* phase centre, J2000, radians                                        */
    double tt_minus_time;    /* TT minus the time scale of time_s, seconds: 69.184 for UTC since
                                2017-01-01, 32.184 for TAI                                          */
    double ut1_minus_time;   /* UT1 minus the time scale of time_s, seconds (DUT1 for UTC, < 0.9 s) */
} mtb_lsrk_params;

/* Workspace bytes of mtb_lsrk_freq_over_c for nrows rows. */
int mtb_lsrk_workspace_size(int nrows, size_t *bytes);

/* Channel frequencies converted from TOPO to LSRK per record, as nu/c in
 * float32: the per-record frequency column PreProcessUVW takes.  Replaces
 * FrequencyConverter (code/mt-imager/lib/components/VisibilityManager/
 * FrequencyConverter.cpp:112-140), which evaluates casacore's
 * MFrequency::Convert(TOPO -> LSRK) once per distinct consecutive record time
 * and stores (float)(nu_LSRK / c).  casacore's measures are not used: the
 * observer's velocity with respect to the kinematic LSR (Earth rotation,
 * Earth's barycentric motion from published mean elements, 20 km/s solar
 * motion towards 18h +30 deg B1900) is computed in FP64 on the device, once
 * per record whose time differs from the previous record's.
 *   time_s   device double [nrows]: MJD seconds (the MeasurementSet TIME
 *            column), in the row order the time-sharing is detected in
 *   chan_hz  device double [nchan]: TOPO channel frequencies, Hz
 *   index    device int [n] or NULL: out[.][k] is for row index[k] (the
 *            baseline-major record order of mtb_sort_index); NULL: n == nrows
 *            and row k; an index outside [0, nrows) writes NaN
 *   out      device float [nchan][n]: nu_LSRK / c, m^-1
 * Enqueued on `stream`; the workspace (mtb_lsrk_workspace_size) is in use
 * until the stream reaches the end of the call. */
int mtb_lsrk_freq_over_c(const mtb_lsrk_params *params, const double *time_s, int nrows, const double *chan_hz,
                         int nchan, const int *index, int n, float *out, void *workspace, size_t workspace_bytes,
                         mtb_stream_t stream);

/* Gridder knobs the autotuner chooses among (fields of mtb_grid_params). */
typedef struct mtb_grid_tuning {
    int tile;             /* bin tile edge                                            */
    int support_bucket;   /* odd supports per bin bucket                              */
    int max_chunk;        /* records per work item                                    */
    int gridder_threads;  /* threads per gridder block (one work item at a time)      */
    int gridder;          /* 3: block-staged items, 5: rolling items, 7: streaming
                             warps (mtb_grid_params)                                   */
    float ms;             /* measured time of one mtb_grid_batch call with these knobs */
} mtb_grid_tuning;

/* Autotuner.  No counterpart in the reference, whose gridder launch shapes are
 * fixed.  Grids the jobs (as mtb_grid_batch) once with every candidate of
 * tile {16, 32, 64} x support_bucket {1, 2} x nine gridder shapes (gridder 3
 * with max_chunk {256, 512} x gridder_threads {256, 512}, gridder 5 with
 * 256-record items, gridders 7 and 8 with max_chunk {256, 512}; 256 threads
 * unless stated), times each call with CUDA events on
 * `stream` (after one untimed call), and writes the fastest to *best and to
 * every job's params.  Every job must start a fresh image (initialize_output
 * = 1): the grids, normalisers and statistics hold the result of a call with
 * the chosen knobs when it returns.  Synchronises `stream` after every call.
 * `candidates` (may be NULL) receives all mtb_grid_autotune_candidate_count()
 * timings (54).  Workspace: mtb_grid_autotune_workspace_size. */
int mtb_grid_autotune_candidate_count(void);
int mtb_grid_autotune_workspace_size(const mtb_grid_job *jobs, int njobs, size_t *bytes);
int mtb_grid_autotune(mtb_grid_job *jobs, int njobs, void *d_workspace, size_t workspace_bytes,
                      mtb_stream_t stream, mtb_grid_tuning *best, mtb_grid_tuning *candidates);

/* Grids one chunk of records into each of up to 64 images -- channels of a cube
 * or unrelated images of any geometry -- with ONE persistent gridder launch fed
 * by a work queue over (image, support bucket, tile) bins.  Every image is
 * preprocessed and binned as by mtb_grid, its work items are concatenated into
 * one queue, and the gridder takes each item's image from it.  The result for
 * every image equals mtb_grid's to the rounding of the FP32 reductions (bit
 * for bit with exact_delta).  All work is enqueued on `stream`; the call can
 * be captured into a CUDA graph. */
int mtb_grid_batch(const mtb_grid_job *jobs, int njobs, void *d_workspace, size_t workspace_bytes,
                   mtb_stream_t stream);

/* The PreProcessUVW operator alone, with its seven outputs in the reference's
 * layout (code/mt-imager/lib/operators/WProjPreProcessUVW.cpp:66-85,
 * WProjPreProcessUVW.cu:112-324), FP64 coordinates.  Workspace: as for
 * mtb_grid with the same record count.
 *   d_gridding_data   int [R][4] {cx, cy*nx+cx, -(cx%S), -(cy%S)}
 *   d_conv_index      int [R]    first table element of the record's sub-kernel
 *   d_to_grid         int [R]    1 = grid (after duplicate compression)
 *   d_to_compress     int [R]    1 = merged into the previous record
 *   d_support         int [R]
 *   d_take_conjugate  float [R]  -1 when w < 0 (u, v negated, imaginary part negated)
 *   d_conv_sum        float [P][R] ConvSums * weight * (1 - flag), flag taken as 0 / 1 */
int mtb_preprocess_uvw(const mtb_grid_params *p, const int *d_conv_info, const int *h_conv_info,
                       const float *d_conv_sums, const float *d_uvw, const float *d_freq,
                       const float *d_weights, const int *d_flags, int nrecords, int *d_gridding_data,
                       int *d_conv_index, int *d_to_grid, int *d_to_compress, int *d_support,
                       float *d_take_conjugate, float *d_conv_sum, void *d_workspace,
                       size_t workspace_bytes, mtb_stream_t stream);

/* mtb_preprocess_uvw for callers that cannot allocate device memory.  No
 * counterpart in the reference.  Some hosts may not call cudaMalloc at all:
 * code running inside an allocator or memory-pool callback, a process whose
 * device memory is partitioned up front by its framework, a plugin that may
 * only use the buffers its host hands it.  This entry point takes no
 * workspace: its scratch lives in a fixed array inside the library's device
 * image (about 28 MB, held by every GPU that loads the library until the
 * process exits), and it calls no allocating routine.  Inputs and outputs are
 * those of mtb_preprocess_uvw and still belong to the caller.
 *   - nrecords above mtb_preprocess_uvw_noalloc_capacity() (1,048,576) is
 *     refused with MTB_ERR_TOO_LARGE; split larger chunks.
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress); make that first call before any stream capture.
 *   - Every call shares the one array, so calls whose work overlaps on the
 *     GPU (different streams or host threads on one device) race and must be
 *     serialised by the caller. */
int mtb_preprocess_uvw_noalloc(const mtb_grid_params *p, const int *d_conv_info, const int *h_conv_info,
                               const float *d_conv_sums, const float *d_uvw, const float *d_freq,
                               const float *d_weights, const int *d_flags, int nrecords, int *d_gridding_data,
                               int *d_conv_index, int *d_to_grid, int *d_to_compress, int *d_support,
                               float *d_take_conjugate, float *d_conv_sum, mtb_stream_t stream);
/* Largest nrecords mtb_preprocess_uvw_noalloc accepts. */
int mtb_preprocess_uvw_noalloc_capacity(void);

/* ------------------------------------------------------------- finalize -- */
enum { MTB_POL_LINEAR = 0, MTB_POL_CIRCULAR = 1 };  /* PolarizationType (mtimager.h:30-37) */

typedef struct mtb_finalize_params {
    int nx, ny, npol;
    int sampling;            /* SincCorrector "sampling" = wproj.convFunction.sampling */
    int pol_type;            /* MTB_POL_LINEAR or MTB_POL_CIRCULAR                     */
    int external_planes;     /* 1: the FP64 FFT planes are the caller's d_planes (of
                                mtb_finalize_planes_bytes bytes) and the workspace holds
                                only the cuFFT work area (for engines that cap scratch
                                buffers, such as GAFW's int buffer size)                */
    void *d_planes;          /* with external_planes: complex128 [P][ny][nx] (device,
                                256-byte aligned); contents need not be kept            */
} mtb_finalize_params;

int mtb_finalize_workspace_size(const mtb_finalize_params *p, size_t *bytes);
int mtb_finalize_planes_bytes(const mtb_finalize_params *p, size_t *bytes);

/* Grid (+ optional compensation term) and normaliser to the corrected Stokes
 * cube: ImageFinalizer::calculate (ImageFinalizer.cpp:60-65). */
int mtb_finalize(const mtb_finalize_params *p, const void *d_grid, const void *d_grid_lo,
                 const float *d_normalizer, float *d_image, void *d_workspace,
                 size_t workspace_bytes, mtb_stream_t stream);

/* ---------------------------------------------------------------- misc -- */
const char *mtb_status_string(int status);
int mtb_version(void);
/* Releases cached cuFFT plans (plans are created on first use per shape). */
void mtb_release_caches(void);
/* Number of this library's own kernels launched so far in the process
 * (cuFFT and CUB launches are not counted). */
unsigned long long mtb_kernel_launch_count(void);
/* Measures the FP32 FMA throughput of the current GPU (TFLOP/s, packed
 * f32x2 FMA chains on every SM): the roofline denominator of the gridder.
 * Synchronises `stream`. */
int mtb_calibrate_fp32(double *tflops, mtb_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* MTB_H */
