/*
 * mtb_engine.h -- imaging request engine (continuous batching on one GPU).
 *
 * No counterpart in the reference, which images one MeasurementSet per
 * process and rebuilds its w-kernels every run
 * (code/mt-imager/lib/components/ConvolutionFunctionsGenerator/
 * WProjectionConvFunction.cpp:186-291).  The engine accepts imaging requests
 * of any geometry and record count while others run:
 *   - a request is admitted when a worker slot is free and its device memory
 *     (grid, compensation grid, delta grid, workspace, staging, image) fits in
 *     the engine's HBM budget, in arrival order;
 *   - each slot owns a CUDA stream, so admitted requests overlap on the GPU;
 *   - w-kernel tables are cached by geometry (LRU within a byte budget) and
 *     shared by every request of that geometry;
 *   - a request's records are streamed in chunks from host memory through
 *     pinned, double-buffered staging, each chunk gridded by mtb_grid; host
 *     copies to and from pinned memory are split over a pool of threads.
 * The image of a request is the same whether it runs alone or in a mix (to
 * the rounding of the FP32 reductions, or exactly with exact_delta).
 */
#ifndef MTB_ENGINE_H
#define MTB_ENGINE_H

#include "mtb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mtb_engine mtb_engine;

typedef struct mtb_engine_config {
    int slots;                    /* requests in flight at once; 0: 4                      */
    size_t hbm_budget_bytes;      /* device memory for admitted requests; 0: 70% of free   */
    size_t kernel_cache_bytes;    /* w-kernel tables kept resident; 0: 4 GiB               */
    int chunk_records;            /* records per mtb_grid call; 0: 4,194,304               */
    int host_threads;             /* threads copying between the caller's host arrays and
                                     pinned memory (shared by the slots); 0: min(8, cores/2) */
} mtb_engine_config;

typedef struct mtb_image_request {
    mtb_wkernel_params geometry;  /* image size, cell, w-planes, oversampling (mtb.h)      */
    int npol;                     /* 1, 2 or 4                                             */
    int pol_type;                 /* MTB_POL_LINEAR / MTB_POL_CIRCULAR                     */
    int compensated;              /* two-float grid (1) or plain FP32 grid (0)             */
    int nrecords;
    /* host inputs, layouts of mtb.h; they must stay valid until the request is done */
    const float *uvw;             /* [3][R]                                                */
    const float *freq;            /* [R]  nu / c                                           */
    const void *vis;              /* complex64 [R][P]                                      */
    const float *weights;         /* [R][P]                                                */
    const int *flags;             /* [R][P]                                                */
    float *image;                 /* host output [P][ny][nx]                               */
    int exact_delta;              /* compensated gridding with an FP64 per-call delta grid
                                     (order-independent result); see mtb_grid_params       */
    long long uvw_row_stride;     /* floats between the u, v and w rows of uvw (a slice of
                                     a longer uvw array); 0: nrecords                      */
    int flags_u8;                 /* 1: flags is uint8 [R][P] (one byte per flag), passed
                                     cast to int *; 0: int32 [R][P]; other values (the
                                     bit-packed flags mtb_grid takes) are refused          */
} mtb_image_request;

typedef struct mtb_image_result {
    int status;                   /* MTB_OK or the first error                             */
    int kernel_cache_hit;         /* 1: the geometry's w-kernels were already resident     */
    double queue_ms;              /* submit -> admission                                   */
    double service_ms;            /* admission -> image on the host                        */
    double latency_ms;            /* submit -> image on the host                           */
    mtb_grid_stats stats;         /* record statistics of the image                        */
} mtb_image_result;

/* Creates the engine on the current device and starts its worker threads. */
int mtb_engine_create(const mtb_engine_config *cfg, mtb_engine **engine);
/* Queues a request; returns at once with a ticket.  Requests larger than the
 * whole budget are refused with MTB_ERR_CAPACITY. */
int mtb_engine_submit(mtb_engine *engine, const mtb_image_request *req, long long *ticket);
/* Blocks until the request is done and returns its result (once per ticket). */
int mtb_engine_wait(mtb_engine *engine, long long ticket, mtb_image_result *result);
/* Cancels a request that has not completed: a queued request is dropped at
 * once; a running one stops at its next chunk boundary (the work already
 * enqueued on its stream completes first) and skips the finalisation.  Its
 * result, from mtb_engine_wait, carries MTB_ERR_CANCELLED and its image is
 * undefined; a request that had already completed keeps its result.
 * Unknown (or already waited-for) tickets return MTB_ERR_BAD_PARAM. */
int mtb_engine_cancel(mtb_engine *engine, long long ticket);
/* Device bytes a request is admitted with. */
int mtb_engine_request_bytes(const mtb_engine *engine, const mtb_image_request *req, size_t *bytes);
/* Finishes the queued requests, stops the workers and frees everything. */
int mtb_engine_destroy(mtb_engine *engine);

#ifdef __cplusplus
}
#endif
#endif /* MTB_ENGINE_H */
