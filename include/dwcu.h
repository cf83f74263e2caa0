/* dwcu.h -- C ABI of the B200-native Richardson-Lucy / Scaled-Heavy-Ball engine.
 *
 * This is the drop-in boundary for deconwolf's `dw --method shb|rl --gpu` path.
 * deconwolf selects its deconvolution method through a function pointer,
 *
 *     typedef float * (*dw_function)(float * restrict im, int64_t M, N, P,
 *                                    float * restrict psf, int64_t pM, pN, pP,
 *                                    dw_opts * s);                (src/dw.h:89-91)
 *
 * called from dw_run (src/dw.c:2841) and deconvolve_tiles (src/dw.c:2137).
 * dwcu_deconvolve() below is that call with plain C types: the dw_opts fields
 * the iteration honours are carried in dwcu_opts, the result goes to a caller
 * buffer, and failures return a status instead of exit().  The reference-side
 * glue that adapts dw_opts and registers deconvolve_shb_cu / deconvolve_rl_cu
 * as dw_functions is deconwolf_b200/glue/method_shb_cu.c.
 *
 * Layout everywhere: float32, x fastest, index = m + n*M + p*M*N (deconwolf's
 * fim layout), no row padding at this boundary.
 *
 * All functions return 0 (DWCU_SUCCESS) or a positive dwcu_status; the text
 * of the last failure on the calling thread is dwcu_last_error().  No
 * function falls back to the CPU: without a usable CUDA device every compute
 * call fails with DWCU_ERROR_CUDA.
 */
#ifndef DWCU_H
#define DWCU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DWCU_ABI_VERSION 1

typedef enum dwcu_status {
    DWCU_SUCCESS = 0,
    DWCU_ERROR_INVALID_VALUE = 1, /* bad argument (sizes, null pointers, options) */
    DWCU_ERROR_UNSUPPORTED = 2,   /* valid for deconwolf, not implemented here (e.g. a job longer than the longest transform, or bq 0/1 periodic margins with an off-centre PSF maximum) */
    DWCU_ERROR_OUT_OF_MEMORY = 3, /* device allocation failed or HBM budget exceeded */
    DWCU_ERROR_CUDA = 4,          /* CUDA runtime / launch failure, or no device */
    DWCU_ERROR_INPUT = 5,         /* non-finite image or PSF values */
    DWCU_ERROR_NOT_READY = 6,     /* asynchronous work still running */
    DWCU_ERROR_CANCELLED = 7,     /* a job was cancelled before it finished */
    DWCU_ERROR_TIMEOUT = 8,       /* a bounded wait gave up */
    DWCU_ERROR_INTERNAL = 9,
    DWCU_ERROR_IO = 10            /* a file could not be read or written (tuning tables) */
} dwcu_status;

/* Enum values equal deconwolf's own (src/dw.h:52-83). */
enum { DWCU_METHOD_RL = 0, DWCU_METHOD_SHB = 2 };
enum { DWCU_START_FLAT = 0, DWCU_START_LP = 1, DWCU_START_IDENTITY = 2 };
enum { DWCU_METRIC_MSE = 0, DWCU_METRIC_IDIV = 1 };
enum { DWCU_ITER_ABS = 0, DWCU_ITER_REL = 1, DWCU_ITER_FIXED = 2 };

/* The dw_opts fields the iteration reads (src/dw.h:104-211), same meaning. */
typedef struct dwcu_opts {
    int32_t method;          /* DWCU_METHOD_SHB (default) or DWCU_METHOD_RL   (dw_opts.method) */
    int32_t n_iter;          /* iterations for DWCU_ITER_FIXED               (dw_opts.nIter) */
    int32_t iter_type;       /* stopping rule, default DWCU_ITER_REL          (dw_opts.iter_type) */
    int32_t maxiter;         /* cap for REL / ABS, default 250                (dw_opts.maxiter) */
    float err_rel;           /* REL threshold, default 0.02                   (dw_opts.err_rel) */
    float err_abs;           /* ABS threshold                                  (dw_opts.err_abs) */
    float bg;                /* background; overwritten when bg_auto          (dw_opts.bg) */
    int32_t bg_auto;         /* 1: bg = max(min(image), 0.01), default 1       (dw_opts.bg_auto) */
    int32_t positivity;      /* SHB: clamp the estimate at bg, default 1      (dw_opts.positivity) */
    int32_t border_quality;  /* 2 (default); 1 and 0 convolve periodically    (dw_opts.borderQuality) */
    int32_t start_condition; /* FLAT (default), IDENTITY or LP (sigma 8)      (dw_opts.start_condition) */
    int32_t metric;          /* IDIV (default) or MSE                         (dw_opts.metric) */
    float alphamax;          /* SHB extrapolation cap, default 1              (dw_opts.alphamax) */
    int32_t device;          /* CUDA device ordinal                            (dw_opts.cl_device) */
    int32_t verbosity;       /* 0 silent; > 0 prints per-iteration lines      (dw_opts.verbosity) */
    int32_t use_graph;       /* FIXED iterations: capture the loop in a CUDA graph (default 1) */
    /* outputs */
    int32_t iterations_done; /* iterations run */
    float *error_trace;      /* optional host array: error of each iteration */
    int32_t trace_capacity;  /* its length */
    int64_t work[3];         /* padded job size used (X, Y, Z) */
    double seconds_setup;    /* device time before the first iteration */
    double seconds_iterate;  /* device time of the iteration loop */
    double seconds_enqueue;  /* host time spent issuing the iterations (graph capture included) */
} dwcu_opts;

/* Defaults of dw_opts_new (src/dw.c:340-413) for the fields above. */
void dwcu_opts_init(dwcu_opts *s);

/* ---------------------------------------------------------------- one call */

/* Deconvolve the host image im (M x N x P) with the host PSF (pM x pN x pP)
 * into the host buffer out (M x N x P).  Replaces the dw_function call
 * s->fun(im, M, N, P, psf, pM, pN, pP, s) (src/dw.c:2841) for the methods
 * deconvolve_shb (src/method_shb.c:77-424), deconvolve_rl
 * (src/method_rl.c:105-400) and deconvolve_shb_cl2 (src/method_shb_cl2.c:
 * 166-602).  im and psf are only read.  SHB returns the iterate before the
 * last update (method_shb.c:385-395), RL the last one (method_rl.c:393);
 * n_iter == 0 copies the image (method_shb.c:101-105). */
int dwcu_deconvolve(const float *im, int64_t M, int64_t N, int64_t P,
                    const float *psf, int64_t pM, int64_t pN, int64_t pP,
                    dwcu_opts *s, float *out);

/* Same with device-resident buffers (device s->device): d_im, d_psf and d_out
 * are device pointers; work is ordered on `stream` (a cudaStream_t, NULL for
 * the default stream) and the call returns after it completes. */
int dwcu_deconvolve_device(const float *d_im, int64_t M, int64_t N, int64_t P,
                           const float *d_psf, int64_t pM, int64_t pN, int64_t pP,
                           dwcu_opts *s, float *d_out, void *stream);

/* The padded job size (X, Y, Z) the engine uses for these sizes, and the
 * device bytes one job needs.  Returns DWCU_ERROR_UNSUPPORTED when no
 * supported FFT length covers the job (see border_quality). */
int dwcu_plan_size(int64_t M, int64_t N, int64_t P, int64_t pM, int64_t pN, int64_t pP,
                   int32_t border_quality, int32_t method, int64_t work[3], int64_t *device_bytes);

/* One image over several GPUs: the dw_function call (as dwcu_deconvolve) with
 * the job split into nparts slabs of z planes, part p holding the planes
 * z = l*nparts + p.  Each part runs the x and y passes of its planes on its
 * GPU; the z pass runs per part on a slab of spectrum columns of every
 * plane, read and written in place over peer access (NVLink) where every
 * pair of the GPUs has it, else on copies gathered from and scattered back
 * to every part (environment DWCU_SLAB_TRANSPOSE=copy forces the copies).
 * devices[p] is part p's GPU (NULL: every part on s->device; parts may
 * share a GPU).  For jobs larger than one GPU's memory, where deconwolf tiles
 * the image (src/dw.c:2001-2229).  Not supported (DWCU_ERROR_UNSUPPORTED):
 * a job z size that needs periodic margins (border_quality 0 / 1 without an
 * exact-size z transform). */
int dwcu_deconvolve_slabs(const float *im, int64_t M, int64_t N, int64_t P,
                          const float *psf, int64_t pM, int64_t pN, int64_t pP,
                          dwcu_opts *s, int32_t nparts, const int32_t *devices, float *out);

/* The share of part `part` of nparts (host arithmetic, no device):
 * info[0] z planes, info[1] image planes, info[2] first z-pass column,
 * info[3] z-pass columns, info[4] columns per plane, info[5] padded Z. */
int dwcu_slab_layout(int64_t M, int64_t N, int64_t P, int64_t pM, int64_t pN, int64_t pP,
                     int32_t border_quality, int32_t nparts, int32_t part, int64_t info[6]);

/* The same split with one process per part (a process per GPU, e.g. under
 * torchrun): each process creates its part, exports the handle of its
 * spectrum, imports every other part's (CUDA IPC), and runs.  The caller
 * provides the collectives; every process calls them at the same points in
 * the same order, with its part's stream:
 *   barrier    work queued on `stream` before the call completes on every
 *              part before work queued after it starts on any part (a
 *              stream-ordered collective such as an NCCL all-reduce on that
 *              stream, or a host barrier after synchronising the stream);
 *   allreduce  the first n doubles of the sync buffer summed (op 0) or their
 *              minimum taken (op 1) over the parts, in place, ordered the
 *              same way.
 * Both return 0 on success.  The plans are the recorded ones (an imported
 * plan table, the same in every process) or the heuristic ones: no process
 * measures plans of its own. */
typedef struct dwcu_slab dwcu_slab;
typedef struct dwcu_slab_sync {
    int (*barrier)(void *ctx, void *stream);
    int (*allreduce)(void *ctx, void *stream, int32_t n, int32_t op);
    void *ctx;
} dwcu_slab_sync;

/* Part `part` of nparts on s->device; sync_buf: the caller's device buffer of
 * at least 4 doubles (the allreduce's data). */
int dwcu_slab_part_create(int64_t M, int64_t N, int64_t P, int64_t pM, int64_t pN, int64_t pP,
                          const dwcu_opts *s, int32_t nparts, int32_t part, double *sync_buf,
                          const dwcu_slab_sync *sync, dwcu_slab **out);
/* The IPC handle (64 bytes) of the part's memory and its spectrum's offset in it. */
int dwcu_slab_part_export(dwcu_slab *sl, void *handle, int64_t *offset);
/* Map another part's spectrum from its exported handle and offset. */
int dwcu_slab_part_import(dwcu_slab *sl, int32_t part, const void *handle, int64_t offset);
/* Set-up, iterations and result: im and psf are the whole image and PSF (host);
 * the part writes its own image planes z = l*nparts + part of `out` (host,
 * M x N x P) and leaves the others untouched; s_out as dwcu_deconvolve's. */
int dwcu_slab_part_run(dwcu_slab *sl, const float *im, const float *psf, float *out, dwcu_opts *s_out);
void dwcu_slab_destroy(dwcu_slab *sl);

/* ---------------------------------------------------------------- jobs */

/* A job keeps its image, OTF, weights and estimates resident on the device
 * so that many jobs (tiles, channels, requests) can be stepped in any
 * interleaving.  Jobs created on the same device share that device's stream
 * unless dwcu_job_set_stream is called. */
typedef struct dwcu_job dwcu_job;

/* Allocate a job for an M x N x P image and pM x pN x pP PSF with options s
 * (copied).  Returns DWCU_ERROR_OUT_OF_MEMORY when the device allocation
 * fails. */
int dwcu_job_create(int64_t M, int64_t N, int64_t P, int64_t pM, int64_t pN, int64_t pP,
                    const dwcu_opts *s, dwcu_job **job);
/* Upload image and PSF (host pointers, or device pointers when on_device)
 * and run the setup: background, OTF, Bertero weights, start estimate. */
int dwcu_job_setup(dwcu_job *job, const float *im, const float *psf, int32_t on_device);
/* Enqueue up to n more iterations (without waiting).  The stopping rule of
 * s->iter_type is applied; REL and ABS read each error back (one small copy
 * per iteration).  *remaining receives how many iterations may still run. */
int dwcu_job_step(dwcu_job *job, int32_t n, int32_t *remaining);
/* Run set-up jobs to completion together: each job with a fixed iteration
 * count replays its iteration loop as one CUDA graph (cached with its
 * device block, so a job of the same sizes on a reused block captures
 * nothing) on a stream of its own; jobs large enough to fill the GPU
 * (>= 32 Mi padded voxels) run one after another on one stream, smaller
 * ones side by side, so tiles and channels of uneven sizes share the GPU;
 * REL/ABS jobs are stepped round-robin.  Replaces the sequential tile loop of deconvolve_tiles
 * (src/dw.c:2093-2153) for the iteration part.  Returns when all are done;
 * results are then read with dwcu_job_result. */
int dwcu_batch_run(dwcu_job **jobs, int32_t n, void *stream);
/* 1 when the job has finished all its iterations. */
int dwcu_job_done(const dwcu_job *job);
/* Wait for the job's queued work; copy the result (host or device pointer)
 * and the error trace.  Fills s-like outputs into *s_out when non-NULL. */
int dwcu_job_result(dwcu_job *job, float *out, int32_t out_on_device, dwcu_opts *s_out);
/* Release the job.  Its device block is kept by the library for the next
 * job of a similar size (at most 64 blocks and half of the device's
 * memory per device); dwcu_release_cache frees those. */
void dwcu_job_destroy(dwcu_job *job);
/* Free the device blocks the library keeps for reuse on `device` (all
 * devices when negative).  No counterpart in the reference, which allocates
 * per call. */
int dwcu_release_cache(int32_t device);
/* Use a caller stream (cudaStream_t) for this job's work. */
int dwcu_job_set_stream(dwcu_job *job, void *stream);
/* Device bytes held by the job. */
int64_t dwcu_job_bytes(const dwcu_job *job);

/* ---------------------------------------------------------------- checkpoints */

/* The state of a job between iterations, for preemption and restarts (the
 * reference has no checkpoint; its --iterdump images cannot be resumed,
 * src/method_shb.c:302-322).  The estimates are two padded real volumes of
 * volume_elems floats: x_k and, for SHB, x_{k-1}. */
typedef struct dwcu_job_state {
    int64_t volume_elems;  /* floats per volume */
    int32_t next_iter;     /* the iteration that runs next; -1 when finished */
    int32_t done_iters;    /* error values in the trace */
    int32_t iter;          /* the stopping rule's counter (dw_iterator_t.iter) */
    float error;           /* the stopping rule's last two error values */
    float lasterror;
    float bg;              /* the background the job uses */
} dwcu_job_state;

/* Copy a set-up job's state to host memory: x_k into x and, for SHB,
 * x_{k-1} into x_prev (st->volume_elems floats each; with x == NULL only *st
 * is filled, to learn the size), and the first done_iters error values into
 * trace (up to trace_capacity; trace may be NULL).  Waits for the job's
 * queued work. */
int dwcu_job_snapshot(dwcu_job *job, float *x, float *x_prev, float *trace, int32_t trace_capacity,
                      dwcu_job_state *st);

/* Continue from a snapshot: `job` was created and set up with the same image,
 * PSF and options as the job snapshotted (the set-up recomputes the OTF,
 * weights and background); its estimates, error trace and iteration state
 * are replaced by the snapshot's, and the next dwcu_job_step continues at
 * st->next_iter.  DWCU_ERROR_INVALID_VALUE for a snapshot of another job
 * size or background. */
int dwcu_job_restore(dwcu_job *job, const float *x, const float *x_prev, const float *trace,
                     const dwcu_job_state *st);

/* ---------------------------------------------------------------- PSF and tiles */

/* Prepare a PSF for an M x N x P job the way dw_run does before the method
 * call (src/dw.c:2797-2826 with psf_autocrop, src/dw.c:1973-1997): normalise
 * to sum 1 (fim_normalize_sum1, src/fim.c:900-912), crop to at most
 * 2*size-1 per axis (size with border_quality 0; psf_autocrop_byImage,
 * src/dw.c:1764-1860), drop outer x/y planes holding less than xycropfactor
 * of the largest y-z plane sum (border_quality > 0 only; psf_autocrop_XY
 * without the FFT lookahead, src/dw.c:1862-1971), normalise again.  out must
 * hold pM*pN*pP floats; out_dims receives the new size. */
int dwcu_psf_prepare(const float *psf, int64_t pM, int64_t pN, int64_t pP,
                     int64_t M, int64_t N, int64_t P, int32_t border_quality,
                     float xycropfactor, float *out, int64_t out_dims[3]);
/* dwcu_psf_prepare on the device: d_psf (device, pM*pN*pP floats, not
 * modified) prepared into d_out (device, room for pM*pN*pP floats) with the
 * same steps and the same float results (the crop decision from float
 * plane sums in the reference's order; the normalisations' double sums in a
 * fixed tree).  Work space is allocated and freed inside; returns after
 * `stream` (NULL: the calling thread's default stream) has drained, with
 * the new size in out_dims.  The tiled path (dwcu_deconvolve_tiled)
 * prepares each tile size's PSF with it. */
int dwcu_psf_prepare_device(const float *d_psf, int64_t pM, int64_t pN, int64_t pP, int64_t M, int64_t N,
                            int64_t P, int32_t border_quality, float xycropfactor, float *d_out, int64_t out_dims[3],
                            int32_t device, void *stream);

/* One tile of a tiling (struct tile, src/tiling.h:29-34): the owned region
 * pos = [m0, m1, n0, n1, p0, p1] and the region deconvolved xpos (pos grown
 * by the overlap and clipped to the image), with their sizes. */
typedef struct dwcu_tile {
    int64_t size[3];
    int64_t pos[6];
    int64_t xpos[6];
    int64_t xsize[3];
} dwcu_tile;

/* The tiling tiling_create(M, N, P, max_size, overlap) builds (src/tiling.c:
 * 22-130): x and y cut into ceil(L / max_size) near-equal sections, tiles
 * ordered x-section outer, y-section inner.  *ntiles receives the count;
 * tiles (capacity entries, may be NULL to query the count) the tiles. */
int dwcu_tiling_create(int64_t M, int64_t N, int64_t P, int64_t max_size, int64_t overlap,
                       dwcu_tile *tiles, int32_t capacity, int32_t *ntiles);

/* Tiled deconvolution, deconvolve_tiles (src/dw.c:2001-2229) with the image
 * and the result in memory instead of temporary raw files: im and out are
 * host M x N x P buffers, psf the PSF as deconvolve_tiles receives it (from
 * dw_run, already normalised and cropped against the whole image).  Per tile
 * the PSF is normalised, cropped against the tile and normalised again, the
 * tile gets +offset (when offset > 0), is deconvolved with options s, gets
 * -offset and is clipped at 0, and is blended into out with the weights of
 * tiling_put_tile (src/tiling.c:412-439), in tile order.  The tiles run as
 * batches (dwcu_batch_run) of as many tiles as fit hbm_budget bytes (<= 0:
 * 85 % of the free device memory).  Fails with DWCU_ERROR_INVALID_VALUE for a
 * tiling of one tile, as the reference does. */
int dwcu_deconvolve_tiled(const float *im, int64_t M, int64_t N, int64_t P,
                          const float *psf, int64_t pM, int64_t pN, int64_t pP,
                          int64_t tile_size, int64_t overlap, float offset, float xycropfactor,
                          double hbm_budget, dwcu_opts *s, float *out);

/* Blend one deconvolved tile (device buffer d_tile, tiles[tid].xsize) into the
 * device volume d_out (M x N x P): minus offset and clipped at 0 when
 * offset > 0 (dw.c:2141-2145), then out += w / sum_w * tile with the weights
 * of tiling_put_tile (src/tiling.c:412-439).  Tiles blended in tile order give
 * deconvolve_tiles' result; tiles spread over several GPUs can be blended
 * per GPU and the volumes summed.  Synchronises the stream. */
int dwcu_tile_blend(float *d_out, int64_t M, int64_t N, int64_t P, const dwcu_tile *tiles, int32_t ntiles,
                    int32_t tid, const float *d_tile, float offset, int32_t device, void *stream);

/* ---------------------------------------------------------------- serving */

/* A request server on one GPU (no counterpart in the reference, which runs
 * one image per process): requests are dw_function calls (host image, host
 * PSF, options, host result buffer) queued from any thread.  A worker thread
 * admits them in arrival order while their device memory (dwcu_plan_size)
 * fits hbm_budget bytes (<= 0: 85 % of the free memory) and at most
 * max_active run, keeps each job's state resident on the device, and
 * interleaves the jobs' iterations on one stream per job, iters_per_turn
 * iterations at a time.  A request's result equals dwcu_deconvolve's on the
 * same inputs.  The caller keeps im, psf and out alive until the request has
 * finished (dwcu_server_wait). */
typedef struct dwcu_server dwcu_server;
typedef struct dwcu_server_stats {
    int64_t submitted, completed, failed, cancelled, active, queued;
    double device_bytes_in_use;
    double latency_p50_s, latency_p99_s, latency_mean_s;  /* submit -> result in the host buffer */
    double voxel_iterations;  /* sum over completed requests of image voxels x iterations */
    double wall_s;            /* first submit -> last completion */
} dwcu_server_stats;
int dwcu_server_create(int32_t device, double hbm_budget, int32_t max_active, int32_t iters_per_turn,
                       dwcu_server **server);
/* Queue one request; *id identifies it.  s->device must be the server's. */
int dwcu_server_submit(dwcu_server *server, const float *im, int64_t M, int64_t N, int64_t P,
                       const float *psf, int64_t pM, int64_t pN, int64_t pP, const dwcu_opts *s,
                       float *out, int64_t *id);
/* Wait up to timeout_s seconds (< 0: no limit) for a request.  Returns
 * DWCU_SUCCESS (result in out, outputs in *s_out), DWCU_ERROR_NOT_READY on
 * timeout, DWCU_ERROR_CANCELLED, or the request's failure status. */
int dwcu_server_wait(dwcu_server *server, int64_t id, double timeout_s, dwcu_opts *s_out);
/* Cancel a request: a queued one never starts, a running one stops after
 * its chunk in flight and releases its memory. */
int dwcu_server_cancel(dwcu_server *server, int64_t id);
int dwcu_server_get_stats(dwcu_server *server, dwcu_server_stats *stats);
/* Cancel queued requests, finish running ones, stop the worker. */
void dwcu_server_destroy(dwcu_server *server);

/* ---------------------------------------------------------------- FFT */

/* 3-D real-to-complex transform of d_in (M x N x P floats, device) into
 * d_out ((M/2+1) x N x P interleaved complex, device), unnormalised, the
 * layout of fftwf_plan_dft_r2c_3d(P, N, M, ...).  Replaces fft() (src/fft.c:
 * 401-415).  M must be even with M/2, N and P supported lengths. */
int dwcu_fft_r2c(const float *d_in, int64_t M, int64_t N, int64_t P, float *d_out, int32_t device,
                 void *stream);
/* Complex-to-real inverse of the above, unnormalised (the caller divides by
 * M*N*P as ifft() does, src/fft.c:383-398).  d_in is not modified. */
int dwcu_fft_c2r(const float *d_in, int64_t M, int64_t N, int64_t P, float *d_out, int32_t device,
                 void *stream);

/* dwcu_fft_r2c without any device-memory allocation.  No counterpart in the
 * reference (deconwolf's fft.c has no allocation-free transform).  Same
 * transform, arguments and result as dwcu_fft_r2c, but the work space is a
 * fixed 32 MiB array in the library's device image (one per device) instead
 * of a cudaMalloc / cudaFree per call: for callers that cannot allocate
 * (a fixed device-memory budget held by their own pool) or cannot afford the
 * device-wide synchronisation of cudaFree while other streams of the GPU are
 * busy.  Transforms whose spectrum, staged input and twiddle tables need more
 * than the work space are rejected with DWCU_ERROR_INVALID_VALUE.  The first
 * call on a device does one-time setup (symbol lookup, kernel attributes),
 * so make that first call before any stream capture.  Calls on one device
 * share the work space, which keeps the last call's contents (each call
 * clears the parts that must start at zero); two calls whose GPU work
 * overlapped would race on it, so calls are serialised by a lock and each
 * returns after its stream has drained.  A NULL stream means the
 * calling thread's default stream (cudaStreamPerThread); pass a stream of
 * your own to keep the transform beside other work.  The caller's current
 * device is left as it was. */
int dwcu_fft_r2c_noalloc(const float *d_in, int64_t M, int64_t N, int64_t P, float *d_out, int32_t device,
                         void *stream);

/* ---------------------------------------------------------------- autotuning */

/* The FFT passes have one or more candidate plans per transform length
 * (radix lists; for the strided line pass also the number of columns per
 * block); candidate 0 is the generator's heuristic choice.  With tuning on
 * (the default; DWCU_AUTOTUNE=0 in the environment turns it off), the first
 * job that needs a length on a device times that length's candidates of
 * each pass kind on a synthetic volume (CUDA events, a few launches each,
 * milliseconds in all) and keeps the fastest; later jobs use the recorded
 * choice.  The first job of a new size therefore takes a little longer to
 * create, and its creation should not happen during stream capture.  The
 * measurement uses a few hundred MB of device memory of its own (outside a
 * server's HBM budget), freed right after; freeing waits for the device, so
 * a serving process that must never stall other streams imports a table
 * (dwcu_tune_import) or runs dwcu_tune_run for its sizes at start-up.
 * Replaces FFTW's planning by measurement (fft_train, src/fft.c:206-319;
 * FFTW_MEASURE, src/dw.c:400) and its wisdom files (src/fft.c:299-316, 355):
 * dwcu_tune_export writes the table as text, dwcu_tune_import reads it back
 * (imported choices apply to every device and are not measured again). */
enum { DWCU_TUNE_OFF = 0, DWCU_TUNE_MEASURE = 1 };
enum { DWCU_PLAN_LINES = 0, DWCU_PLAN_Y = 1, DWCU_PLAN_X = 2 };
int dwcu_tune_set_mode(int32_t mode);
int dwcu_tune_get_mode(int32_t *mode);
/* The selection rule, on candidate times in ms: the index of the fastest,
 * unless it is not faster than candidate 0 by more than `margin` (relative),
 * in which case 0.  Non-finite or negative times are candidates that could
 * not run.  (Pure host logic.) */
int dwcu_tune_select(const float *ms, int32_t n, float margin, int32_t *choice);
/* Candidates of a length for a pass kind (0: length not supported). */
int dwcu_tune_plan_count(int32_t kind, int32_t n, int32_t *count);
/* Radix list (radices[3], 1 = unused) and tile of one candidate: columns per
 * block (lines), rows per block (x), lines per tile (y, always 4). */
int dwcu_tune_plan_info(int32_t kind, int32_t n, int32_t cand, int32_t *radices, int32_t *tile);
/* Use candidate `cand` for this length on every device from now on (cand -1:
 * forget the length, so the next job measures it again). */
int dwcu_tune_force(int32_t kind, int32_t n, int32_t cand);
/* Time the candidates of one length on a device now (if not recorded yet). */
int dwcu_tune_run(int32_t device, int32_t kind, int32_t n);
/* The recorded choice for (device, kind, n): *cand = -1 if none; ms[i] the
 * measured time of candidate i (*nms of them; 0 when imported or forced). */
int dwcu_tune_query(int32_t device, int32_t kind, int32_t n, int32_t *cand, float *ms, int32_t cap, int32_t *nms);
int dwcu_tune_clear(void);
int dwcu_tune_export(const char *path);
int dwcu_tune_import(const char *path);

/* ---------------------------------------------------------------- timing */

/* Per-kernel-class timing.  While enabled, every pass the engine launches
 * is bracketed by CUDA events recorded on the stream it is launched on
 * (inside CUDA graphs too).  dwcu_profile_collect waits for the recorded
 * work, returns one entry per kernel class and clears the records.
 * bytes_per_launch is the algorithmic HBM traffic of one launch (the bytes
 * the pass must read and write), not a measured counter. */
typedef struct dwcu_kernel_stat {
    char name[40];
    int64_t launches;
    double milliseconds;      /* summed event time of all launches */
    double bytes_per_launch;  /* algorithmic bytes of one launch */
} dwcu_kernel_stat;
int dwcu_profile_enable(int32_t on);
int dwcu_profile_collect(dwcu_kernel_stat *stats, int32_t capacity, int32_t *count);

/* ---------------------------------------------------------------- misc */

/* Text of the last failure on this thread ("" if none). */
const char *dwcu_last_error(void);
/* ABI version, for the caller's check. */
int dwcu_abi_version(void);
/* Number of CUDA devices visible (0 without a GPU; never fails). */
int dwcu_device_count(void);
/* Number of kernel launches this thread has issued through the library. */
int64_t dwcu_launch_count(void);
/* Self-test of the device-side bounded waits every pass uses (TMA copies
 * complete on mbarriers; a wait that runs out of polls sets an error word,
 * the block leaves through one exit, and the host turns the word into
 * DWCU_ERROR_TIMEOUT): one block waits at most `polls` polls on a barrier
 * phase that completes only when `arrive` is non-zero.  Returns
 * DWCU_SUCCESS when the phase completed, DWCU_ERROR_TIMEOUT when the wait
 * gave up; the device stays usable either way.  No counterpart in the
 * reference, which exits on any device error. */
int dwcu_selftest_bounded_wait(int32_t device, int32_t arrive, uint32_t polls);
/* Guard bands, a debugging aid in place of a memory checker: with mode 1,
 * jobs created afterwards put 4 KB of a fixed pattern before and after
 * every buffer of their device block, and dwcu_job_destroy compares them
 * with the pattern; a changed band (a write outside its buffer) is counted
 * and reported on stderr.  Mode 2 also overwrites one byte of each job's
 * first band from the host, to check the check.  Mode 0 (the default) adds
 * nothing.  No counterpart in the reference (which relies on AddressSanitizer
 * builds of its host code). */
int dwcu_debug_guards(int32_t mode);
/* Changed guard bands found so far (all jobs, all threads). */
int64_t dwcu_debug_guard_violations(void);

#ifdef __cplusplus
}
#endif
#endif /* DWCU_H */
