/* dwo.h -- oracle: CPU restatement of deconwolf's SHB / RL deconvolution.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (deconwolf_b200/, the
 * C-ABI in include/) may include, link or call this.  Only tests/, the smoke
 * check and bench.py's CPU-baseline leg use it, and only as the checker.
 *
 * The option fields and their meaning follow deconwolf's dw_opts (src/dw.h:
 * 104-211); enum values equal the reference's enums (src/dw.h:52-83).
 */
#ifndef ORACLE_DWO_H
#define ORACLE_DWO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dwo_opts {
    int32_t method;          /* 0 = RL (DW_METHOD_RL), 2 = SHB (DW_METHOD_SHB) */
    int32_t n_iter;          /* nIter */
    int32_t iter_type;       /* 0 ABS, 1 REL, 2 FIXED (dw_iter_type) */
    int32_t maxiter;
    float err_rel;
    float err_abs;
    float bg;                /* in/out: replaced by the automatic value if bg_auto */
    int32_t bg_auto;
    int32_t positivity;
    int32_t border_quality;  /* bq: 0, 1, 2 */
    int32_t start_condition; /* 0 FLAT, 1 LP (Gaussian low-pass, sigma 8), 2 IDENTITY */
    int32_t metric;          /* 0 MSE, 1 IDIV */
    float alphamax;
    int32_t threads;         /* OpenMP threads, <= 0: default */
    int64_t work[3];         /* 0,0,0: the reference's job size; else padded size (bq=2 only) */
    /* outputs */
    int32_t iterations_done;
    float *error_trace;      /* optional, capacity trace_capacity */
    int32_t trace_capacity;
    double loop_seconds;     /* wall time of the iteration loop */
    double setup_seconds;    /* wall time before the loop */
} dwo_opts;

void dwo_opts_default(dwo_opts *s);

/* Deconvolve im (M x N x P, x fastest) with psf (pM x pN x pP).
 * out receives M*N*P floats.  Returns 0 on success, < 0 on a rejected input
 * (the reference exit()s in those cases). */
int dwo_deconvolve(const float *im, int64_t M, int64_t N, int64_t P,
                   const float *psf, int64_t pM, int64_t pN, int64_t pP,
                   dwo_opts *s, float *out);

/* Building blocks exposed for unit tests. */
void dwo_fft_r2c(const float *in, int64_t M, int64_t N, int64_t P, float *out, int threads);
void dwo_fft_c2r(float *in, int64_t M, int64_t N, int64_t P, float *out, int threads);
void dwo_argmax(const float *I, int64_t M, int64_t N, int64_t P,
                int64_t *aM, int64_t *aN, int64_t *aP);
void dwo_circshift(float *A, int64_t M, int64_t N, int64_t P,
                   int64_t sm, int64_t sn, int64_t sp);
float dwo_idiv(const float *y, const float *g, int64_t M, int64_t N, int64_t P,
               int64_t wM, int64_t wN, int64_t wP);

/* fim_gsmooth (in place, M x N x P). */
void dwo_gsmooth(float *V, int64_t M, int64_t N, int64_t P, float sigma);

/* PSF preparation and tiling (dwo.c cites the reference lines). */
float *dwo_psf_autocrop(float *psf, int64_t *pM, int64_t *pN, int64_t *pP, int64_t M, int64_t N, int64_t P,
                        int bq, float xycropfactor);
int dwo_psf_prepare(const float *psf, int64_t pM, int64_t pN, int64_t pP, int64_t M, int64_t N, int64_t P,
                    int bq, float xycropfactor, float *out, int64_t out_dims[3]);
int dwo_tiling_create(int64_t M, int64_t N, int64_t P, int64_t max_size, int64_t overlap, int64_t *tiles,
                      int capacity);
float dwo_tile_weight(const int64_t *tile, int64_t m, int64_t n);
int dwo_deconvolve_tiled(const float *im, int64_t M, int64_t N, int64_t P, const float *psf, int64_t pM,
                         int64_t pN, int64_t pP, int64_t tile_size, int64_t overlap, float offset,
                         float xycropfactor, dwo_opts *s, float *out);

#ifdef __cplusplus
}
#endif
#endif
