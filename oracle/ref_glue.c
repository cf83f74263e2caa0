/* ref_glue.c -- links deconwolf's own CPU method code into oracle/_ref.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles the reference's
 * src/method_shb.c, src/method_rl.c, src/fft.c, src/fim.c, src/dw_util.c,
 * src/quickselect.c, src/ftab.c, src/npio.c and src/tiling.c unmodified, from
 * where they lie in the
 * reference tree, against oracle/include (FFTW-API shim, libtiff type stub).
 * Those files call a handful of helpers that live in src/dw.c, which pulls in
 * every other deconwolf tool and cannot be compiled here; this file restates
 * the helpers the methods need (each cites the dw.c lines it follows) and
 * stubs the TIFF/NPY I/O entry points that the method path never reaches.
 *
 * dwref_deconvolve() is the single entry point: it builds a dw_opts the way
 * dw_opts_new (dw.c:340-413) does, applies the caller's settings, calls the
 * reference's deconvolve_shb / deconvolve_rl through a dw_function pointer
 * and copies the result out.  The per-iteration error trace and iteration
 * timestamps are recorded by the restated iterator.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <math.h>

#include "dw.h"
#include "fim.h"
#include "fft.h"
#include "method_shb.h"
#include "method_rl.h"
#include "tiling.h"
#include "dwo.h"

/* ------------------------------------------------ trace of the iterator */
static float *g_trace;
static int g_trace_cap;
static int g_iters;
static double g_t_first_next, g_t_last_set;
#define DWREF_MAX_TIMES 4096
static double g_t_set[DWREF_MAX_TIMES]; /* end time of each iteration */

static double mono(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double) t.tv_sec + 1e-9 * (double) t.tv_nsec;
}

/* dw.c:219-235 */
dw_iterator_t *dw_iterator_new(const dw_opts *s)
{
    dw_iterator_t *it = calloc(1, sizeof(dw_iterator_t));
    it->error = 1;
    it->lasterror = 1;
    it->itertype = s->iter_type;
    it->abserror = s->err_abs;
    it->relerror = s->err_rel;
    it->iter = -1;
    it->niter = s->nIter;
    if (it->itertype != DW_ITER_FIXED) it->niter = s->maxiter;
    return it;
}

/* dw.c:237-270 */
int dw_iterator_next(dw_iterator_t *it)
{
    if (it->iter < 0) g_t_first_next = mono();
    it->iter++;
    switch (it->itertype) {
    case DW_ITER_FIXED:
        break;
    case DW_ITER_REL:
        if (it->iter < 2) it->lasterror = 2 * it->error * it->relerror;
        if (fabs(it->error - it->lasterror) / it->error < it->relerror) return -1;
        break;
    case DW_ITER_ABS:
        if (it->iter > 0 && it->error < it->abserror) return -1;
        break;
    }
    if (it->iter >= it->niter) return -1;
    return it->iter;
}

/* dw.c:272-276, plus recording for the oracle */
void dw_iterator_set_error(dw_iterator_t *it, float err)
{
    it->lasterror = it->error;
    it->error = err;
    if (g_trace && it->iter >= 0 && it->iter < g_trace_cap) g_trace[it->iter] = err;
    g_iters = it->iter + 1;
    g_t_last_set = mono();
    if (it->iter >= 0 && it->iter < DWREF_MAX_TIMES) g_t_set[it->iter] = g_t_last_set;
}

/* Seconds of each iteration of the last dwref_deconvolve call (the first
 * measured from the loop's first dw_iterator_next); returns the count. */
int dwref_iteration_seconds(double *out, int cap)
{
    int n = g_iters < cap ? g_iters : cap;
    if (n > DWREF_MAX_TIMES) n = DWREF_MAX_TIMES;
    for (int k = 0; k < n; k++) out[k] = g_t_set[k] - (k == 0 ? g_t_first_next : g_t_set[k - 1]);
    return n;
}

void dw_iterator_show(dw_iterator_t *it, const dw_opts *s) { (void) it; (void) s; }
void dw_iterator_free(dw_iterator_t *it) { free(it); }

/* get_fMSE, dw.c:1461-1490 */
float get_fMSE(const float *restrict y, const float *restrict g,
               const int64_t M, const int64_t N, const int64_t P,
               const int64_t wM, const int64_t wN, const int64_t wP)
{
    (void) wP;
    double e = 0;
    for (int64_t c = 0; c < P; c++)
        for (int64_t b = 0; b < N; b++)
            for (int64_t a = 0; a < M; a++) {
                double yv = y[a + b * wM + c * wM * wN];
                double gv = g[a + b * M + c * M * N];
                e += pow(yv - gv, 2);
            }
    return (float) (e / (double) (M * N * P));
}

/* get_fIdiv, dw.c:1492-1524 */
float get_fIdiv(const float *restrict y, const float *restrict g,
                const int64_t M, const int64_t N, const int64_t P,
                const int64_t wM, const int64_t wN, const int64_t wP)
{
    (void) wP;
    double I = 0;
#pragma omp parallel for reduction(+ : I)
    for (int64_t c = 0; c < P; c++)
        for (int64_t b = 0; b < N; b++)
            for (int64_t a = 0; a < M; a++) {
                double yv = y[a + b * wM + c * wM * wN];
                double gv = g[a + b * M + c * M * N];
                if (yv > 0 && gv > 0) I += gv * logf(gv / yv) - (gv - yv);
            }
    return (float) (I / (double) (M * N * P));
}

/* getError, dw.c:1436-1459 */
float getError(const float *restrict y, const float *restrict g,
               const int64_t M, const int64_t N, const int64_t P,
               const int64_t wM, const int64_t wN, const int64_t wP,
               dw_metric metric)
{
    if (metric == DW_METRIC_MSE) return get_fMSE(y, g, M, N, P, wM, wN, wP);
    return get_fIdiv(y, g, M, N, P, wM, wN, wP);
}

/* initial_guess, dw.c:2497-2520 */
fftwf_complex *initial_guess(dw_fft *ff, const int64_t M, const int64_t N, const int64_t P,
                             const int64_t wM, const int64_t wN, const int64_t wP)
{
    float *one = fim_zeros(wM * wN * wP);
    for (int64_t cc = 0; cc < P; cc++)
        for (int64_t bb = 0; bb < N; bb++)
            for (int64_t aa = 0; aa < M; aa++) one[aa + wM * bb + wM * wN * cc] = 1;
    fftwf_complex *Fone = fft(ff, one, wM, wN, wP);
    fim_free(one);
    return Fone;
}

void putdot(const dw_opts *s) { (void) s; }
void fulldump(dw_opts *s, float *A, size_t M, size_t N, size_t P, char *name)
{
    (void) s; (void) A; (void) M; (void) N; (void) P; (void) name;
}
void benchmark_write(dw_opts *s, int iter, double fMSE, const float *x,
                     const int64_t M, const int64_t N, const int64_t P,
                     const int64_t wM, const int64_t wN, const int64_t wP)
{
    (void) s; (void) iter; (void) fMSE; (void) x; (void) M; (void) N; (void) P;
    (void) wM; (void) wN; (void) wP;
}
char *gen_iterdump_name(const dw_opts *s, int it)
{
    (void) s;
    char *n = malloc(64);
    snprintf(n, 64, "itd%05d.tif", it);
    return n;
}
int64_t int64_t_max(int64_t a, int64_t b) { return a > b ? a : b; }
double clockdiff(struct timespec *end, struct timespec *start)
{
    return (double) (end->tv_sec - start->tv_sec) + 1e-9 * (double) (end->tv_nsec - start->tv_nsec);
}

/* ------------------------------------------------ I/O never reached */
static void io_unreachable(const char *f)
{
    fprintf(stderr, "oracle/_ref: %s is not available in the oracle build\n", f);
    abort();
}
ftif_t *fim_tiff_new(FILE *log, int verbose)
{
    ftif_t *f = calloc(1, sizeof(ftif_t));
    f->log = log;
    f->verbose = verbose;
    return f;
}
void fim_tiff_destroy(ftif_t *f) { free(f); }
int fim_tiff_write(ftif_t *f, const char *fName, const float *V, ttags *T,
                   int64_t N, int64_t M, int64_t P)
{
    (void) f; (void) fName; (void) V; (void) T; (void) N; (void) M; (void) P;
    io_unreachable("fim_tiff_write");
    return 1;
}
int fim_tiff_write_float(ftif_t *f, const char *fName, const float *V, const ttags *T,
                         int64_t N, int64_t M, int64_t P)
{
    (void) f; (void) fName; (void) V; (void) T; (void) N; (void) M; (void) P;
    io_unreachable("fim_tiff_write_float");
    return 1;
}
float *fim_tiff_read(ftif_t *f, const char *fName, ttags *T, int64_t *N0, int64_t *M0, int64_t *P0)
{
    (void) f; (void) fName; (void) T; (void) N0; (void) M0; (void) P0;
    io_unreachable("fim_tiff_read");
    return NULL;
}

int fim_tiff_write_opt(ftif_t *f, const char *fName, const float *V, const ttags *T,
                       int64_t N, int64_t M, int64_t P, float scaling)
{
    (void) f; (void) fName; (void) V; (void) T; (void) N; (void) M; (void) P; (void) scaling;
    io_unreachable("fim_tiff_write_opt");
    return 1;
}
int fim_tiff_get_size(ftif_t *f, const char *fname, int64_t *M, int64_t *N, int64_t *P)
{
    (void) f; (void) fname; (void) M; (void) N; (void) P;
    io_unreachable("fim_tiff_get_size");
    return 1;
}
int fim_tiff_to_raw_f32(ftif_t *f, const char *tif_file_name, const char *output_file_name)
{
    (void) f; (void) tif_file_name; (void) output_file_name;
    io_unreachable("fim_tiff_to_raw_f32");
    return 1;
}

/* ------------------------------------------------ entry point */

/* Runs the reference's deconvolve_shb (method 2) or deconvolve_rl (method 0)
 * with the settings in o (dwo_opts field meanings).  o->work is ignored: the
 * reference always uses its own job size.  Returns 0 or a negative code. */
int dwref_deconvolve(const float *im, int64_t M, int64_t N, int64_t P,
                     const float *psf, int64_t pM, int64_t pN, int64_t pP,
                     dwo_opts *o, float *out)
{
    dw_opts *s = calloc(1, sizeof(dw_opts));
    /* defaults from dw_opts_new, dw.c:340-413 */
    s->nThreads_FFT = o->threads > 0 ? o->threads : 1;
    s->nThreads_OMP = s->nThreads_FFT;
    s->fft_inplace = 1;
    s->nIter = o->n_iter;
    s->maxiter = o->maxiter;
    s->err_rel = o->err_rel;
    s->err_abs = o->err_abs;
    s->iter_type = (dw_iter_type) o->iter_type;
    s->verbosity = 0;
    s->method = o->method == 0 ? DW_METHOD_RL : DW_METHOD_SHB;
    s->fun = o->method == 0 ? deconvolve_rl : deconvolve_shb;
    s->borderQuality = o->border_quality;
    s->positivity = o->positivity;
    s->bg = o->bg;
    s->bg_auto = o->bg_auto;
    s->offset = 5;
    s->metric = (dw_metric) o->metric;
    s->fftw3_planning = FFTW_ESTIMATE;
    s->alphamax = o->alphamax;
    s->start_condition = (dw_start_condition) o->start_condition;
    s->xycropfactor = 0.001f;
    s->log = fopen("/dev/null", "w");

    /* fft.c's wisdom path looks under $HOME/.config; point HOME at a path
     * that does not exist so that nothing is created outside the test. */
    char *home = getenv("HOME");
    char *home_saved = home ? strdup(home) : NULL;
    setenv("HOME", "/nonexistent-dwref-home", 1);

    g_trace = o->error_trace;
    g_trace_cap = o->trace_capacity;
    g_iters = 0;
    g_t_first_next = g_t_last_set = 0;

    float *imc = fim_malloc(sizeof(float) * (size_t) M * N * P);
    memcpy(imc, im, sizeof(float) * (size_t) M * N * P);
    float *psfc = fim_malloc(sizeof(float) * (size_t) pM * pN * pP);
    memcpy(psfc, psf, sizeof(float) * (size_t) pM * pN * pP);

    double t0 = mono();
    dw_function fun = s->fun;
    float *res = fun(imc, M, N, P, psfc, pM, pN, pP, s); /* psf is freed by the callee */
    double t1 = mono();
    if (o->n_iter == 0 && o->method == 0) fim_free(psfc); /* RL's nIter==0 path keeps it */

    if (home_saved) { setenv("HOME", home_saved, 1); free(home_saved); }
    else unsetenv("HOME");

    o->bg = s->bg;
    o->iterations_done = g_iters;
    o->loop_seconds = (g_iters > 0) ? g_t_last_set - g_t_first_next : 0;
    o->setup_seconds = (t1 - t0) - o->loop_seconds;
    int rc = 0;
    if (res) {
        memcpy(out, res, sizeof(float) * (size_t) M * N * P);
        fim_free(res);
    } else {
        rc = -1;
    }
    fim_free(imc);
    fclose(s->log);
    free(s);
    return rc;
}

/* ------------------------------------------------ tiling */

float *fim_tiff_read_sub(ftif_t *f, const char *fName, ttags *T, int64_t *M0, int64_t *N0, int64_t *P0, int sub,
                         int64_t sM, int64_t sN, int64_t sP, int64_t wM, int64_t wN, int64_t wP)
{
    (void) f; (void) fName; (void) T; (void) M0; (void) N0; (void) P0; (void) sub;
    (void) sM; (void) sN; (void) sP; (void) wM; (void) wN; (void) wP;
    io_unreachable("fim_tiff_read_sub");
    return NULL;
}

/* The reference's tiling_create (src/tiling.c:70-130), flattened to 18
 * int64 per tile (size[3], pos[6], xpos[6], xsize[3]); returns the count. */
int dwref_tiling_create(int64_t M, int64_t N, int64_t P, int64_t max_size, int64_t overlap, int64_t *tiles,
                        int capacity)
{
    tiling *T = tiling_create(M, N, P, max_size, overlap);
    int nt = T->nTiles;
    if (tiles && capacity >= nt)
        for (int b = 0; b < nt; b++) {
            tile *t = T->tiles[b];
            memcpy(tiles + 18 * b, t->size, 3 * sizeof(int64_t));
            memcpy(tiles + 18 * b + 3, t->pos, 6 * sizeof(int64_t));
            memcpy(tiles + 18 * b + 9, t->xpos, 6 * sizeof(int64_t));
            memcpy(tiles + 18 * b + 15, t->xsize, 3 * sizeof(int64_t));
        }
    tiling_free(T);
    free(T);
    return nt;
}

/* tiling_getWeights (src/tiling.c:215-223) over a whole M x N plane, for
 * pinning the blend weights. */
void dwref_tiling_weights(int64_t M, int64_t N, int64_t P, int64_t max_size, int64_t overlap, int tid,
                          float *w_tile, float *w_sum)
{
    tiling *T = tiling_create(M, N, P, max_size, overlap);
    for (int64_t n = 0; n < N; n++)
        for (int64_t m = 0; m < M; m++) {
            w_tile[m + n * M] = tile_getWeight(T->tiles[tid], m, n, 0);
            w_sum[m + n * M] = tiling_getWeights(T, m, n, 0);
        }
    tiling_free(T);
    free(T);
}

/* deconvolve_tiles (src/dw.c:2093-2153) with the reference's tiling_create,
 * tiling_get_tile, fim_normalize_sum1, fim_add_scalar, fim_project_positive
 * and tiling_put_tile; psf_autocrop lives in dw.c and is the oracle's
 * restatement (dwo_psf_autocrop).  The image and result stay in memory
 * instead of the temporary raw files.  Returns 0, or -3 for one tile. */
int dwref_deconvolve_tiled(const float *im, int64_t M, int64_t N, int64_t P, const float *psf, int64_t pM,
                           int64_t pN, int64_t pP, int64_t tile_size, int64_t overlap, float offset,
                           float xycropfactor, dwo_opts *o, float *out)
{
    tiling *T = tiling_create(M, N, P, tile_size, overlap);
    if (T->nTiles == 1) {
        tiling_free(T);
        free(T);
        return -3;
    }
    memset(out, 0, sizeof(float) * (size_t) (M * N * P));
    int rc = 0;
    for (int tt = 0; tt < T->nTiles && rc == 0; tt++) {
        float *tpsf = fim_copy(psf, (size_t) (pM * pN * pP));
        int64_t tpM = pM, tpN = pN, tpP = pP;
        float *im_tile = tiling_get_tile(T, tt, im);
        int64_t tileM = T->tiles[tt]->xsize[0], tileN = T->tiles[tt]->xsize[1], tileP = T->tiles[tt]->xsize[2];
        fim_normalize_sum1(tpsf, tpM, tpN, tpP);
        float *tp = malloc(sizeof(float) * (size_t) (pM * pN * pP));
        memcpy(tp, tpsf, sizeof(float) * (size_t) (pM * pN * pP));
        fim_free(tpsf);
        tp = dwo_psf_autocrop(tp, &tpM, &tpN, &tpP, tileM, tileN, tileP, o->border_quality, xycropfactor);
        fim_normalize_sum1(tp, tpM, tpN, tpP);
        size_t tv = (size_t) (tileM * tileN * tileP);
        if (offset > 0) fim_add_scalar(im_tile, tv, offset);
        float *res = fim_malloc(sizeof(float) * tv);
        dwo_opts so = *o;
        so.error_trace = NULL;
        so.trace_capacity = 0;
        rc = dwref_deconvolve(im_tile, tileM, tileN, tileP, tp, tpM, tpN, tpP, &so, res);
        o->iterations_done = so.iterations_done;
        fim_free(im_tile);
        free(tp);
        if (rc == 0) {
            if (offset > 0) {
                fim_add_scalar(res, tv, -offset);
                fim_project_positive(res, tv);
            }
            tiling_put_tile(T, tt, out, res);
        }
        fim_free(res);
    }
    tiling_free(T);
    free(T);
    return rc;
}
