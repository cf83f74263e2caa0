/* method_shb_cu.c -- deconwolf methods backed by the B200 engine (libdwcu) */
#include <stdio.h>
#include <string.h>
#include "dw.h"
#include "fim.h"
#include "dwcu.h"

static float *dwcu_method(float *restrict im, const int64_t M, const int64_t N, const int64_t P,
                          float *restrict psf, const int64_t pM, const int64_t pN, const int64_t pP,
                          dw_opts *s, int32_t method)
{
    dwcu_opts o;
    dwcu_opts_init(&o);
    o.method = method;
    o.n_iter = s->nIter;
    o.iter_type = (int32_t) s->iter_type;
    o.maxiter = s->maxiter;
    o.err_rel = s->err_rel;
    o.err_abs = s->err_abs;
    o.bg = s->bg;
    o.bg_auto = s->bg_auto;
    o.positivity = s->positivity;
    o.border_quality = s->borderQuality;
    o.start_condition = (int32_t) s->start_condition;
    o.metric = (int32_t) s->metric;
    o.alphamax = s->alphamax;
    o.device = s->cl_device;
    o.verbosity = s->verbosity;

    float *out = fim_malloc((size_t) M * (size_t) N * (size_t) P * sizeof(float));
    int rc = dwcu_deconvolve(im, M, N, P, psf, pM, pN, pP, &o, out);
    fim_free(psf); /* the dw_function owns the PSF (method_shb.c:191) */
    if (rc != DWCU_SUCCESS) {
        fprintf(s->log, "dwcu: %s (status %d)\n", dwcu_last_error(), rc);
        fprintf(stderr, "dwcu: %s (status %d)\n", dwcu_last_error(), rc);
        fim_free(out);
        return NULL;
    }
    s->bg = o.bg;
    if (s->verbosity > 0)
        printf("dwcu: %d iterations, job %lld x %lld x %lld, %.3f s on the GPU\n", o.iterations_done,
               (long long) o.work[0], (long long) o.work[1], (long long) o.work[2],
               o.seconds_setup + o.seconds_iterate);
    return out;
}

float *deconvolve_shb_cu(float *restrict im, const int64_t M, const int64_t N, const int64_t P,
                         float *restrict psf, const int64_t pM, const int64_t pN, const int64_t pP, dw_opts *s)
{
    return dwcu_method(im, M, N, P, psf, pM, pN, pP, s, DWCU_METHOD_SHB);
}

float *deconvolve_rl_cu(float *restrict im, const int64_t M, const int64_t N, const int64_t P,
                        float *restrict psf, const int64_t pM, const int64_t pN, const int64_t pP, dw_opts *s)
{
    return dwcu_method(im, M, N, P, psf, pM, pN, pP, s, DWCU_METHOD_RL);
}
