/* glue_driver.c -- test driver for deconwolf_b200/glue/method_shb_cu.c.
 *
 * Builds a dw_opts the way dw_opts_new (src/dw.c:340-413) does for the
 * fields the methods read, hands fim_malloc'd copies of the image and PSF to
 * deconvolve_shb_cu / deconvolve_rl_cu through a dw_function pointer (as
 * dw_run does, src/dw.c:2841) and copies the result out.  Compiled against
 * the reference's headers by oracle/Makefile into oracle/_ref/libdwglue.so.
 */
#include <stdlib.h>
#include <string.h>
#include "dw.h"
#include "fim.h"

float *deconvolve_shb_cu(float *restrict im, const int64_t M, const int64_t N, const int64_t P,
                         float *restrict psf, const int64_t pM, const int64_t pN, const int64_t pP, dw_opts *s);
float *deconvolve_rl_cu(float *restrict im, const int64_t M, const int64_t N, const int64_t P,
                        float *restrict psf, const int64_t pM, const int64_t pN, const int64_t pP, dw_opts *s);

int glue_run(const float *im, int64_t M, int64_t N, int64_t P, const float *psf, int64_t pM, int64_t pN,
             int64_t pP, int method, int n_iter, float *out, float *bg_out)
{
    dw_opts *s = calloc(1, sizeof(dw_opts));
    s->nIter = n_iter;
    s->maxiter = 250;
    s->err_rel = 0.02f;
    s->err_abs = 1.0f;
    s->iter_type = DW_ITER_FIXED;
    s->method = method == 0 ? DW_METHOD_RL : DW_METHOD_SHB;
    s->fun = method == 0 ? deconvolve_rl_cu : deconvolve_shb_cu;
    s->borderQuality = 2;
    s->positivity = 1;
    s->bg = 1e-2f;
    s->bg_auto = 1;
    s->metric = DW_METRIC_IDIV;
    s->alphamax = 1.0f;
    s->start_condition = DW_START_FLAT;
    s->cl_device = 0;
    s->log = fopen("/dev/null", "w");
    float *imc = fim_malloc(sizeof(float) * (size_t) (M * N * P));
    memcpy(imc, im, sizeof(float) * (size_t) (M * N * P));
    float *pc = fim_malloc(sizeof(float) * (size_t) (pM * pN * pP));
    memcpy(pc, psf, sizeof(float) * (size_t) (pM * pN * pP));
    dw_function fun = s->fun;
    float *r = fun(imc, M, N, P, pc, pM, pN, pP, s); /* frees pc */
    int rc = 0;
    if (r) {
        memcpy(out, r, sizeof(float) * (size_t) (M * N * P));
        fim_free(r);
    } else {
        rc = -1;
    }
    *bg_out = s->bg;
    fim_free(imc);
    fclose(s->log);
    free(s);
    return rc;
}
