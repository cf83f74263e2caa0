/* psf_glue.c -- TEST INFRASTRUCTURE ONLY: deconwolf's own PSF preparation,
 * for pinning dwcu_psf_prepare.
 *
 * Linked into _ref/libdwpsf.so with the reference's dw.c compiled unmodified
 * (hidden symbols, unused sections dropped by the linker) over _ref/libdwref.so
 * (fim.c, fft.c, dw_util.c).  dwpsf_prepare runs the steps dw_run applies to
 * the PSF before the method (src/dw.c:2799-2826):
 *   fim_normalize_sum1 (fim.c:900-912), psf_autocrop (dw.c:1973-1997:
 *   psf_autocrop_byImage dw.c:1764-1860, psf_autocrop_XY dw.c:1862-1971),
 *   fim_normalize_sum1 again,
 * with the options the GPU path takes (border quality, xy crop factor) and
 * the rest at dw_opts_new's defaults (dw.c:340-413; no FFT lookahead).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dw.h"
#include "fim.h"

float *psf_autocrop(float *psf, int64_t *pM, int64_t *pN, int64_t *pP, int64_t M, int64_t N, int64_t P,
                    dw_opts *s);

__attribute__((visibility("default"))) int dwpsf_prepare(const float *psf_in, int64_t pM, int64_t pN,
                                                         int64_t pP, int64_t M, int64_t N, int64_t P, int bq,
                                                         float xycropfactor, float *out, int64_t *out_dims)
{
    size_t n = (size_t) (pM * pN * pP);
    float *psf = fim_malloc(n * sizeof(float));
    if (!psf) return -1;
    memcpy(psf, psf_in, n * sizeof(float));
    dw_opts *s = dw_opts_new();
    s->borderQuality = bq;
    s->xycropfactor = xycropfactor;
    s->lookahead = 0;
    s->verbosity = 0;
    s->log = fopen("/dev/null", "w");
    FILE *so = stdout;
    stdout = fopen("/dev/null", "w"); /* psf_autocrop_byImage prints warnings */
    fim_normalize_sum1(psf, pM, pN, pP);
    psf = psf_autocrop(psf, &pM, &pN, &pP, M, N, P, s);
    fim_normalize_sum1(psf, pM, pN, pP);
    fclose(stdout);
    stdout = so;
    memcpy(out, psf, (size_t) (pM * pN * pP) * sizeof(float));
    out_dims[0] = pM;
    out_dims[1] = pN;
    out_dims[2] = pP;
    fim_free(psf);
    fclose(s->log);
    s->log = NULL;
    dw_opts_free(&s);
    return 0;
}
