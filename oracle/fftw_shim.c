/* fftw_shim.c -- FFTW-API shim over oracle/cfft.c (test infrastructure only).
 *
 * Implements the functions declared in oracle/include/fftw3.h with the
 * semantics deconwolf's fft.c relies on (fft.c:206-319 plans, 383-415 and
 * 826-863 executes):
 *   - r2c 3-D: dims (n0, n1, n2) with n2 fastest; out-of-place input rows hold
 *     n2 floats, in-place (in == out) rows hold 2*(n2/2+1) floats;
 *   - c2r 3-D: unnormalised inverse, input destroyed, same row rule;
 *   - plans keep their shape and may be executed on other arrays
 *     (fftwf_execute_dft_*), as FFTW's new-array execute allows.
 */
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"
#include "cfft.h"

const char fftwf_version[] = "oracle-fftw-shim (double-precision lines over cfft)";

enum { SHIM_R2C_3D, SHIM_C2R_3D, SHIM_R2C_1D };

struct oracle_fftwf_plan_s {
    int kind;
    int n0, n1, n2;
    void *in, *out;
};

static int shim_threads = 1;

static fftwf_plan mk(int kind, int n0, int n1, int n2, void *in, void *out)
{
    fftwf_plan p = calloc(1, sizeof(*p));
    p->kind = kind;
    p->n0 = n0; p->n1 = n1; p->n2 = n2;
    p->in = in; p->out = out;
    return p;
}

fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float *in,
                                 fftwf_complex *out, unsigned flags)
{
    (void) flags;
    return mk(SHIM_R2C_3D, n0, n1, n2, in, out);
}

fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex *in,
                                 float *out, unsigned flags)
{
    (void) flags;
    return mk(SHIM_C2R_3D, n0, n1, n2, in, out);
}

fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out,
                                 unsigned flags)
{
    (void) flags;
    return mk(SHIM_R2C_1D, 1, 1, n, in, out);
}

void fftwf_execute_dft_r2c(const fftwf_plan p, float *in, fftwf_complex *out)
{
    if (p->kind == SHIM_R2C_1D) {
        cfft_r2c_1d(p->n2, in, (float *) out);
        return;
    }
    int64_t row = ((void *) in == (void *) out) ? 2 * (p->n2 / 2 + 1) : p->n2;
    cfft_r2c_3d(p->n0, p->n1, p->n2, in, row, (float *) out, shim_threads);
}

void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex *in, float *out)
{
    int64_t row = ((void *) in == (void *) out) ? 2 * (p->n2 / 2 + 1) : p->n2;
    cfft_c2r_3d(p->n0, p->n1, p->n2, (float *) in, out, row, shim_threads);
}

void fftwf_execute(const fftwf_plan p)
{
    if (p->kind == SHIM_C2R_3D)
        fftwf_execute_dft_c2r(p, (fftwf_complex *) p->in, (float *) p->out);
    else
        fftwf_execute_dft_r2c(p, (float *) p->in, (fftwf_complex *) p->out);
}

void fftwf_destroy_plan(fftwf_plan p) { free(p); }
int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int nthreads) { shim_threads = nthreads > 0 ? nthreads : 1; }
void fftwf_cleanup(void) {}
void fftwf_cleanup_threads(void) {}
int fftwf_import_wisdom_from_filename(const char *filename) { (void) filename; return 0; }
int fftwf_export_wisdom_to_filename(const char *filename) { (void) filename; return 1; }
