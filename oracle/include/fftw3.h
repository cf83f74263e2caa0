/* fftw3.h -- FFTW-API shim for the oracle build (test infrastructure only).
 *
 * deconwolf's fft.c, fim.c, dw.h and tiling.h include <fftw3.h> and use the
 * single-precision FFTW 3 API.  FFTW is not installed here, so this header
 * declares exactly the subset those files use; oracle/fftw_shim.c implements
 * it on top of oracle/cfft.c.  Names, argument order and flag values follow
 * the public FFTW 3 interface so that the reference sources compile
 * unmodified.  Planner flags are accepted and ignored: every plan is
 * "found", so FFTW_WISDOM_ONLY never returns NULL and no wisdom file is
 * ever written.
 */
#ifndef ORACLE_FFTW3_SHIM_H
#define ORACLE_FFTW3_SHIM_H

#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct oracle_fftwf_plan_s *fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_CONSERVE_MEMORY (1U << 2)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_WISDOM_ONLY (1U << 21)

extern const char fftwf_version[];

fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float *in,
                                 fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex *in,
                                 float *out, unsigned flags);
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out,
                                 unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_execute_dft_r2c(const fftwf_plan p, float *in, fftwf_complex *out);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex *in, float *out);
void fftwf_destroy_plan(fftwf_plan p);
int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int nthreads);
void fftwf_cleanup(void);
void fftwf_cleanup_threads(void);
int fftwf_import_wisdom_from_filename(const char *filename);
int fftwf_export_wisdom_to_filename(const char *filename);

#ifdef __cplusplus
}
#endif
#endif
