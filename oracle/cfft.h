/* cfft.h -- CPU FFT used by the oracle (test infrastructure only).
 *
 * This is NOT part of the product path.  It backs
 *   - the C restatement of deconwolf's SHB/RL iteration (oracle/dwo.c), and
 *   - the FFTW-API shim (oracle/fftw_shim.c) against which the reference's own
 *     method_shb.c / method_rl.c / fft.c / fim.c are compiled into oracle/_ref.
 *
 * The reference calls FFTW 3 (single precision, version not pinned by the
 * reference: CMakeLists.txt:236-240 only does find_package(FFTW)).  FFTW is
 * not present here, so this file restates the published discrete Fourier
 * transform: X[k] = sum_n x[n] exp(sign * 2 pi i n k / N), unnormalised, with
 * FFTW's multi-dimensional real layout (last dimension fastest, r2c keeps
 * N/2+1 outputs along it).  Arithmetic inside a 1-D line is double precision;
 * lines are stored back as float after each axis, as a float FFT stores its
 * intermediate axis results.
 */
#ifndef ORACLE_CFFT_H
#define ORACLE_CFFT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cfft_plan cfft_plan;

/* 1-D complex plan of length n (any n >= 1). */
cfft_plan *cfft_plan_new(int64_t n);
void cfft_plan_free(cfft_plan *p);
/* In-place transform of n interleaved doubles pairs (re, im).
 * sign = -1 forward, +1 backward.  work must hold cfft_work_size(p) doubles. */
void cfft_exec(const cfft_plan *p, double *x, double *work, int sign);
size_t cfft_work_size(const cfft_plan *p);

/* 3-D real transforms on float arrays, dims (n0 slowest, n2 fastest) exactly
 * as fftwf_plan_dft_r2c_3d(n0, n1, n2, ...).
 * r2c: `in` holds real rows of `in_row` floats (n2, or 2*(n2/2+1) in place),
 *      `out` receives (n2/2+1) complex per row.  in == out is allowed.
 * c2r: `in` (complex, destroyed) -> `out` real rows of `out_row` floats. */
void cfft_r2c_3d(int64_t n0, int64_t n1, int64_t n2,
                 const float *in, int64_t in_row, float *out, int nthreads);
void cfft_c2r_3d(int64_t n0, int64_t n1, int64_t n2,
                 float *in, float *out, int64_t out_row, int nthreads);

/* 1-D real-to-complex, for fftwf_plan_dft_r2c_1d. */
void cfft_r2c_1d(int64_t n, const float *in, float *out);

#ifdef __cplusplus
}
#endif
#endif
