/* cfft.c -- CPU FFT for the oracle (test infrastructure only; see cfft.h).
 *
 * Restates the published DFT with a recursive mixed-radix Cooley-Tukey
 * decimation in time (radix 4, 2, 3 and odd primes up to 64) and Bluestein's
 * chirp-z algorithm for lengths with a larger prime factor (the exact job
 * sizes of deconwolf have factors such as 557, 191, 89 and 59).
 * Twiddles are evaluated once per plan with libm cos/sin in double.
 */
#include "cfft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define CFFT_MAXPRIME 64

struct cfft_plan {
    int64_t n;
    int nfac;
    int fac[64];
    double *tw;          /* 2n doubles: exp(-2 pi i j / n) */
    size_t work;         /* doubles of scratch needed by cfft_exec */
    /* Bluestein */
    int blue;
    int64_t L;
    cfft_plan *sub;
    double *chirp;       /* 2n doubles: exp(-pi i j^2 / n) */
    double *bfft;        /* 2L doubles: FFT_L of conj(chirp), wrapped */
};

static const double TWO_PI = 6.283185307179586476925286766559;
static const double ONE_PI = 3.141592653589793238462643383279;

static int factorize(int64_t n, int *fac, int *big)
{
    int nf = 0;
    *big = 0;
    while (n % 4 == 0) { fac[nf++] = 4; n /= 4; }
    while (n % 2 == 0) { fac[nf++] = 2; n /= 2; }
    for (int64_t p = 3; p * p <= n; p += 2) {
        while (n % p == 0) {
            if (p > CFFT_MAXPRIME) *big = 1;
            fac[nf++] = (int) (p > 0x7fffffff ? 0 : p);
            n /= p;
        }
    }
    if (n > 1) {
        if (n > CFFT_MAXPRIME) *big = 1;
        fac[nf++] = (int) (n > 0x7fffffff ? 0 : n);
    }
    return nf;
}

static int64_t next_pow2(int64_t v)
{
    int64_t L = 1;
    while (L < v) L <<= 1;
    return L;
}

cfft_plan *cfft_plan_new(int64_t n)
{
    cfft_plan *p = calloc(1, sizeof(cfft_plan));
    if (!p) return NULL;
    p->n = n;
    int big = 0;
    p->nfac = factorize(n, p->fac, &big);
    if (big) {
        p->blue = 1;
        p->L = next_pow2(2 * n - 1);
        p->sub = cfft_plan_new(p->L);
        p->chirp = malloc(sizeof(double) * 2 * (size_t) n);
        p->bfft = calloc(2 * (size_t) p->L, sizeof(double));
        for (int64_t j = 0; j < n; j++) {
            /* j^2 mod 2n keeps the angle argument small and exact */
            int64_t q = (int64_t) (((__int128) j * j) % (2 * n));
            double a = ONE_PI * (double) q / (double) n;
            p->chirp[2 * j] = cos(a);
            p->chirp[2 * j + 1] = -sin(a);
        }
        /* b_t = conj(chirp_t), placed at t and L - t */
        for (int64_t t = 0; t < n; t++) {
            p->bfft[2 * t] = p->chirp[2 * t];
            p->bfft[2 * t + 1] = -p->chirp[2 * t + 1];
            if (t > 0) {
                p->bfft[2 * (p->L - t)] = p->chirp[2 * t];
                p->bfft[2 * (p->L - t) + 1] = -p->chirp[2 * t + 1];
            }
        }
        double *w = malloc(sizeof(double) * cfft_work_size(p->sub));
        cfft_exec(p->sub, p->bfft, w, -1);
        free(w);
        p->work = 2 * (size_t) p->L + cfft_work_size(p->sub);
    } else {
        p->tw = malloc(sizeof(double) * 2 * (size_t) n);
        for (int64_t j = 0; j < n; j++) {
            double a = TWO_PI * (double) j / (double) n;
            p->tw[2 * j] = cos(a);
            p->tw[2 * j + 1] = -sin(a);
        }
        p->work = 2 * (size_t) n;
    }
    return p;
}

void cfft_plan_free(cfft_plan *p)
{
    if (!p) return;
    free(p->tw);
    free(p->chirp);
    free(p->bfft);
    cfft_plan_free(p->sub);
    free(p);
}

size_t cfft_work_size(const cfft_plan *p) { return p->work; }

/* DFT of length r on t[0..r-1] (interleaved re/im), result in o. */
static void small_dft(int r, const double *t, double *o, int sign,
                      const double *tw, int64_t N)
{
    if (r == 2) {
        o[0] = t[0] + t[2]; o[1] = t[1] + t[3];
        o[2] = t[0] - t[2]; o[3] = t[1] - t[3];
        return;
    }
    if (r == 3) {
        const double c = -0.5, s = sign * 0.86602540378443864676372317075294;
        double ar = t[2] + t[4], ai = t[3] + t[5];
        double br = t[2] - t[4], bi = t[3] - t[5];
        double mr = t[0] + c * ar, mi = t[1] + c * ai;
        o[0] = t[0] + ar; o[1] = t[1] + ai;
        /* + s*i*(b) = (-s*bi, s*br) */
        o[2] = mr - s * bi; o[3] = mi + s * br;
        o[4] = mr + s * bi; o[5] = mi - s * br;
        return;
    }
    if (r == 4) {
        double a0r = t[0] + t[4], a0i = t[1] + t[5];
        double a1r = t[0] - t[4], a1i = t[1] - t[5];
        double a2r = t[2] + t[6], a2i = t[3] + t[7];
        double a3r = t[2] - t[6], a3i = t[3] - t[7];
        /* sign*i*a3 = (-sign*a3i, sign*a3r) */
        double br = -sign * a3i, bi = sign * a3r;
        o[0] = a0r + a2r; o[1] = a0i + a2i;
        o[2] = a1r + br;  o[3] = a1i + bi;
        o[4] = a0r - a2r; o[5] = a0i - a2i;
        o[6] = a1r - br;  o[7] = a1i - bi;
        return;
    }
    /* odd prime r: pair terms r and r-q */
    int h = (r - 1) / 2;
    double sr = t[0], si = t[1];
    for (int q = 1; q < r; q++) { sr += t[2 * q]; si += t[2 * q + 1]; }
    o[0] = sr; o[1] = si;
    int64_t step = N / r;
    for (int q = 1; q <= h; q++) {
        double er = t[0], ei = t[1], fr = 0, fi = 0;
        for (int j = 1; j <= h; j++) {
            int64_t idx = ((int64_t) (j * q) % r) * step;
            double c = tw[2 * idx];
            double s = -tw[2 * idx + 1]; /* sin(2 pi jq/r) */
            double pr = t[2 * j] + t[2 * (r - j)], pi = t[2 * j + 1] + t[2 * (r - j) + 1];
            double mr = t[2 * j] - t[2 * (r - j)], mi = t[2 * j + 1] - t[2 * (r - j) + 1];
            er += c * pr; ei += c * pi;
            fr += s * mr; fi += s * mi;
        }
        /* X_q = e + sign*i*f ; X_{r-q} = e - sign*i*f */
        o[2 * q] = er - sign * fi;     o[2 * q + 1] = ei + sign * fr;
        o[2 * (r - q)] = er + sign * fi; o[2 * (r - q) + 1] = ei - sign * fr;
    }
}

static void rec(const cfft_plan *P, int64_t n, const double *in, int64_t is,
                double *out, const int *fac, int64_t twstride, int sign)
{
    double t[2 * CFFT_MAXPRIME], o[2 * CFFT_MAXPRIME];
    if (n == 1) { out[0] = in[0]; out[1] = in[1]; return; }
    int r = fac[0];
    int64_t m = n / r;
    if (m == 1) {
        for (int q = 0; q < r; q++) { t[2 * q] = in[2 * q * is]; t[2 * q + 1] = in[2 * q * is + 1]; }
        small_dft(r, t, out, sign, P->tw, P->n);
        return;
    }
    for (int q = 0; q < r; q++)
        rec(P, m, in + 2 * q * is, is * r, out + 2 * q * m, fac + 1, twstride * r, sign);
    for (int64_t k = 0; k < m; k++) {
        t[0] = out[2 * k]; t[1] = out[2 * k + 1];
        for (int q = 1; q < r; q++) {
            int64_t idx = (int64_t) q * k * twstride;
            /* the table holds exp(-i a); sign=+1 uses its conjugate */
            double wr = P->tw[2 * idx];
            double wi = (sign < 0) ? P->tw[2 * idx + 1] : -P->tw[2 * idx + 1];
            double xr = out[2 * (q * m + k)], xi = out[2 * (q * m + k) + 1];
            t[2 * q] = xr * wr - xi * wi;
            t[2 * q + 1] = xr * wi + xi * wr;
        }
        small_dft(r, t, o, sign, P->tw, P->n);
        for (int q = 0; q < r; q++) {
            out[2 * (k + q * m)] = o[2 * q];
            out[2 * (k + q * m) + 1] = o[2 * q + 1];
        }
    }
}

void cfft_exec(const cfft_plan *p, double *x, double *work, int sign)
{
    int64_t n = p->n;
    if (n == 1) return;
    if (!p->blue) {
        rec(p, n, x, 1, work, p->fac, 1, sign);
        memcpy(x, work, sizeof(double) * 2 * (size_t) n);
        return;
    }
    int64_t L = p->L;
    double *a = work;
    double *w2 = work + 2 * L;
    /* chirp for this sign: c_j = exp(sign * pi i j^2/n) */
    for (int64_t j = 0; j < n; j++) {
        double cr = p->chirp[2 * j];
        double ci = (sign < 0) ? p->chirp[2 * j + 1] : -p->chirp[2 * j + 1];
        double xr = x[2 * j], xi = x[2 * j + 1];
        a[2 * j] = xr * cr - xi * ci;
        a[2 * j + 1] = xr * ci + xi * cr;
    }
    memset(a + 2 * n, 0, sizeof(double) * 2 * (size_t) (L - n));
    cfft_exec(p->sub, a, w2, -1);
    for (int64_t k = 0; k < L; k++) {
        double br, bi;
        if (sign < 0) {
            br = p->bfft[2 * k]; bi = p->bfft[2 * k + 1];
        } else {
            int64_t kk = (L - k) % L;
            br = p->bfft[2 * kk]; bi = -p->bfft[2 * kk + 1];
        }
        double ar = a[2 * k], ai = a[2 * k + 1];
        a[2 * k] = ar * br - ai * bi;
        a[2 * k + 1] = ar * bi + ai * br;
    }
    cfft_exec(p->sub, a, w2, +1);
    double inv = 1.0 / (double) L;
    for (int64_t k = 0; k < n; k++) {
        double cr = p->chirp[2 * k];
        double ci = (sign < 0) ? p->chirp[2 * k + 1] : -p->chirp[2 * k + 1];
        double yr = a[2 * k] * inv, yi = a[2 * k + 1] * inv;
        x[2 * k] = yr * cr - yi * ci;
        x[2 * k + 1] = yr * ci + yi * cr;
    }
}

/* ---------------------------------------------------------------- 3-D */

#define CBLK 8 /* columns gathered together on the strided axes */

static int nthreads_or_default(int nt)
{
#ifdef _OPENMP
    return nt > 0 ? nt : omp_get_max_threads();
#else
    (void) nt;
    return 1;
#endif
}

/* complex transform along a strided axis of a complex float array.
 * For each of `nouter` outer positions (offset outer*ostride) and each
 * column c in [0, ncol) (offset c), transform the `len` elements at stride
 * `lstride` (all strides in complex elements). */
static void axis_pass(float *data, int64_t nouter, int64_t ostride,
                      int64_t ncol, int64_t len, int64_t lstride, int sign,
                      int nthreads)
{
    cfft_plan *p = cfft_plan_new(len);
    int64_t nblk = (ncol + CBLK - 1) / CBLK;
    int64_t ntask = nouter * nblk;
    int nt = nthreads_or_default(nthreads);
#pragma omp parallel num_threads(nt)
    {
        double *buf = malloc(sizeof(double) * 2 * (size_t) len * CBLK);
        double *work = malloc(sizeof(double) * cfft_work_size(p));
#pragma omp for schedule(static)
        for (int64_t task = 0; task < ntask; task++) {
            int64_t o = task / nblk;
            int64_t c0 = (task % nblk) * CBLK;
            int64_t nc = ncol - c0 < CBLK ? ncol - c0 : CBLK;
            float *base = data + 2 * (o * ostride + c0);
            for (int64_t l = 0; l < len; l++) {
                const float *src = base + 2 * l * lstride;
                for (int64_t c = 0; c < nc; c++) {
                    buf[2 * (c * len + l)] = src[2 * c];
                    buf[2 * (c * len + l) + 1] = src[2 * c + 1];
                }
            }
            for (int64_t c = 0; c < nc; c++)
                cfft_exec(p, buf + 2 * c * len, work, sign);
            for (int64_t l = 0; l < len; l++) {
                float *dst = base + 2 * l * lstride;
                for (int64_t c = 0; c < nc; c++) {
                    dst[2 * c] = (float) buf[2 * (c * len + l)];
                    dst[2 * c + 1] = (float) buf[2 * (c * len + l) + 1];
                }
            }
        }
        free(buf);
        free(work);
    }
    cfft_plan_free(p);
}

void cfft_r2c_3d(int64_t n0, int64_t n1, int64_t n2,
                 const float *in, int64_t in_row, float *out, int nthreads)
{
    int64_t nh = n2 / 2 + 1;
    int64_t nrow = n0 * n1;
    cfft_plan *p = cfft_plan_new(n2);
    int nt = nthreads_or_default(nthreads);
#pragma omp parallel num_threads(nt)
    {
        double *buf = malloc(sizeof(double) * 2 * (size_t) n2);
        double *work = malloc(sizeof(double) * cfft_work_size(p));
#pragma omp for schedule(static)
        for (int64_t r = 0; r < nrow; r++) {
            const float *src = in + r * in_row;
            for (int64_t j = 0; j < n2; j++) { buf[2 * j] = src[j]; buf[2 * j + 1] = 0; }
            cfft_exec(p, buf, work, -1);
            float *dst = out + 2 * r * nh;
            for (int64_t k = 0; k < nh; k++) {
                dst[2 * k] = (float) buf[2 * k];
                dst[2 * k + 1] = (float) buf[2 * k + 1];
            }
        }
        free(buf);
        free(work);
    }
    cfft_plan_free(p);
    if (n1 > 1) axis_pass(out, n0, n1 * nh, nh, n1, nh, -1, nthreads);
    if (n0 > 1) axis_pass(out, n1, nh, nh, n0, n1 * nh, -1, nthreads);
}

void cfft_c2r_3d(int64_t n0, int64_t n1, int64_t n2,
                 float *in, float *out, int64_t out_row, int nthreads)
{
    int64_t nh = n2 / 2 + 1;
    int64_t nrow = n0 * n1;
    if (n0 > 1) axis_pass(in, n1, nh, nh, n0, n1 * nh, +1, nthreads);
    if (n1 > 1) axis_pass(in, n0, n1 * nh, nh, n1, nh, +1, nthreads);
    cfft_plan *p = cfft_plan_new(n2);
    int nt = nthreads_or_default(nthreads);
#pragma omp parallel num_threads(nt)
    {
        double *buf = malloc(sizeof(double) * 2 * (size_t) n2);
        double *work = malloc(sizeof(double) * cfft_work_size(p));
#pragma omp for schedule(static)
        for (int64_t r = 0; r < nrow; r++) {
            const float *src = in + 2 * r * nh;
            for (int64_t k = 0; k < nh; k++) { buf[2 * k] = src[2 * k]; buf[2 * k + 1] = src[2 * k + 1]; }
            /* Hermitian completion; the imaginary parts of the DC and (even
             * n2) Nyquist bins only reach the discarded imaginary output */
            for (int64_t k = nh; k < n2; k++) {
                buf[2 * k] = buf[2 * (n2 - k)];
                buf[2 * k + 1] = -buf[2 * (n2 - k) + 1];
            }
            cfft_exec(p, buf, work, +1);
            float *dst = out + r * out_row;
            for (int64_t j = 0; j < n2; j++) dst[j] = (float) buf[2 * j];
        }
        free(buf);
        free(work);
    }
    cfft_plan_free(p);
}

void cfft_r2c_1d(int64_t n, const float *in, float *out)
{
    cfft_plan *p = cfft_plan_new(n);
    double *buf = malloc(sizeof(double) * 2 * (size_t) n);
    double *work = malloc(sizeof(double) * cfft_work_size(p));
    for (int64_t j = 0; j < n; j++) { buf[2 * j] = in[j]; buf[2 * j + 1] = 0; }
    cfft_exec(p, buf, work, -1);
    for (int64_t k = 0; k < n / 2 + 1; k++) { out[2 * k] = (float) buf[2 * k]; out[2 * k + 1] = (float) buf[2 * k + 1]; }
    free(buf);
    free(work);
    cfft_plan_free(p);
}
