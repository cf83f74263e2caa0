/* dwo.c -- oracle: CPU restatement of deconwolf's SHB / RL iteration.
 *
 * TEST INFRASTRUCTURE ONLY (see dwo.h).  Each function cites the reference
 * source it restates (paths inside the deconwolf tree).  FFTs go through
 * oracle/cfft.c, the same code that backs the FFTW shim used to compile the
 * reference itself into oracle/_ref, so the two agree to the order of the
 * OpenMP reductions.
 */
#include "dwo.h"
#include "cfft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef int64_t i64;

static double now_s(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double) t.tv_sec + 1e-9 * (double) t.tv_nsec;
}

void dwo_opts_default(dwo_opts *s)
{
    /* dw_opts_new, src/dw.c:340-413 (the fields the GPU path honours) */
    memset(s, 0, sizeof(*s));
    s->method = 2;
    s->n_iter = 1;
    s->iter_type = 1;
    s->maxiter = 250;
    s->err_rel = 0.02f;
    s->err_abs = 1.0f;
    s->bg = 1e-2f;
    s->bg_auto = 1;
    s->positivity = 1;
    s->border_quality = 2;
    s->start_condition = 0;
    s->metric = 1;
    s->alphamax = 1.0f;
}

static int nthreads(int t)
{
#ifdef _OPENMP
    return t > 0 ? t : omp_get_max_threads();
#else
    (void) t;
    return 1;
#endif
}

static size_t nch(i64 M, i64 N, i64 P) { return (size_t) (1 + M / 2) * N * P; } /* fft.c:129-133 */

void dwo_fft_r2c(const float *in, i64 M, i64 N, i64 P, float *out, int threads)
{
    /* fft.c:401-415: fftwf_plan_dft_r2c_3d(P, N, M, ...) */
    cfft_r2c_3d(P, N, M, in, M, out, nthreads(threads));
}

void dwo_fft_c2r(float *in, i64 M, i64 N, i64 P, float *out, int threads)
{
    /* unnormalised inverse; fft.c:848-863 normalises afterwards */
    cfft_c2r_3d(P, N, M, in, out, M, nthreads(threads));
}

/* fim_argmax_max, fim.c:269-332: first (lowest linear index) maximum */
void dwo_argmax(const float *I, i64 M, i64 N, i64 P, i64 *aM, i64 *aN, i64 *aP)
{
    size_t MNP = (size_t) M * N * P, amax = 0;
    float mx = I[0];
    for (size_t k = 0; k < MNP; k++)
        if (I[k] > mx) { mx = I[k]; amax = k; }
    i64 p = (i64) (amax / ((size_t) M * N));
    i64 n = (i64) ((amax - (size_t) p * M * N) / M);
    *aP = p;
    *aN = n;
    *aM = (i64) amax - p * M * N - n * M;
}

static i64 mod_i64(i64 a, i64 b)
{
    i64 r = a % b;
    return r < 0 ? r + b : r;
}

/* fim_circshift + shift_vector_buf, fim.c:982-1057 and 1225-1242:
 * new[i] = old[(i - s) mod n] along each axis in turn. */
void dwo_circshift(float *A, i64 M, i64 N, i64 P, i64 sm, i64 sn, i64 sp)
{
    i64 bs = M > N ? M : N;
    bs = bs > P ? bs : P;
    float *buf = malloc(sizeof(float) * (size_t) bs);
    for (i64 c = 0; c < P; c++)
        for (i64 b = 0; b < N; b++) {
            float *v = A + b * M + c * M * N;
            for (i64 i = 0; i < M; i++) buf[i] = v[i];
            for (i64 i = 0; i < M; i++) v[i] = buf[mod_i64(i - sm, M)];
        }
    for (i64 c = 0; c < P; c++)
        for (i64 a = 0; a < M; a++) {
            float *v = A + a + c * M * N;
            for (i64 i = 0; i < N; i++) buf[i] = v[i * M];
            for (i64 i = 0; i < N; i++) v[i * M] = buf[mod_i64(i - sn, N)];
        }
    for (i64 b = 0; b < N; b++)
        for (i64 a = 0; a < M; a++) {
            float *v = A + a + b * M;
            for (i64 i = 0; i < P; i++) buf[i] = v[i * M * N];
            for (i64 i = 0; i < P; i++) v[i * M * N] = buf[mod_i64(i - sp, P)];
        }
    free(buf);
}

/* get_fIdiv, dw.c:1492-1524: mean over the image of g*logf(g/y) - (g - y)
 * for y > 0 and g > 0; y is read with the job strides. */
float dwo_idiv(const float *y, const float *g, i64 M, i64 N, i64 P,
               i64 wM, i64 wN, i64 wP)
{
    (void) wP;
    double I = 0;
#pragma omp parallel for reduction(+ : I)
    for (i64 c = 0; c < P; c++)
        for (i64 b = 0; b < N; b++)
            for (i64 a = 0; a < M; a++) {
                double yv = y[a + b * wM + c * wM * wN];
                double gv = g[a + b * M + c * M * N];
                if (yv > 0 && gv > 0)
                    I += gv * logf((float) (gv / yv)) - (gv - yv);
            }
    return (float) (I / (double) (M * N * P));
}

/* get_fMSE, dw.c:1461-1490 */
static float dwo_mse(const float *y, const float *g, i64 M, i64 N, i64 P, i64 wM, i64 wN)
{
    double e = 0;
    for (i64 c = 0; c < P; c++)
        for (i64 b = 0; b < N; b++)
            for (i64 a = 0; a < M; a++) {
                double d = (double) y[a + b * wM + c * wM * wN] - (double) g[a + b * M + c * M * N];
                e += d * d;
            }
    return (float) (e / (double) (M * N * P));
}

/* ------------------------------------------------------------ iterator */
/* dw_iterator_t and dw_iterator_{new,next,set_error}, dw.h:298-306,
 * dw.c:219-276 */
typedef struct {
    float error, lasterror;
    int iter, niter;
    float relerror, abserror;
    int itertype;
} dwo_it;

static void it_new(dwo_it *it, const dwo_opts *s)
{
    it->error = 1;
    it->lasterror = 1;
    it->itertype = s->iter_type;
    it->abserror = s->err_abs;
    it->relerror = s->err_rel;
    it->iter = -1;
    it->niter = (s->iter_type != 2) ? s->maxiter : s->n_iter;
}

static int it_next(dwo_it *it)
{
    it->iter++;
    if (it->itertype == 1) {
        if (it->iter < 2) it->lasterror = 2 * it->error * it->relerror;
        if (fabs(it->error - it->lasterror) / it->error < it->relerror) return -1;
    } else if (it->itertype == 0) {
        if (it->iter > 0 && it->error < it->abserror) return -1;
    }
    if (it->iter >= it->niter) return -1;
    return it->iter;
}

static void it_set(dwo_it *it, float e)
{
    it->lasterror = it->error;
    it->error = e;
}

/* ------------------------------------------------------------ helpers */

typedef struct {
    i64 M, N, P, wM, wN, wP;
    size_t wMNP;
    float norm;      /* divisor of the inverse transform */
    int threads;
    float *cbuf;     /* complex scratch, nch(w) complex */
} job_t;

/* fft_convolve_cc_f2 / fft_convolve_cc_conj_f2, fft.c:482-521: multiply the
 * spectrum by K (or conj(K)), inverse transform, divide by the job size. */
static void convolve(job_t *J, const float *K, float *F, int conj, float *out)
{
    size_t n = nch(J->wM, J->wN, J->wP);
#pragma omp parallel for
    for (size_t k = 0; k < n; k++) {
        float a = K[2 * k], ac = conj ? -K[2 * k + 1] : K[2 * k + 1];
        float b = F[2 * k], bc = F[2 * k + 1];
        F[2 * k] = a * b - ac * bc;
        F[2 * k + 1] = a * bc + b * ac;
    }
    dwo_fft_c2r(F, J->wM, J->wN, J->wP, out, J->threads);
    float norm = J->norm;
#pragma omp parallel for
    for (size_t k = 0; k < J->wMNP; k++) out[k] /= norm;
}

static float get_error(job_t *J, const float *y, const float *im, int metric)
{
    if (metric == 0) return dwo_mse(y, im, J->M, J->N, J->P, J->wM, J->wN);
    return dwo_idiv(y, im, J->M, J->N, J->P, J->wM, J->wN, J->wP);
}

/* ------------------------------------------------------------ driver */

/* gaussian_kernel, src/fim.c:2077-2106 (normalised to sum 1) */
static float *gauss_kernel(float sigma, size_t *nK)
{
    int len = (int) ceil(3.0 * sigma);
    if (len < 1) len = 1;
    int n = 2 * len + 1;
    float *K = malloc(sizeof(float) * (size_t) n);
    float mid = (n - 1) / 2;
    float s2 = pow(sigma, 2);
    float k0 = 1.0 / sigma / sqrt(2.0 * M_PI);
    double sum = 0;
    for (int kk = 0; kk < n; kk++) {
        float x = (float) kk - mid;
        K[kk] = k0 * exp(-0.5 * pow(x, 2) / s2);
        sum += K[kk];
    }
    for (int kk = 0; kk < n; kk++) K[kk] /= sum;
    *nK = (size_t) n;
    return K;
}

/* fim_conv1_vector with normalized = 1, src/fim.c:1944-2066: products in
 * float, sums in double, kernel renormalised where it leaves the line */
static void conv1_norm(float *V, size_t stride, float *W, size_t nV, const float *K, size_t nK)
{
    const size_t k2 = (nK - 1) / 2;
    size_t b = 0;
    if (nK > nV) {
        for (size_t kk = 0; kk < nV; kk++) {
            double acc0 = 0, kacc = 0;
            size_t from = k2 > kk ? 0 : kk - k2;
            size_t to = kk + k2 + 1 > nV ? nV : kk + k2 + 1;
            for (size_t ll = from; ll < to; ll++) {
                acc0 += V[ll * stride] * K[ll - kk + k2];
                kacc += K[ll - kk + k2];
            }
            W[kk] = acc0 / kacc;
        }
    } else {
        for (size_t vv = 0; vv < k2; vv++) {
            double acc0 = 0, kacc = 0;
            for (size_t kk = k2 - vv; kk < nK; kk++) {
                acc0 = acc0 + K[kk] * V[(vv - k2 + kk) * stride];
                kacc += K[kk];
            }
            W[b++] = acc0 / kacc;
        }
        for (size_t vv = k2; vv + k2 < nV; vv++) {
            double acc = 0;
            for (size_t kk = 0; kk < nK; kk++) acc = acc + K[kk] * V[((vv - k2) + kk) * stride];
            W[b++] = acc;
        }
        for (size_t vv = nV - k2; vv < nV; vv++) {
            double kacc = 0, acc0 = 0;
            for (size_t kk = 0; kk < nV - vv + k2; kk++) {
                acc0 = acc0 + K[kk] * V[(vv - k2 + kk) * stride];
                kacc += K[kk];
            }
            W[b++] = acc0 / kacc;
        }
    }
    for (size_t p = 0; p < nV; p++) V[p * stride] = W[p];
}

/* fim_gsmooth(V, M, N, P, sigma) = fim_gsmooth_aniso(V, ..., sigma, sigma),
 * src/fim.c:2240-2278: x, then y, then z with the kernel trimmed to at most
 * 2P-1 taps (z only when P > 1) */
void dwo_gsmooth(float *V, i64 M, i64 N, i64 P, float sigma)
{
    size_t nK = 0;
    float *K = gauss_kernel(sigma, &nK);
    size_t nb = (size_t) (M > N ? (M > P ? M : P) : (N > P ? N : P));
    float *W = malloc(sizeof(float) * nb);
    for (i64 pp = 0; pp < P; pp++)
        for (i64 nn = 0; nn < N; nn++) conv1_norm(V + pp * M * N + nn * M, 1, W, (size_t) M, K, nK);
    for (i64 pp = 0; pp < P; pp++)
        for (i64 mm = 0; mm < M; mm++) conv1_norm(V + pp * M * N + mm, (size_t) M, W, (size_t) N, K, nK);
    if (P > 1) {
        const float *Ka = K;
        size_t nKa = nK;
        while (nKa > (size_t) (2 * P - 1)) {
            Ka++;
            nKa -= 2;
        }
        for (i64 nn = 0; nn < N; nn++)
            for (i64 mm = 0; mm < M; mm++) conv1_norm(V + mm + M * nn, (size_t) (M * N), W, (size_t) P, Ka, nKa);
    }
    free(W);
    free(K);
}

int dwo_deconvolve(const float *im, i64 M, i64 N, i64 P,
                   const float *psf, i64 pM, i64 pN, i64 pP,
                   dwo_opts *s, float *out)
{
    double t0 = now_s();
    int shb = (s->method == 2);
    size_t MNP = (size_t) M * N * P;
    s->iterations_done = 0;

    /* method_shb.c:101-105, method_rl.c:116-119 */
    if (s->n_iter == 0) {
        memcpy(out, im, sizeof(float) * MNP);
        return 0;
    }

    /* method_shb.c:108-117: bg = max(min(im), 0.01) */
    if (s->bg_auto) {
        float mn = im[0];
        for (size_t k = 0; k < MNP; k++) if (im[k] < mn) mn = im[k];
        s->bg = mn < 1e-2f ? 1e-2f : mn;
    }

    /* method_shb.c:137-153 */
    i64 wM = M + pM - 1, wN = N + pN - 1, wP = P + pP - 1;
    if (s->border_quality == 1) { wM = M + (pM + 1) / 2; wN = N + (pN + 1) / 2; wP = P + (pP + 1) / 2; }
    if (s->border_quality == 0) { wM = M > pM ? M : pM; wN = N > pN ? N : pN; wP = P > pP ? P : pP; }
    size_t wMNP_logical = (size_t) wM * wN * wP;
    int padded = 0;
    if (s->work[0] > 0) {
        if (s->border_quality != 2 || s->work[0] < wM || s->work[1] < wN || s->work[2] < wP) return -1;
        wM = s->work[0]; wN = s->work[1]; wP = s->work[2];
        padded = 1;
    }

    job_t J;
    J.M = M; J.N = N; J.P = P; J.wM = wM; J.wN = wN; J.wP = wP;
    J.wMNP = (size_t) wM * wN * wP;
    J.threads = s->threads;
    /* ifft_inplace, fft.c:860: float MNP = (float) M*N*P (float products) */
    J.norm = (float) wM * (float) wN * (float) wP;
    if (padded) J.norm = (float) ((double) wM * (double) wN * (double) wP);
    size_t wMNP = J.wMNP;
    size_t nc = nch(wM, wN, wP);

    float *K = calloc(2 * nc, sizeof(float));
    float *C = calloc(2 * nc, sizeof(float));
    float *Z = calloc(wMNP, sizeof(float));
    if (!K || !C || !Z) return -3;

    /* OTF, method_shb.c:185-212: insert at the corner (fim_insert,
     * fim.c:585-623), move the argmax to the origin, transform. */
    for (i64 c = 0; c < pP; c++)
        for (i64 b = 0; b < pN; b++)
            for (i64 a = 0; a < pM; a++)
                Z[a + b * wM + c * wM * wN] = psf[a + b * pM + c * pM * pN];
    i64 mM, mN, mP;
    dwo_argmax(Z, wM, wN, wP, &mM, &mN, &mP);
    dwo_circshift(Z, wM, wN, wP, -mM, -mN, -mP);
    {
        float mx = Z[0];
        for (size_t k = 0; k < wMNP; k++) if (Z[k] > mx) mx = Z[k];
        if (Z[0] != mx) { free(K); free(C); free(Z); return -4; } /* method_shb.c:199-203 */
    }
    dwo_fft_r2c(Z, wM, wN, wP, K, s->threads);

    /* Bertero weights, method_shb.c:216-253 (initial_guess, dw.c:2497-2520) */
    float *W = NULL;
    if (s->border_quality > 0) {
        memset(Z, 0, sizeof(float) * wMNP);
        for (i64 c = 0; c < P; c++)
            for (i64 b = 0; b < N; b++)
                for (i64 a = 0; a < M; a++) Z[a + wM * b + wM * wN * c] = 1;
        dwo_fft_r2c(Z, wM, wN, wP, C, s->threads);
        W = malloc(sizeof(float) * wMNP);
        convolve(&J, K, C, 1, W);
        const float sigma = 0.01f;
#pragma omp parallel for
        for (size_t k = 0; k < wMNP; k++)
            W[k] = (W[k] > sigma) ? (float) (1.0 / W[k]) : 0.0f;
    }

    /* fim_sum, fim.c:368-378 */
    double sumd = 0;
    for (size_t k = 0; k < MNP; k++) sumd += (double) im[k];
    float sumg = (float) sumd;

    float *x = malloc(sizeof(float) * wMNP);
    float *xp = malloc(sizeof(float) * wMNP);
    float *y = Z; /* reuse */
    float *xn = shb ? malloc(sizeof(float) * wMNP) : NULL;
    if (s->start_condition == 0) {
        /* method_shb.c:264-268: sumg / wMNP with the job's voxel count */
        float v = sumg / (float) wMNP_logical;
        for (size_t k = 0; k < wMNP; k++) x[k] = v;
    } else {
        /* IDENTITY: the image; LP (method_shb.c:278-285): the image smoothed
         * by fim_gsmooth with sigma 8; both inserted at the corner */
        const float *src = im;
        float *lp = NULL;
        if (s->start_condition == 1) {
            lp = malloc(sizeof(float) * MNP);
            memcpy(lp, im, sizeof(float) * MNP);
            dwo_gsmooth(lp, M, N, P, 8);
            src = lp;
        }
        memset(x, 0, sizeof(float) * wMNP);
        for (i64 c = 0; c < P; c++)
            for (i64 b = 0; b < N; b++)
                for (i64 a = 0; a < M; a++) x[a + wM * b + wM * wN * c] = src[a + M * b + M * N * c];
        free(lp);
    }
    memcpy(xp, x, sizeof(float) * wMNP);

    double t1 = now_s();
    s->setup_seconds = t1 - t0;

    dwo_it it;
    it_new(&it, s);
    while (it_next(&it) >= 0) {
        float err;
        if (shb) {
            /* method_shb.c:325-339: p overwrites xp */
            double alpha = ((float) it.iter - 1.0) / ((float) it.iter + 2.0);
            if (alpha < 0) alpha = 0;
            if (alpha > s->alphamax) alpha = s->alphamax;
            float *p = xp;
            float bg = s->bg;
#pragma omp parallel for
            for (size_t k = 0; k < wMNP; k++) {
                p[k] = x[k] + alpha * (x[k] - xp[k]);
                if (p[k] < bg) p[k] = bg;
            }
            /* iter_shb, method_shb.c:10-74 */
            dwo_fft_r2c(p, wM, wN, wP, C, s->threads);
            convolve(&J, K, C, 0, y);
            err = get_error(&J, y, im, s->metric);
            const double mindiv = 1e-6;
#pragma omp parallel for
            for (i64 cc = 0; cc < wP; cc++)
                for (i64 bb = 0; bb < wN; bb++)
                    for (i64 aa = 0; aa < wM; aa++) {
                        size_t yi = aa + bb * wM + cc * wM * wN;
                        if (aa < M && bb < N && cc < P) {
                            if (fabs(y[yi]) < mindiv) y[yi] = copysign(mindiv, y[yi]);
                            y[yi] = im[aa + bb * M + cc * M * N] / y[yi];
                        } else {
                            y[yi] = 0;
                        }
                    }
            dwo_fft_r2c(y, wM, wN, wP, C, s->threads);
            /* the new estimate goes into xp's buffer (p is consumed) */
            convolve(&J, K, C, 1, xn);
#pragma omp parallel for
            for (size_t k = 0; k < wMNP; k++)
                xn[k] *= W ? p[k] * W[k] : p[k];
            { float *t = xp; xp = xn; xn = t; }
            it_set(&it, err);
            float *t = x; x = xp; xp = t; /* method_shb.c:358-363 */
            if (s->positivity) {
#pragma omp parallel for
                for (size_t k = 0; k < wMNP; k++) if (x[k] < bg) x[k] = bg;
            }
        } else {
            /* iter_rl, method_rl.c:28-102; f = xp is the current guess */
            float *f = xp;
            dwo_fft_r2c(f, wM, wN, wP, C, s->threads);
            convolve(&J, K, C, 0, y);
            err = get_error(&J, y, im, s->metric);
            float bg = s->bg;
#pragma omp parallel for
            for (i64 cc = 0; cc < wP; cc++)
                for (i64 bb = 0; bb < wN; bb++)
                    for (i64 aa = 0; aa < wM; aa++) {
                        size_t yi = aa + bb * wM + cc * wM * wN;
                        if (aa < M && bb < N && cc < P) {
                            y[yi] = (y[yi] > 0) ? im[aa + bb * M + cc * M * N] / y[yi] : bg;
                        } else {
                            y[yi] = 1e-6f;
                        }
                    }
            dwo_fft_r2c(y, wM, wN, wP, C, s->threads);
            convolve(&J, K, C, 1, x);
#pragma omp parallel for
            for (size_t k = 0; k < wMNP; k++)
                x[k] *= W ? f[k] * W[k] : f[k];
            it_set(&it, err);
            /* method_rl.c:353-372: xp = x, clamp at bg when bg > 0 */
            float *t = xp; xp = x; x = t;
            if (bg > 0) {
#pragma omp parallel for
                for (size_t k = 0; k < wMNP; k++) if (xp[k] < bg) xp[k] = bg;
            }
        }
        if (s->error_trace && it.iter < s->trace_capacity) s->error_trace[it.iter] = err;
        s->iterations_done = it.iter + 1;
    }
    s->loop_seconds = now_s() - t1;

    /* SHB returns the iterate before the last update (method_shb.c:385-395);
     * RL returns the newest one (method_rl.c:393).  After the loop above,
     * SHB's newest is x and its predecessor xp; RL's newest is xp. */
    const float *res = xp;
    if (shb && s->iterations_done == 0) res = x;
    for (i64 c = 0; c < P; c++)
        for (i64 b = 0; b < N; b++)
            memcpy(out + b * M + c * M * N, res + b * wM + c * wM * wN, sizeof(float) * M);

    free(K); free(C); free(Z); free(W); free(x); free(xp); free(xn);
    return 0;
}

/* ================================================ PSF preparation, tiling */

/* fim_normalize_sum1, src/fim.c:900-912 (serial double sum) */
static void normalize_sum1(float *p, size_t n)
{
    double s = 0;
    for (size_t k = 0; k < n; k++) s += p[k];
    for (size_t k = 0; k < n; k++) p[k] = (float) (p[k] / s);
}

/* fim_get_cuboid, src/fim.c:659-693, into a new buffer */
static float *cuboid(const float *A, i64 M, i64 N, i64 m0, i64 m1, i64 n0, i64 n1, i64 p0, i64 p1)
{
    i64 m = m1 - m0 + 1, n = n1 - n0 + 1, p = p1 - p0 + 1;
    float *C = malloc(sizeof(float) * (size_t) (m * n * p));
    for (i64 cc = p0; cc <= p1; cc++)
        for (i64 bb = n0; bb <= n1; bb++)
            for (i64 aa = m0; aa <= m1; aa++)
                C[(aa - m0) + (bb - n0) * m + (cc - p0) * m * n] = A[aa + bb * M + cc * M * N];
    return C;
}

/* psf_autocrop, src/dw.c:1973-1997: psf_autocrop_byImage (dw.c:1764-1860)
 * and, for bq > 0 and xycropfactor > 0, psf_autocrop_XY without the FFT
 * lookahead (dw.c:1862-1971).  Takes ownership of psf (malloc'd). */
float *dwo_psf_autocrop(float *psf, i64 *pM, i64 *pN, i64 *pP, i64 M, i64 N, i64 P, int bq,
                        float xycropfactor)
{
    i64 m = *pM, n = *pN, p = *pP;
    i64 mopt = (M - 1) * 2 + 1, nopt = (N - 1) * 2 + 1, popt = (P - 1) * 2 + 1;
    if (bq == 0) { mopt = M; nopt = N; popt = P; }
    if (p < popt) return psf; /* the reference warns and returns before the XY crop */
    if (m > mopt || n > nopt || p > popt) {
        i64 m0 = 0, m1 = m - 1, n0 = 0, n1 = n - 1, p0 = 0, p1 = p - 1;
        if (m > mopt) { m0 = (m - mopt) / 2; m1 = m1 - (m - mopt) / 2; }
        if (n > nopt) { n0 = (n - nopt) / 2; n1 = n1 - (n - nopt) / 2; }
        if (p > popt) { p0 = (p - popt) / 2; p1 = p1 - (p - popt) / 2; }
        float *c = cuboid(psf, m, n, m0, m1, n0, n1, p0, p1);
        free(psf);
        psf = c;
        *pM = m = m1 - m0 + 1;
        *pN = n = n1 - n0 + 1;
        *pP = p = p1 - p0 + 1;
    }
    if (bq <= 0 || xycropfactor <= 0) return psf;
    float maxsum = 0;
    for (i64 xx = 0; xx < m; xx++) {
        float sum = 0;
        for (i64 yy = 0; yy < n; yy++)
            for (i64 zz = 0; zz < p; zz++) sum += psf[xx + yy * m + zz * m * n];
        if (sum > maxsum) maxsum = sum;
    }
    i64 first = -1;
    float sum = 0;
    while (sum < xycropfactor * maxsum && first + 1 < m) {
        first++;
        sum = 0;
        for (i64 yy = 0; yy < n; yy++)
            for (i64 zz = 0; zz < p; zz++) sum += psf[first + yy * m + zz * m * n];
    }
    if (first < 1 || m - 2 * first < 1 || n - 2 * first < 1) return psf;
    float *c = cuboid(psf, m, n, first, m - first - 1, first, n - first - 1, 0, p - 1);
    free(psf);
    *pM = m - 2 * first;
    *pN = n - 2 * first;
    return c;
}

int dwo_psf_prepare(const float *psf, i64 pM, i64 pN, i64 pP, i64 M, i64 N, i64 P, int bq,
                    float xycropfactor, float *out, i64 out_dims[3])
{
    float *p = malloc(sizeof(float) * (size_t) (pM * pN * pP));
    memcpy(p, psf, sizeof(float) * (size_t) (pM * pN * pP));
    normalize_sum1(p, (size_t) (pM * pN * pP));                 /* dw.c:2799 */
    p = dwo_psf_autocrop(p, &pM, &pN, &pP, M, N, P, bq, xycropfactor);
    normalize_sum1(p, (size_t) (pM * pN * pP));                 /* dw.c:2826 */
    memcpy(out, p, sizeof(float) * (size_t) (pM * pN * pP));
    free(p);
    out_dims[0] = pM; out_dims[1] = pN; out_dims[2] = pP;
    return 0;
}

/* tiling_getDivision, src/tiling.c:22-58 (float section width) */
static i64 division(i64 L, i64 m, i64 *divs /* 2 * ceil(L/m) */)
{
    float ns = (float) ceil((double) L / (double) m);
    float width = (float) L / ns;
    i64 n = (i64) ns;
    divs[0] = 0;
    divs[2 * n - 1] = L - 1;
    for (i64 dd = 1; dd < n; dd++) {
        divs[dd * 2 - 1] = (i64) ceilf(width * (float) dd) - 1;
        divs[dd * 2] = divs[dd * 2 - 1] + 1;
    }
    return n;
}

/* tiling_create, src/tiling.c:70-130.  Each tile is 18 int64: size[3],
 * pos[6], xpos[6], xsize[3].  Returns the tile count (tiles may be NULL). */
int dwo_tiling_create(i64 M, i64 N, i64 P, i64 max_size, i64 overlap, i64 *tiles, int capacity)
{
    i64 nM0 = (i64) ceil((double) M / (double) max_size), nN0 = (i64) ceil((double) N / (double) max_size);
    i64 *dM = calloc((size_t) (2 * nM0), sizeof(i64)), *dN = calloc((size_t) (2 * nN0), sizeof(i64));
    i64 nM = division(M, max_size, dM), nN = division(N, max_size, dN);
    int nt = (int) (nM * nN);
    if (tiles && capacity >= nt) {
        int b = 0;
        for (i64 mm = 0; mm < nM; mm++)
            for (i64 nn = 0; nn < nN; nn++, b++) {
                i64 *t = tiles + 18 * b, *size = t, *pos = t + 3, *xpos = t + 9, *xsize = t + 15;
                size[0] = dM[mm * 2 + 1] - dM[mm * 2] + 1;
                size[1] = dN[nn * 2 + 1] - dN[nn * 2] + 1;
                size[2] = P;
                pos[0] = dM[mm * 2]; pos[1] = dM[mm * 2 + 1];
                pos[2] = dN[nn * 2]; pos[3] = dN[nn * 2 + 1];
                pos[4] = 0; pos[5] = P - 1;
                xpos[0] = pos[0] - overlap > 0 ? pos[0] - overlap : 0;
                xpos[1] = pos[1] + overlap < M - 1 ? pos[1] + overlap : M - 1;
                xpos[2] = pos[2] - overlap > 0 ? pos[2] - overlap : 0;
                xpos[3] = pos[3] + overlap < N - 1 ? pos[3] + overlap : N - 1;
                xpos[4] = pos[4]; xpos[5] = pos[5];
                xsize[0] = xpos[1] - xpos[0] + 1;
                xsize[1] = xpos[3] - xpos[2] + 1;
                xsize[2] = xpos[5] - xpos[4] + 1;
            }
    }
    free(dM);
    free(dN);
    return nt;
}

/* getWeight1d, src/tiling.c:169-197 */
static float weight1d(float a, float b, float c, float d, i64 x)
{
    if (x < a || x > d) return 0;
    if (x >= b && x <= c) return 1;
    if (x >= a && x <= b) return (x - a + 1) / (b - a + 1);
    if (x >= c && x <= d) return 1 - (x - c) / (d - c + 1);
    return -1;
}

/* tile_getWeight, src/tiling.c:199-216 */
float dwo_tile_weight(const i64 *t, i64 m, i64 n)
{
    const i64 *pos = t + 3, *xpos = t + 9;
    float wm = weight1d(xpos[0], pos[0], pos[1], xpos[1], m);
    float wn = weight1d(xpos[2], pos[2], pos[3], xpos[3], n);
    return fminf(wm, wn);
}

/* deconvolve_tiles, src/dw.c:2001-2229, in memory: tiles by tiling_get_tile
 * (tiling.c:318-351), per-tile PSF normalise / autocrop / normalise
 * (dw.c:2124-2130), +offset, the method, -offset and projection
 * (dw.c:2132-2145), blended with tiling_put_tile (tiling.c:412-439).
 * s->iterations_done receives the last tile's count.  Returns 0, or a
 * negative code (one tile only: -3). */
int dwo_deconvolve_tiled(const float *im, i64 M, i64 N, i64 P, const float *psf, i64 pM, i64 pN, i64 pP,
                         i64 tile_size, i64 overlap, float offset, float xycropfactor, dwo_opts *s, float *out)
{
    int nt = dwo_tiling_create(M, N, P, tile_size, overlap, NULL, 0);
    if (nt < 2) return -3;
    i64 *tiles = malloc(sizeof(i64) * 18 * (size_t) nt);
    dwo_tiling_create(M, N, P, tile_size, overlap, tiles, nt);
    memset(out, 0, sizeof(float) * (size_t) (M * N * P));
    int rc = 0;
    for (int tt = 0; tt < nt && rc == 0; tt++) {
        const i64 *t = tiles + 18 * tt, *xpos = t + 9, *xsize = t + 15;
        i64 m = xsize[0], n = xsize[1], p = xsize[2];
        size_t tv = (size_t) (m * n * p);
        float *tile = malloc(sizeof(float) * tv);
        for (i64 cc = 0; cc < p; cc++)
            for (i64 bb = 0; bb < n; bb++)
                for (i64 aa = 0; aa < m; aa++)
                    tile[aa + bb * m + cc * m * n] = im[(aa + xpos[0]) + (bb + xpos[2]) * M + (cc + xpos[4]) * M * N];
        i64 a = pM, b = pN, c = pP;
        float *tp = malloc(sizeof(float) * (size_t) (a * b * c));
        memcpy(tp, psf, sizeof(float) * (size_t) (a * b * c));
        normalize_sum1(tp, (size_t) (a * b * c));
        tp = dwo_psf_autocrop(tp, &a, &b, &c, m, n, p, s->border_quality, xycropfactor);
        normalize_sum1(tp, (size_t) (a * b * c));
        if (offset > 0)
            for (size_t k = 0; k < tv; k++) tile[k] += offset;
        float *res = malloc(sizeof(float) * tv);
        dwo_opts so = *s;
        so.error_trace = NULL;
        so.trace_capacity = 0;
        rc = dwo_deconvolve(tile, m, n, p, tp, a, b, c, &so, res);
        s->iterations_done = so.iterations_done;
        if (rc == 0) {
            if (offset > 0)
                for (size_t k = 0; k < tv; k++) {
                    res[k] += -offset;
                    if (res[k] < 0) res[k] = 0;
                }
            for (i64 cc = xpos[4]; cc <= xpos[5]; cc++)
                for (i64 bb = xpos[2]; bb <= xpos[3]; bb++)
                    for (i64 aa = xpos[0]; aa <= xpos[1]; aa++) {
                        float w = dwo_tile_weight(t, aa, bb);
                        float ws = 0;
                        for (int q = 0; q < nt; q++) ws += dwo_tile_weight(tiles + 18 * q, aa, bb);
                        w /= ws;
                        out[aa + bb * M + cc * M * N] += w * res[(aa - xpos[0]) + (bb - xpos[2]) * m + (cc - xpos[4]) * m * n];
                    }
        }
        free(res);
        free(tp);
        free(tile);
    }
    free(tiles);
    return rc;
}
