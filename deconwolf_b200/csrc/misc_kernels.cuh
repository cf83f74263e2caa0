// misc_kernels.cuh -- setup / bookkeeping kernels of a deconvolution job.
//
// All reductions run in a fixed order (fixed partition of the data over
// blocks, fixed order inside a block, one finishing block), so every result
// is bitwise reproducible from run to run and independent of scheduling.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "passes.cuh"

namespace dwcu {

constexpr int kRedThreads = 256;

struct StatsPartial {
    double sum;
    float mn;
    int nonfinite;
};

// Per-block min / double sum / non-finite count over the image rows
// [b*rpb, (b+1)*rpb) (fim_min fim.c:398-408, fim_sum fim.c:368-378).
__global__ void __launch_bounds__(kRedThreads)
k_stats_partial(const float *__restrict__ g, long long GP, int M, long long nrows, long long rpb,
                StatsPartial *__restrict__ part)
{
    __shared__ double ssum[kRedThreads];
    __shared__ float smin[kRedThreads];
    __shared__ int snf[kRedThreads];
    double s = 0.0;
    float mn = INFINITY;
    int nf = 0;
    const long long r0 = (long long) blockIdx.x * rpb;
    const long long r1 = min(nrows, r0 + rpb);
    for (long long r = r0; r < r1; ++r) {
        const float *row = g + r * GP;
        for (int c = threadIdx.x; c < M; c += kRedThreads) {
            float v = row[c];
            if (!isfinite(v)) nf++;
            s += (double) v;
            mn = fminf(mn, v);
        }
    }
    ssum[threadIdx.x] = s;
    smin[threadIdx.x] = mn;
    snf[threadIdx.x] = nf;
    __syncthreads();
    for (int o = kRedThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            ssum[threadIdx.x] += ssum[threadIdx.x + o];
            smin[threadIdx.x] = fminf(smin[threadIdx.x], smin[threadIdx.x + o]);
            snf[threadIdx.x] += snf[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = StatsPartial{ssum[0], smin[0], snf[0]};
}

// Finish the statistics: bg (method_shb.c:108-117), start value
// sumg / wMNP (method_shb.c:255-268, with the job's logical voxel count).
__global__ void __launch_bounds__(kRedThreads)
k_stats_final(const StatsPartial *__restrict__ part, int nb, JobScalars *sc, int bg_auto, float bg_user,
              unsigned long long wmnp_logical)
{
    __shared__ double ssum[kRedThreads];
    __shared__ float smin[kRedThreads];
    __shared__ int snf[kRedThreads];
    double s = 0.0;
    float mn = INFINITY;
    int nf = 0;
    for (int i = threadIdx.x; i < nb; i += kRedThreads) {
        s += part[i].sum;
        mn = fminf(mn, part[i].mn);
        nf += part[i].nonfinite;
    }
    ssum[threadIdx.x] = s;
    smin[threadIdx.x] = mn;
    snf[threadIdx.x] = nf;
    __syncthreads();
    for (int o = kRedThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            ssum[threadIdx.x] += ssum[threadIdx.x + o];
            smin[threadIdx.x] = fminf(smin[threadIdx.x], smin[threadIdx.x + o]);
            snf[threadIdx.x] += snf[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        float gmin = smin[0];
        sc->gmin = gmin;
        sc->sumg = ssum[0];
        sc->bg = bg_auto ? (gmin < 1e-2f ? 1e-2f : gmin) : bg_user;
        const float sumg = (float) ssum[0];
        sc->x0 = sumg / (float) wmnp_logical;
        if (snf[0]) sc->flags |= 1;
    }
}

struct ArgmaxPartial {
    float v;
    long long i;
};

// first maximum (lowest linear index), fim_argmax_max fim.c:269-332
__device__ __forceinline__ void amax_merge(float &v, long long &i, float v2, long long i2)
{
    if (v2 > v || (v2 == v && i2 < i)) {
        v = v2;
        i = i2;
    }
}

__global__ void __launch_bounds__(kRedThreads)
k_argmax_partial(const float *__restrict__ a, long long n, long long per_block, ArgmaxPartial *part, int *flags)
{
    __shared__ float sv[kRedThreads];
    __shared__ long long si[kRedThreads];
    float v = -INFINITY;
    long long idx = LLONG_MAX;
    const long long b0 = (long long) blockIdx.x * per_block;
    const long long b1 = min(n, b0 + per_block);
    int nf = 0;
    for (long long k = b0 + threadIdx.x; k < b1; k += kRedThreads) {
        float x = a[k];
        if (!isfinite(x)) nf = 1;
        amax_merge(v, idx, x, k);
    }
    if (nf) atomicOr(flags, 2);
    sv[threadIdx.x] = v;
    si[threadIdx.x] = idx;
    __syncthreads();
    for (int o = kRedThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            float v2 = sv[threadIdx.x + o];
            long long i2 = si[threadIdx.x + o];
            float v1 = sv[threadIdx.x];
            long long i1 = si[threadIdx.x];
            amax_merge(v1, i1, v2, i2);
            sv[threadIdx.x] = v1;
            si[threadIdx.x] = i1;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = ArgmaxPartial{sv[0], si[0]};
}

__global__ void k_argmax_final(const ArgmaxPartial *part, int nb, long long *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float v = -INFINITY;
    long long i = LLONG_MAX;
    for (int b = 0; b < nb; ++b) amax_merge(v, i, part[b].v, part[b].i);
    *out = i;
}

// Place the PSF into a zeroed X x Y x Z volume so that its first maximum
// lands at the origin (fim_insert fim.c:585-623 followed by fim_circshift
// fim.c:982-1057 by minus the argmax), scaled by `scale` (the inverse
// transform normalisation 1/(X*Y*Z) is folded into the OTF here).
__global__ void k_psf_embed(const float *__restrict__ psf, int pM, int pN, int pP, const long long *amax,
                            float *__restrict__ dst, int X, int Y, int Z, int XP, float scale)
{
    const long long n = (long long) pM * pN * pP;
    const long long am = *amax;
    const int ac = (int) (am / ((long long) pM * pN));
    const int ab = (int) ((am - (long long) ac * pM * pN) / pM);
    const int aa = (int) (am - (long long) ac * pM * pN - (long long) ab * pM);
    for (long long k = blockIdx.x * (long long) blockDim.x + threadIdx.x; k < n;
         k += (long long) gridDim.x * blockDim.x) {
        const int c = (int) (k / ((long long) pM * pN));
        const int b = (int) ((k - (long long) c * pM * pN) / pM);
        const int a = (int) (k - (long long) c * pM * pN - (long long) b * pM);
        int x = (a - aa) % X; if (x < 0) x += X;
        int y = (b - ab) % Y; if (y < 0) y += Y;
        int z = (c - ac) % Z; if (z < 0) z += Z;
        dst[((long long) z * Y + y) * XP + x] = psf[k] * scale;
    }
}

__global__ void k_fill_scalar(float *__restrict__ x, long long n, const JobScalars *sc)
{
    const float v = sc->x0;
    for (long long k = blockIdx.x * (long long) blockDim.x + threadIdx.x; k < n;
         k += (long long) gridDim.x * blockDim.x)
        x[k] = v;
}

// image into the corner of a zeroed real volume (start_condition IDENTITY)
__global__ void k_embed_image(const float *__restrict__ g, long long GP, int M, int N, int P,
                              float *__restrict__ x, int X, int Y)
{
    const long long n = (long long) M * N * P;
    for (long long k = blockIdx.x * (long long) blockDim.x + threadIdx.x; k < n;
         k += (long long) gridDim.x * blockDim.x) {
        const int c = (int) (k / ((long long) M * N));
        const int b = (int) ((k - (long long) c * M * N) / M);
        const int a = (int) (k - (long long) c * M * N - (long long) b * M);
        x[((long long) c * Y + b) * X + a] = g[((long long) c * N + b) * GP + a];
    }
}

// One axis of fim_gsmooth (fim.c:2240-2278): each line convolved with the
// taps as fim_conv1_vector does it with normalized = 1 (fim.c:1944-2066):
// float products summed in double in tap order, the kernel renormalised by
// the sum of the taps that fall inside the line, one rounding to float.
// in and out are M x N x P, x fastest; axis 0, 1, 2 = x, y, z.
struct GaussTaps {
    float k[64];
    int n;
};
__global__ void k_gsmooth_axis(const float *__restrict__ in, float *__restrict__ out, int M, int N, int P, int axis,
                               GaussTaps K)
{
    const long long total = (long long) M * N * P;
    const int nV = axis == 0 ? M : axis == 1 ? N : P;
    const long long stride = axis == 0 ? 1 : axis == 1 ? (long long) M : (long long) M * N;
    const int nK = K.n, k2 = (nK - 1) / 2;
    for (long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < total;
         e += (long long) gridDim.x * blockDim.x) {
        const int a = (int) (e % M);
        const int b = (int) ((e / M) % N);
        const int c = (int) (e / ((long long) M * N));
        const int v = axis == 0 ? a : axis == 1 ? b : c;
        const float *line = in + (e - (long long) v * stride);  // element 0 of this line
        double acc = 0.0, kacc = 0.0;
        float r;
        if (nK > nV) {
            const int from = v > k2 ? v - k2 : 0;
            const int to = v + k2 + 1 > nV ? nV : v + k2 + 1;
            for (int l = from; l < to; ++l) {
                acc += (double) __fmul_rn(line[l * stride], K.k[l - v + k2]);
                kacc += (double) K.k[l - v + k2];
            }
            r = (float) (acc / kacc);
        } else if (v < k2) {
            for (int kk = k2 - v; kk < nK; ++kk) {
                acc += (double) __fmul_rn(K.k[kk], line[(v - k2 + kk) * stride]);
                kacc += (double) K.k[kk];
            }
            r = (float) (acc / kacc);
        } else if (v + k2 < nV) {
            for (int kk = 0; kk < nK; ++kk) acc += (double) __fmul_rn(K.k[kk], line[(v - k2 + kk) * stride]);
            r = (float) acc;
        } else {
            for (int kk = 0; kk < nV - v + k2; ++kk) {
                acc += (double) __fmul_rn(K.k[kk], line[(v - k2 + kk) * stride]);
                kacc += (double) K.k[kk];
            }
            r = (float) (acc / kacc);
        }
        out[e] = r;
    }
}

// Periodic y and/or z (bq 0/1 axes transformed at a larger length): after a
// forward x pass, every spectrum row (y, z) outside [0, wN) x [0, wP) takes
// a copy of the row it wraps to -- [w, w+h) from [0, h), [len-h, len) from
// [w-h, w) -- and the rows in between are cleared.  One thread per 4-wide
// kx block of a row.
__global__ void k_wrap_rows(float2 *__restrict__ S, int Y, int Z, int nkb, int wN, int hy, int wrapy, int wP, int hz,
                            int wrapz)
{
    const long long n = (long long) Z * nkb * Y;
    for (long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < n;
         e += (long long) gridDim.x * blockDim.x) {
        const int y = (int) (e % Y);
        const long long zk = e / Y;
        const int kb = (int) (zk % nkb);
        const int z = (int) (zk / nkb);
        const bool yin = !wrapy || y < wN, zin = !wrapz || z < wP;
        if (yin && zin) continue;
        auto src = [](int v, int w, int h, int len) { return v < w ? v : v < w + h ? v - w : v >= len - h ? v - len + w : -1; };
        const int ys = wrapy ? src(y, wN, hy, Y) : y;
        const int zs = wrapz ? src(z, wP, hz, Z) : z;
        float2 *dst = S + (((long long) z * nkb + kb) * Y + y) * KB;
        if (ys < 0 || zs < 0) {
#pragma unroll
            for (int i = 0; i < KB; ++i) dst[i] = make_float2(0.f, 0.f);
        } else {
            const float2 *from = S + (((long long) zs * nkb + kb) * Y + ys) * KB;
#pragma unroll
            for (int i = 0; i < KB; ++i) dst[i] = from[i];
        }
    }
}

// fim_subregion (fim.c:695-718): the image-sized corner of a job volume
__global__ void k_crop(const float *__restrict__ x, int X, int Y, int M, int N, int P, float *__restrict__ out)
{
    const long long n = (long long) M * N * P;
    for (long long k = blockIdx.x * (long long) blockDim.x + threadIdx.x; k < n;
         k += (long long) gridDim.x * blockDim.x) {
        const int c = (int) (k / ((long long) M * N));
        const int b = (int) ((k - (long long) c * M * N) / M);
        const int a = (int) (k - (long long) c * M * N - (long long) b * M);
        out[k] = x[((long long) c * Y + b) * X + a];
    }
}

// compact half-spectrum (kx fastest, H = X/2+1 per row) <-> blocked layout
__global__ void k_spec_unpack(const float2 *__restrict__ S, int H, int Y, int Z, int nkb, float2 *__restrict__ out)
{
    const long long n = (long long) H * Y * Z;
    for (long long k = blockIdx.x * (long long) blockDim.x + threadIdx.x; k < n;
         k += (long long) gridDim.x * blockDim.x) {
        const int kx = (int) (k % H);
        const long long r = k / H;
        const int y = (int) (r % Y);
        const int z = (int) (r / Y);
        out[k] = S[(((long long) z * nkb + kx / KB) * Y + y) * KB + kx % KB];
    }
}

__global__ void k_spec_pack(const float2 *__restrict__ in, int H, int Y, int Z, int nkb, float2 *__restrict__ S)
{
    const long long n = (long long) H * Y * Z;
    for (long long k = blockIdx.x * (long long) blockDim.x + threadIdx.x; k < n;
         k += (long long) gridDim.x * blockDim.x) {
        const int kx = (int) (k % H);
        const long long r = k / H;
        const int y = (int) (r % Y);
        const int z = (int) (r / Y);
        S[(((long long) z * nkb + kx / KB) * Y + y) * KB + kx % KB] = in[k];
    }
}

// finish one iteration's error: mean over the image of the x-pass partials
// (get_fIdiv dw.c:1492-1524 / get_fMSE dw.c:1461-1490)
__global__ void __launch_bounds__(kRedThreads)
k_err_final(const double *__restrict__ part, int nb, double count, float *err_out)
{
    __shared__ double s[kRedThreads];
    double v = 0.0;
    for (int i = threadIdx.x; i < nb; i += kRedThreads) v += part[i];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = kRedThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *err_out = (float) (s[0] / count);
}

}  // namespace dwcu
