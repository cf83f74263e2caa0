// host.cu -- the parts of dw_run around the iteration: PSF preparation and
// tiled deconvolution with all tiles batched on the GPU.
//
//   dwcu_psf_prepare      fim_normalize_sum1 (src/fim.c:900-912) and
//                         psf_autocrop (src/dw.c:1764-1997)
//   dwcu_tiling_create    tiling_getDivision / tiling_create (src/tiling.c:22-130)
//   dwcu_deconvolve_tiled deconvolve_tiles (src/dw.c:2001-2229) without the
//                         temporary raw files: the image stays on the device,
//                         tiles become jobs that iterate as one batch, and the
//                         weighted blend of tiling_put_tile (src/tiling.c:412-439)
//                         runs as a device kernel per tile, in tile order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dwcu.h"

namespace dwcu {
void record_error(const char *msg);  // engine.cu: the text dwcu_last_error returns
void record_launch();                // engine.cu: dwcu_launch_count
}  // namespace dwcu

namespace dwcu_host {

static int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    dwcu::record_error(buf);
    return code;
}

#define HCU(call)                                                                                      \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return fail(e_ == cudaErrorMemoryAllocation ? DWCU_ERROR_OUT_OF_MEMORY : DWCU_ERROR_CUDA,  \
                        "%s failed: %s", #call, cudaGetErrorString(e_));                               \
    } while (0)

// ------------------------------------------------------------ PSF preparation

// fim_normalize_sum1, fim.c:900-912: divide by the double sum
static void normalize_sum1(std::vector<float> &p)
{
    double s = 0;
    for (float v : p) s += v;
    for (float &v : p) v = (float) (v / s);
}

// fim_get_cuboid, fim.c:659-693
static std::vector<float> cuboid(const std::vector<float> &A, int64_t M, int64_t N, int64_t m0, int64_t m1,
                                 int64_t n0, int64_t n1, int64_t p0, int64_t p1)
{
    const int64_t m = m1 - m0 + 1, n = n1 - n0 + 1, p = p1 - p0 + 1;
    std::vector<float> C((size_t) (m * n * p));
    for (int64_t cc = p0; cc <= p1; ++cc)
        for (int64_t bb = n0; bb <= n1; ++bb)
            for (int64_t aa = m0; aa <= m1; ++aa)
                C[(size_t) ((aa - m0) + (bb - n0) * m + (cc - p0) * m * n)] = A[(size_t) (aa + bb * M + cc * M * N)];
    return C;
}

// psf_autocrop_byImage, dw.c:1764-1860
static void crop_by_image(std::vector<float> &psf, int64_t &pM, int64_t &pN, int64_t &pP, int64_t M, int64_t N,
                          int64_t P, int bq)
{
    int64_t mopt = (M - 1) * 2 + 1, nopt = (N - 1) * 2 + 1, popt = (P - 1) * 2 + 1;
    if (bq == 0) {
        mopt = M;
        nopt = N;
        popt = P;
    }
    if (pP < popt) return;  // the reference warns that the PSF has too few slices
    if (pM > mopt || pN > nopt || pP > popt) {
        int64_t m0 = 0, m1 = pM - 1, n0 = 0, n1 = pN - 1, p0 = 0, p1 = pP - 1;
        if (pM > mopt) { m0 = (pM - mopt) / 2; m1 = m1 - (pM - mopt) / 2; }
        if (pN > nopt) { n0 = (pN - nopt) / 2; n1 = n1 - (pN - nopt) / 2; }
        if (pP > popt) { p0 = (pP - popt) / 2; p1 = p1 - (pP - popt) / 2; }
        psf = cuboid(psf, pM, pN, m0, m1, n0, n1, p0, p1);
        pM = m1 - m0 + 1;
        pN = n1 - n0 + 1;
        pP = p1 - p0 + 1;
    }
}

// psf_autocrop_XY, dw.c:1862-1971 (without the FFTW lookahead benchmark):
// drop outer x (and as many y) planes whose y-z sum is below
// xycropfactor times the largest one; float sums as in the reference
static void crop_xy(std::vector<float> &psf, int64_t &pM, int64_t &pN, int64_t pP, float xycropfactor)
{
    // every x plane's sum in the reference's order (y outer, z inner), all
    // planes at once so that the reads run along x
    std::vector<float> plane((size_t) pM, 0.f);
    for (int64_t yy = 0; yy < pN; ++yy)
        for (int64_t zz = 0; zz < pP; ++zz) {
            const float *row = psf.data() + (size_t) (yy * pM + zz * pM * pN);
            for (int64_t xx = 0; xx < pM; ++xx) plane[(size_t) xx] += row[xx];
        }
    float maxsum = 0;
    for (int64_t xx = 0; xx < pM; ++xx)
        if (plane[(size_t) xx] > maxsum) maxsum = plane[(size_t) xx];
    int64_t first = -1;
    float sum = 0;
    while (sum < xycropfactor * maxsum && first + 1 < pM) {
        first++;
        sum = plane[(size_t) first];
    }
    if (first < 1) return;
    if (pM - 2 * first < 1 || pN - 2 * first < 1) return;
    psf = cuboid(psf, pM, pN, first, pM - first - 1, first, pN - first - 1, 0, pP - 1);
    pM -= 2 * first;
    pN -= 2 * first;
}

// ------------------------------------------------------------ PSF preparation on the device
//
// The same steps as above on a device copy of the PSF, for the GPU's own
// set-up (the tiled path): the double sums of the normalisations as a
// fixed-order tree (a fixed grid of partial sums, then one thread), each
// value divided in double and rounded to float as fim_normalize_sum1 does
// (fim.c:900-912; the reference's own sum is an OpenMP reduction, so its
// order varies with the thread count, which moves the double sum by
// rounding only); the x-plane sums of psf_autocrop_XY in float, one thread
// per plane in the reference's order (y outer, z inner, dw.c:1885-1907), so
// the crop decision is the reference's bit for bit.

constexpr int kPsfSumBlocks = 128;
constexpr int kPsfThreads = 256;

__global__ void k_psf_sum_partial(const float *__restrict__ p, long long n, double *__restrict__ part)
{
    __shared__ double sh[kPsfThreads];
    double s = 0;
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x)
        s += (double) p[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = kPsfThreads / 2; o > 0; o >>= 1) {
        if ((int) threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_psf_sum_final(const double *__restrict__ part, int n, double *__restrict__ out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0;
        for (int i = 0; i < n; ++i) s += part[i];
        *out = s;
    }
}

// out = the cuboid [m0, m0+m) x [n0, n0+n) x [p0, p0+p) of in (M x N x ...),
// divided by *sum when sum is given (fim_get_cuboid, fim.c:659-693)
__global__ void k_psf_crop_scale(const float *__restrict__ in, long long M, long long N, long long m0, long long n0,
                                 long long p0, long long m, long long n, long long p, const double *__restrict__ sum,
                                 float *__restrict__ out)
{
    const long long tot = m * n * p;
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < tot; i += (long long) gridDim.x * blockDim.x) {
        const long long a = i % m, b = (i / m) % n, c = i / (m * n);
        const float v = in[(a + m0) + (b + n0) * M + (c + p0) * M * N];
        out[i] = sum ? (float) ((double) v / *sum) : v;
    }
}

// psf_autocrop_XY's decision (dw.c:1862-1912): the float sum of every x
// plane in the reference's order, the largest of them, and the first plane
// whose sum reaches xycropfactor times it
__global__ void k_psf_plane_sums(const float *__restrict__ p, long long M, long long N, long long P,
                                 float *__restrict__ plane)
{
    const long long xx = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if (xx >= M) return;
    float sum = 0.f;
    for (long long yy = 0; yy < N; ++yy)
        for (long long zz = 0; zz < P; ++zz) sum += p[xx + yy * M + zz * M * N];
    plane[xx] = sum;
}

__global__ void k_psf_first_plane(const float *__restrict__ plane, long long M, float factor, long long *first_out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float maxsum = 0.f;
    for (long long xx = 0; xx < M; ++xx)
        if (plane[xx] > maxsum) maxsum = plane[xx];
    long long first = -1;
    float sum = 0.f;
    while (sum < factor * maxsum && first + 1 < M) {
        first++;
        sum = plane[first];
    }
    *first_out = first;
}

// d_out (room for pM*pN*pP floats) receives the prepared PSF; dims[3] its
// size.  Scratch is allocated here and freed before returning; the call
// waits for its stream (the caller needs the size).
static int psf_prepare_device(const float *d_psf, int64_t pM, int64_t pN, int64_t pP, int64_t M, int64_t N,
                              int64_t P, int bq, float xycropfactor, float *d_out, int64_t dims[3], cudaStream_t st)
{
    const long long n0 = pM * pN * pP;
    char *scratch = nullptr;
    // partials, two sums, the first plane, the x-plane sums, two cuboids
    const size_t o_part = 0, o_sum = 1024 + 8 * kPsfSumBlocks, o_first = o_sum + 256, o_plane = o_first + 256;
    const size_t o_b1 = o_plane + ((size_t) (4 * pM) + 255) / 256 * 256;
    const size_t o_b2 = o_b1 + ((size_t) (4 * n0) + 255) / 256 * 256;
    const size_t bytes = o_b2 + ((size_t) (4 * n0) + 255) / 256 * 256;
    HCU(cudaMalloc(&scratch, bytes));
    struct Free {
        char *p;
        ~Free() { cudaFree(p); }
    } guard{scratch};
    double *part = (double *) (scratch + o_part), *sum1 = (double *) (scratch + o_sum), *sum2 = sum1 + 1;
    long long *first_d = (long long *) (scratch + o_first);
    float *plane = (float *) (scratch + o_plane), *b1 = (float *) (scratch + o_b1), *b2 = (float *) (scratch + o_b2);
    auto dsum = [&](const float *p, long long n, double *out) -> int {
        k_psf_sum_partial<<<kPsfSumBlocks, kPsfThreads, 0, st>>>(p, n, part);
        k_psf_sum_final<<<1, 32, 0, st>>>(part, kPsfSumBlocks, out);
        dwcu::record_launch();
        dwcu::record_launch();
        return cudaGetLastError() == cudaSuccess ? DWCU_SUCCESS : fail(DWCU_ERROR_CUDA, "PSF sum launch failed");
    };
    auto crop = [&](const float *in, long long Mi, long long Ni, long long m0, long long nn0, long long p0,
                    long long m, long long n, long long p, const double *sc, float *out) -> int {
        const long long tot = m * n * p;
        const int blocks = (int) std::min<long long>(148 * 8, (tot + kPsfThreads - 1) / kPsfThreads);
        k_psf_crop_scale<<<std::max(blocks, 1), kPsfThreads, 0, st>>>(in, Mi, Ni, m0, nn0, p0, m, n, p, sc, out);
        dwcu::record_launch();
        return cudaGetLastError() == cudaSuccess ? DWCU_SUCCESS : fail(DWCU_ERROR_CUDA, "PSF crop launch failed");
    };
    // normalise (dw.c:2799), crop against the image (psf_autocrop_byImage)
    int rc = dsum(d_psf, n0, sum1);
    int64_t a0 = 0, a1 = pM - 1, c0 = 0, c1 = pN - 1, e0 = 0, e1 = pP - 1;
    {
        int64_t mopt = (M - 1) * 2 + 1, nopt = (N - 1) * 2 + 1, popt = (P - 1) * 2 + 1;
        if (bq == 0) { mopt = M; nopt = N; popt = P; }
        if (pP >= popt && (pM > mopt || pN > nopt || pP > popt)) {
            if (pM > mopt) { a0 = (pM - mopt) / 2; a1 -= (pM - mopt) / 2; }
            if (pN > nopt) { c0 = (pN - nopt) / 2; c1 -= (pN - nopt) / 2; }
            if (pP > popt) { e0 = (pP - popt) / 2; e1 -= (pP - popt) / 2; }
        }
    }
    int64_t m = a1 - a0 + 1, n = c1 - c0 + 1, p = e1 - e0 + 1;
    if (rc == DWCU_SUCCESS) rc = crop(d_psf, pM, pN, a0, c0, e0, m, n, p, sum1, b1);
    // drop faint outer x and y planes (psf_autocrop_XY)
    long long first = 0;
    if (rc == DWCU_SUCCESS && bq > 0 && xycropfactor > 0) {
        k_psf_plane_sums<<<(int) ((m + 127) / 128), 128, 0, st>>>(b1, m, n, p, plane);
        k_psf_first_plane<<<1, 32, 0, st>>>(plane, m, xycropfactor, first_d);
        dwcu::record_launch();
        dwcu::record_launch();
        if (cudaGetLastError() != cudaSuccess) rc = fail(DWCU_ERROR_CUDA, "PSF plane-sum launch failed");
        if (rc == DWCU_SUCCESS &&
            (cudaMemcpyAsync(&first, first_d, sizeof first, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
             cudaStreamSynchronize(st) != cudaSuccess))
            rc = fail(DWCU_ERROR_CUDA, "reading the PSF crop failed");
    }
    int64_t f = (first >= 1 && m - 2 * first >= 1 && n - 2 * first >= 1) ? first : 0;
    const int64_t m2 = m - 2 * f, n2 = n - 2 * f;
    // the cropped PSF, normalised again (dw.c:2826)
    if (rc == DWCU_SUCCESS) rc = crop(b1, m, n, f, f, 0, m2, n2, p, nullptr, b2);
    if (rc == DWCU_SUCCESS) rc = dsum(b2, m2 * n2 * p, sum2);
    if (rc == DWCU_SUCCESS) rc = crop(b2, m2, n2, 0, 0, 0, m2, n2, p, sum2, d_out);
    if (rc == DWCU_SUCCESS && cudaStreamSynchronize(st) != cudaSuccess)
        rc = fail(DWCU_ERROR_CUDA, "PSF preparation failed on the device");
    dims[0] = m2;
    dims[1] = n2;
    dims[2] = p;
    return rc;
}

}  // namespace dwcu_host

using namespace dwcu_host;

// ------------------------------------------------------------ tiling kernels

namespace {

struct DevTile {
    long long pos[6], xpos[6], xsize[3];
};

// getWeight1d, tiling.c:169-197 (float arithmetic as in the reference)
__host__ __device__ inline float weight1d(float a, float b, float c, float d, long long x)
{
    const float xf = (float) x;
    if (xf < a || xf > d) return 0.f;
    if (xf >= b && xf <= c) return 1.f;
    if (xf >= a && xf <= b) return (xf - a + 1) / (b - a + 1);
    if (xf >= c && xf <= d) return 1 - (xf - c) / (d - c + 1);
    return 0.f;
}

// tile_getWeight, tiling.c:199-216
__host__ __device__ inline float tile_weight(const DevTile &t, long long m, long long n)
{
    const float wm = weight1d((float) t.xpos[0], (float) t.pos[0], (float) t.pos[1], (float) t.xpos[1], m);
    const float wn = weight1d((float) t.xpos[2], (float) t.pos[2], (float) t.pos[3], (float) t.xpos[3], n);
    return fminf(wm, wn);
}

// tiling_get_tile (tiling.c:318-351) plus the offset dw.c adds per tile
__global__ void k_tile_extract(const float *__restrict__ im, long long M, long long N, DevTile t, float offset,
                               float *__restrict__ out)
{
    const long long m = t.xsize[0], n = t.xsize[1], p = t.xsize[2];
    const long long total = m * n * p;
    for (long long k = blockIdx.x * (long long) blockDim.x + threadIdx.x; k < total;
         k += (long long) gridDim.x * blockDim.x) {
        const long long a = k % m, b = (k / m) % n, c = k / (m * n);
        float v = im[(a + t.xpos[0]) + (b + t.xpos[2]) * M + (c + t.xpos[4]) * M * N];
        if (offset > 0) v += offset;
        out[k] = v;
    }
}

// minus the offset, project positive (dw.c:2141-2145), then tiling_put_tile
// (tiling.c:412-439): V += w / sum_w * S, tiles in order
__global__ void k_tile_blend(const float *__restrict__ S, long long M, long long N, const DevTile *__restrict__ tiles,
                             int ntiles, int tid, float offset, float *__restrict__ V)
{
    const DevTile t = tiles[tid];
    const long long m = t.xsize[0], n = t.xsize[1], p = t.xsize[2];
    const long long total = m * n * p;
    for (long long k = blockIdx.x * (long long) blockDim.x + threadIdx.x; k < total;
         k += (long long) gridDim.x * blockDim.x) {
        const long long a = k % m, b = (k / m) % n, c = k / (m * n);
        const long long aa = a + t.xpos[0], bb = b + t.xpos[2], cc = c + t.xpos[4];
        float s = S[k];
        if (offset > 0) {
            s = __fadd_rn(s, -offset);
            if (s < 0) s = 0;
        }
        float w = tile_weight(t, aa, bb);
        float ws = 0;
        for (int q = 0; q < ntiles; ++q) ws = __fadd_rn(ws, tile_weight(tiles[q], aa, bb));
        w = __fdiv_rn(w, ws);
        float &v = V[aa + bb * M + cc * M * N];
        v = __fadd_rn(v, __fmul_rn(w, s));  // no contraction: the CPU blend rounds twice
    }
}

}  // namespace

// ------------------------------------------------------------ C ABI

extern "C" {

int dwcu_psf_prepare(const float *psf, int64_t pM, int64_t pN, int64_t pP, int64_t M, int64_t N, int64_t P,
                     int32_t border_quality, float xycropfactor, float *out, int64_t out_dims[3])
{
    if (!psf || !out || !out_dims) return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    if (pM < 1 || pN < 1 || pP < 1 || M < 1 || N < 1 || P < 1) return fail(DWCU_ERROR_INVALID_VALUE, "bad sizes");
    std::vector<float> p(psf, psf + pM * pN * pP);
    normalize_sum1(p);                                          // dw.c:2799
    crop_by_image(p, pM, pN, pP, M, N, P, border_quality);      // dw.c:1985-1988
    if (border_quality > 0 && xycropfactor > 0) crop_xy(p, pM, pN, pP, xycropfactor);  // dw.c:1990-1996
    normalize_sum1(p);                                          // dw.c:2826
    memcpy(out, p.data(), sizeof(float) * p.size());
    out_dims[0] = pM;
    out_dims[1] = pN;
    out_dims[2] = pP;
    return DWCU_SUCCESS;
}

int dwcu_psf_prepare_device(const float *d_psf, int64_t pM, int64_t pN, int64_t pP, int64_t M, int64_t N,
                            int64_t P, int32_t border_quality, float xycropfactor, float *d_out, int64_t out_dims[3],
                            int32_t device, void *stream)
{
    if (!d_psf || !d_out || !out_dims) return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    if (pM < 1 || pN < 1 || pP < 1 || M < 1 || N < 1 || P < 1) return fail(DWCU_ERROR_INVALID_VALUE, "bad sizes");
    HCU(cudaSetDevice(device));
    cudaStream_t st = stream ? (cudaStream_t) stream : cudaStreamPerThread;
    return psf_prepare_device(d_psf, pM, pN, pP, M, N, P, border_quality, xycropfactor, d_out, out_dims, st);
}

int dwcu_tiling_create(int64_t M, int64_t N, int64_t P, int64_t max_size, int64_t overlap, dwcu_tile *tiles,
                       int32_t capacity, int32_t *ntiles)
{
    if (M < 1 || N < 1 || P < 1 || max_size < 1 || overlap < 0 || !ntiles)
        return fail(DWCU_ERROR_INVALID_VALUE, "bad tiling arguments");
    // tiling_getDivision, tiling.c:22-58 (float section width as in the reference)
    auto division = [](int64_t L, int64_t m, std::vector<int64_t> &divs) {
        const float ns = (float) std::ceil((double) L / (double) m);
        const float width = (float) L / ns;
        const int64_t n = (int64_t) ns;
        divs.assign((size_t) (2 * n), 0);
        divs[0] = 0;
        divs[(size_t) (2 * n - 1)] = L - 1;
        for (int64_t dd = 1; dd < n; ++dd) {
            divs[(size_t) (dd * 2 - 1)] = (int64_t) std::ceil(width * (float) dd) - 1;
            divs[(size_t) (dd * 2)] = divs[(size_t) (dd * 2 - 1)] + 1;
        }
        return n;
    };
    std::vector<int64_t> dM, dN;
    const int64_t nM = division(M, max_size, dM), nN = division(N, max_size, dN);
    *ntiles = (int32_t) (nM * nN);
    if (!tiles) return DWCU_SUCCESS;
    if (capacity < nM * nN) return fail(DWCU_ERROR_INVALID_VALUE, "tile array too small (%lld)", (long long) (nM * nN));
    int b = 0;
    for (int64_t mm = 0; mm < nM; ++mm)  // tiling.c:95-128
        for (int64_t nn = 0; nn < nN; ++nn, ++b) {
            dwcu_tile &t = tiles[b];
            t.size[0] = dM[(size_t) (mm * 2 + 1)] - dM[(size_t) (mm * 2)] + 1;
            t.size[1] = dN[(size_t) (nn * 2 + 1)] - dN[(size_t) (nn * 2)] + 1;
            t.size[2] = P;
            t.pos[0] = dM[(size_t) (mm * 2)]; t.pos[1] = dM[(size_t) (mm * 2 + 1)];
            t.pos[2] = dN[(size_t) (nn * 2)]; t.pos[3] = dN[(size_t) (nn * 2 + 1)];
            t.pos[4] = 0; t.pos[5] = P - 1;
            t.xpos[0] = std::max<int64_t>(0, t.pos[0] - overlap);
            t.xpos[1] = std::min<int64_t>(t.pos[1] + overlap, M - 1);
            t.xpos[2] = std::max<int64_t>(0, t.pos[2] - overlap);
            t.xpos[3] = std::min<int64_t>(t.pos[3] + overlap, N - 1);
            t.xpos[4] = t.pos[4]; t.xpos[5] = t.pos[5];
            t.xsize[0] = t.xpos[1] - t.xpos[0] + 1;
            t.xsize[1] = t.xpos[3] - t.xpos[2] + 1;
            t.xsize[2] = t.xpos[5] - t.xpos[4] + 1;
        }
    return DWCU_SUCCESS;
}

int dwcu_deconvolve_tiled(const float *im, int64_t M, int64_t N, int64_t P, const float *psf, int64_t pM,
                          int64_t pN, int64_t pP, int64_t tile_size, int64_t overlap, float offset,
                          float xycropfactor, double hbm_budget, dwcu_opts *s, float *out)
{
    if (!im || !psf || !out || !s) return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    int32_t nt = 0;
    int rc = dwcu_tiling_create(M, N, P, tile_size, overlap, nullptr, 0, &nt);
    if (rc) return rc;
    if (nt < 2) return fail(DWCU_ERROR_INVALID_VALUE, "only one tile: omit the tile size or decrease it");
    std::vector<dwcu_tile> tiles((size_t) nt);
    dwcu_tiling_create(M, N, P, tile_size, overlap, tiles.data(), nt, &nt);
    HCU(cudaSetDevice(s->device));
    cudaStream_t st = nullptr;
    HCU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const size_t nvox = (size_t) (M * N * P);
    float *d_im = nullptr, *d_out = nullptr;
    DevTile *d_tiles = nullptr;
    std::vector<DevTile> ht((size_t) nt);
    for (int i = 0; i < nt; ++i) {
        memcpy(ht[(size_t) i].pos, tiles[(size_t) i].pos, sizeof ht[0].pos);
        memcpy(ht[(size_t) i].xpos, tiles[(size_t) i].xpos, sizeof ht[0].xpos);
        memcpy(ht[(size_t) i].xsize, tiles[(size_t) i].xsize, sizeof ht[0].xsize);
    }
    auto cleanup = [&]() {
        if (d_im) cudaFree(d_im);
        if (d_out) cudaFree(d_out);
        if (d_tiles) cudaFree(d_tiles);
        if (st) cudaStreamDestroy(st);
    };
#define TCU(call)                                                                       \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            cleanup();                                                                  \
            return fail(e_ == cudaErrorMemoryAllocation ? DWCU_ERROR_OUT_OF_MEMORY : DWCU_ERROR_CUDA, \
                        "%s failed: %s", #call, cudaGetErrorString(e_));                \
        }                                                                               \
    } while (0)
    TCU(cudaMalloc(&d_im, sizeof(float) * nvox));
    TCU(cudaMalloc(&d_out, sizeof(float) * nvox));
    TCU(cudaMalloc(&d_tiles, sizeof(DevTile) * (size_t) nt));
    TCU(cudaMemcpyAsync(d_im, im, sizeof(float) * nvox, cudaMemcpyHostToDevice, st));
    TCU(cudaMemcpyAsync(d_tiles, ht.data(), sizeof(DevTile) * (size_t) nt, cudaMemcpyHostToDevice, st));
    TCU(cudaMemsetAsync(d_out, 0, sizeof(float) * nvox, st));

    // Pageable output pages are touched by a host thread while the tiles
    // iterate, so that the final device-to-host copy does not fault them in
    // (page-locked memory is resident already).
    // (not when the result buffer is the image itself)
    cudaPointerAttributes pa;
    const bool locked = cudaPointerGetAttributes(&pa, out) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();
    const uintptr_t o0 = (uintptr_t) out, i0 = (uintptr_t) im, nb = sizeof(float) * nvox;
    const bool aliased = o0 < i0 + nb && i0 < o0 + nb;
    std::thread prefault;
    if (!locked && !aliased)
        prefault = std::thread([out, nvox]() {
            const size_t chunk = (size_t) 1 << 22;
            for (size_t i = 0; i < nvox; i += chunk) memset(out + i, 0, sizeof(float) * std::min(chunk, nvox - i));
        });
    struct Joiner {
        std::thread &t;
        ~Joiner() { if (t.joinable()) t.join(); }
    } joiner{prefault};

    // per tile: PSF copy normalised and cropped against the tile
    // (dw.c:2112-2130), on the device; tiles of one size share the result
    struct TilePsf {
        int64_t xs[3];
        int64_t d[3];
        float *dev = nullptr;
    };
    std::vector<TilePsf> psfs;
    std::vector<int> psf_of((size_t) nt);
    float *d_psf_in = nullptr;
    auto free_psfs = [&]() {
        for (auto &tp : psfs)
            if (tp.dev) cudaFree(tp.dev);
        if (d_psf_in) cudaFree(d_psf_in);
        d_psf_in = nullptr;
    };
    {
        cudaError_t e = cudaMalloc(&d_psf_in, sizeof(float) * (size_t) (pM * pN * pP));
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_psf_in, psf, sizeof(float) * (size_t) (pM * pN * pP), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {
            free_psfs();
            cleanup();
            return fail(e == cudaErrorMemoryAllocation ? DWCU_ERROR_OUT_OF_MEMORY : DWCU_ERROR_CUDA,
                        "PSF upload failed: %s", cudaGetErrorString(e));
        }
    }
    for (int i = 0; i < nt; ++i) {
        const dwcu_tile &t = tiles[(size_t) i];
        int k = 0;
        while (k < (int) psfs.size() && !(psfs[(size_t) k].xs[0] == t.xsize[0] && psfs[(size_t) k].xs[1] == t.xsize[1] &&
                                          psfs[(size_t) k].xs[2] == t.xsize[2]))
            ++k;
        if (k == (int) psfs.size()) {
            TilePsf tp;
            memcpy(tp.xs, t.xsize, sizeof tp.xs);
            int prc = cudaMalloc(&tp.dev, sizeof(float) * (size_t) (pM * pN * pP)) == cudaSuccess
                          ? DWCU_SUCCESS
                          : fail(DWCU_ERROR_OUT_OF_MEMORY, "tile PSF buffer");
            if (prc == DWCU_SUCCESS)
                prc = psf_prepare_device(d_psf_in, pM, pN, pP, t.xsize[0], t.xsize[1], t.xsize[2], s->border_quality,
                                         xycropfactor, tp.dev, tp.d, st);
            psfs.push_back(tp);
            if (prc != DWCU_SUCCESS) {
                free_psfs();
                cleanup();
                return prc;
            }
        }
        psf_of[(size_t) i] = k;
    }
    // waves of tiles that fit the device-memory budget, each run as one
    // batch; a tile whose job fills the GPU on its own (>= 32 Mi padded
    // voxels, which the batch runner would run one after another anyway)
    // is a wave of its own, so that its job block is reused by the next
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const double budget = hbm_budget > 0 ? hbm_budget : 0.85 * (double) free_b;
    const double large = 32.0 * 1024 * 1024;
    struct TileJob {
        dwcu_job *job = nullptr;
        float *d_tile = nullptr;
    };
    std::vector<TileJob> tj((size_t) nt);
    std::vector<float *> bufs;  // tile buffers, reused by the waves
    size_t buf_elems = 0;
    for (const auto &t : tiles) buf_elems = std::max(buf_elems, (size_t) (t.xsize[0] * t.xsize[1] * t.xsize[2]));
    int next = 0;
    rc = DWCU_SUCCESS;
    while (next < nt && rc == DWCU_SUCCESS) {
        std::vector<int> wave;
        double used = 0;
        for (int i = next; i < nt; ++i) {
            const dwcu_tile &t = tiles[(size_t) i];
            const TilePsf &tp = psfs[(size_t) psf_of[(size_t) i]];
            int64_t w3[3];
            int64_t need = 0;
            rc = dwcu_plan_size(t.xsize[0], t.xsize[1], t.xsize[2], tp.d[0], tp.d[1], tp.d[2], s->border_quality,
                                s->method, w3, &need);
            if (rc) break;
            const bool big = (double) w3[0] * (double) w3[1] * (double) w3[2] >= large;
            need += (int64_t) (sizeof(float) * (t.xsize[0] * t.xsize[1] * t.xsize[2]) * 2);
            if (!wave.empty() && (big || used + (double) need > budget)) break;
            used += (double) need;
            wave.push_back(i);
            if (big) break;
        }
        if (rc) break;
        while (bufs.size() < wave.size()) {
            float *b = nullptr;
            if (cudaMalloc(&b, sizeof(float) * buf_elems) != cudaSuccess) {
                rc = fail(DWCU_ERROR_OUT_OF_MEMORY, "tile buffers");
                break;
            }
            bufs.push_back(b);
        }
        if (rc) break;
        std::vector<dwcu_job *> jobs;
        for (size_t w = 0; w < wave.size(); ++w) {
            const int i = wave[w];
            TileJob &T = tj[(size_t) i];
            const dwcu_tile &t = tiles[(size_t) i];
            const TilePsf &tp = psfs[(size_t) psf_of[(size_t) i]];
            const size_t tv = (size_t) (t.xsize[0] * t.xsize[1] * t.xsize[2]);
            T.d_tile = bufs[w];
            const int blocks = (int) std::min<size_t>(4096, (tv + 255) / 256);
            k_tile_extract<<<blocks, 256, 0, st>>>(d_im, M, N, ht[(size_t) i], offset, T.d_tile);
            dwcu::record_launch();
            if (cudaStreamSynchronize(st) != cudaSuccess) {
                rc = fail(DWCU_ERROR_CUDA, "tile extraction failed");
                break;
            }
            rc = dwcu_job_create(t.xsize[0], t.xsize[1], t.xsize[2], tp.d[0], tp.d[1], tp.d[2], s, &T.job);
            if (rc == DWCU_SUCCESS) rc = dwcu_job_setup(T.job, T.d_tile, tp.dev, 1);
            if (rc) break;
            jobs.push_back(T.job);
        }
        if (rc == DWCU_SUCCESS) rc = dwcu_batch_run(jobs.data(), (int32_t) jobs.size(), st);
        // results in tile order, blended on the device
        for (int i : wave) {
            TileJob &T = tj[(size_t) i];
            const dwcu_tile &t = tiles[(size_t) i];
            const size_t tv = (size_t) (t.xsize[0] * t.xsize[1] * t.xsize[2]);
            if (rc == DWCU_SUCCESS && T.job) {
                dwcu_opts so;
                dwcu_opts_init(&so);
                so.error_trace = nullptr;
                rc = dwcu_job_result(T.job, T.d_tile, 1, &so);
                if (rc == DWCU_SUCCESS) {
                    s->iterations_done = so.iterations_done;
                    const int blocks = (int) std::min<size_t>(4096, (tv + 255) / 256);
                    k_tile_blend<<<blocks, 256, 0, st>>>(T.d_tile, M, N, d_tiles, nt, i, offset, d_out);
                    dwcu::record_launch();
                    if (cudaStreamSynchronize(st) != cudaSuccess) rc = fail(DWCU_ERROR_CUDA, "tile blend failed");
                }
            }
            if (T.job) dwcu_job_destroy(T.job);
            T.job = nullptr;
            T.d_tile = nullptr;
        }
        next = wave.empty() ? nt : wave.back() + 1;
    }
    if (prefault.joinable()) prefault.join();
    if (rc == DWCU_SUCCESS) {
        cudaError_t e = cudaMemcpyAsync(out, d_out, sizeof(float) * nvox, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = fail(DWCU_ERROR_CUDA, "result copy failed: %s", cudaGetErrorString(e));
    }
    for (auto *b : bufs) cudaFree(b);
    free_psfs();
    for (auto &T : tj)
        if (T.job) dwcu_job_destroy(T.job);
    cleanup();
#undef TCU
    return rc;
}

int dwcu_tile_blend(float *d_out, int64_t M, int64_t N, int64_t P, const dwcu_tile *tiles, int32_t ntiles,
                    int32_t tid, const float *d_tile, float offset, int32_t device, void *stream)
{
    if (!d_out || !tiles || !d_tile) return fail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    if (ntiles < 1 || tid < 0 || tid >= ntiles) return fail(DWCU_ERROR_INVALID_VALUE, "bad tile index");
    for (int i = 0; i < ntiles; ++i) {
        const dwcu_tile &t = tiles[i];
        if (t.xpos[0] < 0 || t.xpos[1] >= M || t.xpos[2] < 0 || t.xpos[3] >= N || t.xpos[4] < 0 || t.xpos[5] >= P ||
            t.xsize[0] != t.xpos[1] - t.xpos[0] + 1 || t.xsize[1] != t.xpos[3] - t.xpos[2] + 1 ||
            t.xsize[2] != t.xpos[5] - t.xpos[4] + 1)
            return fail(DWCU_ERROR_INVALID_VALUE, "tile %d does not lie in the image", i);
    }
    HCU(cudaSetDevice(device));
    cudaStream_t st = (cudaStream_t) stream;
    std::vector<DevTile> ht((size_t) ntiles);
    for (int i = 0; i < ntiles; ++i) {
        memcpy(ht[(size_t) i].pos, tiles[i].pos, sizeof ht[0].pos);
        memcpy(ht[(size_t) i].xpos, tiles[i].xpos, sizeof ht[0].xpos);
        memcpy(ht[(size_t) i].xsize, tiles[i].xsize, sizeof ht[0].xsize);
    }
    DevTile *d_tiles = nullptr;
    HCU(cudaMalloc(&d_tiles, sizeof(DevTile) * (size_t) ntiles));
    cudaError_t e = cudaMemcpyAsync(d_tiles, ht.data(), sizeof(DevTile) * (size_t) ntiles, cudaMemcpyHostToDevice, st);
    const dwcu_tile &t = tiles[tid];
    const size_t tv = (size_t) (t.xsize[0] * t.xsize[1] * t.xsize[2]);
    if (e == cudaSuccess) {
        const int blocks = (int) std::min<size_t>(4096, (tv + 255) / 256);
        k_tile_blend<<<blocks, 256, 0, st>>>(d_tile, M, N, d_tiles, ntiles, tid, offset, d_out);
        dwcu::record_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_tiles);
    if (e != cudaSuccess) return fail(DWCU_ERROR_CUDA, "tile blend failed: %s", cudaGetErrorString(e));
    return DWCU_SUCCESS;
}

}  // extern "C"
