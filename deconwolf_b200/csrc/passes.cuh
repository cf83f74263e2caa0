// passes.cuh -- the FFT passes of one RL/SHB iteration (sm_100a).
//
// Data layout in HBM (per job):
//   real volumes  X x Y x Z floats, x fastest, row pitch X (X even)
//   spectrum      (X/2+1) x Y x Z complex, row pitch XC complex (XC even)
//   image g       M x N x P floats, row pitch GP (even)
//
// Line transforms are self-sorting (Stockham) mixed-radix FFTs of length
// N = RA*RB*RC (RC may be 1) with radices <= 16.  One line is handled by
// TPL = N / min(R) threads; in stage s each active thread runs one radix-R_s
// butterfly fully in registers (dft.cuh), and stages exchange through shared
// memory.  The last stage leaves thread t holding elements t + r*N/R_last,
// which is exactly what the first stage of a transform with the reversed
// radix list reads -- so a forward transform followed by an inverse one (the
// OTF multiply in between) or an inverse followed by a forward one (the
// pointwise op in between) hands over in registers, with no extra exchange.
//
// k_lines  : complex transforms along a strided axis (y or z), T adjacent
//            lines per CTA so every global access is T*8 contiguous bytes.
//            Modes: forward, inverse, and convolve = forward, multiply by the
//            OTF (or its conjugate), inverse: the spectrum is read and
//            written once.
// k_xpass  : the x axis, R rows per CTA: optional C2R (Hermitian
//            pre-processing + half-length complex inverse), one pointwise op
//            on the real values (ratio + I-divergence, SHB/RL update, Bertero
//            weights, ...), optional R2C (half-length forward + Hermitian
//            post-processing), all in one kernel.
#pragma once
#include <cstdint>
#include "dft.cuh"
#include "tma.cuh"

namespace dwcu {

__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int cmin(int a, int b) { return a < b ? a : b; }

// Compile-time description of one line length.
template <int RA_, int RB_, int RC_>
struct Rad {
    static constexpr int RA = RA_, RB = RB_, RC = RC_;
    static constexpr int N = RA * RB * RC;
    static constexpr bool THREE = (RC > 1);
    static constexpr int RL = THREE ? RC : RB;  // last radix
    static constexpr int TPL = cmax(cmax(N / RA, N / RB), THREE ? N / RC : 0);
    // padded exchange index: for an even first radix, one spare slot per RA
    // block makes the first stage's stride-RA writes an odd number of
    // float2 apart, which keeps them free of bank conflicts; an odd RA
    // already is, and a spare slot would make the stride even (for RA = 15,
    // every thread of a warp on the same bank), so odd RA is not padded.
    // PADN (the tile size) is the padded bound either way.
    static constexpr int PK = (RA % 2 == 0) ? 1 : 0;
    static constexpr int PADN = N + N / RA + 1;
    static __device__ __forceinline__ int pad(int idx) { return idx + PK * (idx / RA); }
};

// Twiddles of one Stockham stage for butterfly index j: W^r with
// W = W_{NS*R}^{j mod NS}, r = 1 .. R-1.  One value comes from the length-N
// table; the other powers are products of it (squarings for even r), at most
// six products deep, so the twiddles cost one load per stage instead of R-1
// (with most of shared memory in use, the table does not stay in L1).
template <int N, int NS, int R>
__device__ __forceinline__ void stage_twiddles(float2 (&w)[R], int j, const float2 *__restrict__ tw)
{
    constexpr int step = N / (NS * R);
    const int u = (j % NS) * step;
    if constexpr (R > 1) w[1] = __ldg(&tw[u]);
#pragma unroll
    for (int r = 2; r < R; ++r) w[r] = (r % 2 == 0) ? cmul(w[r / 2], w[r / 2]) : cmul(w[r - 1], w[1]);
}
// the table value stage_twiddles loads (for callers that keep it in a register)
template <int N, int NS, int R>
__device__ __forceinline__ float2 stage_twiddle_base(int j, const float2 *__restrict__ tw)
{
    constexpr int step = N / (NS * R);
    return __ldg(&tw[(j % NS) * step]);
}
// stage_twiddles from that value
template <int R>
__device__ __forceinline__ void stage_twiddles_from(float2 (&w)[R], float2 b)
{
    if constexpr (R > 1) w[1] = b;
#pragma unroll
    for (int r = 2; r < R; ++r) w[r] = (r % 2 == 0) ? cmul(w[r / 2], w[r / 2]) : cmul(w[r - 1], w[1]);
}

// one Stockham butterfly on Q rows that share the butterfly index:
// v[q][r] = x_q[j + r*N/R] on entry, multiplied by the stage twiddles w[r]
// (unless NS == 1) and transformed; output r belongs at
// (j/NS)*NS*R + j%NS + r*NS.
template <int NS, int R, int DIR, int Q>
__device__ __forceinline__ void butterfly(float2 (&v)[Q][R], const float2 (&w)[R])
{
    if constexpr (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r)
#pragma unroll
            for (int q = 0; q < Q; ++q) v[q][r] = (DIR < 0) ? cmul(v[q][r], w[r]) : cmulc(v[q][r], w[r]);
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) Dft<R, DIR>::run(v[q]);
}

// Full line transform of Q rows per thread.  On entry thread t (< N/RA)
// holds its first-stage inputs v[q][r] = x_q[t + r*N/RA].  On exit thread t
// (< N/RL) holds o[q][r] = X_q[t + r*N/RL].  smem(q, i) is row q's exchange
// slot for padded index i (RD::pad); every index a thread touches in a stage
// is its base plus a compile-time multiple, so addressing is one add per
// access.  Contains __syncthreads(): call uniformly from the whole block; the
// exchange tiles may be reused by the caller only after another barrier.
// PREF: load each stage's twiddles before the barrier that precedes the
// stage (hides their latency; costs registers across the barrier).
// PP (ping-pong): stage 2 writes a second exchange tile, smem2, so that no
// barrier is needed between its reads and its writes; stage 3 reads smem2.
// HOIST: the stage twiddles come from tb2 / tb3 (stage_twiddle_base of
// stages 2 and 3 for this thread, kept by the caller) instead of the table
// PAD2: the second exchange (stage-2 writes in runs of RA, stage-3
// unit-stride reads) is padded like the first; without it its reads are
// conflict-free.  Measured: unpadded is faster for the x pass (one line per
// thread row), padded for the y pass (four lines interleaved).
template <class RD, int DIR, int Q, bool PREF, bool PP, class SM, class SM2, bool HOIST = false, bool PAD2 = true>
__device__ __forceinline__ void line_fft_impl(float2 (&v)[Q][RD::RA], float2 (&o)[Q][RD::RL], int t,
                                              const float2 *__restrict__ tw, SM smem, SM2 smem2,
                                              float2 tb2 = float2{}, float2 tb3 = float2{});

template <class RD, int DIR, int Q, bool PREF = false, bool PAD2 = true, class SM>
__device__ __forceinline__ void line_fft(float2 (&v)[Q][RD::RA], float2 (&o)[Q][RD::RL], int t,
                                         const float2 *__restrict__ tw, SM smem)
{
    line_fft_impl<RD, DIR, Q, PREF, false, SM, SM, false, PAD2>(v, o, t, tw, smem, smem);
}

template <class RD, int DIR, int Q, bool PREF, bool PP, class SM, class SM2, bool HOIST, bool PAD2>
__device__ __forceinline__ void line_fft_impl(float2 (&v)[Q][RD::RA], float2 (&o)[Q][RD::RL], int t,
                                              const float2 *__restrict__ tw, SM smem, SM2 smem2, float2 tb2,
                                              float2 tb3)
{
    constexpr int P2 = PAD2 ? RD::PK : 0;  // padding of the second exchange
    constexpr int N = RD::N, RA = RD::RA, RB = RD::RB, RC = RD::RC;
    constexpr int M2 = N / RB;  // stage-2 butterflies; read stride, a multiple of RA
    // stage 1 writes t*RA + r  ->  padded t*(RA+PK) + r
    if (t < N / RA) {
        float2 none[RA];
        butterfly<1, RA, DIR, Q>(v, none);
        const int b1 = t * (RA + RD::PK);
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int r = 0; r < RA; ++r) *smem(q, b1 + r) = v[q][r];
    }
    float2 w2[RB];
    if (PREF && t < M2) stage_twiddles<N, RA, RB>(w2, t, tw);
    __syncthreads();
    if constexpr (RD::THREE) {
        constexpr int M3 = N / RC;
        float2 u[Q][RB];
        if (t < M2) {
            const int b2 = RD::pad(t);
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int r = 0; r < RB; ++r) u[q][r] = *smem(q, b2 + r * (M2 + RD::PK * (M2 / RA)));
        }
        if constexpr (!PP) __syncthreads();
        if (t < M2) {
            if constexpr (HOIST) stage_twiddles_from<RB>(w2, tb2);
            else if (!PREF) stage_twiddles<N, RA, RB>(w2, t, tw);
            butterfly<RA, RB, DIR, Q>(u, w2);
            const int base = (t / RA) * RA * RB + t % RA;  // writes base + r*RA
            const int b3 = base + P2 * (base / RA);
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int r = 0; r < RB; ++r) *smem2(q, b3 + r * (RA + P2)) = u[q][r];
        }
        float2 w3[RC];
        if (PREF && t < M3) stage_twiddles<N, RA * RB, RC>(w3, t, tw);
        __syncthreads();
        if (t < M3) {
            const int b4 = t + P2 * (t / RA);
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int r = 0; r < RC; ++r) o[q][r] = *smem2(q, b4 + r * (M3 + P2 * (M3 / RA)));
            if constexpr (HOIST) stage_twiddles_from<RC>(w3, tb3);
            else if (!PREF) stage_twiddles<N, RA * RB, RC>(w3, t, tw);
            butterfly<RA * RB, RC, DIR, Q>(o, w3);
        }
    } else {
        if (t < M2) {
            const int b2 = RD::pad(t);
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int r = 0; r < RB; ++r) o[q][r] = *smem(q, b2 + r * (M2 + RD::PK * (M2 / RA)));
            if constexpr (HOIST) stage_twiddles_from<RB>(w2, tb2);
            else if (!PREF) stage_twiddles<N, RA, RB>(w2, t, tw);
            butterfly<RA, RB, DIR, Q>(o, w2);
        }
    }
}

template <class RD>
using RevRad = Rad<(RD::THREE ? RD::RC : RD::RB), (RD::THREE ? RD::RB : RD::RA), (RD::THREE ? RD::RA : 1)>;

// ------------------------------------------------------------ k_lines

enum LinesMode { LINES_FWD = 0, LINES_INV = 1, LINES_CONV = 2, LINES_CONV_CONJ = 3 };

struct LinesArgs {
    float2 *data;            // spectrum
    const float2 *otf;       // OTF, same layout as data (convolve modes)
    const float2 *tw;        // tw[m] = exp(-2 pi i m / N), m < N
    long long line_stride;   // complex elements between neighbours on a line
    long long outer_stride;  // complex elements between outer blocks
    int ncols;               // adjacent lines (contiguous columns) per outer block
    int ntiles;              // ceil(ncols / T)
    int mode;
    int nin;                 // elements [0, nin) of a line are read; the rest are zero
    int nout;                // elements [0, nout) of a line are written
    // planes mode (a job split by z planes over GPUs): element n of column c
    // is planes[n][col0 + c], plane n on whichever GPU holds it (peer
    // loads and stores); `data` is unused and `line_stride` is the OTF's
    float2 *const *planes = nullptr;
    long long col0 = 0;
};

template <class RD, int T>
struct LinesCfg {
    static constexpr int THREADS = T * cmax(RD::TPL, RevRad<RD>::TPL);
    // exchange tile, then (convolve modes) the OTF tile, prefetched at entry
    static constexpr int XCH_F2 = cmax(RD::PADN, RevRad<RD>::PADN) * T;
    static constexpr size_t SMEM_FFT = sizeof(float2) * (size_t) XCH_F2;
    static constexpr size_t SMEM_BYTES = SMEM_FFT + sizeof(float2) * (size_t) RD::N * T;
    // as many resident CTAs (up to four) as leave at least 64 registers a thread
    static constexpr int MIN_BLOCKS =
        (THREADS * 4 <= 1024 && SMEM_BYTES * 4 <= 225 * 1024) ? 4
        : (THREADS * 3 <= 1024 && SMEM_BYTES * 3 <= 225 * 1024) ? 3
        : (THREADS * 2 <= 1024 && SMEM_BYTES * 2 <= 225 * 1024) ? 2 : 1;
};

template <class RD, int T, bool PL = false>
__global__ void __launch_bounds__(LinesCfg<RD, T>::THREADS, LinesCfg<RD, T>::MIN_BLOCKS)
k_lines(LinesArgs a)
{
    using RV = RevRad<RD>;
    constexpr int N = RD::N;
    extern __shared__ float2 sm[];
    const int line = threadIdx.x;
    const int t = threadIdx.y;
    const int tile = blockIdx.x % a.ntiles;
    const long long outer = blockIdx.x / a.ntiles;
    const int col = tile * T + line;
    const bool valid = col < a.ncols;
    const long long off = outer * a.outer_stride + col;
    float2 *base = a.data + off;
    const long long ls = a.line_stride;
    // element n of this thread's line
    auto elem = [&](int n) -> float2 * {
        if constexpr (PL)
            return a.planes[n] + (a.col0 + col);
        else
            return base + (long long) n * ls;
    };
    const int mode = a.mode;
    auto smem = [&](int, int i) { return sm + (size_t) i * T + line; };
    using Cfg = LinesCfg<RD, T>;
    float2 *sotf = sm + Cfg::XCH_F2;  // OTF tile [n][col] (convolve modes)
    const int col0 = tile * T;
    if (mode >= LINES_CONV && (T % 2) == 0) {
        // the tile's OTF columns arrive while the forward transform runs:
        // 16-byte pieces (two columns) of each of the N rows
        const int tid = t * T + line;
        const float2 *h0 = a.otf + outer * a.outer_stride + col0;
        constexpr int PPR = T / 2;  // pieces per row
        for (int e = tid; e < N * PPR; e += Cfg::THREADS) {
            const int n = e / PPR, p = e - n * PPR;
            if (col0 + 2 * p < a.ncols) cp_async16(sotf + n * T + 2 * p, h0 + (long long) n * ls + 2 * p);
        }
        cp_async_commit();
    }

    float2 v[1][RD::RA];
    if (t < N / RD::RA) {
#pragma unroll
        for (int r = 0; r < RD::RA; ++r) {
            const int n = t + r * (N / RD::RA);
            v[0][r] = (valid && n < a.nin) ? *elem(n) : make_float2(0.f, 0.f);
        }
    }
    float2 o[1][RD::RL];
    if (mode == LINES_INV)
        line_fft<RD, +1, 1>(v, o, t, a.tw, smem);
    else
        line_fft<RD, -1, 1>(v, o, t, a.tw, smem);
    constexpr int SL = N / RD::RL;
    if (mode == LINES_FWD || mode == LINES_INV) {
        if (t < SL && valid) {
#pragma unroll
            for (int r = 0; r < RD::RL; ++r)
                if (t + r * SL < a.nout) *elem(t + r * SL) = o[0][r];
        }
        return;
    }
    // multiply by the OTF (conjugated for the back-projection)
    if constexpr ((T % 2) == 0) {
        cp_async_wait_all();
        __syncthreads();  // every thread's pieces of the OTF tile have landed
        if (t < SL && valid) {
#pragma unroll
            for (int r = 0; r < RD::RL; ++r) {
                const float2 q = sotf[(t + r * SL) * T + line];
                o[0][r] = (mode == LINES_CONV) ? cmul(o[0][r], q) : cmulc(o[0][r], q);
            }
        }
    } else if (t < SL && valid) {
        const float2 *h = a.otf + off;
#pragma unroll
        for (int r = 0; r < RD::RL; ++r) {
            float2 q = __ldg(&h[(long long) (t + r * SL) * ls]);
            o[0][r] = (mode == LINES_CONV) ? cmul(o[0][r], q) : cmulc(o[0][r], q);
        }
    }
    __syncthreads();  // the exchange tile is free again
    float2 q[1][RV::RL];
    line_fft<RV, +1, 1>(o, q, t, a.tw, smem);
    constexpr int SQ = N / RV::RL;
    if (t < SQ && valid) {
#pragma unroll
        for (int r = 0; r < RV::RL; ++r)
            if (t + r * SQ < a.nout) *elem(t + r * SQ) = q[0][r];
    }
}

// ------------------------------------------------------------ spectrum layout
//
// The half-spectrum (kx < X/2+1) is stored blocked by KB = 4 along kx:
//   element (kx, y, z) at  ((z * nkb + kx / KB) * Y + y) * KB + kx % KB
// (nkb = ceil((X/2+1) / KB)).  A y line group (4 neighbouring kx) is then one
// contiguous Y*32-byte block, a z line is strided by the plane size, and the
// two rows y, y+1 of one kx block are 64 contiguous bytes for the x pass.
constexpr int KB = 4;

// ------------------------------------------------------------ k_ypass

struct YArgs {
    float2 *data;
    const float2 *tw;   // tw[m] = exp(-2 pi i m / Y)
    int *err;           // error flags (bounded waits)
    int ntiles;         // Z * nkb
    int dir;            // -1 forward, +1 inverse
};

template <class RD>
struct YCfg {
    static constexpr int Q = 1;                  // lines per thread
    static constexpr int TX = KB / Q;            // threads across the 4 lines
    static constexpr int THREADS = TX * RD::TPL;
    static constexpr int BUF_F2 = RD::PADN * KB;
    // two tile buffers (the next tile's copy lands in one while the other is
    // transformed) and, where it fits, a third exchange tile so that the
    // transform's stages need fewer barriers (line_fft_impl, PP)
    static constexpr bool PP = 3 * sizeof(float2) * (size_t) BUF_F2 + 64 <= 227 * 1024;
    static constexpr size_t SMEM_BYTES = (PP ? 3 : 2) * sizeof(float2) * (size_t) BUF_F2 + 64;
    static constexpr uint32_t TILE_BYTES = (uint32_t) (RD::N * KB * sizeof(float2));
};

// Persistent y transform: one CTA loops over (z, kx-block) tiles; each tile
// (4 lines of length Y, contiguous) arrives by one bulk copy, the next
// tile's copy is in flight while this one is transformed.
template <class RD, int DIR>
__global__ void __launch_bounds__(YCfg<RD>::THREADS)
k_ypass(YArgs a)
{
    using C = YCfg<RD>;
    constexpr int N = RD::N;
    constexpr int Q = C::Q;
    extern __shared__ __align__(128) unsigned char ysm[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(ysm);
    float2 *bufs = reinterpret_cast<float2 *>(ysm + 64);
    const int l0 = threadIdx.x * Q;  // this thread's first line in the tile
    const int t = threadIdx.y;
    const int tid = t * C::TX + threadIdx.x;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    // this thread's stage twiddle values are the same for every tile
    const float2 tb2 = stage_twiddle_base<N, RD::RA, RD::RB>(t < N / RD::RB ? t : 0, a.tw);
    const float2 tb3 = RD::THREE ? stage_twiddle_base<N, RD::RA * RD::RB, (RD::THREE ? RD::RC : 1)>(
                                       t < N / (RD::THREE ? RD::RC : 1) ? t : 0, a.tw)
                                 : make_float2(1.f, 0.f);
    int tile = blockIdx.x;
    if (tid == 0 && tile < a.ntiles) {
        mbar_arrive_expect_tx(&bars[0], C::TILE_BYTES);
        tma_load_1d(bufs, a.data + (size_t) tile * N * KB, C::TILE_BYTES, &bars[0]);
    }
    for (int it = 0; tile < a.ntiles; ++it, tile += gridDim.x) {
        const int b = it & 1;
        float2 *buf = bufs + (size_t) b * C::BUF_F2;
        fence_proxy_async();  // this thread's accesses to the other buffer precede the next bulk copy into it
        __syncthreads();      // the other buffer is no longer read
        const int next = tile + gridDim.x;
        if (tid == 0 && next < a.ntiles) {
            fence_proxy_async();
            mbar_arrive_expect_tx(&bars[b ^ 1], C::TILE_BYTES);
            tma_load_1d(bufs + (size_t) (b ^ 1) * C::BUF_F2, a.data + (size_t) next * N * KB, C::TILE_BYTES,
                        &bars[b ^ 1]);
        }
        if (!wait_all(&bars[b], (it >> 1) & 1, a.err, 1 << 8)) {
            if (tid == 0 && next < a.ntiles) drain(&bars[b ^ 1], ((it + 1) >> 1) & 1);
            return;
        }
        float2 v[Q][RD::RA];
        if (t < N / RD::RA) {
#pragma unroll
            for (int r = 0; r < RD::RA; ++r)
#pragma unroll
                for (int q = 0; q < Q; ++q) v[q][r] = buf[(t + r * (N / RD::RA)) * KB + l0 + q];
        }
        auto smem = [&](int q, int i) { return buf + (size_t) i * KB + l0 + q; };
        float2 o[Q][RD::RL];
        if constexpr (C::PP) {
            // stage 1 writes the third tile (no barrier after the natural-order
            // reads), stage 2 writes the tile buffer back
            float2 *ex = bufs + (size_t) 2 * C::BUF_F2;
            auto smemx = [&](int q, int i) { return ex + (size_t) i * KB + l0 + q; };
            line_fft_impl<RD, DIR, Q, false, true, decltype(smemx), decltype(smem), true>(v, o, t, a.tw, smemx,
                                                                                          smem, tb2, tb3);
        } else {
            __syncthreads();  // natural-order reads done; the buffer becomes the exchange tile
            line_fft<RD, DIR, Q>(v, o, t, a.tw, smem);
        }
        constexpr int SL = N / RD::RL;
        if (t < SL) {
            float2 *dst = a.data + (size_t) tile * N * KB + l0;
#pragma unroll
            for (int r = 0; r < RD::RL; ++r)
#pragma unroll
                for (int q = 0; q < Q; ++q) dst[(size_t) (t + r * SL) * KB + q] = o[q][r];
        }
    }
}

// ------------------------------------------------------------ k_xpass

enum XOp {
    XOP_FWD_COPY = 0,    // src real volume -> R2C
    XOP_FWD_ONES = 1,    // 1 on the image region, 0 elsewhere -> R2C
    XOP_FWD_SHBP = 2,    // p = max(x + a(x - xp), bg) -> R2C
    XOP_RATIO_SHB = 3,   // C2R -> error partial -> ratio (SHB guard) -> R2C
    XOP_RATIO_RL = 4,    // C2R -> error partial -> ratio (RL guard) -> R2C
    XOP_ERROR_ONLY = 5,  // C2R -> error partial
    XOP_UPDATE_SHB = 6,  // C2R -> x' = clamp(t * (p*W)), store -> [p' -> R2C]
    XOP_UPDATE_RL = 7,   // C2R -> x' = clamp(t * (x*W)), store -> [x' -> R2C]
    XOP_WEIGHTS = 8,     // C2R -> W = P1 > 0.01 ? 1/P1 : 0, store
    XOP_STORE = 9,       // C2R -> store real
};

struct JobScalars {
    float bg;        // background level (auto: max(min(g), 0.01))
    float x0;        // flat start value
    double sumg;     // sum of the image in double
    float gmin;
    int flags;       // bit 0/1: non-finite image/PSF; bits 8+: bounded waits that gave up
};

struct XArgs {
    float2 *S;             // spectrum (blocked layout)
    const float2 *tw;      // tw[m] = exp(-2 pi i m / X), m < X (Hermitian pre/post)
    const float2 *twL;     // twL[m] = exp(-2 pi i m / L), m < L (stage twiddles)
    const float *g;        // image, row pitch GP
    const float *src;      // FWD_COPY source / x_k for SHB and RL
    const float *srcp;     // x_{k-1} for SHB
    const float *Wt;       // Bertero weights (may be null)
    float *dst;            // real output (UPDATE: x_{k+1}; WEIGHTS/STORE)
    double *partial;       // per-tile error partials (ops with an error)
    const JobScalars *sc;  // bg, ...
    int *err;              // error flags (bounded waits)
    long long X;           // real row pitch (= real length), multiple of 4
    long long GP;          // image row pitch, multiple of 4
    int Y, Z;              // padded dims
    int M, N, P;           // image dims
    int nkb;               // kx blocks
    int ntiles;            // Z * ceil(Y / R)
    int op;
    int r2c;               // run the forward transform after the op
    int metric;            // 1: I-divergence, 0: squared error
    int positivity;        // SHB: clamp x' at bg
    int rl_clamp;          // RL: clamp x' at bg when bg > 0
    double alpha;          // SHB extrapolation weight of the step being finished
    double alpha_next;     // SHB extrapolation weight of the next step
    // periodic x (wrapx): the row is wM-periodic; before the forward
    // transform, [wM, wM+hx) and [X-hx, X) take copies of [0, hx) and
    // [wM-hx, wM), the rest of [wM, X) is zero
    int wrapx, wM, hx;
};

// The x transform of a real row of X = 2L samples uses a complex transform
// of length L = RD::N: z[n] = x[2n] + i x[2n+1].  The inverse runs with RD,
// the forward with the reversed radix list.  One CTA = one tile of R
// consecutive rows (y0 .. y0+R-1 at one z).  At entry the CTA issues bulk
// copies of its complex rows (the 64-byte kx blocks of the spectrum layout)
// and, on a second barrier, of its real rows; the real rows arrive while the
// inverse transform runs.  Three CTAs share an SM, so one CTA's copies
// overlap the others' arithmetic.
// real slots a family stages: forward: x, x_{k-1}; ratio: the image rows;
// update: x, x_{k-1}, W; C2R-store: none
__host__ __device__ constexpr int x_slots(int fam) { return fam == 0 ? 2 : fam == 1 ? 1 : fam == 2 ? 3 : 0; }

template <class RD, int R, int FAM = 2>
struct XCfg {
    using RV = RevRad<RD>;
    static constexpr int Q = 1;                     // rows per thread
    static constexpr int RY = R / Q;                // thread rows of the block
    static constexpr int L = RD::N;
    static constexpr int X = 2 * L;
    static constexpr int XP = (X + 3) / 4 * 4;  // real row pitch (16-byte rows for bulk copies)
    static constexpr int NKB = (L + 1 + KB - 1) / KB;
    static constexpr int TPL = cmax(RD::TPL, RV::TPL);
    static constexpr int THREADS = RY * TPL;
    static constexpr int ROW_F2 = cmax(cmax(L + 1, RD::PADN), RV::PADN) | 1;
    static constexpr int CPLX_F2 = R * NKB * KB;                  // staged rows, [kb][r][ki]
    // complex area (also the exchange tiles), rounded to 16 bytes
    static constexpr int AREA_F2 = (cmax(CPLX_F2, R * ROW_F2) + 1) / 2 * 2;
    static constexpr int REAL_F = R * XP;                         // one staged real array
    // complex area and three real slots: x (or the image rows g, which no op
    // reads together with x), xp, W
    static constexpr size_t REAL_OFF = 64 + sizeof(float2) * (size_t) AREA_F2;
    // the real slots are also the forward transform's second exchange tile
    // (read by the pointwise op before it), so they hold R padded rows
    static constexpr size_t SLOT_BYTES = x_slots(FAM) * sizeof(float) * (size_t) REAL_F;
    static constexpr size_t XCH2_BYTES = FAM == 3 ? 0 : sizeof(float2) * (size_t) (R * ROW_F2);
    static constexpr size_t REAL_BYTES = SLOT_BYTES > XCH2_BYTES ? SLOT_BYTES : XCH2_BYTES;
    static constexpr size_t RED_OFF = REAL_OFF + (REAL_BYTES + 7) / 8 * 8;
    // the error partials' reduction area: ratio family only
    static constexpr size_t SMEM_BYTES = RED_OFF + (FAM == 1 ? sizeof(double) * THREADS : 0);
    // resident CTAs per SM to aim for (registers are capped to fit them):
    // one-row update tiles of at most five warps take six where their shared
    // memory (plus the 1 KB the hardware reserves per block) fits, which
    // leaves 64 registers a thread (x 2240: no spills; 4.80 -> 4.65 ms per
    // update pass against five), else five
    static constexpr int MIN_BLOCKS =
        (R == 1 && FAM == 2 && THREADS <= 160 && (SMEM_BYTES + 1024) * 6 <= 228 * 1024) ? 6
        : (R == 1 && FAM == 2 && SMEM_BYTES * 5 <= 224 * 1024 && THREADS * 5 <= 2048) ? 5
                                    : (SMEM_BYTES * 4 <= 224 * 1024 && THREADS * 4 <= 2048) ? 4
                                    : (SMEM_BYTES * 3 <= 225 * 1024 && THREADS * 3 <= 2048) ? 3 : 1;
    static_assert(R % Q == 0, "rows per tile");
    static_assert(THREADS >= 32, "the error reduction needs one full warp");
};

__device__ __forceinline__ float shb_p(float xv, float xpv, double alpha, float bg)
{
    // method_shb.c:337-338: p = x + alpha*(x - xp) in double, stored as float; p < bg -> bg
    float p = (float) ((double) xv + alpha * (double) (xv - xpv));
    return p < bg ? bg : p;
}

__device__ __forceinline__ double err_term(float yv, float gv, int metric)
{
    double y = yv, g = gv;
    if (metric == 0) return (y - g) * (y - g);
    // dw.c:1514-1517: g*logf(g/y) - (g - y) for y > 0 and g > 0.  The
    // reference divides in double and rounds to float for logf; the float
    // division gives the same float except in double-rounding ties.
    if (yv > 0.f && gv > 0.f) return g * (double) logf(gv / yv) - (g - y);
    return 0.0;
}

// ops are compiled in four families, one kernel each, so that every kernel's
// code stays small: forward-only, ratio/error, update, and C2R-store ops
enum XFam { XFAM_FWD = 0, XFAM_RATIO = 1, XFAM_UPDATE = 2, XFAM_STORE = 3 };
__host__ __device__ constexpr int x_family(int op)
{
    return op <= XOP_FWD_SHBP ? XFAM_FWD
         : op <= XOP_ERROR_ONLY ? XFAM_RATIO
         : op <= XOP_UPDATE_RL ? XFAM_UPDATE : XFAM_STORE;
}

__device__ __forceinline__ bool op_c2r(int op) { return op >= XOP_RATIO_SHB; }

// err_term with the quotient g/y already computed (q is only read when
// y > 0 and g > 0, where it equals g/y)
__device__ __forceinline__ double err_term_q(float yv, float gv, float q, int metric)
{
    const double y = yv, g = gv;
    if (metric == 0) return (y - g) * (y - g);
    if (yv > 0.f && gv > 0.f) return g * (double) logf(q) - (g - y);
    return 0.0;
}
__device__ __forceinline__ bool op_reads_x(int op)
{
    return op == XOP_FWD_COPY || op == XOP_FWD_SHBP || op == XOP_UPDATE_SHB || op == XOP_UPDATE_RL;
}
__device__ __forceinline__ bool op_reads_xp(int op) { return op == XOP_FWD_SHBP || op == XOP_UPDATE_SHB; }
__device__ __forceinline__ bool op_reads_g(int op) { return op >= XOP_RATIO_SHB && op <= XOP_ERROR_ONLY; }

// The pointwise op of one row: w[r] holds z[n] = (x[2n], x[2n+1]) for
// n = t + r*SL -- the C2R output for the C2R ops -- and is replaced by the
// values handed to the forward transform.  The row's real inputs are staged
// in shared memory (sx: x or the image row, sxp: x_{k-1}, sw: weights).
// The switch is outside the element loop so each op is one straight loop.
template <int FAM, int RL, int SL>
__device__ __forceinline__ void x_row_op(const XArgs &a, int op, int t, long long rbase, const float *sx,
                                         const float *sxp, const float *sw, bool in_img_row, float bg,
                                         float2 (&w)[RL], double &acc)
{
    const int M = a.M;
    // only this family's cases are compiled into the kernel
    if (x_family(op) != FAM) return;
    switch (op) {
    case XOP_FWD_COPY:
        if constexpr (FAM == XFAM_FWD) {
#pragma unroll
            for (int r = 0; r < RL; ++r) w[r] = *reinterpret_cast<const float2 *>(sx + 2 * (t + r * SL));
        }
        break;
    case XOP_FWD_ONES:  // initial_guess, dw.c:2497-2520
        if constexpr (FAM == XFAM_FWD) {
#pragma unroll
            for (int r = 0; r < RL; ++r) {
                const int c0 = 2 * (t + r * SL);
                w[r] = make_float2(in_img_row && c0 < M ? 1.f : 0.f, in_img_row && c0 + 1 < M ? 1.f : 0.f);
            }
        }
        break;
    case XOP_FWD_SHBP:
        if constexpr (FAM == XFAM_FWD) {
#pragma unroll
            for (int r = 0; r < RL; ++r) {
                const int c0 = 2 * (t + r * SL);
                const float2 xv = *reinterpret_cast<const float2 *>(sx + c0);
                const float2 xq = *reinterpret_cast<const float2 *>(sxp + c0);
                w[r] = make_float2(shb_p(xv.x, xq.x, a.alpha, bg), shb_p(xv.y, xq.y, a.alpha, bg));
            }
        }
        break;
    case XOP_RATIO_SHB:
        if constexpr (FAM != XFAM_RATIO) break;
#pragma unroll
        for (int r = 0; r < RL; ++r) {
            const int c0 = 2 * (t + r * SL);
            const bool img0 = in_img_row && c0 < M;
            const bool img1 = in_img_row && c0 + 1 < M;
            const float y0 = w[r].x, y1 = w[r].y;
            const float g0 = img0 ? sx[c0] : 0.f;
            const float g1 = img1 ? sx[c0 + 1] : 0.f;
            // method_shb.c:31-48: |y| < 1e-6 -> +-1e-6; r = g/y on the image, 0 elsewhere.
            // (double)|y| < 1e-6 holds exactly when |y| <= 1e-6f, the float just below 1e-6.
            const float d0 = fabsf(y0) <= 1e-6f ? copysignf(1e-6f, y0) : y0;
            const float d1 = fabsf(y1) <= 1e-6f ? copysignf(1e-6f, y1) : y1;
            const float v0 = img0 ? g0 / d0 : 0.f;
            const float v1 = img1 ? g1 / d1 : 0.f;
            // the error's g/y is the same quotient unless the guard changed y
            // (a branch, so that the second division runs only then)
            float q0 = v0, q1 = v1;
            if (d0 != y0) q0 = g0 / y0;
            if (d1 != y1) q1 = g1 / y1;
            if (img0) acc += err_term_q(y0, g0, q0, a.metric);
            if (img1) acc += err_term_q(y1, g1, q1, a.metric);
            w[r] = make_float2(v0, v1);
        }
        break;
    case XOP_RATIO_RL:
        if constexpr (FAM != XFAM_RATIO) break;
#pragma unroll
        for (int r = 0; r < RL; ++r) {
            const int c0 = 2 * (t + r * SL);
            const bool img0 = in_img_row && c0 < M;
            const bool img1 = in_img_row && c0 + 1 < M;
            const float y0 = w[r].x, y1 = w[r].y;
            const float g0 = img0 ? sx[c0] : 0.f;
            const float g1 = img1 ? sx[c0 + 1] : 0.f;
            // method_rl.c:46-67: r = g/y if y > 0 else bg on the image, 1e-6 elsewhere
            const float v0 = img0 ? (y0 > 0.f ? g0 / y0 : bg) : 1e-6f;
            const float v1 = img1 ? (y1 > 0.f ? g1 / y1 : bg) : 1e-6f;
            if (img0) acc += err_term_q(y0, g0, v0, a.metric);  // q used only when y > 0
            if (img1) acc += err_term_q(y1, g1, v1, a.metric);
            w[r] = make_float2(v0, v1);
        }
        break;
    case XOP_ERROR_ONLY:
        if constexpr (FAM != XFAM_RATIO) break;
#pragma unroll
        for (int r = 0; r < RL; ++r) {
            const int c0 = 2 * (t + r * SL);
            const bool img0 = in_img_row && c0 < M;
            const bool img1 = in_img_row && c0 + 1 < M;
            const float y0 = w[r].x, y1 = w[r].y;
            const float g0 = img0 ? sx[c0] : 0.f;
            const float g1 = img1 ? sx[c0 + 1] : 0.f;
            if (img0) acc += err_term_q(y0, g0, y0 > 0.f ? g0 / y0 : 0.f, a.metric);
            if (img1) acc += err_term_q(y1, g1, y1 > 0.f ? g1 / y1 : 0.f, a.metric);
        }
        break;
    case XOP_UPDATE_SHB:
        // method_shb.c:56-62 (x = Kt r * (p*W)), :366-376 (positivity), and the
        // next extrapolation :333-339; p_k is recomputed from x_k, x_{k-1}
        if constexpr (FAM != XFAM_UPDATE) break;
#pragma unroll
        for (int r = 0; r < RL; ++r) {
            const int c0 = 2 * (t + r * SL);
            const float2 xv = *reinterpret_cast<const float2 *>(sx + c0);
            const float2 xq = *reinterpret_cast<const float2 *>(sxp + c0);
            const float p0 = shb_p(xv.x, xq.x, a.alpha, bg);
            const float p1 = shb_p(xv.y, xq.y, a.alpha, bg);
            float n0, n1;
            if (sw) {
                const float2 ww = *reinterpret_cast<const float2 *>(sw + c0);
                n0 = w[r].x * (p0 * ww.x);
                n1 = w[r].y * (p1 * ww.y);
            } else {
                n0 = w[r].x * p0;
                n1 = w[r].y * p1;
            }
            if (a.positivity) {
                n0 = n0 < bg ? bg : n0;
                n1 = n1 < bg ? bg : n1;
            }
            *reinterpret_cast<float2 *>(a.dst + rbase + c0) = make_float2(n0, n1);
            w[r] = make_float2(shb_p(n0, xv.x, a.alpha_next, bg), shb_p(n1, xv.y, a.alpha_next, bg));
        }
        break;
    case XOP_UPDATE_RL:
        // method_rl.c:84-98 and :362-372
        if constexpr (FAM != XFAM_UPDATE) break;
#pragma unroll
        for (int r = 0; r < RL; ++r) {
            const int c0 = 2 * (t + r * SL);
            const float2 xv = *reinterpret_cast<const float2 *>(sx + c0);
            float n0, n1;
            if (sw) {
                const float2 ww = *reinterpret_cast<const float2 *>(sw + c0);
                n0 = w[r].x * (xv.x * ww.x);
                n1 = w[r].y * (xv.y * ww.y);
            } else {
                n0 = w[r].x * xv.x;
                n1 = w[r].y * xv.y;
            }
            if (a.rl_clamp && bg > 0.f) {
                n0 = n0 < bg ? bg : n0;
                n1 = n1 < bg ? bg : n1;
            }
            *reinterpret_cast<float2 *>(a.dst + rbase + c0) = make_float2(n0, n1);
            w[r] = make_float2(n0, n1);
        }
        break;
    case XOP_WEIGHTS:
        // method_shb.c:224-234: W = 1/P1 where P1 > 0.01, else 0
        if constexpr (FAM != XFAM_STORE) break;
#pragma unroll
        for (int r = 0; r < RL; ++r) {
            const int c0 = 2 * (t + r * SL);
            const float q0 = w[r].x > 0.01f ? (float) (1.0 / (double) w[r].x) : 0.f;
            const float q1 = w[r].y > 0.01f ? (float) (1.0 / (double) w[r].y) : 0.f;
            *reinterpret_cast<float2 *>(a.dst + rbase + c0) = make_float2(q0, q1);
        }
        break;
    case XOP_STORE:
        if constexpr (FAM == XFAM_STORE) {
#pragma unroll
            for (int r = 0; r < RL; ++r) *reinterpret_cast<float2 *>(a.dst + rbase + 2 * (t + r * SL)) = w[r];
        }
        break;
    default:
        break;
    }
}

template <class RD, int R, int FAM>
__global__ void __launch_bounds__(XCfg<RD, R, FAM>::THREADS, XCfg<RD, R, FAM>::MIN_BLOCKS)
k_xpass(XArgs a)
{
    using C = XCfg<RD, R, FAM>;
    using RV = typename C::RV;
    // twiddles loaded ahead of the barriers cost registers across them; the
    // ratio family (four CTAs per SM, few registers) loads them in place
    constexpr bool PREF_TW = (FAM != XFAM_RATIO);
    constexpr int L = C::L;
    constexpr int Q = C::Q;
    constexpr int XP = C::XP;       // real row pitch (a.X == XP)
    constexpr int SL = L / RD::RL;  // op phase: thread t < SL holds n = t + r*SL
    static_assert(RV::RA == RD::RL, "reversed radix list");
    extern __shared__ __align__(128) unsigned char xsm[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(xsm);  // [1]: real rows
    float2 *CB = reinterpret_cast<float2 *>(xsm + 64);
    float *RB = reinterpret_cast<float *>(xsm + C::REAL_OFF);
    double *red = reinterpret_cast<double *>(xsm + C::RED_OFF);
    const int t = threadIdx.x;
    const int ry = threadIdx.y;
    const int tid = ry * C::TPL + t;
    const int op = a.op;
    constexpr bool c2r = (FAM != XFAM_FWD);
    const bool rx = op_reads_x(op), rxp = op_reads_xp(op), rw = rx && (op >= XOP_UPDATE_SHB) && a.Wt != nullptr;
    constexpr bool rg = (FAM == XFAM_RATIO);
    const int ytiles = (a.Y + R - 1) / R;
    const long long plane = (long long) a.nkb * a.Y * KB;  // complex elements per z plane
    const int tile = blockIdx.x;
    const int z = tile / ytiles;
    const int y0 = (tile - z * ytiles) * R;

    if constexpr (FAM == XFAM_RATIO) {
        // (with a periodic x, RL's constant row is not constant over the
        // transform length: such rows take the general path)
        if ((z >= a.P || y0 >= a.N) && !(a.wrapx && op == XOP_RATIO_RL)) {
            // No image row in this tile: the ratio is the same constant on
            // every row (0 for SHB, method_shb.c:44-46; 1e-6 for RL,
            // method_rl.c:62-64) and the rows add nothing to the error, so
            // neither transform is needed: the rows' spectra are c*X at kx = 0
            // and 0 elsewhere.
            if (tid == 0) a.partial[tile] = 0.0;
            if (a.r2c) {
                const float dc = (op == XOP_RATIO_RL) ? 1e-6f * (float) C::X : 0.f;
                float2 *Sz = a.S + (long long) z * plane + (long long) y0 * KB;
                for (int e = tid; e < C::NKB * R * KB; e += C::THREADS) {
                    const int ki = e % KB;
                    const int r2 = (e / KB) % R;
                    const int kb = e / (KB * R);
                    const int k = kb * KB + ki;
                    if (k > L || y0 + r2 >= a.Y) continue;
                    Sz[(long long) kb * a.Y * KB + r2 * KB + ki] = make_float2(k == 0 ? dc : 0.f, 0.f);
                }
            }
            return;
        }
    }

    // ---- bulk copies of this tile (warp 0)
    const bool grow = rg && z < a.P && y0 < a.N;
    const int gr = grow ? min(R, a.N - y0) : 0;
    const uint32_t rbytes = (uint32_t) (R * XP * sizeof(float));
    const uint32_t gbytes = (uint32_t) ((long long) gr * a.GP * sizeof(float));
    const uint32_t cbytes = c2r ? (uint32_t) (C::NKB * R * KB * sizeof(float2)) : 0u;
    const uint32_t real_total = rbytes * ((rx ? 1 : 0) + (rxp ? 1 : 0) + (rw ? 1 : 0)) + gbytes;
    if (tid == 0) {
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    // complex rows: every kx block of this tile is R*32 contiguous bytes;
    // 16-byte asynchronous copies spread over all threads
    if constexpr (c2r) {
        constexpr int PIECES = R * KB * (int) sizeof(float2) / 16;  // per kx block
        const float4 *src = reinterpret_cast<const float4 *>(a.S + (long long) z * plane + (long long) y0 * KB);
        float4 *dst = reinterpret_cast<float4 *>(CB);
        const long long kstride = (long long) a.Y * KB * (long long) sizeof(float2) / 16;
        for (int e = tid; e < C::NKB * PIECES; e += C::THREADS) {
            const int kb = e / PIECES, p = e - kb * PIECES;
            cp_async16(dst + e, src + kb * kstride + p);
        }
        cp_async_commit();
    }
    (void) cbytes;
    __syncthreads();
    if (tid < 32) {
        if (tid == 0) mbar_arrive_expect_tx(&bars[1], real_total);
        __syncwarp();
        const long long row0 = (long long) z * a.Y + y0;
        if (tid == 1 && rx) tma_load_1d(RB, a.src + row0 * XP, rbytes, &bars[1]);
        if (tid == 2 && rxp) tma_load_1d(RB + C::REAL_F, a.srcp + row0 * XP, rbytes, &bars[1]);
        if (tid == 3 && rw) tma_load_1d(RB + 2 * C::REAL_F, a.Wt + row0 * XP, rbytes, &bars[1]);
        if (tid == 4 && gr > 0) tma_load_1d(RB, a.g + ((long long) z * a.N + y0) * a.GP, gbytes, &bars[1]);
    }
    // this thread's rows: ry*Q + q
    auto smem = [&](int q, int i) { return CB + (size_t) (ry * Q + q) * C::ROW_F2 + i; };
    double acc = 0.0;
    const float bg = a.sc->bg;

    float2 w[Q][RD::RL];  // thread t < SL holds z_q[t + r*SL] = x[2n] + i x[2n+1]
#pragma unroll
    for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int r = 0; r < RD::RL; ++r) w[q][r] = make_float2(0.f, 0.f);

    if constexpr (c2r) {
        cp_async_wait_all();
        __syncthreads();  // every thread's copies have landed
        // first-stage inputs Z[k] = (X[k] + X*[L-k]) + i W_X^{-k} (X[k] - X*[L-k]);
        // Im X[0] and Im X[L] are ignored, as by any real inverse transform
        float2 v[Q][RD::RA];
        if (t < L / RD::RA) {
            // W_X^k for k = t + r*L/RA: one table value, times compile-time
            // factors W_X^{r*L/RA} (the table stays out of the L1 cache,
            // which the staging buffers leave small)
            const float2 tb = __ldg(&a.tw[t]);
            static_for<RD::RA>([&](auto rc) {
                constexpr int r = decltype(rc)::value;
                const int k = t + r * (L / RD::RA);
                const int km = L - k;
                const float2 tk = twiddle<C::X, r * (L / RD::RA), -1>(tb);
                const int ik = (k / KB) * (R * KB) + (k % KB);
                const int im = (km / KB) * (R * KB) + (km % KB);
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const int rr = ry * Q + q;
                    float2 xk = CB[ik + rr * KB];
                    float2 xm = CB[im + rr * KB];
                    if (k == 0) { xk.y = 0.f; xm.y = 0.f; }
                    xm.y = -xm.y;
                    float2 s = cadd(xk, xm), d = csub(xk, xm);
                    float2 e = cmulc(d, tk);
                    v[q][r] = make_float2(s.x - e.y, s.y + e.x);
                }
            });
        }
        __syncthreads();  // the staged rows become the exchange tiles
        line_fft<RD, +1, Q, PREF_TW, false>(v, w, t, a.twL, smem);
    }
    if (!wait_all(&bars[1], 0, a.err, 3 << 8)) return;

    // ---- pointwise op on x[2n], x[2n+1], n = t + r*SL
    if (t < SL) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int rr = ry * Q + q;
            const int yy = y0 + rr;
            if (yy < a.Y) {
                const bool in_img_row = yy < a.N && z < a.P;
                const long long rbase = ((long long) z * a.Y + yy) * XP;
                const float *sx = (rg ? RB + rr * a.GP : RB + rr * XP);
                const float *sxp = RB + C::REAL_F + rr * XP;
                const float *sw = rw ? RB + 2 * C::REAL_F + rr * XP : nullptr;
                x_row_op<FAM, RD::RL, SL>(a, op, t, rbase, sx, sxp, sw, in_img_row, bg, w[q], acc);
            }
        }
    }

    if constexpr (rg) {
        // deterministic reduction of the tile's error partial (fixed order;
        // lanes meet in shared memory, then one full warp reduces)
        red[tid] = acc;
        __syncthreads();
        if (tid < 32) {
            double s2 = 0.0;
            for (int i = tid; i < C::THREADS; i += 32) s2 += red[i];
            for (int o = 16; o > 0; o >>= 1) s2 += __shfl_down_sync(0xffffffffu, s2, o);
            if (tid == 0) a.partial[tile] = s2;
        }
    }
    if constexpr (FAM == XFAM_STORE) return;
    if (!a.r2c) return;

    // ---- forward with the reversed radix list; w is its first-stage input
    __syncthreads();  // all reads of the exchange tiles are complete
    if (a.wrapx) {
        // periodic margins of the row (see XArgs), through shared memory
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            float *rowf = reinterpret_cast<float *>(smem(q, 0));
            if (t < SL) {
#pragma unroll
                for (int r = 0; r < RD::RL; ++r) {
                    const int n = t + r * SL;
                    rowf[2 * n] = w[q][r].x;
                    rowf[2 * n + 1] = w[q][r].y;
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float *rowf = reinterpret_cast<const float *>(smem(q, 0));
            if (t < SL) {
#pragma unroll
                for (int r = 0; r < RD::RL; ++r) {
                    const int n = t + r * SL;
                    float e[2];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int c = 2 * n + h;
                        const int src = c < a.wM ? c
                                      : c < a.wM + a.hx ? c - a.wM
                                      : c >= C::X - a.hx ? c - C::X + a.wM : -1;
                        e[h] = src >= 0 ? rowf[src] : 0.f;
                    }
                    w[q][r] = make_float2(e[0], e[1]);
                }
            }
        }
        __syncthreads();
    }
    float2 qo[Q][RV::RL];
    // stage 2 writes the real slots (every pointwise read of them precedes
    // the barrier after stage 1), so stage 3 leaves the exchange tiles free
    float2 *xb2 = reinterpret_cast<float2 *>(RB);
    auto smem2 = [&](int q, int i) { return xb2 + (size_t) (ry * Q + q) * C::ROW_F2 + i; };
    line_fft_impl<RV, -1, Q, PREF_TW, true, decltype(smem), decltype(smem2), false, false>(w, qo, t, a.twL, smem,
                                                                                           smem2);
    constexpr int SQ = L / RV::RL;
    if constexpr (!RV::THREE) __syncthreads();
    if (t < SQ) {
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int r = 0; r < RV::RL; ++r) *smem(q, t + r * SQ) = qo[q][r];
    }
    __syncthreads();
    // ---- Hermitian post-processing X[k] = E[k] + W_X^k O[k], k = 0..L,
    // written to the blocked layout: thread e -> (kb, row, ki)
    float2 *Sz = a.S + (long long) z * plane + (long long) y0 * KB;
    constexpr int TOT = C::NKB * R * KB;
    if constexpr (C::THREADS % (KB * R) == 0) {
        // thread tid handles e = tid + m*THREADS: one row, k = k0 + m*THREADS/R,
        // so W_X^k = W_X^{k0} times compile-time factors
        constexpr int DK = C::THREADS / R;
        constexpr int MAXM = (TOT + C::THREADS - 1) / C::THREADS;
        const int ki0 = tid % KB;
        const int r2 = (tid / KB) % R;
        const int k0 = (tid / (KB * R)) * KB + ki0;
        const float2 tb = __ldg(&a.tw[k0 <= L ? k0 : 0]);
        const float2 *Br = CB + (size_t) r2 * C::ROW_F2;
        const bool row_ok = y0 + r2 < a.Y;
        static_for<MAXM>([&](auto mc) {
            constexpr int m = decltype(mc)::value;
            const int k = k0 + m * DK;
            if (tid + m * C::THREADS < TOT && k <= L && row_ok) {
                float2 zk = Br[k == L ? 0 : k];
                float2 zm = Br[k == 0 ? 0 : L - k];
                zm.y = -zm.y;
                float2 ev = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
                float2 d = csub(zk, zm);
                float2 o = make_float2(0.5f * d.y, -0.5f * d.x);  // -(i/2) d
                const int kb = k / KB;
                Sz[(long long) kb * a.Y * KB + r2 * KB + ki0] = cadd(ev, cmul(o, twiddle<C::X, m * DK, -1>(tb)));
            }
        });
    } else {
        for (int e = tid; e < TOT; e += C::THREADS) {
            const int ki = e % KB;
            const int r2 = (e / KB) % R;
            const int kb = e / (KB * R);
            const int k = kb * KB + ki;
            if (k > L || y0 + r2 >= a.Y) continue;
            const float2 *Br = CB + (size_t) r2 * C::ROW_F2;
            float2 zk = Br[k == L ? 0 : k];
            float2 zm = Br[k == 0 ? 0 : L - k];
            zm.y = -zm.y;
            float2 ev = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
            float2 d = csub(zk, zm);
            float2 o = make_float2(0.5f * d.y, -0.5f * d.x);  // -(i/2) d
            Sz[(long long) kb * a.Y * KB + r2 * KB + ki] = cadd(ev, cmul(o, __ldg(&a.tw[k])));
        }
    }
}

}  // namespace dwcu
