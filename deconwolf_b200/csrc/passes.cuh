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
    // padded exchange index: one spare slot per RA block keeps the
    // stride-RA writes of the first stage free of bank conflicts
    static constexpr int PADN = N + N / RA + 1;
    static __device__ __forceinline__ int pad(int idx) { return idx + idx / RA; }
};

// one Stockham butterfly: v[r] = x[j + r*N/R] on entry; twiddled by
// W_{NS*R}^{r*(j mod NS)} and transformed; output r belongs at
// (j/NS)*NS*R + j%NS + r*NS.
template <int N, int NS, int R, int DIR>
__device__ __forceinline__ void butterfly(float2 (&v)[R], int j, const float2 *__restrict__ tw)
{
    if constexpr (NS > 1) {
        constexpr int step = N / (NS * R);
        const int jm = j % NS;
#pragma unroll
        for (int r = 1; r < R; ++r) {
            float2 w = __ldg(&tw[r * jm * step]);
            v[r] = (DIR < 0) ? cmul(v[r], w) : cmulc(v[r], w);
        }
    }
    Dft<R, DIR>::run(v);
}

// Full line transform.  On entry thread t (< N/RA) holds its first-stage
// input v[r] = x[t + r*N/RA].  On exit thread t (< N/RL) holds
// o[r] = X[t + r*N/RL].  smem(i) gives this line's exchange slot for padded
// index i.  Contains __syncthreads(): call uniformly from the whole block;
// the exchange tile may be reused by the caller only after another barrier.
template <class RD, int DIR, class SM>
__device__ __forceinline__ void line_fft(float2 (&v)[RD::RA], float2 (&o)[RD::RL], int t,
                                         const float2 *__restrict__ tw, SM smem)
{
    constexpr int N = RD::N, RA = RD::RA, RB = RD::RB, RC = RD::RC;
    if (t < N / RA) {
        butterfly<N, 1, RA, DIR>(v, t, tw);
#pragma unroll
        for (int r = 0; r < RA; ++r) *smem(RD::pad(t * RA + r)) = v[r];
    }
    __syncthreads();
    if constexpr (RD::THREE) {
        float2 u[RB];
        if (t < N / RB) {
#pragma unroll
            for (int r = 0; r < RB; ++r) u[r] = *smem(RD::pad(t + r * (N / RB)));
        }
        __syncthreads();
        if (t < N / RB) {
            butterfly<N, RA, RB, DIR>(u, t, tw);
            const int base = (t / RA) * RA * RB + t % RA;
#pragma unroll
            for (int r = 0; r < RB; ++r) *smem(RD::pad(base + r * RA)) = u[r];
        }
        __syncthreads();
        if (t < N / RC) {
#pragma unroll
            for (int r = 0; r < RC; ++r) o[r] = *smem(RD::pad(t + r * (N / RC)));
            butterfly<N, RA * RB, RC, DIR>(o, t, tw);
        }
    } else {
        if (t < N / RB) {
#pragma unroll
            for (int r = 0; r < RB; ++r) o[r] = *smem(RD::pad(t + r * (N / RB)));
            butterfly<N, RA, RB, DIR>(o, t, tw);
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
};

template <class RD, int T>
struct LinesCfg {
    static constexpr int THREADS = T * cmax(RD::TPL, RevRad<RD>::TPL);
    static constexpr size_t SMEM_BYTES =
        sizeof(float2) * (size_t) cmax(RD::PADN, RevRad<RD>::PADN) * T;
};

template <class RD, int T>
__global__ void __launch_bounds__(LinesCfg<RD, T>::THREADS)
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
    const int mode = a.mode;
    auto smem = [&](int i) { return sm + (size_t) i * T + line; };

    float2 v[RD::RA];
    if (t < N / RD::RA) {
#pragma unroll
        for (int r = 0; r < RD::RA; ++r)
            v[r] = valid ? base[(long long) (t + r * (N / RD::RA)) * ls] : make_float2(0.f, 0.f);
    }
    float2 o[RD::RL];
    if (mode == LINES_INV)
        line_fft<RD, +1>(v, o, t, a.tw, smem);
    else
        line_fft<RD, -1>(v, o, t, a.tw, smem);
    constexpr int SL = N / RD::RL;
    if (mode == LINES_FWD || mode == LINES_INV) {
        if (t < SL && valid) {
#pragma unroll
            for (int r = 0; r < RD::RL; ++r) base[(long long) (t + r * SL) * ls] = o[r];
        }
        return;
    }
    // multiply by the OTF (conjugated for the back-projection)
    if (t < SL && valid) {
        const float2 *h = a.otf + off;
#pragma unroll
        for (int r = 0; r < RD::RL; ++r) {
            float2 q = __ldg(&h[(long long) (t + r * SL) * ls]);
            o[r] = (mode == LINES_CONV) ? cmul(o[r], q) : cmulc(o[r], q);
        }
    }
    __syncthreads();  // the exchange tile is free again
    float2 q[RV::RL];
    line_fft<RV, +1>(o, q, t, a.tw, smem);
    constexpr int SQ = N / RV::RL;
    if (t < SQ && valid) {
#pragma unroll
        for (int r = 0; r < RV::RL; ++r) base[(long long) (t + r * SQ) * ls] = q[r];
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
    int flags;       // bit 0: non-finite value in the image or PSF
};

struct XArgs {
    float2 *S;             // spectrum rows, pitch XC
    const float2 *tw;      // tw[m] = exp(-2 pi i m / X), m < X (Hermitian pre/post)
    const float2 *twL;     // twL[m] = exp(-2 pi i m / L), m < L (stage twiddles)
    const float *g;        // image, row pitch GP
    const float *src;      // FWD_COPY source / x_k for SHB and RL
    const float *srcp;     // x_{k-1} for SHB
    const float *Wt;       // Bertero weights (may be null)
    float *dst;            // real output (UPDATE: x_{k+1}; WEIGHTS/STORE)
    double *partial;       // per-CTA error partials (ops with an error)
    const JobScalars *sc;  // bg, ...
    long long XC;          // complex row pitch
    long long X;           // real row pitch (= real length)
    long long GP;
    int Y, Z;              // padded dims
    int M, N, P;           // image dims
    int nrows;             // Y * Z
    int op;
    int r2c;               // run the forward transform after the op
    int metric;            // 1: I-divergence, 0: squared error
    int positivity;        // SHB: clamp x' at bg
    int rl_clamp;          // RL: clamp x' at bg when bg > 0
    double alpha;          // SHB extrapolation weight of the step being finished
    double alpha_next;     // SHB extrapolation weight of the next step
};

// The x transform of a real row of X = 2L samples uses a complex transform
// of length L = RD::N: z[n] = x[2n] + i x[2n+1].  The inverse runs with RD,
// the forward with the reversed radix list.
template <class RD, int R>
struct XCfg {
    using RV = RevRad<RD>;
    static constexpr int L = RD::N;
    static constexpr int TPL = cmax(RD::TPL, RV::TPL);
    static constexpr int THREADS = R * TPL;
    static constexpr int ROW_F2 = cmax(cmax(L + 1, RD::PADN), RV::PADN) | 1;
    static constexpr size_t SMEM_BYTES = sizeof(float2) * (size_t) ROW_F2 * R + sizeof(double) * THREADS;
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
    // dw.c:1514-1517: g*logf(g/y) - (g - y) for y > 0 and g > 0
    if (y > 0 && g > 0) return g * (double) logf((float) (g / y)) - (g - y);
    return 0.0;
}

// the pointwise op on the two real samples c0 = 2n, c0+1 of one row;
// (y0, y1) are the C2R values (unused by the forward-only ops); returns the
// two values handed to the forward transform
__device__ __forceinline__ float2 x_op(const XArgs &a, int op, long long rbase, long long gbase, int c0,
                                       bool img0, bool img1, float y0, float y1, float bg, double &acc)
{
    float v0 = 0.f, v1 = 0.f;
    switch (op) {
    case XOP_FWD_COPY: {
        float2 s = *reinterpret_cast<const float2 *>(a.src + rbase + c0);
        v0 = s.x; v1 = s.y;
    } break;
    case XOP_FWD_ONES:  // initial_guess, dw.c:2497-2520
        v0 = img0 ? 1.f : 0.f;
        v1 = img1 ? 1.f : 0.f;
        break;
    case XOP_FWD_SHBP: {
        float2 xv = *reinterpret_cast<const float2 *>(a.src + rbase + c0);
        float2 xq = *reinterpret_cast<const float2 *>(a.srcp + rbase + c0);
        v0 = shb_p(xv.x, xq.x, a.alpha, bg);
        v1 = shb_p(xv.y, xq.y, a.alpha, bg);
    } break;
    case XOP_RATIO_SHB:
    case XOP_RATIO_RL:
    case XOP_ERROR_ONLY: {
        float g0 = 0.f, g1 = 0.f;
        if (img1) {
            float2 gg = *reinterpret_cast<const float2 *>(a.g + gbase + c0);
            g0 = gg.x; g1 = gg.y;
        } else if (img0) {
            g0 = a.g[gbase + c0];
        }
        if (img0) acc += err_term(y0, g0, a.metric);
        if (img1) acc += err_term(y1, g1, a.metric);
        if (op == XOP_RATIO_SHB) {
            // method_shb.c:31-48: |y| < 1e-6 -> +-1e-6; r = g/y on the image, 0 elsewhere
            float d0 = y0, d1 = y1;
            if ((double) fabsf(d0) < 1e-6) d0 = copysignf(1e-6f, d0);
            if ((double) fabsf(d1) < 1e-6) d1 = copysignf(1e-6f, d1);
            v0 = img0 ? g0 / d0 : 0.f;
            v1 = img1 ? g1 / d1 : 0.f;
        } else if (op == XOP_RATIO_RL) {
            // method_rl.c:46-67: r = g/y if y > 0 else bg on the image, 1e-6 elsewhere
            v0 = img0 ? (y0 > 0.f ? g0 / y0 : bg) : 1e-6f;
            v1 = img1 ? (y1 > 0.f ? g1 / y1 : bg) : 1e-6f;
        }
    } break;
    case XOP_UPDATE_SHB: {
        // method_shb.c:56-62 (x = Kt r * (p*W)), :366-376 (positivity), and the
        // next extrapolation :333-339; p_k is recomputed from x_k, x_{k-1}
        float2 xv = *reinterpret_cast<const float2 *>(a.src + rbase + c0);
        float2 xq = *reinterpret_cast<const float2 *>(a.srcp + rbase + c0);
        float p0 = shb_p(xv.x, xq.x, a.alpha, bg);
        float p1 = shb_p(xv.y, xq.y, a.alpha, bg);
        float n0, n1;
        if (a.Wt) {
            float2 ww = *reinterpret_cast<const float2 *>(a.Wt + rbase + c0);
            n0 = y0 * (p0 * ww.x);
            n1 = y1 * (p1 * ww.y);
        } else {
            n0 = y0 * p0;
            n1 = y1 * p1;
        }
        if (a.positivity) {
            n0 = n0 < bg ? bg : n0;
            n1 = n1 < bg ? bg : n1;
        }
        *reinterpret_cast<float2 *>(a.dst + rbase + c0) = make_float2(n0, n1);
        v0 = shb_p(n0, xv.x, a.alpha_next, bg);
        v1 = shb_p(n1, xv.y, a.alpha_next, bg);
    } break;
    case XOP_UPDATE_RL: {
        // method_rl.c:84-98 and :362-372
        float2 xv = *reinterpret_cast<const float2 *>(a.src + rbase + c0);
        float n0, n1;
        if (a.Wt) {
            float2 ww = *reinterpret_cast<const float2 *>(a.Wt + rbase + c0);
            n0 = y0 * (xv.x * ww.x);
            n1 = y1 * (xv.y * ww.y);
        } else {
            n0 = y0 * xv.x;
            n1 = y1 * xv.y;
        }
        if (a.rl_clamp && bg > 0.f) {
            n0 = n0 < bg ? bg : n0;
            n1 = n1 < bg ? bg : n1;
        }
        *reinterpret_cast<float2 *>(a.dst + rbase + c0) = make_float2(n0, n1);
        v0 = n0;
        v1 = n1;
    } break;
    case XOP_WEIGHTS: {
        // method_shb.c:224-234: W = 1/P1 where P1 > 0.01, else 0
        float q0 = y0 > 0.01f ? (float) (1.0 / (double) y0) : 0.f;
        float q1 = y1 > 0.01f ? (float) (1.0 / (double) y1) : 0.f;
        *reinterpret_cast<float2 *>(a.dst + rbase + c0) = make_float2(q0, q1);
    } break;
    case XOP_STORE:
        *reinterpret_cast<float2 *>(a.dst + rbase + c0) = make_float2(y0, y1);
        break;
    default:
        break;
    }
    return make_float2(v0, v1);
}

template <class RD, int R>
__global__ void __launch_bounds__(XCfg<RD, R>::THREADS)
k_xpass(XArgs a)
{
    using C = XCfg<RD, R>;
    using RV = typename C::RV;
    constexpr int L = C::L;
    constexpr int SL = L / RD::RL;  // op phase: thread t < SL holds n = t + r*SL
    static_assert(RV::RA == RD::RL, "reversed radix list");
    extern __shared__ float2 smx[];
    const int t = threadIdx.x;
    const int rr = threadIdx.y;
    const int row = blockIdx.x * R + rr;
    const bool rvalid = row < a.nrows;
    const int yy = rvalid ? row % a.Y : 0;
    const int zz = rvalid ? row / a.Y : 0;
    float2 *B = smx + (size_t) rr * C::ROW_F2;
    float2 *Srow = a.S + (long long) row * a.XC;
    const int op = a.op;
    const bool c2r = (op >= XOP_RATIO_SHB);
    const bool in_img_row = rvalid && yy < a.N && zz < a.P;
    const float bg = a.sc->bg;
    double acc = 0.0;
    auto smem = [&](int i) { return B + i; };

    float2 w[RD::RL];  // thread t < SL holds z[t + r*SL] = x[2n] + i x[2n+1]
#pragma unroll
    for (int r = 0; r < RD::RL; ++r) w[r] = make_float2(0.f, 0.f);

    if (c2r) {
        if (rvalid)
            for (int k = t; k <= L; k += C::TPL) B[k] = Srow[k];
        __syncthreads();
        // first-stage inputs Z[k] = (X[k] + X*[L-k]) + i W_X^{-k} (X[k] - X*[L-k]);
        // Im X[0] and Im X[L] are ignored, as by any real inverse transform
        float2 v[RD::RA];
        if (t < L / RD::RA) {
#pragma unroll
            for (int r = 0; r < RD::RA; ++r) {
                const int k = t + r * (L / RD::RA);
                float2 xk = B[k];
                float2 xm = B[L - k];
                if (k == 0) { xk.y = 0.f; xm.y = 0.f; }
                xm.y = -xm.y;
                float2 s = cadd(xk, xm), d = csub(xk, xm);
                float2 e = cmulc(d, __ldg(&a.tw[k]));
                v[r] = make_float2(s.x - e.y, s.y + e.x);
            }
        }
        __syncthreads();  // the row buffer becomes the exchange tile
        line_fft<RD, +1>(v, w, t, a.twL, smem);
    }

    // ---- pointwise op on x[2n], x[2n+1], n = t + r*SL
    if (t < SL && rvalid) {
        const long long rbase = (long long) row * a.X;
        const long long gbase = (long long) zz * a.N * a.GP + (long long) yy * a.GP;
#pragma unroll
        for (int r = 0; r < RD::RL; ++r) {
            const int c0 = 2 * (t + r * SL);
            const bool img0 = in_img_row && c0 < a.M;
            const bool img1 = in_img_row && c0 + 1 < a.M;
            w[r] = x_op(a, op, rbase, gbase, c0, img0, img1, w[r].x, w[r].y, bg, acc);
        }
    }

    if (op == XOP_RATIO_SHB || op == XOP_RATIO_RL || op == XOP_ERROR_ONLY) {
        // deterministic block reduction of the error partial (fixed order;
        // the block may end in a partial warp, so lanes meet in shared memory)
        double *red = reinterpret_cast<double *>(smx + (size_t) C::ROW_F2 * R);
        const int tid = threadIdx.y * C::TPL + threadIdx.x;
        red[tid] = acc;
        __syncthreads();
        if (tid < 32) {
            double s = 0.0;
            for (int i = tid; i < C::THREADS; i += 32) s += red[i];
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (tid == 0) a.partial[blockIdx.x] = s;
        }
    }
    if (!a.r2c) return;

    // ---- forward with the reversed radix list; w is its first-stage input
    __syncthreads();  // all reads of the exchange tile are complete
    float2 q[RV::RL];
    line_fft<RV, -1>(w, q, t, a.twL, smem);
    constexpr int SQ = L / RV::RL;
    __syncthreads();
    if (t < SQ) {
#pragma unroll
        for (int r = 0; r < RV::RL; ++r) B[t + r * SQ] = q[r];
    }
    __syncthreads();
    // ---- Hermitian post-processing: X[k] = E[k] + W_X^k O[k], k = 0..L
    if (rvalid) {
        for (int k = t; k <= L; k += C::TPL) {
            float2 zk = B[k == L ? 0 : k];
            float2 zm = B[k == 0 ? 0 : L - k];
            zm.y = -zm.y;
            float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
            float2 d = csub(zk, zm);
            float2 o = make_float2(0.5f * d.y, -0.5f * d.x);  // -(i/2) d
            Srow[k] = cadd(e, cmul(o, __ldg(&a.tw[k])));
        }
    }
}

}  // namespace dwcu
