// dft.cuh -- in-register DFT building blocks for the sm_100a FFT passes.
//
// Every transform here runs on a register array of float2 with compile-time
// length, so all indexing and all twiddle constants fold at compile time.
// Twiddle constants are evaluated by constexpr functions written here from
// the Taylor series of sin and cos after an exact reduction of the angle
// pi*a/b to [0, pi/4] (no library math is used for constants).
//
// Conventions: DIR = -1 is the forward transform X[k] = sum x[n] e^{-2 pi i nk/N},
// DIR = +1 the unnormalised inverse.  Inputs and outputs are in natural order.
#pragma once
#include <cuda_runtime.h>
#include <utility>

#ifndef DW_HD
#define DW_HD __host__ __device__ __forceinline__
#endif

namespace dwcu {

// ------------------------------------------------------------ constants
namespace cx {
constexpr double kPi = 3.14159265358979323846264338327950288;

__host__ __device__ constexpr double taylor_sin(double x)
{
    double x2 = x * x, term = x, sum = x;
    for (int i = 1; i < 14; ++i) {
        term *= -x2 / (double) ((2 * i) * (2 * i + 1));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double taylor_cos(double x)
{
    double x2 = x * x, term = 1.0, sum = 1.0;
    for (int i = 1; i < 14; ++i) {
        term *= -x2 / (double) ((2 * i - 1) * (2 * i));
        sum += term;
    }
    return sum;
}
// cos(pi * a / b), b > 0, any integer a
__host__ __device__ constexpr double cospi_frac(long long a, long long b)
{
    long long m = 2 * b;
    a %= m;
    if (a < 0) a += m;
    if (a > b) a = m - a;              // cos is even, period 2b
    if (2 * a > b) return -cospi_frac(b - a, b);
    if (4 * a > b) return taylor_sin(kPi * (double) (b - 2 * a) / (double) (2 * b));
    return taylor_cos(kPi * (double) a / (double) b);
}
// sin(pi * a / b) = cos(pi/2 - pi*a/b) = cos(pi * (b - 2a) / (2b))
__host__ __device__ constexpr double sinpi_frac(long long a, long long b) { return cospi_frac(b - 2 * a, 2 * b); }
}  // namespace cx

// ------------------------------------------------------------ static_for
template <class F, int... I>
DW_HD void static_for_impl(F &&f, std::integer_sequence<int, I...>)
{
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
DW_HD void static_for(F &&f)
{
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// complex sums as one paired single-precision add on sm_100 (FADD2: both
// lanes rounded to nearest, as two scalar adds).  A translation unit may
// define DW_PAIRED_ADDS 0 first to keep scalar adds (device code is compiled
// per translation unit).
#ifndef DW_PAIRED_ADDS
#define DW_PAIRED_ADDS 1
#endif
DW_HD float2 cadd(float2 a, float2 b)
{
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000 && DW_PAIRED_ADDS
    return __fadd2_rn(a, b);
#else
    return make_float2(a.x + b.x, a.y + b.y);
#endif
}
DW_HD float2 csub(float2 a, float2 b)
{
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000 && DW_PAIRED_ADDS
    return __fadd2_rn(a, make_float2(-b.x, -b.y));
#else
    return make_float2(a.x - b.x, a.y - b.y);
#endif
}
// complex products: with paired instructions, one FMUL2 and one FFMA2
DW_HD float2 cmul(float2 a, float2 b)
{
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000 && DW_PAIRED_ADDS
    const float2 t = __fmul2_rn(a, make_float2(b.x, b.x));
    return __ffma2_rn(make_float2(-a.y, a.x), make_float2(b.y, b.y), t);
#else
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
#endif
}
DW_HD float2 cmulc(float2 a, float2 b)  // a * conj(b)
{
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000 && DW_PAIRED_ADDS
    const float2 t = __fmul2_rn(a, make_float2(b.x, b.x));
    return __ffma2_rn(make_float2(a.y, -a.x), make_float2(b.y, b.y), t);
#else
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
#endif
}
// multiply by DIR*i
template <int DIR>
DW_HD float2 mul_i(float2 v)
{
    return DIR < 0 ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
}

// v * exp(DIR * 2 pi i K / N), K and N compile-time
template <int N, int K, int DIR>
DW_HD float2 twiddle(float2 v)
{
    constexpr int k = ((K % N) + N) % N;
    if constexpr (k == 0) {
        return v;
    } else if constexpr (2 * k == N) {
        return make_float2(-v.x, -v.y);
    } else if constexpr (4 * k == N) {
        return mul_i<DIR>(v);
    } else if constexpr (4 * k == 3 * N) {
        return mul_i<-DIR>(v);
    } else if constexpr ((8 * k) % N == 0) {
        // odd multiples of pi/4: (+-1 +- i)/sqrt(2)
        constexpr float h = 0.70710678118654752440f;
        constexpr float c = (float) cx::cospi_frac(2 * k, N);
        constexpr float s = (float) (DIR * cx::sinpi_frac(2 * k, N));
        constexpr float sc = c > 0 ? h : -h;
        constexpr float ss = s > 0 ? h : -h;
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000 && DW_PAIRED_ADDS
        return __ffma2_rn(make_float2(-v.y, v.x), make_float2(ss, ss), __fmul2_rn(v, make_float2(sc, sc)));
#else
        return make_float2(sc * v.x - ss * v.y, ss * v.x + sc * v.y);
#endif
    } else {
        constexpr float c = (float) cx::cospi_frac(2 * k, N);
        constexpr float s = (float) (DIR * cx::sinpi_frac(2 * k, N));
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000 && DW_PAIRED_ADDS
        return __ffma2_rn(make_float2(-v.y, v.x), make_float2(s, s), __fmul2_rn(v, make_float2(c, c)));
#else
        return make_float2(v.x * c - v.y * s, v.x * s + v.y * c);
#endif
    }
}

// ------------------------------------------------------------ DFT kernels
template <int N, int DIR>
struct Dft;

template <int DIR>
struct Dft<1, DIR> {
    static DW_HD void run(float2 *) {}
};

template <int DIR>
struct Dft<2, DIR> {
    static DW_HD void run(float2 *v)
    {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <int DIR>
struct Dft<3, DIR> {
    static DW_HD void run(float2 *v)
    {
        constexpr float s = DIR * 0.86602540378443864676f;  // DIR*sqrt(3)/2
        float2 a = cadd(v[1], v[2]);
        float2 d = csub(v[1], v[2]);
        float2 m = make_float2(v[0].x - 0.5f * a.x, v[0].y - 0.5f * a.y);
        float2 r = make_float2(-s * d.y, s * d.x);  // i*s*d
        v[0] = cadd(v[0], a);
        v[1] = cadd(m, r);
        v[2] = csub(m, r);
    }
};

template <int DIR>
struct Dft<4, DIR> {
    static DW_HD void run(float2 *v)
    {
        float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        float2 a2 = cadd(v[1], v[3]), a3 = mul_i<DIR>(csub(v[1], v[3]));
        v[0] = cadd(a0, a2);
        v[2] = csub(a0, a2);
        v[1] = cadd(a1, a3);
        v[3] = csub(a1, a3);
    }
};

// odd prime lengths: pair n with N-n
template <int N, int DIR>
struct DftOddPrime {
    static DW_HD void run(float2 *v)
    {
        constexpr int H = (N - 1) / 2;
        float2 A[H + 1], B[H + 1];
        float2 s0 = v[0];
        static_for<H>([&](auto jj) {
            constexpr int j = decltype(jj)::value + 1;
            A[j] = cadd(v[j], v[N - j]);
            B[j] = csub(v[j], v[N - j]);
            s0 = cadd(s0, A[j]);
        });
        float2 x0 = v[0];
        static_for<H>([&](auto qq) {
            constexpr int q = decltype(qq)::value + 1;
            float2 e = x0, f = make_float2(0.f, 0.f);
            static_for<H>([&](auto jj) {
                constexpr int j = decltype(jj)::value + 1;
                constexpr float c = (float) cx::cospi_frac(2 * j * q, N);
                constexpr float s = (float) cx::sinpi_frac(2 * j * q, N);
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000 && DW_PAIRED_ADDS
                e = __ffma2_rn(make_float2(c, c), A[j], e);
                f = __ffma2_rn(make_float2(s, s), B[j], f);
#else
                e.x = fmaf(c, A[j].x, e.x);
                e.y = fmaf(c, A[j].y, e.y);
                f.x = fmaf(s, B[j].x, f.x);
                f.y = fmaf(s, B[j].y, f.y);
#endif
            });
            // X_q = e + DIR*i*f ; X_{N-q} = e - DIR*i*f
            float2 r = mul_i<DIR>(f);
            v[q] = cadd(e, r);
            v[N - q] = csub(e, r);
        });
        v[0] = s0;
    }
};
template <int DIR>
struct Dft<5, DIR> : DftOddPrime<5, DIR> {};
template <int DIR>
struct Dft<7, DIR> : DftOddPrime<7, DIR> {};

// composite: N = A * B, Cooley-Tukey with compile-time twiddles
__host__ __device__ constexpr int dft_first_factor(int n)
{
    return (n % 4 == 0 && n != 8) ? 4 : (n % 2 == 0 ? 2 : (n % 3 == 0 ? 3 : (n % 5 == 0 ? 5 : 7)));
}

__host__ __device__ constexpr int cgcd(int a, int b) { return b == 0 ? a : cgcd(b, a % b); }
// inverse of a modulo m (gcd(a, m) == 1)
__host__ __device__ constexpr int cinv(int a, int m)
{
    int r = 1;
    while ((a * r) % m != 1 % m) ++r;
    return r % m;
}

template <int N, int DIR>
struct Dft {
    static constexpr int A = dft_first_factor(N);
    static constexpr int B = N / A;
    static_assert(A * B == N, "length must be 7-smooth");
    static DW_HD void run(float2 *v)
    {
        if constexpr (cgcd(A, B) == 1) {
            // prime-factor (Good-Thomas) algorithm: input n = (a*B + b*A) mod N,
            // output k = (ka*B*(B^-1 mod A) + kb*A*(A^-1 mod B)) mod N; the
            // sub-transforms need no twiddle factors
            constexpr int CA = B * cinv(B % A, A);  // = 1 mod A, 0 mod B
            constexpr int CB = A * cinv(A % B, B);  // = 0 mod A, 1 mod B
            float2 t[N];
            static_for<B>([&](auto bb) {
                constexpr int b = decltype(bb)::value;
                float2 u[A];
                static_for<A>([&](auto aa) {
                    constexpr int a = decltype(aa)::value;
                    u[a] = v[(a * B + b * A) % N];
                });
                Dft<A, DIR>::run(u);
                static_for<A>([&](auto kk) {
                    constexpr int ka = decltype(kk)::value;
                    t[ka * B + b] = u[ka];
                });
            });
            static_for<A>([&](auto kk) {
                constexpr int ka = decltype(kk)::value;
                float2 w[B];
                static_for<B>([&](auto bb) {
                    constexpr int b = decltype(bb)::value;
                    w[b] = t[ka * B + b];
                });
                Dft<B, DIR>::run(w);
                static_for<B>([&](auto bb) {
                    constexpr int kb = decltype(bb)::value;
                    v[(ka * CA + kb * CB) % N] = w[kb];
                });
            });
            return;
        }
        float2 t[N];
        // A-point DFTs over the subsequences v[b + B*a]
        static_for<B>([&](auto bb) {
            constexpr int b = decltype(bb)::value;
            float2 u[A];
            static_for<A>([&](auto aa) {
                constexpr int a = decltype(aa)::value;
                u[a] = v[b + B * a];
            });
            Dft<A, DIR>::run(u);
            static_for<A>([&](auto kk) {
                constexpr int ka = decltype(kk)::value;
                t[ka * B + b] = twiddle<N, b * ka, DIR>(u[ka]);
            });
        });
        // B-point DFTs; X[ka + A*kb]
        static_for<A>([&](auto kk) {
            constexpr int ka = decltype(kk)::value;
            float2 w[B];
            static_for<B>([&](auto bb) {
                constexpr int b = decltype(bb)::value;
                w[b] = t[ka * B + b];
            });
            Dft<B, DIR>::run(w);
            static_for<B>([&](auto bb) {
                constexpr int kb = decltype(bb)::value;
                v[ka + A * kb] = w[kb];
            });
        });
    }
};

}  // namespace dwcu
