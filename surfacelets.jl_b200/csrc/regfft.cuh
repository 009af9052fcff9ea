// Register-resident FFTs of compile-time length for sm_100a.
//
// A line of N = N1 * N2 points is transformed by N2 threads.  Thread p loads
// x[p + N2 r] (r < N1), runs a DFT of size N1 in registers, multiplies by
// w_N^{p m}, and after one shared-memory exchange runs the DFTs of size N2
// over p for its share of the N1 outputs m (m = p + N2 j):
//
//   X[m + N1 k] = sum_p w_N2^{p k} w_N^{p m} sum_r x[p + N2 r] w_N1^{r m}.
//
// The in-register DFTs are Cooley-Tukey compositions of radix-2/3/4/5/8
// butterflies with compile-time twiddles (constexpr sine/cosine from their
// Taylor series); the w_N^{p m} twiddles come from a float64-designed table.
#pragma once

#include <cuda_runtime.h>

#include "fft_core.cuh"

namespace sfl {

// ── compile-time trigonometry ────────────────────────────────────────────────

// sin and cos of 2 pi k / n, from the Taylor series on the first octant and
// the octant symmetries (exact rational argument reduction).
struct CxSinCos {
    double s, c;
};

constexpr double cx_sin_series(double x) {
    double x2 = x * x, term = x, sum = x;
    for (int n = 1; n < 14; ++n) {
        term *= -x2 / ((2.0 * n) * (2.0 * n + 1));
        sum += term;
    }
    return sum;
}

constexpr double cx_cos_series(double x) {
    double x2 = x * x, term = 1.0, sum = 1.0;
    for (int n = 1; n < 14; ++n) {
        term *= -x2 / ((2.0 * n - 1) * (2.0 * n));
        sum += term;
    }
    return sum;
}

constexpr CxSinCos cx_sincos_frac(long long k, long long n) {
    // angle 2 pi k / n, k reduced to [0, n)
    k %= n;
    if (k < 0) k += n;
    // octant index o = floor(8k / n), remainder angle a = 2 pi (8k - o n) / (8 n) in [0, pi/4)
    long long o = (8 * k) / n;
    long long r = 8 * k - o * n;
    const double pi = 3.14159265358979323846264338327950288;
    double a = 2.0 * pi * (double)r / (8.0 * (double)n);
    double sa = cx_sin_series(a), ca = cx_cos_series(a);
    // pi/4 complement for odd octants: angle = o*pi/4 + a
    double c45 = 0.70710678118654752440084436210484904;
    double s = 0, c = 0;
    switch ((int)o) {
        case 0: s = sa; c = ca; break;
        case 1: s = c45 * (ca + sa); c = c45 * (ca - sa); break;   // pi/4 + a
        case 2: s = ca; c = -sa; break;                           // pi/2 + a
        case 3: s = c45 * (ca - sa); c = -c45 * (ca + sa); break;   // 3pi/4 + a
        case 4: s = -sa; c = -ca; break;
        case 5: s = -c45 * (ca + sa); c = -c45 * (ca - sa); break;
        case 6: s = -ca; c = sa; break;
        default: s = -c45 * (ca - sa); c = c45 * (ca + sa); break;
    }
    return CxSinCos{s, c};
}

// w_n^k = e^{-+2 pi i k/n} as float2 (forward: minus sign).
template <int n, bool INV>
struct CxTw {
    static constexpr float re(int k) { return (float)cx_sincos_frac(k, n).c; }
    static constexpr float im(int k) { return INV ? (float)cx_sincos_frac(k, n).s : -(float)cx_sincos_frac(k, n).s; }
};

template <int n, bool INV>
struct CxTwTable {
    float2 v[n];
    constexpr CxTwTable() : v() {
        for (int k = 0; k < n; ++k) {
            CxSinCos sc = cx_sincos_frac(k, n);
            v[k].x = (float)sc.c;
            v[k].y = INV ? (float)sc.s : -(float)sc.s;
        }
    }
};

// ── in-register DFTs (natural order in and out) ─────────────────────────────

template <int R>
struct SplitOf {
    static constexpr int pick() {
        if (R % 8 == 0 && R != 8) return 8;
        if (R % 4 == 0 && R != 4) return 4;
        if (R % 2 == 0 && R != 2) return 2;
        if (R % 3 == 0 && R != 3) return 3;
        if (R % 5 == 0 && R != 5) return 5;
        return R;
    }
    static constexpr int B = pick();   // inner size
    static constexpr int A = R / B;    // outer size
};

template <int R, bool INV>
struct RegDft {
    __device__ __forceinline__ static void run(float2 (&v)[R]);
};

template <bool INV>
struct RegDft<1, INV> {
    __device__ __forceinline__ static void run(float2 (&)[1]) {}
};

#define SFL_BASE_DFT(R)                                                   \
    template <bool INV>                                                   \
    struct RegDft<R, INV> {                                               \
        __device__ __forceinline__ static void run(float2 (&v)[R]) { Dft<R>::run(v, INV); } \
    };
SFL_BASE_DFT(2)
SFL_BASE_DFT(3)
SFL_BASE_DFT(4)
SFL_BASE_DFT(5)
SFL_BASE_DFT(8)
#undef SFL_BASE_DFT

// Composite or odd-prime sizes.
template <int R, bool INV>
__device__ __forceinline__ void RegDft<R, INV>::run(float2 (&v)[R]) {
    constexpr int B = SplitOf<R>::B;
    constexpr int A = SplitOf<R>::A;
    constexpr CxTwTable<R, INV> tw{};
    if constexpr (B == R) {
        // direct DFT of a prime size
        float2 out[R];
#pragma unroll
        for (int m = 0; m < R; ++m) {
            float2 acc = v[0];
#pragma unroll
            for (int r = 1; r < R; ++r) acc = c_add(acc, c_mul(v[r], tw.v[(r * m) % R]));
            out[m] = acc;
        }
#pragma unroll
        for (int m = 0; m < R; ++m) v[m] = out[m];
    } else {
        // n = a + A b, k = kb + B ka: inner DFT_B over b, twiddle w_R^{a kb}, outer DFT_A over a
        float2 t[R];
#pragma unroll
        for (int a = 0; a < A; ++a) {
            float2 w[B];
#pragma unroll
            for (int b = 0; b < B; ++b) w[b] = v[a + A * b];
            RegDft<B, INV>::run(w);
#pragma unroll
            for (int kb = 0; kb < B; ++kb) t[a + A * kb] = (a * kb) % R == 0 ? w[kb] : c_mul(w[kb], tw.v[(a * kb) % R]);
        }
#pragma unroll
        for (int kb = 0; kb < B; ++kb) {
            float2 w[A];
#pragma unroll
            for (int a = 0; a < A; ++a) w[a] = t[a + A * kb];
            RegDft<A, INV>::run(w);
#pragma unroll
            for (int ka = 0; ka < A; ++ka) v[kb + B * ka] = w[ka];
        }
    }
}

// ── line plans ───────────────────────────────────────────────────────────────

// Split of a supported length N into N1 (in-register size) x N2 (threads per
// line).  N2 divides N1, so the second step is balanced.
template <int N>
struct LinePlan;
#define SFL_LINE_PLAN(N_, N1_, N2_)              \
    template <>                                  \
    struct LinePlan<N_> {                        \
        static constexpr int N1 = N1_;           \
        static constexpr int N2 = N2_;           \
    };
SFL_LINE_PLAN(16, 4, 4)
SFL_LINE_PLAN(32, 8, 4)
SFL_LINE_PLAN(64, 8, 8)
SFL_LINE_PLAN(96, 24, 4)
SFL_LINE_PLAN(128, 16, 8)
SFL_LINE_PLAN(160, 40, 4)
SFL_LINE_PLAN(256, 16, 16)
#undef SFL_LINE_PLAN

// Lengths with a register-resident kernel; every other length takes the
// generic shared-memory Stockham pass.
__host__ __device__ inline bool reg_fft_supported(int n) {
    switch (n) {
        case 16: case 32: case 64: case 96: case 128: case 160: case 256:
            return true;
    }
    return false;
}

// Thread geometry of a register pass: CTA of 256 threads = LP lines x N2.
template <int N>
struct RegGeom {
    static constexpr int N1 = LinePlan<N>::N1;
    static constexpr int N2 = LinePlan<N>::N2;
    static constexpr int M = N1 / N2;                   // step-2 DFTs per thread
    static constexpr int LP = 256 / N2;                 // lines per CTA
    static constexpr int THREADS = LP * N2;             // 256
    static constexpr int XROW = N2 + 1;                 // exchange row pitch (float2)
    static constexpr int XLINE = N1 * XROW + 1;         // exchange line pitch, odd
    static constexpr size_t SMEM = sizeof(float2) * (size_t)LP * XLINE;
};

}  // namespace sfl
