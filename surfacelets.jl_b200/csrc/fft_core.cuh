// Shared-memory mixed-radix Stockham FFT core for sm_100a, and the line
// geometry the pass kernels use to stage tiles of lines through it.
//
// A CTA stages T lines of length n in shared memory (row pitch npad = n + 1
// so that 64-bit accesses of consecutive lines hit distinct banks), runs the
// Stockham stages with radix 8, 5, 4, 3, 2 (and a direct DFT for any other
// prime factor), and hands the tile back to a store op.  Twiddles come from a
// float64-designed table of e^{-2 pi i t/n}, staged in shared memory.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sfl {

constexpr int kMaxStages = 24;

struct FFTShape {
    int n = 1;
    int nstages = 0;
    int radix[kMaxStages] = {};
    const float2* tw = nullptr;   // device: n entries, e^{-2 pi i t / n}
};

// Complex arithmetic on (re, im) register pairs.  Additions, subtractions and
// real scalings use sm_100's paired FP32 instructions (__fadd2_rn,
// __fmul2_rn, __ffma2_rn: one instruction for both components, each rounded
// as its scalar form), which halves the issue slots of the butterflies'
// additions.  The complex product keeps scalar FMUL / FFMA: its cross terms
// pair a component with the other operand's opposite component.
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 c_scale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
// acc + a s, one rounding a component
__device__ __forceinline__ float2 c_fma(float2 a, float s, float2 acc) {
    return __ffma2_rn(a, make_float2(s, s), acc);
}
__device__ __forceinline__ float2 c_conj(float2 a) { return make_float2(a.x, -a.y); }
// The half spectra of two real lines a, b transformed as one complex line
// z = a + i b, from zk = Z[k] and zn = Z[n - k]: A[k] = (zk + conj(zn)) / 2
// and B[k] = (zk - conj(zn)) / (2 i).
__device__ __forceinline__ float2 half_spec_a(float2 zk, float2 zn) {
    return c_scale(__ffma2_rn(zn, make_float2(1.f, -1.f), zk), 0.5f);
}
__device__ __forceinline__ float2 half_spec_b(float2 zk, float2 zn) {
    return c_scale(make_float2(zk.y + zn.y, zn.x - zk.x), 0.5f);
}
// Kahan step s += v with compensation c (Kahan 1965), per component:
// y = v - c; t = s + y; c = (t - s) - y; s = t.  The explicit round-to-nearest
// intrinsics keep the compiler from contracting or reordering it.
__device__ __forceinline__ void kahan_add(float2& s, float2& c, float2 v) {
    const float2 y = c_sub(v, c);
    const float2 t = c_add(s, y);
    c = c_sub(c_sub(t, s), y);
    s = t;
}
// multiply by -i (forward) or +i (inverse)
__device__ __forceinline__ float2 c_rot(float2 a, bool inv) {
    return inv ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <int R>
struct Dft;

template <>
struct Dft<2> {
    __device__ __forceinline__ static void run(float2* v, bool) {
        float2 a = v[0], b = v[1];
        v[0] = c_add(a, b);
        v[1] = c_sub(a, b);
    }
};

template <>
struct Dft<3> {
    __device__ __forceinline__ static void run(float2* v, bool inv) {
        const float c = -0.5f;
        const float s = inv ? -0.86602540378443864676f : 0.86602540378443864676f;
        float2 t1 = c_add(v[1], v[2]);
        // -i (v1 - v2), formed rotated by scalar subtractions
        float2 t2 = make_float2(v[1].y - v[2].y, v[2].x - v[1].x);
        float2 m = c_fma(t1, c, v[0]);
        // -i s (v1 - v2)
        float2 r = c_scale(t2, s);
        v[0] = c_add(v[0], t1);
        v[1] = c_add(m, r);
        v[2] = c_sub(m, r);
    }
};

template <>
struct Dft<4> {
    __device__ __forceinline__ static void run(float2* v, bool inv) {
        float2 t0 = c_add(v[0], v[2]);
        float2 t1 = c_sub(v[0], v[2]);
        float2 t2 = c_add(v[1], v[3]);
        // -+i (v1 - v3), formed rotated by scalar subtractions
        float2 t3 = inv ? make_float2(v[3].y - v[1].y, v[1].x - v[3].x)
                        : make_float2(v[1].y - v[3].y, v[3].x - v[1].x);
        v[0] = c_add(t0, t2);
        v[2] = c_sub(t0, t2);
        v[1] = c_add(t1, t3);
        v[3] = c_sub(t1, t3);
    }
};

template <>
struct Dft<5> {
    __device__ __forceinline__ static void run(float2* v, bool inv) {
        const float c1 = 0.30901699437494742410f;    // cos(2pi/5)
        const float c2 = -0.80901699437494742410f;   // cos(4pi/5)
        const float s1 = inv ? -0.95105651629515357212f : 0.95105651629515357212f;   // sin(2pi/5)
        const float s2 = inv ? -0.58778525229247312917f : 0.58778525229247312917f;   // sin(4pi/5)
        float2 a14 = c_add(v[1], v[4]);
        float2 a23 = c_add(v[2], v[3]);
        // -i d14 and -i d23, formed rotated by scalar subtractions
        float2 e14 = make_float2(v[1].y - v[4].y, v[4].x - v[1].x);
        float2 e23 = make_float2(v[2].y - v[3].y, v[3].x - v[2].x);
        float2 m1 = c_fma(a23, c2, c_fma(a14, c1, v[0]));
        float2 m2 = c_fma(a23, c1, c_fma(a14, c2, v[0]));
        // -i r1 = s1 e14 + s2 e23 ; -i r2 = s2 e14 - s1 e23 ; X1 = m1 - i r1 ; X2 = m2 - i r2
        float2 q1 = c_fma(e23, s2, c_scale(e14, s1));
        float2 q2 = c_fma(e23, -s1, c_scale(e14, s2));
        v[0] = c_add(c_add(v[0], a14), a23);
        v[1] = c_add(m1, q1);
        v[4] = c_sub(m1, q1);
        v[2] = c_add(m2, q2);
        v[3] = c_sub(m2, q2);
    }
};

template <>
struct Dft<8> {
    __device__ __forceinline__ static void run(float2* v, bool inv) {
        float2 e[4] = {v[0], v[2], v[4], v[6]};
        float2 o[4] = {v[1], v[3], v[5], v[7]};
        Dft<4>::run(e, inv);
        Dft<4>::run(o, inv);
        const float h = 0.70710678118654752440f;
        // w8^1 = h(1 -+ i), w8^2 = -+i, w8^3 = h(-1 -+ i)
        float2 o1 = c_scale(inv ? make_float2(o[1].x - o[1].y, o[1].x + o[1].y)
                                : make_float2(o[1].x + o[1].y, o[1].y - o[1].x), h);
        float2 o2 = c_rot(o[2], inv);
        float2 o3 = c_scale(inv ? make_float2(-(o[3].x + o[3].y), o[3].x - o[3].y)
                                : make_float2(o[3].y - o[3].x, -(o[3].x + o[3].y)), h);
        v[0] = c_add(e[0], o[0]);
        v[4] = c_sub(e[0], o[0]);
        v[1] = c_add(e[1], o1);
        v[5] = c_sub(e[1], o1);
        v[2] = c_add(e[2], o2);
        v[6] = c_sub(e[2], o2);
        v[3] = c_add(e[3], o3);
        v[7] = c_sub(e[3], o3);
    }
};

__device__ __forceinline__ float2 twiddle(const float2* tw, int idx, bool inv) {
    float2 w = tw[idx];
    return inv ? make_float2(w.x, -w.y) : w;
}

// One Stockham stage of radix R over T lines (in -> out).
template <int R>
__device__ __forceinline__ void stockham_stage(const float2* __restrict__ in, float2* __restrict__ out, int T,
                                               int n, int npad, int Ns, const float2* tw, bool inv) {
    const int nb = n / R;
    const int total = T * nb;
    const int tstep = n / (Ns * R);
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        int t = idx / nb;
        int j = idx - t * nb;
        const float2* x = in + t * npad;
        float2* y = out + t * npad;
        int k = j % Ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = x[j + r * nb];
        if (Ns > 1) {
            int step = k * tstep;
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = c_mul(v[r], twiddle(tw, r * step, inv));
        }
        Dft<R>::run(v, inv);
        int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) y[base + r * Ns] = v[r];
    }
}

// A stage of any radix R (used for prime factors without a dedicated
// butterfly): each output is a direct sum over the R inputs.
__device__ __forceinline__ void stockham_stage_generic(const float2* __restrict__ in, float2* __restrict__ out,
                                                       int R, int T, int n, int npad, int Ns, const float2* tw,
                                                       bool inv) {
    const int nb = n / R;
    const int total = T * nb * R;
    const int tstep = n / (Ns * R);
    const int rstep = n / R;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        int m = idx % R;
        int q = idx / R;
        int t = q / nb;
        int j = q - t * nb;
        const float2* x = in + t * npad;
        float2* y = out + t * npad;
        int k = j % Ns;
        float2 acc = make_float2(0.f, 0.f);
        for (int r = 0; r < R; ++r) {
            float2 v = x[j + r * nb];
            if (Ns > 1 && r > 0) v = c_mul(v, twiddle(tw, r * k * tstep, inv));
            int e = (r * m) % R;
            acc = c_add(acc, e ? c_mul(v, twiddle(tw, e * rstep, inv)) : v);
        }
        y[(j / Ns) * Ns * R + k + m * Ns] = acc;
    }
}

// All stages; returns the buffer that holds the result (a or b).
__device__ __forceinline__ float2* fft_tile(float2* a, float2* b, int T, const FFTShape& sh, int npad,
                                            const float2* tw, bool inv) {
    int Ns = 1;
    for (int s = 0; s < sh.nstages; ++s) {
        int R = sh.radix[s];
        switch (R) {
            case 2: stockham_stage<2>(a, b, T, sh.n, npad, Ns, tw, inv); break;
            case 3: stockham_stage<3>(a, b, T, sh.n, npad, Ns, tw, inv); break;
            case 4: stockham_stage<4>(a, b, T, sh.n, npad, Ns, tw, inv); break;
            case 5: stockham_stage<5>(a, b, T, sh.n, npad, Ns, tw, inv); break;
            case 8: stockham_stage<8>(a, b, T, sh.n, npad, Ns, tw, inv); break;
            default: stockham_stage_generic(a, b, R, T, sh.n, npad, Ns, tw, inv); break;
        }
        __syncthreads();
        float2* t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

// Lines of a strided array: line l -> (l0, l1, l2) with l0 fastest; element i
// of line l sits at l0*s0 + l1*s1 + l2*s2 + i*si.
struct Lines {
    int nlines = 0;
    int B0 = 1, B1 = 1;
    long long s0 = 0, s1 = 0, s2 = 0, si = 0;
    // ceil(2^32 / B0), ceil(2^32 / B1) where the line index splits by
    // multiply-high division are exact (0: integer division).  l / B =
    // umulhi(l, m) is exact when B is a power of two or l * B < 2^32
    // (Granlund and Montgomery, "Division by invariant integers using
    // multiplication", 1994); fast_div checks that for every l < nlines.
    unsigned m0 = 0, m1 = 0;
    __host__ void fast_div() {
        const unsigned long long lim = 1ull << 32, n = (unsigned long long)nlines + 64;
        m0 = m1 = 0;
        if (B0 > 1 && n * (unsigned long long)B0 < lim) m0 = 0xFFFFFFFFu / (unsigned)B0 + 1u;
        if (B1 > 1 && (n / (unsigned long long)B0 + 1) * (unsigned long long)B1 < lim)
            m1 = 0xFFFFFFFFu / (unsigned)B1 + 1u;
    }
    __device__ __forceinline__ long long base(int l) const {
        const int r = B0 == 1 ? l : (m0 ? (int)__umulhi((unsigned)l, m0) : l / B0);
        const int l0 = l - r * B0;
        const int l2 = B1 == 1 ? r : (m1 ? (int)__umulhi((unsigned)r, m1) : r / B1);
        const int l1 = r - l2 * B1;
        return (long long)l0 * s0 + (long long)l1 * s1 + (long long)l2 * s2;
    }
};

// Shared-memory layout of a pass: [twiddles n][tile a T*npad][tile b T*npad] (+ extra).
__device__ __forceinline__ void load_twiddles(float2* tws, const FFTShape& sh) {
    for (int i = threadIdx.x; i < sh.n; i += blockDim.x) tws[i] = sh.tw[i];
}

}  // namespace sfl
