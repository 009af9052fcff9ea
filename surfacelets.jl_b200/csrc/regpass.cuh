// Line passes on the register-resident FFT of regfft.cuh.
//
// Each CTA holds LP lines x N2 threads.  A thread belongs to one line for the
// whole launch, so all per-line address arithmetic (the divisions of the line
// index into array coordinates) runs once per thread.  Loads and stores are
// ops with a per-line context:
//
//   Ctx line(z, l, valid)   once per thread
//   float2 get(ctx, i)      element i of the line (loads)
//   void put(ctx, k, v)     output k of the line (stores)
//
// Strided lines (element stride != 1) map consecutive lanes to consecutive
// lines, so every warp access is one contiguous run; contiguous lines map
// consecutive lanes to consecutive elements.
#pragma once

#include "passes.cuh"
#include "prof.h"
#include "regfft.cuh"

namespace sfl {

// ── loads ────────────────────────────────────────────────────────────────────

struct RLoadC {
    const float2* src;
    ZMap zm;
    Lines g;
    struct Ctx {
        const float2* p;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        return Ctx{valid ? src + zm.off(z) + g.base(l) : src};
    }
    __device__ __forceinline__ float2 get(const Ctx& c, int i) const { return c.p[(long long)i * g.si]; }
};

// Two real lines as one complex line (for a forward FFT of both).
struct RLoadRPair {
    const float* src;
    ZMap zm;
    Lines g;
    int es;
    struct Ctx {
        const float* a;
        const float* b;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        const float* s = src + zm.off(z);
        int la = 2 * l;
        Ctx c{nullptr, nullptr};
        if (valid && la < g.nlines) c.a = s + g.base(la) * es;
        if (valid && la + 1 < g.nlines) c.b = s + g.base(la + 1) * es;
        return c;
    }
    __device__ __forceinline__ float2 get(const Ctx& c, int i) const {
        long long o = (long long)i * g.si * es;
        return make_float2(c.a ? c.a[o] : 0.f, c.b ? c.b[o] : 0.f);
    }
};

// Two half spectra -> the full spectrum of a + i b (for an inverse FFT of both
// real signals).  The imaginary parts of self-conjugate bins are dropped.
struct RLoadHPair {
    const float2* src;
    ZMap zm;
    Lines g;
    int n;
    float wpair = 1.f;   // weight of the bins that are not self-conjugate (0.5: adjoint of the R2C)
    struct Ctx {
        const float2* a;
        const float2* b;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        const float2* s = src + zm.off(z);
        int la = 2 * l;
        Ctx c{nullptr, nullptr};
        if (valid && la < g.nlines) c.a = s + g.base(la);
        if (valid && la + 1 < g.nlines) c.b = s + g.base(la + 1);
        return c;
    }
    __device__ __forceinline__ float2 get(const Ctx& c, int i) const {
        int k = 2 * i <= n ? i : n - i;
        long long o = (long long)k * g.si;
        float2 A = c.a ? c.a[o] : make_float2(0.f, 0.f);
        float2 B = c.b ? c.b[o] : make_float2(0.f, 0.f);
        if (k == 0 || 2 * k == n) {
            A.y = 0.f;
            B.y = 0.f;
        } else {
            A = c_scale(A, wpair);
            B = c_scale(B, wpair);
        }
        return 2 * i <= n ? make_float2(A.x - B.y, A.y + B.x) : make_float2(A.x + B.y, B.x - A.y);
    }
};

// ── stores ───────────────────────────────────────────────────────────────────

struct RStoreC {
    static constexpr bool kStaged = false;
    float2* dst;
    ZMap zm;
    Lines g;
    struct Ctx {
        float2* p;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        return Ctx{valid ? dst + zm.off(z) + g.base(l) : dst};
    }
    __device__ __forceinline__ void put(const Ctx& c, int k, float2 v) const { c.p[(long long)k * g.si] = v; }
};

// Real and imaginary parts to two real lines, scaled (C2R of both).
struct RStoreRPair {
    static constexpr bool kStaged = false;
    float* dst;
    ZMap zm;
    Lines g;
    int es;
    float scale;
    struct Ctx {
        float* a;
        float* b;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        float* d = dst + zm.off(z);
        int la = 2 * l;
        Ctx c{nullptr, nullptr};
        if (valid && la < g.nlines) c.a = d + g.base(la) * es;
        if (valid && la + 1 < g.nlines) c.b = d + g.base(la + 1) * es;
        return c;
    }
    __device__ __forceinline__ void put(const Ctx& c, int k, float2 v) const {
        long long o = (long long)k * g.si * es;
        if (c.a) c.a[o] = v.x * scale;
        if (c.b) c.b[o] = v.y * scale;
    }
};

// The real part, scaled.
struct RStoreReal {
    static constexpr bool kStaged = false;
    float* dst;
    ZMap zm;
    Lines g;
    int es;
    float scale;
    struct Ctx {
        float* a;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        return Ctx{valid ? dst + zm.off(z) + g.base(l) * es : nullptr};
    }
    __device__ __forceinline__ void put(const Ctx& c, int k, float2 v) const {
        if (c.a) c.a[(long long)k * g.si * es] = v.x * scale;
    }
};

// Unpack z = FFT(a + i b) into the half spectra of a and b (staged through
// shared memory: bin k needs Z[k] and Z[n-k]).
struct RStoreHalfPair {
    static constexpr bool kStaged = true;
    float2* dst;
    ZMap zm;
    Lines g;
    int n;
    float wpair = 1.f;   // weight of the bins that are not self-conjugate (2: adjoint of the C2R)
    struct Ctx {
        float2* a;
        float2* b;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        float2* d = dst + zm.off(z);
        int la = 2 * l;
        Ctx c{nullptr, nullptr};
        if (valid && la < g.nlines) c.a = d + g.base(la);
        if (valid && la + 1 < g.nlines) c.b = d + g.base(la + 1);
        return c;
    }
    __device__ __forceinline__ void staged(const Ctx& c, const float2* Z, int p, int nth) const {
        const int h = n / 2 + 1;
        for (int k = p; k < h; k += nth) {
            float2 zk = Z[k];
            float2 zn = Z[k == 0 ? 0 : n - k];
            long long o = (long long)k * g.si;
            const float w = (k == 0 || 2 * k == n) ? 1.f : wpair;
            if (c.a) c.a[o] = c_scale(half_spec_a(zk, zn), w);
            if (c.b) c.b[o] = c_scale(half_spec_b(zk, zn), w);
        }
    }
};

// Unpack into the full spectra of a and b (all n bins).
struct RStoreFullPair {
    static constexpr bool kStaged = true;
    float2* dst;
    ZMap zm;
    Lines g;
    int n;
    struct Ctx {
        float2* a;
        float2* b;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        float2* d = dst + zm.off(z);
        int la = 2 * l;
        Ctx c{nullptr, nullptr};
        if (valid && la < g.nlines) c.a = d + g.base(la);
        if (valid && la + 1 < g.nlines) c.b = d + g.base(la + 1);
        return c;
    }
    __device__ __forceinline__ void staged(const Ctx& c, const float2* Z, int p, int nth) const {
        for (int k = p; k < n; k += nth) {
            float2 zk = Z[k];
            float2 zn = Z[k == 0 ? 0 : n - k];
            long long o = (long long)k * g.si;
            if (c.a) c.a[o] = half_spec_a(zk, zn);
            if (c.b) c.b[o] = half_spec_b(zk, zn);
        }
    }
};

// ── the kernel ───────────────────────────────────────────────────────────────

// One line of N points per N2 threads: load, in-register DFT_N1, twiddle,
// exchange, in-register DFT_N2 (M per thread).  Leaves the outputs in
// u[j * N2 + k] = X[(p + N2 j) + N1 k].
// The same from values already in registers: v[r] = x[p + N2 r].
template <int N, bool INV>
__device__ __forceinline__ void reg_line_fft_v(float2 (&v)[RegGeom<N>::N1], int p, float2* xl,
                                               const float2* __restrict__ tw,
                                               float2 (&u)[RegGeom<N>::M * RegGeom<N>::N2]) {
    using G = RegGeom<N>;
    constexpr int N1 = G::N1, N2 = G::N2;
    RegDft<N1, INV>::run(v);
#pragma unroll
    for (int m = 1; m < N1; ++m) {
        float2 w = __ldg(&tw[p * m]);
        if (INV) w.y = -w.y;
        v[m] = c_mul(v[m], w);
    }
#pragma unroll
    for (int m = 0; m < N1; ++m) xl[m * G::XROW + p] = v[m];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < G::M; ++j) {
        const int m = p + N2 * j;
        float2 w[N2];
#pragma unroll
        for (int pp = 0; pp < N2; ++pp) w[pp] = xl[m * G::XROW + pp];
        RegDft<N2, INV>::run(w);
#pragma unroll
        for (int k = 0; k < N2; ++k) u[j * N2 + k] = w[k];
    }
}

template <int N, bool INV, class Load>
__device__ __forceinline__ void reg_line_fft(const Load& ld, const typename Load::Ctx& lc, bool valid, int p,
                                             float2* xl, const float2* __restrict__ tw,
                                             float2 (&u)[RegGeom<N>::M * RegGeom<N>::N2]) {
    using G = RegGeom<N>;
    constexpr int N1 = G::N1, N2 = G::N2;
    float2 v[N1];
#pragma unroll
    for (int r = 0; r < N1; ++r) v[r] = valid ? ld.get(lc, p + N2 * r) : make_float2(0.f, 0.f);
    reg_line_fft_v<N, INV>(v, p, xl, tw, u);
}

template <int N, bool INV, class Load, class Store>
__global__ void __launch_bounds__(256) reg_pass_kernel(Load ld, Store st, const float2* __restrict__ tw, int nlines,
                                                       int tfast) {
    using G = RegGeom<N>;
    constexpr int N1 = G::N1, N2 = G::N2, LP = G::LP;
    extern __shared__ float2 xch[];
    const int tid = threadIdx.x;
    int lp, p;
    if (tfast) {
        lp = tid % LP;
        p = tid / LP;
    } else {
        p = tid % N2;
        lp = tid / N2;
    }
    const int l = blockIdx.x * LP + lp;
    const int z = blockIdx.y;
    const bool valid = l < nlines;
    float2* xl = xch + lp * G::XLINE;
    const typename Load::Ctx lc = ld.line(z, l, valid);
    float2 u[G::M * N2];
    reg_line_fft<N, INV>(ld, lc, valid, p, xl, tw, u);
    const typename Store::Ctx sc = st.line(z, l, valid);
    if constexpr (Store::kStaged) {
        __syncthreads();
#pragma unroll
        for (int j = 0; j < G::M; ++j)
#pragma unroll
            for (int k = 0; k < N2; ++k) xl[(p + N2 * j) + N1 * k] = u[j * N2 + k];
        __syncthreads();
        if (valid) st.staged(sc, xl, p, N2);
    } else {
        if (valid) {
#pragma unroll
            for (int j = 0; j < G::M; ++j)
#pragma unroll
                for (int k = 0; k < N2; ++k) st.put(sc, (p + N2 * j) + N1 * k, u[j * N2 + k]);
        }
    }
}

template <int N, bool INV, class Load, class Store>
void launch_reg_n(const Load& ld, const Store& st, const float2* tw, int nlines, int nz, bool tfast,
                  cudaStream_t stream, const char* tag) {
    using G = RegGeom<N>;
    static bool configured = false;
    if (!configured) {
        cuda_check(cudaFuncSetAttribute(reg_pass_kernel<N, INV, Load, Store>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM),
                   "cudaFuncSetAttribute");
        configured = true;
    }
    dim3 grid((nlines + G::LP - 1) / G::LP, nz);
    int tok = prof_begin(tag, stream);
    reg_pass_kernel<N, INV, Load, Store><<<grid, G::THREADS, G::SMEM, stream>>>(ld, st, tw, nlines, tfast ? 1 : 0);
    prof_end(tok, stream);
    cuda_check(cudaGetLastError(), "reg_pass_kernel launch");
}

// Register pass for a supported length; returns false when n has none.
template <bool INV, class Load, class Store>
bool launch_reg(int n, const Load& ld, const Store& st, const float2* tw, int nlines, int nz, bool tfast,
                cudaStream_t stream, const char* tag) {
    switch (n) {
        case 16: launch_reg_n<16, INV>(ld, st, tw, nlines, nz, tfast, stream, tag); return true;
        case 32: launch_reg_n<32, INV>(ld, st, tw, nlines, nz, tfast, stream, tag); return true;
        case 64: launch_reg_n<64, INV>(ld, st, tw, nlines, nz, tfast, stream, tag); return true;
        case 96: launch_reg_n<96, INV>(ld, st, tw, nlines, nz, tfast, stream, tag); return true;
        case 128: launch_reg_n<128, INV>(ld, st, tw, nlines, nz, tfast, stream, tag); return true;
        case 160: launch_reg_n<160, INV>(ld, st, tw, nlines, nz, tfast, stream, tag); return true;
        case 256: launch_reg_n<256, INV>(ld, st, tw, nlines, nz, tfast, stream, tag); return true;
    }
    return false;
}

}  // namespace sfl
