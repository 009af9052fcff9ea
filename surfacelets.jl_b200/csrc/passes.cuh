// Line-pass kernels: a tile of lines is loaded (with a fused pre-op), run
// through the shared-memory FFT, and stored (with a fused post-op).  Used by
// the NSSurfacelet and the decimated drivers.
#pragma once

#include "fft_core.cuh"
#include "plan.h"
#include "prof.h"

namespace sfl {

// ── loads ────────────────────────────────────────────────────────────────────

// Complex lines, optionally scaled.
struct LoadC {
    const float2* src;
    ZMap zm;
    Lines g;
    float scale;
    __device__ __forceinline__ void operator()(float2* tile, int npad, int n, int l0, int T, int z) const {
        const float2* s = src + zm.off(z);
        const int total = T * n;
        const bool ifast = g.si == 1;
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            int t, i;
            if (ifast) {
                i = idx % n;
                t = idx / n;
            } else {
                t = idx % T;
                i = idx / T;
            }
            int l = l0 + t;
            float2 v = make_float2(0.f, 0.f);
            if (l < g.nlines) v = s[g.base(l) + (long long)i * g.si];
            tile[t * npad + i] = scale == 1.f ? v : c_scale(v, scale);
        }
    }
};

// Two real lines per complex line: z = a + i b.  Lines 2(l0+t) and 2(l0+t)+1;
// element (l, i) of the real data at (g.base(l) + i*g.si) * es.
struct LoadRPair {
    const float* src;
    ZMap zm;
    Lines g;
    int es;
    __device__ __forceinline__ void operator()(float2* tile, int npad, int n, int l0, int T, int z) const {
        const float* s = src + zm.off(z);
        const int total = T * n;
        const bool ifast = g.si == 1;
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            int t, i;
            if (ifast) {
                i = idx % n;
                t = idx / n;
            } else {
                t = idx % T;
                i = idx / T;
            }
            int la = 2 * (l0 + t);
            float a = 0.f, b = 0.f;
            if (la < g.nlines) a = s[(g.base(la) + (long long)i * g.si) * es];
            if (la + 1 < g.nlines) b = s[(g.base(la + 1) + (long long)i * g.si) * es];
            tile[t * npad + i] = make_float2(a, b);
        }
    }
};

// Two half spectra (h = n/2+1 bins) -> the full spectrum of z = a + i b whose
// real and imaginary parts are the two real signals (C2R of both at once).  As
// a C2R does, the imaginary parts of the self-conjugate bins are dropped.
struct LoadHPair {
    const float2* src;
    ZMap zm;
    Lines g;
    float wpair = 1.f;   // weight of the bins that are not self-conjugate (0.5: adjoint of the R2C)
    __device__ __forceinline__ void operator()(float2* tile, int npad, int n, int l0, int T, int z) const {
        const float2* s = src + zm.off(z);
        const int h = n / 2 + 1;
        const int total = T * h;
        const bool ifast = g.si == 1;
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            int t, k;
            if (ifast) {
                k = idx % h;
                t = idx / h;
            } else {
                t = idx % T;
                k = idx / T;
            }
            int la = 2 * (l0 + t);
            float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
            if (la < g.nlines) a = s[g.base(la) + (long long)k * g.si];
            if (la + 1 < g.nlines) b = s[g.base(la + 1) + (long long)k * g.si];
            bool selfc = (k == 0) || (2 * k == n);
            if (selfc) {
                a.y = 0.f;
                b.y = 0.f;
            } else {
                a = c_scale(a, wpair);
                b = c_scale(b, wpair);
            }
            tile[t * npad + k] = make_float2(a.x - b.y, a.y + b.x);
            if (!selfc) tile[t * npad + (n - k)] = make_float2(a.x + b.y, b.x - a.y);
        }
    }
};

// ── stores ───────────────────────────────────────────────────────────────────

struct StoreC {
    float2* dst;
    ZMap zm;
    Lines g;
    float scale;
    __device__ __forceinline__ void operator()(const float2* tile, int npad, int n, int l0, int T, int z) const {
        float2* d = dst + zm.off(z);
        const int total = T * n;
        const bool ifast = g.si == 1;
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            int t, i;
            if (ifast) {
                i = idx % n;
                t = idx / n;
            } else {
                t = idx % T;
                i = idx / T;
            }
            int l = l0 + t;
            if (l < g.nlines) {
                float2 v = tile[t * npad + i];
                d[g.base(l) + (long long)i * g.si] = scale == 1.f ? v : c_scale(v, scale);
            }
        }
    }
};

// Unpack z = FFT(a + i b) into the half spectra of a and b (R2C of both).
struct StoreHalfPair {
    float2* dst;
    ZMap zm;
    Lines g;
    float wpair = 1.f;   // weight of the bins that are not self-conjugate (2: adjoint of the C2R)
    __device__ __forceinline__ void operator()(const float2* tile, int npad, int n, int l0, int T, int z) const {
        float2* d = dst + zm.off(z);
        const int h = n / 2 + 1;
        const int total = T * h;
        const bool ifast = g.si == 1;
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            int t, k;
            if (ifast) {
                k = idx % h;
                t = idx / h;
            } else {
                t = idx % T;
                k = idx / T;
            }
            int la = 2 * (l0 + t);
            float2 zk = tile[t * npad + k];
            float2 zm_ = tile[t * npad + (k == 0 ? 0 : n - k)];
            // A = (Z[k] + conj(Z[-k]))/2 ; B = (Z[k] - conj(Z[-k]))/(2i)
            float2 A = half_spec_a(zk, zm_);
            float2 B = half_spec_b(zk, zm_);
            if (k != 0 && 2 * k != n) {
                A = c_scale(A, wpair);
                B = c_scale(B, wpair);
            }
            if (la < g.nlines) d[g.base(la) + (long long)k * g.si] = A;
            if (la + 1 < g.nlines) d[g.base(la + 1) + (long long)k * g.si] = B;
        }
    }
};

// Unpack z = FFT(a + i b) into the full spectra of a and b (all n bins).
struct StoreFullPair {
    float2* dst;
    ZMap zm;
    Lines g;
    __device__ __forceinline__ void operator()(const float2* tile, int npad, int n, int l0, int T, int z) const {
        float2* d = dst + zm.off(z);
        const int total = T * n;
        const bool ifast = g.si == 1;
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            int t, k;
            if (ifast) {
                k = idx % n;
                t = idx / n;
            } else {
                t = idx % T;
                k = idx / T;
            }
            int la = 2 * (l0 + t);
            float2 zk = tile[t * npad + k];
            float2 zm_ = tile[t * npad + (k == 0 ? 0 : n - k)];
            float2 A = half_spec_a(zk, zm_);
            float2 B = half_spec_b(zk, zm_);
            if (la < g.nlines) d[g.base(la) + (long long)k * g.si] = A;
            if (la + 1 < g.nlines) d[g.base(la + 1) + (long long)k * g.si] = B;
        }
    }
};

// Real and imaginary parts of z are the two real output lines, scaled.
struct StoreRPair {
    float* dst;
    ZMap zm;
    Lines g;
    int es;
    float scale;
    __device__ __forceinline__ void operator()(const float2* tile, int npad, int n, int l0, int T, int z) const {
        float* d = dst + zm.off(z);
        const int total = T * n;
        const bool ifast = g.si == 1;
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            int t, i;
            if (ifast) {
                i = idx % n;
                t = idx / n;
            } else {
                t = idx % T;
                i = idx / T;
            }
            int la = 2 * (l0 + t);
            float2 v = tile[t * npad + i];
            if (la < g.nlines) d[(g.base(la) + (long long)i * g.si) * es] = v.x * scale;
            if (la + 1 < g.nlines) d[(g.base(la + 1) + (long long)i * g.si) * es] = v.y * scale;
        }
    }
};

// The real part of each complex line, scaled.
struct StoreReal {
    float* dst;
    ZMap zm;
    Lines g;
    int es;
    float scale;
    __device__ __forceinline__ void operator()(const float2* tile, int npad, int n, int l0, int T, int z) const {
        float* d = dst + zm.off(z);
        const int total = T * n;
        const bool ifast = g.si == 1;
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            int t, i;
            if (ifast) {
                i = idx % n;
                t = idx / n;
            } else {
                t = idx % T;
                i = idx / T;
            }
            int l = l0 + t;
            if (l < g.nlines) d[(g.base(l) + (long long)i * g.si) * es] = tile[t * npad + i].x * scale;
        }
    }
};

// ── the pass kernel ──────────────────────────────────────────────────────────

template <class Load, class Store>
__global__ void __launch_bounds__(256) line_pass_kernel(Load ld, Store st, FFTShape sh, int T, int npad, int inv) {
    extern __shared__ float2 smem[];
    float2* tw = smem;
    float2* a = smem + sh.n + (sh.n & 1);
    float2* b = a + T * npad;
    load_twiddles(tw, sh);
    const int l0 = blockIdx.x * T;
    const int z = blockIdx.y;
    ld(a, npad, sh.n, l0, T, z);
    __syncthreads();
    float2* r = fft_tile(a, b, T, sh, npad, tw, inv != 0);
    st(r, npad, sh.n, l0, T, z);
}

inline size_t pass_smem_bytes(int n, int T) {
    int npad = n + 1;
    return sizeof(float2) * ((size_t)n + (n & 1) + 2 * (size_t)T * npad);
}

// Lines per CTA for length n: about 2K elements per tile.
inline int pass_tile(int n) {
    int T = 2048 / n;
    if (T < 1) T = 1;
    if (T > 64) T = 64;
    return T;
}

template <class Load, class Store>
void launch_pass(const Load& ld, const Store& st, const FFTShape& sh, int nsm_lines, int nz, bool inv,
                 cudaStream_t stream, const char* tag = "pass") {
    int T = pass_tile(sh.n);
    int npad = sh.n + 1;
    size_t smem = pass_smem_bytes(sh.n, T);
    static bool configured = false;
    if (!configured) {
        cuda_check(cudaFuncSetAttribute(line_pass_kernel<Load, Store>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        200 * 1024),
                   "cudaFuncSetAttribute");
        configured = true;
    }
    dim3 grid((nsm_lines + T - 1) / T, nz);
    int tok = prof_begin(tag, stream);
    line_pass_kernel<Load, Store><<<grid, 256, smem, stream>>>(ld, st, sh, T, npad, inv ? 1 : 0);
    prof_end(tok, stream);
    cuda_check(cudaGetLastError(), "line_pass_kernel launch");
}

// Lines of a column-major 3-D array of dims d along axis a (0-based).
inline Lines axis_lines(const int d[3], int a) {
    long long s[3] = {1, d[0], (long long)d[0] * d[1]};
    int o0 = a == 0 ? 1 : 0;
    int o1 = a == 2 ? 1 : 2;
    Lines g;
    g.nlines = d[o0] * d[o1];
    g.B0 = d[o0];
    g.B1 = d[o1];
    g.s0 = s[o0];
    g.s1 = s[o1];
    g.s2 = 0;
    g.si = s[a];
    g.fast_div();
    return g;
}

}  // namespace sfl
