// NSSurfacelet coefficients stored in bfloat16 with one float32 scale per
// subband: subband s = scales[s-1] * c[..., s-1].  The scale is the smallest
// power of two at or above the subband's largest magnitude, so the stored
// values lie in [-1, 1] and the scaling itself is exact (bfloat16 keeps
// float32's exponent range; its 8-bit significand sets the accuracy).
//
// The transforms run in float32 through the item-range building blocks of
// the slab and line pipelines; a chunk of subbands passes through a float32
// scratch of chunk x n1 n2 n3 values (L2-resident at 128^3) on its way to or
// from bfloat16.
#include <cuda_bf16.h>

#include <cmath>

#include "plan.h"
#include "prof.h"

namespace sfl {

namespace {

unsigned grid_blocks(long long n) {
    long long g = (n + 255) / 256;
    return (unsigned)std::max(1LL, std::min(g, 148LL * 8));
}

// Largest magnitude of each band of a chunk (float bits of non-negative
// values order like unsigned integers).
__global__ void band_maxabs_kernel(const float* __restrict__ band, long long n, unsigned* maxbits) {
    const float* b = band + blockIdx.y * n;
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(b[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float wm[32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x + 31) / 32 ? wm[threadIdx.x] : 0.f;
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) atomicMax(maxbits + blockIdx.y, __float_as_uint(m));
    }
}

__device__ __forceinline__ float pow2_scale(unsigned bits) {
    const float m = __uint_as_float(bits);
    if (!(m > 0.f)) return 1.f;
    int e = 0;
    frexpf(m, &e);   // m = f 2^e, f in [0.5, 1)
    return ldexpf(1.f, e);
}

__global__ void band_to_bf16_kernel(const float* __restrict__ band, long long n, const unsigned* __restrict__ maxbits,
                                    const NSItem* __restrict__ items, int item0, __nv_bfloat16* out, float* scales) {
    const float* b = band + blockIdx.y * n;
    const int s = items[item0 + blockIdx.y].s;
    const float scale = pow2_scale(maxbits[blockIdx.y]);
    const float inv = 1.f / scale;   // exact: a power of two
    if (blockIdx.x == 0 && threadIdx.x == 0) scales[s - 1] = scale;
    __nv_bfloat16* o = out + (long long)(s - 1) * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        o[i] = __float2bfloat16_rn(b[i] * inv);
}

__global__ void bf16_to_band_kernel(const __nv_bfloat16* __restrict__ in, const float* __restrict__ scales,
                                    const NSItem* __restrict__ items, int item0, long long n, float* band) {
    float* b = band + blockIdx.y * n;
    const int s = items[item0 + blockIdx.y].s;
    const float scale = scales[s - 1];
    const __nv_bfloat16* c = in + (long long)(s - 1) * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = __bfloat162float(c[i]) * scale;
}

void need_bf16_path(const NSPlan& P) {
    if (P.nch != 1) throw ArgError("bfloat16 coefficients are for Float32 volumes");
}

void ensure_band(NSPlan& P) {
    const size_t need = sizeof(float) * (size_t)P.N * P.group;
    if (P.band.bytes < need) P.band.alloc(need);
    if (P.maxbits.bytes < sizeof(unsigned) * (size_t)P.group) P.maxbits.alloc(sizeof(unsigned) * P.group);
}

}  // namespace

void ns_analyze_bf16(NSPlan& P, const float* x, void* c, float* scales, cudaStream_t st) {
    need_bf16_path(P);
    ensure_band(P);
    float2* X = P.X.as<float2>();
    float* band = P.band.as<float>();
    ns_forward_spectrum(P, x, 1, X, st);
    ZMap vz;
    vz.zstride = P.N;
    for (int i0 = 0, i1; i0 < P.S; i0 = i1) {
        i1 = ns_next_chunk(P, i0);
        const int nz = i1 - i0;
        ns_analyze_range(P, X, band, vz, 1, i0, nz, false, st);
        cuda_check(cudaMemsetAsync(P.maxbits.p, 0, sizeof(unsigned) * nz, st), "cudaMemsetAsync(maxbits)");
        dim3 grid(grid_blocks(P.N), nz);
        int tok = prof_begin("ns_bf16_pack", st);
        band_maxabs_kernel<<<grid, 256, 0, st>>>(band, P.N, P.maxbits.as<unsigned>());
        band_to_bf16_kernel<<<grid, 256, 0, st>>>(band, P.N, P.maxbits.as<unsigned>(), P.items.as<NSItem>(), i0,
                                                  reinterpret_cast<__nv_bfloat16*>(c), scales);
        prof_end(tok, st);
        prof_bytes("ns_bf16_pack", (double)nz * P.N * (4 + 4 + 2));
        cuda_check(cudaGetLastError(), "bfloat16 packing");
    }
}

void ns_synthesize_bf16(NSPlan& P, const void* c, const float* scales, float* x, cudaStream_t st) {
    need_bf16_path(P);
    ensure_band(P);
    float2* A = P.acc.as<float2>();
    float2* K = P.comp.as<float2>();
    float* band = P.band.as<float>();
    ZMap vz;
    vz.zstride = P.N;
    ns_acc_clear(P, A, K, st);
    for (int i0 = 0, i1; i0 < P.S; i0 = i1) {
        i1 = ns_next_chunk(P, i0);
        const int nz = i1 - i0;
        dim3 grid(grid_blocks(P.N), nz);
        int tok = prof_begin("ns_bf16_unpack", st);
        bf16_to_band_kernel<<<grid, 256, 0, st>>>(reinterpret_cast<const __nv_bfloat16*>(c), scales,
                                                  P.items.as<NSItem>(), i0, P.N, band);
        prof_end(tok, st);
        prof_bytes("ns_bf16_unpack", (double)nz * P.N * (2 + 4));
        cuda_check(cudaGetLastError(), "bfloat16 unpacking");
        ns_accumulate_range(P, band, vz, 1, i0, nz, false, A, K, st);
    }
    ns_inverse_spectrum(P, A, x, 1, st);
}

}  // namespace sfl
