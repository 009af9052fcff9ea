// NSSurfacelet soft-threshold denoiser, y = S(soft(A x, tau)): analysis,
// c' = sign(c) max(|c| - tau_s, 0) per subband, synthesis.  On the slab
// pipeline every subband stays on the chip: the analysis axis-3 pass, one
// slab pass that inverts, thresholds and re-transforms (ns_slab_shrink_kernel)
// and the synthesis accumulation, so the coefficients never reach HBM.  The
// line pipeline fuses its axis-1 C2R, the threshold and the axis-1 R2C into
// one kernel on the work slots (axis-1 lengths with a register kernel), or
// else goes through a float32 scratch of one chunk of subbands.
// Either way the result equals synthesize(soft(analyze(x))) of the same
// pipeline bit for bit.
#include "plan.h"
#include "prof.h"

namespace sfl {

namespace {

__global__ void soft_threshold_kernel(float* band, long long n, const float* __restrict__ tau,
                                      const NSItem* __restrict__ items, int item0) {
    float* b = band + blockIdx.y * n;
    const float t = tau[items[item0 + blockIdx.y].s - 1];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float c = b[i];
        b[i] = copysignf(fmaxf(fabsf(c) - t, 0.f), c);
    }
}

}  // namespace

void ns_denoise(NSPlan& P, const float* x, float* y, const float* tau, cudaStream_t st) {
    if (P.nch != 1) throw ArgError("the denoiser is for Float32 volumes");
    float2* X = P.X.as<float2>();
    float2* A = P.acc.as<float2>();
    float2* K = P.comp.as<float2>();
    ns_forward_spectrum(P, x, 1, X, st);
    ns_acc_clear(P, A, K, st);
    const bool fused_lines = !P.slab && ns_line_shrink_supported(P);
    if (!P.slab && !fused_lines) {
        const size_t need = sizeof(float) * (size_t)P.N * P.group;
        if (P.band.bytes < need) P.band.alloc(need);
    }
    ZMap vz;
    vz.zstride = P.N;
    for (int i0 = 0, i1; i0 < P.S; i0 = i1) {
        i1 = ns_next_chunk(P, i0);
        const int nz = i1 - i0;
        if (P.slab) {
            ns_slab_denoise_items(P, X, i0, nz, tau, A, K, st);
            continue;
        }
        if (fused_lines) {
            ns_line_denoise_items(P, X, i0, nz, tau, A, K, st);
            continue;
        }
        float* band = P.band.as<float>();
        ns_analyze_range(P, X, band, vz, 1, i0, nz, false, st);
        const long long g = std::min<long long>((P.N + 255) / 256, 148LL * 8);
        int tok = prof_begin("ns_soft_threshold", st);
        soft_threshold_kernel<<<dim3((unsigned)g, nz), 256, 0, st>>>(band, P.N, tau, P.items.as<NSItem>(), i0);
        prof_end(tok, st);
        cuda_check(cudaGetLastError(), "soft_threshold_kernel");
        ns_accumulate_range(P, band, vz, 1, i0, nz, false, A, K, st);
    }
    ns_inverse_spectrum(P, A, y, 1, st);
}

}  // namespace sfl
