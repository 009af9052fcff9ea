// Pieces shared by the slab passes (ns_slab.cu: one CTA holds a whole slab,
// two CTAs an SM) and the cluster slab passes (ns_slab_cluster.cu: a slab
// split over the two CTAs of a thread-block cluster): launch arguments, line
// geometry, twiddle layout and the warp-local line FFT.
#pragma once

#include "plan.h"
#include "regfft.cuh"

namespace sfl {

constexpr int kSlabThreads = 512;
constexpr int kSlabWarps = kSlabThreads / 32;
constexpr size_t kSlabSmemOneCta = 227 * 1024;   // the most one CTA may hold

struct SlabArgs {
    float2* spec;            // padded spectra, item z at spec + z * spec_zstride
    long long spec_zstride;
    float* vol;              // real volumes (element stride es), item z at vol + vz.off(z)
    ZMap vz;
    int es;
    float scale;             // applied to the C2R outputs
    int P1, n3;
    int nk1, nk2, b2;        // box: rows k1 < nk1, columns as BoxMap
    int units;               // channels x items x n3
    int nzc;                 // items a channel
    long long spec_chstride; // spectra: channel stride (the volume's channels are interleaved floats)
    const float2* twa;       // w_n1^k, k < n1 (float64-designed)
    const float2* twb;       // w_n2^k, k < n2
    const float* tau;        // shrink pass: threshold of subband s at tau[s - 1]
    const NSItem* items;     // shrink pass: the launch's items, from item0
    int item0;
    int* status;             // the plan's device status word (bounded waits record a timeout there)
};

template <int N>
struct SlabLine {
    static constexpr int N1 = LinePlan<N>::N1;
    static constexpr int N2 = LinePlan<N>::N2;
    static constexpr int M = N1 / N2;
    static constexpr int LPW = 32 / N2;             // lines a warp
    static constexpr int LPR = kSlabWarps * LPW;    // lines a round
};

// Twiddles of a line FFT rearranged as tw2[m * N2 + p] = w_N^{p m}: the N2
// lanes of a line read consecutive words.
template <int N>
__device__ __forceinline__ void load_slab_twiddles(float2* tw2, const float2* __restrict__ tw) {
    using L = SlabLine<N>;
    for (int i = threadIdx.x; i < L::N1 * L::N2; i += blockDim.x) {
        const int m = i / L::N2, p = i - m * L::N2;
        tw2[i] = tw[p * m];
    }
}

// Axis-1 pitch of a padded spectrum with h1 bins on axis 1: the smallest
// P1 >= h1 with P1 = 2 mod 4.
constexpr int slab_pitch_c(int h1) { return h1 % 4 == 2 ? h1 : slab_pitch_c(h1 + 1); }

// FFT of one line of N points held by the N2 lanes p of a warp: v[r] holds
// x[p + N2 r] on entry and X[(p + N2 j) + N1 k] at v[j N2 + k] on exit.  The
// exchange runs through the line's own slots base[STRIDE t], t < N, with
// slot (sender q, value m) at t = N2 m + (q ^ (m mod N2)): conflict-free
// writes and reads for STRIDE = 1 and for STRIDE = 2 mod 4.  Lanes of
// invalid lines skip every slot access but keep to the warp barriers.
template <int N, bool INV, int STRIDE>
__device__ __forceinline__ void warp_line_fft(float2 (&v)[LinePlan<N>::N1], int p, bool valid,
                                              const float2* __restrict__ tw2, float2* base) {
    using L = SlabLine<N>;
    constexpr int N1 = L::N1, N2 = L::N2;
    RegDft<N1, INV>::run(v);
#pragma unroll
    for (int m = 1; m < N1; ++m) {
        float2 w = tw2[m * N2 + p];
        if (INV) w.y = -w.y;
        v[m] = c_mul(v[m], w);
    }
    // x[c] = STRIDE (p ^ c): the sender-dependent part of a slot, shared by both sides
    int xo[N2];
#pragma unroll
    for (int c = 0; c < N2; ++c) xo[c] = STRIDE * (p ^ c);
    __syncwarp();   // the line's inputs may have come from its own slots
    if (valid) {
#pragma unroll
        for (int m = 0; m < N1; ++m) base[xo[m & (N2 - 1)] + STRIDE * N2 * m] = v[m];
    }
    __syncwarp();
    const float2* rb = base + STRIDE * N2 * p;
#pragma unroll
    for (int j = 0; j < L::M; ++j) {
        float2 w[N2];
#pragma unroll
        for (int pp = 0; pp < N2; ++pp)
            w[pp] = valid ? rb[xo[pp] + STRIDE * N2 * N2 * j] : make_float2(0.f, 0.f);
        RegDft<N2, INV>::run(w);
#pragma unroll
        for (int k = 0; k < N2; ++k) v[j * N2 + k] = w[k];
    }
    __syncwarp();   // slots are free again
}

// The same line FFT over slots base[stride t] with a run-time stride (a plane
// of another pitch); conflict-free for stride = 1 or 2 mod 4.
template <int N, bool INV>
__device__ __forceinline__ void warp_line_fft_rs(float2 (&v)[LinePlan<N>::N1], int p, bool valid,
                                                 const float2* __restrict__ tw2, float2* base, int stride) {
    using L = SlabLine<N>;
    constexpr int N1 = L::N1, N2 = L::N2;
    RegDft<N1, INV>::run(v);
#pragma unroll
    for (int m = 1; m < N1; ++m) {
        float2 w = tw2[m * N2 + p];
        if (INV) w.y = -w.y;
        v[m] = c_mul(v[m], w);
    }
    int xo[N2];
#pragma unroll
    for (int c = 0; c < N2; ++c) xo[c] = stride * (p ^ c);
    __syncwarp();
    if (valid) {
#pragma unroll
        for (int m = 0; m < N1; ++m) base[xo[m & (N2 - 1)] + stride * N2 * m] = v[m];
    }
    __syncwarp();
    const float2* rb = base + stride * N2 * p;
#pragma unroll
    for (int j = 0; j < L::M; ++j) {
        float2 w[N2];
#pragma unroll
        for (int pp = 0; pp < N2; ++pp)
            w[pp] = valid ? rb[xo[pp] + stride * N2 * N2 * j] : make_float2(0.f, 0.f);
        RegDft<N2, INV>::run(w);
#pragma unroll
        for (int k = 0; k < N2; ++k) v[j * N2 + k] = w[k];
    }
    __syncwarp();
}

// Lane layout of the column-pair phases: p fastest, then the line; with four
// lines a warp, the two lines of a half warp are two apart so that their
// columns fall on disjoint banks (P1 = 2 mod 4).
template <int N>
__device__ __forceinline__ int pair_subline(int s) {
    if (SlabLine<N>::LPW == 4) return s == 1 ? 2 : (s == 2 ? 1 : s);
    return s;
}

// Launches a slab pass of a size with a cluster kernel (ns_slab_cluster.cu).
// KIND: 0 forward, 1 inverse, 2 the denoiser's shrink pass.  Returns false
// when (na, nb) has none.
bool launch_slab_cluster(int kind, int na, int nb, const SlabArgs& a, int sms, cudaStream_t st, const char* tag);
bool slab_cluster_supported(int na, int nb);
bool slab_cluster_resident(int na, int nb);

}  // namespace sfl
