// NSSurfacelet slab pipeline for sm_100a: per subband one line pass along
// axis 3 and one pass over the axis-3 slabs, with the zero rows and columns of
// band-limited masks skipped.
//
// Spectra (the input spectrum X, the per-subband intermediates Y and the
// synthesis accumulator) live on the rfft grid (h1, n2, n3) with the axis-1
// pitch padded to P1 (P1 >= h1, P1 = 2 mod 4): bin (k1, k2, k3) sits at
// k1 + P1 (k2 + n2 k3), so one slab (fixed k3 or n3) is a contiguous block of
// P1 n2 bins that a CTA holds in shared memory.
//
//   analysis of subband s, c_s = irfft(X M_s):
//     line pass  Y_s(k1, k2, n3) = IFFT_3(X M_s)(k1, k2, .) for the lines of
//                the mask's support box (mask applied on load);
//     slab pass  per n3: IFFT_2 of the rows k1 < nk1, then the C2R along
//                axis 1 of two columns at a time, written straight into c_s.
//   synthesis, x = irfft(sum_s M_s rfft(c_s)):
//     slab pass  per n3: R2C along axis 1 (two columns at a time), FFT_2 of
//                the rows in the box -> Y_s;
//     line pass  FFT_3 of Y_s times M_s, summed over the subbands of one mask
//                group in registers, then one Kahan-compensated step into the
//                accumulator (a round trip of it and its compensation per group);
//     then the irfft of the accumulator (line pass and slab pass, no mask).
//
// Support boxes: the group factor B_j of scale j is a product of per-axis
// raised-cosine lowpass profiles of the finer levels
// (src/pyramid/fourier_pyramid.jl:143-150, src/transforms/ns_surfacelet.jl:
// 271-272), so it vanishes outside |k_d| <= b_d.  The plan scans each
// float64-designed group table for its box; lines and rows outside it are
// neither loaded nor transformed, and read as zeros downstream.
//
// Inside the slab pass the N2 lanes of a line sit in one warp, and the
// exchange between the two in-register DFT steps goes through the line's own
// slots of the slab (a row, or the two columns of a pair) with an XOR
// swizzle, so it needs only __syncwarp; CTA-wide barriers separate the
// phases.
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "ns_mask.cuh"
#include "plan.h"
#include "prof.h"
#include "regpass.cuh"
#include "slab_core.cuh"
#include "tma.cuh"

namespace sfl {

namespace {

// ── lines along axis 3 of a padded spectrum, restricted to a box ───────────

// Line l = (k1, j) with k1 fastest; column j maps to k2 = j for j <= b2 and
// to the negative frequencies n2 - (nk2 - j) above.
struct BoxMap {
    int nk1, nk2, b2, n2;
    __device__ __forceinline__ void k12(int l, int& k1, int& k2) const {
        const int j = l / nk1;
        k1 = l - j * nk1;
        k2 = j <= b2 ? j : j + (n2 - nk2);
    }
};

struct L3LoadC {
    const float2* src;
    long long zstride;
    int P1, s3;
    BoxMap bx;
    struct Ctx {
        const float2* p;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        int k1 = 0, k2 = 0;
        if (valid) bx.k12(l, k1, k2);
        return Ctx{src + z * zstride + k1 + P1 * k2};
    }
    __device__ __forceinline__ float2 get(const Ctx& c, int i) const { return c.p[i * s3]; }
};

struct L3StoreC {
    static constexpr bool kStaged = false;
    float2* dst;
    long long zstride;
    int P1, s3;
    BoxMap bx;
    struct Ctx {
        float2* p;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        int k1 = 0, k2 = 0;
        if (valid) bx.k12(l, k1, k2);
        return Ctx{dst + z * zstride + k1 + P1 * k2};
    }
    __device__ __forceinline__ void put(const Ctx& c, int k, float2 v) const { c.p[k * s3] = v; }
};

// X times the analysis (or synthesis) mask of item z, on load.
struct L3LoadMask {
    const float2* X;
    int P1, s3;
    BoxMap bx;
    NSMaskTables tb;
    const NSItem* items;
    int item0;
    int synth;
    struct Ctx {
        const float2* x;
        NSMaskLine m;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        int k1 = 0, k2 = 0;
        if (valid) bx.k12(l, k1, k2);
        Ctx c;
        c.x = X + k1 + P1 * k2;
        c.m = ns_mask_line(tb, items[item0 + z], k1 + tb.h1 * k2, synth != 0);
        return c;
    }
    __device__ __forceinline__ float2 get(const Ctx& c, int i) const {
        return c_scale(c.x[i * s3], ns_mask_at(c.m, i, (long long)tb.h1 * tb.n2));
    }
};

// Resident CTAs an SM the register budget aims at: two (128 registers a
// thread) where the line geometry fits, one for the long-N1 lengths 96 and
// 160 (24 and 40 values a thread) and for 256 in the accumulation.
template <int N>
constexpr int mask_minb() { return (N == 96 || N == 160) ? 1 : 2; }
template <int N>
constexpr int accum_minb() { return (N == 96 || N == 160 || N >= 256) ? 1 : 2; }
// Accumulation lengths whose sums go to shared memory (their register form spills).
template <int N>
constexpr bool accum_sums_shared() { return N == 96 || N == 128 || N == 160; }
template <int N>
constexpr size_t accum_smem() {
    return RegGeom<N>::SMEM + (accum_sums_shared<N>() ? sizeof(float2) * RegGeom<N>::M * RegGeom<N>::N2 * 256 : 0);
}

// Analysis line pass over IPC subbands of one mask group per CTA: a line's X
// times the group factor is loaded once, then per subband scaled by its
// wedge planes, transformed along axis 3 and stored.
//
// Wedge planes constant along axis 3 (plane a of hourglasses 1 and 2, over
// (k1, k2)) are a per-line scalar and commute with the axis-3 FFT, so they
// are applied after it: Y_s = wa_p(k1, k2) IFFT_3(X G wb_q).  With nbq > 0
// the chunk is nbq plane-b wedges q times whole rows of plane-a wedges p
// (item t = p nbq + q); the CTA takes the items q-major, and consecutive
// items of one q share a single FFT.  Every such item uses this order of
// operations whether or not it shares, so the values do not depend on the
// chunking.
// The subbands [k0, k0 + IPC) of one line (X times the group factor in xg):
// per subband its wedge planes, the inverse FFT along axis 3 (shared by the
// subbands of one q when factored) and the store into Y.
template <int N, int IPC>
__device__ __forceinline__ void mask_line_items(const float2 (&xg)[RegGeom<N>::N1], bool valid, int k1, int k2, int p,
                                                float2* xl, const NSMaskTables& tb, const NSItem* __restrict__ items,
                                                int item0, int nz, int k0, int nbq, int rows, int synth, float2* Y,
                                                long long ystride, int P1, int s3, const float2* __restrict__ tw) {
    using Ge = RegGeom<N>;
    constexpr int N1 = Ge::N1, N2 = Ge::N2, E = Ge::M * Ge::N2;
    const int lnat = k1 + tb.h1 * k2;
    auto zof = [&](int k) { return nbq > 0 ? (k % rows) * nbq + k / rows : k; };
    float2 u[E];
#pragma unroll 1
    for (int zz = 0; zz < IPC; ++zz) {
        const int k = k0 + zz;
        if (k >= nz) break;   // uniform across the CTA
        const int z = zof(k);
        const NSMaskLine mk = ns_mask_line(tb, items[item0 + z], lnat, synth != 0);
        const bool wedges = !(mk.low || mk.plain);
        // plane a constant along the line: applied after the FFT
        const bool after = wedges && mk.was == 0;
        const bool reuse = after && nbq > 0 && zz > 0 && (k - 1) / rows == k / rows;   // same q: uniform
        if (!reuse) {
            float2 v[N1];
            if (!wedges) {
#pragma unroll
                for (int r = 0; r < N1; ++r) v[r] = xg[r];
            } else if (after) {
#pragma unroll
                for (int r = 0; r < N1; ++r) v[r] = c_scale(xg[r], mk.wb[(p + N2 * r) * mk.wbs]);
            } else if (mk.wbs == 0) {
                const float b0 = mk.wb[0];
#pragma unroll
                for (int r = 0; r < N1; ++r) v[r] = c_scale(xg[r], mk.wa[(p + N2 * r) * mk.was] * b0);
            } else {
#pragma unroll
                for (int r = 0; r < N1; ++r) {
                    const int i = p + N2 * r;
                    v[r] = c_scale(xg[r], mk.wa[i * mk.was] * mk.wb[i * mk.wbs]);
                }
            }
            reg_line_fft_v<N, true>(v, p, xl, tw, u);
        }
        if (valid) {
            const float a0 = after ? mk.wa[0] : 1.f;
            float2* y = Y + z * ystride + k1 + P1 * k2;
#pragma unroll
            for (int j = 0; j < Ge::M; ++j)
#pragma unroll
                for (int kk = 0; kk < N2; ++kk) {
                    const float2 w = u[j * N2 + kk];
                    y[((p + N2 * j) + N1 * kk) * s3] = after ? c_scale(w, a0) : w;
                }
        }
        __syncthreads();   // the exchange rows are reused by the next subband
    }
}

template <int N, int IPC>
__global__ void __launch_bounds__(256, mask_minb<N>()) ns_slab_mask_group_kernel(const float2* __restrict__ X, int P1, int s3,
                                                                 BoxMap bx, NSMaskTables tb,
                                                                 const NSItem* __restrict__ items, int item0, int nz,
                                                                 int synth, float2* Y, long long ystride,
                                                                 const float2* __restrict__ tw, int nlines,
                                                                 long long xchs, long long ychs, int nbq) {
    using Ge = RegGeom<N>;
    constexpr int N1 = Ge::N1, N2 = Ge::N2, LP = Ge::LP;
    extern __shared__ float2 xch[];
    X += blockIdx.z * xchs;   // channel
    Y += blockIdx.z * ychs;
    const int tid = threadIdx.x;
    const int lp = tid % LP, p = tid / LP;
    const int l = blockIdx.x * LP + lp;
    const bool valid = l < nlines;
    int k1 = 0, k2 = 0;
    if (valid) bx.k12(l, k1, k2);
    float2* xl = xch + lp * Ge::XLINE;
    const long long si = (long long)tb.h1 * tb.n2;
    const int k0 = blockIdx.y * IPC;
    const int rows = nbq > 0 ? nz / nbq : 0;
    const int z0 = nbq > 0 ? (k0 % rows) * nbq + k0 / rows : k0;
    // the group factor of the line (group table, bandpass table or the lowpass factors)
    const NSMaskLine m0 = ns_mask_line(tb, items[item0 + z0], k1 + tb.h1 * k2, synth != 0);
    const float2* xp = X + k1 + P1 * k2;
    float2 xg[N1];
#pragma unroll
    for (int r = 0; r < N1; ++r) {
        const int i = p + N2 * r;
        const float g = m0.low ? m0.lowc * m0.lowv[i] : m0.m[i * si];
        xg[r] = valid ? c_scale(xp[(long long)i * s3], g) : make_float2(0.f, 0.f);
    }
    mask_line_items<N, IPC>(xg, valid, k1, k2, p, xl, tb, items, item0, nz, k0, nbq, rows, synth, Y, ystride, P1, s3,
                            tw);
}

// Synthesis line pass: FFT_3 of every item of a mask group, times its mask,
// summed in float32 over the launch's terms, then added into the accumulator
// with one Kahan step against the compensation grid comp: the compensation
// carries across launches, so the sum over the mask groups of the whole
// synthesis is compensated (src/transforms/ns_surfacelet.jl:292, 355, 383
// accumulate every subband into one spectrum).
//
// A wedge plane constant along axis 3 commutes with the axis-3 FFT, so the
// items that share plane b (and the group factor) are combined first,
// sum_p wa_p(k1, k2) Y_pq, and transformed once: with nbq > 0 the chunk is
// nbq plane-b wedges q times whole rows p (item t = p nbq + q); otherwise
// every item is its own term.  Terms are added in q order.
template <int N>
__global__ void __launch_bounds__(256, accum_minb<N>()) ns_slab_accum_kernel(const float2* __restrict__ Y, long long ystride, int G,
                                                            int P1, int s3, BoxMap bx, NSMaskTables tb,
                                                            const NSItem* __restrict__ items, int item0, int synth,
                                                            float2* acc, float2* comp, const float2* __restrict__ tw,
                                                            int nlines, long long ychs, long long achs, int nbq) {
    using Ge = RegGeom<N>;
    constexpr int N1 = Ge::N1, N2 = Ge::N2, LP = Ge::LP, E = Ge::M * Ge::N2;
    extern __shared__ float2 xch[];
    Y += blockIdx.y * ychs;   // channel
    acc += blockIdx.y * achs;
    comp += blockIdx.y * achs;
    const int tid = threadIdx.x;
    const int lp = tid % LP, p = tid / LP;
    const int l = blockIdx.x * LP + lp;
    const bool valid = l < nlines;
    int k1 = 0, k2 = 0;
    if (valid) bx.k12(l, k1, k2);
    float2* xl = xch + lp * Ge::XLINE;
    // the launch's sums: in registers, or (lengths whose registers would spill) in shared memory after the
    // exchange rows, value q of thread t at [q * 256 + t]
    constexpr bool kSumsShared = accum_sums_shared<N>();
    float2 sr[kSumsShared ? 1 : E];
    float2* ss = xch + LP * Ge::XLINE + tid;
    auto sum = [&](int q) -> float2& {
        if constexpr (kSumsShared)
            return ss[q * Ge::THREADS];
        else
            return sr[q];
    };
#pragma unroll
    for (int q = 0; q < E; ++q) sum(q) = make_float2(0.f, 0.f);
    const long long si_nat = (long long)tb.h1 * tb.n2;
    const int lnat = k1 + tb.h1 * k2;
    // the group factor of the line (group table, bandpass table or the lowpass factors), once for all items
    float gf[E];
    {
        const NSMaskLine m0 = ns_mask_line(tb, items[item0], lnat, synth != 0);
#pragma unroll
        for (int j = 0; j < Ge::M; ++j)
#pragma unroll
            for (int k = 0; k < N2; ++k) {
                const int k3 = (p + N2 * j) + N1 * k;
                gf[j * N2 + k] = m0.low ? m0.lowc * m0.lowv[k3] : m0.m[k3 * si_nat];
            }
    }
    const int rows = nbq > 0 ? G / nbq : 1;
    const int nterms = nbq > 0 ? nbq : G;
    const float2* yl = Y + k1 + P1 * k2;
    // whether an item's plane a is constant along the line (directional item, tight or analysis masks), and
    // that plane's value at the line, for the first kPre items: looked up once, ahead of the loads they scale
    constexpr int kPre = 8;
    const bool wedge_masks = !(synth && !tb.tight);
    float az_pre[kPre];
#pragma unroll
    for (int z = 0; z < kPre; ++z) {
        az_pre[z] = 1.f;
        if (z < G) {
            const NSItem* it = items + item0 + z;
            if (wedge_masks && it->kind == 0 && it->wa_hi != 2) az_pre[z] = ns_wedge_a_line(tb, it, k1, k2);
        }
    }
    for (int t = 0; t < nterms; ++t) {
        const NSItem* it0 = items + item0 + t;
        const bool before = wedge_masks && it0->kind == 0 && it0->wa_hi != 2;   // plane a applied before the FFT
        // the term: sum_p wa_p Y_pq (one item with weight 1 when plane a varies along the line; x 1 is exact).
        // The loads of the next item are in flight while the current one is added.
        const int nt = before ? rows : 1;
        float2 v[N1], yb[N1];
        {
            const float2* yz = yl + t * ystride;
#pragma unroll
            for (int r = 0; r < N1; ++r) yb[r] = valid ? yz[(long long)(p + N2 * r) * s3] : make_float2(0.f, 0.f);
        }
#pragma unroll 1
        for (int pp = 0; pp < nt; ++pp) {
            const int z = nbq > 0 ? pp * nbq + t : t;
            const float az = !before ? 1.f
                                     : (z < kPre ? az_pre[z] : ns_wedge_a_line(tb, items + item0 + z, k1, k2));
            if constexpr (N1 <= 16) {
                // a second buffer for the next item's loads (long lines would spill it)
                float2 cur[N1];
#pragma unroll
                for (int r = 0; r < N1; ++r) cur[r] = yb[r];
                if (pp + 1 < nt) {
                    const float2* yz = yl + (z + nbq) * ystride;
#pragma unroll
                    for (int r = 0; r < N1; ++r)
                        yb[r] = valid ? yz[(long long)(p + N2 * r) * s3] : make_float2(0.f, 0.f);
                }
#pragma unroll
                for (int r = 0; r < N1; ++r)
                    v[r] = pp == 0 ? c_scale(cur[r], az)
                                   : c_fma(cur[r], az, v[r]);
            } else {
                if (pp > 0) {
                    const float2* yz = yl + z * ystride;
#pragma unroll
                    for (int r = 0; r < N1; ++r)
                        yb[r] = valid ? yz[(long long)(p + N2 * r) * s3] : make_float2(0.f, 0.f);
                }
#pragma unroll
                for (int r = 0; r < N1; ++r)
                    v[r] = pp == 0 ? c_scale(yb[r], az)
                                   : c_fma(yb[r], az, v[r]);
            }
        }
        float2 u[E];
        reg_line_fft_v<N, false>(v, p, xl, tw, u);
        // the term's first item carries plane b and the group factor
        const NSMaskLine mk = ns_mask_line(tb, *it0, lnat, synth != 0);
        const bool wedges = !(mk.low || mk.plain);
#pragma unroll
        for (int j = 0; j < Ge::M; ++j)
#pragma unroll
            for (int k = 0; k < N2; ++k) {
                const int k3 = (p + N2 * j) + N1 * k;
                const float g = gf[j * N2 + k];
                const float m = !wedges ? g : (before ? g * mk.wb[k3 * mk.wbs] : g * (mk.wa[k3 * mk.was] * mk.wb[k3 * mk.wbs]));
                float2& tsum = sum(j * N2 + k);
                tsum = make_float2(fmaf(u[j * N2 + k].x, m, tsum.x), fmaf(u[j * N2 + k].y, m, tsum.y));
            }
        __syncthreads();   // the exchange rows are reused by the next term
    }
    if (valid) {
        float2* a = acc + k1 + P1 * k2;
        float2* ca = comp + k1 + P1 * k2;
#pragma unroll
        for (int j = 0; j < Ge::M; ++j)
#pragma unroll
            for (int k = 0; k < N2; ++k) {
                const long long o = (long long)((p + N2 * j) + N1 * k) * s3;
                float2 sv = a[o], cv = ca[o];
                kahan_add(sv, cv, sum(j * N2 + k));
                a[o] = sv;
                ca[o] = cv;
            }
    }
}

// ── slab passes ─────────────────────────────────────────────────────────────

// ── box rows between HBM and shared memory by bulk copies ──────────────────
//
// One cp.async.bulk a box column: the rows k1 < nk1 rounded up to an even
// count (16-byte multiples; the slab pitch P1 = 2 mod 4 is even, so every
// column starts 16-byte aligned).  The extra bin of an odd nk1 lies outside
// the box and is read by no one.  Loads complete on an mbarrier whose wait
// is bounded; stores are waited on for their shared-memory reads only.

// The slab pass's mbarrier, after the slab in shared memory.
template <int NA, int NB>
__device__ __forceinline__ uint64_t* slab_bar(float2* sm) {
    constexpr int P1 = slab_pitch_c(NA / 2 + 1);
    return reinterpret_cast<uint64_t*>(sm + NA + NB + P1 * NB);
}

__device__ __forceinline__ void slab_bar_init(uint64_t* bar) {
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
}

template <int NB, int P1>
__device__ __forceinline__ void slab_bulk_load(float2* S, const float2* src, int nk1, int nk2, int b2,
                                               uint64_t* bar, uint32_t& phase, int* status) {
    const uint32_t bytes = (uint32_t)(((nk1 + 1) & ~1) * sizeof(float2));
    fence_proxy_async();   // this thread's earlier accesses to S ahead of the copies' writes
    if (threadIdx.x == 0) mbar_arrive_expect_tx(bar, bytes * (uint32_t)nk2);
    __syncthreads();
    if ((int)threadIdx.x < nk2) {
        const int j = threadIdx.x;
        const int k2 = j <= b2 ? j : j + (NB - nk2);
        bulk_load(S + P1 * k2, src + P1 * k2, bytes, bar);
    }
    mbar_wait_bounded(bar, phase, status);
    phase ^= 1;
}

template <int NB, int P1>
__device__ __forceinline__ void slab_bulk_store(float2* dst, const float2* S, int nk1, int nk2, int b2) {
    const uint32_t bytes = (uint32_t)(((nk1 + 1) & ~1) * sizeof(float2));
    fence_proxy_async();   // this thread's writes of S visible to the copies
    __syncthreads();
    if ((int)threadIdx.x < nk2) {
        const int j = threadIdx.x;
        const int k2 = j <= b2 ? j : j + (NB - nk2);
        bulk_store(dst + P1 * k2, S + P1 * k2, bytes);
        bulk_commit();
        bulk_wait_read();   // S is rewritten by the next unit
    }
    __syncthreads();
}

// Analysis slab pass (inverse): spectra -> real volumes (element stride ES).
// The exchange slots of a column pair are the pair's two columns read as one
// run of 2 P1 >= NA values.
// FULL: the box spans every row and column (nk1 = NA/2 + 1, nk2 = NB; the
// finest scale), known at compile time so that the box predicates fold away.
template <int NA, int NB, int ES, int MINB, bool FULL>
__global__ void __launch_bounds__(kSlabThreads, MINB) ns_slab_inv_kernel(SlabArgs a) {
    using LA = SlabLine<NA>;
    using LB = SlabLine<NB>;
    constexpr int P1 = slab_pitch_c(NA / 2 + 1);
    constexpr int SL = P1 * NB;
    constexpr long long PLANE = (long long)NA * NB;
    extern __shared__ float2 sm[];
    float2* twA = sm;
    float2* twB = sm + NA;
    float2* S = sm + NA + NB;
    load_slab_twiddles<NA>(twA, a.twa);
    load_slab_twiddles<NB>(twB, a.twb);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nk1 = FULL ? NA / 2 + 1 : a.nk1, nk2 = FULL ? NB : a.nk2, b2 = FULL ? NB : a.b2;
    const int k2hi = NB - (nk2 - b2 - 1);   // first negative-frequency column in the box
    uint64_t* bar = slab_bar<NA, NB>(sm);
    uint32_t phase = 0;
    slab_bar_init(bar);
    const int per = a.nzc * a.n3;
    auto slab_src = [&](int unit) {
        const int ch = unit / per, ur = unit - ch * per;
        const int z = ur / a.n3, s3 = ur - z * a.n3;
        return a.spec + ch * a.spec_chstride + z * a.spec_zstride + (long long)s3 * SL;
    };
    const uint32_t colbytes = (uint32_t)(((nk1 + 1) & ~1) * sizeof(float2));
    bool requested = false;   // the unit's box was requested during the previous unit's C2R
    for (int u = blockIdx.x; u < a.units; u += gridDim.x) {
        const int ch = u / per, ur = u - ch * per;
        const int z = ur / a.n3, s3 = ur - z * a.n3;
        // the output slab (its offset may come from the item table: loaded ahead of the phases)
        float* out = a.vol + ch + a.vz.off(z) + (long long)s3 * PLANE * ES;
        // 1. the box of the slab into shared memory
        if (!requested) {
            slab_bulk_load<NB, P1>(S, slab_src(u), nk1, nk2, b2, bar, phase, a.status);
        } else {
            mbar_wait_bounded(bar, phase, a.status);
            phase ^= 1;
        }
        // the next unit of this CTA, whose box columns are requested as soon as their pair is transformed
        const int un = u + gridDim.x;
        requested = un < a.units;
        const float2* srcn = requested ? slab_src(un) : nullptr;
        // 2. inverse FFT along axis 2 of the rows k1 < nk1; columns outside the box are zero
        {
            const int p = lane & (LB::N2 - 1), s = lane / LB::N2;
            for (int base = 0; base < nk1; base += LB::LPR) {
                if (base + warp * LB::LPW >= nk1) continue;   // warp-uniform
                const int k1 = base + warp * LB::LPW + s;
                const bool valid = k1 < nk1;
                float2* row = S + (valid ? k1 : 0);
                float2 v[LB::N1];
#pragma unroll
                for (int r = 0; r < LB::N1; ++r) {
                    const int k2 = p + LB::N2 * r;
                    const bool in = valid && (k2 <= b2 || k2 >= k2hi);
                    v[r] = in ? row[P1 * k2] : make_float2(0.f, 0.f);
                }
                warp_line_fft<NB, true, P1>(v, p, valid, twB, row);
                if (valid) {
#pragma unroll
                    for (int j = 0; j < LB::M; ++j)
#pragma unroll
                        for (int k = 0; k < LB::N2; ++k) row[P1 * ((p + LB::N2 * j) + LB::N1 * k)] = v[j * LB::N2 + k];
                }
            }
        }
        // the row phase's accesses to every column ahead of the next unit's copies into them
        if (requested) fence_proxy_async();
        __syncthreads();
        // 3. C2R along axis 1, columns 2l and 2l+1 as one complex line; rows k1 >= nk1 are zero
        {
            const int p = lane & (LA::N2 - 1), s = pair_subline<NA>(lane / LA::N2);
            constexpr int npairs = NB / 2;
            for (int base = 0; base < npairs; base += LA::LPR) {
                if (base + warp * LA::LPW >= npairs) continue;   // warp-uniform
                const int l = base + warp * LA::LPW + s;
                const bool valid = l < npairs;
                float2* ca = S + P1 * (2 * (valid ? l : 0));
                float2* cb = ca + P1;
                float2 v[LA::N1];
#pragma unroll
                for (int r = 0; r < LA::N1; ++r) {
                    const int i = p + LA::N2 * r;
                    const int k = 2 * i <= NA ? i : NA - i;
                    float2 A = make_float2(0.f, 0.f), B = make_float2(0.f, 0.f);
                    if (valid && k < nk1) {
                        A = ca[k];
                        B = cb[k];
                    }
                    if (k == 0 || 2 * k == NA) {
                        A.y = 0.f;
                        B.y = 0.f;
                    }
                    v[r] = 2 * i <= NA ? make_float2(A.x - B.y, A.y + B.x) : make_float2(A.x + B.y, B.x - A.y);
                }
                warp_line_fft<NA, true, 1>(v, p, valid, twA, ca);
                if (requested) {
                    // the warp's columns are free (the exchange ended with a warp barrier): lane c of the
                    // first 2 LPW requests column 2 (base + warp LPW) + c of the next unit, if in its box
                    fence_proxy_async();
                    __syncwarp();
                    const int k2 = 2 * (base + warp * LA::LPW) + lane;
                    if (lane < 2 * LA::LPW && k2 < NB && (k2 <= b2 || k2 >= k2hi)) {
                        mbar_expect_tx(bar, colbytes);
                        bulk_load(S + P1 * k2, srcn + P1 * k2, colbytes, bar);
                    }
                }
                if (valid) {
                    float* oa = out + (long long)(2 * l) * NA * ES;
                    float* ob = oa + (long long)NA * ES;
                    const float sc = a.scale;
#pragma unroll
                    for (int j = 0; j < LA::M; ++j)
#pragma unroll
                        for (int k = 0; k < LA::N2; ++k) {
                            const int i1 = (p + LA::N2 * j) + LA::N1 * k;
                            const float2 w = c_scale(v[j * LA::N2 + k], sc);
                            oa[i1 * ES] = w.x;
                            ob[i1 * ES] = w.y;
                        }
                }
            }
        }
        __syncthreads();   // the slab buffer is reused by the next unit
        // every copy of the next unit is issued and announced: the one arrival of the barrier's phase
        if (requested && threadIdx.x == 0) mbar_arrive(bar);
    }
}

// Synthesis / rfft slab pass (forward): real volumes (element stride ES) ->
// spectra (the box rows).
template <int NA, int NB, int ES, int MINB, bool FULL>
__global__ void __launch_bounds__(kSlabThreads, MINB) ns_slab_fwd_kernel(SlabArgs a) {
    using LA = SlabLine<NA>;
    using LB = SlabLine<NB>;
    constexpr int P1 = slab_pitch_c(NA / 2 + 1);
    constexpr int SL = P1 * NB;
    constexpr long long PLANE = (long long)NA * NB;
    constexpr int H1 = NA / 2 + 1;
    constexpr int QA = (H1 + LA::N2 - 1) / LA::N2;   // output bins a lane unpacks
    extern __shared__ float2 sm[];
    float2* twA = sm;
    float2* twB = sm + NA;
    float2* S = sm + NA + NB;
    load_slab_twiddles<NA>(twA, a.twa);
    load_slab_twiddles<NB>(twB, a.twb);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // FULL: the box spans every row and column (as in the inverse pass)
    const int nk1 = FULL ? NA / 2 + 1 : a.nk1, nk2 = FULL ? NB : a.nk2, b2 = FULL ? NB : a.b2;
    for (int u = blockIdx.x; u < a.units; u += gridDim.x) {
        const int per = a.nzc * a.n3;
        const int ch = u / per, ur = u - ch * per;
        const int z = ur / a.n3, s3 = ur - z * a.n3;
        // 1. R2C along axis 1 of columns 2l, 2l+1 (as the real and imaginary parts of one line)
        {
            const int p = lane & (LA::N2 - 1), s = pair_subline<NA>(lane / LA::N2);
            constexpr int npairs = NB / 2;
            const float* in = a.vol + ch + a.vz.off(z) + (long long)s3 * PLANE * ES;
            for (int base = 0; base < npairs; base += LA::LPR) {
                if (base + warp * LA::LPW >= npairs) continue;   // warp-uniform
                const int l = base + warp * LA::LPW + s;
                const bool valid = l < npairs;
                const float* ia = in + (long long)(2 * (valid ? l : 0)) * NA * ES;
                const float* ib = ia + (long long)NA * ES;
                float2 v[LA::N1];
#pragma unroll
                for (int r = 0; r < LA::N1; ++r) {
                    const int i = p + LA::N2 * r;
                    v[r] = valid ? make_float2(ia[i * ES], ib[i * ES]) : make_float2(0.f, 0.f);
                }
                float2* ca = S + P1 * (2 * (valid ? l : 0));
                float2* cb = ca + P1;
                warp_line_fft<NA, false, 1>(v, p, valid, twA, ca);
                // Z in natural order through the pair's slots, then the two half spectra
                if (valid) {
#pragma unroll
                    for (int j = 0; j < LA::M; ++j)
#pragma unroll
                        for (int k = 0; k < LA::N2; ++k) ca[(p + LA::N2 * j) + LA::N1 * k] = v[j * LA::N2 + k];
                }
                __syncwarp();
                float2 ha[QA], hb[QA];
#pragma unroll
                for (int q = 0; q < QA; ++q) {
                    const int k = p + LA::N2 * q;
                    ha[q] = hb[q] = make_float2(0.f, 0.f);
                    if (valid && k < nk1) {
                        const float2 zk = ca[k];
                        const float2 zn = ca[k == 0 ? 0 : NA - k];
                        ha[q] = half_spec_a(zk, zn);
                        hb[q] = half_spec_b(zk, zn);
                    }
                }
                __syncwarp();
                if (valid) {
#pragma unroll
                    for (int q = 0; q < QA; ++q) {
                        const int k = p + LA::N2 * q;
                        if (k < nk1) {
                            ca[k] = ha[q];
                            cb[k] = hb[q];
                        }
                    }
                }
            }
        }
        __syncthreads();
        // 2. forward FFT along axis 2 of the rows k1 < nk1
        {
            const int p = lane & (LB::N2 - 1), s = lane / LB::N2;
            for (int base = 0; base < nk1; base += LB::LPR) {
                if (base + warp * LB::LPW >= nk1) continue;   // warp-uniform
                const int k1 = base + warp * LB::LPW + s;
                const bool valid = k1 < nk1;
                float2* row = S + (valid ? k1 : 0);
                float2 v[LB::N1];
#pragma unroll
                for (int r = 0; r < LB::N1; ++r) v[r] = valid ? row[P1 * (p + LB::N2 * r)] : make_float2(0.f, 0.f);
                warp_line_fft<NB, false, P1>(v, p, valid, twB, row);
                if (valid) {
#pragma unroll
                    for (int j = 0; j < LB::M; ++j)
#pragma unroll
                        for (int k = 0; k < LB::N2; ++k) row[P1 * ((p + LB::N2 * j) + LB::N1 * k)] = v[j * LB::N2 + k];
                }
            }
        }
        __syncthreads();
        // 3. the box of the slab out to the spectrum
        float2* dst = a.spec + ch * a.spec_chstride + z * a.spec_zstride + (long long)s3 * SL;
        slab_bulk_store<NB, P1>(dst, S, nk1, nk2, b2);   // ends with the barrier before S is reused
    }
}

// The denoiser's slab pass (real data): per slab of Y_s, the analysis half
// (inverse FFT along axis 2, C2R along axis 1, 1/N) gives the subband's slab
// in registers; it is soft-thresholded, c' = sign(c) max(|c| - tau_s, 0), and
// the synthesis half (R2C along axis 1, FFT along axis 2 of the box rows)
// writes the box back into the same slab of Y_s.  The subband itself never
// leaves the chip.  Same arithmetic, in the same order, as analyze ->
// threshold -> synthesize through the two slab passes.
template <int NA, int NB, int MINB>
__global__ void __launch_bounds__(kSlabThreads, MINB) ns_slab_shrink_kernel(SlabArgs a) {
    using LA = SlabLine<NA>;
    using LB = SlabLine<NB>;
    constexpr int P1 = slab_pitch_c(NA / 2 + 1);
    constexpr int SL = P1 * NB;
    constexpr int H1 = NA / 2 + 1;
    constexpr int QA = (H1 + LA::N2 - 1) / LA::N2;
    extern __shared__ float2 sm[];
    float2* twA = sm;
    float2* twB = sm + NA;
    float2* S = sm + NA + NB;
    load_slab_twiddles<NA>(twA, a.twa);
    load_slab_twiddles<NB>(twB, a.twb);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nk1 = a.nk1, nk2 = a.nk2, b2 = a.b2;
    const int k2hi = NB - (nk2 - b2 - 1);
    uint64_t* bar = slab_bar<NA, NB>(sm);
    uint32_t phase = 0;
    slab_bar_init(bar);
    for (int u = blockIdx.x; u < a.units; u += gridDim.x) {
        const int per = a.nzc * a.n3;
        const int ch = u / per, ur = u - ch * per;
        const int z = ur / a.n3, s3 = ur - z * a.n3;
        float2* slab = a.spec + ch * a.spec_chstride + z * a.spec_zstride + (long long)s3 * SL;
        const float tau = a.tau[a.items[a.item0 + z].s - 1];
        slab_bulk_load<NB, P1>(S, slab, nk1, nk2, b2, bar, phase, a.status);
        {   // inverse FFT along axis 2 of the box rows
            const int p = lane & (LB::N2 - 1), s = lane / LB::N2;
            for (int base = 0; base < nk1; base += LB::LPR) {
                if (base + warp * LB::LPW >= nk1) continue;   // warp-uniform
                const int k1 = base + warp * LB::LPW + s;
                const bool valid = k1 < nk1;
                float2* row = S + (valid ? k1 : 0);
                float2 v[LB::N1];
#pragma unroll
                for (int r = 0; r < LB::N1; ++r) {
                    const int k2 = p + LB::N2 * r;
                    const bool in = valid && (k2 <= b2 || k2 >= k2hi);
                    v[r] = in ? row[P1 * k2] : make_float2(0.f, 0.f);
                }
                warp_line_fft<NB, true, P1>(v, p, valid, twB, row);
                if (valid) {
#pragma unroll
                    for (int j = 0; j < LB::M; ++j)
#pragma unroll
                        for (int k = 0; k < LB::N2; ++k) row[P1 * ((p + LB::N2 * j) + LB::N1 * k)] = v[j * LB::N2 + k];
                }
            }
        }
        __syncthreads();
        {   // per column pair: C2R, threshold, R2C
            const int p = lane & (LA::N2 - 1), s = pair_subline<NA>(lane / LA::N2);
            constexpr int npairs = NB / 2;
            for (int base = 0; base < npairs; base += LA::LPR) {
                if (base + warp * LA::LPW >= npairs) continue;   // warp-uniform
                const int l = base + warp * LA::LPW + s;
                const bool valid = l < npairs;
                float2* ca = S + P1 * (2 * (valid ? l : 0));
                float2* cb = ca + P1;
                float2 v[LA::N1];
#pragma unroll
                for (int r = 0; r < LA::N1; ++r) {
                    const int i = p + LA::N2 * r;
                    const int k = 2 * i <= NA ? i : NA - i;
                    float2 A = make_float2(0.f, 0.f), B = make_float2(0.f, 0.f);
                    if (valid && k < nk1) {
                        A = ca[k];
                        B = cb[k];
                    }
                    if (k == 0 || 2 * k == NA) {
                        A.y = 0.f;
                        B.y = 0.f;
                    }
                    v[r] = 2 * i <= NA ? make_float2(A.x - B.y, A.y + B.x) : make_float2(A.x + B.y, B.x - A.y);
                }
                warp_line_fft<NA, true, 1>(v, p, valid, twA, ca);
                // the two subband columns, thresholded, in natural order through the pair's slots
                if (valid) {
#pragma unroll
                    for (int j = 0; j < LA::M; ++j)
#pragma unroll
                        for (int k = 0; k < LA::N2; ++k) {
                            const float2 c = v[j * LA::N2 + k];
                            const float xa = c.x * a.scale, xb = c.y * a.scale;
                            ca[(p + LA::N2 * j) + LA::N1 * k] =
                                make_float2(copysignf(fmaxf(fabsf(xa) - tau, 0.f), xa),
                                            copysignf(fmaxf(fabsf(xb) - tau, 0.f), xb));
                        }
                }
                __syncwarp();
#pragma unroll
                for (int r = 0; r < LA::N1; ++r) v[r] = valid ? ca[p + LA::N2 * r] : make_float2(0.f, 0.f);
                warp_line_fft<NA, false, 1>(v, p, valid, twA, ca);
                if (valid) {
#pragma unroll
                    for (int j = 0; j < LA::M; ++j)
#pragma unroll
                        for (int k = 0; k < LA::N2; ++k) ca[(p + LA::N2 * j) + LA::N1 * k] = v[j * LA::N2 + k];
                }
                __syncwarp();
                float2 ha[QA], hb[QA];
#pragma unroll
                for (int q = 0; q < QA; ++q) {
                    const int k = p + LA::N2 * q;
                    ha[q] = hb[q] = make_float2(0.f, 0.f);
                    if (valid && k < nk1) {
                        const float2 zk = ca[k];
                        const float2 zn = ca[k == 0 ? 0 : NA - k];
                        ha[q] = half_spec_a(zk, zn);
                        hb[q] = half_spec_b(zk, zn);
                    }
                }
                __syncwarp();
                if (valid) {
#pragma unroll
                    for (int q = 0; q < QA; ++q) {
                        const int k = p + LA::N2 * q;
                        if (k < nk1) {
                            ca[k] = ha[q];
                            cb[k] = hb[q];
                        }
                    }
                }
            }
        }
        __syncthreads();
        {   // forward FFT along axis 2 of the box rows
            const int p = lane & (LB::N2 - 1), s = lane / LB::N2;
            for (int base = 0; base < nk1; base += LB::LPR) {
                if (base + warp * LB::LPW >= nk1) continue;   // warp-uniform
                const int k1 = base + warp * LB::LPW + s;
                const bool valid = k1 < nk1;
                float2* row = S + (valid ? k1 : 0);
                float2 v[LB::N1];
#pragma unroll
                for (int r = 0; r < LB::N1; ++r) v[r] = valid ? row[P1 * (p + LB::N2 * r)] : make_float2(0.f, 0.f);
                warp_line_fft<NB, false, P1>(v, p, valid, twB, row);
                if (valid) {
#pragma unroll
                    for (int j = 0; j < LB::M; ++j)
#pragma unroll
                        for (int k = 0; k < LB::N2; ++k) row[P1 * ((p + LB::N2 * j) + LB::N1 * k)] = v[j * LB::N2 + k];
                }
            }
        }
        __syncthreads();
        slab_bulk_store<NB, P1>(slab, S, nk1, nk2, b2);   // ends with the barrier before S is reused
    }
}

// ── launch tables ────────────────────────────────────────────────────────────

template <int N>
constexpr int slab_minb() {
    return LinePlan<N>::N1 <= 16 ? 2 : 1;
}

// One CTA a unit up to the resident capacity; CTAs stride over the rest.
// KIND: 0 the forward slab pass, 1 the inverse, 2 the denoiser's shrink pass.
template <int KIND, int NA, int NB, int ES, bool FULL>
void launch_slab_es(const SlabArgs& a, int sms, size_t smem, cudaStream_t st, const char* tag) {
    constexpr int MINB = (slab_minb<NA>() == 2 && slab_minb<NB>() == 2) ? 2 : 1;
    auto kern = KIND == 1 ? ns_slab_inv_kernel<NA, NB, ES, MINB, FULL>
                          : (KIND == 0 ? ns_slab_fwd_kernel<NA, NB, ES, MINB, FULL> : ns_slab_shrink_kernel<NA, NB, MINB>);
    static size_t configured = 0;
    static int resident = 0;
    if (configured < smem) {
        cuda_check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                   "cudaFuncSetAttribute(slab)");
        configured = smem;
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kern, kSlabThreads, smem),
                   "cudaOccupancyMaxActiveBlocksPerMultiprocessor(slab)");
        resident = std::max(resident, 1);
    }
    const int grid = std::max(1, std::min(a.units, resident * sms));
    int tok = prof_begin(tag, st);
    kern<<<grid, kSlabThreads, smem, st>>>(a);
    prof_end(tok, st);
    cuda_check(cudaGetLastError(), "slab kernel launch");
}

template <int KIND, int NA, int NB>
void launch_slab_nn(const SlabArgs& a, int sms, size_t smem, cudaStream_t st, const char* tag) {
    if (a.P1 != slab_pitch_c(NA / 2 + 1)) throw ArgError("slab pitch mismatch");
    const bool full = KIND != 2 && a.nk1 == NA / 2 + 1 && a.nk2 == NB;
    if (a.es == 1) {
        if (full)
            launch_slab_es<KIND, NA, NB, 1, true>(a, sms, smem, st, tag);
        else
            launch_slab_es<KIND, NA, NB, 1, false>(a, sms, smem, st, tag);
    } else {
        if (full)
            launch_slab_es<KIND, NA, NB, 2, true>(a, sms, smem, st, tag);
        else
            launch_slab_es<KIND, NA, NB, 2, false>(a, sms, smem, st, tag);
    }
}

template <int KIND, int NA>
bool launch_slab_n(int nb, const SlabArgs& a, int sms, size_t smem, cudaStream_t st, const char* tag) {
    switch (nb) {
        case 64: launch_slab_nn<KIND, NA, 64>(a, sms, smem, st, tag); return true;
        case 96: launch_slab_nn<KIND, NA, 96>(a, sms, smem, st, tag); return true;
        case 128: launch_slab_nn<KIND, NA, 128>(a, sms, smem, st, tag); return true;
        case 160: launch_slab_nn<KIND, NA, 160>(a, sms, smem, st, tag); return true;
        case 256:
            if constexpr (NA != 256) {   // 256 x 256 slabs run on clusters (ns_slab_cluster.cu)
                launch_slab_nn<KIND, NA, 256>(a, sms, smem, st, tag);
                return true;
            }
            return false;
    }
    return false;
}

template <int KIND>
void launch_slab(int na, int nb, const SlabArgs& a, int sms, size_t smem, cudaStream_t st, const char* tag) {
    if (slab_cluster_supported(na, nb)) {
        if (!launch_slab_cluster(KIND, na, nb, a, sms, st, tag)) throw ArgError("no slab kernel for this size");
        return;
    }
    bool ok = false;
    switch (na) {
        case 64: ok = launch_slab_n<KIND, 64>(nb, a, sms, smem, st, tag); break;
        case 96: ok = launch_slab_n<KIND, 96>(nb, a, sms, smem, st, tag); break;
        case 128: ok = launch_slab_n<KIND, 128>(nb, a, sms, smem, st, tag); break;
        case 160: ok = launch_slab_n<KIND, 160>(nb, a, sms, smem, st, tag); break;
        case 256: ok = launch_slab_n<KIND, 256>(nb, a, sms, smem, st, tag); break;
    }
    if (!ok) throw ArgError("no slab kernel for this size");
}

bool slab_len(int n) { return n == 64 || n == 96 || n == 128 || n == 160 || n == 256; }

int slab_pitch(int h1) { return slab_pitch_c(h1); }

size_t slab_smem(int n1, int n2) {
    return sizeof(float2) * ((size_t)n1 + n2 + (size_t)slab_pitch(n1 / 2 + 1) * n2) + 16;   // + the mbarrier
}

// ── drivers ──────────────────────────────────────────────────────────────────

BoxMap box_map(const NSPlan& P, const NSBox& b) { return BoxMap{b.nk1, b.nk2, b.b2, P.dims[1]}; }

const NSBox& item_box(const NSPlan& P, int item) {
    const NSItem& it = P.items_host[item];
    return P.boxes[it.kind == 1 ? (int)P.boxes.size() - 1 : it.g];
}

SlabArgs slab_args(const NSPlan& P, const NSBox& b, int nz) {
    SlabArgs a{};
    a.P1 = P.P1;
    a.n3 = P.dims[2];
    a.nk1 = b.nk1;
    a.nk2 = b.nk2;
    a.b2 = b.b2;
    a.units = nz * P.dims[2];
    a.nzc = nz;
    a.spec_chstride = 0;
    a.twa = P.ffts.at(P.dims[0])->sh.tw;
    a.twb = P.ffts.at(P.dims[1])->sh.tw;
    a.es = 1;
    a.scale = 1.f;
    a.status = P.status.dev;
    return a;
}

template <bool INV, class Load, class Store>
void line3(const NSPlan& P, const Load& ld, const Store& so, int nlines, int nz, cudaStream_t st, const char* tag) {
    const FFTLen* f = P.ffts.at(P.dims[2]).get();
    if (!launch_reg<INV>(P.dims[2], ld, so, f->sh.tw, nlines, nz, true, st, tag))
        throw ArgError("no register line pass for axis 3 of this size");
}

template <int N>
void launch_slab_accum(const NSPlan& P, const float2* Y, int nz, const BoxMap& bx, int i0, int synth, float2* acc,
                       float2* comp, int nlines, int nch, long long ychs, long long achs, int nbq, cudaStream_t st) {
    using Ge = RegGeom<N>;
    static bool configured = false;
    if (!configured) {
        cuda_check(cudaFuncSetAttribute(ns_slab_accum_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)accum_smem<N>()),
                   "cudaFuncSetAttribute");
        configured = true;
    }
    dim3 grid((nlines + Ge::LP - 1) / Ge::LP, nch);
    int tok = prof_begin("ns_slab_accum_axis3", st);
    ns_slab_accum_kernel<N><<<grid, Ge::THREADS, accum_smem<N>(), st>>>(Y, P.SP, nz, P.P1, P.P1 * P.dims[1], bx, P.tb,
                                                                 P.items.as<NSItem>(), i0, synth, acc, comp,
                                                                 P.ffts.at(P.dims[2])->sh.tw, nlines, ychs, achs, nbq);
    prof_end(tok, st);
    cuda_check(cudaGetLastError(), "ns_slab_accum_kernel launch");
}

template <int N, int IPC>
void launch_mask_group_ipc(const NSPlan& P, const float2* X, float2* Y, int nz, const BoxMap& bx, int i0, int synth,
                           int nlines, int nch, long long xchs, long long ychs, int nbq, cudaStream_t st) {
    using Ge = RegGeom<N>;
    static bool configured = false;
    if (!configured) {
        cuda_check(cudaFuncSetAttribute(ns_slab_mask_group_kernel<N, IPC>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Ge::SMEM),
                   "cudaFuncSetAttribute");
        configured = true;
    }
    const int nblocks = (nlines + Ge::LP - 1) / Ge::LP, ny = (nz + IPC - 1) / IPC;
    dim3 grid(nblocks, ny, nch);
    int tok = prof_begin("ns_slab_mask_axis3", st);
    ns_slab_mask_group_kernel<N, IPC><<<grid, Ge::THREADS, Ge::SMEM, st>>>(
        X, P.P1, P.P1 * P.dims[1], bx, P.tb, P.items.as<NSItem>(), i0, nz, synth, Y, P.SP,
        P.ffts.at(P.dims[2])->sh.tw, nlines, xchs, ychs, nbq);
    prof_end(tok, st);
    cuda_check(cudaGetLastError(), "ns_slab_mask_group_kernel launch");
}

thread_local bool t_concurrent = false;

// Subbands a CTA of the analysis axis-3 pass (the line's X and group factor
// are loaded once for all of them).  An explicit choice is taken as given:
// the plan's (the autotuner's tile), else SFL_MASK_IPC (1, 2, 4 or 8) from
// the environment, read once.  By default up to 8 (a finest-scale group of
// [2,2,3] in one CTA: 2027 vs 2013 Mvox/s for 4 on the bench workload),
// and for launches that run alone halved while the launch would hold fewer
// CTAs than the GPU has SMs (the small boxes of coarse scales: 30 line blocks
// at 128^3 [2,2,3] scale 1): the pass 3.32 -> 2.93 ms a step of eight volumes
// as plain calls, but 2038 -> 2031 Mvox/s in the four-branch graph, where the
// other branches fill the GPU and the split CTAs only reload X.
int mask_ipc(const NSPlan& P, int nz, int nblocks) {
    static const int env_cap = [] {
        const char* e = std::getenv("SFL_MASK_IPC");
        if (!e) return 0;
        const int v = std::atoi(e);
        return v >= 8 ? 8 : (v >= 4 ? 4 : (v >= 2 ? 2 : 1));
    }();
    const int cap = P.ipc > 0 ? P.ipc : (env_cap > 0 ? env_cap : 8);
    const int m = std::min(nz, cap);
    int ipc = m >= 8 ? 8 : (m >= 4 ? 4 : (m >= 2 ? 2 : 1));
    if (P.ipc <= 0 && env_cap == 0 && !t_concurrent)
        while (ipc > 1 && (long long)nblocks * ((nz + ipc - 1) / ipc) < P.sms) ipc /= 2;
    return ipc;
}

template <int N>
void launch_mask_group(const NSPlan& P, const float2* X, float2* Y, int nz, const BoxMap& bx, int i0, int synth,
                       int nlines, int nch, long long xchs, long long ychs, int nbq, cudaStream_t st) {
    switch (mask_ipc(P, nz, (nlines + RegGeom<N>::LP - 1) / RegGeom<N>::LP)) {
        case 8: launch_mask_group_ipc<N, 8>(P, X, Y, nz, bx, i0, synth, nlines, nch, xchs, ychs, nbq, st); return;
        case 4: launch_mask_group_ipc<N, 4>(P, X, Y, nz, bx, i0, synth, nlines, nch, xchs, ychs, nbq, st); return;
        case 2: launch_mask_group_ipc<N, 2>(P, X, Y, nz, bx, i0, synth, nlines, nch, xchs, ychs, nbq, st); return;
        default: launch_mask_group_ipc<N, 1>(P, X, Y, nz, bx, i0, synth, nlines, nch, xchs, ychs, nbq, st); return;
    }
}

// Items [i0, i0 + nz) as nbq plane-b wedges times whole rows of plane-a
// wedges constant along axis 3 (item t = p nbq + q, one mask group): nbq,
// else 0.  Only then do the axis-3 passes share FFTs between items.
int chunk_nbq(const NSPlan& P, int i0, int nz, bool synth_masks) {
    if (nz < 2 || (synth_masks && !P.p.tight)) return 0;
    const NSItem& f = P.items_host[i0];
    if (f.kind != 0 || f.wa_hi == 2) return 0;
    int nb = 1;
    while (nb < nz && P.items_host[i0 + nb].wb_off != f.wb_off) ++nb;
    if (nz % nb != 0) return 0;
    for (int t = 0; t < nz; ++t) {
        const NSItem& it = P.items_host[i0 + t];
        if (it.kind != 0 || it.g != f.g || it.wa_hi == 2 || it.wb_off != P.items_host[i0 + t % nb].wb_off ||
            it.wa_off != P.items_host[i0 + (t / nb) * nb].wa_off)
            return 0;
    }
    return nb;
}

// Algorithmic bytes of one box of a spectrum (complex float32 bins).
double box_bytes(const NSPlan& P, const NSBox& b) { return 8.0 * b.nk1 * b.nk2 * P.dims[2]; }

// Channels: complex volumes run their two real channels in the same launches
// (spectra and intermediates one block per channel, the volume's channels
// interleaved floats), with each channel's arithmetic that of a real volume.
// Y blocks: channel ch of item z at work + ch * (group SP) + z * SP.
long long ych_stride(const NSPlan& P) { return (long long)P.group * P.SP; }

// rfft3 of nch interleaved real channels (element stride es) into the padded
// spectra X + ch SP.
void slab_rfft3(NSPlan& P, const float* x, int es, float2* X, int nch, cudaStream_t st) {
    const NSBox& full = P.boxes_full;
    prof_bytes("ns_slab_r2c", nch * (4.0 * P.N + box_bytes(P, full)));
    prof_bytes("ns_slab_line3", nch * 2 * box_bytes(P, full));
    SlabArgs a = slab_args(P, full, 1);
    a.units *= nch;
    a.spec_chstride = P.SP;
    a.spec = X;
    a.vol = const_cast<float*>(x);
    a.es = es;
    launch_slab<0>(P.dims[0], P.dims[1], a, P.sms, slab_smem(P.dims[0], P.dims[1]), st, "ns_slab_r2c");
    const BoxMap bx = box_map(P, full);
    const int s3 = P.P1 * P.dims[1];
    line3<false>(P, L3LoadC{X, P.SP, P.P1, s3, bx}, L3StoreC{X, P.SP, P.P1, s3, bx}, full.nk1 * full.nk2, nch, st,
                 "ns_slab_line3");
}

// irfft3 of the padded spectra A + ch SP (overwritten) into nch channels.
void slab_irfft3(NSPlan& P, float2* A, float* x, int es, int nch, cudaStream_t st) {
    const NSBox& full = P.boxes_full;
    prof_bytes("ns_slab_line3", nch * 2 * box_bytes(P, full));
    prof_bytes("ns_slab_c2r", nch * (box_bytes(P, full) + 4.0 * P.N));
    const BoxMap bx = box_map(P, full);
    const int s3 = P.P1 * P.dims[1];
    line3<true>(P, L3LoadC{A, P.SP, P.P1, s3, bx}, L3StoreC{A, P.SP, P.P1, s3, bx}, full.nk1 * full.nk2, nch, st,
                "ns_slab_line3");
    SlabArgs a = slab_args(P, full, 1);
    a.units *= nch;
    a.spec_chstride = P.SP;
    a.spec = A;
    a.vol = x;
    a.es = es;
    a.scale = 1.0f / (float)P.N;
    launch_slab<1>(P.dims[0], P.dims[1], a, P.sms, slab_smem(P.dims[0], P.dims[1]), st, "ns_slab_c2r");
}

// The analysis axis-3 pass of items [i0, i0 + nz) (one mask group): X times
// each mask, inverse FFT along axis 3, into Y (the plan's work spectra).
void slab_mask_pass(NSPlan& P, const float2* X, int i0, int nz, bool synth_masks, int nch, cudaStream_t st) {
    const NSBox& b = item_box(P, i0);
    const BoxMap bx = box_map(P, b);
    float2* Y = P.work.as<float2>();
    prof_bytes("ns_slab_mask_axis3", nch * (1.5 * box_bytes(P, b) + nz * box_bytes(P, b)));
    const int nl = b.nk1 * b.nk2, sy = synth_masks ? 1 : 0;
    const long long xc = P.SP, yc = ych_stride(P);
    const int nbq = chunk_nbq(P, i0, nz, synth_masks);
    switch (P.dims[2]) {
        case 16: launch_mask_group<16>(P, X, Y, nz, bx, i0, sy, nl, nch, xc, yc, nbq, st); return;
        case 32: launch_mask_group<32>(P, X, Y, nz, bx, i0, sy, nl, nch, xc, yc, nbq, st); return;
        case 64: launch_mask_group<64>(P, X, Y, nz, bx, i0, sy, nl, nch, xc, yc, nbq, st); return;
        case 96: launch_mask_group<96>(P, X, Y, nz, bx, i0, sy, nl, nch, xc, yc, nbq, st); return;
        case 128: launch_mask_group<128>(P, X, Y, nz, bx, i0, sy, nl, nch, xc, yc, nbq, st); return;
        case 160: launch_mask_group<160>(P, X, Y, nz, bx, i0, sy, nl, nch, xc, yc, nbq, st); return;
        case 256: launch_mask_group<256>(P, X, Y, nz, bx, i0, sy, nl, nch, xc, yc, nbq, st); return;
    }
    throw ArgError("no register line pass for axis 3 of this size");
}

// The synthesis axis-3 pass of items [i0, i0 + nz) from Y into acc + ch SP,
// Kahan-compensated through comp + ch SP.
void slab_accum_pass(NSPlan& P, int i0, int nz, bool analysis_masks, float2* acc, float2* comp, int nch,
                     cudaStream_t st) {
    const NSBox& b = item_box(P, i0);
    const float2* Y = P.work.as<float2>();
    // Y once per item, the group table (4 B a bin), the accumulator and its compensation in and out
    prof_bytes("ns_slab_accum_axis3", nch * (nz * box_bytes(P, b) + 0.5 * box_bytes(P, b) + 4 * box_bytes(P, b)));
    const BoxMap bx = box_map(P, b);
    const int nl = b.nk1 * b.nk2;
    const int sy = analysis_masks ? 0 : 1;
    const long long yc = ych_stride(P), ac = P.SP;
    const int nbq = chunk_nbq(P, i0, nz, !analysis_masks);
    switch (P.dims[2]) {
        case 16: launch_slab_accum<16>(P, Y, nz, bx, i0, sy, acc, comp, nl, nch, yc, ac, nbq, st); return;
        case 32: launch_slab_accum<32>(P, Y, nz, bx, i0, sy, acc, comp, nl, nch, yc, ac, nbq, st); return;
        case 64: launch_slab_accum<64>(P, Y, nz, bx, i0, sy, acc, comp, nl, nch, yc, ac, nbq, st); return;
        case 96: launch_slab_accum<96>(P, Y, nz, bx, i0, sy, acc, comp, nl, nch, yc, ac, nbq, st); return;
        case 128: launch_slab_accum<128>(P, Y, nz, bx, i0, sy, acc, comp, nl, nch, yc, ac, nbq, st); return;
        case 160: launch_slab_accum<160>(P, Y, nz, bx, i0, sy, acc, comp, nl, nch, yc, ac, nbq, st); return;
        case 256: launch_slab_accum<256>(P, Y, nz, bx, i0, sy, acc, comp, nl, nch, yc, ac, nbq, st); return;
    }
    throw ArgError("no register line pass for axis 3 of this size");
}

// Analysis of items [i0, i0 + nz) (one mask group) from X (+ ch SP) into
// volumes at vol + vz.off(z) (+ ch, element stride es).
void slab_analyze_items(NSPlan& P, const float2* X, float* vol, ZMap vz, int es, int i0, int nz, bool synth_masks,
                        int nch, cudaStream_t st) {
    const NSBox& b = item_box(P, i0);
    slab_mask_pass(P, X, i0, nz, synth_masks, nch, st);
    prof_bytes("ns_slab_c2r", nch * nz * (box_bytes(P, b) + 4.0 * P.N));
    SlabArgs a = slab_args(P, b, nz);
    a.units *= nch;
    a.spec_chstride = ych_stride(P);
    a.spec = P.work.as<float2>();
    a.spec_zstride = P.SP;
    a.vol = vol;
    a.vz = vz;
    a.es = es;
    a.scale = 1.0f / (float)P.N;
    launch_slab<1>(P.dims[0], P.dims[1], a, P.sms, slab_smem(P.dims[0], P.dims[1]), st, "ns_slab_c2r");
}

// Synthesis staging of items [i0, i0 + nz) (one mask group) read from
// vol + vz.off(z) (+ ch): slab R2C into work slots slot0.. (+ ch group SP).
void slab_stage_items(NSPlan& P, const float* vol, ZMap vz, int es, int i0, int nz, int slot0, int nch,
                      cudaStream_t st) {
    const NSBox& b = item_box(P, i0);
    prof_bytes("ns_slab_r2c", nch * nz * (4.0 * P.N + box_bytes(P, b)));
    SlabArgs a = slab_args(P, b, nz);
    a.units *= nch;
    a.spec_chstride = ych_stride(P);
    a.spec = P.work.as<float2>() + (long long)slot0 * P.SP;
    a.spec_zstride = P.SP;
    a.vol = const_cast<float*>(vol);
    a.vz = vz;
    a.es = es;
    launch_slab<0>(P.dims[0], P.dims[1], a, P.sms, slab_smem(P.dims[0], P.dims[1]), st, "ns_slab_r2c");
}

// Synthesis accumulation of items [i0, i0 + nz) (one mask group) read from
// vol + vz.off(z) (+ ch) into acc + ch SP.
void slab_synth_items(NSPlan& P, const float* vol, ZMap vz, int es, int i0, int nz, bool analysis_masks,
                      float2* acc, float2* comp, int nch, cudaStream_t st) {
    slab_stage_items(P, vol, vz, es, i0, nz, 0, nch, st);
    slab_accum_pass(P, i0, nz, analysis_masks, acc, comp, nch, st);
}

// The denoiser on items [i0, i0 + nz) (one mask group; real data): the
// analysis axis-3 pass into Y, the shrink slab pass in place, the synthesis
// accumulation.
void slab_denoise_items(NSPlan& P, const float2* X, int i0, int nz, const float* tau, float2* acc, float2* comp,
                        cudaStream_t st) {
    const NSBox& b = item_box(P, i0);
    slab_mask_pass(P, X, i0, nz, false, 1, st);
    prof_bytes("ns_slab_shrink", nz * 2 * box_bytes(P, b));
    SlabArgs a = slab_args(P, b, nz);
    a.spec = P.work.as<float2>();
    a.spec_zstride = P.SP;
    a.scale = 1.0f / (float)P.N;
    a.tau = tau;
    a.items = P.items.as<NSItem>();
    a.item0 = i0;
    launch_slab<2>(P.dims[0], P.dims[1], a, P.sms, slab_smem(P.dims[0], P.dims[1]), st, "ns_slab_shrink");
    slab_accum_pass(P, i0, nz, false, acc, comp, 1, st);
}

// Consecutive items of one mask group, at most P.group of them.
int chunk_end(const NSPlan& P, int i0) {
    auto key = [&](int i) { return P.items_host[i].kind == 1 ? -1 : P.items_host[i].g; };
    int i1 = i0 + 1;
    while (i1 < P.S && i1 - i0 < P.group && key(i1) == key(i0)) ++i1;
    return i1;
}

}  // namespace

void ns_set_concurrent(bool on) { t_concurrent = on; }

bool ns_slab_supported(int n1, int n2, int n3) {
    if (!reg_fft_supported(n3)) return false;
    // one CTA a slab where the slab fits its shared memory (two CTAs an SM up to 112 KB, one above),
    // else two-CTA clusters
    return (slab_len(n1) && slab_len(n2) && slab_smem(n1, n2) <= kSlabSmemOneCta) || slab_cluster_resident(n1, n2);
}

// Support box of a table on the rfft grid (h1, n2, n3), k1 fastest.
NSBox ns_table_box(const std::vector<double>& g, int h1, int n2, int n3) {
    int m1 = -1, m2 = -1;
    for (int k3 = 0; k3 < n3; ++k3)
        for (int k2 = 0; k2 < n2; ++k2) {
            const double* row = g.data() + (size_t)h1 * (k2 + (size_t)n2 * k3);
            for (int k1 = 0; k1 < h1; ++k1)
                if (row[k1] != 0.0) {
                    m1 = std::max(m1, k1);
                    m2 = std::max(m2, std::min(k2, n2 - k2));
                }
        }
    return ns_make_box(m1 + 1, m2, n2);
}

NSBox ns_make_box(int nk1, int b2, int n2) {
    NSBox b;
    b.nk1 = std::max(nk1, 1);
    if (b2 < 0) b2 = 0;
    if (2 * b2 + 1 >= n2) {
        b.nk2 = n2;
        b.b2 = n2;
    } else {
        b.nk2 = 2 * b2 + 1;
        b.b2 = b2;
    }
    return b;
}

void ns_use_slabs(NSPlan& P) {
    if (!ns_slab_supported(P.dims[0], P.dims[1], P.dims[2]))
        throw ArgError("the slab pipeline does not support size " + std::to_string(P.dims[0]) + "x" +
                       std::to_string(P.dims[1]) + "x" + std::to_string(P.dims[2]));
    P.slab = true;
    ns_alloc_scratch(P);
}

void ns_slab_rfft3(NSPlan& P, const float* x, int es, float2* X, cudaStream_t st) { slab_rfft3(P, x, es, X, 1, st); }

void ns_slab_irfft3(NSPlan& P, float2* A, float* x, int es, cudaStream_t st) { slab_irfft3(P, A, x, es, 1, st); }

// Whole transforms, both channels of complex data in every launch.
void ns_slab_analyze(NSPlan& P, const void* x, void* c, cudaStream_t st, bool synth_masks) {
    const int nch = P.nch;
    float2* X = P.X.as<float2>();
    slab_rfft3(P, static_cast<const float*>(x), nch, X, nch, st);
    for (int i0 = 0, i1; i0 < P.S; i0 = i1) {
        i1 = chunk_end(P, i0);
        slab_analyze_items(P, X, static_cast<float*>(c), ns_subband_map(P, i0, nch), nch, i0, i1 - i0, synth_masks,
                           nch, st);
    }
}

void ns_slab_synthesize(NSPlan& P, const void* c, void* x, cudaStream_t st, bool analysis_masks) {
    const int nch = P.nch;
    float2* A = P.acc.as<float2>();
    float2* K = P.comp.as<float2>();
    cuda_check(cudaMemsetAsync(A, 0, sizeof(float2) * P.SP * nch, st), "cudaMemsetAsync(acc)");
    cuda_check(cudaMemsetAsync(K, 0, sizeof(float2) * P.SP * nch, st), "cudaMemsetAsync(comp)");
    for (int i0 = 0, i1; i0 < P.S; i0 = i1) {
        i1 = chunk_end(P, i0);
        slab_synth_items(P, static_cast<const float*>(c), ns_subband_map(P, i0, nch), nch, i0, i1 - i0,
                         analysis_masks, A, K, nch, st);
    }
    slab_irfft3(P, A, static_cast<float*>(x), nch, nch, st);
}

int ns_slab_chunk_end(const NSPlan& P, int i0) { return chunk_end(P, i0); }

void ns_slab_analyze_items(NSPlan& P, const float2* X, float* vol, ZMap vz, int es, int i0, int nz, bool synth_masks,
                           cudaStream_t st) {
    slab_analyze_items(P, X, vol, vz, es, i0, nz, synth_masks, 1, st);
}

void ns_slab_synth_items(NSPlan& P, const float* vol, ZMap vz, int es, int i0, int nz, bool analysis_masks,
                         float2* acc, float2* comp, cudaStream_t st) {
    slab_synth_items(P, vol, vz, es, i0, nz, analysis_masks, acc, comp, 1, st);
}

void ns_slab_denoise_items(NSPlan& P, const float2* X, int i0, int nz, const float* tau, float2* acc, float2* comp,
                           cudaStream_t st) {
    slab_denoise_items(P, X, i0, nz, tau, acc, comp, st);
}

void ns_slab_stage_items(NSPlan& P, const float* vol, ZMap vz, int es, int i0, int nz, int slot0, int nch,
                         cudaStream_t st) {
    slab_stage_items(P, vol, vz, es, i0, nz, slot0, nch, st);
}

void ns_slab_accum_items(NSPlan& P, int i0, int nz, bool analysis_masks, float2* acc, float2* comp, int nch,
                         cudaStream_t st) {
    slab_accum_pass(P, i0, nz, analysis_masks, acc, comp, nch, st);
}

}  // namespace sfl
