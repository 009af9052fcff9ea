// Slab passes for slabs too large for one CTA's shared memory (256 x 256 and
// up: 130 x 256 complex bins are 266 KB), split over the two CTAs of a
// thread-block cluster through distributed shared memory.
//
// CTA rank 0 of a cluster holds the rows k1 < R of the slab's box, rank 1
// the rows k1 >= R (R = NA/4, even, so that both blocks of a column start on
// a 16-byte boundary and move by one cp.async.bulk each), at
// S[(k1 - r R) + PL k2] in its own shared memory (PL = 2 mod 4).  The axis-2 phase (a row's FFT) is local: each CTA
// transforms its own rows.  The axis-1 phase (the C2R / R2C of a column pair)
// needs all h1 rows of two columns: CTA r takes the column pairs
// [r NB/4, (r + 1) NB/4) and reads (or writes) the rows of the other half in
// the peer's shared memory; its line exchange goes through a per-line
// scratch of its own.  Cluster barriers (arrive.release / wait.acquire)
// separate the phases that touch the peer's rows; the two CTAs of a cluster
// step through the same units, so every barrier is met by both.
//
// Per unit (one axis-3 slab of one item), same arithmetic and order as the
// one-CTA slab passes of ns_slab.cu:
//   inverse  load own box rows; IFFT_2 own rows; | C2R of own column pairs
//            (rows from both CTAs) to the volume; |
//   forward  R2C of own column pairs, half spectra into both CTAs' rows; |
//            FFT_2 own rows, out to the spectrum; |
//   shrink   load; IFFT_2; | per own pair: C2R, threshold, R2C, back into
//            both CTAs' rows; | FFT_2 own rows, out.
// (| = cluster barrier.)
#include <algorithm>
#include <cooperative_groups.h>

#include "prof.h"
#include "slab_core.cuh"
#include "tma.cuh"

namespace cg = cooperative_groups;

namespace sfl {

namespace {

constexpr int kClusterCTAs = 2;

template <int NA, int NB>
struct ClusterSlab {
    static constexpr int H1 = NA / 2 + 1;
    static constexpr int R = NA / 4;                                // rows of rank 0; rank 1 has H1 - R
    static constexpr int PL = slab_pitch_c(H1 - R);
    static constexpr int P1 = slab_pitch_c(H1);                     // pitch of the spectra in HBM
    static constexpr int PAIRS = NB / 2 / kClusterCTAs;             // column pairs a CTA
    static constexpr int LINES = kSlabWarps * SlabLine<NA>::LPW;    // axis-1 lines in flight a CTA
    // twiddles (NA + NB), the rows (PL NB), the axis-1 exchange (LINES NA), the mbarrier
    static constexpr size_t SMEM =
        sizeof(float2) * ((size_t)NA + NB + (size_t)PL * NB + (size_t)LINES * NA) + 16;
    static_assert(R % 2 == 0 && PL >= R && PL >= H1 - R + 1, "cluster slab row split");
};

__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" "barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// Own box rows k1 in [r0, r0 + rn) of a slab (pitch P1 in HBM) into S, one
// cp.async.bulk a box column of the rows rounded up to an even count (r0 is
// even and P1 even, so both ends are 16-byte aligned; the extra bin lies
// outside the box, or is the padding bin, and is read by no one).
template <int NB, int P1, int PL>
__device__ __forceinline__ void load_rows(float2* S, const float2* src, int r0, int rn, int nk2, int b2,
                                          uint64_t* bar, uint32_t& phase, int* status) {
    const uint32_t bytes = rn > 0 ? (uint32_t)(((rn + 1) & ~1) * sizeof(float2)) : 0u;
    fence_proxy_async();   // this thread's earlier accesses to S ahead of the copies' writes
    if (threadIdx.x == 0) mbar_arrive_expect_tx(bar, bytes * (uint32_t)nk2);
    __syncthreads();
    if (bytes && (int)threadIdx.x < nk2) {
        const int j = threadIdx.x;
        const int k2 = j <= b2 ? j : j + (NB - nk2);
        bulk_load(S + PL * k2, src + r0 + P1 * k2, bytes, bar);
    }
    mbar_wait_bounded(bar, phase, status);
    phase ^= 1;
}

// Own box rows back to the slab in HBM.  A column's copy covers the rows
// rounded up to an even count: with rank 0's rows all of [0, R) when the box
// reaches rank 1 (R even), so no copy writes a bin of the other CTA.
template <int NB, int P1, int PL>
__device__ __forceinline__ void store_rows(float2* dst, const float2* S, int r0, int rn, int nk2, int b2) {
    const uint32_t bytes = rn > 0 ? (uint32_t)(((rn + 1) & ~1) * sizeof(float2)) : 0u;
    fence_proxy_async();   // this thread's writes of S visible to the copies
    __syncthreads();
    if (bytes && (int)threadIdx.x < nk2) {
        const int j = threadIdx.x;
        const int k2 = j <= b2 ? j : j + (NB - nk2);
        bulk_store(dst + r0 + P1 * k2, S + PL * k2, bytes);
        bulk_commit();
        bulk_wait_read();   // S is rewritten by the next unit
    }
    __syncthreads();
}

// FFT along axis 2 of the own rows kl < rn; on the inverse, the columns
// outside the box read as zero.
template <int NB, int PL, bool INV>
__device__ __forceinline__ void rows_fft(float2* S, const float2* twB, int rn, int nk2, int b2, int warp, int lane) {
    using LB = SlabLine<NB>;
    const int k2hi = NB - (nk2 - b2 - 1);
    const int p = lane & (LB::N2 - 1), s = lane / LB::N2;
    for (int base = 0; base < rn; base += LB::LPR) {
        if (base + warp * LB::LPW >= rn) continue;   // warp-uniform
        const int kl = base + warp * LB::LPW + s;
        const bool valid = kl < rn;
        float2* row = S + (valid ? kl : 0);
        float2 v[LB::N1];
#pragma unroll
        for (int r = 0; r < LB::N1; ++r) {
            const int k2 = p + LB::N2 * r;
            const bool in = valid && (!INV || k2 <= b2 || k2 >= k2hi);
            v[r] = in ? row[PL * k2] : make_float2(0.f, 0.f);
        }
        warp_line_fft<NB, INV, PL>(v, p, valid, twB, row);
        if (valid) {
#pragma unroll
            for (int j = 0; j < LB::M; ++j)
#pragma unroll
                for (int k = 0; k < LB::N2; ++k) row[PL * ((p + LB::N2 * j) + LB::N1 * k)] = v[j * LB::N2 + k];
        }
    }
}

// The full spectrum of (column 2l) + i (column 2l + 1) at v[r] = Z[p + N2 r],
// the rows read from the CTA that holds them.
template <int NA, int NB>
__device__ __forceinline__ void load_pair(float2 (&v)[SlabLine<NA>::N1], float2* S0, float2* S1, int l,
                                          int p, bool valid, int nk1) {
    using C = ClusterSlab<NA, NB>;
    using LA = SlabLine<NA>;
#pragma unroll
    for (int r = 0; r < LA::N1; ++r) {
        const int i = p + LA::N2 * r;
        const int k = 2 * i <= NA ? i : NA - i;
        float2 A = make_float2(0.f, 0.f), B = make_float2(0.f, 0.f);
        if (valid && k < nk1) {
            const int c = k < C::R ? 0 : 1;
            const float2* col = (c ? S1 : S0) + (k - c * C::R) + C::PL * (2 * l);
            A = col[0];
            B = col[C::PL];
        }
        if (k == 0 || 2 * k == NA) {
            A.y = 0.f;
            B.y = 0.f;
        }
        v[r] = 2 * i <= NA ? make_float2(A.x - B.y, A.y + B.x) : make_float2(A.x + B.y, B.x - A.y);
    }
}

// Z (in the exchange slots, natural order) -> the half spectra of the two
// columns, bins k < nk1, into the rows of both CTAs.
template <int NA, int NB>
__device__ __forceinline__ void unpack_pair(const float2* xs, float2* S0, float2* S1, int l, int p,
                                            bool valid, int nk1) {
    using C = ClusterSlab<NA, NB>;
    using LA = SlabLine<NA>;
    constexpr int QA = (C::H1 + LA::N2 - 1) / LA::N2;
    float2 ha[QA], hb[QA];
#pragma unroll
    for (int q = 0; q < QA; ++q) {
        const int k = p + LA::N2 * q;
        ha[q] = hb[q] = make_float2(0.f, 0.f);
        if (valid && k < nk1) {
            const float2 zk = xs[k];
            const float2 zn = xs[k == 0 ? 0 : NA - k];
            ha[q] = half_spec_a(zk, zn);
            hb[q] = half_spec_b(zk, zn);
        }
    }
    if (valid) {
#pragma unroll
        for (int q = 0; q < QA; ++q) {
            const int k = p + LA::N2 * q;
            if (k < nk1) {
                const int c = k < C::R ? 0 : 1;
                float2* col = (c ? S1 : S0) + (k - c * C::R) + C::PL * (2 * l);
                col[0] = ha[q];
                col[C::PL] = hb[q];
            }
        }
    }
}

template <int NA, int NB>
struct ClusterCtx {
    using C = ClusterSlab<NA, NB>;
    float2* twA;
    float2* twB;
    float2* S;
    float2* X;
    float2* S0;   // the rows of rank 0 and rank 1 (generic addresses)
    float2* S1;
    uint64_t* bar;
    uint32_t phase = 0;
    int rank, r0, rn;
    __device__ __forceinline__ ClusterCtx(float2* sm, const SlabArgs& a) {
        cg::cluster_group cl = cg::this_cluster();
        twA = sm;
        twB = sm + NA;
        S = sm + NA + NB;
        X = S + C::PL * NB;
        rank = (int)cl.block_rank();
        S0 = cl.map_shared_rank(S, 0);
        S1 = cl.map_shared_rank(S, 1);
        r0 = rank * C::R;
        rn = min(rank == 0 ? C::R : C::H1 - C::R, a.nk1 - r0);
        bar = reinterpret_cast<uint64_t*>(X + C::LINES * NA);
        if (threadIdx.x == 0) {
            mbar_init(bar, 1);
            fence_barrier_init();
        }
        load_slab_twiddles<NA>(twA, a.twa);
        load_slab_twiddles<NB>(twB, a.twb);
    }
};

template <int NA, int NB, int ES>
__global__ void __launch_bounds__(kSlabThreads, 1) ns_slab_cluster_inv_kernel(SlabArgs a) {
    using C = ClusterSlab<NA, NB>;
    using LA = SlabLine<NA>;
    extern __shared__ float2 sm[];
    ClusterCtx<NA, NB> cx(sm, a);
    cluster_barrier();   // both CTAs of the cluster run before either touches the other's rows
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr long long PLANE = (long long)NA * NB;
    const int nclusters = gridDim.x / kClusterCTAs;
    for (int u = blockIdx.x / kClusterCTAs; u < a.units; u += nclusters) {
        const int per = a.nzc * a.n3;
        const int ch = u / per, ur = u - ch * per;
        const int z = ur / a.n3, s3 = ur - z * a.n3;
        const float2* src = a.spec + ch * a.spec_chstride + z * a.spec_zstride + (long long)s3 * (C::P1 * NB);
        load_rows<NB, C::P1, C::PL>(cx.S, src, cx.r0, cx.rn, a.nk2, a.b2, cx.bar, cx.phase, a.status);
        rows_fft<NB, C::PL, true>(cx.S, cx.twB, cx.rn, a.nk2, a.b2, warp, lane);
        cluster_barrier();   // both halves of every column are final
        {
            const int p = lane & (LA::N2 - 1), s = pair_subline<NA>(lane / LA::N2);
            float* out = a.vol + ch + a.vz.off(z) + (long long)s3 * PLANE * ES;
            float2* xs = cx.X + (warp * LA::LPW + s) * NA;
            for (int base = 0; base < C::PAIRS; base += LA::LPR) {
                const int lo = base + warp * LA::LPW + s;   // own pair index
                const bool valid = lo < C::PAIRS;
                const int l = cx.rank * C::PAIRS + (valid ? lo : 0);
                float2 v[LA::N1];
                load_pair<NA, NB>(v, cx.S0, cx.S1, l, p, valid, a.nk1);
                warp_line_fft<NA, true, 1>(v, p, valid, cx.twA, xs);
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
        cluster_barrier();   // the peer is done reading these rows
    }
}

template <int NA, int NB, int ES>
__global__ void __launch_bounds__(kSlabThreads, 1) ns_slab_cluster_fwd_kernel(SlabArgs a) {
    using C = ClusterSlab<NA, NB>;
    using LA = SlabLine<NA>;
    extern __shared__ float2 sm[];
    ClusterCtx<NA, NB> cx(sm, a);
    cluster_barrier();   // both CTAs run; the twiddles are in place
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr long long PLANE = (long long)NA * NB;
    const int nclusters = gridDim.x / kClusterCTAs;
    for (int u = blockIdx.x / kClusterCTAs; u < a.units; u += nclusters) {
        const int per = a.nzc * a.n3;
        const int ch = u / per, ur = u - ch * per;
        const int z = ur / a.n3, s3 = ur - z * a.n3;
        {
            const int p = lane & (LA::N2 - 1), s = pair_subline<NA>(lane / LA::N2);
            const float* in = a.vol + ch + a.vz.off(z) + (long long)s3 * PLANE * ES;
            float2* xs = cx.X + (warp * LA::LPW + s) * NA;
            for (int base = 0; base < C::PAIRS; base += LA::LPR) {
                const int lo = base + warp * LA::LPW + s;
                const bool valid = lo < C::PAIRS;
                const int l = cx.rank * C::PAIRS + (valid ? lo : 0);
                const float* ia = in + (long long)(2 * l) * NA * ES;
                const float* ib = ia + (long long)NA * ES;
                float2 v[LA::N1];
#pragma unroll
                for (int r = 0; r < LA::N1; ++r) {
                    const int i = p + LA::N2 * r;
                    v[r] = valid ? make_float2(ia[i * ES], ib[i * ES]) : make_float2(0.f, 0.f);
                }
                warp_line_fft<NA, false, 1>(v, p, valid, cx.twA, xs);
                if (valid) {
#pragma unroll
                    for (int j = 0; j < LA::M; ++j)
#pragma unroll
                        for (int k = 0; k < LA::N2; ++k) xs[(p + LA::N2 * j) + LA::N1 * k] = v[j * LA::N2 + k];
                }
                __syncwarp();
                unpack_pair<NA, NB>(xs, cx.S0, cx.S1, l, p, valid, a.nk1);
                __syncwarp();   // the exchange slots are reused by the next pair
            }
        }
        cluster_barrier();   // every row is complete in its CTA
        rows_fft<NB, C::PL, false>(cx.S, cx.twB, cx.rn, a.nk2, a.b2, warp, lane);
        __syncthreads();
        float2* dst = a.spec + ch * a.spec_chstride + z * a.spec_zstride + (long long)s3 * (C::P1 * NB);
        store_rows<NB, C::P1, C::PL>(dst, cx.S, cx.r0, cx.rn, a.nk2, a.b2);
        cluster_barrier();   // the rows are free for the peer's next unit
    }
}

template <int NA, int NB>
__global__ void __launch_bounds__(kSlabThreads, 1) ns_slab_cluster_shrink_kernel(SlabArgs a) {
    using C = ClusterSlab<NA, NB>;
    using LA = SlabLine<NA>;
    extern __shared__ float2 sm[];
    ClusterCtx<NA, NB> cx(sm, a);
    cluster_barrier();   // both CTAs of the cluster run before either touches the other's rows
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nclusters = gridDim.x / kClusterCTAs;
    for (int u = blockIdx.x / kClusterCTAs; u < a.units; u += nclusters) {
        const int per = a.nzc * a.n3;
        const int ch = u / per, ur = u - ch * per;
        const int z = ur / a.n3, s3 = ur - z * a.n3;
        float2* slab = a.spec + ch * a.spec_chstride + z * a.spec_zstride + (long long)s3 * (C::P1 * NB);
        const float tau = a.tau[a.items[a.item0 + z].s - 1];
        load_rows<NB, C::P1, C::PL>(cx.S, slab, cx.r0, cx.rn, a.nk2, a.b2, cx.bar, cx.phase, a.status);
        rows_fft<NB, C::PL, true>(cx.S, cx.twB, cx.rn, a.nk2, a.b2, warp, lane);
        cluster_barrier();
        {
            const int p = lane & (LA::N2 - 1), s = pair_subline<NA>(lane / LA::N2);
            float2* xs = cx.X + (warp * LA::LPW + s) * NA;
            for (int base = 0; base < C::PAIRS; base += LA::LPR) {
                const int lo = base + warp * LA::LPW + s;
                const bool valid = lo < C::PAIRS;
                const int l = cx.rank * C::PAIRS + (valid ? lo : 0);
                float2 v[LA::N1];
                load_pair<NA, NB>(v, cx.S0, cx.S1, l, p, valid, a.nk1);
                warp_line_fft<NA, true, 1>(v, p, valid, cx.twA, xs);
                if (valid) {
#pragma unroll
                    for (int j = 0; j < LA::M; ++j)
#pragma unroll
                        for (int k = 0; k < LA::N2; ++k) {
                            const float2 c = v[j * LA::N2 + k];
                            const float xa = c.x * a.scale, xb = c.y * a.scale;
                            xs[(p + LA::N2 * j) + LA::N1 * k] = make_float2(copysignf(fmaxf(fabsf(xa) - tau, 0.f), xa),
                                                                            copysignf(fmaxf(fabsf(xb) - tau, 0.f), xb));
                        }
                }
                __syncwarp();
#pragma unroll
                for (int r = 0; r < LA::N1; ++r) v[r] = valid ? xs[p + LA::N2 * r] : make_float2(0.f, 0.f);
                warp_line_fft<NA, false, 1>(v, p, valid, cx.twA, xs);
                if (valid) {
#pragma unroll
                    for (int j = 0; j < LA::M; ++j)
#pragma unroll
                        for (int k = 0; k < LA::N2; ++k) xs[(p + LA::N2 * j) + LA::N1 * k] = v[j * LA::N2 + k];
                }
                __syncwarp();
                unpack_pair<NA, NB>(xs, cx.S0, cx.S1, l, p, valid, a.nk1);
                __syncwarp();
            }
        }
        cluster_barrier();   // every row holds the re-transformed columns
        rows_fft<NB, C::PL, false>(cx.S, cx.twB, cx.rn, a.nk2, a.b2, warp, lane);
        __syncthreads();
        store_rows<NB, C::P1, C::PL>(slab, cx.S, cx.r0, cx.rn, a.nk2, a.b2);
        __syncthreads();   // own rows are reloaded by the next unit (the peer writes them only after the next barrier)
    }
}

template <int KIND, int NA, int NB, int ES>
void launch_cluster(const SlabArgs& a, int sms, cudaStream_t st, const char* tag) {
    using C = ClusterSlab<NA, NB>;
    auto kern = KIND == 1 ? ns_slab_cluster_inv_kernel<NA, NB, ES>
                          : (KIND == 0 ? ns_slab_cluster_fwd_kernel<NA, NB, ES> : ns_slab_cluster_shrink_kernel<NA, NB>);
    static bool configured = false;
    static int max_clusters = 0;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClusterCTAs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(kSlabThreads);
    cfg.dynamicSmemBytes = C::SMEM;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (!configured) {
        cuda_check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM),
                   "cudaFuncSetAttribute(cluster slab)");
        cfg.gridDim = dim3(kClusterCTAs * (unsigned)std::max(1, sms / kClusterCTAs));
        cuda_check(cudaOccupancyMaxActiveClusters(&max_clusters, kern, &cfg),
                   "cudaOccupancyMaxActiveClusters(cluster slab)");
        if (max_clusters < 1) throw ArgError("the cluster slab kernel cannot be resident on this device");
        configured = true;
    }
    const int nclusters = std::max(1, std::min(a.units, max_clusters));
    cfg.gridDim = dim3((unsigned)(kClusterCTAs * nclusters));
    int tok = prof_begin(tag, st);
    cuda_check(cudaLaunchKernelEx(&cfg, kern, a), "cluster slab kernel launch");
    prof_end(tok, st);
}

template <int NA, int NB>
void launch_nn(int kind, const SlabArgs& a, int sms, cudaStream_t st, const char* tag) {
    using C = ClusterSlab<NA, NB>;
    if (a.P1 != C::P1) throw ArgError("slab pitch mismatch");
    if (a.nk1 > C::H1 || a.nk2 > NB) throw ArgError("slab box out of range");
    if (kind == 1) {
        if (a.es == 1)
            launch_cluster<1, NA, NB, 1>(a, sms, st, tag);
        else
            launch_cluster<1, NA, NB, 2>(a, sms, st, tag);
    } else if (kind == 0) {
        if (a.es == 1)
            launch_cluster<0, NA, NB, 1>(a, sms, st, tag);
        else
            launch_cluster<0, NA, NB, 2>(a, sms, st, tag);
    } else {
        launch_cluster<2, NA, NB, 1>(a, sms, st, tag);
    }
}

}  // namespace

bool slab_cluster_supported(int na, int nb) { return na == 256 && nb == 256; }

// Whether a two-CTA cluster of the slab kernels fits the current device (a
// partitioned or shared device may not offer it); asked once a device.
bool slab_cluster_resident(int na, int nb) {
    if (!slab_cluster_supported(na, nb)) return false;
    static int cached[64];   // 0 unknown, 1 yes, 2 no
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) return false;
    if (cached[dev] == 0) {
        using C = ClusterSlab<256, 256>;
        auto kern = ns_slab_cluster_inv_kernel<256, 256, 1>;
        int n = 0;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM) == cudaSuccess) {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = kClusterCTAs;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3(kClusterCTAs);
            cfg.blockDim = dim3(kSlabThreads);
            cfg.dynamicSmemBytes = C::SMEM;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) n = 0;
        }
        cudaGetLastError();   // a refused query leaves no sticky error behind
        cached[dev] = n > 0 ? 1 : 2;
    }
    return cached[dev] == 1;
}

bool launch_slab_cluster(int kind, int na, int nb, const SlabArgs& a, int sms, cudaStream_t st, const char* tag) {
    if (na == 256 && nb == 256) {
        static_assert(ClusterSlab<256, 256>::SMEM <= 227 * 1024, "cluster slab exceeds shared memory");
        launch_nn<256, 256>(kind, a, sms, st, tag);
        return true;
    }
    return false;
}

}  // namespace sfl
