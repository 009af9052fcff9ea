// The decimated Surfacelet on the device: SurfBox's construction as in
// src/transforms/surfacelet.jl, src/directional/surfacelet_scale.jl,
// src/directional/irc.jl and src/pyramid/fourier_pyramid.jl.
//
// Forward, per channel:
//   X = FFT(x) (full complex grid; the first pass transforms two real lines
//   per complex FFT and unpacks both full spectra), then per pyramid level:
//   split (lowpass cropped to the next level, highpass in place), and per
//   hourglass K: S_K = X[half_K] V_K / |subband| ; the IRC stages (a 2x2
//   complex butterfly per bin pair) ; the block inverse FFTs along the two
//   decimated axes (segmented line passes) ; the C2R along K, two lines per
//   complex FFT, written straight into the subband's place in the coefficient
//   vector.  The coarse lowpass is Re(bfft(C))/|C|.
// Inverse: the mirror image, with one kernel that forms the Hermitian sum of
// the three hourglasses over the full grid.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "passes.cuh"
#include "plan.h"
#include "regpass.cuh"
#include "slab_core.cuh"

namespace sfl {

struct DecStageDev {
    int m = 0, b = 0;
    DevMem f[4];   // analysis ch0, ch1, synthesis ch0, ch1: (K-half, m) planes
};

struct DecLevelDev {
    int n[3], nlow[3];
    int cnt[3];
    DevMem idx[3], idx_low[3];
    DevMem lw_split, lw_merge, hw;     // box weights (float64-designed)
    DevMem V[3];
    int hd[3][3];                     // [K][d] half-K dims
    std::vector<DecStageDev> stages[3];
    int counts[3][3];                 // [K][d] block counts
    int bsize[3][3];                  // [K][d] block size (K: half length)
    long long first_off[3];           // element offset of hourglass K's first subband
    long long blk_elems[3];
    int nsub[3];
    DevMem S[3];                      // this level's half-K spectra S_K
    DevMem inv[3];                    // box position along axis d of each spectrum index (-1 outside the box)
    bool merge_fused = false;         // the box maps are one to one: the merge runs inside the Hermitian sum
};

// Two side streams and the events that fork them from, and join them back
// to, the caller's stream: the per-level passes of a call, which touch only
// their own level's buffers and coefficients, run on them concurrently (the
// fork-join pattern that stream capture records as graph branches).
struct LevelStreams {
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
    void create() {
        for (auto& x : side) cuda_check(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_check(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "cudaEventCreate");
        for (auto& e : join) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    }
    ~LevelStreams() {
        for (auto& e : join)
            if (e) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        for (auto& x : side)
            if (x) cudaStreamDestroy(x);
    }
};

struct DecPlan {
    SurfDesign design;
    int dims[3];
    int nch = 1;
    int J = 0;
    long long ncoef = 0;
    std::vector<std::unique_ptr<DecLevelDev>> lv;
    std::vector<std::unique_ptr<DevMem>> spectra;   // J + 1 full complex grids
    std::map<int, std::unique_ptr<FFTLen>> ffts;
    LevelStreams ls;
};

void DecPlanDeleter::operator()(DecPlan* d) const { delete d; }
const SurfDesign& dec_design(const DecPlan& d) { return d.design; }

// A table the plan holds on the device, as floats: "ritf" (index = level * 3 +
// K - 1: V_K) or "irc" (index = ((level * 3 + K - 1) * 32 + stage) * 4 +
// which; float2 values as re/im pairs).
const float* dec_plan_table(const DecPlan& d, const std::string& name, int index, long long* count) {
    if (name == "ritf") {
        const int lv = index / 3, K = index % 3;
        if (index < 0 || lv >= (int)d.lv.size()) throw ArgError("table index out of range");
        const int* h = d.lv[lv]->hd[K];
        *count = (long long)h[0] * h[1] * h[2];
        return d.lv[lv]->V[K].as<float>();
    }
    if (name == "irc") {
        const int which = index % 4, stage = (index / 4) % 32, K = (index / 128) % 3, lv = index / 384;
        if (index < 0 || lv >= (int)d.lv.size() || stage >= (int)d.lv[lv]->stages[K].size())
            throw ArgError("table index out of range");
        const DecStageDev& sd = d.lv[lv]->stages[K][stage];
        *count = (long long)(sd.f[which].bytes / sizeof(float));
        return sd.f[which].as<float>();
    }
    throw ArgError("unknown table " + name);
}
int dec_nsubbands(const DecPlan& d) { return (int)d.design.sizes.size(); }
long long dec_ncoeffs(const DecPlan& d) { return d.ncoef; }
void dec_subband_info(const DecPlan& d, int i, int shape[3], long long* offset) {
    for (int k = 0; k < 3; ++k) shape[k] = d.design.sizes[i - 1][k];
    *offset = d.design.offsets[i - 1];
}

// ── kernels ──────────────────────────────────────────────────────────────────

__device__ __forceinline__ long long lin3(int a, int b, int c, int d0, int d1) {
    return a + (long long)d0 * (b + (long long)d1 * c);
}

// Unsigned division by a divisor fixed for a loop: n / d = umulhi(n, m) with
// m = ceil(2^32 / d), after Granlund and Montgomery, "Division by invariant
// integers using multiplication" (1994).  Exact when d is a power of two or
// n * d < 2^32 (n / d gains less than n (d - 2^32 mod d) / (d 2^32) < 1/d);
// the plane pass divides point and pair indices below 2^17 by lengths below
// 2^12.
struct FastDiv {
    unsigned d, m;
    __host__ __device__ explicit FastDiv(unsigned dv) : d(dv), m(dv > 1 ? 0xFFFFFFFFu / dv + 1u : 0u) {}
    __device__ __forceinline__ unsigned div(unsigned n) const { return d > 1 ? __umulhi(n, m) : n; }
};

// The grid kernels below take one point each: a 32 x 8 block over the first two
// axes, blockIdx.z over the third (no index division).
constexpr int kGridBX = 32, kGridBY = 8;
inline dim3 grid3_blocks(int d0, int d1, int d2) {
    return dim3((unsigned)((d0 + kGridBX - 1) / kGridBX), (unsigned)((d1 + kGridBY - 1) / kGridBY), (unsigned)d2);
}
inline dim3 grid3_threads() { return dim3(kGridBX, kGridBY); }
__device__ __forceinline__ bool grid3_point(int d0, int d1, int& a, int& b, int& c) {
    a = blockIdx.x * kGridBX + threadIdx.x;
    b = blockIdx.y * kGridBY + threadIdx.y;
    c = blockIdx.z;
    return a < d0 && b < d1;
}

// src/pyramid/fourier_pyramid.jl:221-231 (file numbering): low = crop(L X)/D^1.5,
// X[box] *= sqrt(1 - L^2).  `low` must be zeroed first.
// lw[q] = L D^-1.5 and hw[q] = sqrt(1 - L^2) on the box, designed in float64.
__global__ void pyr_split_kernel(float2* X, float2* low, int n0, int n1, int l0, int l1, const int* i0,
                                 const int* i1, const int* i2, const int* j0, const int* j1, const int* j2,
                                 const float* lw, const float* hw, int c0, int c1, int c2) {
    int a, b, c;
    if (!grid3_point(c0, c1, a, b, c)) return;
    const long long q = lin3(a, b, c, c0, c1);
    long long xa = lin3(i0[a], i1[b], i2[c], n0, n1);
    float2 v = X[xa];
    low[lin3(j0[a], j1[b], j2[c], l0, l1)] = c_scale(v, lw[q]);
    X[xa] = c_scale(v, hw[q]);
}

// src/pyramid/fourier_pyramid.jl:235-240: X[box] = sqrt(1-L^2) X[box] + L D^1.5 low.
// lw[q] = L D^1.5 and hw[q] = sqrt(1 - L^2) on the box, designed in float64.
__global__ void pyr_merge_kernel(float2* X, const float2* low, int n0, int n1, int l0, int l1, const int* i0,
                                 const int* i1, const int* i2, const int* j0, const int* j1, const int* j2,
                                 const float* lw, const float* hw, int c0, int c1, int c2) {
    int a, b, c;
    if (!grid3_point(c0, c1, a, b, c)) return;
    const long long q = lin3(a, b, c, c0, c1);
    long long xa = lin3(i0[a], i1[b], i2[c], n0, n1);
    float2 h = c_scale(X[xa], hw[q]);
    float2 w = c_scale(low[lin3(j0[a], j1[b], j2[c], l0, l1)], lw[q]);
    X[xa] = c_add(h, w);
}

// S_K = X[half_K] * V_K * s: src/directional/surfacelet_scale.jl:205-206, 292
__global__ void hg_mask_kernel(const float2* X, int n0, int n1, float2* S, int h0, int h1, int h2,
                               const float* V, float s) {
    int a, b, c;
    if (!grid3_point(h0, h1, a, b, c)) return;
    const long long q = lin3(a, b, c, h0, h1);
    S[q] = c_scale(X[lin3(a, b, c, n0, n1)], V[q] * s);
}

// One IRC stage in place on S (half-K dims h): for every bin pair (A, B) of
// the 2b-bin groups along axis m, analysis A <- F0(A)A + F0(B)B,
// B <- F1(A)A + F1(B)B; synthesis A <- G0(A)A + G1(A)B, B <- G0(B)A + G1(B)B.
// src/directional/irc.jl:304-345 (file numbering)
// With conj, the coefficients enter conjugated (the adjoint of a stage is its
// conjugate transpose: the analysis adjoint takes the synthesis form with
// conj(F0), conj(F1); the synthesis adjoint the analysis form with conj(G0),
// conj(G1)).
__global__ void irc_stage_kernel(float2* S, int h0, int h1, int h2, int K, int m, int b, const float2* f0,
                                 const float2* f1, int synth, int conj) {
    int hd[3] = {h0, h1, h2};
    int pd[3] = {h0, h1, h2};
    pd[m] = hd[m] / 2;
    const int nKh = hd[K];
    {
        int c[3];
        if (!grid3_point(pd[0], pd[1], c[0], c[1], c[2])) return;
        int pq = c[m];
        int cA = (pq / b) * 2 * b + (pq % b);
        int cB = cA + b;
        c[m] = cA;
        long long aA = lin3(c[0], c[1], c[2], h0, h1);
        c[m] = cB;
        long long aB = lin3(c[0], c[1], c[2], h0, h1);
        int kK = c[K];
        long long fA = kK + (long long)nKh * cA, fB = kK + (long long)nKh * cB;
        float2 A = S[aA], Bv = S[aB];
        float2 f0A = f0[fA], f0B = f0[fB], f1A = f1[fA], f1B = f1[fB];
        if (conj) {
            f0A.y = -f0A.y;
            f0B.y = -f0B.y;
            f1A.y = -f1A.y;
            f1B.y = -f1B.y;
        }
        float2 nA, nB;
        if (!synth) {
            nA = c_add(c_mul(f0A, A), c_mul(f0B, Bv));
            nB = c_add(c_mul(f1A, A), c_mul(f1B, Bv));
        } else {
            nA = c_add(c_mul(f0A, A), c_mul(f1A, Bv));
            nB = c_add(c_mul(f0B, A), c_mul(f1B, Bv));
        }
        S[aA] = nA;
        S[aB] = nB;
    }
}

// Every IRC stage of hourglass K on one plane k_K of S_K (the plane over the
// two transverse axes), held in shared memory: one HBM round trip for the
// whole cascade instead of one per stage.  Where both block lengths have a
// register line FFT, the block FFTs along the two transverse axes run in the
// same pass (after the stages in the analysis, before them in the
// synthesis): every block lies inside one plane.  The analysis form applies the
// hourglass mask on load (S_K = X[half_K] V_K s, as hg_mask_kernel) and runs
// the stages in order; the synthesis form runs them in reverse with the
// synthesis filters.  Per stage the same butterfly, in the same order of
// operations, as irc_stage_kernel.  One CTA a plane (blockIdx.x = k_K).
constexpr int kIrcPlaneMaxStages = 8;
constexpr int kIrcPlaneThreads = 1024;
constexpr int kIrcPlaneBatch = 4;
struct IrcPlaneStages {
    int n;
    int m[kIrcPlaneMaxStages], b[kIrcPlaneMaxStages];
    const float2* f0[kIrcPlaneMaxStages];
    const float2* f1[kIrcPlaneMaxStages];
};

// The planes of the hourglasses of every pyramid level in one launch: job t
// owns the CTAs [first, first + hd[K]) (one per k_K plane); every hourglass of
// every level has its own S_K buffer.
struct IrcPlaneJob {
    float2* S;
    const float2* X;   // analysis: the level's full spectrum, n0 x n1 x ...
    int n0, n1;
    int K, first;
    int hd[3];
    const float* V;   // analysis: the hourglass mask V_K and the subband scale s
    float s;
    IrcPlaneStages sg;
    // the block FFTs along the two transverse axes, fused: segment lengths (0: run separately) and the
    // twiddle tables w_bs^k of those lengths
    int bs1, bs2;
    const float2* tw1;
    const float2* tw2;
};
constexpr int kIrcPlaneMaxJobs = 12;   // hourglasses of up to four pyramid levels
struct IrcPlaneJobs {
    int n;
    IrcPlaneJob job[kIrcPlaneMaxJobs];
};

// Plane pitch: the first transverse length rounded to 2 mod 4, so that lines
// along either axis of the plane are free of bank conflicts.
__host__ __device__ inline int irc_plane_pitch(int a1) { return a1 % 4 == 0 ? a1 + 2 : a1; }

// Block FFT lengths the plane pass runs itself (register line FFTs of at most
// 16 values a thread, within the 64 registers of a 1024-thread CTA).
__host__ __device__ inline bool irc_plane_block_len(int n) { return n == 16 || n == 32 || n == 64 || n == 128; }

// The segmented FFTs of the plane along one transverse axis: segments of N
// points (the block length), unnormalized, inverse or forward.  Lines of a
// warp sit on consecutive rows (along the first axis) or consecutive columns
// (along the second), so their slots fall on distinct banks.
template <int N, bool INV>
__device__ void irc_plane_seg_fft(float2* pl, int ap, int a1, int a2, bool along1, const float2* tw2s) {
    using LN = SlabLine<N>;
    constexpr int N1 = LN::N1, N2 = LN::N2;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int p = lane & (N2 - 1), sl = lane / N2;
    const int nseg = (along1 ? a1 : a2) / N;
    const int nl = (along1 ? a2 : a1) * nseg;
    for (int b0 = 0; b0 < nl; b0 += nwarps * LN::LPW) {
        if (b0 + warp * LN::LPW >= nl) continue;   // warp-uniform
        const int line = b0 + warp * LN::LPW + sl;
        const bool valid = line < nl;
        const int li = valid ? line : 0;
        float2* base;
        int stride;
        if (along1) {
            const int o2 = li % a2, seg = li / a2;
            base = pl + (long long)o2 * ap + seg * N;
            stride = 1;
        } else {
            const int o1 = li % a1, seg = li / a1;
            base = pl + o1 + (long long)seg * N * ap;
            stride = ap;
        }
        float2 v[N1];
#pragma unroll
        for (int r = 0; r < N1; ++r) v[r] = valid ? base[stride * (p + N2 * r)] : make_float2(0.f, 0.f);
        warp_line_fft_rs<N, INV>(v, p, valid, tw2s, base, stride);
        if (valid) {
#pragma unroll
            for (int j = 0; j < LN::M; ++j)
#pragma unroll
                for (int k = 0; k < N2; ++k) base[stride * ((p + N2 * j) + N1 * k)] = v[j * N2 + k];
        }
    }
}

template <bool INV>
__device__ void irc_plane_block_ffts(float2* pl, int ap, int a1, int a2, int bs, bool along1, const float2* tw2s) {
    switch (bs) {
        case 16: irc_plane_seg_fft<16, INV>(pl, ap, a1, a2, along1, tw2s); break;
        case 32: irc_plane_seg_fft<32, INV>(pl, ap, a1, a2, along1, tw2s); break;
        case 64: irc_plane_seg_fft<64, INV>(pl, ap, a1, a2, along1, tw2s); break;
        case 128: irc_plane_seg_fft<128, INV>(pl, ap, a1, a2, along1, tw2s); break;
    }
}

template <int N>
__device__ void irc_plane_twiddles(float2* tw2s, const float2* tw) {
    load_slab_twiddles<N>(tw2s, tw);
}

__device__ void irc_plane_load_twiddles(float2* tw2s, const float2* tw, int bs) {
    switch (bs) {
        case 16: irc_plane_twiddles<16>(tw2s, tw); break;
        case 32: irc_plane_twiddles<32>(tw2s, tw); break;
        case 64: irc_plane_twiddles<64>(tw2s, tw); break;
        case 128: irc_plane_twiddles<128>(tw2s, tw); break;
    }
}

template <bool SYNTH>
__global__ void __launch_bounds__(kIrcPlaneThreads) irc_plane_kernel(const __grid_constant__ IrcPlaneJobs jobs) {
    extern __shared__ float2 pl[];
    int t0 = 0;
    while (t0 + 1 < jobs.n && (int)blockIdx.x >= jobs.job[t0 + 1].first) ++t0;
    const IrcPlaneJob& jb = jobs.job[t0];
    const float2* __restrict__ X = jb.X;
    const int n0 = jb.n0, n1 = jb.n1;
    float2* S = jb.S;
    const int K = jb.K;
    const float* __restrict__ V = jb.V;
    const float s = jb.s;
    const IrcPlaneStages& sg = jb.sg;
    // extents and strides of the hourglass axis K and the transverse axes m1 < m2, as scalars
    const int h0 = jb.hd[0], h1 = jb.hd[1], h2 = jb.hd[2];
    const long long p1 = h0, p2 = (long long)h0 * h1;   // S_K strides of axes 1, 2
    const long long x1 = n0, x2 = (long long)n0 * n1;   // X strides of axes 1, 2
    const int nKh = K == 0 ? h0 : (K == 1 ? h1 : h2);
    const int a1 = K == 0 ? h1 : h0, a2 = K == 2 ? h1 : h2;
    const long long sK = K == 0 ? 1 : (K == 1 ? p1 : p2), s1 = K == 0 ? p1 : 1, s2 = K == 2 ? p1 : p2;
    const long long xK = K == 0 ? 1 : (K == 1 ? x1 : x2), xa = K == 0 ? x1 : 1, xb = K == 2 ? x1 : x2;
    const int kK = blockIdx.x - jb.first;
    const long long base = (long long)kK * sK;
    const long long xbase = (long long)kK * xK;
    const int tot = a1 * a2;
    const FastDiv fa1((unsigned)a1);
    const int ap = irc_plane_pitch(a1);                  // the plane's row pitch in shared memory
    float2* cf = pl + (long long)ap * a2;                // a stage's two filter rows
    float2* tws = cf + 2 * (a1 > a2 ? a1 : a2);          // block-FFT twiddles: bs1 then bs2 entries
    const bool fused = jb.bs1 > 0 && jb.bs2 > 0;
    if (fused) {
        irc_plane_load_twiddles(tws, jb.tw1, jb.bs1);
        irc_plane_load_twiddles(tws + jb.bs1, jb.tw2, jb.bs2);
    }
    // kIrcPlaneBatch independent loads in flight per thread (one CTA an SM holds the plane)
    for (int q0 = threadIdx.x; q0 < tot; q0 += kIrcPlaneBatch * blockDim.x) {
        float2 v[kIrcPlaneBatch];
#pragma unroll
        for (int u = 0; u < kIrcPlaneBatch; ++u) {
            const int q = q0 + u * blockDim.x;
            v[u] = make_float2(0.f, 0.f);
            if (q < tot) {
                const int i2 = (int)fa1.div((unsigned)q), i1 = q - i2 * a1;
                const long long g = base + i1 * s1 + i2 * s2;
                if (!SYNTH) {
                    v[u] = c_scale(X[xbase + i1 * xa + i2 * xb], V[g] * s);
                } else {
                    v[u] = S[g];
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kIrcPlaneBatch; ++u) {
            const int q = q0 + u * blockDim.x;
            if (q < tot) {
                const int i2 = (int)fa1.div((unsigned)q);
                pl[(q - i2 * a1) + ap * i2] = v[u];
            }
        }
    }
    __syncthreads();
    if (SYNTH && fused) {
        // subband -> block: the forward block FFTs along both transverse axes, then the stages in reverse
        irc_plane_block_ffts<false>(pl, ap, a1, a2, jb.bs1, true, tws);
        __syncthreads();
        irc_plane_block_ffts<false>(pl, ap, a1, a2, jb.bs2, false, tws + jb.bs1);
        __syncthreads();
    }
    for (int t = 0; t < sg.n; ++t) {
        const int u = SYNTH ? sg.n - 1 - t : t;
        const int b = sg.b[u];
        const bool first = sg.m[u] == (K == 0 ? 1 : 0);   // along the plane's first axis m1
        const int half = (first ? a1 : a2) / 2;
        const int npairs = half * (first ? a2 : a1);
        const FastDiv fo((unsigned)(first ? half : a1)), fb((unsigned)b);
        // the stage's filter row at k_K (over the stage's axis) into shared memory
        const int am = first ? a1 : a2;
        for (int i = threadIdx.x; i < am; i += blockDim.x) {
            cf[i] = sg.f0[u][kK + (long long)nKh * i];
            cf[am + i] = sg.f1[u][kK + (long long)nKh * i];
        }
        __syncthreads();
        for (int q = threadIdx.x; q < npairs; q += blockDim.x) {
            // consecutive threads on consecutive words of the plane: the pair index runs fastest along
            // the first axis, the other index along the second
            const int qd = (int)fo.div((unsigned)q), qr = q - qd * (int)fo.d;
            const int pq = first ? qr : qd, o = first ? qd : qr;
            const int pb = (int)fb.div((unsigned)pq);
            const int cA = pb * 2 * b + (pq - pb * b), cB = cA + b;
            const int qA = first ? cA + ap * o : o + ap * cA;
            const int qB = first ? cB + ap * o : o + ap * cB;
            const float2 A = pl[qA], Bv = pl[qB];
            const float2 f0A = cf[cA], f0B = cf[cB], f1A = cf[am + cA], f1B = cf[am + cB];
            float2 nA, nB;
            if (!SYNTH) {
                nA = c_add(c_mul(f0A, A), c_mul(f0B, Bv));
                nB = c_add(c_mul(f1A, A), c_mul(f1B, Bv));
            } else {
                nA = c_add(c_mul(f0A, A), c_mul(f1A, Bv));
                nB = c_add(c_mul(f0B, A), c_mul(f1B, Bv));
            }
            pl[qA] = nA;
            pl[qB] = nB;
        }
        __syncthreads();
    }
    if (!SYNTH && fused) {
        // block -> subband, first half: the inverse block FFTs along both transverse axes
        irc_plane_block_ffts<true>(pl, ap, a1, a2, jb.bs1, true, tws);
        __syncthreads();
        irc_plane_block_ffts<true>(pl, ap, a1, a2, jb.bs2, false, tws + jb.bs1);
        __syncthreads();
    }
    for (int q = threadIdx.x; q < tot; q += blockDim.x) {
        const int i2 = (int)fa1.div((unsigned)q), i1 = q - i2 * a1;
        S[base + i1 * s1 + i2 * s2] = pl[i1 + ap * i2];
    }
}

// X = sum_K (1/3) V_K S_K on each half and the conjugate mirror on the rest:
// src/directional/surfacelet_scale.jl:231-257
struct HermArgs {
    const float2* S[3];
    const float* V[3];
};
// With MERGE, the pyramid merge of the level (pyr_merge_kernel) on the box
// points in the same pass: X = sqrt(1-L^2) X + L D^1.5 low there, with the
// same arithmetic, located by the inverse box maps.
struct MergeArgs {
    const int* inv[3];
    const int* jl[3];
    const float* lw;
    const float* hw;
    const float2* low;
    int c0, c1, l0, l1;
};
template <bool MERGE>
__global__ void hermitian_sum_kernel(float2* X, int n0, int n1, int n2, HermArgs ha, float third, MergeArgs mg) {
    int n[3] = {n0, n1, n2};
    {
        int k[3];
        if (!grid3_point(n0, n1, k[0], k[1], k[2])) return;
        const long long q = lin3(k[0], k[1], k[2], n0, n1);
        float2 v = make_float2(0.f, 0.f);
#pragma unroll
        for (int K = 0; K < 3; ++K) {
            int hd[3] = {n0, n1, n2};
            hd[K] = n[K] / 2 + 1;
            if (k[K] < hd[K]) {
                long long a = lin3(k[0], k[1], k[2], hd[0], hd[1]);
                v = c_fma(ha.S[K][a], third * ha.V[K][a], v);
            } else {
                const int m0 = k[0] ? n0 - k[0] : 0, m1 = k[1] ? n1 - k[1] : 0, m2 = k[2] ? n2 - k[2] : 0;
                long long a = lin3(m0, m1, m2, hd[0], hd[1]);
                v = c_fma(c_conj(ha.S[K][a]), third * ha.V[K][a], v);
            }
        }
        if (MERGE) {
            const int a = mg.inv[0][k[0]], b = mg.inv[1][k[1]], c = mg.inv[2][k[2]];
            if ((a | b | c) >= 0) {
                const long long qb = lin3(a, b, c, mg.c0, mg.c1);
                const float2 h = c_scale(v, mg.hw[qb]);
                const float2 w = c_scale(mg.low[lin3(mg.jl[0][a], mg.jl[1][b], mg.jl[2][c], mg.l0, mg.l1)], mg.lw[qb]);
                v = c_add(h, w);
            }
        }
        X[q] = v;
    }
}

// Adjoint of the hourglass masks of the analysis: X = sum_K pad_K(V_K s_K S_K),
// zero outside each half grid.
__global__ void hg_adjoint_sum_kernel(float2* X, int n0, int n1, int n2, HermArgs ha, float s0, float s1, float s2) {
    int n[3] = {n0, n1, n2};
    const float sK[3] = {s0, s1, s2};
    {
        int k[3];
        if (!grid3_point(n0, n1, k[0], k[1], k[2])) return;
        const long long q = lin3(k[0], k[1], k[2], n0, n1);
        float2 v = make_float2(0.f, 0.f);
#pragma unroll
        for (int K = 0; K < 3; ++K) {
            int hd[3] = {n0, n1, n2};
            hd[K] = n[K] / 2 + 1;
            if (k[K] < hd[K]) {
                long long a = lin3(k[0], k[1], k[2], hd[0], hd[1]);
                v = c_fma(ha.S[K][a], sK[K] * ha.V[K][a], v);
            }
        }
        X[q] = v;
    }
}

// Adjoint of the Hermitian sum of the synthesis, for hourglass K: on its half
// grid S_K[a] = (1/3) V_K[a] (X[a] + conj(X[-a]) where -a lies outside the
// half grid along K).
__global__ void herm_gather_kernel(const float2* X, int n0, int n1, int n2, float2* S, const float* V, int K,
                                   float third) {
    int n[3] = {n0, n1, n2};
    int hd[3] = {n0, n1, n2};
    hd[K] = n[K] / 2 + 1;
    {
        int a[3];
        if (!grid3_point(hd[0], hd[1], a[0], a[1], a[2])) return;
        const long long q = lin3(a[0], a[1], a[2], hd[0], hd[1]);
        float2 v = X[lin3(a[0], a[1], a[2], n0, n1)];
        const int mK = a[K] ? n[K] - a[K] : 0;
        if (mK >= hd[K]) {
            const int m0 = a[0] ? n0 - a[0] : 0, m1 = a[1] ? n1 - a[1] : 0, m2 = a[2] ? n2 - a[2] : 0;
            v = c_add(v, c_conj(X[lin3(m0, m1, m2, n0, n1)]));
        }
        S[q] = c_scale(v, third * V[q]);
    }
}

__global__ void cscale_kernel(float2* X, long long n, float s) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        X[q] = c_scale(X[q], s);
}

// Block <-> subband address map of hourglass K at one level.  Line l of S_K
// along K is (c_a, c_b) over the two other axes a < b.
struct BlockMap {
    int K, ax, bx;
    int ha;            // extent of S_K along a (lines: l = c_a + ha * c_b)
    int ba, bb, ca;    // block sizes along a, b; block count along a
    long long first, blk;
    int sd0, sd1;      // subband dims along axes 0, 1
    long long sK;      // element stride of axis K inside a subband
    __device__ __forceinline__ long long addr(int l, int i) const {
        int c_a = l % ha, c_b = l / ha;
        int pa = c_a / ba, ra = c_a - pa * ba;
        int pb = c_b / bb, rb = c_b - pb * bb;
        int e[3];
        e[K] = i;
        e[ax] = ra;
        e[bx] = rb;
        return first + (long long)(pa + ca * pb) * blk + e[0] + (long long)sd0 * (e[1] + (long long)sd1 * e[2]);
    }
};

// C2R output of two block lines into the subbands (element stride es).
struct StoreRPairBlocks {
    float* dst;
    BlockMap bm;
    int nlines;
    int es;
    __device__ __forceinline__ void operator()(const float2* tile, int npad, int n, int l0, int T, int) const {
        const int total = T * n;
        const bool ifast = bm.K == 0;
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
            if (la < nlines) dst[bm.addr(la, i) * es] = v.x;
            if (la + 1 < nlines) dst[bm.addr(la + 1, i) * es] = v.y;
        }
    }
};

// Two subband lines along K packed as one complex line (R2C input).
struct LoadRPairBlocks {
    const float* src;
    BlockMap bm;
    int nlines;
    int es;
    __device__ __forceinline__ void operator()(float2* tile, int npad, int n, int l0, int T, int) const {
        const int total = T * n;
        const bool ifast = bm.K == 0;
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
            float a = la < nlines ? src[bm.addr(la, i) * es] : 0.f;
            float b = la + 1 < nlines ? src[bm.addr(la + 1, i) * es] : 0.f;
            tile[t * npad + i] = make_float2(a, b);
        }
    }
};

// Register-pass versions of the two block ops (see regpass.cuh).
struct RStoreRPairBlocks {
    static constexpr bool kStaged = false;
    float* dst;
    BlockMap bm;
    int nlines;
    int es;
    struct Ctx {
        long long a, b;
    };
    __device__ __forceinline__ Ctx line(int, int l, bool valid) const {
        int la = 2 * l;
        return Ctx{valid && la < nlines ? bm.addr(la, 0) : -1, valid && la + 1 < nlines ? bm.addr(la + 1, 0) : -1};
    }
    __device__ __forceinline__ void put(const Ctx& c, int k, float2 v) const {
        if (c.a >= 0) dst[(c.a + k * bm.sK) * es] = v.x;
        if (c.b >= 0) dst[(c.b + k * bm.sK) * es] = v.y;
    }
};

struct RLoadRPairBlocks {
    const float* src;
    BlockMap bm;
    int nlines;
    int es;
    struct Ctx {
        long long a, b;
    };
    __device__ __forceinline__ Ctx line(int, int l, bool valid) const {
        int la = 2 * l;
        return Ctx{valid && la < nlines ? bm.addr(la, 0) : -1, valid && la + 1 < nlines ? bm.addr(la + 1, 0) : -1};
    }
    __device__ __forceinline__ float2 get(const Ctx& c, int i) const {
        float a = c.a >= 0 ? src[(c.a + i * bm.sK) * es] : 0.f;
        float b = c.b >= 0 ? src[(c.b + i * bm.sK) * es] : 0.f;
        return make_float2(a, b);
    }
};

// ── set-up ───────────────────────────────────────────────────────────────────

template <class T>
static void upload_vec(DevMem& m, const std::vector<T>& v) {
    m.alloc(sizeof(T) * (v.empty() ? 1 : v.size()));
    if (!v.empty()) cuda_check(cudaMemcpy(m.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
}

void dec_plan_create(Plan& plan, const sfl_surf_params& p, const int dims[3], int dtype) {
    for (int d = 0; d < 3; ++d)
        if (dims[d] > 8192) throw ArgError("axis lengths above 8192 are not supported by this library");
    std::unique_ptr<DecPlan> D(new DecPlan);
    D->design = surf_design(p, dims, false);   // factors only: the tables are composed on the device
    const SurfDesign& S = D->design;
    for (int d = 0; d < 3; ++d) D->dims[d] = dims[d];
    D->nch = dtype == SFL_COMPLEX64 ? 2 : 1;
    D->J = p.scales;
    D->ncoef = S.offsets.back();
    for (int j = 0; j < D->J; ++j) {
        std::unique_ptr<DecLevelDev> L(new DecLevelDev);
        const PyrLevel& pl = S.pyramid[j];
        const ScaleDesign& sc = S.scales[j];
        for (int d = 0; d < 3; ++d) {
            L->n[d] = pl.n[d];
            L->nlow[d] = pl.nlow[d];
            L->cnt[d] = (int)pl.idx[d].size();
            upload_vec(L->idx[d], pl.idx[d]);
            upload_vec(L->idx_low[d], pl.idx_low[d]);
        }
        {
            // inverse box maps: spectrum index -> box position, where every
            // spectrum index is in the box at most once
            bool one_to_one = true;
            for (int d = 0; d < 3; ++d) {
                std::vector<int> inv((size_t)L->n[d], -1);
                for (int a = 0; a < L->cnt[d]; ++a) {
                    const int i = pl.idx[d][a];
                    if (i < 0 || i >= L->n[d] || inv[i] >= 0) {
                        one_to_one = false;
                        break;
                    }
                    inv[i] = a;
                }
                upload_vec(L->inv[d], inv);
            }
            L->merge_fused = one_to_one;
        }
        {
            // src/pyramid/fourier_pyramid.jl:221-240 (file numbering): the
            // separable lowpass L on the box, its D^-+1.5 scalings and
            // sqrt(1 - L^2), in float64.
            double Dv = (double)pl.D.p / (double)pl.D.q;
            double D15 = std::pow(Dv, 1.5);
            size_t nbox = (size_t)L->cnt[0] * L->cnt[1] * L->cnt[2];
            std::vector<float> ls(nbox), lm(nbox), hw(nbox);
            size_t q = 0;
            for (int c = 0; c < L->cnt[2]; ++c)
                for (int b = 0; b < L->cnt[1]; ++b)
                    for (int a = 0; a < L->cnt[0]; ++a, ++q) {
                        double Lv = pl.prof[0][a] * pl.prof[1][b] * pl.prof[2][c];
                        ls[q] = (float)(Lv / D15);
                        lm[q] = (float)(Lv * D15);
                        hw[q] = (float)std::sqrt(1 - Lv * Lv);
                    }
            upload_vec(L->lw_split, ls);
            upload_vec(L->lw_merge, lm);
            upload_vec(L->hw, hw);
        }
        int first = S.level_first[j];   // 0-based index of the level's first subband
        {
            float* Vp[3];
            for (int K = 0; K < 3; ++K) {
                for (int d = 0; d < 3; ++d) L->hd[K][d] = d == K ? sc.n[K] / 2 + 1 : sc.n[d];
                L->V[K].alloc(sizeof(float) * (size_t)L->hd[K][0] * L->hd[K][1] * L->hd[K][2]);
                Vp[K] = L->V[K].as<float>();
            }
            ritf_masks_device(sc.n, sc.P, Vp, 0);
        }
        for (int K = 0; K < 3; ++K) {
            for (const IRCStage& st : sc.stages[K]) {
                DecStageDev sd;
                sd.m = st.m - 1;
                sd.b = st.b;
                float2* fp[4];
                for (int w = 0; w < 4; ++w) {
                    sd.f[w].alloc(sizeof(float2) * (size_t)st.fac.nKh * st.fac.nm);
                    fp[w] = sd.f[w].as<float2>();
                }
                irc_slices_device(st.fac, fp, 0);
                L->stages[K].push_back(std::move(sd));
            }
            int nb = 1;
            for (int d = 0; d < 3; ++d) {
                L->counts[K][d] = 1 << sc.lv[K][d];
                L->bsize[K][d] = d == K ? sc.n[K] / 2 + 1 : sc.n[d] / L->counts[K][d];
                nb *= L->counts[K][d];
            }
            L->nsub[K] = nb;
            L->first_off[K] = S.offsets[first];
            L->blk_elems[K] = (long long)sc.n[K] * L->bsize[K][(K + 1) % 3] * L->bsize[K][(K + 2) % 3];
            first += nb;
        }
        D->lv.push_back(std::move(L));
    }
    // spectra: the input of every level and the coarse lowpass
    for (int j = 0; j <= D->J; ++j) {
        const int* n = j < D->J ? S.pyramid[j].n : S.pyramid[D->J - 1].nlow;
        std::unique_ptr<DevMem> m(new DevMem);
        m->alloc(sizeof(float2) * (size_t)n[0] * n[1] * n[2]);
        D->spectra.push_back(std::move(m));
    }
    for (auto& L : D->lv)
        for (int K = 0; K < 3; ++K) {
            const int* h = L->hd[K];
            L->S[K].alloc(sizeof(float2) * (size_t)h[0] * h[1] * h[2]);
        }
    D->ls.create();
    plan.dec.reset(D.release());
}

// ── drivers ──────────────────────────────────────────────────────────────────

namespace {

// The grid of irc_stage_kernel: one thread a bin pair, over S_K's dims with
// axis m halved.
dim3 irc_stage_grid(const int* hd, int m) {
    int pd[3] = {hd[0], hd[1], hd[2]};
    pd[m] /= 2;
    return grid3_blocks(pd[0], pd[1], pd[2]);
}

unsigned grid_for(long long total) {
    long long g = (total + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    if (g < 1) g = 1;
    return (unsigned)g;
}

// Full complex FFT of a real volume (dims d, element stride es) into X.
void fft_real_full(DecPlan& D, const float* x, int es, const int d[3], float2* X, cudaStream_t st) {
    Lines gin = axis_lines(d, 0);
    FFTLen* f0 = get_fft(D.ffts, d[0]);
    int pairs = (gin.nlines + 1) / 2;
    if (!launch_reg<false>(d[0], RLoadRPair{x, ZMap{}, gin, es}, RStoreFullPair{X, ZMap{}, gin, d[0]}, f0->sh.tw,
                           pairs, 1, false, st, "dec_fft_r2c")) {
        LoadRPair ld{x, ZMap{}, gin, es};
        StoreFullPair sto{X, ZMap{}, gin};
        launch_pass(ld, sto, f0->sh, pairs, 1, false, st, "dec_fft_r2c");
    }
    for (int a = 1; a < 3; ++a) {
        Lines g = axis_lines(d, a);
        FFTLen* f = get_fft(D.ffts, d[a]);
        if (launch_reg<false>(d[a], RLoadC{X, ZMap{}, g}, RStoreC{X, ZMap{}, g}, f->sh.tw, g.nlines, 1, true, st,
                              "dec_fft_c2c"))
            continue;
        LoadC l2{X, ZMap{}, g, 1.f};
        StoreC s2{X, ZMap{}, g, 1.f};
        launch_pass(l2, s2, f->sh, g.nlines, 1, false, st, "dec_fft_c2c");
    }
}

// Re(bfft(X)) * scale into a real volume (element stride es).
void ifft_full_real(DecPlan& D, float2* X, const int d[3], float* out, int es, float scale, cudaStream_t st) {
    for (int a = 2; a >= 1; --a) {
        Lines g = axis_lines(d, a);
        FFTLen* f = get_fft(D.ffts, d[a]);
        if (launch_reg<true>(d[a], RLoadC{X, ZMap{}, g}, RStoreC{X, ZMap{}, g}, f->sh.tw, g.nlines, 1, true, st,
                             "dec_fft_c2c"))
            continue;
        LoadC l2{X, ZMap{}, g, 1.f};
        StoreC s2{X, ZMap{}, g, 1.f};
        launch_pass(l2, s2, f->sh, g.nlines, 1, true, st, "dec_fft_c2c");
    }
    Lines g0 = axis_lines(d, 0);
    FFTLen* f0 = get_fft(D.ffts, d[0]);
    if (launch_reg<true>(d[0], RLoadC{X, ZMap{}, g0}, RStoreReal{out, ZMap{}, g0, es, scale}, f0->sh.tw, g0.nlines,
                         1, false, st, "dec_fft_real"))
        return;
    LoadC l0{X, ZMap{}, g0, 1.f};
    StoreReal s0{out, ZMap{}, g0, es, scale};
    launch_pass(l0, s0, f0->sh, g0.nlines, 1, true, st, "dec_fft_real");
}

// Lines of the segmented FFTs along axis m of a half-K spectrum (dims hd):
// blocks of length bl.
Lines block_lines(const int hd[3], int m, int bl) {
    long long str[3] = {1, hd[0], (long long)hd[0] * hd[1]};
    int o[2], k = 0;
    for (int d = 0; d < 3; ++d)
        if (d != m) o[k++] = d;
    Lines g;
    g.B0 = hd[o[0]];
    g.B1 = hd[o[1]];
    g.s0 = str[o[0]];
    g.s1 = str[o[1]];
    g.s2 = (long long)bl * str[m];
    g.si = str[m];
    g.nlines = hd[o[0]] * hd[o[1]] * (hd[m] / bl);
    g.fast_div();
    return g;
}

// Segmented FFTs along axis m of a half-K spectrum: blocks of length bl.
void block_fft(DecPlan& D, float2* S, const int hd[3], int m, int bl, bool inv, cudaStream_t st) {
    const Lines g = block_lines(hd, m, bl);
    FFTLen* f = get_fft(D.ffts, bl);
    bool tf = g.si != 1;
    bool done = inv ? launch_reg<true>(bl, RLoadC{S, ZMap{}, g}, RStoreC{S, ZMap{}, g}, f->sh.tw, g.nlines, 1, tf, st,
                                       "dec_block_fft")
                    : launch_reg<false>(bl, RLoadC{S, ZMap{}, g}, RStoreC{S, ZMap{}, g}, f->sh.tw, g.nlines, 1, tf,
                                        st, "dec_block_fft");
    if (done) return;
    LoadC ld{S, ZMap{}, g, 1.f};
    StoreC sto{S, ZMap{}, g, 1.f};
    launch_pass(ld, sto, f->sh, g.nlines, 1, inv, st, "dec_block_fft");
}

// Block FFTs of several spectra in one register pass: item z (grid.y) has its
// own spectrum and line geometry (same length); lines past an item's count
// read zeros and store nothing.
constexpr int kMaxLineJobs = 6;
struct LineJobs {
    int n = 0;
    float2* base[kMaxLineJobs];
    Lines g[kMaxLineJobs];
};
struct RLoadCJobs {
    LineJobs j;
    struct Ctx {
        const float2* p;
        long long si;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        const bool ok = valid && l < j.g[z].nlines;
        return Ctx{ok ? j.base[z] + j.g[z].base(l) : nullptr, j.g[z].si};
    }
    __device__ __forceinline__ float2 get(const Ctx& c, int i) const {
        return c.p ? c.p[(long long)i * c.si] : make_float2(0.f, 0.f);
    }
};
struct RStoreCJobs {
    static constexpr bool kStaged = false;
    LineJobs j;
    struct Ctx {
        float2* p;
        long long si;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        const bool ok = valid && l < j.g[z].nlines;
        return Ctx{ok ? j.base[z] + j.g[z].base(l) : nullptr, j.g[z].si};
    }
    __device__ __forceinline__ void put(const Ctx& c, int k, float2 v) const {
        if (c.p) c.p[(long long)k * c.si] = v;
    }
};

// Up to three line passes of one loader / store type as the jobs of one
// register-pass launch (grid.y = job): each job keeps its own geometry, and
// lines past a job's own count are invalid for it.
template <class L>
struct LoadJobs {
    L j[3];
    struct Ctx {
        typename L::Ctx c;
        int z;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const { return Ctx{j[z].line(0, l, valid), z}; }
    __device__ __forceinline__ float2 get(const Ctx& c, int i) const { return j[c.z].get(c.c, i); }
};
template <class S>
struct StoreJobs {
    static constexpr bool kStaged = S::kStaged;
    S j[3];
    struct Ctx {
        typename S::Ctx c;
        int z;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const { return Ctx{j[z].line(0, l, valid), z}; }
    __device__ __forceinline__ void put(const Ctx& c, int k, float2 v) const { j[c.z].put(c.c, k, v); }
    __device__ __forceinline__ void staged(const Ctx& c, const float2* xl, int p, int n2) const {
        j[c.z].staged(c.c, xl, p, n2);
    }
};

// The block FFTs of every hourglass of level L along both transverse axes,
// grouped into one launch per (block length, line layout); lengths without a
// register pass run one segmented pass per spectrum and axis.
void block_fft_level(DecPlan& D, DecLevelDev& L, bool inv, const bool skip[3], cudaStream_t st) {
    struct Item {
        int K, m, bl;
        bool tf;
        bool done;
    };
    Item items[6];
    int ni = 0;
    for (int K = 0; K < 3; ++K)
        for (int m = 0; m < 3; ++m)
            if (m != K && !skip[K]) items[ni++] = Item{K, m, L.bsize[K][m], m != 0, false};
    for (int a = 0; a < ni; ++a) {
        if (items[a].done) continue;
        LineJobs jobs;
        int member[kMaxLineJobs];   // the item of each job
        int nlines = 0;
        bool inGroup[3] = {false, false, false};
        for (int b = a; b < ni; ++b) {
            if (items[b].done || items[b].bl != items[a].bl || items[b].tf != items[a].tf) continue;
            const int K = items[b].K;
            // one job per spectrum in a launch (the two axes of S_K would race), and the axes of an
            // hourglass in their order
            bool earlier_pending = false;
            for (int c = 0; c < b; ++c)
                if (items[c].K == K && !items[c].done) earlier_pending = true;
            if (inGroup[K] || earlier_pending) continue;
            inGroup[K] = true;
            member[jobs.n] = b;
            jobs.base[jobs.n] = L.S[K].as<float2>();
            jobs.g[jobs.n] = block_lines(L.hd[K], items[b].m, items[b].bl);
            nlines = std::max(nlines, jobs.g[jobs.n].nlines);
            ++jobs.n;
            items[b].done = true;
        }
        const int bl = items[a].bl;
        FFTLen* f = get_fft(D.ffts, bl);
        const bool ok = inv ? launch_reg<true>(bl, RLoadCJobs{jobs}, RStoreCJobs{jobs}, f->sh.tw, nlines, jobs.n,
                                               items[a].tf, st, "dec_block_fft")
                            : launch_reg<false>(bl, RLoadCJobs{jobs}, RStoreCJobs{jobs}, f->sh.tw, nlines, jobs.n,
                                                items[a].tf, st, "dec_block_fft");
        if (!ok) {
            // no register pass for this length: one generic segmented pass per spectrum and axis
            for (int t = 0; t < jobs.n; ++t) {
                const Item& it = items[member[t]];
                block_fft(D, jobs.base[t], L.hd[it.K], it.m, bl, inv, st);
            }
        }
    }
}

BlockMap block_map(const DecLevelDev& L, int K) {
    BlockMap bm;
    bm.K = K;
    bm.ax = K == 0 ? 1 : 0;
    bm.bx = K == 2 ? 1 : 2;
    bm.ha = L.hd[K][bm.ax];
    bm.ba = L.bsize[K][bm.ax];
    bm.bb = L.bsize[K][bm.bx];
    bm.ca = L.counts[K][bm.ax];
    bm.first = L.first_off[K];
    bm.blk = L.blk_elems[K];
    int sd[3];
    for (int d = 0; d < 3; ++d) sd[d] = d == K ? L.n[K] : L.bsize[K][d];
    bm.sd0 = sd[0];
    bm.sd1 = sd[1];
    bm.sK = K == 0 ? 1 : (K == 1 ? (long long)sd[0] : (long long)sd[0] * sd[1]);
    return bm;
}

Lines k_lines(const DecLevelDev& L, int K) {
    const int* hd = L.hd[K];
    long long str[3] = {1, hd[0], (long long)hd[0] * hd[1]};
    int a = K == 0 ? 1 : 0, b = K == 2 ? 1 : 2;
    Lines g;
    g.nlines = hd[a] * hd[b];
    g.B0 = hd[a];
    g.B1 = hd[b];
    g.s0 = str[a];
    g.s1 = str[b];
    g.s2 = 0;
    g.si = str[K];
    g.fast_div();
    return g;
}

// Split of level j; with adjoint, the adjoint of the merge (the same gather
// with the merge's D^1.5 weights).
void pyr_split(DecPlan& D, int j, cudaStream_t st, bool adjoint = false) {
    DecLevelDev& L = *D.lv[j];
    float2* X = D.spectra[j]->as<float2>();
    float2* low = D.spectra[j + 1]->as<float2>();
    cuda_check(cudaMemsetAsync(low, 0, D.spectra[j + 1]->bytes, st), "memset");
    {
        int tok = prof_begin("dec_pyr_split", st);
        pyr_split_kernel<<<grid3_blocks(L.cnt[0], L.cnt[1], L.cnt[2]), grid3_threads(), 0, st>>>(
            X, low, L.n[0], L.n[1], L.nlow[0], L.nlow[1], L.idx[0].as<int>(), L.idx[1].as<int>(), L.idx[2].as<int>(),
            L.idx_low[0].as<int>(), L.idx_low[1].as<int>(), L.idx_low[2].as<int>(),
            adjoint ? L.lw_merge.as<float>() : L.lw_split.as<float>(), L.hw.as<float>(), L.cnt[0], L.cnt[1], L.cnt[2]);
        prof_end(tok, st);
    }
    cuda_check(cudaGetLastError(), "pyr_split_kernel");
}

// Merge of level j; with adjoint, the adjoint of the split (the same scatter
// with the split's D^-1.5 weights).
void pyr_merge(DecPlan& D, int j, cudaStream_t st, bool adjoint = false) {
    DecLevelDev& L = *D.lv[j];
    float2* X = D.spectra[j]->as<float2>();
    const float2* low = D.spectra[j + 1]->as<float2>();
    {
        int tok = prof_begin("dec_pyr_merge", st);
        pyr_merge_kernel<<<grid3_blocks(L.cnt[0], L.cnt[1], L.cnt[2]), grid3_threads(), 0, st>>>(
            X, low, L.n[0], L.n[1], L.nlow[0], L.nlow[1], L.idx[0].as<int>(), L.idx[1].as<int>(), L.idx[2].as<int>(),
            L.idx_low[0].as<int>(), L.idx_low[1].as<int>(), L.idx_low[2].as<int>(),
            adjoint ? L.lw_split.as<float>() : L.lw_merge.as<float>(), L.hw.as<float>(), L.cnt[0], L.cnt[1], L.cnt[2]);
        prof_end(tok, st);
    }
    cuda_check(cudaGetLastError(), "pyr_merge_kernel");
}

// The fused plane pass holds one k_K plane of S_K (n_m1 x n_m2 complex values)
// and one stage's two filter rows in shared memory: up to 227 KB, and at most
// kIrcPlaneMaxStages stages.
size_t irc_plane_smem(const DecLevelDev& L, int K) {
    const int m1 = K == 0 ? 1 : 0, m2 = K == 2 ? 1 : 2;
    const int a1 = L.hd[K][m1], a2 = L.hd[K][m2];
    // the padded plane, a stage's two filter rows and the two block lengths' twiddles
    return sizeof(float2) * ((size_t)irc_plane_pitch(a1) * a2 + 2 * (size_t)std::max(a1, a2) + (size_t)a1 + a2);
}

// Whether the plane pass of hourglass K also runs its block FFTs (both block
// lengths with a register line FFT).
bool irc_plane_fuses_blocks(const DecLevelDev& L, int K) {
    const int m1 = K == 0 ? 1 : 0, m2 = K == 2 ? 1 : 2;
    return irc_plane_block_len(L.bsize[K][m1]) && irc_plane_block_len(L.bsize[K][m2]);
}

bool irc_plane_fits(const DecLevelDev& L, int K) {
    return irc_plane_smem(L, K) <= 227 * 1024 && L.stages[K].size() <= (size_t)kIrcPlaneMaxStages;
}

IrcPlaneStages irc_plane_stages(const DecLevelDev& L, int K, bool synth) {
    IrcPlaneStages ps{};
    ps.n = (int)L.stages[K].size();
    for (int t = 0; t < ps.n; ++t) {
        const DecStageDev& sg = L.stages[K][t];
        ps.m[t] = sg.m;
        ps.b[t] = sg.b;
        ps.f0[t] = sg.f[synth ? 2 : 0].as<float2>();
        ps.f1[t] = sg.f[synth ? 3 : 1].as<float2>();
    }
    return ps;
}

template <bool SYNTH>
void irc_plane_configure(size_t smem) {
    static size_t configured = 0;
    if (smem > configured) {
        cuda_check(cudaFuncSetAttribute(irc_plane_kernel<SYNTH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem),
                   "cudaFuncSetAttribute(irc_plane)");
        configured = smem;
    }
}

// Whether the plane pass of level L runs hourglass K (its plane fits; the
// synthesis has nothing to do without stages) and whether it runs K's block
// FFTs too.
template <bool SYNTH>
bool irc_plane_runs(const DecLevelDev& L, int K) {
    return irc_plane_fits(L, K) && !(SYNTH && L.stages[K].empty());
}
template <bool SYNTH>
bool irc_plane_fuses(const DecLevelDev& L, int K) {
    return irc_plane_runs<SYNTH>(L, K) && irc_plane_fuses_blocks(L, K);
}

// One launch of the plane pass over every level's hourglasses whose plane
// fits (analysis: with the mask on load from the level spectrum; synthesis:
// hourglasses without stages have nothing to do), the finest level's planes
// first so that the coarser levels' smaller planes fill the last wave.
template <bool SYNTH>
void irc_plane_launch_levels(DecPlan& D, cudaStream_t st) {
    IrcPlaneJobs jobs{};
    size_t smem = 0;
    int blocks = 0;
    auto flush = [&] {
        if (jobs.n == 0) return;
        irc_plane_configure<SYNTH>(smem);
        int tok = prof_begin("dec_irc_plane", st);
        irc_plane_kernel<SYNTH><<<blocks, kIrcPlaneThreads, smem, st>>>(jobs);
        prof_end(tok, st);
        cuda_check(cudaGetLastError(), "irc_plane_kernel");
        jobs = IrcPlaneJobs{};
        smem = 0;
        blocks = 0;
    };
    for (int j = 0; j < D.J; ++j) {
        DecLevelDev& L = *D.lv[j];
        for (int K = 0; K < 3; ++K) {
            if (!irc_plane_runs<SYNTH>(L, K)) continue;
            if (jobs.n == kIrcPlaneMaxJobs) flush();
            IrcPlaneJob& jb = jobs.job[jobs.n++];
            jb.S = L.S[K].as<float2>();
            jb.X = D.spectra[j]->as<float2>();
            jb.n0 = L.n[0];
            jb.n1 = L.n[1];
            jb.K = K;
            jb.first = blocks;
            for (int d = 0; d < 3; ++d) jb.hd[d] = L.hd[K][d];
            jb.V = L.V[K].as<float>();
            int sb[3];
            for (int d = 0; d < 3; ++d) sb[d] = d == K ? L.n[K] : L.bsize[K][d];
            jb.s = (float)(1.0 / ((double)sb[0] * sb[1] * sb[2]));
            jb.sg = irc_plane_stages(L, K, SYNTH);
            if (irc_plane_fuses<SYNTH>(L, K)) {
                const int m1 = K == 0 ? 1 : 0, m2 = K == 2 ? 1 : 2;
                jb.bs1 = L.bsize[K][m1];
                jb.bs2 = L.bsize[K][m2];
                jb.tw1 = get_fft(D.ffts, jb.bs1)->sh.tw;
                jb.tw2 = get_fft(D.ffts, jb.bs2)->sh.tw;
            }
            blocks += L.hd[K][K];
            smem = std::max(smem, irc_plane_smem(L, K));
        }
    }
    flush();
}

// Level j of the analysis after the plane pass (irc_plane_launch_levels<false>,
// which ran the mask, every stage and, where both lengths allow, the block
// FFTs of each hourglass whose plane fits): the other hourglasses' mask and
// stages, the block FFTs the plane pass did not run, and the C2R along K
// into the subbands.
void scale_forward(DecPlan& D, int j, float* c, int es, cudaStream_t st) {
    DecLevelDev& L = *D.lv[j];
    const float2* X = D.spectra[j]->as<float2>();
    bool fuse[3];
    for (int K = 0; K < 3; ++K) fuse[K] = irc_plane_fuses<false>(L, K);
    for (int K = 0; K < 3; ++K) {
        const int* hd = L.hd[K];
        float2* S = L.S[K].as<float2>();
        int sb[3];
        for (int d = 0; d < 3; ++d) sb[d] = d == K ? L.n[K] : L.bsize[K][d];
        float s = (float)(1.0 / ((double)sb[0] * sb[1] * sb[2]));
        if (!irc_plane_fits(L, K)) {
            int tok = prof_begin("dec_hg_mask", st);
            hg_mask_kernel<<<grid3_blocks(hd[0], hd[1], hd[2]), grid3_threads(), 0, st>>>(
                X, L.n[0], L.n[1], S, hd[0], hd[1], hd[2], L.V[K].as<float>(), s);
            prof_end(tok, st);
            cuda_check(cudaGetLastError(), "hg_mask_kernel");
            for (auto& sg : L.stages[K]) {
                {
                    int tok = prof_begin("dec_irc", st);
                    irc_stage_kernel<<<irc_stage_grid(hd, sg.m), grid3_threads(), 0, st>>>(
                        S, hd[0], hd[1], hd[2], K, sg.m, sg.b, sg.f[0].as<float2>(), sg.f[1].as<float2>(), 0, 0);
                    prof_end(tok, st);
                }
                cuda_check(cudaGetLastError(), "irc_stage_kernel");
            }
        }
    }
    // the block FFTs of the other hourglasses, grouped by length and layout
    block_fft_level(D, L, true, fuse, st);
    // the C2R along K into the subbands: the hourglasses of one length and line layout in one launch
    bool done[3] = {false, false, false};
    for (int K = 0; K < 3; ++K) {
        if (done[K]) continue;
        LoadJobs<RLoadHPair> lj{};
        StoreJobs<RStoreRPairBlocks> sj{};
        int nj = 0, pairs = 0;
        for (int K2 = K; K2 < 3; ++K2) {
            if (done[K2] || L.n[K2] != L.n[K] || (K2 != 0) != (K != 0)) continue;
            Lines gk = k_lines(L, K2);
            lj.j[nj] = RLoadHPair{L.S[K2].as<float2>(), ZMap{}, gk, L.n[K2]};
            sj.j[nj] = RStoreRPairBlocks{c, block_map(L, K2), gk.nlines, es};
            pairs = std::max(pairs, (gk.nlines + 1) / 2);
            done[K2] = true;
            ++nj;
        }
        FFTLen* f = get_fft(D.ffts, L.n[K]);
        if (!launch_reg<true>(L.n[K], lj, sj, f->sh.tw, pairs, nj, K != 0, st, "dec_c2r_blocks")) {
            for (int t = 0; t < nj; ++t) {
                const RLoadHPair& l1 = lj.j[t];
                LoadHPair ld{l1.src, ZMap{}, l1.g};
                StoreRPairBlocks sto{c, sj.j[t].bm, l1.g.nlines, es};
                launch_pass(ld, sto, f->sh, (l1.g.nlines + 1) / 2, 1, true, st, "dec_c2r_blocks");
            }
        }
    }
}

// Level j of the synthesis up to the plane pass (irc_plane_launch_levels<true>,
// which runs every stage, in reverse, and where both lengths allow the block
// FFTs before them, of each hourglass whose plane fits): the R2C along K out
// of the subbands, the block FFTs the plane pass does not run and the other
// hourglasses' stages.
void scale_inverse(DecPlan& D, int j, const float* c, int es, cudaStream_t st) {
    DecLevelDev& L = *D.lv[j];
    // the R2C along K out of the subbands: the hourglasses of one length and line layout in one launch
    bool done[3] = {false, false, false};
    for (int K = 0; K < 3; ++K) {
        if (done[K]) continue;
        LoadJobs<RLoadRPairBlocks> lj{};
        StoreJobs<RStoreHalfPair> sj{};
        int nj = 0, pairs = 0;
        for (int K2 = K; K2 < 3; ++K2) {
            if (done[K2] || L.n[K2] != L.n[K] || (K2 != 0) != (K != 0)) continue;
            Lines gk = k_lines(L, K2);
            lj.j[nj] = RLoadRPairBlocks{c, block_map(L, K2), gk.nlines, es};
            sj.j[nj] = RStoreHalfPair{L.S[K2].as<float2>(), ZMap{}, gk, L.n[K2]};
            pairs = std::max(pairs, (gk.nlines + 1) / 2);
            done[K2] = true;
            ++nj;
        }
        FFTLen* f = get_fft(D.ffts, L.n[K]);
        if (!launch_reg<false>(L.n[K], lj, sj, f->sh.tw, pairs, nj, K != 0, st, "dec_r2c_blocks")) {
            for (int t = 0; t < nj; ++t) {
                const RStoreHalfPair& s1 = sj.j[t];
                LoadRPairBlocks ld{c, lj.j[t].bm, s1.g.nlines, es};
                StoreHalfPair sto{s1.dst, ZMap{}, s1.g};
                launch_pass(ld, sto, f->sh, (s1.g.nlines + 1) / 2, 1, false, st, "dec_r2c_blocks");
            }
        }
    }
    // the block FFTs of the hourglasses whose plane pass does not run them, grouped by length and layout
    bool fuse[3];
    for (int K = 0; K < 3; ++K) fuse[K] = irc_plane_fuses<true>(L, K);
    block_fft_level(D, L, false, fuse, st);
    for (int K = 0; K < 3; ++K) {
        const int* hd = L.hd[K];
        float2* S = L.S[K].as<float2>();
        if (!irc_plane_fits(L, K)) {
            for (int s = (int)L.stages[K].size() - 1; s >= 0; --s) {
                auto& sg = L.stages[K][s];
                {
                    int tok = prof_begin("dec_irc", st);
                    irc_stage_kernel<<<irc_stage_grid(hd, sg.m), grid3_threads(), 0, st>>>(S, hd[0], hd[1], hd[2], K, sg.m, sg.b,
                                                                        sg.f[2].as<float2>(), sg.f[3].as<float2>(), 1,
                                                                        0);
                    prof_end(tok, st);
                }
                cuda_check(cudaGetLastError(), "irc_stage_kernel");
            }
        }
    }
}

// Level j of the synthesis after the plane pass: the Hermitian sum of its
// three hourglasses into the level spectrum, then the pyramid merge with the
// coarser spectrum (inside the same pass where the box maps are one to one).
void scale_inverse_sum_merge(DecPlan& D, int j, cudaStream_t st) {
    DecLevelDev& L = *D.lv[j];
    HermArgs ha;
    for (int K = 0; K < 3; ++K) {
        ha.S[K] = L.S[K].as<float2>();
        ha.V[K] = L.V[K].as<float>();
    }
    MergeArgs mg{};
    if (L.merge_fused) {
        for (int d = 0; d < 3; ++d) {
            mg.inv[d] = L.inv[d].as<int>();
            mg.jl[d] = L.idx_low[d].as<int>();
        }
        mg.lw = L.lw_merge.as<float>();
        mg.hw = L.hw.as<float>();
        mg.low = D.spectra[j + 1]->as<float2>();
        mg.c0 = L.cnt[0];
        mg.c1 = L.cnt[1];
        mg.l0 = L.nlow[0];
        mg.l1 = L.nlow[1];
    }
    {
        int tok = prof_begin("dec_herm_sum", st);
        const dim3 g = grid3_blocks(L.n[0], L.n[1], L.n[2]);
        float2* X = D.spectra[j]->as<float2>();
        if (L.merge_fused)
            hermitian_sum_kernel<true><<<g, grid3_threads(), 0, st>>>(X, L.n[0], L.n[1], L.n[2], ha, 1.0f / 3.0f, mg);
        else
            hermitian_sum_kernel<false><<<g, grid3_threads(), 0, st>>>(X, L.n[0], L.n[1], L.n[2], ha, 1.0f / 3.0f, mg);
        prof_end(tok, st);
    }
    cuda_check(cudaGetLastError(), "hermitian_sum_kernel");
    if (!L.merge_fused) pyr_merge(D, j, st);
}

// Adjoint of scale_forward: the subbands of level j (real, in c) to the
// level's spectrum.  Per hourglass: a_k * R2C along K (a_k = 2 off the
// self-conjugate bins: the adjoint of the C2R), forward block FFTs (adjoint of
// the backward ones), the IRC stages in reverse order conjugate-transposed;
// then the zero-padded sum of V_K s_K S_K.
void scale_forward_adjoint(DecPlan& D, int j, const float* c, int es, cudaStream_t st) {
    DecLevelDev& L = *D.lv[j];
    HermArgs ha;
    float sK[3];
    for (int K = 0; K < 3; ++K) {
        const int* hd = L.hd[K];
        float2* S = L.S[K].as<float2>();
        Lines gk = k_lines(L, K);
        FFTLen* f = get_fft(D.ffts, L.n[K]);
        BlockMap bm = block_map(L, K);
        int pairs = (gk.nlines + 1) / 2;
        if (!launch_reg<false>(L.n[K], RLoadRPairBlocks{c, bm, gk.nlines, es},
                               RStoreHalfPair{S, ZMap{}, gk, L.n[K], 2.f}, f->sh.tw, pairs, 1, K != 0, st,
                               "dec_r2c_blocks")) {
            LoadRPairBlocks ld{c, bm, gk.nlines, es};
            StoreHalfPair sto{S, ZMap{}, gk, 2.f};
            launch_pass(ld, sto, f->sh, pairs, 1, false, st, "dec_r2c_blocks");
        }
        for (int m = 0; m < 3; ++m)
            if (m != K) block_fft(D, S, hd, m, L.bsize[K][m], false, st);
        for (int sg_i = (int)L.stages[K].size() - 1; sg_i >= 0; --sg_i) {
            auto& sg = L.stages[K][sg_i];
            int tok = prof_begin("dec_irc", st);
            irc_stage_kernel<<<irc_stage_grid(hd, sg.m), grid3_threads(), 0, st>>>(S, hd[0], hd[1], hd[2], K, sg.m, sg.b,
                                                                sg.f[0].as<float2>(), sg.f[1].as<float2>(), 1, 1);
            prof_end(tok, st);
            cuda_check(cudaGetLastError(), "irc_stage_kernel");
        }
        int sb[3];
        for (int d = 0; d < 3; ++d) sb[d] = d == K ? L.n[K] : L.bsize[K][d];
        sK[K] = (float)(1.0 / ((double)sb[0] * sb[1] * sb[2]));
        ha.S[K] = S;
        ha.V[K] = L.V[K].as<float>();
    }
    int tok = prof_begin("dec_hg_adjoint", st);
    hg_adjoint_sum_kernel<<<grid3_blocks(L.n[0], L.n[1], L.n[2]), grid3_threads(), 0, st>>>(D.spectra[j]->as<float2>(), L.n[0], L.n[1], L.n[2], ha,
                                                          sK[0], sK[1], sK[2]);
    prof_end(tok, st);
    cuda_check(cudaGetLastError(), "hg_adjoint_sum_kernel");
}

// Adjoint of scale_inverse: the level's spectrum to its subbands.  Per
// hourglass: the gather adjoint to the Hermitian sum, the synthesis IRC
// stages in forward order conjugate-transposed, backward block FFTs, and the
// C2R along K of S / a_k (the adjoint of the R2C).
void scale_inverse_adjoint(DecPlan& D, int j, float* c, int es, cudaStream_t st) {
    DecLevelDev& L = *D.lv[j];
    for (int K = 0; K < 3; ++K) {
        const int* hd = L.hd[K];
        float2* S = L.S[K].as<float2>();
        {
            int tok = prof_begin("dec_herm_gather", st);
            herm_gather_kernel<<<grid3_blocks(hd[0], hd[1], hd[2]), grid3_threads(), 0, st>>>(D.spectra[j]->as<float2>(), L.n[0], L.n[1], L.n[2], S,
                                                               L.V[K].as<float>(), K, 1.0f / 3.0f);
            prof_end(tok, st);
            cuda_check(cudaGetLastError(), "herm_gather_kernel");
        }
        for (auto& sg : L.stages[K]) {
            int tok = prof_begin("dec_irc", st);
            irc_stage_kernel<<<irc_stage_grid(hd, sg.m), grid3_threads(), 0, st>>>(S, hd[0], hd[1], hd[2], K, sg.m, sg.b,
                                                                sg.f[2].as<float2>(), sg.f[3].as<float2>(), 0, 1);
            prof_end(tok, st);
            cuda_check(cudaGetLastError(), "irc_stage_kernel");
        }
        for (int m = 0; m < 3; ++m)
            if (m != K) block_fft(D, S, hd, m, L.bsize[K][m], true, st);
        Lines gk = k_lines(L, K);
        FFTLen* f = get_fft(D.ffts, L.n[K]);
        BlockMap bm = block_map(L, K);
        int pairs = (gk.nlines + 1) / 2;
        if (!launch_reg<true>(L.n[K], RLoadHPair{S, ZMap{}, gk, L.n[K], 0.5f}, RStoreRPairBlocks{c, bm, gk.nlines, es},
                              f->sh.tw, pairs, 1, K != 0, st, "dec_c2r_blocks")) {
            LoadHPair ld{S, ZMap{}, gk, 0.5f};
            StoreRPairBlocks sto{c, bm, gk.nlines, es};
            launch_pass(ld, sto, f->sh, pairs, 1, true, st, "dec_c2r_blocks");
        }
    }
}

// f(j, stream) for the levels j = 0 .. J-1, level 0 on st and the others on
// the plan's side streams, all after the work already on st; st waits for
// all of them.
template <class F>
void per_level(DecPlan& D, cudaStream_t st, F f) {
    if (D.J < 2) {
        for (int j = 0; j < D.J; ++j) f(j, st);
        return;
    }
    LevelStreams& ls = D.ls;
    cuda_check(cudaEventRecord(ls.fork, st), "cudaEventRecord");
    const int nside = std::min(D.J - 1, 2);
    for (int k = 0; k < nside; ++k) cuda_check(cudaStreamWaitEvent(ls.side[k], ls.fork, 0), "cudaStreamWaitEvent");
    for (int j = 0; j < D.J; ++j) f(j, j == 0 ? st : ls.side[(j - 1) % 2]);
    for (int k = 0; k < nside; ++k) {
        cuda_check(cudaEventRecord(ls.join[k], ls.side[k]), "cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(st, ls.join[k], 0), "cudaStreamWaitEvent");
    }
}

void cscale(float2* X, long long n, float s, cudaStream_t st) {
    int tok = prof_begin("dec_scale", st);
    cscale_kernel<<<grid_for(n), 256, 0, st>>>(X, n, s);
    prof_end(tok, st);
    cuda_check(cudaGetLastError(), "cscale_kernel");
}

}  // namespace

void dec_analyze(DecPlan& D, const void* x, void* c, cudaStream_t st) {
    const int es = D.nch;
    const SurfDesign& S = D.design;
    for (int ch = 0; ch < D.nch; ++ch) {
        const float* xin = reinterpret_cast<const float*>(x) + ch;
        float* cout = reinterpret_cast<float*>(c) + ch;
        fft_real_full(D, xin, es, D.dims, D.spectra[0]->as<float2>(), st);
        // every split first (split j leaves level j's highpass in spectrum j), so
        // that one plane pass covers the hourglasses of all levels
        for (int j = 0; j < D.J; ++j) pyr_split(D, j, st);
        irc_plane_launch_levels<false>(D, st);
        // the levels' block FFTs and C2R, and the lowpass (after the coarsest level), concurrently
        const int* nl = S.pyramid[D.J - 1].nlow;
        const float scale = (float)(1.0 / ((double)nl[0] * nl[1] * nl[2]));
        per_level(D, st, [&](int j, cudaStream_t s) {
            scale_forward(D, j, cout, es, s);
            if (j == D.J - 1) ifft_full_real(D, D.spectra[D.J]->as<float2>(), nl, cout, es, scale, s);
        });
    }
}

void dec_synthesize(DecPlan& D, const void* c, void* x, cudaStream_t st) {
    const int es = D.nch;
    const SurfDesign& S = D.design;
    for (int ch = 0; ch < D.nch; ++ch) {
        const float* cin = reinterpret_cast<const float*>(c) + ch;
        float* xout = reinterpret_cast<float*>(x) + ch;
        const int* nl = S.pyramid[D.J - 1].nlow;
        // the levels' R2C and block FFTs, and the lowpass FFT (before the coarsest level), concurrently
        per_level(D, st, [&](int j, cudaStream_t s) {
            if (j == D.J - 1) fft_real_full(D, cin, es, nl, D.spectra[D.J]->as<float2>(), s);
            scale_inverse(D, j, cin, es, s);
        });
        irc_plane_launch_levels<true>(D, st);
        for (int j = D.J - 1; j >= 0; --j) scale_inverse_sum_merge(D, j, st);
        float scale = (float)(1.0 / ((double)D.dims[0] * D.dims[1] * D.dims[2]));
        ifft_full_real(D, D.spectra[0]->as<float2>(), D.dims, xout, es, scale, st);
    }
}

// x = A^T c, the adjoint of dec_analyze under the real inner products of the
// volume and the coefficient vector: every stage of the analysis replaced by
// its adjoint, in reverse order (FFT -> Re(bfft), split -> merge with the
// split weights, hourglass mask -> zero-padded V_K s, IRC -> conjugate
// transpose, backward block FFT -> forward, C2R -> a_k R2C, the lowpass's
// Re(bfft)/M -> FFT/M).
void dec_adjoint_analyze(DecPlan& D, const void* c, void* x, cudaStream_t st) {
    const int es = D.nch;
    const SurfDesign& S = D.design;
    for (int ch = 0; ch < D.nch; ++ch) {
        const float* cin = reinterpret_cast<const float*>(c) + ch;
        float* xout = reinterpret_cast<float*>(x) + ch;
        const int* nl = S.pyramid[D.J - 1].nlow;
        const long long M = (long long)nl[0] * nl[1] * nl[2];
        fft_real_full(D, cin, es, nl, D.spectra[D.J]->as<float2>(), st);
        cscale(D.spectra[D.J]->as<float2>(), M, (float)(1.0 / (double)M), st);
        for (int j = D.J - 1; j >= 0; --j) {
            scale_forward_adjoint(D, j, cin, es, st);
            pyr_merge(D, j, st, true);
        }
        ifft_full_real(D, D.spectra[0]->as<float2>(), D.dims, xout, es, 1.0f, st);
    }
}

// c = S^T x, the adjoint of dec_synthesize: FFT/N of x, then per level the
// adjoint of the merge (a split with the merge weights) and of the scale's
// inverse, and Re(bfft) of the coarse spectrum into the lowpass.
void dec_adjoint_synthesize(DecPlan& D, const void* x, void* c, cudaStream_t st) {
    const int es = D.nch;
    const SurfDesign& S = D.design;
    for (int ch = 0; ch < D.nch; ++ch) {
        const float* xin = reinterpret_cast<const float*>(x) + ch;
        float* cout = reinterpret_cast<float*>(c) + ch;
        const long long N = (long long)D.dims[0] * D.dims[1] * D.dims[2];
        fft_real_full(D, xin, es, D.dims, D.spectra[0]->as<float2>(), st);
        cscale(D.spectra[0]->as<float2>(), N, (float)(1.0 / (double)N), st);
        for (int j = 0; j < D.J; ++j) {
            pyr_split(D, j, st, true);
            scale_inverse_adjoint(D, j, cout, es, st);
        }
        const int* nl = S.pyramid[D.J - 1].nlow;
        ifft_full_real(D, D.spectra[D.J]->as<float2>(), nl, cout, es, 1.0f, st);
    }
}

}  // namespace sfl
