// Plane-major NSSurfacelet passes: the 3-D real FFTs of the cascade as one
// pencil pass along axis 1 and one plane pass over axes (2, 3).
//
// Spectra live in plane-major order on the rfft grid: element (k1, k2, k3) at
// k2 + n2 (k3 + n3 k1), so plane k1 is one contiguous block of E = n2 n3
// points.
//
//   pencil pass: the real FFT along axis 1 of a tile of 2 LP lines, two lines
//     per complex FFT; real data is staged through shared memory so that the
//     column-major volume is read and written in contiguous runs, and the
//     spectra are read and written with consecutive lanes on consecutive
//     lines (one contiguous run per plane).
//   plane pass: a CTA owns one plane (and one subband): the FFT along axis 3
//     reads the plane straight from global memory (consecutive lanes on
//     consecutive columns) with the subband mask fused into the load and
//     leaves the plane in shared memory; the FFT along axis 2 runs on its
//     rows and writes (or mask-accumulates) straight to global memory.
//
// Per subband the analysis is one plane pass and one pencil pass (instead of
// three line passes), and the synthesis likewise.
#include "ns_mask.cuh"
#include "passes.cuh"
#include "plan.h"
#include "prof.h"
#include "regfft.cuh"
#include "tma.cuh"

namespace sfl {

enum PlaneMode { kPlaneFwd = 0, kPlaneInvMask = 1, kPlaneFwdMaskAcc = 2, kPlaneInvSum = 3 };

struct PlaneArgs {
    const float2* in;      // input spectra (plane-major)
    long long in_z;        // stride between items of the input (0: shared)
    float2* out;           // output spectra
    long long out_z;
    float2* acc;           // partial accumulators (kPlaneFwdMaskAcc: one per item slot; kPlaneInvSum: summed)
    int npart;             // kPlaneInvSum: partials summed on load
    int init;              // kPlaneFwdMaskAcc: first contribution (store instead of add)
    NSMaskTables tb;       // G / Bl in plane-major order
    const NSItem* items;
    int item0;
    int synth;
    const float2* twr;     // twiddles of the row length (n2)
    const float2* twc;     // twiddles of the column length (n3)
    int n2, n3;
    long long E;           // plane size n2 n3
    long long H;           // spectrum size h1 n2 n3
    int* status;           // device status word (bounded waits)
};

// Row pitch (float2) of the plane in shared memory: room for the row FFT's
// padded exchange (N1 (N2 + 1) slots) and 8 mod 16, so that two rows in a
// half-warp fall on disjoint banks.
template <int NR>
struct PlanePitch {
    using G = RegGeom<NR>;
    static constexpr int need = NR > G::N1 * (G::N2 + 1) ? NR : G::N1 * (G::N2 + 1);
    static constexpr int value = need + ((8 - need % 16) + 16) % 16;
};

// Mask of item `it` at plane-major point (k1, k2, k3), linear index q.
__device__ __forceinline__ float ns_mask_p(const NSMaskTables& tb, const NSItem& it, int k1, int k2, int k3,
                                           long long q, bool synth) {
    if (it.kind == 1) {
        const float* v = tb.vec;
        return v[tb.low_off[0] + k1] * v[tb.low_off[1] + k2] * v[tb.low_off[2] + k3];
    }
    if (synth && !tb.tight) return tb.Bl[(long long)it.lv * tb.H + q];
    float g = tb.G[(long long)it.g * tb.H + q];
    int kk[3] = {k1, k2, k3};
    float wa = tb.planes[it.wa_off + kk[it.wa_lo] + it.wa_dlo * kk[it.wa_hi]];
    float wb = tb.planes[it.wb_off + kk[it.wb_lo] + it.wb_dlo * kk[it.wb_hi]];
    return (g * wa) * wb;
}

// Per-CTA wedge-plane addressing: the value of a wedge plane at in-plane
// point (col = k2, row = k3) of plane k1 is planes[base + col * sc + row * sr].
struct WedgeAddr {
    int base, sc, sr;
};

__device__ __forceinline__ WedgeAddr wedge_addr(int off, int lo, int hi, int dlo, int k1) {
    // plane over axes (lo, hi), index off + k_lo + dlo * k_hi, axes 0 = k1, 1 = k2 (col), 2 = k3 (row)
    WedgeAddr w{off, 0, 0};
    if (lo == 0) {
        w.base += k1;
        if (hi == 1) w.sc = dlo; else w.sr = dlo;
    } else {   // (1, 2)
        w.sc = 1;
        w.sr = dlo;
    }
    return w;
}

template <int NR, int NC, int MODE>
__global__ void __launch_bounds__(512) plane_kernel(PlaneArgs a) {
    using GC = RegGeom<NC>;   // column FFT (along axis 3)
    using GR = RegGeom<NR>;   // row FFT (along axis 2)
    constexpr int PITCH = PlanePitch<NR>::value;
    constexpr int T = 512;
    constexpr bool kTmaIn = MODE != kPlaneInvSum;                            // plane staged by bulk copies
    constexpr bool kMaskTab = MODE == kPlaneInvMask || MODE == kPlaneFwdMaskAcc;
    constexpr bool kBulkOut = MODE == kPlaneFwd || MODE == kPlaneInvMask;    // rows leave by bulk stores
    extern __shared__ __align__(16) unsigned char smraw[];
    float2* plane = reinterpret_cast<float2*>(smraw);                          // [NC][PITCH]
    float* gbuf = reinterpret_cast<float*>(plane + NC * PITCH);              // [NC][NR] mask plane
    uint64_t* bar = reinterpret_cast<uint64_t*>(gbuf + (kMaskTab ? NC * NR : 0));
    const int tid = threadIdx.x;
    const int k1 = blockIdx.x;
    const int z = blockIdx.y;
    const long long pbase = (long long)k1 * a.E;
    const bool invc = MODE == kPlaneInvMask || MODE == kPlaneInvSum;
    NSItem it{};
    if (kMaskTab) it = a.items[a.item0 + z];
    // the item's mask on this plane: a table plane (G or, for the synthesis of
    // an untight bank, the bandpass B), the lowpass's separable factors, and
    // the two wedge planes
    const bool low = kMaskTab && it.kind == 1;
    const bool plain = kMaskTab && !low && a.synth && !a.tb.tight;
    const float* mtab = !kMaskTab || low ? nullptr
                        : plain ? a.tb.Bl + (long long)it.lv * a.H + pbase
                                : a.tb.G + (long long)it.g * a.H + pbase;
    WedgeAddr wa{0, 0, 0}, wb{0, 0, 0};
    float lowc = 0.f;
    if (kMaskTab && !low && !plain) {
        wa = wedge_addr(it.wa_off, it.wa_lo, it.wa_hi, it.wa_dlo, k1);
        wb = wedge_addr(it.wb_off, it.wb_lo, it.wb_hi, it.wb_dlo, k1);
    }
    if (low) lowc = a.tb.vec[a.tb.low_off[0] + k1];
    auto mask_at = [&](int col, int row) -> float {
        if (low) return lowc * a.tb.vec[a.tb.low_off[1] + col] * a.tb.vec[a.tb.low_off[2] + row];
        float g = gbuf[row * NR + col];
        if (plain) return g;
        const float* P = a.tb.planes;
        return (g * __ldg(&P[wa.base + col * wa.sc + row * wa.sr])) * __ldg(&P[wb.base + col * wb.sc + row * wb.sr]);
    };

    // ── stage the plane (and its mask plane) with bulk copies ──
    if (kTmaIn) {
        const float2* src = a.in + (MODE == kPlaneInvMask ? 0 : (long long)z * a.in_z) + pbase;
        const uint32_t bytes = (uint32_t)(NC * NR * sizeof(float2)) + (mtab ? (uint32_t)(NC * NR * sizeof(float)) : 0u);
        if (tid == 0) {
            mbar_init(bar, 1);
            fence_barrier_init();
        }
        __syncthreads();
        if (tid == 0) mbar_arrive_expect_tx(bar, bytes);
        __syncthreads();
        for (int r = tid; r < NC; r += T) {
            bulk_load(plane + r * PITCH, src + (long long)r * NR, NR * sizeof(float2), bar);
            if (mtab) bulk_load(gbuf + r * NR, mtab + (long long)r * NR, NR * sizeof(float), bar);
        }
        mbar_wait_bounded(bar, 0, a.status);
    }

    // ── column FFTs along axis 3 ──
    {
        constexpr int N1 = GC::N1, N2 = GC::N2;
        constexpr int CPR = T / N2;                  // columns per round
        constexpr int ROUNDS = (NR + CPR - 1) / CPR;
        const int cl = tid % CPR, p = tid / CPR;
#pragma unroll 1
        for (int rd = 0; rd < ROUNDS; ++rd) {
            const int col = rd * CPR + cl;
            const bool ok = col < NR;
            float2 v[N1];
#pragma unroll
            for (int r = 0; r < N1; ++r) {
                const int row = p + N2 * r;
                float2 x = make_float2(0.f, 0.f);
                if (ok) {
                    if (MODE == kPlaneInvSum) {
                        // Kahan sum of the partial accumulators, from global memory
                        const long long e = (long long)row * NR + col;
                        float2 cmp = make_float2(0.f, 0.f);
                        for (int q = 0; q < a.npart; ++q) {
                            float2 y = c_sub(a.acc[q * a.H + pbase + e], cmp);
                            float2 t = c_add(x, y);
                            cmp = c_sub(c_sub(t, x), y);
                            x = t;
                        }
                    } else {
                        x = plane[row * PITCH + col];
                        if (MODE == kPlaneInvMask) x = c_scale(x, mask_at(col, row));
                    }
                }
                v[r] = x;
            }
            if (invc) RegDft<N1, true>::run(v); else RegDft<N1, false>::run(v);
#pragma unroll
            for (int m = 1; m < N1; ++m) {
                float2 w = __ldg(&a.twc[p * m]);
                if (invc) w.y = -w.y;
                v[m] = c_mul(v[m], w);
            }
            __syncthreads();    // every input row of this round's columns has been read
            if (ok) {
#pragma unroll
                for (int m = 0; m < N1; ++m) plane[(m * N2 + p) * PITCH + col] = v[m];
            }
            __syncthreads();
            float2 u[GC::M * N2];
#pragma unroll
            for (int j = 0; j < GC::M; ++j) {
                const int m = p + N2 * j;
                float2 w[N2];
#pragma unroll
                for (int pp = 0; pp < N2; ++pp) w[pp] = ok ? plane[(m * N2 + pp) * PITCH + col] : make_float2(0.f, 0.f);
                if (invc) RegDft<N2, true>::run(w); else RegDft<N2, false>::run(w);
#pragma unroll
                for (int k = 0; k < N2; ++k) u[j * N2 + k] = w[k];
            }
            __syncthreads();
            if (ok) {
#pragma unroll
                for (int j = 0; j < GC::M; ++j)
#pragma unroll
                    for (int k = 0; k < N2; ++k) plane[((p + N2 * j) + N1 * k) * PITCH + col] = u[j * N2 + k];
            }
        }
    }
    __syncthreads();

    // ── row FFTs along axis 2 ──
    {
        constexpr int N1 = GR::N1, N2 = GR::N2;
        constexpr int RPR = T / N2;                  // rows per round
        constexpr int ROUNDS = (NC + RPR - 1) / RPR;
        constexpr int XR = N2 + 1;
        const int p = tid % N2, rl = tid / N2;
#pragma unroll 1
        for (int rd = 0; rd < ROUNDS; ++rd) {
            const int row = rd * RPR + rl;
            const bool ok = row < NC;
            float2* prow = plane + (ok ? row : 0) * PITCH;
            float2 v[N1];
#pragma unroll
            for (int r = 0; r < N1; ++r) v[r] = ok ? prow[p + N2 * r] : make_float2(0.f, 0.f);
            if (invc) RegDft<N1, true>::run(v); else RegDft<N1, false>::run(v);
#pragma unroll
            for (int m = 1; m < N1; ++m) {
                float2 w = __ldg(&a.twr[p * m]);
                if (invc) w.y = -w.y;
                v[m] = c_mul(v[m], w);
            }
            __syncwarp();
            if (ok) {
#pragma unroll
                for (int m = 0; m < N1; ++m) prow[m * XR + p] = v[m];
            }
            __syncwarp();
            float2 u[GR::M * N2];
#pragma unroll
            for (int j = 0; j < GR::M; ++j) {
                const int m = p + N2 * j;
                float2 w[N2];
#pragma unroll
                for (int pp = 0; pp < N2; ++pp) w[pp] = ok ? prow[m * XR + pp] : make_float2(0.f, 0.f);
                if (invc) RegDft<N2, true>::run(w); else RegDft<N2, false>::run(w);
#pragma unroll
                for (int k = 0; k < N2; ++k) u[j * N2 + k] = w[k];
            }
            if (kBulkOut) {
                __syncwarp();   // the row's exchange slots are read; its outputs go back in place
                if (ok) {
#pragma unroll
                    for (int j = 0; j < GR::M; ++j)
#pragma unroll
                        for (int k = 0; k < N2; ++k) prow[(p + N2 * j) + N1 * k] = u[j * N2 + k];
                }
            } else if (ok) {
#pragma unroll
                for (int j = 0; j < GR::M; ++j)
#pragma unroll
                    for (int k = 0; k < N2; ++k) {
                        const int k2 = (p + N2 * j) + N1 * k;
                        const long long e = (long long)row * NR + k2;
                        if (MODE == kPlaneFwdMaskAcc) {
                            float2* dst = a.acc + (long long)z * a.H + pbase + e;
                            const float2 y = c_scale(u[j * N2 + k], mask_at(k2, row));
                            if (a.init)
                                *dst = y;
                            else
                                atomicAdd(dst, y);   // a single contribution per launch: a fire-and-forget add
                        } else {
                            a.out[pbase + e] = u[j * N2 + k];
                        }
                    }
            }
        }
    }

    // ── rows back to global memory with bulk stores ──
    if (kBulkOut) {
        fence_proxy_async();
        __syncthreads();
        float2* dst = a.out + (MODE == kPlaneInvMask ? (long long)z * a.out_z : 0) + pbase;
        for (int r = tid; r < NC; r += T) {
            bulk_store(dst + (long long)r * NR, plane + r * PITCH, NR * sizeof(float2));
            bulk_commit();
        }
        bulk_wait_read();
    }
}

template <int NR, int NC, int MODE>
struct PlaneSmem {
    static constexpr bool kMaskTab = MODE == kPlaneInvMask || MODE == kPlaneFwdMaskAcc;
    static constexpr size_t bytes = sizeof(float2) * (size_t)NC * PlanePitch<NR>::value +
                                    (kMaskTab ? sizeof(float) * (size_t)NC * NR : 0) + 16;
};

// ── pencil passes along axis 1 ────────────────────────────────────────────────

// Real lines (column-major volume; element stride es; item z at zm.off(z))
// -> plane-major half spectra out + z * H: two lines per complex FFT.
struct PencilArgs {
    const float* rin;       // r2c: real input
    float* rout;            // c2r: real output
    const float2* cin;      // c2r: spectra
    float2* cout;           // r2c: spectra
    ZMap zm;                // real side item offsets
    long long cz;           // spectrum side item stride
    int es;
    float scale;
    int n1;                 // line length (real)
    int nlines;             // n2 n3
    long long E;            // plane stride of the spectra
    const float2* tw;
};

template <int N>
struct PencilGeom {
    using G = RegGeom<N>;
    static constexpr int LPAIR = G::LP;           // line pairs per CTA
    static constexpr int NL = 2 * LPAIR;          // real lines per CTA
    static constexpr int RP = N + 4;              // real tile row pitch (floats), 4 mod 32: pairs of rows on disjoint banks
    static constexpr int H = N / 2 + 1;
    // shared memory: the real tile (NL x RP floats) and the FFT exchange / complex tile
    static constexpr size_t XBYTES = sizeof(float2) * (size_t)LPAIR * G::XLINE;
    static constexpr size_t RBYTES = sizeof(float) * (size_t)NL * RP;
    static constexpr size_t CBYTES = sizeof(float2) * (size_t)2 * LPAIR * H;
    static constexpr size_t bytes = (XBYTES > RBYTES ? (XBYTES > CBYTES ? XBYTES : CBYTES) : (RBYTES > CBYTES ? RBYTES : CBYTES));
};

template <int N>
__global__ void __launch_bounds__(256) pencil_r2c_kernel(PencilArgs a) {
    using PG = PencilGeom<N>;
    using G = typename PG::G;
    constexpr int N1 = G::N1, N2 = G::N2, LPAIR = PG::LPAIR, NL = PG::NL, RP = PG::RP, H = PG::H;
    extern __shared__ float2 sm[];
    float* rt = reinterpret_cast<float*>(sm);
    const int tid = threadIdx.x;
    const int z = blockIdx.y;
    const int L0 = blockIdx.x * NL;            // first real line of the tile
    const float* src = a.rin + a.zm.off(z);
    // stage the real tile: consecutive lanes on consecutive elements of a line
    for (int idx = tid; idx < NL * N; idx += 256) {
        const int i = idx % N, ln = idx / N;
        const int L = L0 + ln;
        rt[ln * RP + i] = L < a.nlines ? src[((long long)L * a.n1 + i) * a.es] : 0.f;
    }
    __syncthreads();
    // FFT of pair l = lines 2l, 2l+1 of the tile
    const int p = tid % N2, l = tid / N2;
    float2 v[N1];
#pragma unroll
    for (int r = 0; r < N1; ++r) v[r] = make_float2(rt[(2 * l) * RP + p + N2 * r], rt[(2 * l + 1) * RP + p + N2 * r]);
    RegDft<N1, false>::run(v);
#pragma unroll
    for (int m = 1; m < N1; ++m) v[m] = c_mul(v[m], __ldg(&a.tw[p * m]));
    __syncthreads();     // the real tile is dead; its space becomes the exchange
    float2* xl = sm + l * G::XLINE;
#pragma unroll
    for (int m = 0; m < N1; ++m) xl[m * G::XROW + p] = v[m];
    __syncthreads();
    float2 u[G::M * N2];
#pragma unroll
    for (int j = 0; j < G::M; ++j) {
        const int m = p + N2 * j;
        float2 w[N2];
#pragma unroll
        for (int pp = 0; pp < N2; ++pp) w[pp] = xl[m * G::XROW + pp];
        RegDft<N2, false>::run(w);
#pragma unroll
        for (int k = 0; k < N2; ++k) u[j * N2 + k] = w[k];
    }
    __syncthreads();
    // Z of pair l in natural order: zt[l][k], k < N  (complex tile reuses the space)
    float2* zt = sm;
#pragma unroll
    for (int j = 0; j < G::M; ++j)
#pragma unroll
        for (int k = 0; k < N2; ++k) zt[l * (N + 1) + (p + N2 * j) + N1 * k] = u[j * N2 + k];
    __syncthreads();
    // unpack and store: consecutive lanes on consecutive pairs (lines), one plane at a time
    float2* dst = a.cout + (long long)z * a.cz;
    for (int idx = tid; idx < LPAIR * H; idx += 256) {
        const int pl = idx % LPAIR, k = idx / LPAIR;
        const float2 zk = zt[pl * (N + 1) + k];
        const float2 zn = zt[pl * (N + 1) + (k == 0 ? 0 : N - k)];
        const int La = L0 + 2 * pl;
        const long long o = (long long)k * a.E;
        if (La < a.nlines) dst[o + La] = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
        if (La + 1 < a.nlines) dst[o + La + 1] = make_float2(0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x));
    }
}

template <int N>
__global__ void __launch_bounds__(256) pencil_c2r_kernel(PencilArgs a) {
    using PG = PencilGeom<N>;
    using G = typename PG::G;
    constexpr int N1 = G::N1, N2 = G::N2, LPAIR = PG::LPAIR, NL = PG::NL, RP = PG::RP, H = PG::H;
    extern __shared__ float2 sm[];
    const int tid = threadIdx.x;
    const int z = blockIdx.y;
    const int L0 = blockIdx.x * NL;
    const float2* src = a.cin + (long long)z * a.cz;
    // stage the half spectra of the tile's lines: ht[line][k], consecutive lanes on consecutive lines
    float2* ht = sm;
    for (int idx = tid; idx < NL * H; idx += 256) {
        const int ln = idx % NL, k = idx / NL;
        const int L = L0 + ln;
        ht[ln * H + k] = L < a.nlines ? src[(long long)k * a.E + L] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const int p = tid % N2, l = tid / N2;
    float2 v[N1];
#pragma unroll
    for (int r = 0; r < N1; ++r) {
        const int i = p + N2 * r;
        const int k = 2 * i <= N ? i : N - i;
        float2 A = ht[(2 * l) * H + k], B = ht[(2 * l + 1) * H + k];
        if (k == 0 || 2 * k == N) {
            A.y = 0.f;
            B.y = 0.f;
        }
        v[r] = 2 * i <= N ? make_float2(A.x - B.y, A.y + B.x) : make_float2(A.x + B.y, B.x - A.y);
    }
    RegDft<N1, true>::run(v);
#pragma unroll
    for (int m = 1; m < N1; ++m) {
        float2 w = __ldg(&a.tw[p * m]);
        w.y = -w.y;
        v[m] = c_mul(v[m], w);
    }
    __syncthreads();
    float2* xl = sm + l * G::XLINE;
#pragma unroll
    for (int m = 0; m < N1; ++m) xl[m * G::XROW + p] = v[m];
    __syncthreads();
    float2 u[G::M * N2];
#pragma unroll
    for (int j = 0; j < G::M; ++j) {
        const int m = p + N2 * j;
        float2 w[N2];
#pragma unroll
        for (int pp = 0; pp < N2; ++pp) w[pp] = xl[m * G::XROW + pp];
        RegDft<N2, true>::run(w);
#pragma unroll
        for (int k = 0; k < N2; ++k) u[j * N2 + k] = w[k];
    }
    __syncthreads();
    // real tile: line 2l = Re, line 2l+1 = Im
    float* rt = reinterpret_cast<float*>(sm);
#pragma unroll
    for (int j = 0; j < G::M; ++j)
#pragma unroll
        for (int k = 0; k < N2; ++k) {
            const int i = (p + N2 * j) + N1 * k;
            rt[(2 * l) * RP + i] = u[j * N2 + k].x * a.scale;
            rt[(2 * l + 1) * RP + i] = u[j * N2 + k].y * a.scale;
        }
    __syncthreads();
    float* dst = a.rout + a.zm.off(z);
    for (int idx = tid; idx < NL * N; idx += 256) {
        const int i = idx % N, ln = idx / N;
        const int L = L0 + ln;
        if (L < a.nlines) dst[((long long)L * a.n1 + i) * a.es] = rt[ln * RP + i];
    }
}

// ── launch helpers ───────────────────────────────────────────────────────────

template <int NR, int NC, int MODE>
static void launch_plane_nm(const PlaneArgs& a, int nplanes, int nz, cudaStream_t st, const char* tag) {
    static bool configured = false;
    constexpr size_t smem = PlaneSmem<NR, NC, MODE>::bytes;
    if (!configured) {
        cuda_check(cudaFuncSetAttribute(plane_kernel<NR, NC, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem),
                   "cudaFuncSetAttribute(plane)");
        configured = true;
    }
    int tok = prof_begin(tag, st);
    plane_kernel<NR, NC, MODE><<<dim3(nplanes, nz), 512, smem, st>>>(a);
    prof_end(tok, st);
    cuda_check(cudaGetLastError(), "plane_kernel launch");
}

template <int MODE>
static bool launch_plane(int n2, int n3, const PlaneArgs& a, int nplanes, int nz, cudaStream_t st, const char* tag) {
#define SFL_PLANE_CASE(A, B)                                                    \
    if (n2 == A && n3 == B) {                                                   \
        launch_plane_nm<A, B, MODE>(a, nplanes, nz, st, tag);                   \
        return true;                                                            \
    }
    SFL_PLANE_CASE(64, 64)
    SFL_PLANE_CASE(96, 96)
    SFL_PLANE_CASE(128, 128)
    SFL_PLANE_CASE(64, 128)
    SFL_PLANE_CASE(128, 64)
#undef SFL_PLANE_CASE
    return false;
}

bool ns_plane_supported(int n1, int n2, int n3) {
    bool pencil = n1 == 64 || n1 == 96 || n1 == 128 || n1 == 160 || n1 == 256;
    bool plane = (n2 == 64 && n3 == 64) || (n2 == 96 && n3 == 96) || (n2 == 128 && n3 == 128) ||
                 (n2 == 64 && n3 == 128) || (n2 == 128 && n3 == 64);
    return pencil && plane;
}

template <int N>
static void launch_pencil_n(bool r2c, const PencilArgs& a, int nz, cudaStream_t st, const char* tag) {
    using PG = PencilGeom<N>;
    static bool cfg_r = false, cfg_c = false;
    bool& cfg = r2c ? cfg_r : cfg_c;
    if (!cfg) {
        if (r2c)
            cuda_check(cudaFuncSetAttribute(pencil_r2c_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)PG::bytes),
                       "cudaFuncSetAttribute(pencil)");
        else
            cuda_check(cudaFuncSetAttribute(pencil_c2r_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)PG::bytes),
                       "cudaFuncSetAttribute(pencil)");
        cfg = true;
    }
    dim3 grid((a.nlines + PG::NL - 1) / PG::NL, nz);
    int tok = prof_begin(tag, st);
    if (r2c)
        pencil_r2c_kernel<N><<<grid, 256, PG::bytes, st>>>(a);
    else
        pencil_c2r_kernel<N><<<grid, 256, PG::bytes, st>>>(a);
    prof_end(tok, st);
    cuda_check(cudaGetLastError(), "pencil kernel launch");
}

static void launch_pencil(bool r2c, int n1, const PencilArgs& a, int nz, cudaStream_t st) {
    const char* tag = r2c ? "ns_pencil_r2c" : "ns_pencil_c2r";
    switch (n1) {
        case 64: launch_pencil_n<64>(r2c, a, nz, st, tag); return;
        case 96: launch_pencil_n<96>(r2c, a, nz, st, tag); return;
        case 128: launch_pencil_n<128>(r2c, a, nz, st, tag); return;
        case 160: launch_pencil_n<160>(r2c, a, nz, st, tag); return;
        case 256: launch_pencil_n<256>(r2c, a, nz, st, tag); return;
    }
    throw ArgError("no pencil kernel for this length");
}

// ── drivers ──────────────────────────────────────────────────────────────────

namespace {

PlaneArgs plane_args(NSPlan& P) {
    PlaneArgs a{};
    a.tb = P.tbp;
    a.items = P.items.as<NSItem>();
    a.twr = get_fft(P.ffts, P.dims[1])->sh.tw;
    a.twc = get_fft(P.ffts, P.dims[2])->sh.tw;
    a.n2 = P.dims[1];
    a.n3 = P.dims[2];
    a.E = (long long)P.dims[1] * P.dims[2];
    a.H = P.H;
    a.status = P.status.dev;
    return a;
}

PencilArgs pencil_args(NSPlan& P) {
    PencilArgs a{};
    a.n1 = P.dims[0];
    a.nlines = P.dims[1] * P.dims[2];
    a.E = (long long)P.dims[1] * P.dims[2];
    a.tw = get_fft(P.ffts, P.dims[0])->sh.tw;
    a.cz = P.H;
    return a;
}

ZMap sub_map(NSPlan& P, int i0, int es) {
    ZMap zc;
    zc.items = P.items.as<NSItem>();
    zc.item0 = i0;
    zc.sub_stride = P.N * es;
    return zc;
}

// X = rfft3(x) in plane-major order
void rfft3_p(NSPlan& P, const float* x, int es, float2* X, cudaStream_t st) {
    PencilArgs pa = pencil_args(P);
    pa.rin = x;
    pa.cout = X;
    pa.es = es;
    launch_pencil(true, P.dims[0], pa, 1, st);
    PlaneArgs a = plane_args(P);
    a.in = X;
    a.out = X;
    launch_plane<kPlaneFwd>(P.dims[1], P.dims[2], a, P.h1, 1, st, "ns_plane_fwd");
}

}  // namespace

void ns_plane_analyze(NSPlan& P, const void* x, void* c, cudaStream_t st, bool synth_masks) {
    const int es = P.nch;
    float2* X = P.X.as<float2>();
    float2* W = P.work.as<float2>();
    for (int ch = 0; ch < P.nch; ++ch) {
        rfft3_p(P, reinterpret_cast<const float*>(x) + ch, es, X, st);
        for (int i0 = 0; i0 < P.S; i0 += P.group) {
            int nz = std::min(P.group, P.S - i0);
            PlaneArgs a = plane_args(P);
            a.in = X;
            a.out = W;
            a.out_z = P.H;
            a.item0 = i0;
            a.synth = synth_masks ? 1 : 0;
            launch_plane<kPlaneInvMask>(P.dims[1], P.dims[2], a, P.h1, nz, st, "ns_plane_inv_mask");
            PencilArgs pa = pencil_args(P);
            pa.cin = W;
            pa.rout = reinterpret_cast<float*>(c) + ch;
            pa.zm = sub_map(P, i0, es);
            pa.es = es;
            pa.scale = 1.0f / (float)P.N;
            launch_pencil(false, P.dims[0], pa, nz, st);
        }
    }
}

void ns_plane_synthesize(NSPlan& P, const void* c, void* x, cudaStream_t st, bool analysis_masks) {
    const int es = P.nch;
    float2* W = P.work.as<float2>();
    float2* A = P.acc.as<float2>();
    for (int ch = 0; ch < P.nch; ++ch) {
        int nparts = std::min(P.group, P.S);
        for (int i0 = 0; i0 < P.S; i0 += P.group) {
            int nz = std::min(P.group, P.S - i0);
            PencilArgs pa = pencil_args(P);
            pa.rin = reinterpret_cast<const float*>(c) + ch;
            pa.cout = W;
            pa.zm = sub_map(P, i0, es);
            pa.es = es;
            launch_pencil(true, P.dims[0], pa, nz, st);
            PlaneArgs a = plane_args(P);
            a.in = W;
            a.in_z = P.H;
            a.acc = A;
            a.init = i0 == 0 ? 1 : 0;
            a.item0 = i0;
            a.synth = analysis_masks ? 0 : 1;
            launch_plane<kPlaneFwdMaskAcc>(P.dims[1], P.dims[2], a, P.h1, nz, st, "ns_plane_fwd_acc");
        }
        // x = irfft3(sum of the partial accumulators)
        PlaneArgs a = plane_args(P);
        a.acc = A;
        a.npart = nparts;
        a.out = W;
        launch_plane<kPlaneInvSum>(P.dims[1], P.dims[2], a, P.h1, 1, st, "ns_plane_inv_sum");
        PencilArgs pa = pencil_args(P);
        pa.cin = W;
        pa.rout = reinterpret_cast<float*>(x) + ch;
        pa.es = es;
        pa.scale = 1.0f / (float)P.N;
        launch_pencil(false, P.dims[0], pa, 1, st);
    }
}

// ── streaming on the plane pipeline ──────────────────────────────────────────
// The same kernels and the same accumulator slots (item position mod group),
// so streaming agrees with the materialized transform bit for bit.

void ns_plane_stream_analyze_begin(NSPlan& P, const void* x, cudaStream_t st) {
    for (int ch = 0; ch < P.nch; ++ch) rfft3_p(P, reinterpret_cast<const float*>(x) + ch, P.nch, P.X.as<float2>() + ch * P.H, st);
}

void ns_plane_stream_analyze_one(NSPlan& P, int pos, void* band, cudaStream_t st) {
    float2* W = P.work.as<float2>();
    for (int ch = 0; ch < P.nch; ++ch) {
        PlaneArgs a = plane_args(P);
        a.in = P.X.as<float2>() + ch * P.H;
        a.out = W;
        a.out_z = P.H;
        a.item0 = pos;
        launch_plane<kPlaneInvMask>(P.dims[1], P.dims[2], a, P.h1, 1, st, "ns_plane_inv_mask");
        PencilArgs pa = pencil_args(P);
        pa.cin = W;
        pa.rout = reinterpret_cast<float*>(band) + ch;
        pa.es = P.nch;
        pa.scale = 1.0f / (float)P.N;
        launch_pencil(false, P.dims[0], pa, 1, st);
    }
}

// Accumulator of channel ch, slot q: channels keep separate sets of slots.
static float2* acc_slot(NSPlan& P, int ch) { return P.acc.as<float2>() + (long long)ch * P.group * P.H; }

void ns_plane_stream_synth_push(NSPlan& P, int pos, const void* band, cudaStream_t st) {
    float2* W = P.work.as<float2>();
    for (int ch = 0; ch < P.nch; ++ch) {
        PencilArgs pa = pencil_args(P);
        pa.rin = reinterpret_cast<const float*>(band) + ch;
        pa.cout = W;
        pa.es = P.nch;
        launch_pencil(true, P.dims[0], pa, 1, st);
        PlaneArgs a = plane_args(P);
        a.in = W;
        a.in_z = P.H;
        a.acc = acc_slot(P, ch) + (long long)(pos % P.group) * P.H;
        a.init = pos < P.group ? 1 : 0;
        a.item0 = pos;
        launch_plane<kPlaneFwdMaskAcc>(P.dims[1], P.dims[2], a, P.h1, 1, st, "ns_plane_fwd_acc");
    }
}

void ns_plane_stream_synth_end(NSPlan& P, void* x, cudaStream_t st) {
    float2* W = P.work.as<float2>();
    for (int ch = 0; ch < P.nch; ++ch) {
        PlaneArgs a = plane_args(P);
        a.acc = acc_slot(P, ch);
        a.npart = std::min(P.group, P.S);
        a.out = W;
        launch_plane<kPlaneInvSum>(P.dims[1], P.dims[2], a, P.h1, 1, st, "ns_plane_inv_sum");
        PencilArgs pa = pencil_args(P);
        pa.cin = W;
        pa.rout = reinterpret_cast<float*>(x) + ch;
        pa.es = P.nch;
        pa.scale = 1.0f / (float)P.N;
        launch_pencil(false, P.dims[0], pa, 1, st);
    }
}

}  // namespace sfl
