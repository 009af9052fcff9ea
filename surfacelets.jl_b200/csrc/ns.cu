// NSSurfacelet on the device: the cascade of src/transforms/ns_surfacelet.jl
// as line passes over the rfft grid (h1, n2, n3).
//
//   analysis, per subband s:   c_s = irfft(X * M_s)
//     pass 3 (axis 3, inverse) loads X and multiplies by M_s on the fly,
//     pass 2 (axis 2, inverse), pass 1 (axis 1, C2R of two lines at once,
//     scaled by 1/N) writes c_s straight into the coefficient array.
//   synthesis:                 x = irfft(sum_s rfft(c_s) * M_s)
//     pass 1 (R2C of two lines at once), pass 2, then pass 3 runs the FFT of
//     every subband of a group in one CTA and accumulates M_s * F_s in
//     registers with Kahan compensation; one accumulator round trip per group.
//
// M_s = (B_j hg_i) * w_a * w_b is evaluated per element from float32 tables
// designed in float64: the group factor B_j hg_i on the rfft grid (one table
// per scale and hourglass) and the wedge planes; M_s itself is never
// materialized.
#include <cmath>
#include <cstring>

#include "ns_mask.cuh"
#include "passes.cuh"
#include "plan.h"
#include "regpass.cuh"
#include "tma.cuh"

namespace sfl {

constexpr int kAccMax = 16;   // accumulator registers per thread (tile elements / 256)

// Pass 3 of the synthesis: for every item of the group, load its lines along
// axis 3 from work + z*H, FFT, multiply by its mask and accumulate, with Kahan
// compensation, into registers; then one round trip of acc/comp.
__global__ void __launch_bounds__(256) ns_accum_kernel(const float2* __restrict__ work, long long H, int G,
                                                       NSMaskTables tb, const NSItem* __restrict__ items,
                                                       int item0, int synth, float2* acc, float2* comp, int init,
                                                       FFTShape sh, int T, int npad) {
    extern __shared__ float2 smem[];
    float2* tw = smem;
    float2* a = smem + sh.n + (sh.n & 1);
    float2* b = a + T * npad;
    load_twiddles(tw, sh);
    const int n = sh.n;
    const int nlines = tb.h1 * tb.n2;
    const long long si = (long long)tb.h1 * tb.n2;
    const int l0 = blockIdx.x * T;
    const int total = T * n;
    float2 s[kAccMax], c[kAccMax];
#pragma unroll
    for (int e = 0; e < kAccMax; ++e) {
        s[e] = make_float2(0.f, 0.f);
        c[e] = make_float2(0.f, 0.f);
    }
    if (!init) {
#pragma unroll
        for (int e = 0; e < kAccMax; ++e) {
            int idx = threadIdx.x + e * blockDim.x;
            if (idx < total) {
                int t = idx % T, i = idx / T, l = l0 + t;
                if (l < nlines) {
                    s[e] = acc[l + (long long)i * si];
                    c[e] = comp[l + (long long)i * si];
                }
            }
        }
    }
    for (int z = 0; z < G; ++z) {
        const float2* src = work + (long long)z * H;
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            int t = idx % T, i = idx / T, l = l0 + t;
            a[t * npad + i] = l < nlines ? src[l + (long long)i * si] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        float2* r = fft_tile(a, b, T, sh, npad, tw, false);
        const NSItem it = items[item0 + z];
#pragma unroll
        for (int e = 0; e < kAccMax; ++e) {
            int idx = threadIdx.x + e * blockDim.x;
            if (idx < total) {
                int t = idx % T, i = idx / T, l = l0 + t;
                if (l < nlines) {
                    int k1 = l % tb.h1, k2 = l / tb.h1;
                    float m = ns_mask(tb, it, k1, k2, i, l + (long long)i * si, synth != 0);
                    float2 v = c_scale(r[t * npad + i], m);
                    // Kahan: y = v - c ; t = s + y ; c = (t - s) - y ; s = t
                    float2 y = c_sub(v, c[e]);
                    float2 tt = c_add(s[e], y);
                    c[e] = c_sub(c_sub(tt, s[e]), y);
                    s[e] = tt;
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int e = 0; e < kAccMax; ++e) {
        int idx = threadIdx.x + e * blockDim.x;
        if (idx < total) {
            int t = idx % T, i = idx / T, l = l0 + t;
            if (l < nlines) {
                acc[l + (long long)i * si] = s[e];
                comp[l + (long long)i * si] = c[e];
            }
        }
    }
}

// Synthesis pass 3 on the register FFT: every item of the group is
// transformed along axis 3 and accumulated (Kahan) in registers.
template <int N>
__global__ void __launch_bounds__(256) ns_accum_reg_kernel(const float2* __restrict__ work, long long H, int G,
                                                           NSMaskTables tb, const NSItem* __restrict__ items,
                                                           int item0, int synth, float2* acc, float2* comp, int init,
                                                           const float2* __restrict__ tw, int nlines) {
    using Ge = RegGeom<N>;
    constexpr int N1 = Ge::N1, N2 = Ge::N2, LP = Ge::LP, E = Ge::M * Ge::N2;
    extern __shared__ float2 xch[];
    const int tid = threadIdx.x;
    const int lp = tid % LP, p = tid / LP;
    const int l = blockIdx.x * LP + lp;
    const bool valid = l < nlines;
    const long long si = (long long)tb.h1 * tb.n2;
    float2* xl = xch + lp * Ge::XLINE;
    float2 s[E], c[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        s[e] = make_float2(0.f, 0.f);
        c[e] = make_float2(0.f, 0.f);
    }
    if (!init && valid) {
#pragma unroll
        for (int j = 0; j < Ge::M; ++j)
#pragma unroll
            for (int k = 0; k < N2; ++k) {
                long long q = l + (long long)((p + N2 * j) + N1 * k) * si;
                s[j * N2 + k] = acc[q];
                c[j * N2 + k] = comp[q];
            }
    }
    for (int z = 0; z < G; ++z) {
        RLoadC ld{work + (long long)z * H, ZMap{}, Lines{}};
        ld.g.si = si;
        RLoadC::Ctx lc{ld.src + (valid ? l : 0)};
        float2 u[E];
        reg_line_fft<N, false>(ld, lc, valid, p, xl, tw, u);
        const NSMaskLine mk = ns_mask_line(tb, items[item0 + z], valid ? l : 0, synth != 0);
#pragma unroll
        for (int j = 0; j < Ge::M; ++j)
#pragma unroll
            for (int k = 0; k < N2; ++k) {
                const int k3 = (p + N2 * j) + N1 * k;
                float2 v = c_scale(u[j * N2 + k], ns_mask_at(mk, k3, si));
                const int e = j * N2 + k;
                float2 y = c_sub(v, c[e]);
                float2 t = c_add(s[e], y);
                c[e] = c_sub(c_sub(t, s[e]), y);
                s[e] = t;
            }
        __syncthreads();   // the exchange rows are reused by the next item
    }
    if (valid) {
#pragma unroll
        for (int j = 0; j < Ge::M; ++j)
#pragma unroll
            for (int k = 0; k < N2; ++k) {
                long long q = l + (long long)((p + N2 * j) + N1 * k) * si;
                acc[q] = s[j * N2 + k];
                comp[q] = c[j * N2 + k];
            }
    }
}

template <int N>
static void launch_accum_reg(const float2* W, long long H, int nz, const NSMaskTables& tb, const NSItem* items,
                             int i0, int synth, float2* acc, float2* comp, int init, const float2* tw, int nlines,
                             cudaStream_t st) {
    using Ge = RegGeom<N>;
    static bool configured = false;
    if (!configured) {
        cuda_check(cudaFuncSetAttribute(ns_accum_reg_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)Ge::SMEM),
                   "cudaFuncSetAttribute");
        configured = true;
    }
    dim3 grid((nlines + Ge::LP - 1) / Ge::LP);
    int tok = prof_begin("ns_accum_axis3", st);
    ns_accum_reg_kernel<N><<<grid, Ge::THREADS, Ge::SMEM, st>>>(W, H, nz, tb, items, i0, synth, acc, comp, init, tw,
                                                                nlines);
    prof_end(tok, st);
    cuda_check(cudaGetLastError(), "ns_accum_reg_kernel launch");
}

// ── set-up ───────────────────────────────────────────────────────────────────

static std::vector<int> factorize(int n) {
    std::vector<int> f;
    for (int r : {8, 4, 2, 3, 5}) {
        while (n % r == 0) {
            f.push_back(r);
            n /= r;
        }
    }
    for (int p = 7; n > 1; p += 2) {
        while (n % p == 0) {
            f.push_back(p);
            n /= p;
        }
    }
    return f;
}

FFTLen* get_fft(std::map<int, std::unique_ptr<FFTLen>>& cache, int n) {
    auto it = cache.find(n);
    if (it != cache.end()) return it->second.get();
    std::unique_ptr<FFTLen> f(new FFTLen);
    std::vector<int> r = factorize(n);
    if ((int)r.size() > kMaxStages) throw ArgError("FFT length has too many factors");
    f->sh.n = n;
    f->sh.nstages = (int)r.size();
    for (size_t i = 0; i < r.size(); ++i) f->sh.radix[i] = r[i];
    std::vector<float2> tw(n);
    for (int t = 0; t < n; ++t) {
        // e^{-2 pi i t/n} designed in float64
        long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)t / (long double)n;
        tw[t] = make_float2((float)std::cos((double)a), (float)std::sin((double)a));
    }
    f->tw.alloc(sizeof(float2) * n);
    cuda_check(cudaMemcpy(f->tw.p, tw.data(), sizeof(float2) * n, cudaMemcpyHostToDevice), "twiddle upload");
    f->sh.tw = f->tw.as<float2>();
    FFTLen* raw = f.get();
    cache[n] = std::move(f);
    return raw;
}

template <class T>
static void upload(DevMem& m, const std::vector<T>& v) {
    m.alloc(sizeof(T) * (v.empty() ? 1 : v.size()));
    if (!v.empty()) cuda_check(cudaMemcpy(m.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
}

static std::vector<float> to_f32(const std::vector<double>& v) {
    std::vector<float> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) o[i] = (float)v[i];
    return o;
}

// With ndfb, the standalone directional bank of one level count
// (src/directional/ndfb.jl:91-104; HourglassFB at level 0): the same cascade
// with the hourglass masks alone as group factors, no pyramid and no lowpass.
void ns_plan_init(NSPlan& P, const sfl_ns_params& p, const int dims[3], int dtype, bool ndfb) {
    for (int d = 0; d < 3; ++d)
        if (dims[d] > 8192) throw ArgError("axis lengths above 8192 are not supported by this library");
    P.ndfb = ndfb;
    P.design = ns_design(p, dims, !ndfb, false);
    const NSDesign& D = P.design;
    P.p = p;
    for (int d = 0; d < 3; ++d) P.dims[d] = dims[d];
    P.h1 = dims[0] / 2 + 1;
    P.N = (long long)dims[0] * dims[1] * dims[2];
    P.H = (long long)P.h1 * dims[1] * dims[2];
    P.S = ndfb ? 3 * (1 << p.direction_levels[0]) : ns_nsubbands(p);
    P.nch = dtype == SFL_COMPLEX64 ? 2 : 1;
    const int J = p.scales;

    // tables: group masks (and level bandpasses when not tight), designed in
    // float64 on the device, with the support box of each
    NSMaskTables& tb = P.tb;
    ns_design_tables_device(P);
    if (ndfb) {
        P.boxes.push_back(ns_make_box(P.h1, dims[1], dims[1]));   // no lowpass; keeps the table indexing uniform
        P.boxes_full = ns_make_box(P.h1, dims[1], dims[1]);
    } else {
        // lowpass box from its per-axis factors
        int m1 = -1, m2 = -1;
        const auto& a1 = D.pa[J][0];
        const auto& a2 = D.pa[J][1];
        for (int k = 0; k < (int)a1.size(); ++k)
            if (a1[k] != 0.0) m1 = std::max(m1, k);
        for (int k = 0; k < (int)a2.size(); ++k)
            if (a2[k] != 0.0) m2 = std::max(m2, std::min(k, dims[1] - k));
        P.boxes.push_back(ns_make_box(m1 + 1, m2, dims[1]));
        P.boxes_full = ns_make_box(P.h1, dims[1], dims[1]);
    }
    std::vector<float> vec;
    for (int d = 0; d < 3; ++d) {
        tb.low_off[d] = (int)vec.size();
        if (ndfb)
            vec.resize(vec.size() + (d == 0 ? P.h1 : dims[d]), 1.0f);
        else
            for (double x : D.pa[J][d]) vec.push_back((float)x);
    }
    upload(P.vec, vec);
    std::vector<float> planes;
    // plane_off[j][i][plane][w]
    std::vector<std::array<std::array<std::vector<int>, 2>, 3>> off(J);
    for (int j = 0; j < J; ++j)
        for (int i = 0; i < 3; ++i)
            for (int q = 0; q < 2; ++q) {
                const WedgePlanes& W = D.wedges[j][i][q];
                for (const auto& w : W.w) {
                    off[j][i][q].push_back((int)planes.size());
                    for (double x : w) planes.push_back((float)x);
                }
            }
    upload(P.planes, planes);
    tb.G = P.G.as<float>();
    tb.Bl = P.Bl.as<float>();
    tb.H = P.H;
    tb.vec = P.vec.as<float>();
    tb.planes = P.planes.as<float>();
    tb.h1 = P.h1;
    tb.n2 = dims[1];
    tb.n3 = dims[2];
    tb.tight = p.tight ? 1 : 0;

    // items in streaming order: directional subbands ascending, then the lowpass.
    // Subband index: src/transforms/ns_surfacelet.jl:222-242, 430
    std::vector<NSItem> items;
    int offset = ndfb ? 0 : 1;   // the bank's subband index: ((i-1) na + (p-1)) nb + q, src/directional/ndfb.jl:184-190
    for (int j = 1; j <= J; ++j) {
        int L = p.direction_levels[j - 1];
        int na = 1 << ((L + 1) / 2), nb = 1 << (L / 2);
        for (int i = 1; i <= 3; ++i)
            for (int a = 1; a <= na; ++a)
                for (int b = 1; b <= nb; ++b) {
                    NSItem it{};
                    it.s = offset + ((i - 1) * na + (a - 1)) * nb + b;
                    it.kind = 0;
                    it.lv = J - j;
                    it.i = i;
                    it.g = 3 * (j - 1) + (i - 1);
                    const WedgePlanes& Wa = D.wedges[j - 1][i - 1][0];
                    const WedgePlanes& Wb = D.wedges[j - 1][i - 1][1];
                    it.wa_off = off[j - 1][i - 1][0][a - 1];
                    it.wb_off = off[j - 1][i - 1][1][b - 1];
                    it.wa_lo = Wa.lo - 1;
                    it.wa_hi = Wa.hi - 1;
                    it.wa_dlo = Wa.dlo;
                    it.wb_lo = Wb.lo - 1;
                    it.wb_hi = Wb.hi - 1;
                    it.wb_dlo = Wb.dlo;
                    items.push_back(it);
                }
        offset += 3 * na * nb;
    }
    if (!ndfb) {
        NSItem low{};
        low.s = 1;
        low.kind = 1;
        low.lv = J;
        low.i = 1;
        items.push_back(low);
    }
    P.items_host = items;
    upload(P.items, items);

    get_fft(P.ffts, dims[0]);
    get_fft(P.ffts, dims[1]);
    get_fft(P.ffts, dims[2]);

    P.status.alloc();
    P.group = std::min(8, P.S);
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&P.sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    P.P1 = P.h1;
    while (P.P1 % 4 != 2) ++P.P1;
    P.SP = (long long)P.P1 * dims[1] * dims[2];
    P.slab = ns_slab_supported(dims[0], dims[1], dims[2]);
    ns_alloc_scratch(P);
}

// Spectrum-sized scratch for the selected pipeline and group size.
void ns_alloc_scratch(NSPlan& P) {
    const long long spec = P.slab ? P.SP : P.H;
    P.X.alloc(sizeof(float2) * spec * P.nch);
    P.work.alloc(sizeof(float2) * spec * P.group * (P.slab ? P.nch : 1));
    if (P.slab) {
        P.acc.alloc(sizeof(float2) * spec * P.nch);
        P.comp.alloc(sizeof(float2) * spec * P.nch);
    } else {
        P.acc.alloc(sizeof(float2) * P.H * std::max(P.nch, P.group * P.nch));
        P.comp.alloc(sizeof(float2) * P.H * P.nch);
    }
}

// ── passes ───────────────────────────────────────────────────────────────────

namespace {

// rfft grid of the plan
struct Grid {
    int d[3];
};

Grid half_grid(const NSPlan& P) { return Grid{{P.h1, P.dims[1], P.dims[2]}}; }

// R2C along axis 1 of nz real volumes (element stride es) into nz spectra.
void pass_r2c(NSPlan& P, const float* src, ZMap zin, int es, float2* dst, long long dst_zstride, int nz,
              cudaStream_t st) {
    FFTLen* f = get_fft(P.ffts, P.dims[0]);
    Lines gin = axis_lines(P.dims, 0);
    Grid hg = half_grid(P);
    Lines gout = axis_lines(hg.d, 0);
    ZMap zo;
    zo.zstride = dst_zstride;
    int pairs = (gin.nlines + 1) / 2;
    if (launch_reg<false>(f->sh.n, RLoadRPair{src, zin, gin, es}, RStoreHalfPair{dst, zo, gout, f->sh.n}, f->sh.tw,
                          pairs, nz, false, st, "ns_r2c_axis1"))
        return;
    LoadRPair ld{src, zin, gin, es};
    StoreHalfPair sto{dst, zo, gout};
    launch_pass(ld, sto, f->sh, pairs, nz, false, st, "ns_r2c_axis1");
}

// C2R along axis 1 of nz spectra into nz real volumes, scaled.
void pass_c2r(NSPlan& P, const float2* src, long long src_zstride, float* dst, ZMap zout, int es, float scale,
              int nz, cudaStream_t st) {
    FFTLen* f = get_fft(P.ffts, P.dims[0]);
    Grid hg = half_grid(P);
    Lines gin = axis_lines(hg.d, 0);
    Lines gout = axis_lines(P.dims, 0);
    ZMap zi;
    zi.zstride = src_zstride;
    int pairs = (gout.nlines + 1) / 2;
    if (launch_reg<true>(f->sh.n, RLoadHPair{src, zi, gin, f->sh.n}, RStoreRPair{dst, zout, gout, es, scale},
                         f->sh.tw, pairs, nz, false, st, "ns_c2r_axis1"))
        return;
    LoadHPair ld{src, zi, gin};
    StoreRPair sto{dst, zout, gout, es, scale};
    launch_pass(ld, sto, f->sh, pairs, nz, true, st, "ns_c2r_axis1");
}

// Complex FFT along axis a (1 or 2, 0-based) of nz spectra.
void pass_c2c(NSPlan& P, const float2* src, float2* dst, long long zstride, int axis, bool inv, int nz,
              cudaStream_t st) {
    Grid hg = half_grid(P);
    FFTLen* f = get_fft(P.ffts, hg.d[axis]);
    Lines g = axis_lines(hg.d, axis);
    ZMap zm;
    zm.zstride = zstride;
    const char* tag = axis == 1 ? "ns_c2c_axis2" : "ns_c2c_axis3";
    bool tf = g.si != 1;
    bool done = inv ? launch_reg<true>(f->sh.n, RLoadC{src, zm, g}, RStoreC{dst, zm, g}, f->sh.tw, g.nlines, nz, tf,
                                       st, tag)
                    : launch_reg<false>(f->sh.n, RLoadC{src, zm, g}, RStoreC{dst, zm, g}, f->sh.tw, g.nlines, nz,
                                        tf, st, tag);
    if (done) return;
    LoadC ld{src, zm, g, 1.f};
    StoreC sto{dst, zm, g, 1.f};
    launch_pass(ld, sto, f->sh, g.nlines, nz, inv, st, tag);
}

void rfft3(NSPlan& P, const float* x, int es, float2* X, cudaStream_t st) {
    pass_r2c(P, x, ZMap{}, es, X, 0, 1, st);
    pass_c2c(P, X, X, 0, 1, false, 1, st);
    pass_c2c(P, X, X, 0, 2, false, 1, st);
}

void irfft3(NSPlan& P, const float2* A, float* x, int es, cudaStream_t st) {
    float2* W = P.work.as<float2>();
    pass_c2c(P, A, W, 0, 2, true, 1, st);
    pass_c2c(P, W, W, 0, 1, true, 1, st);
    pass_c2r(P, W, 0, x, ZMap{}, es, 1.0f / (float)P.N, 1, st);
}

// Analysis of items [i0, i0 + nz) from spectrum X into the coefficients
// (item z written at cbase + zc.off(z), element stride es).
void analyze_items(NSPlan& P, const float2* X, float* cbase, ZMap zc, int es, int i0, int nz, bool synth_masks,
                   cudaStream_t st) {
    float2* W = P.work.as<float2>();
    Grid hg = half_grid(P);
    FFTLen* f3 = get_fft(P.ffts, P.dims[2]);
    Lines g3 = axis_lines(hg.d, 2);
    ZMap zw;
    zw.zstride = P.H;
    if (!launch_reg<true>(f3->sh.n, RLoadNSMask{X, P.tb, P.items.as<NSItem>(), i0, synth_masks ? 1 : 0},
                          RStoreC{W, zw, g3}, f3->sh.tw, g3.nlines, nz, true, st, "ns_mask_axis3")) {
        LoadNSMask ld{X, P.tb, P.items.as<NSItem>(), i0, synth_masks ? 1 : 0};
        StoreC sto{W, zw, g3, 1.f};
        launch_pass(ld, sto, f3->sh, g3.nlines, nz, true, st, "ns_mask_axis3");
    }
    pass_c2c(P, W, W, P.H, 1, true, nz, st);
    pass_c2r(P, W, P.H, cbase, zc, es, 1.0f / (float)P.N, nz, st);
}

// The forward axis-1 and axis-2 passes of nz subband volumes into work slots
// slot0.. (one channel).
void stage_items(NSPlan& P, const float* cbase, ZMap zc, int es, int nz, int slot0, cudaStream_t st) {
    float2* W = P.work.as<float2>() + (long long)slot0 * P.H;
    pass_r2c(P, cbase, zc, es, W, P.H, nz, st);
    pass_c2c(P, W, W, P.H, 1, false, nz, st);
}

// The axis-3 pass of work slots 0..nz-1 times the masks of items i0.., summed
// into acc (Kahan-compensated through comp).
void accum_items(NSPlan& P, int i0, int nz, bool analysis_masks, float2* acc, float2* comp, bool init,
                 cudaStream_t st) {
    float2* W = P.work.as<float2>();
    FFTLen* f3 = get_fft(P.ffts, P.dims[2]);
    int n = f3->sh.n;
    {
        int nl = P.h1 * P.dims[1];
        const NSItem* it = P.items.as<NSItem>();
        int sy = analysis_masks ? 0 : 1;
        switch (n) {
            case 16: launch_accum_reg<16>(W, P.H, nz, P.tb, it, i0, sy, acc, comp, init, f3->sh.tw, nl, st); return;
            case 32: launch_accum_reg<32>(W, P.H, nz, P.tb, it, i0, sy, acc, comp, init, f3->sh.tw, nl, st); return;
            case 64: launch_accum_reg<64>(W, P.H, nz, P.tb, it, i0, sy, acc, comp, init, f3->sh.tw, nl, st); return;
            case 96: launch_accum_reg<96>(W, P.H, nz, P.tb, it, i0, sy, acc, comp, init, f3->sh.tw, nl, st); return;
            case 128: launch_accum_reg<128>(W, P.H, nz, P.tb, it, i0, sy, acc, comp, init, f3->sh.tw, nl, st); return;
            case 160: launch_accum_reg<160>(W, P.H, nz, P.tb, it, i0, sy, acc, comp, init, f3->sh.tw, nl, st); return;
            case 256: launch_accum_reg<256>(W, P.H, nz, P.tb, it, i0, sy, acc, comp, init, f3->sh.tw, nl, st); return;
        }
    }
    int T = pass_tile(n);
    while (T > 1 && T * n > kAccMax * 256) --T;
    if (T * n > kAccMax * 256) throw ArgError("axis 3 is too long for the accumulating pass of this library");
    int npad = n + 1;
    size_t smem = pass_smem_bytes(n, T);
    static bool configured = false;
    if (!configured) {
        cuda_check(cudaFuncSetAttribute(ns_accum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024),
                   "cudaFuncSetAttribute");
        configured = true;
    }
    int nlines = P.h1 * P.dims[1];
    dim3 grid((nlines + T - 1) / T);
    int tok = prof_begin("ns_accum_axis3", st);
    ns_accum_kernel<<<grid, 256, smem, st>>>(W, P.H, nz, P.tb, P.items.as<NSItem>(), i0,
                                             analysis_masks ? 0 : 1, acc, comp, init ? 1 : 0,
                                             f3->sh, T, npad);
    prof_end(tok, st);
    cuda_check(cudaGetLastError(), "ns_accum_kernel launch");
}

void synth_items(NSPlan& P, const float* cbase, ZMap zc, int es, int i0, int nz, bool analysis_masks, float2* acc,
                 float2* comp, bool init, cudaStream_t st) {
    stage_items(P, cbase, zc, es, nz, 0, st);
    accum_items(P, i0, nz, analysis_masks, acc, comp, init, st);
}

// The denoiser's axis-1 step on the line pipeline, one kernel per pair of
// lines: C2R of the two half-spectrum lines (scaled by 1/N), the soft
// threshold of subband z's tau on both real lines, and their R2C, in place in
// the work slots.  The same arithmetic as pass_c2r, soft_threshold_kernel and
// pass_r2c one after the other, so the result is theirs bit for bit.
template <int N>
__global__ void __launch_bounds__(256) reg_shrink_axis1_kernel(RLoadHPair ld, RStoreHalfPair sto,
                                                               const float2* __restrict__ tw, int nlines,
                                                               float scale, const float* __restrict__ tau,
                                                               const NSItem* __restrict__ items, int item0) {
    using G = RegGeom<N>;
    constexpr int N1 = G::N1, N2 = G::N2, LP = G::LP;
    extern __shared__ float2 xch[];
    const int tid = threadIdx.x;
    const int p = tid % N2, lp = tid / N2;
    const int l = blockIdx.x * LP + lp;
    const int z = blockIdx.y;
    const bool valid = l < nlines;
    float2* xl = xch + lp * G::XLINE;
    const float t = tau[items[item0 + z].s - 1];
    const RLoadHPair::Ctx lc = ld.line(z, l, valid);
    float2 u[G::M * N2];
    reg_line_fft<N, true>(ld, lc, valid, p, xl, tw, u);
    const bool hasb = lc.b != nullptr;
#pragma unroll
    for (int q = 0; q < G::M * N2; ++q) {
        const float a = __fmul_rn(u[q].x, scale);
        const float b = hasb ? __fmul_rn(u[q].y, scale) : 0.f;
        u[q] = make_float2(copysignf(fmaxf(fabsf(a) - t, 0.f), a), hasb ? copysignf(fmaxf(fabsf(b) - t, 0.f), b) : 0.f);
    }
    // back to natural order: thread p takes x[p + N2 r]
    __syncthreads();
#pragma unroll
    for (int j = 0; j < G::M; ++j)
#pragma unroll
        for (int k = 0; k < N2; ++k) xl[(p + N2 * j) + N1 * k] = u[j * N2 + k];
    __syncthreads();
    float2 v[N1];
#pragma unroll
    for (int r = 0; r < N1; ++r) v[r] = xl[p + N2 * r];
    __syncthreads();
    reg_line_fft_v<N, false>(v, p, xl, tw, u);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < G::M; ++j)
#pragma unroll
        for (int k = 0; k < N2; ++k) xl[(p + N2 * j) + N1 * k] = u[j * N2 + k];
    __syncthreads();
    if (valid) sto.staged(sto.line(z, l, valid), xl, p, N2);
}

template <int N>
void launch_shrink_axis1(const RLoadHPair& ld, const RStoreHalfPair& sto, const float2* tw, int nlines, int nz,
                         float scale, const float* tau, const NSItem* items, int item0, cudaStream_t st) {
    using G = RegGeom<N>;
    static bool configured = false;
    if (!configured) {
        cuda_check(cudaFuncSetAttribute(reg_shrink_axis1_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)G::SMEM),
                   "cudaFuncSetAttribute");
        configured = true;
    }
    dim3 grid((nlines + G::LP - 1) / G::LP, nz);
    int tok = prof_begin("ns_shrink_axis1", st);
    reg_shrink_axis1_kernel<N><<<grid, G::THREADS, G::SMEM, st>>>(ld, sto, tw, nlines, scale, tau, items, item0);
    prof_end(tok, st);
    cuda_check(cudaGetLastError(), "reg_shrink_axis1_kernel launch");
}

}  // namespace

// ── item ranges: the building blocks of the slab and line pipelines ─────────

long long ns_spec_elems(const NSPlan& P) { return P.slab ? P.SP : P.H; }

void ns_forward_spectrum(NSPlan& P, const float* x, int es, float2* X, cudaStream_t st) {
    if (P.slab)
        ns_slab_rfft3(P, x, es, X, st);
    else
        rfft3(P, x, es, X, st);
}

int ns_next_chunk(const NSPlan& P, int i0) {
    return P.slab ? ns_slab_chunk_end(P, i0) : std::min(P.S, i0 + P.group);
}

void ns_analyze_range(NSPlan& P, const float2* X, float* vol, ZMap vz, int es, int i0, int nz, bool synth_masks,
                      cudaStream_t st) {
    if (P.slab)
        ns_slab_analyze_items(P, X, vol, vz, es, i0, nz, synth_masks, st);
    else
        analyze_items(P, X, vol, vz, es, i0, nz, synth_masks, st);
}

void ns_acc_clear(NSPlan& P, float2* acc, float2* comp, cudaStream_t st) {
    cuda_check(cudaMemsetAsync(acc, 0, sizeof(float2) * ns_spec_elems(P), st), "cudaMemsetAsync(acc)");
    cuda_check(cudaMemsetAsync(comp, 0, sizeof(float2) * ns_spec_elems(P), st), "cudaMemsetAsync(comp)");
}

float2* ns_comp_grid(NSPlan& P, int ch) { return P.comp.as<float2>() + ch * ns_spec_elems(P); }

void ns_accumulate_range(NSPlan& P, const float* vol, ZMap vz, int es, int i0, int nz, bool analysis_masks,
                         float2* acc, float2* comp, cudaStream_t st) {
    if (P.slab)
        ns_slab_synth_items(P, vol, vz, es, i0, nz, analysis_masks, acc, comp, st);
    else
        synth_items(P, vol, vz, es, i0, nz, analysis_masks, acc, comp, false, st);
}

void ns_stage_range(NSPlan& P, const float* vol, ZMap vz, int es, int i0, int nz, int slot0, int nch,
                    cudaStream_t st) {
    if (slot0 < 0 || slot0 + nz > P.group) throw ArgError("work slots out of range");
    if (P.slab) {
        ns_slab_stage_items(P, vol, vz, es, i0, nz, slot0, nch, st);
    } else {
        if (nch != 1) throw ArgError("the line pipeline stages one channel at a time");
        stage_items(P, vol, vz, es, nz, slot0, st);
    }
}

void ns_accum_staged(NSPlan& P, int i0, int nz, bool analysis_masks, float2* acc, float2* comp, int nch,
                     cudaStream_t st) {
    if (P.slab) {
        ns_slab_accum_items(P, i0, nz, analysis_masks, acc, comp, nch, st);
    } else {
        if (nch != 1) throw ArgError("the line pipeline stages one channel at a time");
        accum_items(P, i0, nz, analysis_masks, acc, comp, false, st);
    }
}

bool ns_line_shrink_supported(const NSPlan& P) {
    switch (P.dims[0]) {
        case 16: case 32: case 64: case 96: case 128: case 160: case 256:
            return true;
    }
    return false;
}

void ns_line_denoise_items(NSPlan& P, const float2* X, int i0, int nz, const float* tau, float2* acc, float2* comp,
                           cudaStream_t st) {
    float2* W = P.work.as<float2>();
    Grid hg = half_grid(P);
    FFTLen* f3 = get_fft(P.ffts, P.dims[2]);
    Lines g3 = axis_lines(hg.d, 2);
    ZMap zw;
    zw.zstride = P.H;
    if (!launch_reg<true>(f3->sh.n, RLoadNSMask{X, P.tb, P.items.as<NSItem>(), i0, 0}, RStoreC{W, zw, g3},
                          f3->sh.tw, g3.nlines, nz, true, st, "ns_mask_axis3")) {
        LoadNSMask ld{X, P.tb, P.items.as<NSItem>(), i0, 0};
        StoreC sto{W, zw, g3, 1.f};
        launch_pass(ld, sto, f3->sh, g3.nlines, nz, true, st, "ns_mask_axis3");
    }
    pass_c2c(P, W, W, P.H, 1, true, nz, st);
    FFTLen* f1 = get_fft(P.ffts, P.dims[0]);
    const Lines gh = axis_lines(hg.d, 0);
    const int pairs = (axis_lines(P.dims, 0).nlines + 1) / 2;
    const RLoadHPair ld{W, zw, gh, f1->sh.n};
    const RStoreHalfPair sto{W, zw, gh, f1->sh.n};
    const float sc = 1.0f / (float)P.N;
    const NSItem* it = P.items.as<NSItem>();
    switch (P.dims[0]) {
        case 16: launch_shrink_axis1<16>(ld, sto, f1->sh.tw, pairs, nz, sc, tau, it, i0, st); break;
        case 32: launch_shrink_axis1<32>(ld, sto, f1->sh.tw, pairs, nz, sc, tau, it, i0, st); break;
        case 64: launch_shrink_axis1<64>(ld, sto, f1->sh.tw, pairs, nz, sc, tau, it, i0, st); break;
        case 96: launch_shrink_axis1<96>(ld, sto, f1->sh.tw, pairs, nz, sc, tau, it, i0, st); break;
        case 128: launch_shrink_axis1<128>(ld, sto, f1->sh.tw, pairs, nz, sc, tau, it, i0, st); break;
        case 160: launch_shrink_axis1<160>(ld, sto, f1->sh.tw, pairs, nz, sc, tau, it, i0, st); break;
        case 256: launch_shrink_axis1<256>(ld, sto, f1->sh.tw, pairs, nz, sc, tau, it, i0, st); break;
        default: throw ArgError("no register pass for axis 1 of this size");
    }
    pass_c2c(P, W, W, P.H, 1, false, nz, st);
    accum_items(P, i0, nz, false, acc, comp, false, st);
}

void ns_inverse_spectrum(NSPlan& P, float2* A, float* x, int es, cudaStream_t st) {
    if (P.slab)
        ns_slab_irfft3(P, A, x, es, st);
    else
        irfft3(P, A, x, es, st);
}

ZMap ns_subband_map(const NSPlan& P, int i0, int es) {
    ZMap zc;
    zc.items = P.items.as<NSItem>();
    zc.item0 = i0;
    zc.sub_stride = P.N * es;
    return zc;
}

void ns_analyze(NSPlan& P, const void* x, void* c, cudaStream_t st, bool synth_masks) {
    if (P.slab) return ns_slab_analyze(P, x, c, st, synth_masks);
    const int es = P.nch;
    float2* X = P.X.as<float2>();
    for (int ch = 0; ch < P.nch; ++ch) {
        ns_forward_spectrum(P, reinterpret_cast<const float*>(x) + ch, es, X, st);
        for (int i0 = 0, i1; i0 < P.S; i0 = i1) {
            i1 = ns_next_chunk(P, i0);
            ns_analyze_range(P, X, reinterpret_cast<float*>(c) + ch, ns_subband_map(P, i0, es), es, i0, i1 - i0,
                             synth_masks, st);
        }
    }
}

void ns_synthesize(NSPlan& P, const void* c, void* x, cudaStream_t st, bool analysis_masks) {
    if (P.slab) return ns_slab_synthesize(P, c, x, st, analysis_masks);
    const int es = P.nch;
    float2* A = P.acc.as<float2>();
    float2* K = P.comp.as<float2>();
    for (int ch = 0; ch < P.nch; ++ch) {
        ns_acc_clear(P, A, K, st);
        for (int i0 = 0, i1; i0 < P.S; i0 = i1) {
            i1 = ns_next_chunk(P, i0);
            ns_accumulate_range(P, reinterpret_cast<const float*>(c) + ch, ns_subband_map(P, i0, es), es, i0,
                                i1 - i0, analysis_masks, A, K, st);
        }
        ns_inverse_spectrum(P, A, reinterpret_cast<float*>(x) + ch, es, st);
    }
}

// ── bounded-wait self-test ──────────────────────────────────────────────────

// One CTA waits, with a short iteration limit, on an mbarrier that expects
// one arrival nobody makes (no copy is issued): the wait runs out and records
// its status through the same path as the bulk-copy waits.
__global__ void selftest_wait_kernel(int* status, long long limit) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
        mbar_wait_bounded(&bar, 0, status, limit);
    }
}

void ns_selftest_wait(NSPlan& P, cudaStream_t st) {
    selftest_wait_kernel<<<1, 32, 0, st>>>(P.status.dev, 4096);
    cuda_check(cudaGetLastError(), "selftest_wait_kernel launch");
}

// ── streaming ────────────────────────────────────────────────────────────────

void ns_stream_analyze_begin(NSPlan& P, const void* x, cudaStream_t st) {
    for (int ch = 0; ch < P.nch; ++ch)
        ns_forward_spectrum(P, reinterpret_cast<const float*>(x) + ch, P.nch, P.X.as<float2>() + ch * ns_spec_elems(P),
                            st);
    P.stream_mode = 1;
    P.stream_pos = 0;
}

int ns_stream_analyze_next(NSPlan& P, void* band, int* index, cudaStream_t st) {
    if (P.stream_mode != 1) throw StateError("no streaming analysis is open on this plan");
    if (P.stream_pos >= P.S) {
        P.stream_mode = 0;
        return SFL_DONE;
    }
    const NSItem& it = P.items_host[P.stream_pos];
    for (int ch = 0; ch < P.nch; ++ch)
        ns_analyze_range(P, P.X.as<float2>() + ch * ns_spec_elems(P), reinterpret_cast<float*>(band) + ch, ZMap{},
                         P.nch, P.stream_pos, 1, false, st);
    *index = it.s;
    P.stream_pos += 1;
    return SFL_OK;
}

void ns_stream_synth_begin(NSPlan& P, cudaStream_t) {
    P.stream_mode = 2;
    P.stream_pos = 0;
}

int ns_stream_synth_next_index(NSPlan& P, int* index) {
    if (P.stream_mode != 2) throw StateError("no streaming synthesis is open on this plan");
    if (P.stream_pos >= P.S) return SFL_DONE;
    *index = P.items_host[P.stream_pos].s;
    return SFL_OK;
}

void ns_stream_synth_push(NSPlan& P, const void* band, cudaStream_t st) {
    if (P.stream_mode != 2) throw StateError("no streaming synthesis is open on this plan");
    if (P.stream_pos >= P.S) throw StateError("every subband has already been pushed");
    {
        const long long E = ns_spec_elems(P);
        if (P.stream_pos == 0) {
            for (int ch = 0; ch < P.nch; ++ch) ns_acc_clear(P, P.acc.as<float2>() + ch * E, ns_comp_grid(P, ch), st);
            P.stream_chunk0 = 0;
        }
        if (P.slab || P.nch == 1) {
            // stage the subband in the work slot of its position in the mask
            // group; the axis-3 accumulation runs once per group
            const int c0 = P.stream_chunk0, c1 = ns_next_chunk(P, c0);
            ns_stage_range(P, reinterpret_cast<const float*>(band), ZMap{}, P.nch, P.stream_pos, 1,
                           P.stream_pos - c0, P.nch, st);
            if (P.stream_pos + 1 == c1) {
                ns_accum_staged(P, c0, c1 - c0, false, P.acc.as<float2>(), P.comp.as<float2>(), P.nch, st);
                P.stream_chunk0 = c1;
            }
        } else {
            // complex data on the line pipeline: the work slots hold one channel
            for (int ch = 0; ch < P.nch; ++ch)
                ns_accumulate_range(P, reinterpret_cast<const float*>(band) + ch, ZMap{}, P.nch, P.stream_pos, 1,
                                    false, P.acc.as<float2>() + ch * E, ns_comp_grid(P, ch), st);
        }
    }
    P.stream_pos += 1;
}

void ns_stream_synth_end(NSPlan& P, void* x, cudaStream_t st) {
    if (P.stream_mode != 2 || P.stream_pos != P.S)
        throw StateError("streaming synthesis ended before every subband was pushed");
    for (int ch = 0; ch < P.nch; ++ch)
        ns_inverse_spectrum(P, P.acc.as<float2>() + ch * ns_spec_elems(P), reinterpret_cast<float*>(x) + ch, P.nch, st);
    P.stream_mode = 0;
}

}  // namespace sfl
