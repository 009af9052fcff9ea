// NSSurfacelet mask evaluation and the mask-multiplying loads of the
// analysis' first inverse pass (lines along axis 3 of the rfft grid), shared
// by the NS drivers.
#pragma once

#include "passes.cuh"
#include "plan.h"
#include "regpass.cuh"

namespace sfl {

// Mask of item `it` at rfft-grid point (k1, k2, k3), linear index q.  synth
// selects the synthesis mask, which is B_j alone when the bank is not tight
// (src/transforms/ns_surfacelet.jl:226-227, 237-238).  The group factor
// B_j hg_i comes from a float64-designed table; the wedge planes are
// square-rooted in float64 too, so only well-conditioned float32 products
// remain here.
__device__ __forceinline__ float ns_mask(const NSMaskTables& tb, const NSItem& it, int k1, int k2, int k3,
                                         long long q, bool synth) {
    if (it.kind == 1) {
        // lowpass a1 a2 a3: src/transforms/ns_surfacelet.jl:358-371
        const float* v = tb.vec;
        return v[tb.low_off[0] + k1] * v[tb.low_off[1] + k2] * v[tb.low_off[2] + k3];
    }
    if (synth && !tb.tight) return tb.Bl[(long long)it.lv * tb.H + q];
    float G = tb.G[(long long)it.g * tb.H + q];
    // wedge planes: src/transforms/ns_surfacelet.jl:376-427
    int kk[3] = {k1, k2, k3};
    float wa = tb.planes[it.wa_off + kk[it.wa_lo] + it.wa_dlo * kk[it.wa_hi]];
    float wb = tb.planes[it.wb_off + kk[it.wb_lo] + it.wb_dlo * kk[it.wb_hi]];
    return (G * wa) * wb;
}

// Pass-3 load of the analysis: lines along axis 3 of X, times the mask of
// item z.  Line l = (k1, k2) with k1 fastest.
struct LoadNSMask {
    const float2* X;
    NSMaskTables tb;
    const NSItem* items;
    int item0;
    int synth;
    __device__ __forceinline__ void operator()(float2* tile, int npad, int n, int l0, int T, int z) const {
        const NSItem it = items[item0 + z];
        const int nlines = tb.h1 * tb.n2;
        const long long si = (long long)tb.h1 * tb.n2;
        const int total = T * n;
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            int t = idx % T;
            int i = idx / T;
            int l = l0 + t;
            float2 v = make_float2(0.f, 0.f);
            if (l < nlines) {
                int k1 = l % tb.h1, k2 = l / tb.h1;
                long long q = l + (long long)i * si;
                v = c_scale(X[q], ns_mask(tb, it, k1, k2, i, q, synth != 0));
            }
            tile[t * npad + i] = v;
        }
    }
};

// Per-line mask context of an NS item for lines along axis 3 (line l =
// (k1, k2), element k3): mask(k3) = m[k3 * si] * wa(k3) * wb(k3), each plane
// either constant along the line or stepping with k3.
struct NSMaskLine {
    const float* m;       // group table (or level bandpass) at the line's first point
    const float* wa;
    const float* wb;
    int was, wbs;         // steps of the planes along k3 (0: constant)
    int plain;            // 1: the mask is m alone (bandpass of an untight synthesis)
    int low;              // 1: lowpass a1 a2 a3
    float lowc;           // a1[k1] a2[k2]
    const float* lowv;    // a3
};

__device__ __forceinline__ NSMaskLine ns_mask_line(const NSMaskTables& tb, const NSItem& it, int l, bool synth) {
    NSMaskLine c;
    const int k1 = l % tb.h1, k2 = l / tb.h1;
    c.low = it.kind == 1;
    c.plain = 0;
    c.m = nullptr;
    c.wa = c.wb = nullptr;
    c.was = c.wbs = 0;
    c.lowc = 0.f;
    c.lowv = nullptr;
    if (c.low) {
        c.lowc = tb.vec[tb.low_off[0] + k1] * tb.vec[tb.low_off[1] + k2];
        c.lowv = tb.vec + tb.low_off[2];
        return c;
    }
    if (synth && !tb.tight) {
        c.plain = 1;
        c.m = tb.Bl + (long long)it.lv * tb.H + l;
        return c;
    }
    c.m = tb.G + (long long)it.g * tb.H + l;
    const int kk[3] = {k1, k2, 0};
    // a plane over (lo, hi): index off + k_lo + dlo * k_hi; axis 3 can only be hi
    c.wa = tb.planes + it.wa_off + kk[it.wa_lo] + (it.wa_hi == 2 ? 0 : it.wa_dlo * kk[it.wa_hi]);
    c.was = it.wa_hi == 2 ? it.wa_dlo : 0;
    c.wb = tb.planes + it.wb_off + kk[it.wb_lo] + (it.wb_hi == 2 ? 0 : it.wb_dlo * kk[it.wb_hi]);
    c.wbs = it.wb_hi == 2 ? it.wb_dlo : 0;
    return c;
}

// Plane a of a directional item at (k1, k2), for a plane constant along axis 3
// (it.wa_hi != 2): the per-line scalar of NSMaskLine's wa[0], read with only
// the plane's four fields.
__device__ __forceinline__ float ns_wedge_a_line(const NSMaskTables& tb, const NSItem* it, int k1, int k2) {
    const int off = it->wa_off, lo = it->wa_lo, hi = it->wa_hi, dlo = it->wa_dlo;
    const int klo = lo == 0 ? k1 : k2, khi = hi == 0 ? k1 : k2;
    return tb.planes[off + klo + dlo * khi];
}

__device__ __forceinline__ float ns_mask_at(const NSMaskLine& c, int k3, long long si) {
    if (c.low) return c.lowc * c.lowv[k3];
    float g = c.m[(long long)k3 * si];
    if (c.plain) return g;
    return (g * c.wa[k3 * c.was]) * c.wb[k3 * c.wbs];
}

// Analysis pass-3 load for the register kernel: X times the mask of item z.
struct RLoadNSMask {
    const float2* X;
    NSMaskTables tb;
    const NSItem* items;
    int item0;
    int synth;
    struct Ctx {
        const float2* x;
        NSMaskLine m;
        long long si;
    };
    __device__ __forceinline__ Ctx line(int z, int l, bool valid) const {
        Ctx c;
        c.si = (long long)tb.h1 * tb.n2;
        c.x = X + (valid ? l : 0);
        c.m = ns_mask_line(tb, items[item0 + z], valid ? l : 0, synth != 0);
        return c;
    }
    __device__ __forceinline__ float2 get(const Ctx& c, int i) const {
        return c_scale(c.x[i * c.si], ns_mask_at(c.m, i, c.si));
    }
};

}  // namespace sfl
