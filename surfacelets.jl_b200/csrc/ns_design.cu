// NSSurfacelet (and NDFB) mask tables designed on the device, in float64:
// per bin of the rfft grid, m1 = f0(M1) from the separable factors the host
// computes (the axis-1-contracted mapping kernel, the Bernstein tables of
// axes 2 and 3, m2), then every group table B_j sqrt(W_i) (or W_i, or the
// hourglass mask alone for the standalone bank) and the level bandpasses
// B_j of an untight bank, rounded to float32; and the support box of each
// table.  The arithmetic repeats the host design's (src/directional/
// hourglass.jl:172-189, 289-303; src/transforms/ns_surfacelet.jl:265-272)
// operation for operation, without fused multiply-adds, so the tables are
// the host design's bit for bit; only the O(N (order+1)^2) contraction and
// the O(N S) products move to the GPU.
#include <algorithm>
#include <vector>

#include "plan.h"

namespace sfl {

namespace {

struct NSDesignArgs {
    int h1, n2, n3, np, poly, tight, ndfb, J, ngroups, nbl;
    long long H;
    const double* t1;
    const double* b2;
    const double* b3;
    const double* m2;
    const double* pa;   // per level: the axis-1 | axis-2 | axis-3 vectors
    const double* pl;
    float* G;
    float* Bl;
    int* box;           // per table: max k1, max |k2| of its nonzero bins
};

__device__ __forceinline__ double halfband_dev(double x, int m) {
    const double u = __ddiv_rn(__dadd_rn(1.0, x), 2.0);
    const double v = __ddiv_rn(__dsub_rn(1.0, x), 2.0);
    if (u == 0.0) return 0.0;
    double s = 0.0, c = 1.0, vk = 1.0;
    for (int k = 0; k <= m; ++k) {
        s = __dadd_rn(s, __dmul_rn(c, vk));
        c = __ddiv_rn(__dmul_rn(c, (double)(m + k + 1)), (double)(k + 1));
        vk = __dmul_rn(vk, v);
    }
    double um = 1.0;
    for (int k = 0; k <= m; ++k) um = __dmul_rn(um, u);
    return __dmul_rn(um, s);
}

// B_lv at (k1, k2, k3): a0 a1 a2 sqrt(max(1 - (l0 l1 l2)^2, 0)).
__device__ __forceinline__ double bandpass(const NSDesignArgs& a, int lv, int k1, int k2, int k3) {
    const int stride = a.h1 + a.n2 + a.n3;
    const double* A = a.pa + (long long)lv * stride;
    const double* Lp = a.pl + (long long)lv * stride;
    const double L = __dmul_rn(__dmul_rn(Lp[k1], Lp[a.h1 + k2]), Lp[a.h1 + a.n2 + k3]);
    const double r = __dsub_rn(1.0, __dmul_rn(L, L));
    return __dmul_rn(__dmul_rn(__dmul_rn(A[k1], A[a.h1 + k2]), A[a.h1 + a.n2 + k3]), __dsqrt_rn(r < 0.0 ? 0.0 : r));
}

__device__ __forceinline__ void track_box(int* box, int t, bool nz, int k1, int k2abs) {
    // warp maxima first, one atomic a warp
    const int m1 = __reduce_max_sync(0xffffffffu, nz ? k1 : -1);
    const int m2 = __reduce_max_sync(0xffffffffu, nz ? k2abs : -1);
    if ((threadIdx.x & 31) == 0 && m1 >= 0) {
        atomicMax(box + 2 * t, m1);
        atomicMax(box + 2 * t + 1, m2);
    }
}

__global__ void ns_design_kernel(NSDesignArgs a) {
    const long long Hr = (a.H + 31) / 32 * 32;   // whole warps in every iteration
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < Hr;
         q += (long long)gridDim.x * blockDim.x) {
        const bool in = q < a.H;
        const long long e = in ? q : 0;
        const int k1 = (int)(e % a.h1);
        const long long r = e / a.h1;
        const int k2 = (int)(r % a.n2), k3 = (int)(r / a.n2);
        const int np = a.np;
        double s = 0.0;
        for (int j3 = 0; j3 < np; ++j3) {
            double u = 0.0;
            const double* tp = a.t1 + np * (j3 + (long long)np * k1);
            for (int j2 = 0; j2 < np; ++j2) u = __dadd_rn(u, __dmul_rn(tp[j2], a.b2[j2 + np * k2]));
            s = __dadd_rn(s, __dmul_rn(u, a.b3[j3 + np * k3]));
        }
        const double f1 = halfband_dev(s, a.poly);
        const double f2 = a.m2[k2 + (long long)a.n2 * k3];
        const int k2abs = k2 < a.n2 - k2 ? k2 : a.n2 - k2;
        for (int g = 0; g < a.ngroups; ++g) {
            const int i = g % 3 + 1;
            const double w1 = i == 1 ? f1 : __dsub_rn(1.0, f1);
            const double w2 = i == 1 ? 1.0 : (i == 2 ? f2 : __dsub_rn(1.0, f2));
            const double w = __dmul_rn(w1, w2);
            const double hg = a.tight ? __dsqrt_rn(w < 0.0 ? 0.0 : w) : w;
            const double v = a.ndfb ? hg : __dmul_rn(bandpass(a, a.J - 1 - g / 3, k1, k2, k3), hg);
            if (in) a.G[g * a.H + e] = (float)v;
            track_box(a.box, g, in && v != 0.0, k1, k2abs);
        }
        for (int lv = 0; lv < a.nbl; ++lv) {
            const double v = a.ndfb ? 1.0 : bandpass(a, lv, k1, k2, k3);
            if (in) a.Bl[lv * a.H + e] = (float)v;
            track_box(a.box, a.ngroups + lv, in && v != 0.0, k1, k2abs);
        }
    }
}

template <class T>
void put(DevMem& m, const std::vector<T>& v) {
    m.alloc(sizeof(T) * (v.empty() ? 1 : v.size()));
    if (!v.empty()) cuda_check(cudaMemcpy(m.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
}

}  // namespace

void ns_design_tables_device(NSPlan& P) {
    const NSDesign& D = P.design;
    const int J = P.p.scales, h1 = P.h1, n2 = P.dims[1], n3 = P.dims[2];
    const bool ndfb = P.ndfb;
    const int ngroups = ndfb ? 3 : 3 * J;
    const int nbl = P.p.tight ? 0 : (ndfb ? 1 : J);
    std::vector<double> pa, pl;
    const int nlv = ndfb ? 0 : J;
    for (int lv = 0; lv < nlv; ++lv)
        for (int d = 0; d < 3; ++d) {
            pa.insert(pa.end(), D.pa[lv][d].begin(), D.pa[lv][d].end());
            pl.insert(pl.end(), D.pl[lv][d].begin(), D.pl[lv][d].end());
        }
    DevMem t1, b2, b3, m2, dpa, dpl, box;
    put(t1, D.hg.t1);
    put(b2, D.hg.b2);
    put(b3, D.hg.b3);
    put(m2, D.hg.m2);
    put(dpa, pa);
    put(dpl, pl);
    box.alloc(sizeof(int) * 2 * (ngroups + nbl));
    cuda_check(cudaMemset(box.p, 0xff, box.bytes), "cudaMemset(box)");   // -1
    P.G.alloc(sizeof(float) * ngroups * P.H);
    P.Bl.alloc(sizeof(float) * (nbl ? nbl * P.H : 1));
    NSDesignArgs a{};
    a.h1 = h1;
    a.n2 = n2;
    a.n3 = n3;
    a.np = D.hg.np;
    a.poly = P.p.halfband_order;
    a.tight = P.p.tight ? 1 : 0;
    a.ndfb = ndfb ? 1 : 0;
    a.J = J;
    a.ngroups = ngroups;
    a.nbl = nbl;
    a.H = P.H;
    a.t1 = t1.as<double>();
    a.b2 = b2.as<double>();
    a.b3 = b3.as<double>();
    a.m2 = m2.as<double>();
    a.pa = dpa.as<double>();
    a.pl = dpl.as<double>();
    a.G = P.G.as<float>();
    a.Bl = P.Bl.as<float>();
    a.box = box.as<int>();
    int dev = 0, sms = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    const long long blocks = std::max<long long>(1, std::min<long long>((P.H + 255) / 256, (long long)sms * 8));
    ns_design_kernel<<<(unsigned)blocks, 256>>>(a);
    cuda_check(cudaGetLastError(), "ns_design_kernel launch");
    std::vector<int> hb(2 * (ngroups + nbl));
    cuda_check(cudaMemcpy(hb.data(), box.p, sizeof(int) * hb.size(), cudaMemcpyDeviceToHost), "box readback");
    P.boxes.clear();
    for (int g = 0; g < ngroups; ++g) P.boxes.push_back(ns_make_box(hb[2 * g] + 1, hb[2 * g + 1], n2));
    if (!ndfb)
        for (int lv = 0; lv < nbl; ++lv) {
            // the synthesis bandpass B_j covers the group factors of its level
            const NSBox bb = ns_make_box(hb[2 * (ngroups + lv)] + 1, hb[2 * (ngroups + lv) + 1], n2);
            for (int i = 0; i < 3; ++i) P.boxes[3 * (J - 1 - lv) + i] = bb;
        }
}

}  // namespace sfl
