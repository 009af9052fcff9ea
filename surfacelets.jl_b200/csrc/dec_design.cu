// Design tables of the decimated Surfacelet composed on the device: the ritf
// hourglass masks V_K (src/directional/ritf.jl:89-108) over the half-K grids
// and the IRC filter slices of every stage (src/directional/irc.jl:49-67).
//
// The host supplies the separable factors (design.cpp): the 2-D diamond
// planes P[K][m] of the ritf construction and the 1-D tables of one stage's
// ladder filters (IRCFactors).  Every per-bin step here is one IEEE double
// operation through a round-to-nearest intrinsic (no contraction), in the
// order of the host's ritf_compose and irc_slice_values, so the tables equal
// the host's float64 design bit for bit before the rounding to float32.
#include <vector>

#include "design.h"
#include "plan.h"

namespace sfl {

namespace {

// V_K at (i0, i1, i2) of the half-K grid: h_K = P[K][a] P[K][b] (a < b the
// other two axes), tot = (h_0 + h_1) + h_2, V_K = sqrt((3 h_K) / tot).
__global__ void ritf_compose_kernel(const double* __restrict__ planes, int3 n, int K, int3 hd, long long total,
                                    long long off01, long long off02, long long off10, long long off12,
                                    long long off20, long long off21, float* __restrict__ V) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += stride) {
        const int i0 = (int)(e % hd.x);
        const long long r = e / hd.x;
        const int i1 = (int)(r % hd.y);
        const int i2 = (int)(r / hd.y);
        // plane P[K][m] holds (i_K, i_m) at i_K + n_K i_m
        const double h0 = __dmul_rn(planes[off01 + i0 + (long long)n.x * i1], planes[off02 + i0 + (long long)n.x * i2]);
        const double h1 = __dmul_rn(planes[off10 + i1 + (long long)n.y * i0], planes[off12 + i1 + (long long)n.y * i2]);
        const double h2 = __dmul_rn(planes[off20 + i2 + (long long)n.z * i0], planes[off21 + i2 + (long long)n.z * i1]);
        const double tot = __dadd_rn(__dadd_rn(h0, h1), h2);
        const double hk = K == 0 ? h0 : (K == 1 ? h1 : h2);
        V[e] = __double2float_rn(__dsqrt_rn(__ddiv_rn(__dmul_rn(3.0, hk), tot)));
    }
}

// The four slice planes of one IRC stage at (k, c), entry k + nKh c:
// analysis channel 0/1 (x 0.5), synthesis channel 0/1.
__global__ void irc_slice_kernel(const double* __restrict__ f, int nKh, int nm, int W, int ng, int nq, double r,
                                 long long o_t, long long o_bK, long long o_sth, long long o_cth, long long o_sph,
                                 long long o_cph, float2* __restrict__ a0, float2* __restrict__ a1,
                                 float2* __restrict__ s0, float2* __restrict__ s1) {
    const long long total = (long long)nKh * nm;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += stride) {
        const int k = (int)(e % nKh);
        const int c = (int)(e / nKh);
        const int g = c / W, l = c - g * W;
        double s = 0.0, sw = 0.0, cw = 0.0;
        for (int i = 0; i < nq; ++i) {
            const double st = f[o_sth + (long long)i * W + l], ct = f[o_cth + (long long)i * W + l];
            const long long q = ((long long)i * ng + g) * nKh + k;
            const double sp = f[o_sph + q], cp = f[o_cph + q];
            const double sq = __dadd_rn(__dmul_rn(st, cp), __dmul_rn(ct, sp));
            if (i == 0) {
                sw = sq;
                cw = __dsub_rn(__dmul_rn(ct, cp), __dmul_rn(st, sp));
            }
            s = __dadd_rn(s, __dmul_rn(f[o_t + i], sq));
        }
        const double bm = __dmul_rn(2.0, s);
        const double B = __dmul_rn(-f[o_bK + k], bm);
        const double B2 = __dmul_rn(B, B);
        const double h0 = __dmul_rn(r, __dadd_rn(1.0, B));
        const double h1 = __dmul_rn(r, __dsub_rn(__dsub_rn(2.0, B), B2));
        const double g0 = __dmul_rn(r, __dsub_rn(__dadd_rn(2.0, B), B2));
        const double g1 = __dmul_rn(r, __dsub_rn(1.0, B));
        a0[e] = make_float2(__double2float_rn(__dmul_rn(0.5, h0)), 0.f);
        a1[e] = make_float2(__double2float_rn(__dmul_rn(0.5, __dmul_rn(cw, h1))),
                            __double2float_rn(__dmul_rn(0.5, __dmul_rn(sw, h1))));
        s0[e] = make_float2(__double2float_rn(g0), 0.f);
        s1[e] = make_float2(__double2float_rn(__dmul_rn(cw, g1)), __double2float_rn(-__dmul_rn(sw, g1)));
    }
}

unsigned blocks_for(long long total) {
    long long b = (total + 255) / 256;
    return (unsigned)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

void ritf_masks_device(const int n[3], const std::vector<double> P[3][3], float* const V[3], cudaStream_t st) {
    // the six planes in one buffer, P[K][m] at off[K][m]
    std::vector<double> all;
    long long off[3][3] = {};
    for (int K = 0; K < 3; ++K)
        for (int m = 0; m < 3; ++m) {
            if (m == K) continue;
            off[K][m] = (long long)all.size();
            all.insert(all.end(), P[K][m].begin(), P[K][m].end());
        }
    DevMem buf;
    buf.alloc(sizeof(double) * all.size());
    cuda_check(cudaMemcpyAsync(buf.p, all.data(), sizeof(double) * all.size(), cudaMemcpyHostToDevice, st),
               "ritf planes upload");
    for (int K = 0; K < 3; ++K) {
        int3 hd = make_int3(n[0], n[1], n[2]);
        if (K == 0) hd.x = n[0] / 2 + 1;
        if (K == 1) hd.y = n[1] / 2 + 1;
        if (K == 2) hd.z = n[2] / 2 + 1;
        const long long total = (long long)hd.x * hd.y * hd.z;
        ritf_compose_kernel<<<blocks_for(total), 256, 0, st>>>(buf.as<double>(), make_int3(n[0], n[1], n[2]), K, hd,
                                                               total, off[0][1], off[0][2], off[1][0], off[1][2],
                                                               off[2][0], off[2][1], V[K]);
        cuda_check(cudaGetLastError(), "ritf_compose_kernel launch");
    }
    cuda_check(cudaStreamSynchronize(st), "ritf design");   // the planes buffer is freed on return
}

void irc_slices_device(const IRCFactors& F, float2* const out[4], cudaStream_t st) {
    std::vector<double> all;
    auto put = [&](const std::vector<double>& v) {
        const long long o = (long long)all.size();
        all.insert(all.end(), v.begin(), v.end());
        return o;
    };
    const long long o_t = put(F.t), o_bK = put(F.bK), o_sth = put(F.sth), o_cth = put(F.cth), o_sph = put(F.sph),
                    o_cph = put(F.cph);
    DevMem buf;
    buf.alloc(sizeof(double) * all.size());
    cuda_check(cudaMemcpyAsync(buf.p, all.data(), sizeof(double) * all.size(), cudaMemcpyHostToDevice, st),
               "irc factors upload");
    const long long total = (long long)F.nKh * F.nm;
    irc_slice_kernel<<<blocks_for(total), 256, 0, st>>>(buf.as<double>(), F.nKh, F.nm, F.W, F.ng, F.nq, F.r, o_t, o_bK,
                                                        o_sth, o_cth, o_sph, o_cph, out[0], out[1], out[2], out[3]);
    cuda_check(cudaGetLastError(), "irc_slice_kernel launch");
    cuda_check(cudaStreamSynchronize(st), "irc design");
}

}  // namespace sfl
