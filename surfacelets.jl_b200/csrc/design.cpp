// Float64 table design and parameter rules.  Each function names the
// reference code (Surfacelets.jl file:line) whose arithmetic it follows.
#include "design.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <sstream>

namespace sfl {

namespace {

const double kPi = 3.14159265358979323846;

long long gcdll(long long a, long long b) {
    a = a < 0 ? -a : a;
    b = b < 0 ? -b : b;
    while (b) {
        long long t = a % b;
        a = b;
        b = t;
    }
    return a;
}

Rat rnorm(Rat r) {
    long long g = gcdll(r.p, r.q);
    if (g == 0) return {0, 1};
    r.p /= g;
    r.q /= g;
    if (r.q < 0) {
        r.p = -r.p;
        r.q = -r.q;
    }
    return r;
}
Rat radd(Rat a, Rat b) { return rnorm({a.p * b.q + b.p * a.q, a.q * b.q}); }
Rat rsub(Rat a, Rat b) { return rnorm({a.p * b.q - b.p * a.q, a.q * b.q}); }
Rat rmul(Rat a, Rat b) { return rnorm({a.p * b.p, a.q * b.q}); }
long long rceil(Rat a) {
    a = rnorm(a);
    long long d = a.p / a.q;
    if (a.p % a.q != 0 && a.p > 0) d += 1;
    return d;
}
long long rfloor(Rat a) {
    a = rnorm(a);
    long long d = a.p / a.q;
    if (a.p % a.q != 0 && a.p < 0) d -= 1;
    return d;
}

double binom(int n, int k) {
    double r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return std::round(r);
}

std::string fmt_vec(const int32_t* v, int n) {
    std::ostringstream s;
    s << "[";
    for (int i = 0; i < n; ++i) s << (i ? ", " : "") << v[i];
    s << "]";
    return s.str();
}

std::string fmt_real(double x) {
    // Julia prints an integral Float64 with a trailing ".0".
    std::ostringstream s;
    if (std::isfinite(x) && x == std::floor(x) && std::fabs(x) < 1e15) {
        s << (long long)x << ".0";
    } else {
        s.precision(17);
        s << x;
    }
    return s.str();
}

}  // namespace

std::string fmt_dims(const int d[3]) {
    std::ostringstream s;
    s << "(" << d[0] << ", " << d[1] << ", " << d[2] << ")";
    return s.str();
}

// src/filters/bernstein.jl:64-67
std::vector<double> dft_frequencies(int n, bool half) {
    int m = half ? n / 2 + 1 : n;
    std::vector<double> w(m);
    for (int k = 0; k < m; ++k) w[k] = 2 * kPi * k / n;
    return w;
}

// src/filters/bernstein.jl:72-79
std::vector<double> folded_frequencies(int n, bool half) {
    if (half) return dft_frequencies(n, true);
    std::vector<double> w(n);
    for (int k = 0; k < n; ++k) {
        double v = 2 * kPi * k / n;
        w[k] = v > kPi ? v - 2 * kPi : v;
    }
    return w;
}

// src/filters/bernstein.jl:36-53
std::vector<double> bernstein_table(int N, const std::vector<double>& omega) {
    if (N < 1) throw ArgError("Bernstein order must be ≥ 1");
    std::vector<double> bin(N + 1);
    for (int j = 0; j <= N; ++j) bin[j] = binom(N, j);
    std::vector<double> tbl((size_t)(N + 1) * omega.size());
    for (size_t k = 0; k < omega.size(); ++k) {
        double x = std::sin(omega[k] / 2);
        x = x * x;
        x = std::min(std::max(x, 0.0), 1.0);
        double y = 1 - x;
        for (int j = 0; j <= N; ++j) tbl[j + (N + 1) * k] = bin[j] * std::pow(x, j) * std::pow(y, N - j);
    }
    return tbl;
}

// src/filters/bernstein.jl:171-190 — the sum first, scaled last.  The powers
// are running products, so the device-side design (ns_design.cu) repeats the
// same roundings.
double halfband_split(double x, int m) {
    if (m < 0) throw ArgError("polynomial order must be ≥ 0");
    double u = (1 + x) / 2;
    double v = (1 - x) / 2;
    if (u == 0) return 0.0;
    double s = 0, c = 1, vk = 1;
    for (int k = 0; k <= m; ++k) {
        s += c * vk;
        c = c * (m + k + 1) / (k + 1);
        vk *= v;
    }
    double um = 1;
    for (int k = 0; k <= m; ++k) um *= u;
    return um * s;
}

// src/filters/bernstein.jl:196-203
double soft_step(double s, double b, double w, int poly) {
    if (w <= 0) return s >= b ? 1.0 : 0.0;
    double u = (s - b) / w;
    u = std::min(std::max(u, -1.0), 1.0);
    return halfband_split(u, poly);
}

// src/pyramid/fourier_pyramid.jl:155-160 (file numbering)
void rcos_edges(int n, Rat w, Rat t, int& P, int& Q) {
    Rat h{n, 2};
    P = (int)rceil(rmul(h, radd(w, t)));
    Q = (int)rfloor(rmul(h, rsub(w, t)));
}

static double rcos(double x) { return x <= 0 ? 0.0 : (x >= 1 ? 1.0 : (1 - std::cos(kPi * x)) / 2); }

// src/pyramid/fourier_pyramid.jl:163-174 (file numbering)
std::vector<double> rcos_axis(int n, Rat w, Rat t, int& P) {
    int Q;
    rcos_edges(n, w, t, P, Q);
    std::vector<double> prof(n);
    for (int k = 0; k < n; ++k) {
        int f = std::abs(k <= n / 2 ? k : k - n);
        prof[k] = f <= P ? std::sqrt(rcos(double(P - f) / double(P - Q))) : 0.0;
    }
    return prof;
}

// ── NSSurfacelet ──────────────────────────────────────────────────────────────

// src/types/transforms.jl:93-104, 149-154
void ns_check_params(const sfl_ns_params& p) {
    if (p.scales < 1) throw ArgError("scales must be ≥ 1, got " + std::to_string(p.scales));
    if (p.scales > SFL_MAX_SCALES)
        throw ArgError("scales must be ≤ " + std::to_string(SFL_MAX_SCALES) + " in this library, got " +
                       std::to_string(p.scales));
    for (int j = 0; j < p.scales; ++j)
        if (p.direction_levels[j] < 0)
            throw ArgError("direction_levels entries must be ≥ 0, got " + fmt_vec(p.direction_levels, p.scales));
    for (int j = 0; j < p.scales; ++j)
        if (p.direction_levels[j] > 12)
            throw ArgError("direction_levels entries must be ≤ 12 in this library, got " +
                           fmt_vec(p.direction_levels, p.scales));
    if (p.bernstein_order < 1)
        throw ArgError("bernstein_order must be ≥ 1, got " + std::to_string(p.bernstein_order));
    if (p.halfband_order < 0)
        throw ArgError("halfband_order must be ≥ 0, got " + std::to_string(p.halfband_order));
    if (!(p.transition >= 0)) throw ArgError("transition must be ≥ 0, got " + fmt_real(p.transition));
}

// src/types/transforms.jl:157
int ns_nbands(const sfl_ns_params& p, int j) { return 3 * (1 << p.direction_levels[j - 1]); }

// src/transforms/ns_surfacelet.jl:527
int ns_nsubbands(const sfl_ns_params& p) {
    int s = 1;
    for (int j = 1; j <= p.scales; ++j) s += ns_nbands(p, j);
    return s;
}

// Per-axis pyramid factors: src/pyramid/fourier_pyramid.jl:256-263 (file numbering)
static void rc_responses(int J, int n, int nbins, std::vector<std::vector<double>>& acc,
                         std::vector<std::vector<double>>& prof) {
    prof.assign(J, {});
    for (int j = 1; j <= J; ++j) {
        int P;
        std::vector<double> full = rcos_axis(n, Rat{1, 1LL << j}, Rat{1, 3 * (1LL << j)}, P);
        prof[j - 1].assign(full.begin(), full.begin() + nbins);
    }
    acc.assign(J + 1, std::vector<double>(nbins, 1.0));
    for (int j = 0; j < J; ++j)
        for (int b = 0; b < nbins; ++b) acc[j + 1][b] = acc[j][b] * prof[j][b];
}

// src/transforms/ns_surfacelet.jl:98-115
void ns_check_size(const sfl_ns_params& p, const int dims[3]) {
    for (int d = 0; d < 3; ++d)
        if (dims[d] < 1) throw ArgError("volume size must be positive, got " + fmt_dims(dims));
    int nb[3] = {dims[0] / 2 + 1, dims[1], dims[2]};
    std::vector<std::vector<double>> acc[3], prof[3];
    for (int d = 0; d < 3; ++d) rc_responses(p.scales, dims[d], nb[d], acc[d], prof[d]);
    for (int j = 0; j < p.scales; ++j) {
        bool empty = true;
        for (int d = 0; d < 3 && empty; ++d)
            for (int b = 0; b < nb[d]; ++b)
                if (!(acc[d][j][b] == 0 || prof[d][j][b] == 1)) {
                    empty = false;
                    break;
                }
        if (empty)
            throw ArgError("size " + fmt_dims(dims) + " is too small for " + std::to_string(p.scales) +
                           " scales: scale " + std::to_string(p.scales - j) + " would be empty");
    }
}

// Canonical signed slope: src/directional/ndfb_wedges.jl:78, 97-106
static double wedge_ratio(double wr, double wt, bool ref_self, bool tr_self) {
    if (wr == 0) return 0.0;
    if (ref_self) return std::fabs(wt) / std::fabs(wr);
    if (tr_self) return wt / std::fabs(wr);
    return wt / wr;
}

// src/directional/ndfb_wedges.jl:25-32
static double wedge_weight(double s, int idx, int nw, double transition, int poly) {
    if (nw == 1) return 1.0;
    double delta = 2.0 / nw;
    double width = transition * delta;
    double lo = idx == 1 ? 1.0 : soft_step(s, -1.0 + (idx - 1) * delta, width, poly);
    double hi = idx == nw ? 0.0 : soft_step(s, -1.0 + idx * delta, width, poly);
    return lo - hi;
}

static void transverse_axes(int i, int& a, int& b) {
    if (i == 1) {
        a = 2;
        b = 3;
    } else if (i == 2) {
        a = 1;
        b = 3;
    } else {
        a = 1;
        b = 2;
    }
}

// src/directional/ndfb_wedges.jl:45-69, oriented as :112-113
static WedgePlanes wedge_masks_plane(const int dims[3], int ref, int tr, int l, int poly, double transition,
                                     bool tight) {
    WedgePlanes W;
    W.ref = ref;
    W.tr = tr;
    W.lo = std::min(ref, tr);
    W.hi = std::max(ref, tr);
    int nref = dims[ref - 1], ntr = dims[tr - 1];
    std::vector<double> wref = folded_frequencies(nref, ref == 1);
    std::vector<double> wtr = folded_frequencies(ntr, tr == 1);
    int dref = (int)wref.size(), dtr = (int)wtr.size();
    W.dlo = ref < tr ? dref : dtr;
    W.dhi = ref < tr ? dtr : dref;
    int nw = 1 << l;
    W.w.assign(nw, std::vector<double>((size_t)dref * dtr, 1.0));
    if (l == 0) return W;
    for (int q = 0; q < dtr; ++q)
        for (int pp = 0; pp < dref; ++pp) {
            bool rs = (2 * pp) % nref == 0;
            bool ts = (2 * q) % ntr == 0;
            double s = wedge_ratio(wref[pp], wtr[q], rs, ts);
            size_t at = ref < tr ? (size_t)pp + (size_t)dref * q : (size_t)q + (size_t)dtr * pp;
            for (int k = 1; k <= nw; ++k) {
                double v = wedge_weight(s, k, nw, transition, poly);
                W.w[k - 1][at] = tight ? std::sqrt(std::max(v, 0.0)) : v;
            }
        }
    return W;
}

// src/directional/hourglass.jl:172-189 and src/filters/bernstein.jl:97-151
// The separable parts of the hourglass tables (src/directional/hourglass.jl:
// 172-189): the Bernstein tables of axes 2 and 3, the 3-D mapping kernel
// contracted along axis 1, t1[j2, j3, k1], and m2 = f0(M2) on (n2, n3).
NSHourglassFactors ns_hourglass_factors(const int dims[3], int order, int poly) {
    NSHourglassFactors F;
    int n1 = dims[0], n2 = dims[1], n3 = dims[2], h1 = n1 / 2 + 1;
    int np = order + 1;
    F.np = np;
    std::vector<double> b1 = bernstein_table(order, dft_frequencies(n1, true));
    F.b2 = bernstein_table(order, dft_frequencies(n2, false));
    F.b3 = bernstein_table(order, dft_frequencies(n3, false));
    const std::vector<double>& b2 = F.b2;
    const std::vector<double>& b3 = F.b3;
    // c[j1,j2,j3] = sign(j1 - max(j2, j3)): group (1,) of mapping_coefficients.
    auto c3 = [&](int j1, int j2, int j3) {
        int b = std::max(j2, j3);
        return j1 > b ? 1.0 : (j1 < b ? -1.0 : 0.0);
    };
    // contract axis 1: t1[j2, j3, k1]
    F.t1.assign((size_t)np * np * h1, 0.0);
    for (int k1 = 0; k1 < h1; ++k1)
        for (int j3 = 0; j3 < np; ++j3)
            for (int j2 = 0; j2 < np; ++j2) {
                double s = 0;
                for (int j1 = 0; j1 < np; ++j1) s += c3(j1, j2, j3) * b1[j1 + np * k1];
                F.t1[j2 + np * (j3 + (size_t)np * k1)] = s;
            }
    // 2-D kernel on (w2, w3): c2[j2, j3] = sign(j2 - j3)
    std::vector<double> t((size_t)np * n3, 0.0);   // t[j2, k3] = sum_j3 c2 b3[j3, k3]
    for (int k3 = 0; k3 < n3; ++k3)
        for (int j2 = 0; j2 < np; ++j2) {
            double s = 0;
            for (int j3 = 0; j3 < np; ++j3) s += (j2 > j3 ? 1.0 : (j2 < j3 ? -1.0 : 0.0)) * b3[j3 + np * k3];
            t[j2 + np * k3] = s;
        }
    F.m2.assign((size_t)n2 * n3, 0.0);
    for (int k3 = 0; k3 < n3; ++k3)
        for (int k2 = 0; k2 < n2; ++k2) {
            double s = 0;
            for (int j2 = 0; j2 < np; ++j2) s += b2[j2 + np * k2] * t[j2 + np * k3];
            F.m2[k2 + (size_t)n2 * k3] = halfband_split(s, poly);
        }
    return F;
}

// m1 = f0(M1) on the rfft grid: the contraction along axes 2 and 3 (the
// device design does the same per bin, in the same order).
void ns_design_fill_m1(NSDesign& D) {
    if (!D.m1.empty()) return;
    const NSHourglassFactors& F = D.hg;
    const int h1 = D.h1, n2 = D.dims[1], n3 = D.dims[2], np = F.np;
    D.m1.assign((size_t)h1 * n2 * n3, 0.0);
    std::vector<double> t2(np);
    for (int k3 = 0; k3 < n3; ++k3)
        for (int k2 = 0; k2 < n2; ++k2)
            for (int k1 = 0; k1 < h1; ++k1) {
                double s = 0;
                for (int j3 = 0; j3 < np; ++j3) {
                    double u = 0;
                    for (int j2 = 0; j2 < np; ++j2) u += F.t1[j2 + np * (j3 + (size_t)np * k1)] * F.b2[j2 + np * k2];
                    s += u * F.b3[j3 + np * k3];
                }
                D.m1[k1 + (size_t)h1 * (k2 + (size_t)n2 * k3)] = halfband_split(s, D.p.halfband_order);
            }
}

// src/transforms/ns_surfacelet.jl:98-123, 178-185
NSDesign ns_design(const sfl_ns_params& p, const int dims[3], bool pyramid, bool with_m1) {
    ns_check_params(p);
    if (pyramid) ns_check_size(p, dims);
    NSDesign D;
    for (int d = 0; d < 3; ++d) D.dims[d] = dims[d];
    D.h1 = dims[0] / 2 + 1;
    D.p = p;
    D.hg = ns_hourglass_factors(dims, p.bernstein_order, p.halfband_order);
    D.m2 = D.hg.m2;
    if (with_m1) ns_design_fill_m1(D);
    D.wedges.resize(p.scales);
    for (int j = 0; j < p.scales; ++j) {
        int L = p.direction_levels[j];
        int la = (L + 1) / 2, lb = L / 2;
        for (int i = 1; i <= 3; ++i) {
            int a, b;
            transverse_axes(i, a, b);
            D.wedges[j][i - 1][0] = wedge_masks_plane(dims, i, a, la, p.halfband_order, p.transition, p.tight);
            D.wedges[j][i - 1][1] = wedge_masks_plane(dims, i, b, lb, p.halfband_order, p.transition, p.tight);
        }
    }
    int nb[3] = {D.h1, dims[1], dims[2]};
    std::vector<std::vector<double>> acc[3], prof[3];
    for (int d = 0; d < 3; ++d) rc_responses(p.scales, dims[d], nb[d], acc[d], prof[d]);
    D.pa.resize(p.scales + 1);
    D.pl.resize(p.scales);
    for (int lv = 0; lv <= p.scales; ++lv)
        for (int d = 0; d < 3; ++d) D.pa[lv][d] = acc[d][lv];
    for (int lv = 0; lv < p.scales; ++lv)
        for (int d = 0; d < 3; ++d) D.pl[lv][d] = prof[d][lv];
    return D;
}

// The hourglass mask of the standalone bank: sqrt(W_i) when tight, W_i
// otherwise (src/directional/hourglass.jl:264-303, 400-412).
std::vector<double> ns_hourglass_mask(const NSDesign& D, int i) {
    const int h1 = D.h1, n2 = D.dims[1], n3 = D.dims[2];
    std::vector<double> G((size_t)h1 * n2 * n3);
    for (int k3 = 0; k3 < n3; ++k3)
        for (int k2 = 0; k2 < n2; ++k2)
            for (int k1 = 0; k1 < h1; ++k1) {
                size_t q = k1 + (size_t)h1 * (k2 + (size_t)n2 * k3);
                double f1 = D.m1[q], f2 = D.m2[k2 + (size_t)n2 * k3];
                double w1 = i == 1 ? f1 : 1 - f1;
                double w2 = i == 1 ? 1.0 : (i == 2 ? f2 : 1 - f2);
                double w = w1 * w2;
                G[q] = D.p.tight ? std::sqrt(std::max(w, 0.0)) : w;
            }
    return G;
}

// src/transforms/ns_surfacelet.jl:265-272 (_hg_factor, _bandpass), 278-303
std::vector<double> ns_group_mask(const NSDesign& D, int lv, int i, bool hourglass) {
    const int h1 = D.h1, n2 = D.dims[1], n3 = D.dims[2];
    std::vector<double> G((size_t)h1 * n2 * n3);
    const auto& a = D.pa[lv];
    const auto& l = D.pl[lv];
    for (int k3 = 0; k3 < n3; ++k3)
        for (int k2 = 0; k2 < n2; ++k2)
            for (int k1 = 0; k1 < h1; ++k1) {
                size_t q = k1 + (size_t)h1 * (k2 + (size_t)n2 * k3);
                double L = l[0][k1] * l[1][k2] * l[2][k3];
                double B = a[0][k1] * a[1][k2] * a[2][k3] * std::sqrt(std::max(1 - L * L, 0.0));
                if (!hourglass) {
                    G[q] = B;
                    continue;
                }
                double f1 = D.m1[q], f2 = D.m2[k2 + (size_t)n2 * k3];
                double w1 = i == 1 ? f1 : 1 - f1;
                double w2 = i == 1 ? 1.0 : (i == 2 ? f2 : 1 - f2);
                double w = w1 * w2;
                G[q] = B * (D.p.tight ? std::sqrt(std::max(w, 0.0)) : w);
            }
    return G;
}

// ── Decimated Surfacelet ──────────────────────────────────────────────────────

// src/types/transforms.jl:270-278 with the wedge split of ndfb_wedges.jl:19
void surf_levels_from_int(int L, int out[3][3]) {
    int la = L >= 0 ? (L + 1) / 2 : -((-L) / 2);
    int lb = L >= 0 ? L / 2 : -((-L + 1) / 2);
    for (int K = 1; K <= 3; ++K) {
        int a, b;
        transverse_axes(K, a, b);
        for (int m = 1; m <= 3; ++m) out[K - 1][m - 1] = m == a ? la : (m == b ? lb : 0);
    }
}

// src/pyramid/fourier_pyramid.jl:148-153
void surf_pyramid_mode(double mode, Rat w[2], Rat t[2], Rat D[2]) {
    if (mode == 1) {
        w[0] = {1, 2}; w[1] = {1, 4}; t[0] = {1, 6}; t[1] = {1, 12}; D[0] = {1, 1}; D[1] = {2, 1};
    } else if (mode == 1.5) {
        w[0] = {1, 2}; w[1] = {3, 8}; t[0] = {1, 7}; t[1] = {1, 9}; D[0] = {3, 2}; D[1] = {2, 1};
    } else if (mode == 2) {
        w[0] = {1, 3}; w[1] = {1, 3}; t[0] = {1, 7}; t[1] = {1, 7}; D[0] = {2, 1}; D[1] = {2, 1};
    } else {
        throw ArgError("pyramid_ratio must be 1, 1.5 or 2, got " + fmt_real(mode));
    }
}

static const int kCbdOrders[] = {4, 6, 8, 10, 12, 14, 16, 18};

// The 1-D odd ladder taps t_q (q = 1, 3, ..., bo-1) of SurfBox's checkerboard
// filters of order bo.  A table that must equal SurfBox's for coefficient
// parity; it is the one in src/filters/checkerboard.jl:26-53.
static const std::vector<double>& cbd_ladder(int bo) {
    static const std::vector<double> t4 = {-0.6262169131293146, -0.2391935764853579};
    static const std::vector<double> t6 = {-0.6263429050738657, -0.18302382681237633, -0.10753046674888095};
    static const std::vector<double> t8 = {-0.627819441355453, -0.1868110527281001, -0.08821345831338342,
                                           -0.05299463507171143};
    static const std::vector<double> t10 = {-0.6290391996524649, -0.19023436487159193, -0.09316419099049718,
                                            -0.04787638089257991, -0.02729049477362672};
    static const std::vector<double> t12 = {-0.6299909650161403, -0.19294788893803155, -0.09719811683520764,
                                            -0.05257765509290852, -0.027224347419537415, -0.014421093056370137};
    static const std::vector<double> t14 = {-0.6307470366053054, -0.19509552613399547, -0.10042251574577052,
                                            -0.056418179282558024, -0.03113763249657735, -0.015819995468636647,
                                            -0.007750295209451851};
    static const std::vector<double> t16 = {-0.631356163548133, -0.19683521105934682, -0.10304471724680653,
                                            -0.05956342644490844, -0.03441276144847804, -0.018849533868796398,
                                            -0.009297418074817033, -0.004215553479603451};
    static const std::vector<double> t18 = {-0.6318535467876545, -0.19826135647461407, -0.10520738123671233,
                                            -0.06218709792109189, -0.037184557113685186, -0.021472356755448885,
                                            -0.011535270028700011, -0.00549634585408209, -0.0023119823375261405};
    switch (bo) {
        case 4: return t4;
        case 6: return t6;
        case 8: return t8;
        case 10: return t10;
        case 12: return t12;
        case 14: return t14;
        case 16: return t16;
        case 18: return t18;
    }
    throw ArgError("checkerboard_order must be one of [4, 6, 8, 10, 12, 14, 16, 18], got " + std::to_string(bo));
}

// src/types/transforms.jl:231-251
void surf_check_params(const sfl_surf_params& p) {
    if (p.scales < 1) throw ArgError("scales must be ≥ 1, got " + std::to_string(p.scales));
    if (p.scales > SFL_MAX_SCALES)
        throw ArgError("scales must be ≤ " + std::to_string(SFL_MAX_SCALES) + " in this library, got " +
                       std::to_string(p.scales));
    for (int j = 0; j < p.scales; ++j)
        for (int K = 0; K < 3; ++K)
            for (int m = 0; m < 3; ++m)
                if (m != K && p.levels[j][K][m] < 0) throw ArgError("directional levels must be ≥ 0");
    for (int j = 0; j < p.scales; ++j)
        for (int K = 0; K < 3; ++K)
            for (int m = 0; m < 3; ++m)
                if (m != K && p.levels[j][K][m] > 12)
                    throw ArgError("directional levels must be ≤ 12 in this library");
    Rat w[2], t[2], D[2];
    surf_pyramid_mode(p.pyramid_ratio, w, t, D);
    cbd_ladder(p.checkerboard_order);
    if (!(p.diamond_length % 2 == 1 && p.diamond_length >= 3))
        throw ArgError("diamond_length must be an odd integer ≥ 3, got " + std::to_string(p.diamond_length));
    if (!(p.kaiser_beta > 0)) throw ArgError("kaiser_beta must be > 0, got " + fmt_real(p.kaiser_beta));
    if (!(p.diamond_power % 2 == 0 && p.diamond_power > 0))
        throw ArgError("diamond_power must be a positive even integer, got " + std::to_string(p.diamond_power));
}

int surf_nsubbands_scale(const int lv[3][3]) {
    int s = 0;
    for (int K = 0; K < 3; ++K) s += 1 << (lv[K][0] + lv[K][1] + lv[K][2]);
    return s;
}

static void levels_of(const sfl_surf_params& p, int j, int lv[3][3]) {
    for (int K = 0; K < 3; ++K)
        for (int m = 0; m < 3; ++m) lv[K][m] = m == K ? 0 : p.levels[j][K][m];
}

static std::string fmt_ratio(double r) {
    std::ostringstream s;
    s << r;
    std::string v = s.str();
    if (v.find('.') == std::string::npos) v += ".0";
    return v;
}

// The first reason an axis does not fit, or "": src/transforms/surfacelet.jl:230-249
static std::string axis_problem(const sfl_surf_params& p, int a, int n) {
    int J = p.scales;
    Rat w[2], t[2], D[2];
    surf_pyramid_mode(p.pyramid_ratio, w, t, D);
    for (int j = 1; j <= J; ++j) {
        int s = J - j + 1;
        std::string where = "at scale " + std::to_string(s) + " of " + std::to_string(J) +
                            " (1 the coarsest) the length is " + std::to_string(n);
        if (n % 2 != 0) return where + ", which must be even";
        int lv[3][3];
        levels_of(p, s - 1, lv);
        int mx = 0;
        for (int K = 0; K < 3; ++K) mx = std::max(mx, lv[K][a - 1]);
        long long c = 1LL << mx;
        if (n % c != 0)
            return where + ", which the directional levels must split into " + std::to_string(c) + " wedge blocks";
        int k = j == 1 ? 0 : 1;
        Rat Dk = D[k];
        if ((n * Dk.q) % Dk.p != 0)
            return where + ", which resampling by " + std::to_string(Dk.p) + "/" + std::to_string(Dk.q) +
                   " needs to be a multiple of " + std::to_string(Dk.p);
        int nlow = (int)(n * Dk.q / Dk.p);
        int P, Q;
        rcos_edges(n, w[k], t[k], P, Q);
        if (!(2 * P <= nlow)) return where + ", too small for the pyramid's lowpass";
        n = nlow;
    }
    return "";
}

// src/transforms/surfacelet.jl:253-269
void surf_check_size(const sfl_surf_params& p, const int dims[3]) {
    for (int a = 1; a <= 3; ++a) {
        std::string problem = axis_problem(p, a, dims[a - 1]);
        if (problem.empty()) continue;
        int n = dims[a - 1];
        int near = 0;
        for (int d = 1; d <= 4 * n + 64 && near == 0; ++d) {
            for (int m : {n - d, n + d}) {
                if (m >= 1 && axis_problem(p, a, m).empty()) {
                    near = m;
                    break;
                }
            }
        }
        std::string hint = near > 0 ? "; the nearest length that fits is " + std::to_string(near) : "";
        throw ArgError("a volume of size " + fmt_dims(dims) + " does not fit Surfacelet(scales = " +
                       std::to_string(p.scales) + ", pyramid_ratio = " + fmt_ratio(p.pyramid_ratio) +
                       "): axis " + std::to_string(a) + ": " + problem + hint);
    }
}

// src/pyramid/fourier_pyramid.jl:181-216 (file numbering)
std::vector<PyrLevel> fourier_pyramid(const int dims[3], int J, double mode) {
    Rat w[2], t[2], D[2];
    surf_pyramid_mode(mode, w, t, D);
    std::vector<PyrLevel> out;
    int n[3] = {dims[0], dims[1], dims[2]};
    for (int j = 1; j <= J; ++j) {
        int k = j == 1 ? 0 : 1;
        PyrLevel lv;
        lv.D = D[k];
        for (int d = 0; d < 3; ++d) {
            if ((n[d] * D[k].q) % D[k].p != 0) {
                throw ArgError("a pyramid level with factor " + std::to_string(D[k].p) + "//" +
                               std::to_string(D[k].q) + " cannot divide size " + fmt_dims(n));
            }
        }
        for (int d = 0; d < 3; ++d) {
            lv.n[d] = n[d];
            lv.nlow[d] = (int)(n[d] * D[k].q / D[k].p);
        }
        for (int a = 0; a < 3; ++a) {
            int P;
            std::vector<double> full = rcos_axis(n[a], w[k], t[k], P);
            if (!(2 * P <= lv.nlow[a])) throw ArgError("size " + std::to_string(n[a]) + " is too small for the pyramid");
            for (int f = 0; f <= P; ++f) {
                lv.idx[a].push_back(f);
                lv.idx_low[a].push_back(f);
            }
            for (int f = n[a] - P; f < n[a]; ++f) lv.idx[a].push_back(f);
            for (int f = lv.nlow[a] - P; f < lv.nlow[a]; ++f) lv.idx_low[a].push_back(f);
            for (int f : lv.idx[a]) lv.prof[a].push_back(full[f]);
        }
        out.push_back(lv);
        for (int d = 0; d < 3; ++d) n[d] = lv.nlow[d];
    }
    return out;
}

// src/transforms/surfacelet.jl:275-290
std::vector<std::array<int, 3>> surf_layout_sizes(const sfl_surf_params& p, const int dims[3]) {
    surf_check_size(p, dims);
    std::vector<PyrLevel> pyr = fourier_pyramid(dims, p.scales, p.pyramid_ratio);
    std::vector<std::array<int, 3>> sizes;
    const PyrLevel& last = pyr.back();
    sizes.push_back({last.nlow[0], last.nlow[1], last.nlow[2]});
    for (int j = 1; j <= p.scales; ++j) {
        const int* n = pyr[p.scales - j].n;
        int lv[3][3];
        levels_of(p, j - 1, lv);
        for (int K = 0; K < 3; ++K) {
            int counts[3];
            for (int d = 0; d < 3; ++d) counts[d] = 1 << lv[K][d];
            for (int d = 0; d < 3; ++d)
                if (n[d] % counts[d] != 0)
                    throw ArgError("scale " + std::to_string(j) + " of size " + fmt_dims(n) +
                                   " cannot be split into " + fmt_dims(counts) + " wedge blocks in hourglass " +
                                   std::to_string(K + 1));
            std::array<int, 3> sb;
            for (int d = 0; d < 3; ++d) sb[d] = d == K ? n[K] : n[d] / counts[d];
            int cnt = counts[0] * counts[1] * counts[2];
            for (int c = 0; c < cnt; ++c) sizes.push_back(sb);
        }
    }
    return sizes;
}

// Modified Bessel I0 by SurfBox's truncated series: src/directional/ritf.jl:24-37
static double ritf_I0(double x) {
    x /= 2;
    double y = 1, z = 1, t = 1;
    int k = 1;
    while (t > 1.0e-10 * y) {
        z = z * x / k;
        k += 1;
        t = z * z;
        y += t;
    }
    return y;
}

static double sinc(double x) { return x == 0 ? 1.0 : std::sin(kPi * x) / (kPi * x); }

// src/directional/ritf.jl:40-52
static std::vector<double> ritf_window(int n, double beta) {
    double den = ritf_I0(beta);
    int half = (n - 1) / 2;
    std::vector<double> wh(half + 1);
    for (int i = 0; i <= half; ++i) {
        double v = 2.0 * i / (n - 1) - 1;
        wh[i] = ritf_I0(beta * std::sqrt(1 - v * v)) / den;
    }
    std::vector<double> w(n);
    for (int i = 0; i <= half; ++i) w[i] = wh[i];
    for (int i = 0; i < half; ++i) w[half + 1 + i] = wh[half - 1 - i];
    for (int i = 0; i < n; ++i) w[i] *= sinc((double)(i - half) / 2);
    return w;
}

// src/directional/ritf.jl:58-73
static double ritf_diamond(const std::vector<double>& w, double a, double b) {
    int half = ((int)w.size() - 1) / 2;
    double al = (a + b) / 2, be = (a - b) / 2;
    double cea = 0, ceb = 0, coa = 0, cob = 0;
    for (int i = 0; i < (int)w.size(); ++i) {
        int u = i - half;
        if (u % 2 == 0) {
            cea += w[i] * std::cos(u * al);
            ceb += w[i] * std::cos(u * be);
        } else {
            coa += w[i] * std::cos(u * al);
            cob += w[i] * std::cos(u * be);
        }
    }
    return cea * ceb + coa * cob;
}

// src/directional/ritf.jl:76-84: the planes D(w_K + pi, w_m)^lambda, m != K.
void ritf_planes(const int n[3], int msize, double beta, int lambda, std::vector<double> P[3][3]) {
    for (int d = 0; d < 3; ++d)
        if (n[d] % 2 != 0) throw ArgError("the hourglass stage needs even dimensions, got " + fmt_dims(n));
    std::vector<double> w = ritf_window(msize, beta);
    for (int K = 0; K < 3; ++K)
        for (int m = 0; m < 3; ++m) {
            P[K][m].clear();
            if (m == K) continue;
            int nK = n[K], nm = n[m];
            P[K][m].resize((size_t)nK * nm);
            for (int l = 0; l < nm; ++l)
                for (int k = 0; k < nK; ++k) {
                    double a = 2 * kPi * k / nK + kPi;
                    double b = 2 * kPi * l / nm;
                    P[K][m][k + (size_t)nK * l] = std::pow(ritf_diamond(w, a, b), lambda);
                }
        }
}

// src/directional/ritf.jl:89-108: V_K on the half-K grid.  The order of the
// operations is the device kernel's (dec_design.cu): h_K = P_a P_b (m
// ascending), tot = (h_1 + h_2) + h_3, V = sqrt((3 h_K) / tot).
void ritf_compose(const int n[3], const std::vector<double> P[3][3], std::vector<double> V[3]) {
    auto hg = [&](int K, int i0, int i1, int i2) {
        int idx[3] = {i0, i1, i2};
        double acc = 1.0;
        for (int m = 0; m < 3; ++m) {
            if (m == K) continue;
            acc *= P[K][m][idx[K] + (size_t)n[K] * idx[m]];
        }
        return acc;
    };
    for (int K = 0; K < 3; ++K) {
        int hd[3] = {n[0], n[1], n[2]};
        hd[K] = n[K] / 2 + 1;
        V[K].resize((size_t)hd[0] * hd[1] * hd[2]);
        for (int i2 = 0; i2 < hd[2]; ++i2)
            for (int i1 = 0; i1 < hd[1]; ++i1)
                for (int i0 = 0; i0 < hd[0]; ++i0) {
                    double h0 = hg(0, i0, i1, i2), h1 = hg(1, i0, i1, i2), h2 = hg(2, i0, i1, i2);
                    double tot = h0 + h1 + h2;
                    double hk = K == 0 ? h0 : (K == 1 ? h1 : h2);
                    V[K][i0 + (size_t)hd[0] * (i1 + (size_t)hd[1] * i2)] = std::sqrt(3 * hk / tot);
                }
    }
}

void ritf_masks(const int n[3], int msize, double beta, int lambda, std::vector<double> V[3]) {
    std::vector<double> P[3][3];
    ritf_planes(n, msize, beta, lambda, P);
    ritf_compose(n, P, V);
}

// Checkerboard responses: src/filters/checkerboard.jl:71-91
static double cbd_b(const std::vector<double>& t, double w) {
    double s = 0;
    for (size_t i = 0; i < t.size(); ++i) s += t[i] * std::sin((2.0 * (i + 1) - 1) * w);
    return 2 * s;
}

// src/directional/irc.jl:49-67 with the ladder responses of
// src/filters/checkerboard.jl:80-91: stage le on axis m of length nm splits
// it into groups of W = nm >> (le - 1) bins; bin c = g W + l has
// w_m = 2 pi l / W + sf_g w_K, sf_g = 2^(le-1) - 1 - 2g.
IRCFactors irc_factors(int nKh, int nK, int nm, int le, int bo) {
    const std::vector<double>& t = cbd_ladder(bo);
    IRCFactors F;
    F.nKh = nKh;
    F.nm = nm;
    F.W = nm >> (le - 1);
    F.ng = nm / F.W;
    F.nq = (int)t.size();
    F.t = t;
    F.r = 1 / std::sqrt(2.0);
    F.bK.resize(nKh);
    for (int k = 0; k < nKh; ++k) F.bK[k] = cbd_b(t, 2 * kPi * k / nK);
    F.sth.resize((size_t)F.nq * F.W);
    F.cth.resize((size_t)F.nq * F.W);
    for (int i = 0; i < F.nq; ++i)
        for (int l = 0; l < F.W; ++l) {
            const double th = (2.0 * (i + 1) - 1) * (2 * kPi * l / F.W);
            F.sth[(size_t)i * F.W + l] = std::sin(th);
            F.cth[(size_t)i * F.W + l] = std::cos(th);
        }
    F.sph.resize((size_t)F.nq * F.ng * nKh);
    F.cph.resize((size_t)F.nq * F.ng * nKh);
    for (int i = 0; i < F.nq; ++i)
        for (int g = 0; g < F.ng; ++g) {
            const int sf = (1 << (le - 1)) - 1 - 2 * g;
            for (int k = 0; k < nKh; ++k) {
                const double ph = (2.0 * (i + 1) - 1) * (sf * (2 * kPi * k / nK));
                F.sph[((size_t)i * F.ng + g) * nKh + k] = std::sin(ph);
                F.cph[((size_t)i * F.ng + g) * nKh + k] = std::cos(ph);
            }
        }
    return F;
}

// B = -b(w_K) b(w_m); analysis H0 = (1 + B)/sqrt2, H1 = e^{i w_m} (2 - B - B^2)/sqrt2,
// both x 0.5; synthesis G0 = (2 + B - B^2)/sqrt2, G1 = e^{-i w_m} (1 - B)/sqrt2.
// Every step below is one IEEE operation, in the order dec_design.cu uses.
void irc_slice_values(const IRCFactors& F, int k, int c, std::complex<double> out[4]) {
    const int g = c / F.W, l = c - g * F.W;
    double s = 0, sw = 0, cw = 0;
    for (int i = 0; i < F.nq; ++i) {
        const double st = F.sth[(size_t)i * F.W + l], ct = F.cth[(size_t)i * F.W + l];
        const size_t q = ((size_t)i * F.ng + g) * F.nKh + k;
        const double sp = F.sph[q], cp = F.cph[q];
        const double sq = st * cp + ct * sp;   // sin(q_i w_m)
        if (i == 0) {
            sw = sq;
            cw = ct * cp - st * sp;             // cos(w_m)
        }
        s = s + F.t[i] * sq;
    }
    const double bm = 2 * s;
    const double B = -F.bK[k] * bm;
    const double B2 = B * B;
    const double h0 = F.r * (1 + B);
    const double h1 = F.r * ((2 - B) - B2);
    const double g0 = F.r * ((2 + B) - B2);
    const double g1 = F.r * (1 - B);
    out[0] = {0.5 * h0, 0.0};
    out[1] = {0.5 * (cw * h1), 0.5 * (sw * h1)};
    out[2] = {g0, 0.0};
    out[3] = {cw * g1, -(sw * g1)};
}

// src/directional/irc.jl:76-91: the stages of hourglass K, axes m ascending.
std::vector<IRCStage> irc_stages(const int hdims[3], int nK, int K, const int levels[3], int bo, bool values) {
    std::vector<IRCStage> out;
    for (int m = 1; m <= 3; ++m) {
        if (m == K) continue;
        int lv = levels[m - 1];
        if (lv < 0) throw ArgError("directional levels must be ≥ 0");
        if (hdims[m - 1] % (1 << lv) != 0)
            throw ArgError("axis " + std::to_string(m) + " of length " + std::to_string(hdims[m - 1]) +
                           " cannot be split " + std::to_string(lv) + " times");
        for (int le = 1; le <= lv; ++le) {
            IRCStage st;
            st.m = m;
            st.b = hdims[m - 1] >> le;
            const int nKh = hdims[K - 1], nm = hdims[m - 1];
            st.fac = irc_factors(nKh, nK, nm, le, bo);
            if (values) {
                for (int c = 0; c < 2; ++c) {
                    st.ana[c].resize((size_t)nKh * nm);
                    st.syn[c].resize((size_t)nKh * nm);
                }
                for (int cc = 0; cc < nm; ++cc)
                    for (int k = 0; k < nKh; ++k) {
                        std::complex<double> v[4];
                        irc_slice_values(st.fac, k, cc, v);
                        const size_t e = k + (size_t)nKh * cc;
                        st.ana[0][e] = v[0];
                        st.ana[1][e] = v[1];
                        st.syn[0][e] = v[2];
                        st.syn[1][e] = v[3];
                    }
            }
            out.push_back(std::move(st));
        }
    }
    return out;
}

// src/transforms/surfacelet.jl:73-102, 136-149
SurfDesign surf_design(const sfl_surf_params& p, const int dims[3], bool tables) {
    surf_check_params(p);
    SurfDesign S;
    for (int d = 0; d < 3; ++d) S.dims[d] = dims[d];
    S.p = p;
    S.sizes = surf_layout_sizes(p, dims);
    S.pyramid = fourier_pyramid(dims, p.scales, p.pyramid_ratio);
    int J = p.scales;
    for (int j = 1; j <= J; ++j) {
        ScaleDesign sc;
        for (int d = 0; d < 3; ++d) sc.n[d] = S.pyramid[j - 1].n[d];
        levels_of(p, J - j, sc.lv);
        ritf_planes(sc.n, p.diamond_length, p.kaiser_beta, p.diamond_power, sc.P);
        if (tables) ritf_compose(sc.n, sc.P, sc.V);
        for (int K = 1; K <= 3; ++K) {
            int hd[3] = {sc.n[0], sc.n[1], sc.n[2]};
            hd[K - 1] = sc.n[K - 1] / 2 + 1;
            sc.stages[K - 1] = irc_stages(hd, sc.n[K - 1], K, sc.lv[K - 1], p.checkerboard_order, tables);
        }
        S.scales.push_back(std::move(sc));
    }
    S.offsets.assign(S.sizes.size() + 1, 0);
    for (size_t i = 0; i < S.sizes.size(); ++i)
        S.offsets[i + 1] = S.offsets[i] + (int64_t)S.sizes[i][0] * S.sizes[i][1] * S.sizes[i][2];
    std::vector<int> counts;
    for (int j = 0; j < J; ++j) counts.push_back(surf_nsubbands_scale(S.scales[j].lv));
    S.level_first.resize(J);
    for (int j = 0; j < J; ++j) {
        int s = 1;
        for (int k = j + 1; k < J; ++k) s += counts[k];
        S.level_first[j] = s;
    }
    return S;
}

}  // namespace sfl
