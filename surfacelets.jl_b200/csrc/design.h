// Float64 design of every table the kernels read: the NSSurfacelet hourglass
// responses, wedge planes and pyramid factors, and the decimated transform's
// pyramid profiles, ritf hourglass masks and checkerboard (IRC) filter slices.
// Also the parameter and size rules of both transforms, with the reference's
// error messages.  Host-only C++; no CUDA.
#pragma once

#include <array>
#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/surfacelets_b200.h"

namespace sfl {

// Errors that map to the reference's ArgumentError / DimensionMismatch.
struct ArgError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct DimError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// Exact rationals for the pyramid edges (the reference uses Julia Rationals).
struct Rat {
    long long p, q;
};

std::string fmt_dims(const int d[3]);

// ── Filter design (src/filters/bernstein.jl, src/pyramid/fourier_pyramid.jl) ──
std::vector<double> dft_frequencies(int n, bool half);
std::vector<double> folded_frequencies(int n, bool half);
// (N+1) x m table, entry [j + (N+1)*k].
std::vector<double> bernstein_table(int N, const std::vector<double>& omega);
double halfband_split(double x, int m);
double soft_step(double s, double b, double w, int poly);
void rcos_edges(int n, Rat w, Rat t, int& P, int& Q);
std::vector<double> rcos_axis(int n, Rat w, Rat t, int& P);

// ── NSSurfacelet ──────────────────────────────────────────────────────────────

// One wedge plane set: the 2^l planes of hourglass i along transverse axis tr,
// each indexed (lo axis, hi axis) of the two axes it depends on, lo fastest.
struct WedgePlanes {
    int ref = 0, tr = 0;        // 1-based axes
    int lo = 0, hi = 0;         // 1-based axes, lo < hi
    int dlo = 0, dhi = 0;       // plane extents (axis 1 is the half grid)
    std::vector<std::vector<double>> w;
};

// The separable parts of the hourglass tables: Bernstein tables of axes 2
// and 3 ((order + 1) x n), the mapping kernel contracted along axis 1
// (t1[j2, j3, k1]) and m2.
struct NSHourglassFactors {
    int np = 0;
    std::vector<double> t1, b2, b3, m2;
};

struct NSDesign {
    int dims[3] = {0, 0, 0};
    int h1 = 0;
    sfl_ns_params p{};
    NSHourglassFactors hg;
    std::vector<double> m1;   // f0(M1) on (h1, n2, n3), column-major (ns_design_fill_m1; empty until then)
    std::vector<double> m2;   // f0(M2) on (n2, n3)
    // wedges[j][i][plane]: scale j (coarse first), hourglass i, plane a/b;
    // square-rooted when tight.
    std::vector<std::array<std::array<WedgePlanes, 2>, 3>> wedges;
    // Per pyramid level (0 = finest) and axis, on that axis's rfft bins:
    // pa[lv] = prod_{i<lv} l_i (J+1 levels), pl[lv] = l_lv (J levels).
    std::vector<std::array<std::vector<double>, 3>> pa, pl;
};

// Group mask of hourglass i (1..3) at pyramid level lv on the rfft grid:
// B_lv * sqrt(max(W_i, 0)) when tight, B_lv * W_i otherwise; with
// hourglass = false, B_lv alone.  Float64 throughout: in float32 the
// cancellations in 1 - (l1 l2 l3)^2 and 1 - f0 cost up to 1.5e-4 absolute
// after the square root.
std::vector<double> ns_group_mask(const NSDesign& D, int lv, int i, bool hourglass);

void ns_check_params(const sfl_ns_params& p);
void ns_check_size(const sfl_ns_params& p, const int dims[3]);
int ns_nbands(const sfl_ns_params& p, int j);      // scale j 1-based
int ns_nsubbands(const sfl_ns_params& p);
// pyramid = false: the standalone directional bank (no pyramid, no size rule).
// with_m1 = false leaves m1 to the device design (ns_design.cu) or to
// ns_design_fill_m1.
NSDesign ns_design(const sfl_ns_params& p, const int dims[3], bool pyramid = true, bool with_m1 = true);
NSHourglassFactors ns_hourglass_factors(const int dims[3], int order, int poly);
void ns_design_fill_m1(NSDesign& D);
std::vector<double> ns_hourglass_mask(const NSDesign& D, int i);

// ── Decimated Surfacelet ──────────────────────────────────────────────────────

struct PyrLevel {
    int n[3], nlow[3];
    Rat D;
    std::vector<int> idx[3], idx_low[3];
    std::vector<double> prof[3];
};

// The separable factors of one IRC stage's filter slices
// (src/directional/irc.jl:49-67, the ladder filters of
// src/filters/checkerboard.jl:71-91): b(w) = 2 sum_i t_i sin(q_i w), q_i =
// 2i + 1, at w_K = 2 pi k / n_K and at w_m = theta_l + phi_{g,k} with
// theta_l = 2 pi l / W and phi_{g,k} = sf_g w_K.  sin(q_i w_m) and cos(w_m)
// come from these 1-D tables by angle addition, so every later step is an
// exact IEEE multiply or add: the host (irc_slice_values) and the device
// (dec_design.cu) give the same float64 values bit for bit.
struct IRCFactors {
    int nKh = 0, nm = 0, W = 0, ng = 0, nq = 0;
    double r = 0;                    // 1/sqrt(2)
    std::vector<double> t;           // ladder taps t_i
    std::vector<double> bK;          // b(w_K), k < nKh
    std::vector<double> sth, cth;    // sin, cos(q_i theta_l): [i * W + l]
    std::vector<double> sph, cph;    // sin, cos(q_i phi_{g,k}): [(i * ng + g) * nKh + k]
};

struct IRCStage {
    int m = 0;      // 1-based axis decimated
    int b = 0;      // block size after the stage
    IRCFactors fac;
    // (K-half, m) planes, entry [k + nKh * c]: analysis channel 0/1 (x 0.5),
    // synthesis channel 0/1 (filled only when the host tables are asked for).
    std::vector<std::complex<double>> ana[2], syn[2];
};

struct ScaleDesign {
    int n[3];
    int lv[3][3];                  // [K][m]
    std::vector<double> P[3][3];   // ritf diamond planes [K][m] (n_K x n_m, k fastest), m != K
    std::vector<double> V[3];      // V_K on the half-K grid, column-major (host tables only)
    std::vector<IRCStage> stages[3];
};

struct SurfDesign {
    int dims[3];
    sfl_surf_params p{};
    std::vector<PyrLevel> pyramid;       // finest first
    std::vector<ScaleDesign> scales;     // per pyramid level, finest first
    std::vector<std::array<int, 3>> sizes;   // subband sizes, layout order
    std::vector<int64_t> offsets;        // element offsets (size nsub + 1)
    std::vector<int> level_first;        // [level] 0-based index of its first subband
};

void surf_levels_from_int(int L, int out[3][3]);
void surf_check_params(const sfl_surf_params& p);
void surf_pyramid_mode(double mode, Rat w[2], Rat t[2], Rat D[2]);
void surf_check_size(const sfl_surf_params& p, const int dims[3]);
std::vector<std::array<int, 3>> surf_layout_sizes(const sfl_surf_params& p, const int dims[3]);
int surf_nsubbands_scale(const int lv[3][3]);
std::vector<PyrLevel> fourier_pyramid(const int dims[3], int J, double mode);
// The 2-D factors of the ritf masks: P[K][m] = D(w_K + pi, w_m)^lambda on
// (n_K, n_m), m != K (src/directional/ritf.jl:58-84).
void ritf_planes(const int n[3], int msize, double beta, int lambda, std::vector<double> P[3][3]);
// V_K = sqrt(3 h_K / (h_1 + h_2 + h_3)), h_K the product of P[K][m] over m != K
// (src/directional/ritf.jl:89-108), from the planes.
void ritf_compose(const int n[3], const std::vector<double> P[3][3], std::vector<double> V[3]);
void ritf_masks(const int n[3], int msize, double beta, int lambda, std::vector<double> V[3]);
IRCFactors irc_factors(int nKh, int nK, int nm, int le, int bo);
// Slice values at (k, c): analysis channel 0/1 (x 0.5), synthesis channel 0/1.
void irc_slice_values(const IRCFactors& F, int k, int c, std::complex<double> out[4]);
std::vector<IRCStage> irc_stages(const int hdims[3], int nK, int K, const int levels[3], int bo, bool values = true);
// tables = false: the pyramid, layout, ritf planes and IRC factors only (the
// device composes V_K and the slices from them, dec_design.cu).
SurfDesign surf_design(const sfl_surf_params& p, const int dims[3], bool tables = true);

}  // namespace sfl
