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

struct IRCStage {
    int m = 0;      // 1-based axis decimated
    int b = 0;      // block size after the stage
    // (K-half, m) planes, entry [k + nKh * c]: analysis channel 0/1 (x 0.5),
    // synthesis channel 0/1.
    std::vector<std::complex<double>> ana[2], syn[2];
};

struct ScaleDesign {
    int n[3];
    int lv[3][3];                  // [K][m]
    std::vector<double> V[3];      // V_K on the half-K grid, column-major
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
void ritf_masks(const int n[3], int msize, double beta, int lambda, std::vector<double> V[3]);
std::vector<IRCStage> irc_stages(const int hdims[3], int nK, int K, const int levels[3], int bo);
SurfDesign surf_design(const sfl_surf_params& p, const int dims[3]);

}  // namespace sfl
