// Internal types shared by the host planner (plan.cpp), the CUDA kernels
// (kernels.cu) and the C ABI (api.cu).
//
// Storage model.  The reference evolves the nodal state (mode, field, r,
// theta) and projects every RHS field back onto its fixed-(s,m) band
// (include/teuk/spatial_pipeline.hpp:756-766), so an accepted state is always
// S_m * c for band coefficients c (S_m = synthesis matrix).  This engine
// keeps exactly those band coefficients: for every parent mode m a
// "segment" of nr rows, each row holding the three evolved fields
// (P, Q, psi) x n_ell(m) complex modal values.  Radial SBP operators act on
// each ell column (they commute with the angular transforms), the angular
// Laplacian is diagonal, and the only theta coupling left -- the Kerr
// C_T(theta) and i s a cos(theta) factors of psi_t -- is applied as
// analysis * diag(.) * synthesis on the Gauss-Legendre nodes, i.e. the
// reference's own quadrature.  Fields that the linear pipeline freezes
// (include/teuk/spatial_pipeline.hpp:623-649) are kept on the host.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace teuk_b200 {

inline constexpr int kFieldCount = 13;
inline constexpr int kEvolvedFields = 3;  // P, Q, psi
inline constexpr int kMaxEll = 64;        // per-row modal values
inline constexpr int kMaxTheta = 96;      // Gauss-Legendre nodes
inline constexpr int kSpinWeight = -2;

enum Disc : int { kD42 = 0, kD84 = 1, kD105 = 2 };

// Per-discretization geometry (include/teuk/sbp*.hpp).
struct DiscInfo {
  int boundary_rows;   // closure rows (4, 8, 11)
  int boundary_width;  // closure stencil columns (6, 12, 16)
  int interior_half;   // interior stencil half width (2, 4, 5)
  int diss_order;      // undivided difference order p (3, 5, 6)
  int norm_rows;       // rows with a non-unit norm weight (4, 8, 11)
  int min_points;      // radial_minimum_points (8, 16, 22)
};
DiscInfo disc_info(int disc);

// ---------------------------------------------------------------- device
// descriptors (plain structs copied to the device)
struct InstanceDesc {
  double mass;
  double spin;
  double length;       // compactification length L
  double spacing;      // h
  double inv_spacing;  // 1/h
  double damping;      // reduction damping (FreeDamped) or 0
  double dissipation;  // sigma
  double dt;
  int nr;
  int ntheta;
  int trig_offset;  // doubles into the trig pool: sin(theta)[nt], cos(theta)[nt]
  int reduction;    // 0 free damped, 1 stage constrained
  int disc;
  int coef_row0;    // first row of this solve in the coefficient table
  int wide_row0;    // first row in the wide node table (-1: no wide bands)
};

struct SegmentDesc {
  long long offset;  // complex offset of row 0 in each state buffer
  int instance;
  int m;
  int n_ell;
  int ell_min;
  int mat_offset;    // doubles into the matrix pool: St[n_ell][nt], At[nt][n_ell]
  int row_stride;    // complex values per row = 3 * n_ell
};

struct TileDesc {
  int segment;
  int r0;
  int r1;
  int pad;
};

// Coefficient tables in __constant__ memory (host-built, binary64 exact as
// the reference evaluates its rational literals).
struct SbpConstants {
  // h*D closure rows, left side: [disc][row][column]
  double left[3][11][16];
  // interior stencil c_k, k = 1..half (antisymmetric): [disc][k]
  double interior[3][6];
  // dissipation: -(A^T A)_ij / H_ii for the special left rows
  // [disc][row][column], row < 11, column < 18; interior symmetric stencil
  // -C(k), k = 0..p
  double diss_left[3][11][18];
  double diss_interior[3][7];
};

// ---------------------------------------------------------------- host plan
struct Config {
  double mass = 1.0;
  double spin = 0.0;
  double length = 1.0;
  int nr = 0;
  int ntheta = 0;
  int ell_max_first = 0;
  int ell_max_second = 0;
  std::vector<int> modes;    // sorted, unique
  std::vector<int> parents;  // sorted, unique
  std::vector<int> targets;  // sorted, unique
  double damping = 0.1;
  double dissipation = 0.0;
  int reduction = 0;
  int disc = kD42;
  int source_mode = 0;
  double source_start_time = 0.0;
  double constraint_tolerance = 0.0;
  int required_passes = 1;
};

struct ModePlan {
  int m = 0;
  int mode_index = 0;  // position in the sorted registry
  bool parent = false;
  int ell_min = 0;
  int n_ell = 0;
  std::vector<double> synthesis;  // [nt][n_ell]
  std::vector<double> analysis;   // [n_ell][nt]
  long long segment = -1;         // segment id in the batch (parents only)
};

struct InstancePlan {
  Config config;
  double horizon = 0.0;  // R_H = L^2 / r_+
  double spacing = 0.0;
  std::vector<double> x, weights, theta, sinv, cosv;
  std::vector<ModePlan> modes;  // registry order
  // activation latch (SourceActivationState)
  int active = 0;
  double activation_time = -1.0;
  int consecutive_passes = 0;
  double last_eligibility_time = -1.0;
  std::size_t value_count() const {
    return config.modes.size() * static_cast<std::size_t>(kFieldCount) *
           static_cast<std::size_t>(config.nr) *
           static_cast<std::size_t>(config.ntheta);
  }
};

// Validates like the reference constructor and builds the angular plans.
// Throws std::invalid_argument / std::runtime_error with the reference's
// messages.
InstancePlan build_instance_plan(const Config& config);

// Reference-identical host math (include/teuk/angular.hpp).
void gauss_legendre(int nodes, std::vector<double>& x,
                    std::vector<double>& weights);
double spin_weighted_harmonic_theta(int ell, int m, int spin, double theta);
double outer_horizon_radius(double mass, double spin);
SbpConstants build_sbp_constants();
// Diagonal SBP norm weight H_ii / h (include/teuk/radial_discretization.hpp).
double sbp_norm_weight(int disc, int n, int index);
// Dense h*D row for host-side use (initial data): value of the SBP first
// derivative of `line` (stride 2 doubles for complex parts) at `row`.
void sbp_derivative_line(int disc, const double* line_re_im, int n,
                         double inv_spacing, double* out_re_im);

// Teukolsky point coefficients (include/teuk/teukolsky.hpp:38-85), split into
// theta-independent parts and the theta-dependent pieces.
struct RowCoefficients {
  double c0;      // C_T without the -a^2 sin^2 theta term
  double K;       // radial advection
  double HR;      // radial principal
  double g_re;    // Re G_m (theta independent)
  double g_im_m;  // Im G_m without the 2 s a cos(theta) term
  double q_re, q_im;
  double c_re, c_im;  // psi coefficient
};

// Checks of initialize_compactified_gaussian_pulse
// (include/teuk/pipeline_initial_data.hpp:211-250) with its messages.
void validate_gaussian(const InstancePlan& plan, double center, double width,
                       const std::vector<int>& ell,
                       const std::vector<int>& m_values);
// Radial profile of the pulse at R (Gaussian, or the compact bump).
double gaussian_profile(double R, double center, double width,
                        bool compact_support);

// Gaussian initial data of one instance, nodal (m,13,r,theta) host array in
// the reference's order; returns the Galerkin residual.
double gaussian_initial_state(const InstancePlan& plan, double center,
                              double width, bool compact_support,
                              const std::vector<int>& ell,
                              const std::vector<int>& m,
                              const std::vector<double>& amp_re,
                              const std::vector<double>& amp_im,
                              std::vector<double>& nodal);

}  // namespace teuk_b200
