// Host-side planning for the B200 engine: reference-identical angular
// matrices, SBP coefficient tables, construction-time validation and the
// Gaussian / Galerkin initial data.  Everything here runs once per solve at
// set-up; nothing here runs inside a time step.
#include <algorithm>
#include <cmath>
#include <limits>
#include <numbers>
#include <stdexcept>
#include <string>
#include <utility>

#include "engine.h"
#include "sbp_tables.h"

namespace teuk_b200 {

DiscInfo disc_info(const int disc) {
  switch (disc) {
    case kD42: return {4, 6, 2, 3, 4, 8};
    case kD84: return {8, 12, 4, 5, 8, 16};
    case kD105: return {11, 16, 5, 6, 11, 22};
  }
  throw std::invalid_argument("unknown radial discretization");
}

// ------------------------------------------------------------------ angular
// Gauss-Legendre nodes by Newton iteration on P_n in long double, the
// procedure of include/teuk/angular.hpp:69-115 (same start values, update,
// stopping rule and weight formula) so node and weight bits agree.
namespace {

std::pair<long double, long double> legendre_pair(const int degree,
                                                  const long double x) {
  long double previous = 1.0L;
  if (degree == 0) return {previous, 0.0L};
  long double current = x;
  for (int ell = 2; ell <= degree; ++ell) {
    const long double next =
        ((2.0L * ell - 1.0L) * x * current - (ell - 1.0L) * previous) / ell;
    previous = current;
    current = next;
  }
  return {current, previous};
}

long double power_ld(long double base, int exponent) {
  long double result = 1.0L;
  while (exponent != 0) {
    if ((exponent & 1) != 0) result *= base;
    base *= base;
    exponent >>= 1;
  }
  return result;
}

long double log_factorial(const int n) {
  return std::lgammal(static_cast<long double>(n) + 1.0L);
}

// Wigner small-d, Condon-Shortley phase, as the long-double factorial sum of
// include/teuk/angular.hpp:170-206.
double wigner_d(const int ell, const int m_prime, const int m,
                const double theta) {
  const int k_min = std::max(0, m - m_prime);
  const int k_max = std::min(ell + m, ell - m_prime);
  const long double log_norm =
      0.5L * (log_factorial(ell + m) + log_factorial(ell - m) +
              log_factorial(ell + m_prime) + log_factorial(ell - m_prime));
  const long double c = std::cos(0.5L * static_cast<long double>(theta));
  const long double s = std::sin(0.5L * static_cast<long double>(theta));
  long double value = 0.0L;
  for (int k = k_min; k <= k_max; ++k) {
    const long double log_coefficient =
        log_norm - log_factorial(ell + m - k) - log_factorial(k) -
        log_factorial(m_prime - m + k) - log_factorial(ell - m_prime - k);
    long double term = std::exp(log_coefficient) *
                       power_ld(c, 2 * ell + m - m_prime - 2 * k) *
                       power_ld(s, m_prime - m + 2 * k);
    if (((m_prime - m + k) & 1) != 0) term = -term;
    value += term;
  }
  return static_cast<double>(value);
}

}  // namespace

void gauss_legendre(const int nodes, std::vector<double>& x,
                    std::vector<double>& weights) {
  if (nodes <= 0) {
    throw std::invalid_argument("Gauss-Legendre node count must be positive");
  }
  x.assign(static_cast<std::size_t>(nodes), 0.0);
  weights.assign(static_cast<std::size_t>(nodes), 0.0);
  const int half = (nodes + 1) / 2;
  const long double tolerance =
      8.0L * std::numeric_limits<long double>::epsilon();
  for (int i = 0; i < half; ++i) {
    long double root = std::cos(std::numbers::pi_v<long double> *
                                (i + 0.75L) / (nodes + 0.5L));
    long double derivative = 0.0L;
    for (int iteration = 0; iteration < 100; ++iteration) {
      const auto [pn, pm] = legendre_pair(nodes, root);
      derivative = nodes * (root * pn - pm) / (root * root - 1.0L);
      const long double update = pn / derivative;
      root -= update;
      if (std::abs(update) <= tolerance * (1.0L + std::abs(root))) break;
      if (iteration == 99) {
        throw std::runtime_error("Gauss-Legendre root iteration failed");
      }
    }
    const auto [pn, pm] = legendre_pair(nodes, root);
    derivative = nodes * (root * pn - pm) / (root * root - 1.0L);
    const long double weight =
        2.0L / ((1.0L - root * root) * derivative * derivative);
    const auto low = static_cast<std::size_t>(i);
    const auto high = static_cast<std::size_t>(nodes - 1 - i);
    x[low] = static_cast<double>(-root);
    x[high] = static_cast<double>(root);
    weights[low] = static_cast<double>(weight);
    weights[high] = static_cast<double>(weight);
  }
}

double spin_weighted_harmonic_theta(const int ell, const int m,
                                    const int spin, const double theta) {
  if (ell < 0 || std::abs(spin) > ell || std::abs(m) > ell) {
    throw std::invalid_argument("spin-weighted mode requires ell >= |s|,|m|");
  }
  const double phase = (std::abs(spin) & 1) != 0 ? -1.0 : 1.0;
  return phase *
         std::sqrt((2.0 * ell + 1.0) / (4.0 * std::numbers::pi_v<double>)) *
         wigner_d(ell, m, -spin, theta);
}

double outer_horizon_radius(const double mass, const double spin) {
  return mass + std::sqrt(mass * mass - spin * spin);
}

// ---------------------------------------------------------------- SBP tables
namespace {

double rational(const teuk_sbp_rational r) { return r.num / r.den; }

// Interior antisymmetric stencil c_k (k = 1..half) of h*D.
void interior_stencil(const int disc, double* c) {
  switch (disc) {
    case kD42:
      c[1] = 2.0 / 3.0;
      c[2] = -1.0 / 12.0;
      break;
    case kD84:
      c[1] = 4.0 / 5.0;
      c[2] = -1.0 / 5.0;
      c[3] = 4.0 / 105.0;
      c[4] = -1.0 / 280.0;
      break;
    case kD105:
      c[1] = 5.0 / 6.0;
      c[2] = -5.0 / 21.0;
      c[3] = 5.0 / 84.0;
      c[4] = -5.0 / 504.0;
      c[5] = 1.0 / 1260.0;
      break;
  }
}

double norm_weight(const int disc, const int n, const int index) {
  const int distance = std::min(index, n - 1 - index);
  switch (disc) {
    case kD42: return distance < 4 ? rational(teuk_d42_norm[distance]) : 1.0;
    case kD84: return distance < 8 ? rational(teuk_d84_norm[distance]) : 1.0;
    case kD105:
      return distance < 11 ? rational(teuk_d105_norm[distance]) : 1.0;
  }
  return 1.0;
}

// Left closure coefficient of h*D (row < boundary_rows, column < width).
double left_coefficient(const int disc, const int row, const int column) {
  switch (disc) {
    case kD42: return rational(teuk_d42_left[row][column]);
    case kD84: return rational(teuk_d84_left[row][column]);
    case kD105: {
      double q = 0.0;
      if (column < 11) {
        q = rational(teuk_d105_left_q[row][column]);
      } else {
        // Columns 11..15 of the closure block follow the centred interior
        // row (skew symmetry of Q).
        const int offset = column - row;
        static const teuk_sbp_rational interior[6] = {
            {0.0, 1.0},  {5.0, 6.0},    {-5.0, 21.0},
            {5.0, 84.0}, {-5.0, 504.0}, {1.0, 1260.0}};
        if (offset >= 1 && offset <= 5) q = rational(interior[offset]);
      }
      // D10-5 closure rows are Q(row, :) / H(row) with H taken at the
      // minimum grid size (22) exactly as the reference normalises them.
      return q / rational(teuk_d105_norm[row]);
    }
  }
  return 0.0;
}

const int binomial_difference[3][7] = {
    {-1, 3, -3, 1, 0, 0, 0},
    {-1, 5, -10, 10, -5, 1, 0},
    {1, -6, 15, -20, 15, -6, 1},
};

}  // namespace

double sbp_norm_weight(const int disc, const int n, const int index) {
  return norm_weight(disc, n, index);
}

SbpConstants build_sbp_constants() {
  SbpConstants c{};
  for (int disc = 0; disc < 3; ++disc) {
    const DiscInfo info = disc_info(disc);
    for (int row = 0; row < info.boundary_rows; ++row) {
      for (int column = 0; column < info.boundary_width; ++column) {
        c.left[disc][row][column] = left_coefficient(disc, row, column);
      }
    }
    interior_stencil(disc, c.interior[disc]);
    // Dissipation Q = -(sigma/h) H^-1 A^T A with A the undivided p-th
    // difference (include/teuk/radial_discretization.hpp:163-234).  Rows
    // below max(p, norm_rows) are tabulated for a grid long enough that
    // the right closure does not reach them; the rest use the symmetric
    // interior stencil -C(k).
    const int p = info.diss_order;
    const int* b = binomial_difference[disc];
    const int special = std::max(p, info.norm_rows);
    const int n_model = 64;
    for (int i = 0; i < special; ++i) {
      const double w = norm_weight(disc, n_model, i);
      for (int j = 0; j <= i + p && j < 18; ++j) {
        double sum = 0.0;
        const int first = std::max(0, i - p);
        for (int row = first; row <= i; ++row) {
          const int alpha = i - row;
          const int beta = j - row;
          if (beta >= 0 && beta <= p) sum += b[alpha] * b[beta];
        }
        c.diss_left[disc][i][j] = -sum / w;
      }
    }
    for (int k = 0; k <= p; ++k) {
      double sum = 0.0;
      for (int alpha = 0; alpha + k <= p; ++alpha) {
        sum += b[alpha] * b[alpha + k];
      }
      c.diss_interior[disc][k] = -sum;
    }
  }
  return c;
}

void sbp_derivative_line(const int disc, const double* line, const int n,
                         const double inv_spacing, double* out) {
  const DiscInfo info = disc_info(disc);
  double interior[6] = {0, 0, 0, 0, 0, 0};
  interior_stencil(disc, interior);
  for (int row = 0; row < n; ++row) {
    for (int part = 0; part < 2; ++part) {
      double result = 0.0;
      if (row < info.boundary_rows) {
        for (int column = 0; column < info.boundary_width; ++column) {
          result += left_coefficient(disc, row, column) *
                    line[2 * column + part];
        }
      } else if (row + info.boundary_rows >= n) {
        const int reflected = n - 1 - row;
        for (int column = 0; column < info.boundary_width; ++column) {
          result -= left_coefficient(disc, reflected, column) *
                    line[2 * (n - 1 - column) + part];
        }
      } else {
        for (int k = info.interior_half; k >= 1; --k) {
          result += interior[k] *
                    (line[2 * (row + k) + part] - line[2 * (row - k) + part]);
        }
      }
      out[2 * row + part] = inv_spacing * result;
    }
  }
}

// ---------------------------------------------------------------- validation
namespace {

std::vector<int> sorted_unique(std::vector<int> values, const char* what) {
  std::sort(values.begin(), values.end());
  if (std::adjacent_find(values.begin(), values.end()) != values.end()) {
    throw std::invalid_argument(std::string("duplicate ") + what);
  }
  return values;
}

bool contains(const std::vector<int>& sorted, const int value) {
  return std::binary_search(sorted.begin(), sorted.end(), value);
}

}  // namespace

InstancePlan build_instance_plan(const Config& input) {
  InstancePlan plan;
  Config& c = plan.config;
  c = input;
  // ModeRegistry (include/teuk/modes.hpp:42-80)
  c.modes = sorted_unique(c.modes, "mode");
  c.parents = sorted_unique(c.parents, "parent mode");
  c.targets = sorted_unique(c.targets, "target mode");
  if (c.modes.empty()) {
    throw std::invalid_argument("ModeRegistry requires at least one mode");
  }
  if (c.targets.empty()) {
    throw std::invalid_argument(
        "ModeRegistry requires at least one target mode");
  }
  if (c.parents.empty()) {
    throw std::invalid_argument(
        "ModeRegistry requires at least one parent mode");
  }
  for (const int p : c.parents) {
    if (!contains(c.modes, p)) {
      throw std::invalid_argument("parent mode " + std::to_string(p) +
                                  " is not stored");
    }
  }
  for (const int t : c.targets) {
    if (!contains(c.modes, t)) {
      throw std::invalid_argument("target mode " + std::to_string(t) +
                                  " is not stored");
    }
  }
  // SpatialPipelineStorage (include/teuk/pipeline_storage.hpp:56-79)
  for (const int m : c.modes) {
    if (m == std::numeric_limits<int>::min() || !contains(c.modes, -m)) {
      throw std::invalid_argument(
          "spatial pipeline modes must be closed under m -> -m");
    }
  }
  if (!(c.mass > 0.0) || !std::isfinite(c.mass) || !std::isfinite(c.spin) ||
      std::abs(c.spin) > c.mass || !(c.length > 0.0) ||
      !std::isfinite(c.length)) {
    throw std::invalid_argument("Kerr parameters are invalid");
  }
  if (c.disc < 0 || c.disc > 2) {
    throw std::invalid_argument("unknown radial discretization");
  }
  if (c.reduction != 0 && c.reduction != 1) {
    throw std::invalid_argument("unsupported reduction mode");
  }
  // UniformRadialGrid (include/teuk/grid.hpp:15-29)
  if (c.nr < 5) {
    throw std::invalid_argument(
        "fourth-order radial differences require at least five points");
  }
  plan.horizon = c.length * c.length / outer_horizon_radius(c.mass, c.spin);
  if (!(plan.horizon > 0.0)) {
    throw std::invalid_argument(
        "radial grid upper bound must exceed its lower bound");
  }
  plan.spacing = (plan.horizon - 0.0) / static_cast<double>(c.nr - 1);
  // SpatialPipeline constructor (include/teuk/spatial_pipeline.hpp:315-343)
  const int exact_product_nodes =
      (2 * c.ell_max_first + c.ell_max_second + 2) / 2;
  if (c.nr < disc_info(c.disc).min_points) {
    throw std::invalid_argument(
        "full pipeline radial grid is too small for selected discretization");
  }
  if (c.ell_max_first < 3 || c.ell_max_second < 3 ||
      c.ntheta < std::max({c.ell_max_first + 1, c.ell_max_second + 1,
                           exact_product_nodes})) {
    throw std::invalid_argument(
        "full pipeline angular bands require exact-product padding");
  }
  if (c.ntheta > kMaxTheta) {
    throw std::invalid_argument("theta node count exceeds the engine limit");
  }
  if (!(c.dissipation >= 0.0) || !std::isfinite(c.dissipation)) {
    throw std::invalid_argument("pipeline dissipation must be nonnegative");
  }
  if (!std::isfinite(c.damping)) {
    throw std::invalid_argument("reduction damping must be finite");
  }
  if (!std::isfinite(c.source_start_time) || c.source_start_time < 0.0 ||
      !std::isfinite(c.constraint_tolerance) ||
      c.constraint_tolerance < 0.0 || c.required_passes < 1) {
    throw std::invalid_argument("pipeline source policy is invalid");
  }
  // SignedModeAngularCoordinator (include/teuk/angular_coordinator.hpp:75-88)
  for (const int m : c.parents) {
    if (std::abs(m) > c.ell_max_first) {
      throw std::invalid_argument(
          "angular coordinator active mode is outside its stored band");
    }
  }
  for (const int m : c.targets) {
    if (std::abs(m) > c.ell_max_second) {
      throw std::invalid_argument(
          "angular coordinator active mode is outside its stored band");
    }
  }

  gauss_legendre(c.ntheta, plan.x, plan.weights);
  const std::size_t nt = static_cast<std::size_t>(c.ntheta);
  plan.theta.resize(nt);
  plan.sinv.resize(nt);
  plan.cosv.resize(nt);
  for (std::size_t j = 0; j < nt; ++j) {
    plan.theta[j] = std::acos(plan.x[j]);
    // sin(theta) itself; the kernel forms a^2 sin(theta) sin(theta) in the
    // reference's multiplication order.
    plan.sinv[j] = std::sin(plan.theta[j]);
    plan.cosv[j] = std::cos(plan.theta[j]);
  }
  const double pi = std::numbers::pi_v<double>;
  for (std::size_t index = 0; index < c.modes.size(); ++index) {
    ModePlan mp;
    mp.m = c.modes[index];
    mp.mode_index = static_cast<int>(index);
    mp.parent = contains(c.parents, mp.m);
    if (mp.parent) {
      mp.ell_min = std::max(std::abs(kSpinWeight), std::abs(mp.m));
      if (c.ell_max_first < mp.ell_min) {
        throw std::invalid_argument(
            "ell_max is below the minimum allowed ell");
      }
      mp.n_ell = c.ell_max_first - mp.ell_min + 1;
      if (mp.n_ell > c.ntheta) {
        throw std::invalid_argument(
            "angular transform needs at least as many nodes as modes");
      }
      if (mp.n_ell > kMaxEll) {
        throw std::invalid_argument("angular band exceeds the engine limit");
      }
      const std::size_t ne = static_cast<std::size_t>(mp.n_ell);
      mp.synthesis.assign(nt * ne, 0.0);
      mp.analysis.assign(ne * nt, 0.0);
      for (std::size_t j = 0; j < nt; ++j) {
        for (std::size_t l = 0; l < ne; ++l) {
          const int ell = mp.ell_min + static_cast<int>(l);
          const double basis = spin_weighted_harmonic_theta(
              ell, mp.m, kSpinWeight, plan.theta[j]);
          mp.synthesis[j * ne + l] = basis;
          mp.analysis[l * nt + j] = 2.0 * pi * plan.weights[j] * basis;
        }
      }
    }
    plan.modes.push_back(std::move(mp));
  }
  if (c.source_mode == 2 && c.source_start_time == 0.0) {
    plan.active = 1;
    plan.activation_time = 0.0;
    plan.consecutive_passes = c.required_passes;
  }
  return plan;
}

// ---------------------------------------------------------------- initial data
namespace {

struct Cx {
  double re = 0.0;
  double im = 0.0;
};
Cx operator+(const Cx a, const Cx b) { return {a.re + b.re, a.im + b.im}; }
Cx operator-(const Cx a, const Cx b) { return {a.re - b.re, a.im - b.im}; }
Cx operator*(const Cx a, const Cx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
Cx operator*(const double s, const Cx a) { return {s * a.re, s * a.im}; }
// |c|+|d| scaled division.
Cx operator/(const Cx x, const Cx y) {
  const double s = std::fabs(y.re) + std::fabs(y.im);
  const double xr = x.re / s, xi = x.im / s, yr = y.re / s, yi = -y.im / s;
  const double d = yr * yr + yi * yi;
  return {(xr * yr - xi * yi) / d, (xr * yi + xi * yr) / d};
}
double magnitude(const Cx a) { return std::hypot(a.re, a.im); }

RowCoefficients row_coefficients(const Config& c, const double R,
                                 const int m) {
  const double M = c.mass, a = c.spin, L = c.length;
  const double L2 = L * L, L4 = L2 * L2, R2 = R * R, a2 = a * a;
  const double mrl = M * R / L2;
  const double s = static_cast<double>(kSpinWeight);
  const double mm = static_cast<double>(m);
  RowCoefficients r{};
  r.c0 = 8.0 * M * (2.0 * M - a2 * R / L2) * (1.0 + 2.0 * mrl);
  r.K = L2 - (8.0 * M * M - a2) * R2 / L2 + 4.0 * a2 * M * R * R2 / L4;
  r.HR = R2 / L4 * (L4 - 2.0 * L2 * M * R + a2 * R2);
  r.g_re = 2.0 * (2.0 * M * (-s + (2.0 + s) * 2.0 * mrl - 3.0 * a2 * R2 / L4) -
                  a2 * R / L2);
  r.g_im_m = 2.0 * a * mm * (1.0 + 4.0 * mrl);
  r.q_re = 2.0 * R * (1.0 + s - (3.0 + s) * mrl + 2.0 * a2 * R2 / L4);
  r.q_im = -(2.0 * a * mm * R2 / L2);
  r.c_re = -2.0 * R * ((1.0 + s) * M / L2 - a2 * R / L4);
  r.c_im = -(2.0 * a * mm * R / L2);
  return r;
}

std::vector<Cx> dense_solve(std::vector<Cx> matrix, std::vector<Cx> rhs) {
  const std::size_t n = rhs.size();
  double scale = 0.0;
  for (const Cx v : matrix) scale = std::max(scale, magnitude(v));
  const double floor =
      128.0 * std::numeric_limits<double>::epsilon() * scale;
  for (std::size_t col = 0; col < n; ++col) {
    std::size_t pivot = col;
    double best = magnitude(matrix[col * n + col]);
    for (std::size_t row = col + 1; row < n; ++row) {
      const double cand = magnitude(matrix[row * n + col]);
      if (cand > best) {
        pivot = row;
        best = cand;
      }
    }
    if (!std::isfinite(best) || best <= floor) {
      throw std::runtime_error("singular Galerkin initialization matrix");
    }
    if (pivot != col) {
      for (std::size_t j = col; j < n; ++j) {
        std::swap(matrix[col * n + j], matrix[pivot * n + j]);
      }
      std::swap(rhs[col], rhs[pivot]);
    }
    const Cx diag = matrix[col * n + col];
    for (std::size_t row = col + 1; row < n; ++row) {
      const Cx factor = matrix[row * n + col] / diag;
      matrix[row * n + col] = Cx{};
      for (std::size_t j = col + 1; j < n; ++j) {
        matrix[row * n + j] = matrix[row * n + j] - factor * matrix[col * n + j];
      }
      rhs[row] = rhs[row] - factor * rhs[col];
    }
  }
  std::vector<Cx> x(n);
  for (std::size_t rev = 0; rev < n; ++rev) {
    const std::size_t row = n - 1 - rev;
    Cx v = rhs[row];
    for (std::size_t col = row + 1; col < n; ++col) {
      v = v - matrix[row * n + col] * x[col];
    }
    x[row] = v / matrix[row * n + row];
  }
  return x;
}

double relative_residual(const std::vector<Cx>& matrix,
                         const std::vector<Cx>& x,
                         const std::vector<Cx>& rhs) {
  const std::size_t n = rhs.size();
  double res2 = 0.0, rhs2 = 0.0;
  for (std::size_t row = 0; row < n; ++row) {
    Cx r{-rhs[row].re, -rhs[row].im};
    for (std::size_t col = 0; col < n; ++col) {
      r = r + matrix[row * n + col] * x[col];
    }
    res2 += magnitude(r) * magnitude(r);
    rhs2 += magnitude(rhs[row]) * magnitude(rhs[row]);
  }
  return std::sqrt(res2) /
         std::max(std::sqrt(rhs2), std::numeric_limits<double>::min());
}

}  // namespace

// Restates initialize_compactified_gaussian_pulse
// (include/teuk/pipeline_initial_data.hpp:211-339) for the first-order
// fields: psi = profile(R) * S_m seed, Q = D psi with the production radial
// operator, P from the projected C_T^{-1} Galerkin system (:142-207), then
// projection of every field onto its band.  Higher fields start at zero.
void validate_gaussian(const InstancePlan& plan, const double center,
                       const double width, const std::vector<int>& ell,
                       const std::vector<int>& m_values) {
  const Config& c = plan.config;
  const int ell_max = c.ell_max_first;
  if (ell_max < 2 || c.ntheta < ell_max + 1) {
    throw std::invalid_argument(
        "initial-data angular band does not fit the pipeline grid");
  }
  if (!(width > 0.0) || center < 0.0 || center > plan.horizon) {
    throw std::invalid_argument(
        "Gaussian center must be on-grid and width must be positive");
  }
  if (ell.empty()) {
    throw std::invalid_argument("Gaussian pulse needs at least one mode");
  }
  for (std::size_t i = 0; i < ell.size(); ++i) {
    if (!std::binary_search(c.parents.begin(), c.parents.end(),
                            m_values[i])) {
      throw std::invalid_argument("Gaussian seed m is not a first-order mode");
    }
    if (ell[i] < std::max(2, std::abs(m_values[i])) || ell[i] > ell_max) {
      throw std::invalid_argument("Gaussian seed ell is outside the band");
    }
    for (std::size_t j = 0; j < i; ++j) {
      if (ell[j] == ell[i] && m_values[j] == m_values[i]) {
        throw std::invalid_argument("duplicate Gaussian (ell,m) seed");
      }
    }
  }
}

double gaussian_profile(const double R, const double center,
                        const double width, const bool compact_support) {
  const double x = (R - center) / width;
  if (!compact_support) return std::exp(-x * x);
  if (std::abs(R - center) >= width) return 0.0;
  return std::exp(1.0 - 1.0 / (1.0 - x * x));
}

double gaussian_initial_state(const InstancePlan& plan, const double center,
                              const double width, const bool compact_support,
                              const std::vector<int>& ell,
                              const std::vector<int>& m_values,
                              const std::vector<double>& amp_re,
                              const std::vector<double>& amp_im,
                              std::vector<double>& nodal) {
  const Config& c = plan.config;
  const int nr = c.nr;
  const int nt = c.ntheta;
  const std::size_t nmodes = c.modes.size();
  validate_gaussian(plan, center, width, ell, m_values);
  const auto at = [&](const std::size_t mode, const int field, const int r,
                      const int j) -> std::size_t {
    return 2 * (((mode * kFieldCount + static_cast<std::size_t>(field)) *
                     static_cast<std::size_t>(nr) +
                 static_cast<std::size_t>(r)) *
                    static_cast<std::size_t>(nt) +
                static_cast<std::size_t>(j));
  };
  nodal.assign(2 * plan.value_count(), 0.0);
  const auto profile = [&](const double R) {
    return gaussian_profile(R, center, width, compact_support);
  };
  // psi
  for (std::size_t mode = 0; mode < nmodes; ++mode) {
    const ModePlan& mp = plan.modes[mode];
    if (!mp.parent) continue;
    const std::size_t ne = static_cast<std::size_t>(mp.n_ell);
    std::vector<Cx> seed(ne);
    for (std::size_t i = 0; i < ell.size(); ++i) {
      if (m_values[i] == mp.m) {
        Cx& s = seed[static_cast<std::size_t>(ell[i] - mp.ell_min)];
        s = s + Cx{amp_re[i], amp_im[i]};
      }
    }
    std::vector<Cx> angular(static_cast<std::size_t>(nt));
    for (int j = 0; j < nt; ++j) {
      Cx v{};
      for (std::size_t l = 0; l < ne; ++l) {
        v = v + mp.synthesis[static_cast<std::size_t>(j) * ne + l] * seed[l];
      }
      angular[static_cast<std::size_t>(j)] = v;
    }
    for (int r = 0; r < nr; ++r) {
      const double prof = profile(plan.spacing * static_cast<double>(r));
      for (int j = 0; j < nt; ++j) {
        const Cx v = prof * angular[static_cast<std::size_t>(j)];
        nodal[at(mode, 2, r, j)] = v.re;
        nodal[at(mode, 2, r, j) + 1] = v.im;
      }
    }
  }
  // Q = D psi
  std::vector<double> line(2 * static_cast<std::size_t>(nr));
  std::vector<double> dline(2 * static_cast<std::size_t>(nr));
  for (std::size_t mode = 0; mode < nmodes; ++mode) {
    for (int j = 0; j < nt; ++j) {
      for (int r = 0; r < nr; ++r) {
        line[2 * r] = nodal[at(mode, 2, r, j)];
        line[2 * r + 1] = nodal[at(mode, 2, r, j) + 1];
      }
      sbp_derivative_line(c.disc, line.data(), nr, 1.0 / plan.spacing,
                          dline.data());
      for (int r = 0; r < nr; ++r) {
        nodal[at(mode, 1, r, j)] = dline[2 * r];
        nodal[at(mode, 1, r, j) + 1] = dline[2 * r + 1];
      }
    }
  }
  // P: Galerkin zero time derivative in the retained band.
  double max_residual = 0.0;
  for (std::size_t mode = 0; mode < nmodes; ++mode) {
    const ModePlan& mp = plan.modes[mode];
    if (!mp.parent) continue;
    const std::size_t ne = static_cast<std::size_t>(mp.n_ell);
    std::vector<Cx> matrix(ne * ne), rhs(ne);
    for (int r = 0; r < nr; ++r) {
      std::fill(matrix.begin(), matrix.end(), Cx{});
      std::fill(rhs.begin(), rhs.end(), Cx{});
      const RowCoefficients rc =
          row_coefficients(c, plan.spacing * static_cast<double>(r), mp.m);
      for (int j = 0; j < nt; ++j) {
        const double sin_t = plan.sinv[static_cast<std::size_t>(j)];
        const double time = rc.c0 - c.spin * c.spin * sin_t * sin_t;
        const double inverse_time = 1.0 / time;
        const Cx G{rc.g_re,
                   rc.g_im_m + 2.0 * (kSpinWeight * c.spin *
                                      plan.cosv[static_cast<std::size_t>(j)])};
        const Cx Q{nodal[at(mode, 1, r, j)], nodal[at(mode, 1, r, j) + 1]};
        const Cx psi{nodal[at(mode, 2, r, j)], nodal[at(mode, 2, r, j) + 1]};
        const Cx nodal_rhs = inverse_time * ((-2.0 * rc.K) * Q + G * psi);
        for (std::size_t row = 0; row < ne; ++row) {
          const double a = mp.analysis[row * static_cast<std::size_t>(nt) +
                                       static_cast<std::size_t>(j)];
          rhs[row] = rhs[row] + a * nodal_rhs;
          for (std::size_t col = 0; col < ne; ++col) {
            matrix[row * ne + col].re +=
                a * inverse_time *
                mp.synthesis[static_cast<std::size_t>(j) * ne + col];
          }
        }
      }
      const std::vector<Cx> p = dense_solve(matrix, rhs);
      max_residual = std::max(max_residual, relative_residual(matrix, p, rhs));
      for (int j = 0; j < nt; ++j) {
        Cx v{};
        for (std::size_t l = 0; l < ne; ++l) {
          v = v + mp.synthesis[static_cast<std::size_t>(j) * ne + l] * p[l];
        }
        nodal[at(mode, 0, r, j)] = v.re;
        nodal[at(mode, 0, r, j) + 1] = v.im;
      }
    }
  }
  if (!std::isfinite(max_residual) || max_residual > 2.0e-12) {
    throw std::runtime_error(
        "Galerkin initial-time-derivative solve failed its residual check");
  }
  // Band projection of the first-order fields (the others are zero).
  std::vector<Cx> modal;
  for (std::size_t mode = 0; mode < nmodes; ++mode) {
    const ModePlan& mp = plan.modes[mode];
    for (int f = 0; f < 3; ++f) {
      for (int r = 0; r < nr; ++r) {
        if (!mp.parent) {
          for (int j = 0; j < nt; ++j) {
            nodal[at(mode, f, r, j)] = 0.0;
            nodal[at(mode, f, r, j) + 1] = 0.0;
          }
          continue;
        }
        const std::size_t ne = static_cast<std::size_t>(mp.n_ell);
        modal.assign(ne, Cx{});
        for (std::size_t l = 0; l < ne; ++l) {
          Cx v{};
          for (int j = 0; j < nt; ++j) {
            v = v + mp.analysis[l * static_cast<std::size_t>(nt) +
                                static_cast<std::size_t>(j)] *
                        Cx{nodal[at(mode, f, r, j)],
                           nodal[at(mode, f, r, j) + 1]};
          }
          modal[l] = v;
        }
        for (int j = 0; j < nt; ++j) {
          Cx v{};
          for (std::size_t l = 0; l < ne; ++l) {
            v = v + mp.synthesis[static_cast<std::size_t>(j) * ne + l] *
                        modal[l];
          }
          nodal[at(mode, f, r, j)] = v.re;
          nodal[at(mode, f, r, j) + 1] = v.im;
        }
      }
    }
  }
  return max_residual;
}

}  // namespace teuk_b200
