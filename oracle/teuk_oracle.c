/*
 * CPU restatement of the teuk-kokkos linear RK4 path (test infrastructure;
 * see teuk_oracle.h).  Plain C11, binary64 complex arithmetic written out
 * as (re, im) pairs in the reference's operation order.
 */
#include "teuk_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../teuk-kokkos_b200/csrc/sbp_tables.h"

#define FIELDS 13
#define SPIN (-2)
static const long double PI_L = 3.141592653589793238462643383279502884L;
static const double PI_D = 3.141592653589793;

static char g_error[512];

static int fail(const int code, const char* message) {
  snprintf(g_error, sizeof g_error, "%s", message);
  return code;
}

const char* oracle_last_error(void) { return g_error; }

typedef struct {
  double re, im;
} cx;

static cx cx_add(cx a, cx b) { return (cx){a.re + b.re, a.im + b.im}; }
static cx cx_sub(cx a, cx b) { return (cx){a.re - b.re, a.im - b.im}; }
static cx cx_mul(cx a, cx b) {
  return (cx){a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
static cx cx_rmul(double s, cx a) { return (cx){s * a.re, s * a.im}; }
static cx cx_rdiv(cx a, double d) { return (cx){a.re / d, a.im / d}; }

/* ------------------------------------------------------------ angular */
/* Gauss-Legendre nodes: include/teuk/angular.hpp:69-115 */
static void legendre_pair(int degree, long double x, long double* p,
                          long double* previous) {
  long double prev = 1.0L;
  if (degree == 0) {
    *p = prev;
    *previous = 0.0L;
    return;
  }
  long double cur = x;
  for (int ell = 2; ell <= degree; ++ell) {
    const long double next =
        ((2.0L * ell - 1.0L) * x * cur - (ell - 1.0L) * prev) / ell;
    prev = cur;
    cur = next;
  }
  *p = cur;
  *previous = prev;
}

int oracle_gauss_legendre(const int n, double* x, double* w) {
  if (n <= 0) return fail(-1, "Gauss-Legendre node count must be positive");
  const int half = (n + 1) / 2;
  const long double tol = 8.0L * 1.0842021724855044340e-19L; /* LDBL_EPSILON */
  for (int i = 0; i < half; ++i) {
    long double root = cosl(PI_L * (i + 0.75L) / (n + 0.5L));
    long double pn, pm, derivative = 0.0L;
    for (int it = 0; it < 100; ++it) {
      legendre_pair(n, root, &pn, &pm);
      derivative = n * (root * pn - pm) / (root * root - 1.0L);
      const long double update = pn / derivative;
      root -= update;
      if (fabsl(update) <= tol * (1.0L + fabsl(root))) break;
      if (it == 99) return fail(-2, "Gauss-Legendre root iteration failed");
    }
    legendre_pair(n, root, &pn, &pm);
    derivative = n * (root * pn - pm) / (root * root - 1.0L);
    const long double weight =
        2.0L / ((1.0L - root * root) * derivative * derivative);
    x[i] = (double)(-root);
    x[n - 1 - i] = (double)root;
    w[i] = (double)weight;
    w[n - 1 - i] = (double)weight;
  }
  return 0;
}

static long double ipow_l(long double base, int e) {
  long double r = 1.0L;
  while (e != 0) {
    if (e & 1) r *= base;
    base *= base;
    e >>= 1;
  }
  return r;
}

static long double lfact(int n) { return lgammal((long double)n + 1.0L); }

/* Wigner small-d (include/teuk/angular.hpp:170-206) */
static double wigner_d(int ell, int mp, int m, double theta) {
  const int kmin = m - mp > 0 ? m - mp : 0;
  const int kmax = (ell + m) < (ell - mp) ? (ell + m) : (ell - mp);
  const long double lnorm =
      0.5L * (lfact(ell + m) + lfact(ell - m) + lfact(ell + mp) +
              lfact(ell - mp));
  const long double c = cosl(0.5L * (long double)theta);
  const long double s = sinl(0.5L * (long double)theta);
  long double value = 0.0L;
  for (int k = kmin; k <= kmax; ++k) {
    const long double lc = lnorm - lfact(ell + m - k) - lfact(k) -
                           lfact(mp - m + k) - lfact(ell - mp - k);
    long double term = expl(lc) * ipow_l(c, 2 * ell + m - mp - 2 * k) *
                       ipow_l(s, mp - m + 2 * k);
    if ((mp - m + k) & 1) term = -term;
    value += term;
  }
  return (double)value;
}

/* spin_weighted_harmonic_theta (include/teuk/angular.hpp:211-217) */
static double swsh(int ell, int m, int spin, double theta) {
  const double phase = (abs(spin) & 1) ? -1.0 : 1.0;
  return phase * sqrt((2.0 * ell + 1.0) / (4.0 * PI_D)) *
         wigner_d(ell, m, -spin, theta);
}

/* ------------------------------------------------------------ SBP */
static double rat(teuk_sbp_rational r) { return r.num / r.den; }

static int boundary_rows(int disc) { return disc == 0 ? 4 : disc == 1 ? 8 : 11; }
static int boundary_width(int disc) { return disc == 0 ? 6 : disc == 1 ? 12 : 16; }
static int min_points(int disc) { return disc == 0 ? 8 : disc == 1 ? 16 : 22; }

static double norm_weight(int disc, int n, int index) {
  const int d = index < n - 1 - index ? index : n - 1 - index;
  if (disc == 0) return d < 4 ? rat(teuk_d42_norm[d]) : 1.0;
  if (disc == 1) return d < 8 ? rat(teuk_d84_norm[d]) : 1.0;
  return d < 11 ? rat(teuk_d105_norm[d]) : 1.0;
}

/* closure coefficient of h*D (sbp.hpp:34-74, sbp84.hpp:36-122,
 * sbp105.hpp:62-207) */
static double left_coef(int disc, int row, int col) {
  if (disc == 0) return col < 6 ? rat(teuk_d42_left[row][col]) : 0.0;
  if (disc == 1) return col < 12 ? rat(teuk_d84_left[row][col]) : 0.0;
  double q = 0.0;
  if (col < 11) {
    q = rat(teuk_d105_left_q[row][col]);
  } else {
    const int off = col - row;
    if (off == 1) q = 5.0 / 6.0;
    else if (off == 2) q = -5.0 / 21.0;
    else if (off == 3) q = 5.0 / 84.0;
    else if (off == 4) q = -5.0 / 504.0;
    else if (off == 5) q = 1.0 / 1260.0;
  }
  return q / rat(teuk_d105_norm[row]);
}

/* radial_first_derivative_strided_at (radial_discretization.hpp:131-145) */
static cx derivative_at(int disc, const cx* v, int stride, int n, int r,
                        double inv_h) {
  const int br = boundary_rows(disc), w = boundary_width(disc);
  cx result = {0.0, 0.0};
#define V(i) v[(size_t)(i) * (size_t)stride]
  if (r < br) {
    for (int c = 0; c < w; ++c) {
      result = cx_add(result, cx_rmul(left_coef(disc, r, c), V(c)));
    }
  } else if (r + br >= n) {
    const int rr = n - 1 - r;
    for (int c = 0; c < w; ++c) {
      result = cx_sub(result, cx_rmul(left_coef(disc, rr, c), V(n - 1 - c)));
    }
  } else if (disc == 0) {
    cx t = cx_sub(V(r - 2), cx_rmul(8.0, V(r - 1)));
    t = cx_add(t, cx_rmul(8.0, V(r + 1)));
    t = cx_sub(t, V(r + 2));
    result = cx_rdiv(t, 12.0);
  } else if (disc == 1) {
    result = cx_rdiv(cx_sub(V(r - 4), V(r + 4)), 280.0);
    result = cx_add(result, cx_rdiv(cx_rmul(4.0, cx_add(cx_rmul(-1.0, V(r - 3)),
                                                        V(r + 3))), 105.0));
    result = cx_add(result, cx_rdiv(cx_sub(V(r - 2), V(r + 2)), 5.0));
    result = cx_add(result, cx_rdiv(cx_rmul(4.0, cx_add(cx_rmul(-1.0, V(r - 1)),
                                                        V(r + 1))), 5.0));
  } else {
    result = cx_rdiv(cx_add(cx_rmul(-1.0, V(r - 5)), V(r + 5)), 1260.0);
    result = cx_add(result, cx_rdiv(cx_rmul(5.0, cx_sub(V(r - 4), V(r + 4))),
                                     504.0));
    result = cx_add(result, cx_rdiv(cx_rmul(5.0, cx_add(cx_rmul(-1.0, V(r - 3)),
                                                         V(r + 3))), 84.0));
    result = cx_add(result, cx_rdiv(cx_rmul(5.0, cx_sub(V(r - 2), V(r + 2))),
                                     21.0));
    result = cx_add(result, cx_rdiv(cx_rmul(5.0, cx_add(cx_rmul(-1.0, V(r - 1)),
                                                        V(r + 1))), 6.0));
  }
#undef V
  return cx_rmul(inv_h, result);
}

/* radial_compatible_dissipation_at, strided form
 * (radial_discretization.hpp:163-234) */
static cx dissipation_at(int disc, const cx* v, int stride, int n, int index,
                         double h, double strength) {
  static const double b[3][7] = {{-1, 3, -3, 1, 0, 0, 0},
                                 {-1, 5, -10, 10, -5, 1, 0},
                                 {1, -6, 15, -20, 15, -6, 1}};
  const int order = disc == 2 ? 6 : disc == 1 ? 5 : 3;
  const int first = index > order ? index - order : 0;
  const int last = index < n - order ? index : n - order - 1;
  cx normal = {0.0, 0.0};
  for (int row = first; row <= last; ++row) {
    cx diff = {0.0, 0.0};
    for (int c = 0; c <= order; ++c) {
      diff = cx_add(diff, cx_rmul(b[disc][c],
                                  v[(size_t)(row + c) * (size_t)stride]));
    }
    normal = cx_add(normal, cx_rmul(b[disc][index - row], diff));
  }
  const double scale = -strength / (h * norm_weight(disc, n, index));
  return cx_rmul(scale, normal);
}

int oracle_sbp_matrix(int disc, int n, double* D, double* H) {
  if (disc < 0 || disc > 2) return fail(-1, "unknown radial discretization");
  cx* unit = calloc((size_t)n, sizeof(cx));
  if (!unit) return fail(-5, "allocation failed");
  for (int col = 0; col < n; ++col) {
    memset(unit, 0, (size_t)n * sizeof(cx));
    unit[col].re = 1.0;
    for (int row = 0; row < n; ++row) {
      D[(size_t)row * (size_t)n + (size_t)col] =
          derivative_at(disc, unit, 1, n, row, 1.0).re;
    }
  }
  for (int row = 0; row < n; ++row) H[row] = norm_weight(disc, n, row);
  free(unit);
  return 0;
}

/* ------------------------------------------------------------ pipeline */
typedef struct {
  int m, parent, ell_min, n_ell;
  double* S; /* [nt][ne] */
  double* A; /* [ne][nt] */
} mode_plan;

struct oracle_pipeline {
  double mass, spin, length, damping, dissipation, h;
  int nr, nt, ell_max, disc, reduction, nmodes;
  int* modes;
  mode_plan* plan;
  double *theta;
  size_t count; /* complex values */
  cx *state, *stage, *k1, *k2, *k3, *k4, *lap, *scratch;
};

static int cmp_int(const void* a, const void* b) {
  const int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

static size_t at(const oracle_pipeline* p, int mode, int f, int r, int j) {
  return (((size_t)mode * FIELDS + (size_t)f) * (size_t)p->nr + (size_t)r) *
             (size_t)p->nt + (size_t)j;
}

int oracle_destroy(oracle_pipeline* p) {
  if (!p) return 0;
  for (int i = 0; i < p->nmodes; ++i) {
    free(p->plan[i].S);
    free(p->plan[i].A);
  }
  free(p->plan);
  free(p->modes);
  free(p->theta);
  free(p->state);
  free(p->stage);
  free(p->k1);
  free(p->k2);
  free(p->k3);
  free(p->k4);
  free(p->lap);
  free(p->scratch);
  free(p);
  return 0;
}

int oracle_create(const teuk_b200_config* c, oracle_pipeline** out) {
  if (!c || !out) return fail(-1, "null argument");
  if (c->source_mode != TEUK_B200_SOURCE_DISABLED) {
    return fail(-4, "the oracle restates the linear (disabled) pipeline only");
  }
  if (c->radial_points < min_points(c->discretization) ||
      c->discretization < 0 || c->discretization > 2) {
    return fail(-1, "radial grid is too small for selected discretization");
  }
  oracle_pipeline* p = calloc(1, sizeof *p);
  if (!p) return fail(-5, "allocation failed");
  p->mass = c->mass;
  p->spin = c->spin;
  p->length = c->compactification_length;
  p->damping = c->reduction == TEUK_B200_FREE_DAMPED ? c->reduction_damping : 0.0;
  p->dissipation = c->dissipation;
  p->nr = c->radial_points;
  p->nt = c->theta_nodes;
  p->ell_max = c->ell_max_first;
  p->disc = c->discretization;
  p->reduction = c->reduction;
  p->nmodes = c->mode_count;
  const double r_plus = c->mass + sqrt(c->mass * c->mass - c->spin * c->spin);
  const double horizon = c->compactification_length *
                         c->compactification_length / r_plus;
  p->h = (horizon - 0.0) / (double)(p->nr - 1);
  p->modes = malloc(sizeof(int) * (size_t)p->nmodes);
  memcpy(p->modes, c->modes, sizeof(int) * (size_t)p->nmodes);
  qsort(p->modes, (size_t)p->nmodes, sizeof(int), cmp_int);
  double* x = malloc(sizeof(double) * (size_t)p->nt);
  double* w = malloc(sizeof(double) * (size_t)p->nt);
  p->theta = malloc(sizeof(double) * (size_t)p->nt);
  oracle_gauss_legendre(p->nt, x, w);
  for (int j = 0; j < p->nt; ++j) p->theta[j] = acos(x[j]);
  p->plan = calloc((size_t)p->nmodes, sizeof(mode_plan));
  for (int i = 0; i < p->nmodes; ++i) {
    mode_plan* mp = &p->plan[i];
    mp->m = p->modes[i];
    for (int k = 0; k < c->parent_count; ++k) {
      if (c->parents[k] == mp->m) mp->parent = 1;
    }
    if (!mp->parent) continue;
    mp->ell_min = abs(mp->m) > 2 ? abs(mp->m) : 2;
    mp->n_ell = p->ell_max - mp->ell_min + 1;
    mp->S = malloc(sizeof(double) * (size_t)(p->nt * mp->n_ell));
    mp->A = malloc(sizeof(double) * (size_t)(p->nt * mp->n_ell));
    for (int j = 0; j < p->nt; ++j) {
      for (int l = 0; l < mp->n_ell; ++l) {
        const double basis = swsh(mp->ell_min + l, mp->m, SPIN, p->theta[j]);
        mp->S[j * mp->n_ell + l] = basis;
        mp->A[l * p->nt + j] = 2.0 * PI_D * w[j] * basis;
      }
    }
  }
  free(x);
  free(w);
  p->count = (size_t)p->nmodes * FIELDS * (size_t)p->nr * (size_t)p->nt;
  cx** bufs[] = {&p->state, &p->stage, &p->k1, &p->k2, &p->k3, &p->k4,
                 &p->scratch};
  for (size_t i = 0; i < sizeof bufs / sizeof bufs[0]; ++i) {
    *bufs[i] = calloc(p->count, sizeof(cx));
    if (!*bufs[i]) {
      oracle_destroy(p);
      return fail(-5, "allocation failed");
    }
  }
  p->lap = calloc((size_t)p->nmodes * (size_t)p->nr * (size_t)p->nt, sizeof(cx));
  *out = p;
  return 0;
}

int oracle_set_state(oracle_pipeline* p, const double* s, size_t count) {
  if (count != p->count) return fail(-1, "state complex count does not match");
  memcpy(p->state, s, count * sizeof(cx));
  return 0;
}

int oracle_get_state(oracle_pipeline* p, double* s, size_t count) {
  if (count != p->count) return fail(-1, "state complex count does not match");
  memcpy(s, p->state, count * sizeof(cx));
  return 0;
}

/* analyze -> (diag) -> synthesize one nodal line of nt values */
static void band_line(const oracle_pipeline* p, const mode_plan* mp,
                      const cx* in, size_t in_stride, cx* out,
                      size_t out_stride, int laplacian) {
  cx modal[128];
  for (int l = 0; l < mp->n_ell; ++l) {
    cx v = {0.0, 0.0};
    for (int j = 0; j < p->nt; ++j) {
      v = cx_add(v, cx_rmul(mp->A[l * p->nt + j], in[(size_t)j * in_stride]));
    }
    if (laplacian) {
      const int ell = mp->ell_min + l;
      v = cx_rmul(-(double)((ell - SPIN) * (ell + SPIN + 1)), v);
    }
    modal[l] = v;
  }
  for (int j = 0; j < p->nt; ++j) {
    cx v = {0.0, 0.0};
    for (int l = 0; l < mp->n_ell; ++l) {
      v = cx_add(v, cx_rmul(mp->S[j * mp->n_ell + l], modal[l]));
    }
    out[(size_t)j * out_stride] = v;
  }
}

/* teukolsky_coefficients (include/teuk/teukolsky.hpp:38-85) */
typedef struct {
  double time, K, HR;
  cx G, q, c;
} coefs;

static coefs coefficients(const oracle_pipeline* p, double R, double theta,
                          int m) {
  const double M = p->mass, a = p->spin, L = p->length;
  const double L2 = L * L, L4 = L2 * L2, R2 = R * R, a2 = a * a;
  const double mrl = M * R / L2;
  const double s = (double)SPIN, mm = (double)m;
  coefs k;
  k.time = 8.0 * M * (2.0 * M - a2 * R / L2) * (1.0 + 2.0 * mrl) -
           a2 * sin(theta) * sin(theta);
  k.K = L2 - (8.0 * M * M - a2) * R2 / L2 + 4.0 * a2 * M * R * R2 / L4;
  k.HR = R2 / L4 * (L4 - 2.0 * L2 * M * R + a2 * R2);
  const cx g1 = {0.0, 2.0 * a * mm * (1.0 + 4.0 * mrl)};
  const double g2_re =
      2.0 * M * (-s + (2.0 + s) * 2.0 * mrl - 3.0 * a2 * R2 / L4) - a2 * R / L2;
  const cx g2 = {2.0 * g2_re, 2.0 * (s * a * cos(theta))};
  k.G = cx_add(g1, g2);
  k.q = (cx){2.0 * R * (1.0 + s - (3.0 + s) * mrl + 2.0 * a2 * R2 / L4),
             -(2.0 * a * mm * R2 / L2)};
  k.c = (cx){-2.0 * R * ((1.0 + s) * M / L2 - a2 * R / L4),
             -(2.0 * a * mm * R / L2)};
  return k;
}

static int is_parent(const oracle_pipeline* p, int mode) {
  return p->plan[mode].parent;
}

static void evaluate(oracle_pipeline* p, const cx* stage, cx* out) {
  const int nr = p->nr, nt = p->nt;
  const double inv_h = 1.0 / p->h;
  memset(out, 0, p->count * sizeof(cx));
  cx* dpsi = malloc(sizeof(cx) * (size_t)nr);
  cx* qeff = malloc(sizeof(cx) * (size_t)nr);
  cx* dq = malloc(sizeof(cx) * (size_t)nr);
  cx* vel = malloc(sizeof(cx) * (size_t)nr);
  cx* dvel = malloc(sizeof(cx) * (size_t)nr);
  for (int mode = 0; mode < p->nmodes; ++mode) {
    const mode_plan* mp = &p->plan[mode];
    cx* lap = p->lap + (size_t)mode * (size_t)nr * (size_t)nt;
    for (int r = 0; r < nr; ++r) {
      if (is_parent(p, mode)) {
        band_line(p, mp, stage + at(p, mode, 2, r, 0), 1,
                  lap + (size_t)r * (size_t)nt, 1, 1);
      } else {
        memset(lap + (size_t)r * (size_t)nt, 0, sizeof(cx) * (size_t)nt);
      }
    }
    for (int j = 0; j < nt; ++j) {
      const cx* P = stage + at(p, mode, 0, 0, j);
      const cx* Q = stage + at(p, mode, 1, 0, j);
      const cx* psi = stage + at(p, mode, 2, 0, j);
      for (int r = 0; r < nr; ++r) {
        dpsi[r] = derivative_at(p->disc, psi, nt, nr, r, inv_h);
        qeff[r] = p->reduction == TEUK_B200_STAGE_CONSTRAINED ? dpsi[r]
                                                              : Q[(size_t)r * nt];
      }
      for (int r = 0; r < nr; ++r) {
        dq[r] = derivative_at(p->disc, qeff, 1, nr, r, inv_h);
        const coefs k = coefficients(p, p->h * (double)r, p->theta[j], mp->m);
        cx num = cx_add(P[(size_t)r * nt], cx_rmul(2.0 * k.K, qeff[r]));
        num = cx_sub(num, cx_mul(k.G, psi[(size_t)r * nt]));
        vel[r] = cx_rdiv(num, k.time);
      }
      for (int r = 0; r < nr; ++r) {
        dvel[r] = derivative_at(p->disc, vel, 1, nr, r, inv_h);
      }
      for (int r = 0; r < nr; ++r) {
        const coefs k = coefficients(p, p->h * (double)r, p->theta[j], mp->m);
        cx pt = cx_rmul(k.HR, dq[r]);
        pt = cx_add(pt, cx_mul(k.q, qeff[r]));
        pt = cx_add(pt, cx_mul(k.c, psi[(size_t)r * nt]));
        pt = cx_add(pt, lap[(size_t)r * nt + j]);
        const cx constraint = cx_sub(Q[(size_t)r * nt], dpsi[r]);
        cx qt = cx_sub(dvel[r], cx_rmul(p->damping, constraint));
        cx vt = vel[r];
        if (p->dissipation > 0.0) {
          pt = cx_add(pt, dissipation_at(p->disc, P, nt, nr, r, p->h,
                                         p->dissipation));
          qt = cx_add(qt, dissipation_at(p->disc, Q, nt, nr, r, p->h,
                                         p->dissipation));
          vt = cx_add(vt, dissipation_at(p->disc, psi, nt, nr, r, p->h,
                                         p->dissipation));
        }
        out[at(p, mode, 0, r, j)] = pt;
        out[at(p, mode, 1, r, j)] = qt;
        out[at(p, mode, 2, r, j)] = vt;
      }
    }
    /* band projection of P_t, Q_t, psi_t (zero for non-parent modes) */
    for (int f = 0; f < 3; ++f) {
      for (int r = 0; r < nr; ++r) {
        cx* line = out + at(p, mode, f, r, 0);
        if (is_parent(p, mode)) {
          cx tmp[256];
          memcpy(tmp, line, sizeof(cx) * (size_t)nt);
          band_line(p, mp, tmp, 1, line, 1, 0);
        } else {
          memset(line, 0, sizeof(cx) * (size_t)nt);
        }
      }
    }
  }
  free(dpsi);
  free(qeff);
  free(dq);
  free(vel);
  free(dvel);
}

int oracle_evaluate_rhs(oracle_pipeline* p, const double* stage,
                        double* output, size_t count) {
  if (count != p->count) return fail(-1, "state complex count does not match");
  memcpy(p->scratch, stage, count * sizeof(cx));
  evaluate(p, p->scratch, (cx*)output);
  return 0;
}

/* device_classical_rk4_step (include/teuk/device_rk4.hpp:84-128) */
int oracle_step(oracle_pipeline* p, double dt, int steps) {
  const size_t n = p->count;
  for (int s = 0; s < steps; ++s) {
    evaluate(p, p->state, p->k1);
    for (size_t i = 0; i < n; ++i) {
      p->stage[i] = cx_add(p->state[i], cx_rmul(0.5 * dt, p->k1[i]));
    }
    evaluate(p, p->stage, p->k2);
    for (size_t i = 0; i < n; ++i) {
      p->stage[i] = cx_add(p->state[i], cx_rmul(0.5 * dt, p->k2[i]));
    }
    evaluate(p, p->stage, p->k3);
    for (size_t i = 0; i < n; ++i) {
      p->stage[i] = cx_add(p->state[i], cx_rmul(dt, p->k3[i]));
    }
    evaluate(p, p->stage, p->k4);
    const double scale = dt / 6.0;
    for (size_t i = 0; i < n; ++i) {
      cx sum = cx_add(p->k1[i], cx_rmul(2.0, p->k2[i]));
      sum = cx_add(sum, cx_rmul(2.0, p->k3[i]));
      sum = cx_add(sum, p->k4[i]);
      p->state[i] = cx_add(p->state[i], cx_rmul(scale, sum));
    }
  }
  return 0;
}
