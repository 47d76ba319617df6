// Second-order stage graph on the GPU (see second_order.h).  Every kernel
// below restates one reference kernel or point function in this engine's own
// CUDA; the file:line of each is given where it is defined.  All arithmetic
// is binary64; complex/complex division scales by |c|+|d|.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numbers>
#include <stdexcept>
#include <string>

#include "second_order.h"
#include "split_precision.cuh"
#include "teuk_b200.h"

namespace teuk_b200 {

__constant__ SbpConstants c_sbp_nodal;

namespace {

// ------------------------------------------------------------- slots
enum Field : int {
  kFirstP = 0, kFirstQ = 1, kFirstPsi = 2, kG = 3, kLambda = 4, kH = 5,
  kB = 6, kPi = 7, kC = 8, kU = 9, kSecondP = 10, kSecondQ = 11,
  kSecondPsi = 12
};
enum Scratch : int { kDrPsi = 0, kEffQ = 1, kDrQ = 2, kVel = 3, kDrVel = 4 };
enum Recon : int { rG = 0, rLambda = 1, rH = 2, rB = 3, rPi = 4, rC = 5, rU = 6 };
enum AngIn : int {
  aEth1F = 0, aEth2G = 1, aEth2C = 2, aEth2Pi = 3, aEthP1BSharp = 4,
  aEthP2CSharp = 5
};
enum Sharp : int { shB = 0, shC = 1, shBDt = 2, shCDt = 3 };
enum Extra : int { xEth1B = 0, xEthP1F = 1, xEth1BT = 2, xEthP1FT = 3 };
enum SrcField : int {
  sF = 0, sG = 1, sH = 2, sLambda = 3, sPi = 4, sB = 5, sC = 6, sU = 7
};
enum SrcDeriv : int {
  dDelta1F = 0, dDelta3U = 1, dEth2C = 2, dEthP2CSharp = 3, dEth1B = 4,
  dDelta2C = 5, dDelta2G = 6, dEth2G = 7, dEthP1F = 8, dDelta2CSharp = 9,
  dEthP1BSharp = 10
};
enum Coord : int {
  cFirst = 0, cSecond, cG, cB, cPi, cC, cScalar, cBSharp, cCSharp, cT,
  cCount
};
enum OpKind : int { kProject = 0, kLaplacian = 1, kEth = 2, kEthPrime = 3 };

constexpr int kBlock = 256;
// resident 256-thread blocks per SM that the heaviest pointwise kernels
// (Teukolsky RHS, reconstruction passes 2 and 3; 88-94 registers when
// unbounded) are compiled for: three blocks instead of two per SM, more warps
// per scheduler for their latency-bound loops over grid points
constexpr int kPointBlocks = 3;
constexpr int kMaxNodes = 96;  // theta nodes per row held by one warp
constexpr double kTwoPi = 2.0 * std::numbers::pi_v<double>;

// ------------------------------------------------------------- complex
struct C2 {
  double re, im;
};
__device__ __forceinline__ C2 mk(const double re, const double im) {
  return {re, im};
}
__device__ __forceinline__ C2 ld(const double2 v) { return {v.x, v.y}; }
__device__ __forceinline__ double2 st(const C2 v) {
  return make_double2(v.re, v.im);
}
__device__ __forceinline__ C2 operator+(const C2 a, const C2 b) {
  return {a.re + b.re, a.im + b.im};
}
__device__ __forceinline__ C2 operator-(const C2 a, const C2 b) {
  return {a.re - b.re, a.im - b.im};
}
__device__ __forceinline__ C2 operator-(const C2 a) { return {-a.re, -a.im}; }
__device__ __forceinline__ C2 operator*(const C2 a, const C2 b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ C2 operator*(const double s, const C2 a) {
  return {s * a.re, s * a.im};
}
__device__ __forceinline__ C2 operator*(const C2 a, const double s) {
  return {a.re * s, a.im * s};
}
__device__ __forceinline__ C2 operator/(const C2 a, const double d) {
  return {a.re / d, a.im / d};
}
__device__ __forceinline__ C2 operator/(const C2 x, const C2 y) {
  const double s = fabs(y.re) + fabs(y.im);
  const double xr = x.re / s, xi = x.im / s;
  const double yr = y.re / s, yi = -y.im / s;
  const double d = yr * yr + yi * yi;
  return {(xr * yr - xi * yi) / d, (xr * yi + xi * yr) / d};
}
__device__ __forceinline__ C2 conj(const C2 a) { return {a.re, -a.im}; }
__device__ __forceinline__ double cabs2(const C2 a) { return hypot(a.re, a.im); }

// Jet1<Complex>: value and common-stage tangent (include/teuk/jet.hpp).
struct J {
  C2 v, d;
};
__device__ __forceinline__ J operator+(const J a, const J b) {
  return {a.v + b.v, a.d + b.d};
}
__device__ __forceinline__ J operator-(const J a) { return {-a.v, -a.d}; }
__device__ __forceinline__ J operator*(const J a, const J b) {
  return {a.v * b.v, a.d * b.v + a.v * b.d};
}
__device__ __forceinline__ J operator*(const J a, const C2 f) {
  return {a.v * f, a.d * f};
}
__device__ __forceinline__ J operator*(const C2 f, const J a) { return a * f; }
__device__ __forceinline__ J operator*(const double f, const J a) {
  return a * mk(f, 0.0);
}
__device__ __forceinline__ J operator/(const J a, const C2 f) {
  return {a.v / f, a.d / f};
}
__device__ __forceinline__ J jconj(const J a) { return {conj(a.v), conj(a.d)}; }

// ------------------------------------------------------------- geometry
struct Geo {
  double mass, spin, length, spacing, inv_spacing, horizon;
  double damping, dissipation;
  int nr, nt, modes, disc, reduction;
};

// Kerr background point (include/teuk/background.hpp:28-72).
struct Bg {
  C2 mu0, tau0, pi0, psi20, rho0, eps0;
};
__device__ Bg background(const Geo& g, const double R, const double c,
                         const double s) {
  const double L2 = g.length * g.length, L4 = L2 * L2, a = g.spin;
  const double sqrt_two = sqrt(2.0);
  const C2 minus_radial = mk(-L2, a * R * c);
  const C2 angular = mk(L2, -a * R * c);
  const C2 angular2 = angular * angular;
  const double real_pi = L4 + a * a * R * R * c * c;
  Bg b;
  b.mu0 = mk(1.0, 0.0) / minus_radial;
  b.tau0 = (mk(0.0, 1.0) * a * s) / (sqrt_two * angular2);
  b.pi0 = (mk(0.0, -1.0) * a * s) / (sqrt_two * real_pi);
  const C2 ingoing = mk(L2, a * R * c);
  const C2 optical = angular2 * ingoing;
  b.rho0 = mk(-0.5 * (L4 - 2.0 * L2 * g.mass * R + a * a * R * R), 0.0) /
           optical;
  b.eps0 = 0.5 * mk(L2 * g.mass - a * a * R, -a * (L2 - g.mass * R) * c) /
           optical;
  b.psi20 = mk(-g.mass, 0.0) / (angular2 * angular);
  return b;
}

// Delta_n (include/teuk/ghp.hpp:12-24)
__device__ __forceinline__ C2 delta_n(const Geo& g, const C2 value,
                                      const C2 dt_value, const C2 dr_value,
                                      const int n, const double R) {
  const double L2 = g.length * g.length;
  const double tc = 2.0 + 4.0 * g.mass * R / L2;
  const double rc = R / L2;
  return tc * dt_value + rc * (R * dr_value + static_cast<double>(n) * value);
}

// thorn_n (include/teuk/ghp.hpp:28-64)
__device__ C2 thorn_n(const Geo& g, const C2 value, const C2 dt_value,
                      const C2 dr_value, const int n, const int spin,
                      const int boost, const int m, const double R,
                      const double c, const C2 eps0) {
  const double L2 = g.length * g.length, L4 = L2 * L2, a = g.spin;
  const double den = L4 + a * a * R * R * c * c;
  const double tc = R * 2.0 * g.mass * (2.0 * g.mass - a * a * R / L2) / den;
  const double rc = -0.5 * (L2 - 2.0 * g.mass * R + a * a * R * R / L2) / den;
  const int p = spin + boost, q = -spin + boost;
  const C2 im_term = (R * (mk(0.0, 1.0) * a * static_cast<double>(m) * value)) / den;
  return tc * dt_value + rc * (R * dr_value + static_cast<double>(n) * value) +
         im_term -
         R * ((static_cast<double>(p) * eps0 + static_cast<double>(q) * conj(eps0)) *
              value);
}

// eth_n / eth'_n point formulas (include/teuk/ghp.hpp:69-115)
__device__ C2 eth_point(const Geo& g, const C2 value, const C2 dt_value,
                        const C2 raised, const int spin, const int boost,
                        const double R, const double s, const double c) {
  const double L2 = g.length * g.length, a = g.spin;
  const double sqrt_two = sqrt(2.0);
  const int p = spin + boost;
  const C2 den = mk(L2, -a * R * c);
  const C2 derivative =
      ((mk(0.0, -1.0) * a * s) * dt_value + raised) / (sqrt_two * den);
  const C2 connection = (((mk(0.0, -1.0) * static_cast<double>(p)) * a * R * s) *
                         value) / ((sqrt_two * den) * den);
  return derivative + connection;
}
__device__ C2 ethprime_point(const Geo& g, const C2 value, const C2 dt_value,
                             const C2 lowered, const int spin, const int boost,
                             const double R, const double s, const double c) {
  const double L2 = g.length * g.length, a = g.spin;
  const double sqrt_two = sqrt(2.0);
  const int q = -spin + boost;
  const C2 den = mk(L2, a * R * c);
  const C2 derivative =
      ((mk(0.0, 1.0) * a * s) * dt_value + lowered) / (sqrt_two * den);
  const C2 connection = (((mk(0.0, 1.0) * static_cast<double>(q)) * a * R * s) *
                         value) / ((sqrt_two * den) * den);
  return derivative + connection;
}

// reconstruction_time_derivative (include/teuk/reconstruction.hpp:109-121)
__device__ __forceinline__ C2 recon_dt(const Geo& g, const C2 value,
                                       const C2 dr, const C2 delta_rhs,
                                       const int n, const double R) {
  const double L2 = g.length * g.length;
  const double den = 2.0 + 4.0 * g.mass * R / L2;
  const C2 radial = (R * R / L2) * dr + (static_cast<double>(n) * R / L2) * value;
  return (delta_rhs - radial) / den;
}

// SBP first derivative, strided (include/teuk/radial_discretization.hpp:131-145)
template <int DISC>
__device__ C2 sbp_d(const double2* line, const long long stride, const int n,
                    const int r, const double inv_h) {
  constexpr int BR = DISC == kD42 ? 4 : DISC == kD84 ? 8 : 11;
  constexpr int W = DISC == kD42 ? 6 : DISC == kD84 ? 12 : 16;
  constexpr int HALF = DISC == kD42 ? 2 : DISC == kD84 ? 4 : 5;
  C2 acc = mk(0.0, 0.0);
  if (r < BR) {
    for (int c = 0; c < W; ++c) {
      acc = acc + c_sbp_nodal.left[DISC][r][c] * ld(line[c * stride]);
    }
  } else if (r + BR >= n) {
    const int rr = n - 1 - r;
    for (int c = 0; c < W; ++c) {
      acc = acc - c_sbp_nodal.left[DISC][rr][c] * ld(line[(n - 1 - c) * stride]);
    }
  } else {
    for (int k = HALF; k >= 1; --k) {
      acc = acc + c_sbp_nodal.interior[DISC][k] *
                      (ld(line[(r + k) * stride]) - ld(line[(r - k) * stride]));
    }
  }
  return inv_h * acc;
}

// -(A^T A v)(r)/H_rr (include/teuk/radial_discretization.hpp:163-234)
template <int DISC>
__device__ C2 sbp_diss(const double2* line, const long long stride,
                       const int n, const int r) {
  constexpr int P = DISC == kD42 ? 3 : DISC == kD84 ? 5 : 6;
  constexpr int SPECIAL = DISC == kD42 ? 4 : DISC == kD84 ? 8 : 11;
  C2 acc = mk(0.0, 0.0);
  if (r < SPECIAL) {
    for (int j = 0; j <= r + P; ++j) {
      acc = acc + c_sbp_nodal.diss_left[DISC][r][j] * ld(line[j * stride]);
    }
  } else if (r >= n - SPECIAL) {
    const int rr = n - 1 - r;
    for (int j = 0; j <= rr + P; ++j) {
      acc = acc + c_sbp_nodal.diss_left[DISC][rr][j] * ld(line[(n - 1 - j) * stride]);
    }
  } else {
    acc = c_sbp_nodal.diss_interior[DISC][0] * ld(line[r * stride]);
    for (int k = 1; k <= P; ++k) {
      acc = acc + c_sbp_nodal.diss_interior[DISC][k] *
                      (ld(line[(r + k) * stride]) + ld(line[(r - k) * stride]));
    }
  }
  return acc;
}

__device__ __forceinline__ C2 deriv(const int disc, const double2* line,
                                    const long long stride, const int n,
                                    const int r, const double inv_h) {
  if (disc == kD105) return sbp_d<kD105>(line, stride, n, r, inv_h);
  if (disc == kD84) return sbp_d<kD84>(line, stride, n, r, inv_h);
  return sbp_d<kD42>(line, stride, n, r, inv_h);
}
__device__ __forceinline__ C2 diss(const int disc, const double2* line,
                                   const long long stride, const int n,
                                   const int r) {
  if (disc == kD105) return sbp_diss<kD105>(line, stride, n, r);
  if (disc == kD84) return sbp_diss<kD84>(line, stride, n, r);
  return sbp_diss<kD42>(line, stride, n, r);
}

// ------------------------------------------------------------- indexing
struct Arr {
  double2* p;
  int slots;
  __device__ __forceinline__ double2* at(const Geo& g, const int mode,
                                         const int slot, const int r,
                                         const int t) const {
    return p + ((static_cast<long long>(mode) * slots + slot) * g.nr + r) *
                   g.nt + t;
  }
  __device__ __forceinline__ const double2* line(const Geo& g, const int mode,
                                                 const int slot,
                                                 const int t) const {
    return p + (static_cast<long long>(mode) * slots + slot) * g.nr * g.nt + t;
  }
};

struct Trig {
  const double* theta_sin;  // sin(acos x)
  const double* theta_cos;  // cos(acos x)
  const double* grid_sin;   // sqrt(1 - x^2)
  const double* grid_cos;   // x
  const int* mvals;
  const int* sharp;
};

// ------------------------------------------------------------- angular op
struct AngularOpParams {
  int kind;
  Arr in;
  int in_slot;
  Arr dt;
  int dt_slot;
  Arr out;
  int out_slot;
  const int* active;
  const int* a_off;
  const int* s_off;
  const int* o_off;   // output synthesis matrix (s, s+1 or s-1)
  const int* diag_off;
  const int* ne;
  const int* lmin;
  const int* ne_o;
  const int* lmin_o;
  const double* pool;
  int spin, boost;
};

// Fused SignedModeAngularCoordinator::{project, laplacian, eth, ethprime}
// (include/teuk/angular_coordinator.hpp:125-230 with
// DeviceAngularPlan::analyze/synthesize and DeviceGhpAngularPlan::eth/ethprime,
// angular_device.hpp:177-243, ghp_device.hpp:210-248): one warp per
// (mode, radial) row.
__global__ void angular_op_kernel(const Geo g, const Trig tr,
                                  const AngularOpParams p) {
  __shared__ double2 modal[kBlock / 32][kMaxNodes];
  __shared__ double2 row_in[kBlock / 32][kMaxNodes];  // the input row
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long rows = static_cast<long long>(g.modes) * g.nr;
  for (long long row = blockIdx.x * (kBlock / 32) + warp; row < rows;
       row += static_cast<long long>(gridDim.x) * (kBlock / 32)) {
    const int mode = static_cast<int>(row / g.nr);
    const int r = static_cast<int>(row - static_cast<long long>(mode) * g.nr);
    double2* out = p.out.at(g, mode, p.out_slot, r, 0);
    if (!p.active[mode]) {
      for (int j = lane; j < g.nt; j += 32) out[j] = make_double2(0.0, 0.0);
      continue;
    }
    // one coalesced read of the input row (every lane needs all of it)
    const double2* in = p.in.at(g, mode, p.in_slot, r, 0);
    double2* x = row_in[warp];
    for (int j = lane; j < g.nt; j += 32) x[j] = in[j];
    __syncwarp();
    const int ne = p.ne[mode];
    const double* A = p.pool + p.a_off[mode];
    const double* diag = p.pool + p.diag_off[mode];
    for (int l = lane; l < ne; l += 32) {
      C2 v = mk(0.0, 0.0);
      for (int j = 0; j < g.nt; ++j) v = v + A[j * ne + l] * ld(x[j]);
      if (p.kind != kProject) v = diag[l] * v;
      modal[warp][l] = st(v);
    }
    __syncwarp();
    const int ne_o = p.ne_o[mode];
    const int shift = p.lmin_o[mode] - p.lmin[mode];
    const double* S = p.pool + p.o_off[mode];
    double2 result[kMaxNodes / 32];
    for (int k = 0, j = lane; j < g.nt; j += 32, ++k) {
      C2 v = mk(0.0, 0.0);
      for (int l = 0; l < ne_o; ++l) {
        const int src = l + shift;  // align onto the output band
        if (src >= 0 && src < ne) v = v + S[l * g.nt + j] * ld(modal[warp][src]);
      }
      if (p.kind == kEth || p.kind == kEthPrime) {
        const double2* dtv = p.dt.at(g, mode, p.dt_slot, r, 0);
        const double R = g.spacing * static_cast<double>(r);
        v = p.kind == kEth
                ? eth_point(g, ld(x[j]), ld(dtv[j]), v, p.spin, p.boost, R,
                            tr.grid_sin[j], tr.grid_cos[j])
                : ethprime_point(g, ld(x[j]), ld(dtv[j]), v, p.spin,
                                 p.boost, R, tr.grid_sin[j], tr.grid_cos[j]);
      }
      result[k] = st(v);
    }
    // in-place projection: every lane read the input row before the stores;
    // the next row's staging waits for every lane's reads of this one
    for (int k = 0, j = lane; j < g.nt; j += 32, ++k) out[j] = result[k];
    __syncwarp();
  }
}

// ------------------------------------------------------------- tile operator
// The four operations of angular_op_kernel through one composite nodal
// matrix per (coordinator, operation, mode), built on the host:
//   T = S_out diag(d) A   (nt x nt),   out[r][j] = sum_k T[j][k] x[r][k],
// then the GHP point formula for eth / eth'.  A CTA takes 32 radial rows of
// one mode (a warp 8), stages them in shared memory and multiplies on the
// tensor cores: in FP64 (mma.sync m8n8k4), or in split precision.
//
// Split precision: the digit scheme of split_precision.cuh (BF16 digit
// slices, exact FP32 accumulation, FP64 recombination).
constexpr int kTileRows = 8;     // complex rows of one MMA row tile
constexpr int kTileWarps = 4;    // two warps per row tile, each half the nodes
constexpr int kTileCtaRows = 16; // two row tiles per CTA
constexpr int kTileMaxNodes = 64;                // nodes of the tile kernel
constexpr int kTileStride = kTileMaxNodes + 4;   // staged row stride
constexpr int kTileLoads = kTileCtaRows * kTileMaxNodes / (kTileWarps * 32);
constexpr int kSplitSlices = split::kSlices;
constexpr int kPrecisionFp64 = 0;
constexpr int kPrecisionSplit = 1;

struct AngularTileParams {
  int kind;
  Arr in;
  int in_slot;
  Arr dt;
  int dt_slot;
  Arr out;
  int out_slot;
  const int* active;
  // per mode: FP64 fragment offset (doubles), split fragment offset (uint2),
  // split column-scale offset (doubles), n_ell of the source band; 4 ints
  // per mode
  const int* offsets;
  const double* fp64;    // [n8][k4][lane] B fragments of T^T
  const uint2* split;    // [n8][k16][slice][lane] BF16 digit fragments
  const double* scales;  // 2^(F_j - 14) per output node
  int spin, boost;
};

__device__ __forceinline__ void dmma_tile(double& c0, double& c1, const double a,
                                          const double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, "
      "{%0,%1};\n"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}

// Stages rows [r0, r0 + rows) of one (mode, slot) plane into split real /
// imaginary shared arrays, K padded with zeros; every thread issues all of
// its loads before its first store.
__device__ __forceinline__ void stage_tile_rows(const double2* src,
                                                const int rows, const int nt,
                                                const int kpad,
                                                double (*re)[kTileStride],
                                                double (*im)[kTileStride]) {
  double2 v[kTileLoads];
#pragma unroll
  for (int u = 0; u < kTileLoads; ++u) {
    const int i = threadIdx.x + u * kTileWarps * 32;
    const int row = i / kpad, k = i - row * kpad;
    v[u] = make_double2(0.0, 0.0);
    if (row < rows && k < nt) v[u] = src[row * nt + k];
  }
#pragma unroll
  for (int u = 0; u < kTileLoads; ++u) {
    const int i = threadIdx.x + u * kTileWarps * 32;
    const int row = i / kpad, k = i - row * kpad;
    if (row < kTileCtaRows) {
      re[row][k] = v[u].x;
      im[row][k] = v[u].y;
    }
  }
}

// Asynchronous 16-byte global -> shared copies (no register round trip), so
// every copy of the operator's fragments is in flight at once.
__device__ __forceinline__ void copy_async_16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                   static_cast<unsigned>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void copy_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// 8-byte words of one operator's fragments.  FP64 projections run as two
// GEMMs, analysis (B = A^T, n_ell columns) then synthesis (B = S^T, K =
// n_ell), so that their output is the synthesis of band coefficients, band
// limited to rounding of its own size as the reference's is; the other FP64
// operations and every split-precision one use the composite nodal matrix.
__host__ __device__ constexpr int tile_operator_words(const int prec, const int kind,
                                                      const int nt, const int ne) {
  const int n8 = (nt + 7) / 8, k4 = (nt + 3) / 4;
  if (prec == kPrecisionSplit) return n8 * ((nt + 15) / 16) * kSplitSlices * 32;
  if (kind == kProject) return ((ne + 7) / 8) * k4 * 32 + n8 * ((ne + 3) / 4) * 32;
  return n8 * k4 * 32;
}

// Dynamic shared memory of the tile operator: the four staged planes and the
// operator's fragments (`frag_words` 8-byte words).
__host__ __device__ constexpr size_t tile_smem_bytes(const int frag_words) {
  return sizeof(double) * (4 * kTileCtaRows * kTileStride +
                           static_cast<size_t>(frag_words));
}

// Independent operations launched together: CTAs [first_block[i],
// first_block[i + 1]) run operation i.
constexpr int kTileMaxOps = 6;
struct AngularTileBatch {
  int count;
  int first_block[kTileMaxOps + 1];
  AngularTileParams ops[kTileMaxOps];
};

template <int PREC>
__global__ void __launch_bounds__(kTileWarps * 32)
    angular_tile_kernel(const Geo g, const Trig tr, const AngularTileBatch batch) {
  int which = 0;
  while (which + 1 < batch.count && static_cast<int>(blockIdx.x) >= batch.first_block[which + 1]) {
    ++which;
  }
  const AngularTileParams& p = batch.ops[which];
  const int block = static_cast<int>(blockIdx.x) - batch.first_block[which];
  extern __shared__ __align__(16) double tile_smem[];
  double (*xr)[kTileStride] = reinterpret_cast<double (*)[kTileStride]>(tile_smem);
  double (*xi)[kTileStride] = xr + kTileCtaRows;
  double (*dr)[kTileStride] = xi + kTileCtaRows;  // d_T x (eth / eth')
  double (*di)[kTileStride] = dr + kTileCtaRows;
  double* sfrag = tile_smem + 4 * kTileCtaRows * kTileStride;
  const int nt = g.nt;
  const int tiles = (g.nr + kTileCtaRows - 1) / kTileCtaRows;
  const int mode = block / tiles;
  const int r0 = (block - mode * tiles) * kTileCtaRows;
  const int rows = min(kTileCtaRows, g.nr - r0);
  double2* out = p.out.at(g, mode, p.out_slot, r0, 0);
  if (!p.active[mode]) {
    for (int i = threadIdx.x; i < rows * nt; i += blockDim.x) {
      out[i] = make_double2(0.0, 0.0);
    }
    return;
  }
  const bool ghp = p.kind == kEth || p.kind == kEthPrime;
  // K padded to the MMA's k granularity; padding columns and rows past the
  // grid are zero
  const int kpad = PREC == kPrecisionSplit ? (nt + 15) / 16 * 16 : (nt + 3) / 4 * 4;
  {  // the mode's operator fragments, copied asynchronously while the rows load
    const double* src = PREC == kPrecisionSplit
                            ? reinterpret_cast<const double*>(p.split + p.offsets[4 * mode + 1])
                            : p.fp64 + p.offsets[4 * mode];
    const int words = tile_operator_words(PREC, p.kind, nt, p.offsets[4 * mode + 3]);
    for (int i = 2 * threadIdx.x; i < words; i += 2 * blockDim.x) {
      copy_async_16(sfrag + i, src + i);
    }
  }
  stage_tile_rows(p.in.at(g, mode, p.in_slot, r0, 0), rows, nt, kpad, xr, xi);
  if (ghp) stage_tile_rows(p.dt.at(g, mode, p.dt_slot, r0, 0), rows, nt, kpad, dr, di);
  copy_async_wait_all();
  // every read of the input rows happens before any store below (the
  // operation may run in place)
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = lane >> 2, q = lane & 3;
  const int half = warp & 1;                        // output node tiles n % 2
  const int row = (warp >> 1) * kTileRows + grp;    // CTA-local row of this lane
  const int n8 = (nt + 7) / 8;
  const double R = g.spacing * static_cast<double>(r0 + row);
  const bool live = row < rows;
  const auto finish = [&](const int j, double re, double im) {
    if (!live || j >= nt) return;
    C2 v = mk(re, im);
    if (ghp) {
      const C2 x = mk(xr[row][j], xi[row][j]);
      const C2 dtv = mk(dr[row][j], di[row][j]);
      v = p.kind == kEth ? eth_point(g, x, dtv, v, p.spin, p.boost, R,
                                     tr.grid_sin[j], tr.grid_cos[j])
                         : ethprime_point(g, x, dtv, v, p.spin, p.boost, R,
                                          tr.grid_sin[j], tr.grid_cos[j]);
    }
    out[row * nt + j] = st(v);
  };
  constexpr int kHalfN8 = kTileMaxNodes / 16;  // n tiles of one warp
  if (PREC == kPrecisionFp64 && p.kind == kProject) {
    // analysis: band coefficients c(row, l), l < n_ell, over K = nodes
    const int ne = p.offsets[4 * mode + 3];
    const int k4 = kpad / 4, n1 = (ne + 7) / 8, kl4 = (ne + 3) / 4;
    const double* f1 = sfrag;
    const double* f2 = sfrag + n1 * k4 * 32;
    double acc[kHalfN8][4];
#pragma unroll
    for (int h = 0; h < kHalfN8; ++h) {
      acc[h][0] = acc[h][1] = acc[h][2] = acc[h][3] = 0.0;
    }
#pragma unroll
    for (int ks = 0; ks < kTileMaxNodes / 4; ++ks) {
      if (ks < k4) {
        const double ar = xr[row][ks * 4 + q];
        const double ai = xi[row][ks * 4 + q];
#pragma unroll
        for (int h = 0; h < kHalfN8; ++h) {
          const int n = 2 * h + half;
          if (n < n1) {
            const double b = f1[(n * k4 + ks) * 32 + lane];
            dmma_tile(acc[h][0], acc[h][1], ar, b);
            dmma_tile(acc[h][2], acc[h][3], ai, b);
          }
        }
      }
    }
    // the coefficients go through the (unused) d_T planes: zero beyond
    // n_ell (their fragments are zero), K-padded for the synthesis
#pragma unroll
    for (int h = 0; h < kHalfN8; ++h) {
      const int n = 2 * h + half;
      if (n < n1) {
        dr[row][n * 8 + 2 * q] = acc[h][0];
        dr[row][n * 8 + 2 * q + 1] = acc[h][1];
        di[row][n * 8 + 2 * q] = acc[h][2];
        di[row][n * 8 + 2 * q + 1] = acc[h][3];
      }
    }
    __syncthreads();
    // synthesis over K = n_ell
#pragma unroll
    for (int h = 0; h < kHalfN8; ++h) {
      acc[h][0] = acc[h][1] = acc[h][2] = acc[h][3] = 0.0;
    }
#pragma unroll
    for (int ks = 0; ks < kTileMaxNodes / 4; ++ks) {
      if (ks < kl4) {
        const double ar = dr[row][ks * 4 + q];
        const double ai = di[row][ks * 4 + q];
#pragma unroll
        for (int h = 0; h < kHalfN8; ++h) {
          const int n = 2 * h + half;
          if (n < n8) {
            const double b = f2[(n * kl4 + ks) * 32 + lane];
            dmma_tile(acc[h][0], acc[h][1], ar, b);
            dmma_tile(acc[h][2], acc[h][3], ai, b);
          }
        }
      }
    }
#pragma unroll
    for (int h = 0; h < kHalfN8; ++h) {
      const int n = 2 * h + half;
      if (n < n8) {
        finish(n * 8 + 2 * q, acc[h][0], acc[h][2]);
        finish(n * 8 + 2 * q + 1, acc[h][1], acc[h][3]);
      }
    }
  } else if constexpr (PREC == kPrecisionFp64) {
    const int k4 = kpad / 4;
    const double* frag = sfrag;
    double acc[kHalfN8][4];
#pragma unroll
    for (int h = 0; h < kHalfN8; ++h) {
      acc[h][0] = acc[h][1] = acc[h][2] = acc[h][3] = 0.0;
    }
    // unrolled over the largest K so the fragment loads of later k steps
    // issue ahead of the MMAs that wait for earlier ones
#pragma unroll
    for (int ks = 0; ks < kTileMaxNodes / 4; ++ks) {
      if (ks < k4) {
        const double ar = xr[row][ks * 4 + q];
        const double ai = xi[row][ks * 4 + q];
#pragma unroll
        for (int h = 0; h < kHalfN8; ++h) {
          const int n = 2 * h + half;
          if (n < n8) {
            const double b = frag[(n * k4 + ks) * 32 + lane];
            dmma_tile(acc[h][0], acc[h][1], ar, b);
            dmma_tile(acc[h][2], acc[h][3], ai, b);
          }
        }
      }
    }
#pragma unroll
    for (int h = 0; h < kHalfN8; ++h) {
      const int n = 2 * h + half;
      if (n < n8) {
        finish(n * 8 + 2 * q, acc[h][0], acc[h][2]);
        finish(n * 8 + 2 * q + 1, acc[h][1], acc[h][3]);
      }
    }
  } else {
    const int k16 = kpad / 16;
    constexpr int kMaxK16 = kTileMaxNodes / 16;
    // per real row (this lane's row: real part, imaginary part) scale over
    // the K nodes; the four lanes of a quad hold the whole row
    double mr = 0.0, mi = 0.0;
#pragma unroll
    for (int ks = 0; ks < kMaxK16; ++ks) {
      if (ks < k16) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int k = ks * 16 + 2 * q + (e & 1) + 8 * (e >> 1);
          mr = fmax(mr, fabs(xr[row][k]));
          mi = fmax(mi, fabs(xi[row][k]));
        }
      }
    }
#pragma unroll
    for (int o = 1; o <= 2; o <<= 1) {
      mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
      mi = fmax(mi, __shfl_xor_sync(0xffffffffu, mi, o));
    }
    const int er = split::exponent(mr), ei = split::exponent(mi);
    const double down_r = ldexp(1.0, -er), down_i = ldexp(1.0, -ei);
    // A fragments: rows 0-7 real parts, rows 8-15 imaginary parts of the
    // tile's 8 complex rows; every slice of every k step
    unsigned a[kMaxK16][kSplitSlices][4];
#pragma unroll
    for (int ks = 0; ks < kMaxK16; ++ks) {
      if (ks < k16) {
        float t[4][2][kSplitSlices];  // [k offset][re, im][slice]
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int k = ks * 16 + 2 * q + (e & 1) + 8 * (e >> 1);
          split::digits(xr[row][k] * down_r, t[e][0]);
          split::digits(xi[row][k] * down_i, t[e][1]);
        }
#pragma unroll
        for (int s = 0; s < kSplitSlices; ++s) {
          a[ks][s][0] = split::pack(t[0][0][s], t[1][0][s]);
          a[ks][s][1] = split::pack(t[0][1][s], t[1][1][s]);
          a[ks][s][2] = split::pack(t[2][0][s], t[3][0][s]);
          a[ks][s][3] = split::pack(t[2][1][s], t[3][1][s]);
        }
      }
    }
    const uint2* frag = reinterpret_cast<const uint2*>(sfrag);
    const double* colscale = p.scales + p.offsets[4 * mode + 2];
    const double up_r = ldexp(1.0, er), up_i = ldexp(1.0, ei);
    for (int n = half; n < n8; n += 2) {
      float d[kSplitSlices][4];  // accumulator of digit pairs with s + t = u
#pragma unroll
      for (int u = 0; u < kSplitSlices; ++u) {
        d[u][0] = d[u][1] = d[u][2] = d[u][3] = 0.0f;
      }
#pragma unroll
      for (int ks = 0; ks < kMaxK16; ++ks) {
        if (ks < k16) {
          uint2 b[kSplitSlices];
#pragma unroll
          for (int t = 0; t < kSplitSlices; ++t) {
            b[t] = frag[((n * k16 + ks) * kSplitSlices + t) * 32 + lane];
          }
#pragma unroll
          for (int s = 0; s < kSplitSlices; ++s) {
#pragma unroll
            for (int t = 0; t + s < kSplitSlices; ++t) {
              split::mma_bf16(d[s + t], a[ks][s], b[t]);
            }
          }
        }
      }
      double v[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) v[c] = split::recombine(d, c);
      const int j = n * 8 + 2 * q;
      const double s0 = colscale[j], s1 = colscale[j + 1];
      finish(j, v[0] * up_r * s0, v[2] * up_i * s0);
      finish(j + 1, v[1] * up_r * s1, v[3] * up_i * s1);
    }
  }
}

// ------------------------------------------------------------- Teukolsky
// Point coefficients (include/teuk/teukolsky.hpp:38-85) at (R, theta, m).
struct TC {
  double time, K, HR;
  C2 G, q, c;
};
__device__ TC teuk_coefs(const Geo& g, const double R, const double sin_t,
                         const double cos_t, const int m) {
  const double M = g.mass, a = g.spin, L = g.length;
  const double L2 = L * L, L4 = L2 * L2, R2 = R * R, a2 = a * a;
  const double mrl = M * R / L2;
  const double s = -2.0, mm = static_cast<double>(m);
  TC k;
  k.time = 8.0 * M * (2.0 * M - a2 * R / L2) * (1.0 + 2.0 * mrl) -
           a2 * sin_t * sin_t;
  k.K = L2 - (8.0 * M * M - a2) * R2 / L2 + 4.0 * a2 * M * R * R2 / L4;
  k.HR = R2 / L4 * (L4 - 2.0 * L2 * M * R + a2 * R2);
  const C2 g1 = mk(0.0, 2.0 * a * mm * (1.0 + 4.0 * mrl));
  const double g2 = 2.0 * M * (-s + (2.0 + s) * 2.0 * mrl - 3.0 * a2 * R2 / L4) -
                    a2 * R / L2;
  k.G = g1 + mk(2.0 * g2, 2.0 * (s * a * cos_t));
  k.q = mk(2.0 * R * (1.0 + s - (3.0 + s) * mrl + 2.0 * a2 * R2 / L4),
           -(2.0 * a * mm * R2 / L2));
  k.c = mk(-2.0 * R * ((1.0 + s) * M / L2 - a2 * R / L4),
           -(2.0 * a * mm * R / L2));
  return k;
}

struct TeukParams {
  Arr stage;
  int f0;  // first field offset (P) of the triple: 0 or 10
  Arr scratch;
  Arr lap;
  int lap_slot;
  const double2* forcing;  // (mode, r, theta) or null for zero
  Arr out;
};

// TeukolskyPrepareReductionFunctor (include/teuk/full_spatial.hpp:99-134)
__global__ void teuk_prepare_kernel(const Geo g, const TeukParams p) {
  const long long total = static_cast<long long>(g.modes) * g.nr * g.nt;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < total; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int t = static_cast<int>(i % g.nt);
    const int r = static_cast<int>((i / g.nt) % g.nr);
    const int mode = static_cast<int>(i / (static_cast<long long>(g.nt) * g.nr));
    const C2 dpsi = deriv(g.disc, p.stage.line(g, mode, p.f0 + 2, t), g.nt,
                          g.nr, r, g.inv_spacing);
    *p.scratch.at(g, mode, kDrPsi, r, t) = st(dpsi);
    *p.scratch.at(g, mode, kEffQ, r, t) =
        g.reduction == 1 ? st(dpsi) : *p.stage.at(g, mode, p.f0 + 1, r, t);
  }
}

// TeukolskySpatialPrimitivesFunctor (include/teuk/full_spatial.hpp:136-182)
__global__ void teuk_primitives_kernel(const Geo g, const Trig tr,
                                       const TeukParams p) {
  const long long total = static_cast<long long>(g.modes) * g.nr * g.nt;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < total; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int t = static_cast<int>(i % g.nt);
    const int r = static_cast<int>((i / g.nt) % g.nr);
    const int mode = static_cast<int>(i / (static_cast<long long>(g.nt) * g.nr));
    const C2 dq = deriv(g.disc, p.scratch.line(g, mode, kEffQ, t), g.nt, g.nr,
                        r, g.inv_spacing);
    *p.scratch.at(g, mode, kDrQ, r, t) = st(dq);
    const TC k = teuk_coefs(g, g.spacing * r, tr.theta_sin[t], tr.theta_cos[t],
                            tr.mvals[mode]);
    const C2 P = ld(*p.stage.at(g, mode, p.f0, r, t));
    const C2 Q = ld(*p.scratch.at(g, mode, kEffQ, r, t));
    const C2 psi = ld(*p.stage.at(g, mode, p.f0 + 2, r, t));
    const C2 vel = (P + (2.0 * k.K) * Q - k.G * psi) / k.time;
    *p.scratch.at(g, mode, kVel, r, t) = st(vel);
  }
}

// TeukolskyRhsFunctor (include/teuk/full_spatial.hpp:184-280)
__global__ void __launch_bounds__(kBlock, kPointBlocks) teuk_rhs_kernel(const Geo g, const Trig tr,
                                const TeukParams p) {
  const long long total = static_cast<long long>(g.modes) * g.nr * g.nt;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < total; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int t = static_cast<int>(i % g.nt);
    const int r = static_cast<int>((i / g.nt) % g.nr);
    const int mode = static_cast<int>(i / (static_cast<long long>(g.nt) * g.nr));
    const C2 dvel = deriv(g.disc, p.scratch.line(g, mode, kVel, t), g.nt,
                          g.nr, r, g.inv_spacing);
    *p.scratch.at(g, mode, kDrVel, r, t) = st(dvel);
    const TC k = teuk_coefs(g, g.spacing * r, tr.theta_sin[t], tr.theta_cos[t],
                            tr.mvals[mode]);
    const C2 Qe = ld(*p.scratch.at(g, mode, kEffQ, r, t));
    const C2 psi = ld(*p.stage.at(g, mode, p.f0 + 2, r, t));
    const C2 constraint = ld(*p.stage.at(g, mode, p.f0 + 1, r, t)) -
                          ld(*p.scratch.at(g, mode, kDrPsi, r, t));
    const C2 lap = ld(*p.lap.at(g, mode, p.lap_slot, r, t));
    const C2 forcing =
        p.forcing != nullptr
            ? ld(p.forcing[(static_cast<long long>(mode) * g.nr + r) * g.nt + t])
            : mk(0.0, 0.0);
    C2 pt = k.HR * ld(*p.scratch.at(g, mode, kDrQ, r, t)) + k.q * Qe +
            k.c * psi + lap + forcing;
    C2 qt = dvel - g.damping * constraint;
    C2 vt = ld(*p.scratch.at(g, mode, kVel, r, t));
    if (g.dissipation > 0.0) {
      // the tables hold -(A^T A)/H, so sigma/h completes the operator
      const double scale = g.dissipation * g.inv_spacing;
      pt = pt + scale * diss(g.disc, p.stage.line(g, mode, p.f0, t), g.nt, g.nr, r);
      qt = qt + scale * diss(g.disc, p.stage.line(g, mode, p.f0 + 1, t), g.nt, g.nr, r);
      vt = vt + scale * diss(g.disc, p.stage.line(g, mode, p.f0 + 2, t), g.nt, g.nr, r);
    }
    *p.out.at(g, mode, p.f0, r, t) = st(pt);
    *p.out.at(g, mode, p.f0 + 1, r, t) = st(qt);
    *p.out.at(g, mode, p.f0 + 2, r, t) = st(vt);
  }
}

// ------------------------------------------------------------- reconstruction
__global__ void recon_radial_kernel(const Geo g, const Arr stage, Arr out) {
  const long long total = static_cast<long long>(g.modes) * 7 * g.nr * g.nt;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < total; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int t = static_cast<int>(i % g.nt);
    const int r = static_cast<int>((i / g.nt) % g.nr);
    const long long mf = i / (static_cast<long long>(g.nt) * g.nr);
    const int f = static_cast<int>(mf % 7), mode = static_cast<int>(mf / 7);
    *out.at(g, mode, f, r, t) = st(deriv(g.disc, stage.line(g, mode, kG + f, t),
                                         g.nt, g.nr, r, g.inv_spacing));
  }
}

struct ReconParams {
  Arr stage;
  Arr out;
  Arr rr;   // radial derivatives, compact slots
  Arr ang;  // reconstruction angular inputs
};

// evaluate_sbp_reconstruction_full_pass{1,2,3}
// (include/teuk/full_spatial.hpp:494-695, reconstruction.hpp:46-121)
template <int PASS>
__global__ void __launch_bounds__(kBlock, kPointBlocks) recon_pass_kernel(const Geo g, const Trig tr,
                                  const ReconParams p) {
  const long long total = static_cast<long long>(g.modes) * g.nr * g.nt;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < total; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int t = static_cast<int>(i % g.nt);
    const int r = static_cast<int>((i / g.nt) % g.nr);
    const int mode = static_cast<int>(i / (static_cast<long long>(g.nt) * g.nr));
    const double R = g.spacing * r;
    const double R2 = R * R;
    const Bg b = background(g, R, tr.theta_cos[t], tr.theta_sin[t]);
    const auto S = [&](const int f) { return ld(*p.stage.at(g, mode, f, r, t)); };
    const auto D = [&](const int f) { return ld(*p.rr.at(g, mode, f, r, t)); };
    const auto A = [&](const int f) { return ld(*p.ang.at(g, mode, f, r, t)); };
    if (PASS == 1) {
      const C2 G = S(kG), Lm = S(kLambda), F = S(kFirstPsi);
      const C2 dG = (-4.0 * R) * b.mu0 * G + A(aEth1F) - (R * b.tau0) * F;
      const C2 dL = -R * (b.mu0 + conj(b.mu0)) * Lm - F;
      *p.out.at(g, mode, kG, r, t) = st(recon_dt(g, G, D(rG), dG, 2, R));
      *p.out.at(g, mode, kLambda, r, t) = st(recon_dt(g, Lm, D(rLambda), dL, 1, R));
    } else if (PASS == 2) {
      const C2 mu_bar = conj(b.mu0), pi_bar = conj(b.pi0);
      const C2 G = S(kG), Lm = S(kLambda), H = S(kH), B = S(kB), Pi = S(kPi),
               C = S(kC);
      const C2 dH = (-3.0 * R) * b.mu0 * H + A(aEth2G) - (2.0 * R) * b.tau0 * G;
      const C2 dB = R * (b.mu0 - mu_bar) * B - 2.0 * Lm;
      const C2 dPi = -G - R * (pi_bar + b.tau0) * Lm +
                     (0.5 * R2) * b.mu0 * (pi_bar + b.tau0) * B;
      const C2 dC = -R * mu_bar * C - 2.0 * Pi - R * b.tau0 * B;
      *p.out.at(g, mode, kH, r, t) = st(recon_dt(g, H, D(rH), dH, 3, R));
      *p.out.at(g, mode, kB, r, t) = st(recon_dt(g, B, D(rB), dB, 1, R));
      *p.out.at(g, mode, kPi, r, t) = st(recon_dt(g, Pi, D(rPi), dPi, 2, R));
      *p.out.at(g, mode, kC, r, t) = st(recon_dt(g, C, D(rC), dC, 2, R));
    } else {
      const int sh = tr.sharp[mode];
      const C2 mu_bar = conj(b.mu0), pi_bar = conj(b.pi0), tau_bar = conj(b.tau0);
      const C2 C = S(kC), U = S(kU), Pi = S(kPi), H = S(kH);
      const C2 Pi_s = conj(ld(*p.stage.at(g, sh, kPi, r, t)));
      const C2 B_s = conj(ld(*p.stage.at(g, sh, kB, r, t)));
      const C2 C_s = conj(ld(*p.stage.at(g, sh, kC, r, t)));
      const C2 u_transport = -R * mu_bar * U;
      const C2 c_eth = -R * b.mu0 * A(aEth2C);
      const C2 c_conn = -R2 * b.mu0 * (pi_bar + 2.0 * b.tau0) * C;
      const C2 pi_eth = -2.0 * A(aEth2Pi);
      const C2 pi_conn = (-2.0 * R) * pi_bar * Pi;
      const C2 psi2 = -2.0 * H;
      const C2 sharp_pi = (-2.0 * R) * b.pi0 * Pi_s;
      const C2 sharp_b_eth = -R * b.pi0 * A(aEthP1BSharp);
      const C2 sharp_b_conn = R2 * b.pi0 * b.pi0 * B_s;
      const C2 sharp_c_eth = R * b.mu0 * A(aEthP2CSharp);
      const C2 sharp_c_conn = R2 * ((-3.0 * b.mu0) * b.pi0 + (2.0 * mu_bar) * b.pi0 -
                                    (2.0 * b.mu0) * tau_bar) * C_s;
      const C2 dU = u_transport + c_eth + c_conn + pi_eth + pi_conn + psi2 +
                    sharp_pi + sharp_b_eth + sharp_b_conn + sharp_c_eth +
                    sharp_c_conn;
      *p.out.at(g, mode, kU, r, t) = st(recon_dt(g, U, D(rU), dU, 3, R));
    }
  }
}

// pack_sharp_fields (include/teuk/spatial_pipeline.hpp:895-931)
__global__ void pack_sharp_kernel(const Geo g, const Trig tr, const Arr stage,
                                  const Arr dt, Arr work) {
  const long long total = static_cast<long long>(g.modes) * g.nr * g.nt;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < total; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int t = static_cast<int>(i % g.nt);
    const int r = static_cast<int>((i / g.nt) % g.nr);
    const int mode = static_cast<int>(i / (static_cast<long long>(g.nt) * g.nr));
    const int src = tr.sharp[mode];
    *work.at(g, mode, shB, r, t) = st(conj(ld(*stage.at(g, src, kB, r, t))));
    *work.at(g, mode, shC, r, t) = st(conj(ld(*stage.at(g, src, kC, r, t))));
    *work.at(g, mode, shBDt, r, t) = st(conj(ld(*dt.at(g, src, kB, r, t))));
    *work.at(g, mode, shCDt, r, t) = st(conj(ld(*dt.at(g, src, kC, r, t))));
  }
}

// independent reconstruction constraints
// (include/teuk/spatial_pipeline.hpp:768-893, reconstruction_constraints.hpp:30-81)
struct ConstraintParams {
  Arr stage, dt, first_scratch, rr, ang, constraints, terms;
};
__global__ void constraints_kernel(const Geo g, const Trig tr,
                                   const ConstraintParams p) {
  const long long total = static_cast<long long>(g.modes) * g.nr * g.nt;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < total; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int t = static_cast<int>(i % g.nt);
    const int r = static_cast<int>((i / g.nt) % g.nr);
    const int mode = static_cast<int>(i / (static_cast<long long>(g.nt) * g.nr));
    const double R = g.spacing * r;
    const double c = tr.grid_cos[t];
    const Bg b = background(g, R, c, tr.grid_sin[t]);
    const auto S = [&](const int f) { return ld(*p.stage.at(g, mode, f, r, t)); };
    const C2 F = S(kFirstPsi), G = S(kG), H = S(kH);
    const int m = tr.mvals[mode];
    const C2 thorn1F = thorn_n(g, F, ld(*p.dt.at(g, mode, kFirstPsi, r, t)),
                               ld(*p.first_scratch.at(g, mode, kDrPsi, r, t)),
                               1, -2, -2, m, R, c, b.eps0);
    const C2 thorn2G = thorn_n(g, G, ld(*p.dt.at(g, mode, kG, r, t)),
                               ld(*p.rr.at(g, mode, rG, r, t)), 2, -1, -1, m, R,
                               c, b.eps0);
    const C2 ethp2G = ld(*p.ang.at(g, mode, 0, r, t));
    const C2 ethp3H = ld(*p.ang.at(g, mode, 1, r, t));
    const double R2 = R * R, R3 = R2 * R;
    const C2 psi3_left = R * ethp2G + (4.0 * R2) * b.pi0 * G + b.rho0 * F;
    const C2 psi3_right = thorn1F + (3.0 * R2) * b.psi20 * S(kLambda);
    const C2 bg_terms = b.psi20 * ((-3.0 * R3) * b.mu0 * S(kC) -
                                   (1.5 * R3) * b.tau0 * S(kB) -
                                   (3.0 * R2) * S(kPi));
    const C2 psi2_left = thorn2G - 2.0 * b.rho0 * G;
    const C2 psi2_right = R * ethp3H + (3.0 * R2) * b.pi0 * H - bg_terms;
    const C2 U_sharp = conj(ld(*p.stage.at(g, tr.sharp[mode], kU, r, t)));
    const C2 hll_left = S(kU) / b.mu0;
    const C2 hll_right = U_sharp / conj(b.mu0);
    *p.constraints.at(g, mode, 0, r, t) = st(psi3_left - psi3_right);
    *p.constraints.at(g, mode, 1, r, t) = st(psi2_left - psi2_right);
    *p.constraints.at(g, mode, 2, r, t) = st(hll_left - hll_right);
    *p.terms.at(g, mode, 0, r, t) = st(psi3_left);
    *p.terms.at(g, mode, 1, r, t) = st(psi3_right);
    *p.terms.at(g, mode, 2, r, t) = st(psi2_left);
    *p.terms.at(g, mode, 3, r, t) = st(psi2_right);
    *p.terms.at(g, mode, 4, r, t) = st(hll_left);
    *p.terms.at(g, mode, 5, r, t) = st(hll_right);
  }
}

// ------------------------------------------------------------- source
struct SourceInputParams {
  Arr stage, dt, ddt, first_scratch, tangent_scratch, rr, rr_t, ang, ang_t,
      extra, fields, field_t, deriv, deriv_t;
};
// prepare_source_inputs (include/teuk/spatial_pipeline.hpp:961-1181)
__global__ void source_inputs_kernel(const Geo g, const Trig tr,
                                     const SourceInputParams p) {
  const long long total = static_cast<long long>(g.modes) * g.nr * g.nt;
  const int state_slots[8] = {kFirstPsi, kG, kH, kLambda, kPi, kB, kC, kU};
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < total; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int t = static_cast<int>(i % g.nt);
    const int r = static_cast<int>((i / g.nt) % g.nr);
    const int mode = static_cast<int>(i / (static_cast<long long>(g.nt) * g.nr));
    const int sh = tr.sharp[mode];
    const double R = g.spacing * r;
    for (int k = 0; k < 8; ++k) {
      *p.fields.at(g, mode, k, r, t) = *p.stage.at(g, mode, state_slots[k], r, t);
      *p.field_t.at(g, mode, k, r, t) = *p.dt.at(g, mode, state_slots[k], r, t);
    }
    const auto V = [&](const Arr& a, const int m, const int f) {
      return ld(*a.at(g, m, f, r, t));
    };
    const auto set = [&](const int slot, const C2 v, const C2 d) {
      *p.deriv.at(g, mode, slot, r, t) = st(v);
      *p.deriv_t.at(g, mode, slot, r, t) = st(d);
    };
    set(dDelta1F,
        delta_n(g, V(p.stage, mode, kFirstPsi), V(p.dt, mode, kFirstPsi),
                V(p.first_scratch, mode, kDrPsi), 1, R),
        delta_n(g, V(p.dt, mode, kFirstPsi), V(p.ddt, mode, kFirstPsi),
                V(p.tangent_scratch, mode, kDrPsi), 1, R));
    set(dDelta3U,
        delta_n(g, V(p.stage, mode, kU), V(p.dt, mode, kU), V(p.rr, mode, rU), 3, R),
        delta_n(g, V(p.dt, mode, kU), V(p.ddt, mode, kU), V(p.rr_t, mode, rU), 3, R));
    set(dEth2C, V(p.ang, mode, aEth2C), V(p.ang_t, mode, aEth2C));
    set(dEthP2CSharp, V(p.ang, mode, aEthP2CSharp), V(p.ang_t, mode, aEthP2CSharp));
    set(dEth1B, V(p.extra, mode, xEth1B), V(p.extra, mode, xEth1BT));
    set(dDelta2C,
        delta_n(g, V(p.stage, mode, kC), V(p.dt, mode, kC), V(p.rr, mode, rC), 2, R),
        delta_n(g, V(p.dt, mode, kC), V(p.ddt, mode, kC), V(p.rr_t, mode, rC), 2, R));
    set(dDelta2G,
        delta_n(g, V(p.stage, mode, kG), V(p.dt, mode, kG), V(p.rr, mode, rG), 2, R),
        delta_n(g, V(p.dt, mode, kG), V(p.ddt, mode, kG), V(p.rr_t, mode, rG), 2, R));
    set(dEth2G, V(p.ang, mode, aEth2G), V(p.ang_t, mode, aEth2G));
    set(dEthP1F, V(p.extra, mode, xEthP1F), V(p.extra, mode, xEthP1FT));
    set(dDelta2CSharp,
        delta_n(g, conj(V(p.stage, sh, kC)), conj(V(p.dt, sh, kC)),
                conj(V(p.rr, sh, rC)), 2, R),
        delta_n(g, conj(V(p.dt, sh, kC)), conj(V(p.ddt, sh, kC)),
                conj(V(p.rr_t, sh, rC)), 2, R));
    set(dEthP1BSharp, V(p.ang, mode, aEthP1BSharp), V(p.ang_t, mode, aEthP1BSharp));
  }
}

struct InnerParams {
  Arr fields, field_t, deriv, deriv_t;
  Arr sum, sum_t;        // (mode, 2, r, theta)
  Arr pair, pair_t;      // (pair, 2, r, theta)
  const int* index1;
  const int* index2;
  const int* offsets;
  const int* targets;
  int target_count;
};

// corrected_ordered_pair_source with its Jet1 tangent
// (include/teuk/second_order.hpp:74-142, source_tangent_spatial.hpp:65-226)
__global__ void inner_source_kernel(const Geo g, const Trig tr,
                                    const InnerParams p) {
  const long long total = static_cast<long long>(p.target_count) * g.nr * g.nt;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < total; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int t = static_cast<int>(i % g.nt);
    const int r = static_cast<int>((i / g.nt) % g.nr);
    const int slot = static_cast<int>(i / (static_cast<long long>(g.nt) * g.nr));
    const int target = p.targets[slot];
    const double R = g.spacing * r, R2 = R * R;
    const Bg b = background(g, R, tr.grid_cos[t], tr.grid_sin[t]);
    const C2 mu_bar = conj(b.mu0), pi_bar = conj(b.pi0), tau_bar = conj(b.tau0);
    J totD{mk(0, 0), mk(0, 0)}, totT{mk(0, 0), mk(0, 0)};
    for (int pi = p.offsets[slot]; pi < p.offsets[slot + 1]; ++pi) {
      const int m1 = p.index1[pi], m2 = p.index2[pi];
      const int s1 = tr.sharp[m1], s2 = tr.sharp[m2];
      const auto fld = [&](const int m, const int c) {
        return J{ld(*p.fields.at(g, m, c, r, t)), ld(*p.field_t.at(g, m, c, r, t))};
      };
      const auto der = [&](const int m, const int c) {
        return J{ld(*p.deriv.at(g, m, c, r, t)), ld(*p.deriv_t.at(g, m, c, r, t))};
      };
      const J F1 = fld(m1, sF), G1 = fld(m1, sG), L1 = fld(m1, sLambda),
              Pi1 = fld(m1, sPi), B1 = fld(m1, sB), C1 = fld(m1, sC),
              U1 = fld(m1, sU);
      const J F2 = fld(m2, sF), G2 = fld(m2, sG), H2 = fld(m2, sH),
              B2 = fld(m2, sB), C2v = fld(m2, sC), U2 = fld(m2, sU);
      const J U2s = jconj(fld(s2, sU)), C2s = jconj(fld(s2, sC)),
              C1s = jconj(fld(s1, sC)), B1s = jconj(fld(s1, sB)),
              Pi2s = jconj(fld(s2, sPi)), B2s = jconj(fld(s2, sB));
      const J d1F2 = der(m2, dDelta1F), d3U2 = der(m2, dDelta3U),
              e2C2 = der(m2, dEth2C), ep2C2s = der(m2, dEthP2CSharp),
              e1B2 = der(m2, dEth1B), d2C2 = der(m2, dDelta2C),
              d2G2 = der(m2, dDelta2G), e2G2 = der(m2, dEth2G),
              ep1F2 = der(m2, dEthP1F), d2C2s = der(m2, dDelta2CSharp),
              ep1B2s = der(m2, dEthP1BSharp);
      const J sd0102 = 0.5 * U1 * (d1F2 / b.mu0 + R * F2);
      const J sd03 = F1 * (0.5 * R * e2C2);
      const J sd04 = F1 * ((0.5 * R2) * (pi_bar + 2.0 * b.tau0) * C2v);
      const J sd05 = F1 * (d3U2 / b.mu0 + R * U2s);
      const J sd06 = F1 * (-0.5 * R * ep2C2s);
      const J sd07 = F1 * ((0.5 * R2) * (5.0 * b.pi0 + 4.0 * tau_bar) * C2s);
      const J sd08 = -0.5 * G1 * (R * e1B2);
      const J sd09 = -0.5 * G1 * (R2 * (pi_bar + b.tau0) * B2);
      const J sd10 = -0.5 * G1 * (R * d2C2);
      const J sd11 = -0.5 * G1 * (R2 * (-2.0 * b.mu0 + mu_bar) * C2v);
      const J sd12 = -R * C1 * d2G2;
      const J sd13 = 0.5 * R * B1 * e2G2;
      const J sd14 = 4.0 * R * Pi1 * G2;
      const J sd15 = -3.0 * R * L1 * H2;
      const J st0102 = -C1s * (d1F2 + R * (b.mu0 + 2.0 * mu_bar) * F2);
      const J st03 = 0.5 * B1s * ep1F2;
      const J st04 = F1 * Pi2s;
      const J st05 = -F1 * d2C2s;
      const J st06 = F1 * ep1B2s;
      const J st07 = F1 * (-0.5 * R * (b.pi0 + tau_bar) * B2s);
      const J D = sd0102 + sd03 + sd04 + sd05 + sd06 + sd07 + sd08 + sd09 +
                  sd10 + sd11 + sd12 + sd13 + sd14 + sd15;
      const J T = st0102 + st03 + st04 + st05 + st06 + st07;
      *p.pair.at(g, pi, 0, r, t) = st(D.v);
      *p.pair.at(g, pi, 1, r, t) = st(T.v);
      *p.pair_t.at(g, pi, 0, r, t) = st(D.d);
      *p.pair_t.at(g, pi, 1, r, t) = st(T.d);
      totD = totD + D;
      totT = totT + T;
    }
    *p.sum.at(g, target, 0, r, t) = st(totD.v);
    *p.sum.at(g, target, 1, r, t) = st(totT.v);
    *p.sum_t.at(g, target, 0, r, t) = st(totD.d);
    *p.sum_t.at(g, target, 1, r, t) = st(totT.d);
  }
}

// evaluate_spatial_outer_source_from_ethprime
// (include/teuk/source_spatial.hpp:358-424, second_order.hpp:152-182)
__global__ void outer_source_kernel(const Geo g, const Trig tr, const Arr inner,
                                    const Arr inner_t, const double2* ethp_t,
                                    double2* source_over_r3, double2* forcing) {
  const long long total = static_cast<long long>(g.modes) * g.nr * g.nt;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < total; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int t = static_cast<int>(i % g.nt);
    const int r = static_cast<int>((i / g.nt) % g.nr);
    const int mode = static_cast<int>(i / (static_cast<long long>(g.nt) * g.nr));
    const double R = g.spacing * r;
    const C2 Dv = ld(*inner.at(g, mode, 0, r, t));
    const C2 Tv = ld(*inner.at(g, mode, 1, r, t));
    const C2 dD = deriv(g.disc, inner.line(g, mode, 0, t), g.nt, g.nr, r,
                        g.inv_spacing);
    const C2 delta3D = delta_n(g, Dv, ld(*inner_t.at(g, mode, 0, r, t)), dD, 3, R);
    const double c = tr.grid_cos[t];
    const Bg b = background(g, R, c, tr.grid_sin[t]);
    const C2 s01 = delta3D;
    const C2 s02 = R * (4.0 * b.mu0 + conj(b.mu0)) * Dv;
    const C2 s03 = R * ld(ethp_t[i]);
    const C2 s04 = R * R * (4.0 * b.pi0 - conj(b.tau0)) * Tv;
    const C2 source = s01 + s02 + s03 + s04;
    source_over_r3[i] = st(source);
    const double L2 = g.length * g.length, L4 = L2 * L2;
    const double norm = 2.0 * (L4 + g.spin * g.spin * R * R * c * c);
    forcing[i] = st(norm * source);
  }
}

// ------------------------------------------------------------- RK4 + norms
__global__ void axpy_kernel(const double2* y, const double2* k, double2* out,
                            const double scale, const long long n) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < n; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    out[i] = st(ld(y[i]) + scale * ld(k[i]));
  }
}
__global__ void accumulate_kernel(double2* y, const double2* k1,
                                  const double2* k2, const double2* k3,
                                  const double2* k4, const double scale,
                                  const long long n) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < n; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const C2 sum = ld(k1[i]) + 2.0 * ld(k2[i]) + 2.0 * ld(k3[i]) + ld(k4[i]);
    y[i] = st(ld(y[i]) + scale * sum);
  }
}

__device__ void atomic_max_double(double* address, const double value) {
  unsigned long long* a = reinterpret_cast<unsigned long long*>(address);
  unsigned long long old = *a;
  while (__longlong_as_double(static_cast<long long>(old)) < value) {
    const unsigned long long assumed = old;
    old = atomicCAS(a, assumed,
                    static_cast<unsigned long long>(__double_as_longlong(value)));
    if (old == assumed) break;
  }
}

// SourceConstraintEvaluator::sample, first reduction
// (include/teuk/source_activation.hpp:127-160)
__global__ void norms_natural_kernel(const Geo g, const Arr residuals,
                                     const Arr terms, const double* weights,
                                     double* acc, int* finite) {
  // acc: [0..2] weighted c^2, [3..5] weighted l^2, [6..8] weighted r^2,
  //      [9..11] max c^2, [12..14] max natural^2, [15..17] max normalized^2
  const long long total = static_cast<long long>(g.modes) * g.nr * g.nt;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < total; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int t = static_cast<int>(i % g.nt);
    const int r = static_cast<int>((i / g.nt) % g.nr);
    const int mode = static_cast<int>(i / (static_cast<long long>(g.nt) * g.nr));
    const double w = g.spacing * weights[g.nt + r] * kTwoPi * weights[t];
    for (int f = 0; f < 3; ++f) {
      const double c = cabs2(ld(*residuals.at(g, mode, f, r, t)));
      const double l = cabs2(ld(*terms.at(g, mode, 2 * f, r, t)));
      const double rr = cabs2(ld(*terms.at(g, mode, 2 * f + 1, r, t)));
      if (!isfinite(c) || !isfinite(l) || !isfinite(rr)) {
        atomicExch(finite, 0);
        continue;
      }
      atomicAdd(&acc[f], w * c * c);
      atomicAdd(&acc[3 + f], w * l * l);
      atomicAdd(&acc[6 + f], w * rr * rr);
      atomic_max_double(&acc[9 + f], c * c);
      atomic_max_double(&acc[12 + f], fmax(l * l, rr * rr));
    }
  }
}

// second reduction (include/teuk/source_activation.hpp:161-186)
__global__ void norms_normalized_kernel(const Geo g, const Arr residuals,
                                        const Arr terms, double* acc,
                                        int* finite) {
  const double floor = 64.0 * 2.220446049250313e-16;
  const long long total = static_cast<long long>(g.modes) * g.nr * g.nt;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < total; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int t = static_cast<int>(i % g.nt);
    const int r = static_cast<int>((i / g.nt) % g.nr);
    const int mode = static_cast<int>(i / (static_cast<long long>(g.nt) * g.nr));
    for (int f = 0; f < 3; ++f) {
      const double c = cabs2(ld(*residuals.at(g, mode, f, r, t)));
      const double l = cabs2(ld(*terms.at(g, mode, 2 * f, r, t)));
      const double rr = cabs2(ld(*terms.at(g, mode, 2 * f + 1, r, t)));
      const double scale = sqrt(acc[12 + f]);
      const double den = l + rr + floor * scale;
      const double normalized = den > 0.0 ? c / den : 0.0;
      if (isfinite(normalized)) {
        atomic_max_double(&acc[15 + f], normalized * normalized);
      } else {
        atomicExch(finite, 0);
      }
    }
  }
}

__device__ __forceinline__ double dwarp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double dwarp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ bool finite2(const C2 v) {
  return isfinite(v.re) && isfinite(v.im);
}

// One warp-reduced sum / max per slot and iteration; the first lane adds
// them to the device accumulators.
__device__ void reduce_slot(const DiagnosticsLaunch& p, const int slot,
                            const double value, const int lane) {
  const double s = dwarp_sum(value);
  const double m = dwarp_max(value);
  if (lane == 0) {
    atomicAdd(&p.sums[slot], s);
    atomicMax(&p.maxima[slot],
              static_cast<unsigned long long>(__double_as_longlong(m)));
  }
}

__global__ void diagnostics_kernel(const DiagnosticsLaunch p) {
  // flags: 0 state, 1 rhs, 2 first constraint, 3 second constraint,
  // 4 source, 5 forcing, 6 scri, 7 horizon
  const int lane = threadIdx.x & 31;
  const long long total = static_cast<long long>(p.modes) * p.nr * p.nt;
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  const long long rounds = (total + stride - 1) / stride;
  for (long long k = 0; k < rounds; ++k) {
    const long long i = k * stride + blockIdx.x * static_cast<long long>(blockDim.x) +
                        threadIdx.x;
    const bool in = i < total;
    int t = 0, r = 0, mode = 0;
    if (in) {
      t = static_cast<int>(i % p.nt);
      r = static_cast<int>((i / p.nt) % p.nr);
      mode = static_cast<int>(i / (static_cast<long long>(p.nt) * p.nr));
    }
    const bool scri = in && r == 0, horizon = in && r + 1 == p.nr;
    const auto bad = [&](const int flag) {
      atomicExch(&p.finite[flag], 0);
      if (scri) atomicExch(&p.finite[6], 0);
      if (horizon) atomicExch(&p.finite[7], 0);
    };
    const auto at = [&](const double2* a, const int f) {
      return a + ((static_cast<long long>(mode) * kFieldCount + f) * p.nr + r) * p.nt + t;
    };
    for (int f = 0; f < kFieldCount; ++f) {
      double sv = 0.0, rv = 0.0;
      if (in) {
        const C2 v = ld(*at(p.state, f));
        if (finite2(v)) {
          sv = v.re * v.re + v.im * v.im;
        } else {
          bad(0);
        }
        if (p.rhs != nullptr) {
          const C2 w = ld(*at(p.rhs, f));
          if (finite2(w)) {
            rv = w.re * w.re + w.im * w.im;
          } else {
            bad(1);
          }
        }
      }
      reduce_slot(p, f, sv, lane);
      reduce_slot(p, kFieldCount + f, rv, lane);
    }
    for (int c = 0; c < 2; ++c) {
      double v2 = 0.0;
      if (in) {
        const int q = c == 0 ? kFirstQ : kSecondQ;
        const int psi = c == 0 ? kFirstPsi : kSecondPsi;
        const C2 d = deriv(p.disc, at(p.state, psi) - static_cast<long long>(r) * p.nt,
                           p.nt, p.nr, r, p.inv_spacing);
        const C2 v = ld(*at(p.state, q)) - d;
        if (finite2(v)) {
          v2 = v.re * v.re + v.im * v.im;
        } else {
          atomicExch(&p.finite[2 + c], 0);
        }
      }
      reduce_slot(p, 2 * kFieldCount + c, v2, lane);
    }
    for (int c = 0; c < 2; ++c) {
      const double2* a = c == 0 ? p.source : p.forcing;
      double v2 = 0.0;
      if (in && a != nullptr) {
        const C2 v = ld(a[i]);
        if (finite2(v)) {
          v2 = v.re * v.re + v.im * v.im;
        } else {
          bad(4 + c);
        }
      }
      reduce_slot(p, 2 * kFieldCount + 2 + c, v2, lane);
    }
  }
}

int grid_for(const long long n) {
  const long long b = (n + kBlock - 1) / kBlock;
  return static_cast<int>(b < 8192 ? (b > 0 ? b : 1) : 8192);
}

void check(const cudaError_t err, const char* what) {
  if (err != cudaSuccess) {
    throw DeviceError(std::string(what) + ": " + cudaGetErrorString(err));
  }
}

// complex values per (mode, r, theta) point: nine 13-field buffers (state,
// RK stage, k1..k4, RHS input/output, tangent RHS) plus the scratch slots
constexpr std::size_t kFullBuffers = 9;
constexpr std::size_t kScratchSlots = 3 + 6 + 6 + 2 + 3 + 6 + 4 + 4 + 5 + 5 + 5 +
                                      7 + 7 + 8 + 8 + 11 + 11 + 2 + 2 + 2 + 2 +
                                      1 + 1 + 1;

}  // namespace

// ------------------------------------------------------------- host side
struct NodalPipeline::Buffers {
  Geo geo{};
  Trig trig{};
  size_t plane = 0;  // complex values per (mode, slot)
  // device allocations (double2 unless noted)
  double2 *state = nullptr, *stage = nullptr, *k[4] = {nullptr, nullptr, nullptr, nullptr};
  double2 *rhs_in = nullptr, *rhs_out = nullptr;
  double2 *lin_ang = nullptr, *rec_ang = nullptr, *rec_ang_t = nullptr,
          *ind_ang = nullptr, *constraints = nullptr, *terms = nullptr,
          *extra = nullptr, *sharp = nullptr, *first_scr = nullptr,
          *first_t_scr = nullptr, *second_scr = nullptr, *rr = nullptr,
          *rr_t = nullptr, *tangent = nullptr, *src_f = nullptr,
          *src_ft = nullptr, *src_d = nullptr, *src_dt = nullptr, *sum = nullptr,
          *sum_t = nullptr, *pairs = nullptr, *pairs_t = nullptr,
          *proj = nullptr, *proj_t = nullptr, *ethp_t = nullptr,
          *source = nullptr, *forcing = nullptr;
  double* pool = nullptr;
  // composite tile operators (angular_tile_kernel)
  double* tile_fp64 = nullptr;
  uint2* tile_split = nullptr;
  double* tile_scales = nullptr;
  const int* tile_offsets[cCount][4] = {};
  double* trig_data = nullptr;
  int* ints = nullptr;
  double* norm_acc = nullptr;
  int* finite = nullptr;
  double* weights = nullptr;
  std::vector<void*> owned;
  // per-coordinator device tables
  struct CoordDev {
    const int *active, *a_off, *s_off, *up_off, *down_off, *lap_diag,
        *raise_diag, *lower_diag, *ne, *lmin, *ne_up, *lmin_up, *ne_down,
        *lmin_down;
  } coords[cCount];
  const int *index1 = nullptr, *index2 = nullptr, *offsets = nullptr,
            *targets = nullptr;
  int target_count = 0;
  int pair_count = 0;

  template <class T>
  T* alloc(const size_t count) {
    void* p = nullptr;
    check(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)), "cudaMalloc");
    check(cudaMemset(p, 0, std::max<size_t>(count, 1) * sizeof(T)), "cudaMemset");
    owned.push_back(p);
    return static_cast<T*>(p);
  }
  ~Buffers() {
    for (void* p : owned) cudaFree(p);
  }
};

NodalPipeline::NodalPipeline(const InstancePlan& plan, const int precision,
                             const int replicas)
    : plan_(plan), precision_(precision), replicas_(replicas),
      active_(replicas), buf_(std::make_unique<Buffers>()) {
  if (precision != kPrecisionFp64 && precision != kPrecisionSplit) {
    throw std::invalid_argument("unknown transform precision");
  }
  const Config& c = plan_.config;
  if (replicas < 1) throw std::invalid_argument("replica count must be positive");
  // Replicas share one latch, so only solves whose source is on from the
  // start (no constraint-driven or time-driven switch) are replicated.
  if (replicas > 1 && !(c.source_mode == TEUK_B200_SOURCE_UNRESTRICTED &&
                        c.source_start_time == 0.0)) {
    throw std::invalid_argument(
        "replicated second-order pipelines need the Unrestricted source from t = 0");
  }
  if (c.ntheta > kMaxNodes) {
    throw std::invalid_argument(
        "the second-order pipeline supports at most 96 theta nodes");
  }
  Buffers& b = *buf_;
  b.geo.mass = c.mass;
  b.geo.spin = c.spin;
  b.geo.length = c.length;
  b.geo.spacing = plan_.spacing;
  b.geo.inv_spacing = 1.0 / plan_.spacing;
  b.geo.horizon = plan_.horizon;
  b.geo.damping = c.reduction == 0 ? c.damping : 0.0;
  b.geo.dissipation = c.dissipation;
  b.geo.nr = c.nr;
  b.geo.nt = c.ntheta;
  b.geo.modes = static_cast<int>(c.modes.size()) * replicas;
  b.geo.disc = c.disc;
  b.geo.reduction = c.reduction;
  check(upload_nodal_sbp_constants(), "upload SBP constants");

  // one replica's modes; buffers and tables hold `replicas` of them, replica
  // k in modes [k nm, (k + 1) nm)
  const size_t nm1 = c.modes.size();
  const size_t nm = nm1 * static_cast<size_t>(replicas);
  b.plane = static_cast<size_t>(c.nr) * static_cast<size_t>(c.ntheta);
  const size_t full = nm * kFieldCount * b.plane;
  b.state = b.alloc<double2>(full);
  b.stage = b.alloc<double2>(full);
  for (auto& k : b.k) k = b.alloc<double2>(full);
  b.rhs_in = b.alloc<double2>(full);
  b.rhs_out = b.alloc<double2>(full);
  b.tangent = b.alloc<double2>(full);
  const auto slots = [&](const size_t s) { return b.alloc<double2>(nm * s * b.plane); };
  b.lin_ang = slots(3);
  b.rec_ang = slots(6);
  b.rec_ang_t = slots(6);
  b.ind_ang = slots(2);
  b.constraints = slots(3);
  b.terms = slots(6);
  b.extra = slots(4);
  b.sharp = slots(4);
  b.first_scr = slots(5);
  b.first_t_scr = slots(5);
  b.second_scr = slots(5);
  b.rr = slots(7);
  b.rr_t = slots(7);
  b.src_f = slots(8);
  b.src_ft = slots(8);
  b.src_d = slots(11);
  b.src_dt = slots(11);
  b.sum = slots(2);
  b.sum_t = slots(2);
  b.proj = slots(2);
  b.proj_t = slots(2);
  b.ethp_t = slots(1);
  b.source = slots(1);
  b.forcing = slots(1);

  // ordered pairs, target-major then m1-major (include/teuk/modes.hpp:184-202)
  const auto index_of = [&](const int m) {
    return static_cast<int>(std::lower_bound(c.modes.begin(), c.modes.end(), m) -
                            c.modes.begin());
  };
  const auto is_parent = [&](const int m) {
    return std::binary_search(c.parents.begin(), c.parents.end(), m);
  };
  for (const int target : c.targets) {
    pair_offsets_.push_back(static_cast<int>(pair_index1_.size()));
    targets_.push_back(index_of(target));
    for (const int m1 : c.parents) {
      const int m2 = target - m1;
      if (!is_parent(m2)) continue;
      pair_index1_.push_back(index_of(m1));
      pair_index2_.push_back(index_of(m2));
    }
  }
  pair_offsets_.push_back(static_cast<int>(pair_index1_.size()));
  pairs_per_replica_ = static_cast<int>(pair_index1_.size());
  targets_per_replica_ = static_cast<int>(targets_.size());
  // replicate the pair tables, offset by each replica's first mode and pair
  {
    const std::vector<int> i1 = pair_index1_, i2 = pair_index2_,
                           po = pair_offsets_, tg = targets_;
    const int P = pairs_per_replica_, nmi = static_cast<int>(nm1);
    pair_offsets_.clear();
    for (int k = 1; k < replicas; ++k) {
      for (size_t j = 0; j < i1.size(); ++j) {
        pair_index1_.push_back(i1[j] + k * nmi);
        pair_index2_.push_back(i2[j] + k * nmi);
      }
      for (const int t : tg) targets_.push_back(t + k * nmi);
    }
    for (int k = 0; k < replicas; ++k) {
      for (size_t j = 0; j + 1 < po.size(); ++j) pair_offsets_.push_back(po[j] + k * P);
    }
    pair_offsets_.push_back(P * replicas);
  }
  b.pair_count = pairs_per_replica_ * replicas;
  b.target_count = targets_per_replica_ * replicas;
  b.pairs = b.alloc<double2>(std::max<size_t>(pair_index1_.size(), 1) * 2 * b.plane);
  b.pairs_t = b.alloc<double2>(std::max<size_t>(pair_index1_.size(), 1) * 2 * b.plane);

  build_coordinators();
  tile_operators_ = c.ntheta <= kTileMaxNodes;
  if (precision_ == kPrecisionSplit && !tile_operators_) {
    throw std::invalid_argument(
        "split-precision transforms support at most 64 theta nodes");
  }
  if (tile_operators_) {
    build_tile_operators();
    // the largest operator: a projection with n_ell = ntheta (FP64), any
    // operation (split)
    tile_fp64_words_ = tile_operator_words(kPrecisionFp64, kProject, c.ntheta, c.ntheta);
    tile_split_words_ = tile_operator_words(kPrecisionSplit, kProject, c.ntheta, c.ntheta);
    // the dynamic shared-memory opt-in is an attribute of the function on
    // the current device: set on every construction (cheap), so pipelines
    // on any device of the process may launch
    const int most = static_cast<int>(tile_smem_bytes(std::max(
        tile_operator_words(kPrecisionFp64, kProject, kTileMaxNodes, kTileMaxNodes),
        tile_operator_words(kPrecisionSplit, kProject, kTileMaxNodes, kTileMaxNodes))));
    check(cudaFuncSetAttribute(angular_tile_kernel<kPrecisionFp64>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, most),
          "tile operator shared memory");
    check(cudaFuncSetAttribute(angular_tile_kernel<kPrecisionSplit>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, most),
          "tile operator shared memory");
  }

  // integer tables: mvals, sharp, pairs, coordinator tables
  std::vector<int> ints;
  const auto push = [&](const std::vector<int>& v) {
    const size_t off = ints.size();
    ints.insert(ints.end(), v.begin(), v.end());
    if (v.empty()) ints.push_back(0);
    return off;
  };
  // per-mode tables of every replica
  const auto replicate = [&](const std::vector<int>& v) {
    std::vector<int> out;
    for (int k = 0; k < replicas; ++k) out.insert(out.end(), v.begin(), v.end());
    return out;
  };
  std::vector<int> sharp(nm);
  for (size_t i = 0; i < nm; ++i) {
    sharp[i] = index_of(-c.modes[i % nm1]) + static_cast<int>((i / nm1) * nm1);
  }
  const size_t off_m = push(replicate(c.modes)), off_sh = push(sharp);
  const size_t off_i1 = push(pair_index1_), off_i2 = push(pair_index2_),
               off_po = push(pair_offsets_), off_tg = push(targets_);
  size_t coord_offsets[cCount][14];
  for (int k = 0; k < cCount; ++k) {
    const AngularCoordinator& a = coordinators_[k];
    const std::vector<int>* lists[14] = {
        &a.active, &a.analysis, &a.synthesis, &a.raised, &a.lowered,
        nullptr, nullptr, nullptr, &a.n_ell, &a.ell_min, &a.n_ell_up,
        &a.ell_min_up, &a.n_ell_down, &a.ell_min_down};
    for (int l = 0; l < 14; ++l) {
      coord_offsets[k][l] = lists[l] ? push(replicate(*lists[l])) : 0;
    }
  }
  // pool offsets of each mode's Laplacian / raising / lowering diagonal
  for (int k = 0; k < cCount; ++k) {
    coord_offsets[k][5] = push(replicate(coordinator_diag_[k][0]));
    coord_offsets[k][6] = push(replicate(coordinator_diag_[k][1]));
    coord_offsets[k][7] = push(replicate(coordinator_diag_[k][2]));
  }
  b.ints = b.alloc<int>(ints.size());
  check(cudaMemcpy(b.ints, ints.data(), ints.size() * sizeof(int),
                   cudaMemcpyHostToDevice),
        "upload tables");
  b.trig.mvals = b.ints + off_m;
  b.trig.sharp = b.ints + off_sh;
  b.index1 = b.ints + off_i1;
  b.index2 = b.ints + off_i2;
  b.offsets = b.ints + off_po;
  b.targets = b.ints + off_tg;
  for (int k = 0; k < cCount; ++k) {
    auto& d = b.coords[k];
    d.active = b.ints + coord_offsets[k][0];
    d.a_off = b.ints + coord_offsets[k][1];
    d.s_off = b.ints + coord_offsets[k][2];
    d.up_off = b.ints + coord_offsets[k][3];
    d.down_off = b.ints + coord_offsets[k][4];
    d.lap_diag = b.ints + coord_offsets[k][5];
    d.raise_diag = b.ints + coord_offsets[k][6];
    d.lower_diag = b.ints + coord_offsets[k][7];
    d.ne = b.ints + coord_offsets[k][8];
    d.lmin = b.ints + coord_offsets[k][9];
    d.ne_up = b.ints + coord_offsets[k][10];
    d.lmin_up = b.ints + coord_offsets[k][11];
    d.ne_down = b.ints + coord_offsets[k][12];
    d.lmin_down = b.ints + coord_offsets[k][13];
  }
  b.pool = b.alloc<double>(matrices_.size());
  check(cudaMemcpy(b.pool, matrices_.data(), matrices_.size() * sizeof(double),
                   cudaMemcpyHostToDevice),
        "upload matrices");
  if (tile_operators_) {
    b.tile_fp64 = b.alloc<double>(tile_fp64_.size());
    b.tile_split = b.alloc<uint2>(tile_split_.size());
    b.tile_scales = b.alloc<double>(tile_scales_.size());
    check(cudaMemcpy(b.tile_fp64, tile_fp64_.data(),
                     tile_fp64_.size() * sizeof(double), cudaMemcpyHostToDevice),
          "upload tile operators");
    check(cudaMemcpy(b.tile_split, tile_split_.data(),
                     tile_split_.size() * sizeof(uint2), cudaMemcpyHostToDevice),
          "upload split tile operators");
    check(cudaMemcpy(b.tile_scales, tile_scales_.data(),
                     tile_scales_.size() * sizeof(double), cudaMemcpyHostToDevice),
          "upload tile operator scales");
    std::vector<int> offs;
    for (int k = 0; k < cCount; ++k) {
      for (int kind = 0; kind < 4; ++kind) {
        const auto v = replicate(tile_offsets_[k][kind]);  // 4 ints per mode
        offs.insert(offs.end(), v.begin(), v.end());
      }
    }
    int* d_offs = b.alloc<int>(offs.size());
    check(cudaMemcpy(d_offs, offs.data(), offs.size() * sizeof(int),
                     cudaMemcpyHostToDevice),
          "upload tile operator offsets");
    size_t at = 0;
    for (int k = 0; k < cCount; ++k) {
      for (int kind = 0; kind < 4; ++kind) {
        b.tile_offsets[k][kind] = d_offs + at;
        at += tile_offsets_[k][kind].size() * static_cast<size_t>(replicas);
      }
    }
  }
  // trig: theta_sin, theta_cos, grid_sin, grid_cos
  const size_t nt = static_cast<size_t>(c.ntheta);
  std::vector<double> trig(4 * nt);
  for (size_t j = 0; j < nt; ++j) {
    trig[j] = plan_.sinv[j];
    trig[nt + j] = plan_.cosv[j];
    trig[2 * nt + j] = std::sqrt(1.0 - plan_.x[j] * plan_.x[j]);
    trig[3 * nt + j] = plan_.x[j];
  }
  b.trig_data = b.alloc<double>(trig.size());
  check(cudaMemcpy(b.trig_data, trig.data(), trig.size() * sizeof(double),
                   cudaMemcpyHostToDevice),
        "upload trig");
  b.trig.theta_sin = b.trig_data;
  b.trig.theta_cos = b.trig_data + nt;
  b.trig.grid_sin = b.trig_data + 2 * nt;
  b.trig.grid_cos = b.trig_data + 3 * nt;
  // constraint weights: theta weights then radial norm weights
  std::vector<double> w(nt + static_cast<size_t>(c.nr));
  for (size_t j = 0; j < nt; ++j) w[j] = plan_.weights[j];
  for (int r = 0; r < c.nr; ++r) w[nt + r] = sbp_norm_weight(c.disc, c.nr, r);
  b.weights = b.alloc<double>(w.size());
  check(cudaMemcpy(b.weights, w.data(), w.size() * sizeof(double),
                   cudaMemcpyHostToDevice),
        "upload weights");
  b.norm_acc = b.alloc<double>(18);
  b.finite = b.alloc<int>(1);
  activation_ = {plan_.active != 0, plan_.activation_time,
                 plan_.consecutive_passes, plan_.last_eligibility_time};
  check(cudaDeviceSynchronize(), "nodal pipeline setup");
  check(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking),
        "cudaStreamCreate");
  stream_ = own_stream_;
}

NodalPipeline::~NodalPipeline() {
  for (StepGraph& g : graphs_) release_graph(g);
  buf_.reset();
  if (own_stream_ != nullptr) cudaStreamDestroy(own_stream_);
}

void NodalPipeline::set_stream(cudaStream_t stream) {
  stream_ = stream != nullptr ? stream : own_stream_;
}

void NodalPipeline::build_coordinators() {
  const Config& c = plan_.config;
  const size_t nm = c.modes.size();
  const int nt = c.ntheta;
  struct Spec {
    int spin, boost;
    bool second;
  };
  const Spec specs[cCount] = {{-2, -2, false}, {-2, -2, true}, {-1, -1, false},
                              {-2, 0, false},  {-1, 0, false}, {-1, 1, false},
                              {0, 0, false},   {2, 0, false},  {1, 1, false},
                              {-1, -2, true}};
  const double pi = std::numbers::pi_v<double>;
  const auto add_matrix = [&](const int spin, const int m, const int ell_max,
                              const bool analysis, int& ell_min, int& ne) {
    ell_min = std::max(std::abs(spin), std::abs(m));
    ne = ell_max - ell_min + 1;
    if (ne <= 0) {
      throw std::invalid_argument("ell_max is below the minimum allowed ell");
    }
    if (ne > nt) {
      throw std::invalid_argument(
          "angular transform needs at least as many nodes as modes");
    }
    const int off = static_cast<int>(matrices_.size());
    matrices_.resize(matrices_.size() + static_cast<size_t>(ne * nt));
    for (int j = 0; j < nt; ++j) {
      for (int l = 0; l < ne; ++l) {
        const double basis = spin_weighted_harmonic_theta(
            ell_min + l, m, spin, plan_.theta[static_cast<size_t>(j)]);
        // stored so that a warp's lanes read consecutive entries: the
        // analysis (lanes over ell) node-major, the synthesis (lanes over
        // nodes) ell-major
        if (analysis) {
          matrices_[static_cast<size_t>(off + j * ne + l)] =
              2.0 * pi * plan_.weights[static_cast<size_t>(j)] * basis;
        } else {
          matrices_[static_cast<size_t>(off + l * nt + j)] = basis;
        }
      }
    }
    return off;
  };
  coordinators_.resize(cCount);
  for (int k = 0; k < cCount; ++k) {
    const Spec& s = specs[k];
    AngularCoordinator& a = coordinators_[k];
    a.spin = s.spin;
    a.boost = s.boost;
    a.ell_max = s.second ? c.ell_max_second : c.ell_max_first;
    const std::vector<int>& act = s.second ? c.targets : c.parents;
    a.active.assign(nm, 0);
    a.analysis.assign(nm, 0);
    a.synthesis.assign(nm, 0);
    a.raised.assign(nm, 0);
    a.lowered.assign(nm, 0);
    a.n_ell.assign(nm, 0);
    a.ell_min.assign(nm, 0);
    a.n_ell_up.assign(nm, 0);
    a.ell_min_up.assign(nm, 0);
    a.n_ell_down.assign(nm, 0);
    a.ell_min_down.assign(nm, 0);
    for (int d = 0; d < 3; ++d) coordinator_diag_[k][d].assign(nm, 0);
    for (size_t i = 0; i < nm; ++i) {
      const int m = c.modes[i];
      if (!std::binary_search(act.begin(), act.end(), m)) continue;
      if (std::abs(m) > a.ell_max) {
        throw std::invalid_argument(
            "angular coordinator active mode is outside its stored band");
      }
      a.active[i] = 1;
      int lmin = 0, ne = 0, lu = 0, nu = 0, ldn = 0, nd = 0;
      a.analysis[i] = add_matrix(s.spin, m, a.ell_max, true, lmin, ne);
      a.synthesis[i] = add_matrix(s.spin, m, a.ell_max, false, lmin, ne);
      a.raised[i] = add_matrix(s.spin + 1, m, a.ell_max, false, lu, nu);
      a.lowered[i] = add_matrix(s.spin - 1, m, a.ell_max, false, ldn, nd);
      a.n_ell[i] = ne;
      a.ell_min[i] = lmin;
      a.n_ell_up[i] = nu;
      a.ell_min_up[i] = lu;
      a.n_ell_down[i] = nd;
      a.ell_min_down[i] = ldn;
      // diagonal factors (include/teuk/angular.hpp:129-165)
      for (int d = 0; d < 3; ++d) {
        coordinator_diag_[k][d][i] = static_cast<int>(matrices_.size());
        for (int l = 0; l < ne; ++l) {
          const int ell = lmin + l;
          const int sp = s.spin;
          double v = 0.0;
          if (d == 0) v = -static_cast<double>((ell - sp) * (ell + sp + 1));
          if (d == 1) v = std::sqrt(static_cast<double>((ell - sp) * (ell + sp + 1)));
          if (d == 2) v = -std::sqrt(static_cast<double>((ell + sp) * (ell - sp + 1)));
          matrices_.push_back(v);
        }
      }
    }
  }
}

// Composite nodal matrices T = S_out diag(d) A of every (coordinator,
// operation, active mode), accumulated in long double and rounded once, and
// their tensor-core fragment layouts: FP64 B fragments of T^T for
// mma.sync m8n8k4, and BF16 digit fragments with per-column power-of-two
// scales for the split-precision m16n8k16 path.
void NodalPipeline::build_tile_operators() {
  const Config& c = plan_.config;
  const int nt = c.ntheta;
  const size_t nm = c.modes.size();
  const int n8 = (nt + 7) / 8, k4 = (nt + 3) / 4, k16 = (nt + 15) / 16;
  std::vector<double> T(static_cast<size_t>(nt) * nt);
  for (int k = 0; k < cCount; ++k) {
    const AngularCoordinator& a = coordinators_[k];
    for (int kind = 0; kind < 4; ++kind) {
      std::vector<int>& offs = tile_offsets_[k][kind];
      offs.assign(4 * nm, 0);
      for (size_t i = 0; i < nm; ++i) {
        if (!a.active[i]) continue;
        const int ne = a.n_ell[i], lmin = a.ell_min[i];
        int o_off = a.synthesis[i], ne_o = ne, lmin_o = lmin, diag = -1;
        if (kind == kLaplacian) diag = coordinator_diag_[k][0][i];
        if (kind == kEth) {
          o_off = a.raised[i];
          ne_o = a.n_ell_up[i];
          lmin_o = a.ell_min_up[i];
          diag = coordinator_diag_[k][1][i];
        } else if (kind == kEthPrime) {
          o_off = a.lowered[i];
          ne_o = a.n_ell_down[i];
          lmin_o = a.ell_min_down[i];
          diag = coordinator_diag_[k][2][i];
        }
        const int shift = lmin_o - lmin;
        const double* A = matrices_.data() + a.analysis[i];  // [node][ell]
        const double* S = matrices_.data() + o_off;          // [ell][node]
        for (int j = 0; j < nt; ++j) {
          for (int kk = 0; kk < nt; ++kk) {
            long double v = 0.0L;
            for (int l = 0; l < ne_o; ++l) {
              const int src = l + shift;
              if (src < 0 || src >= ne) continue;
              long double term = static_cast<long double>(S[l * nt + j]) *
                                 static_cast<long double>(A[kk * ne + src]);
              if (diag >= 0) term *= static_cast<long double>(matrices_[diag + src]);
              v += term;
            }
            T[static_cast<size_t>(j) * nt + kk] = static_cast<double>(v);
          }
        }
        const auto at = [&](const int j, const int kk) {
          return (j < nt && kk < nt) ? T[static_cast<size_t>(j) * nt + kk] : 0.0;
        };
        offs[4 * i] = static_cast<int>(tile_fp64_.size());
        offs[4 * i + 3] = ne;
        if (kind == kProject) {
          // two GEMMs: B fragments of A^T (K = nodes, N = ell), then of S^T
          // (K = ell, N = nodes)
          const int n1 = (ne + 7) / 8, kl4 = (ne + 3) / 4;
          const auto Av = [&](const int l, const int kk) {
            return (l < ne && kk < nt) ? A[kk * ne + l] : 0.0;
          };
          const auto Sv = [&](const int j, const int l) {
            return (j < nt && l < ne) ? S[l * nt + j] : 0.0;
          };
          for (int n = 0; n < n1; ++n) {
            for (int ks = 0; ks < k4; ++ks) {
              for (int lane = 0; lane < 32; ++lane) {
                tile_fp64_.push_back(Av(n * 8 + lane / 4, ks * 4 + lane % 4));
              }
            }
          }
          for (int n = 0; n < n8; ++n) {
            for (int ks = 0; ks < kl4; ++ks) {
              for (int lane = 0; lane < 32; ++lane) {
                tile_fp64_.push_back(Sv(n * 8 + lane / 4, ks * 4 + lane % 4));
              }
            }
          }
        } else {
          for (int n = 0; n < n8; ++n) {
            for (int ks = 0; ks < k4; ++ks) {
              for (int lane = 0; lane < 32; ++lane) {
                tile_fp64_.push_back(at(n * 8 + lane / 4, ks * 4 + lane % 4));
              }
            }
          }
        }
        // split: per output node j a power-of-two scale and five digits
        std::vector<float> digits(static_cast<size_t>(n8) * 8 * k16 * 16 * kSplitSlices, 0.0f);
        const auto digit = [&](const int j, const int kk, const int t) -> float& {
          return digits[((static_cast<size_t>(j) * k16 * 16) + kk) * kSplitSlices + t];
        };
        offs[4 * i + 2] = static_cast<int>(tile_scales_.size());
        for (int j = 0; j < n8 * 8; ++j) {
          double m = 0.0;
          for (int kk = 0; kk < nt; ++kk) m = std::max(m, std::fabs(at(j, kk)));
          const int e = split::host_exponent(m);
          tile_scales_.push_back(j < nt ? std::ldexp(1.0, e - 14) : 0.0);
          for (int kk = 0; kk < nt; ++kk) {
            float t[kSplitSlices];
            split::host_digits(at(j, kk) * std::ldexp(1.0, -e), t);
            for (int s = 0; s < kSplitSlices; ++s) digit(j, kk, s) = t[s];
          }
        }
        offs[4 * i + 1] = static_cast<int>(tile_split_.size());
        for (int n = 0; n < n8; ++n) {
          for (int ks = 0; ks < k16; ++ks) {
            for (int t = 0; t < kSplitSlices; ++t) {
              for (int lane = 0; lane < 32; ++lane) {
                const int j = n * 8 + lane / 4, kk = ks * 16 + 2 * (lane % 4);
                uint2 f;
                f.x = split::host_pack(digit(j, kk, t), digit(j, kk + 1, t));
                f.y = split::host_pack(digit(j, kk + 8, t), digit(j, kk + 9, t));
                tile_split_.push_back(f);
              }
            }
          }
        }
      }
    }
  }
  if (tile_fp64_.empty()) tile_fp64_.push_back(0.0);
  if (tile_split_.empty()) tile_split_.push_back(uint2{0u, 0u});
  if (tile_scales_.empty()) tile_scales_.push_back(0.0);
}

void NodalPipeline::sync_check(const char* what) {
  check(cudaGetLastError(), what);
}

void NodalPipeline::evaluate(const double2* stage_in, double2* out) {
  Buffers& b = *buf_;
  const Geo& g = b.geo;
  const Trig& tr = b.trig;
  cudaStream_t s = stream_;
  const long long points = static_cast<long long>(g.modes) * g.nr * g.nt;
  const int gp = grid_for(points);
  const int ga = grid_for(static_cast<long long>(g.modes) * g.nr * 32);
  const Arr stage{const_cast<double2*>(stage_in), kFieldCount};
  const Arr output{out, kFieldCount};

  // Angular operations on the tile operator are queued and launched
  // together while they are independent: a queued operation that writes a
  // plane another queued one reads or writes (or reads a plane one writes)
  // flushes the queue first, and so does every other kernel below.
  struct TileQueue {
    NodalPipeline& self;
    Buffers& b;
    const Geo& g;
    const Trig& tr;
    cudaStream_t s;
    struct Plane {
      const double2* p;
      int slots, slot;
      bool operator==(const Plane& o) const {
        return p == o.p && slots == o.slots && slot == o.slot;
      }
    };
    // pending operations by arithmetic: projections always run the FP64
    // two-GEMM path (their output must be band limited relative to itself,
    // as the reference's checkpoints require); the others follow the
    // pipeline's precision
    AngularTileBatch batch[2]{};  // [kPrecisionFp64], [kPrecisionSplit]
    std::vector<Plane> reads, writes;
    int pending() const { return batch[0].count + batch[1].count; }
    void launch(const int prec) {
      AngularTileBatch& bt = batch[prec];
      if (bt.count == 0) return;
      const int tiles = g.modes * ((g.nr + kTileCtaRows - 1) / kTileCtaRows);
      for (int i = 0; i <= bt.count; ++i) bt.first_block[i] = i * tiles;
      const int words = prec == kPrecisionSplit ? self.tile_split_words_
                                                : self.tile_fp64_words_;
      const size_t bytes = tile_smem_bytes(words);
      const unsigned grid = static_cast<unsigned>(bt.count * tiles);
      if (prec == kPrecisionSplit) {
        angular_tile_kernel<kPrecisionSplit><<<grid, kTileWarps * 32, bytes, s>>>(g, tr, bt);
      } else {
        angular_tile_kernel<kPrecisionFp64><<<grid, kTileWarps * 32, bytes, s>>>(g, tr, bt);
      }
      bt.count = 0;
    }
    // the pending operations are mutually independent, so the two launches
    // may run in either order
    void flush() {
      launch(kPrecisionFp64);
      launch(kPrecisionSplit);
      reads.clear();
      writes.clear();
    }
    static bool contains(const std::vector<Plane>& v, const Plane& x) {
      return std::find(v.begin(), v.end(), x) != v.end();
    }
    void add(const int coord, const int kind, const Arr in, const int in_slot,
             const Arr dt, const int dt_slot, const Arr o, const int out_slot,
             const int spin, const int boost) {
      const bool ghp = kind == kEth || kind == kEthPrime;
      const Plane r1{in.p, in.slots, in_slot}, r2{dt.p, dt.slots, dt_slot},
          w{o.p, o.slots, out_slot};
      const int prec = kind == kProject ? kPrecisionFp64 : self.precision_;
      if (batch[prec].count == kTileMaxOps || contains(writes, r1) ||
          (ghp && contains(writes, r2)) || contains(writes, w) ||
          contains(reads, w)) {
        flush();
      }
      const auto& d = b.coords[coord];
      AngularTileParams& tp = batch[prec].ops[batch[prec].count++];
      tp = AngularTileParams{};
      tp.kind = kind;
      tp.in = in;
      tp.in_slot = in_slot;
      tp.dt = dt;
      tp.dt_slot = dt_slot;
      tp.out = o;
      tp.out_slot = out_slot;
      tp.active = d.active;
      tp.offsets = b.tile_offsets[coord][kind];
      tp.fp64 = b.tile_fp64;
      tp.split = b.tile_split;
      tp.scales = b.tile_scales;
      tp.spin = spin;
      tp.boost = boost;
      reads.push_back(r1);
      if (ghp) reads.push_back(r2);
      writes.push_back(w);
    }
  } tile_queue{*this, b, g, tr, s};
  const auto flush = [&] { tile_queue.flush(); };

  const auto op = [&](const int coord, const int kind, const Arr in,
                      const int in_slot, const Arr dt, const int dt_slot,
                      const Arr o, const int out_slot) {
    const auto& d = b.coords[coord];
    AngularOpParams p{};
    p.kind = kind;
    p.in = in;
    p.in_slot = in_slot;
    p.dt = dt;
    p.dt_slot = dt_slot;
    p.out = o;
    p.out_slot = out_slot;
    p.active = d.active;
    p.a_off = d.a_off;
    p.pool = b.pool;
    p.spin = coordinators_[coord].spin;
    p.boost = coordinators_[coord].boost;
    p.ne = d.ne;
    p.lmin = d.lmin;
    if (kind == kProject || kind == kLaplacian) {
      p.o_off = d.s_off;
      p.ne_o = d.ne;
      p.lmin_o = d.lmin;
      p.diag_off = d.lap_diag;
    } else if (kind == kEth) {
      p.o_off = d.up_off;
      p.ne_o = d.ne_up;
      p.lmin_o = d.lmin_up;
      p.diag_off = d.raise_diag;
    } else {
      p.o_off = d.down_off;
      p.ne_o = d.ne_down;
      p.lmin_o = d.lmin_down;
      p.diag_off = d.lower_diag;
    }
    if (tile_operators_) {
      tile_queue.add(coord, kind, in, in_slot, dt, dt_slot, o, out_slot,
                     p.spin, p.boost);
      return;
    }
    angular_op_kernel<<<ga, kBlock, 0, s>>>(g, tr, p);
  };
  const auto teuk = [&](const Arr st_, const int f0, const Arr scratch,
                        const Arr lap, const int lap_slot,
                        const double2* forcing, const Arr o) {
    flush();
    TeukParams p{st_, f0, scratch, lap, lap_slot, forcing, o};
    teuk_prepare_kernel<<<gp, kBlock, 0, s>>>(g, p);
    teuk_primitives_kernel<<<gp, kBlock, 0, s>>>(g, tr, p);
    teuk_rhs_kernel<<<gp, kBlock, 0, s>>>(g, tr, p);
  };
  const auto project3 = [&](const int coord, const Arr o, const int f0) {
    for (int f = 0; f < 3; ++f) op(coord, kProject, o, f0 + f, o, 0, o, f0 + f);
  };
  const Arr lin{b.lin_ang, 3}, first_scr{b.first_scr, 5},
      first_t_scr{b.first_t_scr, 5}, second_scr{b.second_scr, 5},
      tangent{b.tangent, kFieldCount}, sharp{b.sharp, 4};
  const auto chain = [&](const Arr st_, const Arr o, double2* rr_p,
                         double2* ang_p) {
    const Arr rr{rr_p, 7}, ang{ang_p, 6};
    flush();
    recon_radial_kernel<<<grid_for(points * 7), kBlock, 0, s>>>(g, st_, rr);
    op(cFirst, kEth, st_, kFirstPsi, o, kFirstPsi, ang, aEth1F);
    ReconParams rp{st_, o, rr, ang};
    flush();
    recon_pass_kernel<1><<<gp, kBlock, 0, s>>>(g, tr, rp);
    op(cG, kProject, o, kG, o, 0, o, kG);
    op(cFirst, kProject, o, kLambda, o, 0, o, kLambda);
    op(cG, kEth, st_, kG, o, kG, ang, aEth2G);
    flush();
    recon_pass_kernel<2><<<gp, kBlock, 0, s>>>(g, tr, rp);
    op(cScalar, kProject, o, kH, o, 0, o, kH);
    op(cB, kProject, o, kB, o, 0, o, kB);
    op(cPi, kProject, o, kPi, o, 0, o, kPi);
    op(cC, kProject, o, kC, o, 0, o, kC);
    op(cC, kEth, st_, kC, o, kC, ang, aEth2C);
    op(cPi, kEth, st_, kPi, o, kPi, ang, aEth2Pi);
    flush();
    pack_sharp_kernel<<<gp, kBlock, 0, s>>>(g, tr, st_, o, sharp);
    op(cBSharp, kEthPrime, sharp, shB, sharp, shBDt, ang, aEthP1BSharp);
    op(cCSharp, kEthPrime, sharp, shC, sharp, shCDt, ang, aEthP2CSharp);
    flush();
    recon_pass_kernel<3><<<gp, kBlock, 0, s>>>(g, tr, rp);
    op(cScalar, kProject, o, kU, o, 0, o, kU);
  };

  // first-order triple (include/teuk/spatial_pipeline.hpp:483-497)
  op(cFirst, kLaplacian, stage, kFirstPsi, stage, 0, lin, 0);
  teuk(stage, kFirstP, first_scr, lin, 0, nullptr, output);
  project3(cFirst, output, kFirstP);
  // reconstruction and independent constraints (:517-520, 768-893)
  chain(stage, output, b.rr, b.rec_ang);
  const Arr ind{b.ind_ang, 2};
  op(cG, kEthPrime, stage, kG, output, kG, ind, 0);
  op(cScalar, kEthPrime, stage, kH, output, kH, ind, 1);
  ConstraintParams cp{stage, output, first_scr, Arr{b.rr, 7}, ind,
                      Arr{b.constraints, 3}, Arr{b.terms, 6}};
  flush();
  constraints_kernel<<<gp, kBlock, 0, s>>>(g, tr, cp);
  // stage tangent (:526-546)
  op(cFirst, kLaplacian, output, kFirstPsi, output, 0, lin, 1);
  teuk(output, kFirstP, first_t_scr, lin, 1, nullptr, tangent);
  project3(cFirst, tangent, kFirstP);
  chain(output, tangent, b.rr_t, b.rec_ang_t);
  // source angular derivatives (:933-959)
  const Arr extra{b.extra, 4};
  op(cB, kEth, stage, kB, output, kB, extra, xEth1B);
  op(cFirst, kEthPrime, stage, kFirstPsi, output, kFirstPsi, extra, xEthP1F);
  op(cB, kEth, output, kB, tangent, kB, extra, xEth1BT);
  op(cFirst, kEthPrime, output, kFirstPsi, tangent, kFirstPsi, extra, xEthP1FT);
  // source inputs, inner source, projection, outer source (:961-1209)
  SourceInputParams sp{stage,          output,          tangent,
                       first_scr,      first_t_scr,     Arr{b.rr, 7},
                       Arr{b.rr_t, 7}, Arr{b.rec_ang, 6}, Arr{b.rec_ang_t, 6},
                       extra,          Arr{b.src_f, 8}, Arr{b.src_ft, 8},
                       Arr{b.src_d, 11}, Arr{b.src_dt, 11}};
  flush();
  source_inputs_kernel<<<gp, kBlock, 0, s>>>(g, tr, sp);
  check(cudaMemsetAsync(b.sum, 0, sizeof(double2) * g.modes * 2 * b.plane, s),
        "zero inner source");
  check(cudaMemsetAsync(b.sum_t, 0, sizeof(double2) * g.modes * 2 * b.plane, s),
        "zero inner source tangent");
  InnerParams ip{Arr{b.src_f, 8}, Arr{b.src_ft, 8}, Arr{b.src_d, 11},
                 Arr{b.src_dt, 11}, Arr{b.sum, 2}, Arr{b.sum_t, 2},
                 Arr{b.pairs, 2}, Arr{b.pairs_t, 2}, b.index1, b.index2,
                 b.offsets, b.targets, b.target_count};
  if (b.target_count > 0) {
    inner_source_kernel<<<grid_for(static_cast<long long>(b.target_count) * g.nr * g.nt),
                          kBlock, 0, s>>>(g, tr, ip);
  }
  const Arr sum{b.sum, 2}, sum_t{b.sum_t, 2}, proj{b.proj, 2}, proj_t{b.proj_t, 2};
  op(cSecond, kProject, sum, 0, sum, 0, proj, 0);
  op(cSecond, kProject, sum_t, 0, sum_t, 0, proj_t, 0);
  op(cT, kProject, sum, 1, sum, 0, proj, 1);
  op(cT, kProject, sum_t, 1, sum_t, 0, proj_t, 1);
  op(cT, kEthPrime, proj, 1, proj_t, 1, Arr{b.ethp_t, 1}, 0);
  flush();
  outer_source_kernel<<<gp, kBlock, 0, s>>>(g, tr, proj, proj_t, b.ethp_t,
                                            b.source, b.forcing);
  if (!activation_.active) {
    check(cudaMemsetAsync(b.forcing, 0, sizeof(double2) * points, s),
          "latched forcing");
  }
  // second-order triple with forcing (:566-583)
  op(cSecond, kLaplacian, stage, kSecondPsi, stage, 0, lin, 2);
  teuk(stage, kSecondP, second_scr, lin, 2, b.forcing, output);
  project3(cSecond, output, kSecondP);
  flush();
  sync_check("second-order RHS");
}

ConstraintNorms NodalPipeline::sample_constraints() {
  Buffers& b = *buf_;
  const Geo& g = b.geo;
  cudaStream_t s = stream_;
  check(cudaMemsetAsync(b.norm_acc, 0, 18 * sizeof(double), s), "zero norms");
  const int one = 1;
  check(cudaMemcpyAsync(b.finite, &one, sizeof(int), cudaMemcpyHostToDevice, s),
        "finite flag");
  const long long points = static_cast<long long>(g.modes) * g.nr * g.nt;
  norms_natural_kernel<<<grid_for(points), kBlock, 0, s>>>(
      g, Arr{b.constraints, 3}, Arr{b.terms, 6}, b.weights, b.norm_acc, b.finite);
  norms_normalized_kernel<<<grid_for(points), kBlock, 0, s>>>(
      g, Arr{b.constraints, 3}, Arr{b.terms, 6}, b.norm_acc, b.finite);
  double acc[18];
  int finite = 1;
  check(cudaMemcpyAsync(acc, b.norm_acc, sizeof(acc), cudaMemcpyDeviceToHost, s),
        "norms read");
  check(cudaMemcpyAsync(&finite, b.finite, sizeof(int), cudaMemcpyDeviceToHost, s),
        "finite read");
  check(cudaStreamSynchronize(s), "constraint norms");
  // include/teuk/source_activation.hpp:188-225
  ConstraintNorms n;
  n.all_finite = finite != 0;
  const double floor = 64.0 * std::numeric_limits<double>::epsilon();
  const double weight_sum = static_cast<double>(g.modes) * (g.horizon - 0.0) *
                            4.0 * std::numbers::pi_v<double>;
  for (int f = 0; f < 3; ++f) {
    n.absolute_maximum[f] = std::sqrt(acc[9 + f]);
    n.normalized_maximum[f] = std::sqrt(acc[15 + f]);
    n.weighted_rms[f] = std::sqrt(acc[f] / weight_sum);
    const double left = std::sqrt(acc[3 + f]);
    const double right = std::sqrt(acc[6 + f]);
    const double natural = std::max(left, right);
    const double den = left + right + floor * natural;
    n.normalized_weighted[f] = den > 0.0 ? std::sqrt(acc[f]) / den : 0.0;
    n.controlling_normalized =
        std::max(n.controlling_normalized,
                 std::max(n.normalized_maximum[f], n.normalized_weighted[f]));
  }
  if (!n.all_finite || !std::isfinite(n.controlling_normalized)) {
    n.all_finite = false;
    n.controlling_normalized = std::numeric_limits<double>::infinity();
  }
  return n;
}

// consider_source_activation (include/teuk/spatial_pipeline.hpp:1242-1289)
void NodalPipeline::consider_activation(const double accepted_time) {
  const Config& c = plan_.config;
  if (!std::isfinite(accepted_time) || accepted_time < 0.0) {
    throw std::invalid_argument(
        "source activation requires a finite accepted-state time");
  }
  if (activation_.active || accepted_time < c.source_start_time ||
      accepted_time <= activation_.last_eligibility_time) {
    return;
  }
  if (c.source_mode == TEUK_B200_SOURCE_DISABLED) return;
  if (c.source_mode == TEUK_B200_SOURCE_UNRESTRICTED) {
    activation_.last_eligibility_time = accepted_time;
    activation_.consecutive_passes = c.required_passes;
    activation_.active = true;
    activation_.activation_time = accepted_time;
    return;
  }
  evaluate(buf_->state, buf_->rhs_out);
  norms_ = sample_constraints();
  independent_max_ = std::max({norms_.absolute_maximum[0],
                               norms_.absolute_maximum[1],
                               norms_.absolute_maximum[2]});
  const bool passed = norms_.all_finite &&
                      norms_.controlling_normalized <= c.constraint_tolerance;
  activation_.last_eligibility_time = accepted_time;
  activation_.consecutive_passes =
      passed ? std::min(activation_.consecutive_passes + 1, c.required_passes)
             : 0;
  if (activation_.consecutive_passes >= c.required_passes) {
    activation_.active = true;
    activation_.activation_time = accepted_time;
  }
}

// advance_fixed_source_step + device_classical_rk4_step
// (include/teuk/spatial_pipeline.hpp:1291-1310, device_rk4.hpp:84-128)
void NodalPipeline::advance_fixed(const double, const double dt) {
  if (!(dt > 0.0)) return;
  // One RK4 step is replayed from a CUDA graph per (latch state, dt,
  // stream): the latch is host state read while the step is recorded, and
  // it only changes between steps.
  StepGraph& g = graphs_[activation_.active ? 1 : 0];
  if (g.exec == nullptr || g.dt != dt || g.stream != stream_) {
    release_graph(g);
    check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal),
          "begin step capture");
    try {
      record_step(dt);
    } catch (...) {
      cudaGraph_t discard = nullptr;
      cudaStreamEndCapture(stream_, &discard);
      if (discard != nullptr) cudaGraphDestroy(discard);
      throw;
    }
    check(cudaStreamEndCapture(stream_, &g.graph), "end step capture");
    check(cudaGraphInstantiate(&g.exec, g.graph, 0), "instantiate step");
    g.dt = dt;
    g.stream = stream_;
  }
  check(cudaGraphLaunch(g.exec, stream_), "step graph launch");
}

void NodalPipeline::release_graph(StepGraph& g) {
  if (g.exec != nullptr) cudaGraphExecDestroy(g.exec);
  if (g.graph != nullptr) cudaGraphDestroy(g.graph);
  g = StepGraph{};
}

void NodalPipeline::record_step(const double dt) {
  Buffers& b = *buf_;
  const long long n = static_cast<long long>(value_count());
  const int grid = grid_for(n);
  cudaStream_t s = stream_;
  evaluate(b.state, b.k[0]);
  axpy_kernel<<<grid, kBlock, 0, s>>>(b.state, b.k[0], b.stage, 0.5 * dt, n);
  evaluate(b.stage, b.k[1]);
  axpy_kernel<<<grid, kBlock, 0, s>>>(b.state, b.k[1], b.stage, 0.5 * dt, n);
  evaluate(b.stage, b.k[2]);
  axpy_kernel<<<grid, kBlock, 0, s>>>(b.state, b.k[2], b.stage, dt, n);
  evaluate(b.stage, b.k[3]);
  accumulate_kernel<<<grid, kBlock, 0, s>>>(b.state, b.k[0], b.k[1], b.k[2],
                                            b.k[3], dt / 6.0, n);
  sync_check("second-order RK4 step");
}

// SpatialPipeline::step (include/teuk/spatial_pipeline.hpp:590-620)
void NodalPipeline::step(const double time, const double dt) {
  if (!std::isfinite(time) || !std::isfinite(dt) || time < 0.0 || !(dt > 0.0)) {
    throw std::invalid_argument("pipeline step requires finite positive time data");
  }
  const double end_time = time + dt;
  if (!std::isfinite(end_time)) {
    throw std::invalid_argument("pipeline step end time is not finite");
  }
  const double start_time = plan_.config.source_start_time;
  if (!activation_.active && time >= start_time) consider_activation(time);
  if (!activation_.active && time < start_time && start_time < end_time) {
    advance_fixed(time, start_time - time);
    consider_activation(start_time);
    advance_fixed(start_time, end_time - start_time);
  } else {
    advance_fixed(time, dt);
  }
  if (!activation_.active && end_time >= start_time) consider_activation(end_time);
}

void NodalPipeline::reset_activation() {
  const Config& c = plan_.config;
  activation_ = {};
  norms_ = {};
  independent_max_ = 0.0;
  if (c.source_mode == TEUK_B200_SOURCE_UNRESTRICTED &&
      c.source_start_time == 0.0) {
    activation_.active = true;
    activation_.activation_time = 0.0;
    activation_.consecutive_passes = c.required_passes;
  }
}

void NodalPipeline::restore_activation(const SourceActivation& s) {
  activation_ = s;
}

void NodalPipeline::set_state(const double* state, const int memory) {
  const size_t bytes = value_count() * sizeof(double2);
  check(cudaMemcpyAsync(buf_->state, state, bytes,
                        memory == TEUK_B200_HOST ? cudaMemcpyHostToDevice
                                                 : cudaMemcpyDeviceToDevice,
                        stream_),
        "set_state");
  check(cudaStreamSynchronize(stream_), "set_state");
}

void NodalPipeline::get_state(double* state, const int memory) {
  const size_t bytes = value_count() * sizeof(double2);
  check(cudaMemcpyAsync(state, buf_->state, bytes,
                        memory == TEUK_B200_HOST ? cudaMemcpyDeviceToHost
                                                 : cudaMemcpyDeviceToDevice,
                        stream_),
        "get_state");
  check(cudaStreamSynchronize(stream_), "get_state");
}

void NodalPipeline::evaluate_rhs(const double* stage, double* out,
                                 const int memory, double) {
  const size_t bytes = value_count() * sizeof(double2);
  const cudaMemcpyKind in_kind =
      memory == TEUK_B200_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  check(cudaMemcpyAsync(buf_->rhs_in, stage, bytes, in_kind, stream_), "rhs in");
  // the storage RHS (rhs_out) is left to the latch check, as the reference
  // leaves storage().rhs() alone when a caller evaluates its own views
  evaluate(buf_->rhs_in, buf_->k[3]);
  check(cudaMemcpyAsync(out, buf_->k[3], bytes,
                        memory == TEUK_B200_HOST ? cudaMemcpyDeviceToHost
                                                 : cudaMemcpyDeviceToDevice,
                        stream_),
        "rhs out");
  check(cudaStreamSynchronize(stream_), "evaluate_rhs");
}

void NodalPipeline::set_active_replicas(const int k) {
  if (k < 1 || k > replicas_) {
    throw std::invalid_argument("active replica count outside the pipeline's room");
  }
  if (k == active_) return;
  check(cudaStreamSynchronize(stream_), "replica change");
  const int nm1 = static_cast<int>(plan_.config.modes.size());
  active_ = k;
  buf_->geo.modes = nm1 * k;
  buf_->target_count = targets_per_replica_ * k;
  buf_->pair_count = pairs_per_replica_ * k;
  for (StepGraph& g : graphs_) release_graph(g);  // recorded for the old count
}

void NodalPipeline::set_replica_state(const int k, const double* state,
                                      const int memory) {
  if (k < 0 || k >= replicas_) throw std::invalid_argument("replica index out of range");
  const size_t n = plan_.value_count();
  check(cudaMemcpyAsync(buf_->state + static_cast<size_t>(k) * n, state,
                        n * sizeof(double2),
                        memory == TEUK_B200_HOST ? cudaMemcpyHostToDevice
                                                 : cudaMemcpyDeviceToDevice,
                        stream_),
        "set replica state");
  check(cudaStreamSynchronize(stream_), "set replica state");
}

void NodalPipeline::get_replica_state(const int k, double* state,
                                      const int memory) {
  if (k < 0 || k >= replicas_) throw std::invalid_argument("replica index out of range");
  const size_t n = plan_.value_count();
  check(cudaMemcpyAsync(state, buf_->state + static_cast<size_t>(k) * n,
                        n * sizeof(double2),
                        memory == TEUK_B200_HOST ? cudaMemcpyDeviceToHost
                                                 : cudaMemcpyDeviceToDevice,
                        stream_),
        "get replica state");
  check(cudaStreamSynchronize(stream_), "get replica state");
}

void NodalPipeline::copy_replica_from(const NodalPipeline& src, const int src_k,
                                      const int dst_k) {
  if (src_k < 0 || src_k >= src.replicas_ || dst_k < 0 || dst_k >= replicas_ ||
      src.plan_.value_count() != plan_.value_count()) {
    throw std::invalid_argument("replica copy between different shapes");
  }
  const size_t n = plan_.value_count();
  // the source's pending steps come first
  check(cudaStreamSynchronize(src.stream_), "replica copy");
  check(cudaMemcpyAsync(buf_->state + static_cast<size_t>(dst_k) * n,
                        src.buf_->state + static_cast<size_t>(src_k) * n,
                        n * sizeof(double2), cudaMemcpyDeviceToDevice, stream_),
        "replica copy");
  check(cudaStreamSynchronize(stream_), "replica copy");
}

void NodalPipeline::endpoint_slice(const int field, const int radial,
                                   std::vector<double2>& out, const int replica) {
  const Config& c = plan_.config;
  const size_t nm = c.modes.size(), nt = static_cast<size_t>(c.ntheta);
  if (replica < 0 || replica >= active_) {
    throw std::invalid_argument("replica index out of range");
  }
  out.resize(nm * nt);
  for (size_t mode0 = 0; mode0 < nm; ++mode0) {
    const size_t mode = mode0 + static_cast<size_t>(replica) * nm;
    const size_t off = ((mode * kFieldCount + static_cast<size_t>(field)) *
                            static_cast<size_t>(c.nr) +
                        static_cast<size_t>(radial)) *
                       nt;
    check(cudaMemcpyAsync(out.data() + mode0 * nt, buf_->state + off,
                          nt * sizeof(double2), cudaMemcpyDeviceToHost, stream_),
          "endpoint slice");
  }
  check(cudaStreamSynchronize(stream_), "endpoint slice");
}

std::size_t nodal_footprint_bytes(const InstancePlan& plan) {
  const Config& c = plan.config;
  const std::size_t plane = static_cast<std::size_t>(c.nr) *
                            static_cast<std::size_t>(c.ntheta);
  std::size_t pairs = 0;
  for (const int target : c.targets) {
    for (const int m1 : c.parents) {
      if (std::binary_search(c.parents.begin(), c.parents.end(), target - m1)) {
        ++pairs;
      }
    }
  }
  const std::size_t complex_count =
      (kFullBuffers * kFieldCount + kScratchSlots) * c.modes.size() * plane +
      4 * std::max<std::size_t>(pairs, 1) * plane;
  return complex_count * sizeof(double2);
}

cudaError_t launch_diagnostics(const DiagnosticsLaunch& p, cudaStream_t stream) {
  const long long total = static_cast<long long>(p.modes) * p.nr * p.nt;
  diagnostics_kernel<<<grid_for(total), kBlock, 0, stream>>>(p);
  return cudaGetLastError();
}

const double2* NodalPipeline::state_device() const { return buf_->state; }
const double2* NodalPipeline::storage_rhs_device() const { return buf_->rhs_out; }
const double2* NodalPipeline::source_device() const { return buf_->source; }
const double2* NodalPipeline::forcing_device() const { return buf_->forcing; }

cudaError_t upload_nodal_sbp_constants() {
  const SbpConstants constants = build_sbp_constants();
  return cudaMemcpyToSymbol(c_sbp_nodal, &constants, sizeof(SbpConstants));
}

}  // namespace teuk_b200
