// CUDA kernels (sm_100a) of the B200 engine.
//
// stage_kernel is the hot path: one CTA per radial tile of one (solve, m)
// segment.  It
//   0. streams the tile's radial slab (plus halo) of the RK stage input
//      u = y + c k into shared memory (coalesced 16-byte loads),
//   1. evaluates psi_t = (P + 2K Q - G psi) / C_T on the tile rows plus a
//      derivative halo -- pointwise in band space for a = 0, and through
//      the Gauss-Legendre quadrature A diag(.) S for a != 0 (the implicit
//      Kerr ell-coupling of include/teuk/full_spatial.hpp:136-182 followed by
//      the band projection of include/teuk/spatial_pipeline.hpp:756-766),
//   2. applies the SBP first derivatives (closures + interior) and the
//      norm-compatible dissipation on every ell column, assembles P_t, Q_t,
//      psi_t (include/teuk/full_spatial.hpp:184-280, teukolsky.hpp:117-146)
//      and performs this stage's RK4 update (include/teuk/device_rk4.hpp:
//      84-128) in the same pass.
// All arithmetic is binary64.
#include <cstdio>
#include <mutex>
#include <type_traits>
#include <unordered_map>

#include "kernels.h"
#include "split_precision.cuh"

namespace teuk_b200 {

__constant__ SbpConstants c_sbp;

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kCoefCount = 10;

template <int DISC>
struct DiscTraits;
template <>
struct DiscTraits<kD42> {
  static constexpr int BR = 4, W = 6, HALF = 2, P = 3, SPECIAL = 4;
};
template <>
struct DiscTraits<kD84> {
  static constexpr int BR = 8, W = 12, HALF = 4, P = 5, SPECIAL = 8;
};
template <>
struct DiscTraits<kD105> {
  static constexpr int BR = 11, W = 16, HALF = 5, P = 6, SPECIAL = 11;
};

__device__ __forceinline__ double2 cadd(const double2 a, const double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(const double2 a, const double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 cscale(const double s, const double2 a) {
  return make_double2(s * a.x, s * a.y);
}
__device__ __forceinline__ double2 cmul(const double2 a, const double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cfma(const double s, const double2 a,
                                        const double2 acc) {
  return make_double2(fma(s, a.x, acc.x), fma(s, a.y, acc.y));
}

// Teukolsky point coefficients split into theta-independent parts
// (include/teuk/teukolsky.hpp:38-85); see RowCoefficients in engine.h.
__device__ void row_coefficients(const InstanceDesc& in, const int m,
                                 const int radial, double* out) {
  const double M = in.mass, a = in.spin, L = in.length;
  const double R = in.spacing * static_cast<double>(radial);
  const double L2 = L * L, L4 = L2 * L2, R2 = R * R, a2 = a * a;
  const double mrl = M * R / L2;
  const double s = static_cast<double>(kSpinWeight);
  const double mm = static_cast<double>(m);
  out[0] = 8.0 * M * (2.0 * M - a2 * R / L2) * (1.0 + 2.0 * mrl);
  out[1] = L2 - (8.0 * M * M - a2) * R2 / L2 + 4.0 * a2 * M * R * R2 / L4;
  out[2] = R2 / L4 * (L4 - 2.0 * L2 * M * R + a2 * R2);
  out[3] = 2.0 * (2.0 * M * (-s + (2.0 + s) * 2.0 * mrl - 3.0 * a2 * R2 / L4) -
                  a2 * R / L2);
  out[4] = 2.0 * a * mm * (1.0 + 4.0 * mrl);
  out[5] = 2.0 * R * (1.0 + s - (3.0 + s) * mrl + 2.0 * a2 * R2 / L4);
  out[6] = -(2.0 * a * mm * R2 / L2);
  out[7] = -2.0 * R * ((1.0 + s) * M / L2 - a2 * R / L4);
  out[8] = -(2.0 * a * mm * R / L2);
  out[9] = 1.0 / out[0];
}

// h * (D v)(r): v(q) = base[(q - s0) * stride], q in the resident slab.
template <int DISC>
__device__ __forceinline__ double2 sbp_derivative(const double2* base,
                                                  const int stride,
                                                  const int s0, const int r,
                                                  const int nr) {
  using T = DiscTraits<DISC>;
  double2 acc = make_double2(0.0, 0.0);
  if (r < T::BR) {
#pragma unroll
    for (int c = 0; c < T::W; ++c) {
      acc = cfma(c_sbp.left[DISC][r][c], base[(c - s0) * stride], acc);
    }
  } else if (r + T::BR >= nr) {
    const int rr = nr - 1 - r;
#pragma unroll
    for (int c = 0; c < T::W; ++c) {
      acc = cfma(-c_sbp.left[DISC][rr][c],
                 base[(nr - 1 - c - s0) * stride], acc);
    }
  } else {
    const double2* center = base + (r - s0) * stride;
#pragma unroll
    for (int k = T::HALF; k >= 1; --k) {
      acc = cfma(c_sbp.interior[DISC][k],
                 csub(center[k * stride], center[-k * stride]), acc);
    }
  }
  return acc;
}

// -(A^T A v)(r) / H_rr for the norm-compatible dissipation
// (include/teuk/radial_discretization.hpp:163-234); caller scales by sigma/h.
template <int DISC>
__device__ __forceinline__ double2 sbp_dissipation(const double2* base,
                                                   const int stride,
                                                   const int s0, const int r,
                                                   const int nr) {
  using T = DiscTraits<DISC>;
  double2 acc = make_double2(0.0, 0.0);
  if (r < T::SPECIAL) {
    for (int j = 0; j <= r + T::P; ++j) {
      acc = cfma(c_sbp.diss_left[DISC][r][j], base[(j - s0) * stride], acc);
    }
  } else if (r >= nr - T::SPECIAL) {
    const int rr = nr - 1 - r;
    for (int j = 0; j <= rr + T::P; ++j) {
      acc = cfma(c_sbp.diss_left[DISC][rr][j],
                 base[(nr - 1 - j - s0) * stride], acc);
    }
  } else {
    const double2* center = base + (r - s0) * stride;
    acc = cscale(c_sbp.diss_interior[DISC][0], center[0]);
#pragma unroll
    for (int k = 1; k <= T::P; ++k) {
      acc = cfma(c_sbp.diss_interior[DISC][k],
                 cadd(center[k * stride], center[-k * stride]), acc);
    }
  }
  return acc;
}

// Shared-memory geometry of one launch group (padded strides chosen so the
// 8x4 / 4x8 fragment loads of the FP64 MMA hit 32 distinct banks).
struct SmemLayout {
  int ne4, ne8, nt4, nt8;  // padded ell / theta extents
  int xs;                  // stride of the per-warp band staging rows
  int ts;                  // stride of the per-warp nodal staging columns
  int ss;                  // synthesis matrix row stride
  int as;                  // analysis matrix row stride
  __host__ __device__ static int round_up(const int v, const int m) {
    return (v + m - 1) / m * m;
  }
  __host__ __device__ static int bank_stride(const int v) {
    return 16 * ((v + 15) / 16) + 4;
  }
  __host__ __device__ explicit SmemLayout(const StageLaunch& p) {
    ne4 = round_up(p.max_ell, 4);
    ne8 = round_up(p.max_ell, 8);
    nt4 = round_up(p.max_theta, 4);
    nt8 = round_up(p.max_theta, 8);
    xs = bank_stride(ne4);
    ts = bank_stride(nt8);
    ss = bank_stride(ne4);
    as = bank_stride(nt4);
  }
  // double counts
  __host__ __device__ int warp_x() const { return 16 * xs; }
  __host__ __device__ int warp_t() const { return 8 * ts; }
  __host__ __device__ int synthesis() const { return nt8 * ss; }
  __host__ __device__ int analysis() const { return ne8 * as; }
};

// D = A * B + D for one 8x8x4 FP64 tile (mma.sync m8n8k4, FP64 tensor path).
__device__ __forceinline__ void dmma(double& c0, double& c1, const double a,
                                     const double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, "
      "{%0,%1};\n"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}

// psi_t = A diag(1/C_T) S (P + 2K Q - G0 psi) - i A diag(2 s a cos/C_T) S psi
// for rows [t0, t1) of one tile, four rows per warp iteration:
//   synthesis  C(j, col) = S(j, l) X(l, col), col = (row, {v1.re, v1.im,
//              psi.re, psi.im})            -> pointwise t_j on the nodes
//   analysis   psi_t(l, col2) = A(l, j) T(j, col2), col2 = (row, re/im).
__device__ void psi_t_transforms(const SmemLayout& L, const int ne,
                                 const int nt, const int t0, const int t1,
                                 const double2* u, const int s0, const int rs,
                                 const double2* qcol, const int qstride,
                                 const int qbase, const double* coef,
                                 const double* Sm, const double* Am,
                                 const double* sinv, const double* cosv,
                                 const double spin, double* xw, double* tw,
                                 double2* psit, const int warp,
                                 const int lane) {
  const double a2 = spin * spin;
  const double sa2 = 2.0 * (static_cast<double>(kSpinWeight) * spin);
  const int rows = t1 - t0;
  const int quad = lane & 3;
  const int group = lane >> 2;
  for (int b0 = warp * 4; b0 < rows; b0 += kWarps * 4) {
    // stage the band vectors of four rows: v1 = P + 2K Q - G0 psi, psi
    for (int idx = lane; idx < 4 * L.ne4; idx += 32) {
      const int rho = idx / L.ne4;
      const int l = idx - rho * L.ne4;
      const int rr = b0 + rho;
      double2 v1 = make_double2(0.0, 0.0), psi = make_double2(0.0, 0.0);
      if (rr < rows && l < ne) {
        const int r = t0 + rr;
        const double* cf = coef + rr * kCoefCount;
        const double2* row = u + (r - s0) * rs;
        const double2 Q = qcol[(r - qbase) * qstride + l];
        psi = row[2 * ne + l];
        v1 = csub(cadd(row[l], cscale(2.0 * cf[1], Q)),
                  cmul(make_double2(cf[3], cf[4]), psi));
      }
      xw[(rho * 4 + 0) * L.xs + l] = v1.x;
      xw[(rho * 4 + 1) * L.xs + l] = v1.y;
      xw[(rho * 4 + 2) * L.xs + l] = psi.x;
      xw[(rho * 4 + 3) * L.xs + l] = psi.y;
    }
    __syncwarp();
    // synthesis on the nodes and the pointwise Kerr factor
    for (int mt = 0; mt < L.nt8 / 8; ++mt) {
      double acc[2][2];
#pragma unroll
      for (int n = 0; n < 2; ++n) acc[n][0] = acc[n][1] = 0.0;
      for (int ks = 0; ks < L.ne4 / 4; ++ks) {
        const double a = Sm[(mt * 8 + group) * L.ss + ks * 4 + quad];
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          const double b = xw[(n * 8 + group) * L.xs + ks * 4 + quad];
          dmma(acc[n][0], acc[n][1], a, b);
        }
      }
      const int j = mt * 8 + group;
      // 1 / C_T for the two rows this lane finishes, issued before the
      // shuffles so the reciprocals overlap them
      double inv[2], gam = 0.0;
      const bool node = j < nt;
      if (node) gam = sa2 * cosv[j];
#pragma unroll
      for (int n = 0; n < 2; ++n) {
        const int rr = b0 + 2 * n + (quad >> 1);
        inv[n] = 0.0;
        if (rr < rows && node) {
          inv[n] = 1.0 / (coef[rr * kCoefCount] - a2 * sinv[j] * sinv[j]);
        }
      }
#pragma unroll
      for (int n = 0; n < 2; ++n) {
        // lane quad 0/2 holds a_j of a row, quad 1/3 holds b_j of that row
        const double o0 = __shfl_xor_sync(0xffffffffu, acc[n][0], 1);
        const double o1 = __shfl_xor_sync(0xffffffffu, acc[n][1], 1);
        if ((quad & 1) == 0) {
          const int rho = 2 * n + (quad >> 1);
          tw[(rho * 2 + 0) * L.ts + j] = (acc[n][0] + gam * o1) * inv[n];
          tw[(rho * 2 + 1) * L.ts + j] = (acc[n][1] - gam * o0) * inv[n];
        }
      }
    }
    __syncwarp();
    // analysis back onto the band
    for (int mt = 0; mt < L.ne8 / 8; ++mt) {
      // two accumulator pairs (even / odd K steps) halve the MMA chain
      double c0 = 0.0, c1 = 0.0, d0 = 0.0, d1 = 0.0;
      const int ksteps = L.nt4 / 4;
      int ks = 0;
      for (; ks + 1 < ksteps; ks += 2) {
        const double a = Am[(mt * 8 + group) * L.as + ks * 4 + quad];
        const double b = tw[group * L.ts + ks * 4 + quad];
        const double a2n = Am[(mt * 8 + group) * L.as + ks * 4 + 4 + quad];
        const double b2n = tw[group * L.ts + ks * 4 + 4 + quad];
        dmma(c0, c1, a, b);
        dmma(d0, d1, a2n, b2n);
      }
      if (ks < ksteps) {
        const double a = Am[(mt * 8 + group) * L.as + ks * 4 + quad];
        const double b = tw[group * L.ts + ks * 4 + quad];
        dmma(c0, c1, a, b);
      }
      c0 += d0;
      c1 += d1;
      const int l = mt * 8 + group;
      const int rr = b0 + quad;
      if (rr < rows && l < ne) psit[rr * ne + l] = make_double2(c0, c1);
    }
    __syncwarp();
  }
}

// psi_t_transforms for one padded shape known at compile time: the
// synthesis and analysis A-fragments are loaded once per warp and stay in
// registers for every row block.
template <int MTS, int KSS, int MTA, int KSA>
__device__ void psi_t_transforms_fixed(
    const SmemLayout& L, const int ne, const int nt, const int t0,
    const int t1, const double2* u, const int s0, const int rs,
    const double2* qcol, const int qstride, const int qbase,
    const double* coef, const double* Sm, const double* Am,
    const double* sinv, const double* cosv, const double spin, double* xw,
    double* tw, double2* psit, const int warp, const int lane) {
  const double a2 = spin * spin;
  const double sa2 = 2.0 * (static_cast<double>(kSpinWeight) * spin);
  const int rows = t1 - t0;
  const int quad = lane & 3;
  const int group = lane >> 2;
  double fs[MTS][KSS], fa[MTA][KSA];
#pragma unroll
  for (int mt = 0; mt < MTS; ++mt) {
#pragma unroll
    for (int ks = 0; ks < KSS; ++ks) {
      fs[mt][ks] = Sm[(mt * 8 + group) * L.ss + ks * 4 + quad];
    }
  }
#pragma unroll
  for (int mt = 0; mt < MTA; ++mt) {
#pragma unroll
    for (int ks = 0; ks < KSA; ++ks) {
      fa[mt][ks] = Am[(mt * 8 + group) * L.as + ks * 4 + quad];
    }
  }
  for (int b0 = warp * 4; b0 < rows; b0 += kWarps * 4) {
    for (int idx = lane; idx < 4 * L.ne4; idx += 32) {
      const int rho = idx / L.ne4;
      const int l = idx - rho * L.ne4;
      const int rr = b0 + rho;
      double2 v1 = make_double2(0.0, 0.0), psi = make_double2(0.0, 0.0);
      if (rr < rows && l < ne) {
        const int r = t0 + rr;
        const double* cf = coef + rr * kCoefCount;
        const double2* row = u + (r - s0) * rs;
        const double2 Q = qcol[(r - qbase) * qstride + l];
        psi = row[2 * ne + l];
        v1 = csub(cadd(row[l], cscale(2.0 * cf[1], Q)),
                  cmul(make_double2(cf[3], cf[4]), psi));
      }
      xw[(rho * 4 + 0) * L.xs + l] = v1.x;
      xw[(rho * 4 + 1) * L.xs + l] = v1.y;
      xw[(rho * 4 + 2) * L.xs + l] = psi.x;
      xw[(rho * 4 + 3) * L.xs + l] = psi.y;
    }
    __syncwarp();
    double bx[2][KSS];
#pragma unroll
    for (int n = 0; n < 2; ++n) {
#pragma unroll
      for (int ks = 0; ks < KSS; ++ks) {
        bx[n][ks] = xw[(n * 8 + group) * L.xs + ks * 4 + quad];
      }
    }
#pragma unroll
    for (int mt = 0; mt < MTS; ++mt) {
      double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
      for (int ks = 0; ks < KSS; ++ks) {
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          dmma(acc[n][0], acc[n][1], fs[mt][ks], bx[n][ks]);
        }
      }
      const int j = mt * 8 + group;
      double inv[2], gam = 0.0;
      const bool node = j < nt;
      if (node) gam = sa2 * cosv[j];
#pragma unroll
      for (int n = 0; n < 2; ++n) {
        const int rr = b0 + 2 * n + (quad >> 1);
        inv[n] = 0.0;
        if (rr < rows && node) {
          inv[n] = 1.0 / (coef[rr * kCoefCount] - a2 * sinv[j] * sinv[j]);
        }
      }
#pragma unroll
      for (int n = 0; n < 2; ++n) {
        const double o0 = __shfl_xor_sync(0xffffffffu, acc[n][0], 1);
        const double o1 = __shfl_xor_sync(0xffffffffu, acc[n][1], 1);
        if ((quad & 1) == 0) {
          const int rho = 2 * n + (quad >> 1);
          tw[(rho * 2 + 0) * L.ts + j] = (acc[n][0] + gam * o1) * inv[n];
          tw[(rho * 2 + 1) * L.ts + j] = (acc[n][1] - gam * o0) * inv[n];
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < MTA; ++mt) {
      double c[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
      for (int ks = 0; ks < KSA; ++ks) {
        const double b = tw[group * L.ts + ks * 4 + quad];
        dmma(c[ks & 1][0], c[ks & 1][1], fa[mt][ks], b);
      }
      const int l = mt * 8 + group;
      const int rr = b0 + quad;
      if (rr < rows && l < ne) {
        psit[rr * ne + l] = make_double2(c[0][0] + c[1][0], c[0][1] + c[1][1]);
      }
    }
    __syncwarp();
  }
}

// The same psi_t on the FP64 CUDA cores: one warp per row, lanes over the
// Gauss-Legendre nodes for the synthesis and over ell for the analysis.
__device__ void psi_t_scalar(const SmemLayout& L, const int ne, const int nt,
                             const int t0, const int t1, const double2* u,
                             const int s0, const int rs, const double2* qcol,
                             const int qstride, const int qbase,
                             const double* coef, const double* Sm,
                             const double* Am, const double* sinv,
                             const double* cosv, const double spin,
                             double* xw, double* tw, double2* psit,
                             const int warp, const int lane) {
  const double a2 = spin * spin;
  const double sa2 = 2.0 * (static_cast<double>(kSpinWeight) * spin);
  double2* v1 = reinterpret_cast<double2*>(xw);
  double2* tj = reinterpret_cast<double2*>(tw);
  for (int rr = warp; rr < t1 - t0; rr += kWarps) {
    const int r = t0 + rr;
    const double* cf = coef + rr * kCoefCount;
    const double2* row = u + (r - s0) * rs;
    const double2 G0 = make_double2(cf[3], cf[4]);
    for (int l = lane; l < ne; l += 32) {
      const double2 Q = qcol[(r - qbase) * qstride + l];
      v1[l] = csub(cadd(row[l], cscale(2.0 * cf[1], Q)),
                   cmul(G0, row[2 * ne + l]));
    }
    __syncwarp();
    for (int j = lane; j < nt; j += 32) {
      double2 sa = make_double2(0.0, 0.0);
      double2 sb = make_double2(0.0, 0.0);
      for (int l = 0; l < ne; ++l) {
        const double s = Sm[j * L.ss + l];
        sa = cfma(s, v1[l], sa);
        sb = cfma(s, row[2 * ne + l], sb);
      }
      const double gamma = sa2 * cosv[j];
      const double ct = cf[0] - a2 * sinv[j] * sinv[j];
      tj[j] = make_double2((sa.x + gamma * sb.y) / ct,
                           (sa.y - gamma * sb.x) / ct);
    }
    __syncwarp();
    for (int l = lane; l < ne; l += 32) {
      double2 acc = make_double2(0.0, 0.0);
      for (int j = 0; j < nt; ++j) acc = cfma(Am[l * L.as + j], tj[j], acc);
      psit[rr * ne + l] = acc;
    }
    __syncwarp();
  }
}

#ifndef TEUK_TRANSFORM_MMA
#define TEUK_TRANSFORM_MMA 1
#endif

// Register window of RB output rows plus a halo of H rows on each side.
template <int RB, int H>
__device__ __forceinline__ void load_window(double2 (&w)[RB + 2 * H],
                                            const double2* col,
                                            const int stride, const int base,
                                            const int ra) {
#pragma unroll
  for (int i = 0; i < RB + 2 * H; ++i) {
    w[i] = col[(ra - H + i - base) * stride];
  }
}

template <int DISC, int RB, int H>
__device__ __forceinline__ double2 window_derivative(
    const double2 (&w)[RB + 2 * H], const int i) {
  using T = DiscTraits<DISC>;
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll
  for (int k = T::HALF; k >= 1; --k) {
    acc = cfma(c_sbp.interior[DISC][k], csub(w[i + H + k], w[i + H - k]), acc);
  }
  return acc;
}

template <int DISC, int RB, int H>
__device__ __forceinline__ double2 window_dissipation(
    const double2 (&w)[RB + 2 * H], const int i) {
  using T = DiscTraits<DISC>;
  double2 acc = cscale(c_sbp.diss_interior[DISC][0], w[i + H]);
#pragma unroll
  for (int k = 1; k <= T::P; ++k) {
    acc = cfma(c_sbp.diss_interior[DISC][k], cadd(w[i + H + k], w[i + H - k]),
               acc);
  }
  return acc;
}

// Hint the L2 to fetch [ptr, ptr + bytes) (bulk prefetch; no completion to
// wait for, no effect on results).  Sizes are multiples of 16 bytes.
__device__ __forceinline__ void l2_prefetch(const double2* ptr,
                                            long long count) {
  const char* c = reinterpret_cast<const char*>(ptr);
  long long bytes = count * static_cast<long long>(sizeof(double2));
  while (bytes > 0) {
    const unsigned chunk =
        bytes > 65536 ? 65536u : static_cast<unsigned>(bytes);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                 :
                 : "l"(c), "r"(chunk)
                 : "memory");
    c += chunk;
    bytes -= chunk;
  }
}

// L2 prefetch of what tile t reads from HBM: its slab of RK stage inputs
// (rows within H of the tile) and the own-row inputs of its RK update.
__device__ void prefetch_tile(const StageLaunch& p, const int t, const int H,
                              const bool slab, const bool update) {
  const TileDesc tile = p.tiles[t];
  const SegmentDesc seg = p.segments[tile.segment];
  const int nr = p.instances[seg.instance].nr;
  const long long rs = 3LL * seg.n_ell;
  if (slab) {
    const int s0 = max(0, tile.r0 - H), s1 = min(nr, tile.r1 + H);
    const long long off = seg.offset + s0 * rs, n = (s1 - s0) * rs;
    if (p.stage == kStage4) {
      l2_prefetch(p.kA + off, n);
    } else {
      l2_prefetch(p.y + off, n);
      if (p.stage == kStage2) l2_prefetch(p.kA + off, n);
      if (p.stage == kStage3) l2_prefetch(p.kB + off, n);
    }
  }
  if (update) {
    const long long off = seg.offset + tile.r0 * rs;
    const long long n = (tile.r1 - tile.r0) * rs;
    if (p.stage == kStage2) l2_prefetch(p.kA + off, n);
    if (p.stage == kStage3) {
      l2_prefetch(p.y + off, n);
      l2_prefetch(p.acc + off, n);
    }
    if (p.stage == kStage4) l2_prefetch(p.acc + off, n);
  }
}

#ifndef TEUK_ROW_BLOCK
#define TEUK_ROW_BLOCK 2
#endif
constexpr int kRowBlock = TEUK_ROW_BLOCK;

template <int DISC, int SC>
__global__ void __launch_bounds__(kThreads, 2)
    stage_kernel(const StageLaunch p) {
  using T = DiscTraits<DISC>;
  extern __shared__ double2 smem[];
  const TileDesc tile = p.tiles[blockIdx.x];
  const SegmentDesc seg = p.segments[tile.segment];
  const InstanceDesc in = p.instances[seg.instance];
  const SmemLayout L(p);
  const int nr = in.nr;
  const int ne = seg.n_ell;
  const int nt = in.ntheta;
  const int rs = 3 * ne;
  constexpr int H = SC ? (T::P > 2 * T::HALF ? T::P : 2 * T::HALF) : T::P;
  constexpr int HD = T::HALF;
  const int r0 = tile.r0, r1 = tile.r1;
  const int s0 = max(0, r0 - H), s1 = min(nr, r1 + H);
  const int t0 = max(0, r0 - HD), t1 = min(nr, r1 + HD);
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;

  double2* u = smem;                        // slab rows x rs
  double2* psit = u + p.slab_capacity;      // t-rows x ne
  double2* qeff = psit + p.dslab_capacity;  // t-rows x ne (SC)
  double* dbase = reinterpret_cast<double*>(qeff + (SC ? p.dslab_capacity : 0));
  double* xw = dbase + warp * (L.warp_x() + L.warp_t());
  double* tw = xw + L.warp_x();
  double* Sm = dbase + kWarps * (L.warp_x() + L.warp_t());
  double* Am = Sm + L.synthesis();
  double* sinv = Am + L.analysis();
  double* cosv = sinv + L.nt8;
  double* coef = cosv + L.nt8;  // t-rows x kCoefCount

  // L2 prefetches: the own-row RK update inputs of this tile, and the slab
  // and update inputs of the tile that takes this CTA's slot next
  if (tid == 0 && p.prefetch_stride > 0) {
    prefetch_tile(p, blockIdx.x, H, false, true);
    const int next = blockIdx.x + p.prefetch_stride;
    if (next < p.tile_count) prefetch_tile(p, next, H, true, true);
  }

  // ---- phase 0: RK stage input over the slab, matrices, coefficients
  {
    const long long base = seg.offset + static_cast<long long>(s0) * rs;
    const int count = (s1 - s0) * rs;
    const double hdt = 0.5 * in.dt;
    const double2* __restrict__ y = p.y + base;
    constexpr int U = 8;
    if (p.stage == kStage1 || p.stage == kRhsOnly || p.stage == kStage4) {
      const double2* __restrict__ src = p.stage == kStage4 ? p.kA + base : y;
      for (int i0 = tid; i0 < count; i0 += kThreads * U) {
        double2 v[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
          const int i = i0 + k * kThreads;
          if (i < count) v[k] = __ldg(src + i);
        }
#pragma unroll
        for (int k = 0; k < U; ++k) {
          const int i = i0 + k * kThreads;
          if (i < count) u[i] = v[k];
        }
      }
    } else {
      const double2* __restrict__ kk =
          (p.stage == kStage2 ? p.kA : p.kB) + base;
      for (int i0 = tid; i0 < count; i0 += kThreads * U) {
        double2 yv[U], kv[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
          const int i = i0 + k * kThreads;
          if (i < count) {
            yv[k] = __ldg(y + i);
            kv[k] = __ldg(kk + i);
          }
        }
#pragma unroll
        for (int k = 0; k < U; ++k) {
          const int i = i0 + k * kThreads;
          if (i < count) {
            u[i] = make_double2(yv[k].x + hdt * kv[k].x,
                                yv[k].y + hdt * kv[k].y);
          }
        }
      }
    }
    if (in.spin != 0.0) {
      const double* S = p.matrices + seg.mat_offset;  // St[l][j]
      const double* A = S + ne * nt;                  // At[j][l]
      for (int i = tid; i < L.nt8 * L.ne4; i += kThreads) {
        const int j = i / L.ne4, l = i - (i / L.ne4) * L.ne4;
        Sm[j * L.ss + l] = (j < nt && l < ne) ? S[l * nt + j] : 0.0;
      }
      for (int i = tid; i < L.ne8 * L.nt4; i += kThreads) {
        const int l = i / L.nt4, j = i - (i / L.nt4) * L.nt4;
        Am[l * L.as + j] = (j < nt && l < ne) ? A[j * ne + l] : 0.0;
      }
      for (int j = tid; j < L.nt8; j += kThreads) {
        sinv[j] = j < nt ? p.trig[in.trig_offset + j] : 0.0;
        cosv[j] = j < nt ? p.trig[in.trig_offset + nt + j] : 0.0;
      }
      // zero the nodal staging columns beyond the analysis K extent
      for (int i = lane; i < L.warp_t(); i += 32) tw[i] = 0.0;
    }
    for (int r = t0 + tid; r < t1; r += kThreads) {
      row_coefficients(in, seg.m, r, coef + (r - t0) * kCoefCount);
    }
  }
  __syncthreads();

  // effective Q (include/teuk/full_spatial.hpp:99-134)
  const double2* qcol;
  int qstride, qbase;
  if (SC) {
    for (int i = tid; i < (t1 - t0) * ne; i += kThreads) {
      const int r = t0 + i / ne;
      const int l = i - (i / ne) * ne;
      qeff[i] = cscale(in.inv_spacing,
                       sbp_derivative<DISC>(u + 2 * ne + l, rs, s0, r, nr));
    }
    __syncthreads();
    qcol = qeff;
    qstride = ne;
    qbase = t0;
  } else {
    qcol = u + ne;
    qstride = rs;
    qbase = s0;
  }

  // ---- phase 1: psi_t on rows [t0, t1)
  if (in.spin == 0.0) {
    for (int i = tid; i < (t1 - t0) * ne; i += kThreads) {
      const int rr = i / ne;
      const int l = i - rr * ne;
      const int r = t0 + rr;
      const double* cf = coef + rr * kCoefCount;
      const double2 P = u[(r - s0) * rs + l];
      const double2 Q = qcol[(r - qbase) * qstride + l];
      const double2 psi = u[(r - s0) * rs + 2 * ne + l];
      const double2 G = make_double2(cf[3], cf[4]);
      const double2 num = csub(cadd(P, cscale(2.0 * cf[1], Q)), cmul(G, psi));
      psit[i] = cscale(cf[9], num);
    }
  } else if (TEUK_TRANSFORM_MMA && L.nt8 == 32 && L.ne4 == 16 &&
             L.ne8 == 16 && L.nt4 == 28) {
    psi_t_transforms_fixed<4, 4, 2, 7>(L, ne, nt, t0, t1, u, s0, rs, qcol,
                                       qstride, qbase, coef, Sm, Am, sinv,
                                       cosv, in.spin, xw, tw, psit, warp,
                                       lane);
  } else if (TEUK_TRANSFORM_MMA) {
    psi_t_transforms(L, ne, nt, t0, t1, u, s0, rs, qcol, qstride, qbase, coef,
                     Sm, Am, sinv, cosv, in.spin, xw, tw, psit, warp, lane);
  } else {
    psi_t_scalar(L, ne, nt, t0, t1, u, s0, rs, qcol, qstride, qbase, coef, Sm,
                 Am, sinv, cosv, in.spin, xw, tw, psit, warp, lane);
  }
  __syncthreads();

  // ---- phase 2: RHS assembly and RK update on rows [r0, r1)
  const double inv_h = in.inv_spacing;
  const double diss_scale = in.dissipation * inv_h;
  const bool dissipate = in.dissipation > 0.0;
  const double damping = in.damping;
  const double dt = in.dt;
  const double dt6 = in.dt / 6.0;
  const int chunks = (r1 - r0 + kRowBlock - 1) / kRowBlock;
  const int items = chunks * ne;
  // With at most one work item per thread the stage results are parked in
  // the slab (after every window has read it) and the RK update runs as one
  // coalesced streaming pass over the tile's rows; otherwise each item
  // updates its own rows directly.
  const bool park = items <= kThreads;
  for (int item0 = 0; item0 < items; item0 += kThreads) {
    const int item = item0 + tid;
    const bool active = item < items;
    int l = 0, ra = r0, rows = 0;
    double2 kP[kRowBlock], kQ[kRowBlock], kpsi[kRowBlock];
    if (active) {
      const int chunk = item / ne;
      l = item - chunk * ne;
      ra = r0 + chunk * kRowBlock;
      rows = min(kRowBlock, r1 - ra);
      const int ell = seg.ell_min + l;
      const double lambda = -static_cast<double>((ell - kSpinWeight) *
                                                 (ell + kSpinWeight + 1));
      const bool interior =
          rows == kRowBlock && ra >= T::BR && ra + kRowBlock + T::BR <= nr;
      if (interior) {
        {  // psi: D psi (constraint), dissipation, (c_psi + lambda) psi
          double2 w[kRowBlock + 2 * T::P];
          load_window<kRowBlock, T::P>(w, u + 2 * ne + l, rs, s0, ra);
  #pragma unroll
          for (int i = 0; i < kRowBlock; ++i) {
            const double* cf = coef + (ra + i - t0) * kCoefCount;
            const double2 dpsi =
                cscale(inv_h, window_derivative<DISC, kRowBlock, T::P>(w, i));
            kQ[i] = cscale(damping, dpsi);
            kpsi[i] = dissipate
                          ? cscale(diss_scale,
                                   window_dissipation<DISC, kRowBlock, T::P>(w, i))
                          : make_double2(0.0, 0.0);
            const double2 psi = w[i + T::P];
            kP[i] = cadd(cmul(make_double2(cf[7], cf[8]), psi),
                         cscale(lambda, psi));
          }
        }
        {  // Q: -gamma Q, dissipation; free-damped: H_R D Q + q Q
          double2 w[kRowBlock + 2 * T::P];
          load_window<kRowBlock, T::P>(w, u + ne + l, rs, s0, ra);
  #pragma unroll
          for (int i = 0; i < kRowBlock; ++i) {
            const double* cf = coef + (ra + i - t0) * kCoefCount;
            const double2 Q = w[i + T::P];
            kQ[i] = csub(kQ[i], cscale(damping, Q));
            if (dissipate) {
              kQ[i] = cfma(diss_scale,
                           window_dissipation<DISC, kRowBlock, T::P>(w, i),
                           kQ[i]);
            }
            if (!SC) {
              const double2 dq =
                  cscale(inv_h, window_derivative<DISC, kRowBlock, T::P>(w, i));
              kP[i] = cadd(kP[i], cscale(cf[2], dq));
              kP[i] = cadd(kP[i], cmul(make_double2(cf[5], cf[6]), Q));
            }
          }
        }
        if (SC) {  // stage-constrained effective Q = D psi
          double2 w[kRowBlock + 2 * T::HALF];
          load_window<kRowBlock, T::HALF>(w, qeff + l, ne, t0, ra);
  #pragma unroll
          for (int i = 0; i < kRowBlock; ++i) {
            const double* cf = coef + (ra + i - t0) * kCoefCount;
            const double2 dq = cscale(
                inv_h, window_derivative<DISC, kRowBlock, T::HALF>(w, i));
            kP[i] = cadd(kP[i], cscale(cf[2], dq));
            kP[i] = cadd(kP[i], cmul(make_double2(cf[5], cf[6]), w[i + T::HALF]));
          }
        }
        if (dissipate) {  // P: dissipation only
          double2 w[kRowBlock + 2 * T::P];
          load_window<kRowBlock, T::P>(w, u + l, rs, s0, ra);
  #pragma unroll
          for (int i = 0; i < kRowBlock; ++i) {
            kP[i] = cfma(diss_scale,
                         window_dissipation<DISC, kRowBlock, T::P>(w, i), kP[i]);
          }
        }
        {  // psi_t: D psi_t into Q_t, psi_t itself
          double2 w[kRowBlock + 2 * T::HALF];
          load_window<kRowBlock, T::HALF>(w, psit + l, ne, t0, ra);
  #pragma unroll
          for (int i = 0; i < kRowBlock; ++i) {
            kQ[i] = cadd(kQ[i], cscale(inv_h, window_derivative<DISC, kRowBlock,
                                                                T::HALF>(w, i)));
            kpsi[i] = cadd(kpsi[i], w[i + T::HALF]);
          }
        }
      } else {
        for (int i = 0; i < rows; ++i) {
          const int r = ra + i;
          const double* cf = coef + (r - t0) * kCoefCount;
          const double2* urow = u + (r - s0) * rs;
          const double2 Qs = urow[ne + l];
          const double2 psi = urow[2 * ne + l];
          const double2 Qe = qcol[(r - qbase) * qstride + l];
          const double2 dpsi =
              cscale(inv_h, sbp_derivative<DISC>(u + 2 * ne + l, rs, s0, r, nr));
          const double2 dq = cscale(
              inv_h, sbp_derivative<DISC>(qcol + l, qstride, qbase, r, nr));
          const double2 dpsit =
              cscale(inv_h, sbp_derivative<DISC>(psit + l, ne, t0, r, nr));
          double2 P_t = cscale(cf[2], dq);
          P_t = cadd(P_t, cmul(make_double2(cf[5], cf[6]), Qe));
          P_t = cadd(P_t, cmul(make_double2(cf[7], cf[8]), psi));
          P_t = cadd(P_t, cscale(lambda, psi));
          double2 Q_t = csub(dpsit, cscale(damping, csub(Qs, dpsi)));
          double2 psi_t = psit[(r - t0) * ne + l];
          if (dissipate) {
            P_t = cfma(diss_scale, sbp_dissipation<DISC>(u + l, rs, s0, r, nr),
                       P_t);
            Q_t = cfma(diss_scale,
                       sbp_dissipation<DISC>(u + ne + l, rs, s0, r, nr), Q_t);
            psi_t = cfma(diss_scale,
                         sbp_dissipation<DISC>(u + 2 * ne + l, rs, s0, r, nr),
                         psi_t);
          }
          kP[i] = P_t;
          kQ[i] = Q_t;
          kpsi[i] = psi_t;
        }
      }
    }
    if (park) {
      __syncthreads();  // every window has finished reading the slab
      if (active) {
        for (int i = 0; i < rows; ++i) {
          double2* dst = u + (ra + i - s0) * rs + l;
          dst[0] = kP[i];
          dst[ne] = kQ[i];
          dst[2 * ne] = kpsi[i];
        }
      }
    } else if (active) {
        // RK update: every own-row input is loaded before any store so the
        // global loads are in flight together.
        const long long g0 = seg.offset + static_cast<long long>(ra) * rs + l;
        double2 in0[kRowBlock][3], in1[kRowBlock][3];
        const double2* __restrict__ src0 =
            p.stage == kStage2 ? p.kA : (p.stage == kStage3 ? p.y : p.acc);
        const double2* __restrict__ src1 = p.acc;
    #pragma unroll
        for (int i = 0; i < kRowBlock; ++i) {
    #pragma unroll
          for (int f = 0; f < 3; ++f) {
            in0[i][f] = make_double2(0.0, 0.0);
            in1[i][f] = make_double2(0.0, 0.0);
            if (i < rows && p.stage != kStage1 && p.stage != kRhsOnly) {
              const long long gi = g0 + static_cast<long long>(i) * rs + f * ne;
              in0[i][f] = src0[gi];
              if (p.stage == kStage3) in1[i][f] = src1[gi];
            }
          }
        }
    #pragma unroll
        for (int i = 0; i < kRowBlock; ++i) {
          if (i >= rows) break;
          const double2 k[3] = {kP[i], kQ[i], kpsi[i]};
    #pragma unroll
          for (int f = 0; f < 3; ++f) {
            const long long gi = g0 + static_cast<long long>(i) * rs + f * ne;
            switch (p.stage) {
              case kStage1:
              case kRhsOnly:
                p.kA[gi] = k[f];
                break;
              case kStage2:  // in0 = k1
                p.kB[gi] = k[f];
                p.acc[gi] = cfma(2.0, k[f], in0[i][f]);
                break;
              case kStage3: {  // in0 = y, in1 = k1 + 2 k2
                const double2 acc = cfma(2.0, k[f], in1[i][f]);
                p.acc[gi] = cfma(dt6, acc, in0[i][f]);
                p.kA[gi] = cfma(dt, k[f], in0[i][f]);
                break;
              }
              case kStage4:  // in0 = y + dt/6 (k1 + 2 k2 + 2 k3)
                p.y[gi] = cfma(dt6, k[f], in0[i][f]);
                break;
            }
          }
        }
    }
  }
  if (park) {
    __syncthreads();
    const int count = (r1 - r0) * rs;
    const double2* kk = u + (r0 - s0) * rs;
    const long long g0 = seg.offset + static_cast<long long>(r0) * rs;
    constexpr int V = 4;
    for (int i0 = tid; i0 < count; i0 += kThreads * V) {
      double2 a[V], b[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const int i = i0 + v * kThreads;
        a[v] = b[v] = make_double2(0.0, 0.0);
        if (i < count) {
          switch (p.stage) {
            case kStage2: a[v] = p.kA[g0 + i]; break;
            case kStage3: a[v] = p.y[g0 + i]; b[v] = p.acc[g0 + i]; break;
            case kStage4: a[v] = p.acc[g0 + i]; break;
            default: break;
          }
        }
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const int i = i0 + v * kThreads;
        if (i >= count) break;
        const double2 k = kk[i];
        const long long g = g0 + i;
        switch (p.stage) {
          case kStage1:
          case kRhsOnly:
            p.kA[g] = k;
            break;
          case kStage2:  // a = k1
            p.kB[g] = k;
            p.acc[g] = cfma(2.0, k, a[v]);
            break;
          case kStage3: {  // a = y, b = k1 + 2 k2
            const double2 acc = cfma(2.0, k, b[v]);
            p.acc[g] = cfma(dt6, acc, a[v]);
            p.kA[g] = cfma(dt, k, a[v]);
            break;
          }
          case kStage4:  // a = y + dt/6 (k1 + 2 k2 + 2 k3)
            p.y[g] = cfma(dt6, k, a[v]);
            break;
        }
      }
    }
  }
}

#include "stream_kernel.cuh"

// Launch set-up of one kernel on one device: the dynamic shared-memory
// opt-in (an attribute of the function on each device), the SM count, the
// registers the compiled kernel is launched with and the resident CTAs for
// a shared-memory size.  Kept per device, because one process may run
// pipelines on several devices, and behind a mutex, because several host
// threads may launch at once.
struct KernelSetup {
  int configured_bytes = 0;
  int sms = 0;
  int launch_regs = -1;
  size_t resident_bytes = 0;
  int resident = 0;
};

class KernelSetups {
 public:
  // Runs `body(setup)` on the calling device's record under the lock.
  template <class Body>
  cudaError_t with(Body&& body) {
    int device = 0;
    const cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return err;
    std::lock_guard<std::mutex> lock(mutex_);
    return body(per_device_[device], device);
  }

 private:
  std::mutex mutex_;
  std::unordered_map<int, KernelSetup> per_device_;
};

static_assert(kSplitRecord == kSplitRecordUint4, "split record size");
static_assert(kSplitScales == kSplitScaleDoubles, "split scale count");

template <int DISC, int SC, int PREC, int STAGE>
cudaError_t launch_stream_stage(const StageLaunch& p, cudaStream_t stream) {
  const size_t bytes = StreamLayout(SC).total;
  auto kernel = stream_stage_kernel<DISC, SC, PREC, STAGE>;
  static KernelSetups setups;
  int sms = 0;
  const cudaError_t setup_err = setups.with([&](KernelSetup& k, const int device) {
    if (k.configured_bytes != static_cast<int>(bytes)) {
      const cudaError_t err = cudaFuncSetAttribute(
          kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
          static_cast<int>(bytes));
      if (err != cudaSuccess) return err;
      k.configured_bytes = static_cast<int>(bytes);
    }
    if (k.sms == 0) {
      const cudaError_t err = cudaDeviceGetAttribute(
          &k.sms, cudaDevAttrMultiProcessorCount, device);
      if (err != cudaSuccess) return err;
    }
    // The warpgroups' setmaxnreg requests must fit the registers the CTA
    // is launched with; a larger request would never be granted.
    if (k.launch_regs < 0) {
      cudaFuncAttributes attributes{};
      const cudaError_t err = cudaFuncGetAttributes(&attributes, kernel);
      if (err != cudaSuccess) return err;
      k.launch_regs = attributes.numRegs;
    }
    if (k.launch_regs != kStreamLaunchRegs ||
        k.launch_regs * kStreamThreads < kStreamRegisterDemand) {
      return cudaErrorInvalidConfiguration;
    }
    sms = k.sms;
    return cudaSuccess;
  });
  if (setup_err != cudaSuccess) return setup_err;
  const int grid = p.strip_count < sms ? p.strip_count : sms;
  kernel<<<grid, kStreamThreads, bytes, stream>>>(p);
  return cudaGetLastError();
}

template <int DISC, int SC, int PREC>
cudaError_t launch_stream_typed(const StageLaunch& p, cudaStream_t stream) {
  switch (p.stage) {
    case kStage1: return launch_stream_stage<DISC, SC, PREC, kStage1>(p, stream);
    case kStage2: return launch_stream_stage<DISC, SC, PREC, kStage2>(p, stream);
    case kStage3: return launch_stream_stage<DISC, SC, PREC, kStage3>(p, stream);
    case kStage4: return launch_stream_stage<DISC, SC, PREC, kStage4>(p, stream);
    default: return launch_stream_stage<DISC, SC, PREC, kRhsOnly>(p, stream);
  }
}

template <int DISC, int STAGE>
cudaError_t launch_wide_stage(const StageLaunch& p, cudaStream_t stream) {
  const size_t bytes = WideLayout().total;
  auto kernel = stream_wide_kernel<DISC, STAGE>;
  static KernelSetups setups;
  int sms = 0;
  const cudaError_t setup_err = setups.with([&](KernelSetup& k, const int device) {
    if (k.configured_bytes != static_cast<int>(bytes)) {
      const cudaError_t err = cudaFuncSetAttribute(
          kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
          static_cast<int>(bytes));
      if (err != cudaSuccess) return err;
      k.configured_bytes = static_cast<int>(bytes);
    }
    if (k.sms == 0) {
      const cudaError_t err = cudaDeviceGetAttribute(
          &k.sms, cudaDevAttrMultiProcessorCount, device);
      if (err != cudaSuccess) return err;
    }
    // the setmaxnreg requests must fit the launch allocation
    if (k.launch_regs < 0) {
      cudaFuncAttributes attributes{};
      const cudaError_t err = cudaFuncGetAttributes(&attributes, kernel);
      if (err != cudaSuccess) return err;
      k.launch_regs = attributes.numRegs;
    }
    if (k.launch_regs != kStreamLaunchRegs) return cudaErrorInvalidConfiguration;
    sms = k.sms;
    return cudaSuccess;
  });
  if (setup_err != cudaSuccess) return setup_err;
  const int grid = p.strip_count < sms ? p.strip_count : sms;
  kernel<<<grid, kStreamThreads, bytes, stream>>>(p);
  return cudaGetLastError();
}

template <int DISC>
cudaError_t launch_wide_typed(const StageLaunch& p, cudaStream_t stream) {
  switch (p.stage) {
    case kStage1: return launch_wide_stage<DISC, kStage1>(p, stream);
    case kStage2: return launch_wide_stage<DISC, kStage2>(p, stream);
    case kStage3: return launch_wide_stage<DISC, kStage3>(p, stream);
    case kStage4: return launch_wide_stage<DISC, kStage4>(p, stream);
    default: return launch_wide_stage<DISC, kRhsOnly>(p, stream);
  }
}

template <int DISC, int SC>
cudaError_t launch_typed(const StageLaunch& p, cudaStream_t stream) {
  if (p.strips != nullptr && p.strip_count > 0) {
    if (p.wide != 0) {
      // free-damped FP64 only (the host never builds other wide groups)
      if (SC != 0 || p.precision != 0) return cudaErrorInvalidValue;
      return launch_wide_typed<DISC>(p, stream);
    }
    return p.precision == 1 ? launch_stream_typed<DISC, SC, 1>(p, stream)
                            : launch_stream_typed<DISC, SC, 0>(p, stream);
  }
  const size_t bytes = stage_smem_bytes(p);
  auto kernel = stage_kernel<DISC, SC>;
  static KernelSetups setups;
  int resident = 0;
  const cudaError_t setup_err = setups.with([&](KernelSetup& k, const int device) {
    // The opt-in limit is raised to the largest size requested so far on
    // this device (never inside a launch sequence that needs less).
    if (static_cast<int>(bytes) > k.configured_bytes) {
      const cudaError_t err = cudaFuncSetAttribute(
          kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
          static_cast<int>(bytes));
      if (err != cudaSuccess) return err;
      k.configured_bytes = static_cast<int>(bytes);
    }
    // resident CTAs for this shared-memory size, cached per size
    if (bytes != k.resident_bytes) {
      int sms = 0, per_sm = 0;
      cudaError_t err =
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
      if (err == cudaSuccess) {
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel,
                                                            kThreads, bytes);
      }
      if (err != cudaSuccess) return err;
      k.resident = sms * per_sm;
      k.resident_bytes = bytes;
    }
    resident = k.resident;
    return cudaSuccess;
  });
  if (setup_err != cudaSuccess) return setup_err;
  StageLaunch q = p;
  q.prefetch_stride = resident;
  kernel<<<p.tile_count, kThreads, bytes, stream>>>(q);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- conversions
__global__ void nodal_to_modal_kernel(const ConvertLaunch p) {
  // one thread per (segment, r, field, ell)
  const long long total = static_cast<long long>(p.segment_count) * p.nr * 3 *
                          p.max_ell;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) +
                       threadIdx.x;
       idx < total; idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int l = static_cast<int>(idx % p.max_ell);
    long long rest = idx / p.max_ell;
    const int f = static_cast<int>(rest % 3);
    rest /= 3;
    const int r = static_cast<int>(rest % p.nr);
    const int s = static_cast<int>(rest / p.nr);
    const SegmentDesc seg = p.segments[s];
    if (l >= seg.n_ell) continue;
    const int mode = p.segment_modes[s];
    const int ne = seg.n_ell;
    const double* A = p.matrices + seg.mat_offset + ne * p.ntheta;  // At[j][l]
    const double2* line =
        p.nodal_in +
        ((static_cast<long long>(mode) * kFieldCount + f) * p.nr + r) *
            p.ntheta;
    double2 acc = make_double2(0.0, 0.0);
    for (int j = 0; j < p.ntheta; ++j) acc = cfma(A[j * ne + l], line[j], acc);
    p.modal[seg.offset + static_cast<long long>(r) * 3 * ne + f * ne + l] = acc;
  }
}

__global__ void modal_to_nodal_kernel(const ConvertLaunch p) {
  const long long total =
      static_cast<long long>(p.segment_count) * p.nr * 3 * p.ntheta;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) +
                       threadIdx.x;
       idx < total; idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(idx % p.ntheta);
    long long rest = idx / p.ntheta;
    const int f = static_cast<int>(rest % 3);
    rest /= 3;
    const int r = static_cast<int>(rest % p.nr);
    const int s = static_cast<int>(rest / p.nr);
    const SegmentDesc seg = p.segments[s];
    const int mode = p.segment_modes[s];
    const int ne = seg.n_ell;
    const double* St = p.matrices + seg.mat_offset;  // St[l][j]
    const double2* row =
        p.modal + seg.offset + static_cast<long long>(r) * 3 * ne + f * ne;
    double2 acc = make_double2(0.0, 0.0);
    for (int l = 0; l < ne; ++l) acc = cfma(St[l * p.ntheta + j], row[l], acc);
    p.nodal_out[((static_cast<long long>(mode) * kFieldCount + f) * p.nr + r) *
                    p.ntheta +
                j] = acc;
  }
}

__global__ void frozen_scan_kernel(const double2* nodal,
                                   const int* parent_mask, const int modes,
                                   const int plane_values, int* flag) {
  const long long total =
      static_cast<long long>(modes) * kFieldCount * plane_values;
  bool nonzero = false;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) +
                       threadIdx.x;
       idx < total; idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long plane = idx / plane_values;
    const int field = static_cast<int>(plane % kFieldCount);
    const int mode = static_cast<int>(plane / kFieldCount);
    if (field < 3 && parent_mask[mode] != 0) continue;
    const double2 v = nodal[idx];
    nonzero |= (v.x != 0.0) || (v.y != 0.0);
  }
  if (__any_sync(0xffffffffu, nonzero) && (threadIdx.x & 31) == 0) {
    atomicOr(flag, 1);
  }
}

__global__ void endpoint_gather_kernel(const double2* y,
                                       const SegmentDesc* segments,
                                       const InstanceDesc* instances,
                                       const int segment_count,
                                       const int max_ell, double2* out) {
  const int total = segment_count * 2 * max_ell;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += gridDim.x * blockDim.x) {
    const int l = idx % max_ell;
    const int boundary = (idx / max_ell) % 2;
    const int s = idx / (2 * max_ell);
    const SegmentDesc seg = segments[s];
    double2 value = make_double2(0.0, 0.0);
    if (l < seg.n_ell) {
      const int nr = instances[seg.instance].nr;
      const int r = boundary == 0 ? 0 : nr - 1;
      value = y[seg.offset + static_cast<long long>(r) * 3 * seg.n_ell +
                2 * seg.n_ell + l];
    }
    out[idx] = value;
  }
}

}  // namespace

size_t stage_smem_bytes(const StageLaunch& p) {
  const SmemLayout L(p);
  const size_t complex_count =
      static_cast<size_t>(p.slab_capacity) +
      static_cast<size_t>(p.dslab_capacity) * (p.reduction == 1 ? 2 : 1);
  const size_t double_count =
      static_cast<size_t>(kWarps) * (L.warp_x() + L.warp_t()) +
      static_cast<size_t>(L.synthesis() + L.analysis()) +
      2 * static_cast<size_t>(L.nt8) +
      static_cast<size_t>(p.coef_rows) * kCoefCount;
  return complex_count * sizeof(double2) + double_count * sizeof(double);
}

cudaError_t launch_coefficient_table(const InstanceDesc* instance_device,
                                     const double* trig, const int nr,
                                     const int row0, double* table,
                                     double* node_table, const int node_row0,
                                     const int node_record,
                                     cudaStream_t stream) {
  if (nr <= 0) return cudaSuccess;
  coefficient_table_kernel<<<(nr + 127) / 128, 128, 0, stream>>>(
      instance_device, trig, nr,
      table != nullptr ? table + static_cast<long long>(row0) * kCoefCount
                       : nullptr,
      node_table + static_cast<long long>(node_row0) * node_record,
      node_record);
  return cudaGetLastError();
}

size_t stream_smem_bytes(const int reduction, const bool wide) {
  if (wide) return WideLayout().total;
  return StreamLayout(reduction == 1 ? 1 : 0).total;
}

cudaError_t upload_sbp_constants(const SbpConstants& constants) {
  return cudaMemcpyToSymbol(c_sbp, &constants, sizeof(SbpConstants));
}

cudaError_t launch_stage(const StageLaunch& p, cudaStream_t stream) {
  if (p.tile_count <= 0) return cudaSuccess;
  const bool sc = p.reduction == 1;
  switch (p.disc) {
    case kD42:
      return sc ? launch_typed<kD42, 1>(p, stream)
                : launch_typed<kD42, 0>(p, stream);
    case kD84:
      return sc ? launch_typed<kD84, 1>(p, stream)
                : launch_typed<kD84, 0>(p, stream);
    case kD105:
      return sc ? launch_typed<kD105, 1>(p, stream)
                : launch_typed<kD105, 0>(p, stream);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_nodal_to_modal(const ConvertLaunch& p,
                                  cudaStream_t stream) {
  if (p.segment_count == 0) return cudaSuccess;
  const long long total =
      static_cast<long long>(p.segment_count) * p.nr * 3 * p.max_ell;
  const int blocks = static_cast<int>((total + 255) / 256 < 65536
                                          ? (total + 255) / 256
                                          : 65536);
  nodal_to_modal_kernel<<<blocks, 256, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_modal_to_nodal(const ConvertLaunch& p,
                                  cudaStream_t stream) {
  if (p.segment_count == 0) return cudaSuccess;
  const long long total =
      static_cast<long long>(p.segment_count) * p.nr * 3 * p.ntheta;
  const int blocks = static_cast<int>((total + 255) / 256 < 65536
                                          ? (total + 255) / 256
                                          : 65536);
  modal_to_nodal_kernel<<<blocks, 256, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_frozen_scan(const double2* nodal, const int* parent_mask,
                               const int modes, const int plane_values,
                               int* flag, cudaStream_t stream) {
  const long long total =
      static_cast<long long>(modes) * kFieldCount * plane_values;
  const long long wanted = (total + 255) / 256;
  const int blocks = static_cast<int>(wanted < 4096 ? (wanted > 0 ? wanted : 1)
                                                    : 4096);
  frozen_scan_kernel<<<blocks, 256, 0, stream>>>(nodal, parent_mask, modes,
                                                 plane_values, flag);
  return cudaGetLastError();
}

namespace {

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) {
    v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

// doubles of one warp's scratch: the Galerkin matrix and its copy, the
// right-hand side and its copy, the solution, the seed's nodal values, the
// 1/C_T factors and the nodal right-hand side
__host__ __device__ inline int gaussian_warp_doubles(const int ne, const int nt) {
  return 2 * ne * ne + 6 * ne + 5 * nt;
}

// initialize_compactified_gaussian_pulse in band space, one warp per
// (segment, r) row: the Galerkin system of
// include/teuk/pipeline_initial_data.hpp:142-207 built on the
// Gauss-Legendre nodes and solved by Gaussian elimination with partial
// pivoting (first maximal pivot, 128 eps singularity floor) and back
// substitution, then the relative residual check.
__global__ void gaussian_band_kernel(const GaussianLaunch p) {
  extern __shared__ double gsm[];
  const int warps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const InstanceDesc& in = p.instance;
  const int nr = in.nr, nt = in.ntheta;
  double* base = gsm + warp * gaussian_warp_doubles(p.max_ell, nt);
  const double* sinv = p.trig + in.trig_offset;
  const double* cosv = sinv + nt;
  const double a2 = in.spin * in.spin;
  const long long rows = static_cast<long long>(p.segment_count) * nr;
  for (long long row = static_cast<long long>(blockIdx.x) * warps + warp;
       row < rows; row += static_cast<long long>(gridDim.x) * warps) {
    const int s = static_cast<int>(row / nr);
    const int r = static_cast<int>(row - static_cast<long long>(s) * nr);
    const SegmentDesc seg = p.segments[s];
    const int ne = seg.n_ell;
    double* M = base;
    double* M0 = M + ne * ne;
    double* rhs = M0 + ne * ne;
    double* rhs0 = rhs + 2 * ne;
    double* x = rhs0 + 2 * ne;
    double* ang = x + 2 * ne;
    double* inv = ang + 2 * nt;
    double* nod = inv + nt;
    const double* St = p.matrices + seg.mat_offset;  // St[l][j]
    const double* At = St + ne * nt;                 // At[j][l]
    const double2* seed = p.seeds + static_cast<long long>(s) * p.max_ell;
    const double prof = p.profile[r], dprof = p.profile[nr + r];
    double cf[kCoefCount];
    row_coefficients(in, seg.m, r, cf);
    for (int j = lane; j < nt; j += 32) {
      double re = 0.0, im = 0.0;
      for (int l = 0; l < ne; ++l) {
        const double sv = St[l * nt + j];
        re += sv * seed[l].x;
        im += sv * seed[l].y;
      }
      ang[2 * j] = re;
      ang[2 * j + 1] = im;
      const double it = 1.0 / (cf[0] - a2 * sinv[j] * sinv[j]);
      inv[j] = it;
      const double gre = cf[3];
      const double gim = cf[4] + 2.0 * (kSpinWeight * in.spin * cosv[j]);
      const double qre = dprof * re, qim = dprof * im;
      const double pre = prof * re, pim = prof * im;
      const double k2 = -2.0 * cf[1];
      nod[2 * j] = it * (k2 * qre + (gre * pre - gim * pim));
      nod[2 * j + 1] = it * (k2 * qim + (gre * pim + gim * pre));
    }
    __syncwarp();
    for (int l = lane; l < ne; l += 32) {
      double re = 0.0, im = 0.0;
      for (int j = 0; j < nt; ++j) {
        const double a = At[j * ne + l];
        re += a * nod[2 * j];
        im += a * nod[2 * j + 1];
      }
      rhs[2 * l] = rhs0[2 * l] = re;
      rhs[2 * l + 1] = rhs0[2 * l + 1] = im;
    }
    double scale = 0.0;
    for (int idx = lane; idx < ne * ne; idx += 32) {
      const int i = idx / ne, c = idx - (idx / ne) * ne;
      double v = 0.0;
      for (int j = 0; j < nt; ++j) v += At[j * ne + i] * inv[j] * St[c * nt + j];
      M[idx] = M0[idx] = v;
      scale = fmax(scale, fabs(v));
    }
    scale = warp_max(scale);
    __syncwarp();
    const double floor = 128.0 * 2.220446049250313e-16 * scale;
    bool ok = true;
    for (int col = 0; col < ne; ++col) {
      double best = -1.0;
      int piv = ne;
      for (int i = col + lane; i < ne; i += 32) {
        const double v = fabs(M[i * ne + col]);
        if (v > best) {
          best = v;
          piv = i;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int op = __shfl_xor_sync(0xffffffffu, piv, o);
        if (ob > best || (ob == best && op < piv)) {
          best = ob;
          piv = op;
        }
      }
      if (!isfinite(best) || best <= floor) {
        if (lane == 0) atomicExch(p.singular, 1);
        ok = false;
        break;
      }
      if (piv != col) {
        for (int j = col + lane; j < ne; j += 32) {
          const double t = M[col * ne + j];
          M[col * ne + j] = M[piv * ne + j];
          M[piv * ne + j] = t;
        }
        if (lane == 0) {
          const double tr = rhs[2 * col], ti = rhs[2 * col + 1];
          rhs[2 * col] = rhs[2 * piv];
          rhs[2 * col + 1] = rhs[2 * piv + 1];
          rhs[2 * piv] = tr;
          rhs[2 * piv + 1] = ti;
        }
      }
      __syncwarp();
      const double diag = M[col * ne + col];
      for (int i = col + 1 + lane; i < ne; i += 32) {
        const double f = M[i * ne + col] / diag;
        M[i * ne + col] = 0.0;
        for (int j = col + 1; j < ne; ++j) M[i * ne + j] -= f * M[col * ne + j];
        rhs[2 * i] -= f * rhs[2 * col];
        rhs[2 * i + 1] -= f * rhs[2 * col + 1];
      }
      __syncwarp();
    }
    if (!ok) continue;  // uniform across the warp
    if (lane == 0) {
      for (int i = ne - 1; i >= 0; --i) {
        double re = rhs[2 * i], im = rhs[2 * i + 1];
        for (int c = i + 1; c < ne; ++c) {
          re -= M[i * ne + c] * x[2 * c];
          im -= M[i * ne + c] * x[2 * c + 1];
        }
        x[2 * i] = re / M[i * ne + i];
        x[2 * i + 1] = im / M[i * ne + i];
      }
    }
    __syncwarp();
    double res2 = 0.0, rhs2 = 0.0;
    for (int i = lane; i < ne; i += 32) {
      double re = -rhs0[2 * i], im = -rhs0[2 * i + 1];
      for (int c = 0; c < ne; ++c) {
        re += M0[i * ne + c] * x[2 * c];
        im += M0[i * ne + c] * x[2 * c + 1];
      }
      const double h = hypot(re, im), g = hypot(rhs0[2 * i], rhs0[2 * i + 1]);
      res2 += h * h;
      rhs2 += g * g;
    }
    res2 = warp_sum(res2);
    rhs2 = warp_sum(rhs2);
    if (lane == 0) {
      const double rel = sqrt(res2) / fmax(sqrt(rhs2), 2.2250738585072014e-308);
      atomicMax(p.worst_residual,
                static_cast<unsigned long long>(__double_as_longlong(rel)));
    }
    double2* yrow = p.y + seg.offset + static_cast<long long>(r) * 3 * ne;
    for (int l = lane; l < ne; l += 32) {
      yrow[l] = make_double2(x[2 * l], x[2 * l + 1]);
      yrow[ne + l] = make_double2(dprof * seed[l].x, dprof * seed[l].y);
      yrow[2 * ne + l] = make_double2(prof * seed[l].x, prof * seed[l].y);
    }
    __syncwarp();
  }
}

}  // namespace

size_t gaussian_smem_bytes(const int max_ell, const int ntheta,
                           int* warps_per_block) {
  const size_t per_warp =
      sizeof(double) * static_cast<size_t>(gaussian_warp_doubles(max_ell, ntheta));
  int warps = static_cast<int>((96 * 1024) / per_warp);
  warps = warps < 1 ? 1 : (warps > 8 ? 8 : warps);
  if (warps_per_block != nullptr) *warps_per_block = warps;
  return per_warp * static_cast<size_t>(warps);
}

cudaError_t launch_gaussian_band(const GaussianLaunch& p, cudaStream_t stream) {
  int warps = 1;
  const size_t bytes = gaussian_smem_bytes(p.max_ell, p.instance.ntheta, &warps);
  static KernelSetups setups;
  const cudaError_t setup_err = setups.with([&](KernelSetup& k, int) {
    if (static_cast<int>(bytes) > k.configured_bytes) {
      const cudaError_t err = cudaFuncSetAttribute(
          gaussian_band_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
          static_cast<int>(bytes));
      if (err != cudaSuccess) return err;
      k.configured_bytes = static_cast<int>(bytes);
    }
    return cudaSuccess;
  });
  if (setup_err != cudaSuccess) return setup_err;
  const long long rows = static_cast<long long>(p.segment_count) * p.instance.nr;
  if (rows == 0) return cudaSuccess;
  long long blocks = (rows + warps - 1) / warps;
  if (blocks > 65535) blocks = 65535;
  gaussian_band_kernel<<<static_cast<unsigned>(blocks), 32 * warps, bytes,
                         stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_endpoint_gather(const double2* y,
                                   const SegmentDesc* segments,
                                   const InstanceDesc* instances,
                                   const int segment_count, const int max_ell,
                                   double2* out, cudaStream_t stream) {
  if (segment_count == 0) return cudaSuccess;
  const int total = segment_count * 2 * max_ell;
  const int blocks = (total + 255) / 256;
  endpoint_gather_kernel<<<blocks, 256, 0, stream>>>(
      y, segments, instances, segment_count, max_ell, out);
  return cudaGetLastError();
}

}  // namespace teuk_b200
