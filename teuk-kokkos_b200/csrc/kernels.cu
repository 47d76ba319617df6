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

#include "kernels.h"

namespace teuk_b200 {

__constant__ SbpConstants c_sbp;

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kCoefCount = 9;

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

template <int DISC, int SC>
__global__ void __launch_bounds__(kThreads)
    stage_kernel(const StageLaunch p) {
  using T = DiscTraits<DISC>;
  extern __shared__ double2 smem[];
  const TileDesc tile = p.tiles[blockIdx.x];
  const SegmentDesc seg = p.segments[tile.segment];
  const InstanceDesc in = p.instances[seg.instance];
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

  double2* u = smem;                                   // slab rows x rs
  double2* psit = u + p.slab_capacity;                 // t-rows x ne
  double2* qeff = psit + p.dslab_capacity;             // t-rows x ne (SC)
  double2* wbuf = qeff + (SC ? p.dslab_capacity : 0);  // warps x (nt + ne)
  double* St = reinterpret_cast<double*>(wbuf + kWarps * (p.max_theta + p.max_ell));
  double* At = St + p.matrix_capacity;
  double* sinv = At + p.matrix_capacity;
  double* cosv = sinv + p.max_theta;
  double* coef = cosv + p.max_theta;  // t-rows x kCoefCount

  // ---- phase 0: RK stage input over the slab, matrices, coefficients
  {
    const long long base = seg.offset + static_cast<long long>(s0) * rs;
    const int count = (s1 - s0) * rs;
    const double hdt = 0.5 * in.dt;
    const double2* __restrict__ y = p.y + base;
    if (p.stage == kStage1 || p.stage == kRhsOnly) {
      for (int i = tid; i < count; i += kThreads) u[i] = __ldg(y + i);
    } else if (p.stage == kStage4) {
      const double2* __restrict__ k = p.kA + base;
      for (int i = tid; i < count; i += kThreads) u[i] = __ldg(k + i);
    } else {
      const double2* __restrict__ k = (p.stage == kStage2 ? p.kA : p.kB) + base;
      for (int i = tid; i < count; i += kThreads) {
        const double2 yv = __ldg(y + i);
        const double2 kv = __ldg(k + i);
        u[i] = make_double2(yv.x + hdt * kv.x, yv.y + hdt * kv.y);
      }
    }
    const double* S = p.matrices + seg.mat_offset;  // St[l][j]
    const double* A = S + ne * nt;                  // At[j][l]
    for (int i = tid; i < ne * nt; i += kThreads) {
      St[i] = S[i];
      At[i] = A[i];
    }
    for (int j = tid; j < nt; j += kThreads) {
      sinv[j] = p.trig[in.trig_offset + j];
      cosv[j] = p.trig[in.trig_offset + nt + j];
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
  const double a = in.spin;
  if (a == 0.0) {
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
      psit[i] = make_double2(num.x / cf[0], num.y / cf[0]);
    }
  } else {
    double2* v1 = wbuf + warp * (p.max_theta + p.max_ell);
    double2* tj = v1 + p.max_ell;
    const double a2 = a * a;
    const double sa2 = 2.0 * (static_cast<double>(kSpinWeight) * a);
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
          const double s = St[l * nt + j];
          sa = cfma(s, v1[l], sa);
          sb = cfma(s, row[2 * ne + l], sb);
        }
        // t_j = (a_j - i gamma_j b_j) / C_T_j, gamma_j = 2 s a cos(theta_j)
        const double gamma = sa2 * cosv[j];
        const double ct = cf[0] - a2 * sinv[j] * sinv[j];
        tj[j] = make_double2((sa.x + gamma * sb.y) / ct,
                             (sa.y - gamma * sb.x) / ct);
      }
      __syncwarp();
      for (int l = lane; l < ne; l += 32) {
        double2 acc = make_double2(0.0, 0.0);
        for (int j = 0; j < nt; ++j) acc = cfma(At[j * ne + l], tj[j], acc);
        psit[rr * ne + l] = acc;
      }
      __syncwarp();
    }
  }
  __syncthreads();

  // ---- phase 2: RHS assembly and RK update on rows [r0, r1)
  const double inv_h = in.inv_spacing;
  const double diss_scale = in.dissipation * inv_h;
  const double damping = in.damping;
  const double dt = in.dt;
  const double dt6 = in.dt / 6.0;
  const int items = (r1 - r0) * ne;
  for (int i = tid; i < items; i += kThreads) {
    const int rr = i / ne;
    const int l = i - rr * ne;
    const int r = r0 + rr;
    const double* cf = coef + (r - t0) * kCoefCount;
    const double2* urow = u + (r - s0) * rs;
    const double2 Qs = urow[ne + l];
    const double2 psi = urow[2 * ne + l];
    const double2 Qe = qcol[(r - qbase) * qstride + l];
    const double2 dpsi =
        cscale(inv_h, sbp_derivative<DISC>(u + 2 * ne + l, rs, s0, r, nr));
    const double2 dq = cscale(inv_h, sbp_derivative<DISC>(qcol + l, qstride,
                                                          qbase, r, nr));
    const double2 dpsit =
        cscale(inv_h, sbp_derivative<DISC>(psit + l, ne, t0, r, nr));
    const int ell = seg.ell_min + l;
    const double lambda = -static_cast<double>((ell - kSpinWeight) *
                                               (ell + kSpinWeight + 1));
    double2 kP = cscale(cf[2], dq);
    kP = cadd(kP, cmul(make_double2(cf[5], cf[6]), Qe));
    kP = cadd(kP, cmul(make_double2(cf[7], cf[8]), psi));
    kP = cadd(kP, cscale(lambda, psi));
    double2 kQ = csub(dpsit, cscale(damping, csub(Qs, dpsi)));
    double2 kpsi = psit[(r - t0) * ne + l];
    if (in.dissipation > 0.0) {
      kP = cfma(diss_scale, sbp_dissipation<DISC>(u + l, rs, s0, r, nr), kP);
      kQ = cfma(diss_scale, sbp_dissipation<DISC>(u + ne + l, rs, s0, r, nr),
                kQ);
      kpsi = cfma(diss_scale,
                  sbp_dissipation<DISC>(u + 2 * ne + l, rs, s0, r, nr), kpsi);
    }
    const long long g = seg.offset + static_cast<long long>(r) * rs + l;
    const double2 k[3] = {kP, kQ, kpsi};
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const long long gi = g + f * ne;
      switch (p.stage) {
        case kStage1:
        case kRhsOnly:
          p.kA[gi] = k[f];
          break;
        case kStage2: {
          const double2 k1 = p.kA[gi];
          p.kB[gi] = k[f];
          p.acc[gi] = cfma(2.0, k[f], k1);
          break;
        }
        case kStage3: {
          const double2 yv = p.y[gi];
          const double2 acc = cfma(2.0, k[f], p.acc[gi]);
          p.acc[gi] = cfma(dt6, acc, yv);
          p.kA[gi] = cfma(dt, k[f], yv);
          break;
        }
        case kStage4:
          p.y[gi] = cfma(dt6, k[f], p.acc[gi]);
          break;
      }
    }
  }
}

template <int DISC, int SC>
cudaError_t launch_typed(const StageLaunch& p, cudaStream_t stream) {
  const size_t bytes = stage_smem_bytes(p);
  auto kernel = stage_kernel<DISC, SC>;
  // The opt-in limit is raised once per instantiation to the largest size
  // requested so far (never inside a launch sequence that needs less).
  static int configured_bytes = 0;
  if (static_cast<int>(bytes) > configured_bytes) {
    cudaError_t err = cudaFuncSetAttribute(
        kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
        static_cast<int>(bytes));
    if (err != cudaSuccess) return err;
    configured_bytes = static_cast<int>(bytes);
  }
  kernel<<<p.tile_count, kThreads, bytes, stream>>>(p);
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
  const size_t complex_count =
      static_cast<size_t>(p.slab_capacity) +
      static_cast<size_t>(p.dslab_capacity) * (p.reduction == 1 ? 2 : 1) +
      static_cast<size_t>(kWarps) * (p.max_theta + p.max_ell);
  const size_t double_count = 2 * static_cast<size_t>(p.matrix_capacity) +
                              2 * static_cast<size_t>(p.max_theta) +
                              static_cast<size_t>(p.coef_rows) * kCoefCount;
  return complex_count * sizeof(double2) + double_count * sizeof(double);
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
