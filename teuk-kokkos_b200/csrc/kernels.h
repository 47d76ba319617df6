// Launch interface of the CUDA kernels (kernels.cu) used by the C ABI.
#pragma once

#include <cuda_runtime.h>

#include "engine.h"

namespace teuk_b200 {

// RK stage selector of stage_kernel.  kRhsOnly evaluates k = f(y) into kA
// without touching y / kB / acc (evaluate_rhs).
enum StageKind : int {
  kStage1 = 1,
  kStage2 = 2,
  kStage3 = 3,
  kStage4 = 4,
  kRhsOnly = 5
};

struct StageLaunch {
  double2* y;
  double2* kA;
  double2* kB;
  double2* acc;
  const InstanceDesc* instances;
  const SegmentDesc* segments;
  const TileDesc* tiles;  // tiles of this launch group
  const double* matrices;
  const double* trig;
  int tile_count;
  int disc;
  int reduction;  // 0 free damped, 1 stage constrained
  int stage;
  // shared-memory carve-up capacities (elements), host-computed per group
  int slab_capacity;   // double2
  int dslab_capacity;  // double2
  int matrix_capacity; // doubles per matrix
  int coef_rows;       // rows of coefficient records
  int max_theta;
  int max_ell;
  // CTAs resident at once (SMs x CTAs per SM), set by launch_stage: the
  // tile blockIdx + prefetch_stride starts when this CTA's slot frees up
  int prefetch_stride;
  // Radial strips for the streaming kernel (null: tile kernel only).  A
  // strip is a TileDesc whose rows are at least kStripMinRows long.
  const TileDesc* strips;
  int strip_count;
  // device word set to a non-zero code when a streaming-kernel wait timed
  // out (read by the host after the step)
  int* error;
  // Teukolsky row coefficients of every solve, kCoefRecord doubles per
  // radial row (coefficient_table_kernel); the m-dependent imaginary parts
  // (entries 4, 6, 8) are stored for m = 1 and scaled by m where used.
  const double* coef_table;
  // 1 / C_T(r, theta_j) of every solve on its Gauss-Legendre nodes,
  // kNodeRecord doubles per radial row (zero beyond the solve's nodes)
  const double* node_table;
  // Transform precision of Kerr bands on the streaming kernel: 0 FP64,
  // 1 split precision (BF16 digit slices, split_precision.cuh) with the
  // per-segment digit records below (kSplitRecordUint4 uint4 and
  // kSplitScaleDoubles doubles per segment, indexed by segment).  Tile-kernel
  // bands always run FP64.
  int precision;
  const uint4* split_frags;
  const double* split_scales;
  // 1: the strips run the wide streaming kernel (WideGeom), whose node
  // table rows have kWideMaxNodes doubles
  int wide;
  // Failure-detection test hook (-1: off): in stage-1 launches the producer
  // of CTA 0 never issues this chunk, so the waits for it run out and the
  // launch reports a timeout through `error`.
  int withhold_chunk;
};

// Streaming kernel eligibility of a band (segment): n_ell <= 16, and at
// most 32 Gauss-Legendre nodes per row in its solve.
inline constexpr int kStreamMaxEll = 16;
inline constexpr int kStreamMaxNodes = 32;
// Wide streaming kernel eligibility: n_ell <= 24, at most 48 nodes, the
// free-damped reduction and FP64 transforms.  Its node table has
// kWideMaxNodes doubles per radial row.
inline constexpr int kWideMaxEll = 24;
inline constexpr int kWideMaxNodes = 48;

inline constexpr int kSplitRecordUint4 = 4 * 5 * 32;
inline constexpr int kSplitScaleDoubles = kStreamMaxNodes + kStreamMaxEll;
inline constexpr int kCoefRecord = 10;
inline constexpr int kNodeRecord = kStreamMaxNodes;
// Fills the coefficient table rows of one solve, table[(row0 + r) * 10 + k]
// (none when table is null), and its node-inverse rows,
// node_table[(node_row0 + r) * node_record + j] (node_record: kNodeRecord,
// or kWideMaxNodes for the wide table);
// `trig` is the device trig pool the instance's trig_offset points into.
cudaError_t launch_coefficient_table(const InstanceDesc* instance_device,
                                     const double* trig, int nr, int row0,
                                     double* table, double* node_table,
                                     int node_row0, int node_record,
                                     cudaStream_t stream);
inline constexpr int kStripMinRows = 64;
// Radial strips per CTA the host aims for when it splits segments.
inline constexpr int kStripsPerCta = 8;
// Dynamic shared memory of the streaming kernel (wide: its wide form).
size_t stream_smem_bytes(int reduction, bool wide = false);

// Dynamic shared memory bytes for one launch description.
size_t stage_smem_bytes(const StageLaunch& launch);
cudaError_t upload_sbp_constants(const SbpConstants& constants);
cudaError_t launch_stage(const StageLaunch& launch, cudaStream_t stream);

// Nodal (m,13,r,theta) complex array of one instance <-> modal segments.
struct ConvertLaunch {
  const double2* nodal_in;  // nodal -> modal source
  double2* nodal_out;       // modal -> nodal destination
  double2* modal;           // state buffer base
  const SegmentDesc* segments;
  const int* segment_modes;  // registry index of each listed segment
  const double* matrices;
  int segment_count;
  int nr;
  int ntheta;
  int mode_count;  // registry modes of the instance
  int max_ell;
};
cudaError_t launch_nodal_to_modal(const ConvertLaunch& launch,
                                  cudaStream_t stream);
cudaError_t launch_modal_to_nodal(const ConvertLaunch& launch,
                                  cudaStream_t stream);

// Sets *flag to 1 when any value of a frozen (mode, field) plane of the
// nodal state is non-zero.  parent_mask[mode] is 1 for parent modes, whose
// first three fields are evolved (not frozen).
cudaError_t launch_frozen_scan(const double2* nodal, const int* parent_mask,
                               int modes, int plane_values, int* flag,
                               cudaStream_t stream);

// Gather psi modal coefficients at r = 0 and r = nr-1 of every segment into
// out[(2 * segment + boundary) * max_ell + ell].
cudaError_t launch_endpoint_gather(const double2* y,
                                   const SegmentDesc* segments,
                                   const InstanceDesc* instances,
                                   int segment_count, int max_ell,
                                   double2* out, cudaStream_t stream);

// Gaussian initial data of one solve written straight into band storage
// (include/teuk/pipeline_initial_data.hpp:142-339 in band space): psi =
// profile(R) seed, Q = (D profile)(R) seed, and P from the per-row Galerkin
// system A diag(1/C_T) S p = A [C_T^{-1} (-2K Q + G psi)], solved by one warp
// per (segment, radial row) with partial pivoting.
struct GaussianLaunch {
  double2* y;
  const SegmentDesc* segments;  // the solve's segments (parents)
  int segment_count;
  InstanceDesc instance;
  const double* matrices;
  const double* trig;      // sin(theta) then cos(theta) at instance.trig_offset
  const double2* seeds;    // segment-major, max_ell complex seeds each
  const double* profile;   // profile(R_r) [nr], then (D profile)(R_r) [nr]
  int max_ell;
  unsigned long long* worst_residual;  // bits of the largest relative residual
  int* singular;                       // set when a pivot falls below the floor
};
size_t gaussian_smem_bytes(int max_ell, int ntheta, int* warps_per_block);
cudaError_t launch_gaussian_band(const GaussianLaunch& launch,
                                 cudaStream_t stream);

}  // namespace teuk_b200
