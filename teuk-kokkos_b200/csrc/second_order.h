// Second-order (quadratic-source) pipeline on the GPU: the stage graph of
// SpatialPipeline::evaluate_rhs_at_time for the ConstraintAware and
// Unrestricted source policies (include/teuk/spatial_pipeline.hpp:517-587),
// its RK4 step with the source-activation latch (:590-620, :1225-1310).
//
// Storage follows the reference: every field lives nodally on the
// Gauss-Legendre grid in (mode, slot, radial, theta) order, because the
// quadratic source multiplies fields of different m pointwise.  Each angular
// operator of a SignedModeAngularCoordinator (project, Laplacian, eth,
// eth') is one fused launch over all modes and radial rows.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <stdexcept>
#include <vector>

#include "engine.h"

namespace teuk_b200 {

// One SignedModeAngularCoordinator: (spin, boost, ell_max, active modes).
struct AngularCoordinator {
  int spin = 0;
  int boost = 0;
  int ell_max = 0;
  std::vector<int> active;  // per registry mode: 1 if it has resources
  // per registry mode, offsets into the matrix pool (0 when inactive)
  std::vector<int> analysis;        // A_s   [ne_s][nt]
  std::vector<int> synthesis;       // S_s   [nt][ne_s]
  std::vector<int> raised;          // S_s+1 [nt][ne_s+1]
  std::vector<int> lowered;         // S_s-1 [nt][ne_s-1]
  std::vector<int> n_ell, ell_min;  // source band
  std::vector<int> n_ell_up, ell_min_up, n_ell_down, ell_min_down;
};

struct SourceActivation {
  bool active = false;
  double activation_time = -1.0;
  int consecutive_passes = 0;
  double last_eligibility_time = -1.0;
};

struct ConstraintNorms {
  double absolute_maximum[3] = {0, 0, 0};
  double normalized_maximum[3] = {0, 0, 0};
  double weighted_rms[3] = {0, 0, 0};
  double normalized_weighted[3] = {0, 0, 0};
  double controlling_normalized = 0.0;
  bool all_finite = true;
};

// Uploads the SBP tables used by the nodal kernels to the current device.
cudaError_t upload_nodal_sbp_constants();

// A CUDA runtime failure inside the nodal pipeline.
struct DeviceError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// Device bytes a NodalPipeline allocates for `plan`.
std::size_t nodal_footprint_bytes(const InstancePlan& plan);

// Reductions of PipelineDiagnostics::sample
// (include/teuk/pipeline_diagnostics.hpp:143-291) over nodal
// (mode, 13, r, theta) arrays; a null rhs / source / forcing reads as zero.
struct DiagnosticsLaunch {
  const double2* state;
  const double2* rhs;
  const double2* source;   // (mode, r, theta)
  const double2* forcing;  // (mode, r, theta)
  int modes, nr, nt, disc;
  double inv_spacing;
  double* sums;                // 30: 13 state, 13 rhs, 4 scalars
  unsigned long long* maxima;  // 30, as bits of nonnegative doubles
  int* finite;                 // 8 flags, 1 = finite
};
cudaError_t launch_diagnostics(const DiagnosticsLaunch& launch,
                               cudaStream_t stream);

class NodalPipeline {
 public:
  struct Buffers;
  // precision 0: FP64 transforms; 1: split-precision (BF16 digits, FP32
  // accumulation, FP64 recombination) tensor-core transforms.
  // replicas > 1: room for that many independent solves of the same plan,
  // replica k in modes [k n, (k + 1) n) of every array (n = the plan's
  // modes), all stepped by the same launches; each replica's results equal
  // the solve alone bit for bit (every kernel works per mode and grid point,
  // and the pair tables stay inside a replica).  Replicas share one latch,
  // so they need the Unrestricted source from t = 0.
  explicit NodalPipeline(const InstancePlan& plan, int precision = 0,
                         int replicas = 1);
  int precision() const { return precision_; }
  int replicas() const { return replicas_; }
  int active_replicas() const { return active_; }
  // Steps advance replicas [0, k) only (1 <= k <= replicas()).
  void set_active_replicas(int k);
  // State of replica k (the plan's value_count() complex values).
  void set_replica_state(int k, const double* state, int memory);
  void get_replica_state(int k, double* state, int memory);
  // Device copy of replica src_k of `src` (same plan) into replica dst_k.
  void copy_replica_from(const NodalPipeline& src, int src_k, int dst_k);
  ~NodalPipeline();
  NodalPipeline(const NodalPipeline&) = delete;
  NodalPipeline& operator=(const NodalPipeline&) = delete;

  const InstancePlan& plan() const { return plan_; }
  // complex values of the active replicas' states
  size_t value_count() const {
    return plan_.value_count() * static_cast<size_t>(active_);
  }
  void set_stream(cudaStream_t stream);
  cudaStream_t stream() const { return stream_; }

  void set_state(const double* state, int memory);
  void get_state(double* state, int memory);
  void evaluate_rhs(const double* stage, double* out, int memory,
                    double time);
  void step(double time, double dt);
  void reset_activation();
  void restore_activation(const SourceActivation& s);
  SourceActivation activation() const { return activation_; }
  const ConstraintNorms& constraint_norms() const { return norms_; }
  // Endpoint psi of the first-order (field 2) or second-order (field 12)
  // state of one replica: (mode, theta) nodal values at radial index
  // `radial`.
  void endpoint_slice(int field, int radial, std::vector<double2>& out,
                      int replica = 0);
  // Storage views of the reference pipeline: state, storage rhs (written by
  // the latch check), source_over_r3, forcing.
  const double2* state_device() const;
  const double2* storage_rhs_device() const;
  const double2* source_device() const;
  const double2* forcing_device() const;
  double independent_constraint_maximum() const { return independent_max_; }

 private:
  void build_coordinators();
  void build_tile_operators();
  void evaluate(const double2* stage, double2* out);
  void consider_activation(double accepted_time);
  void advance_fixed(double time, double dt);
  struct StepGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double dt = 0.0;
    cudaStream_t stream = nullptr;
  };
  void record_step(double dt);
  static void release_graph(StepGraph& g);
  ConstraintNorms sample_constraints();
  void sync_check(const char* what);

  InstancePlan plan_;
  int precision_ = 0;
  int replicas_ = 1;
  int active_ = 1;
  int pairs_per_replica_ = 0;
  int targets_per_replica_ = 0;
  // composite tile operators: used when ntheta <= 64
  bool tile_operators_ = false;
  int tile_fp64_words_ = 0;   // 8-byte words of one FP64 operator
  int tile_split_words_ = 0;  // 8-byte words of one split operator
  std::vector<double> tile_fp64_;
  std::vector<uint2> tile_split_;
  std::vector<double> tile_scales_;
  std::vector<int> tile_offsets_[10][4];  // [coordinator][operation]: 3 per mode
  std::vector<int> pair_index1_, pair_index2_, pair_offsets_, targets_;
  std::vector<AngularCoordinator> coordinators_;
  // per coordinator: pool offsets of the Laplacian / raising / lowering
  // diagonals of each registry mode
  std::vector<int> coordinator_diag_[10][3];
  std::vector<double> matrices_;
  SourceActivation activation_;
  double independent_max_ = 0.0;  // sqrt(source_constraint_max_squared)
  ConstraintNorms norms_;
  StepGraph graphs_[2];  // latch off / on
  cudaStream_t own_stream_ = nullptr;
  cudaStream_t stream_ = nullptr;
  std::unique_ptr<Buffers> buf_;
};

}  // namespace teuk_b200
