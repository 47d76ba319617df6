// teuk_b200.hpp -- C++ facade of the B200 engine shaped like the
// reference's teuk::SpatialPipeline (include/teuk/spatial_pipeline.hpp:
// 144-1364), for host code that called the reference class directly
// (teuk_solver's run_solver, include/teuk/solver_driver.hpp:127-317).
//
// It is header-only over the C ABI in teuk_b200.h: status codes come back as
// the exception types the reference throws (std::invalid_argument for
// shape/policy/time errors, std::runtime_error otherwise).  Kokkos::View
// arguments become host or device pointers to complex128 arrays in the same
// (mode, field, radial, theta) order.
#pragma once

#include <complex>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "teuk_b200.h"

namespace teuk_b200 {

using Complex = std::complex<double>;

enum class RadialDiscretization { D42 = TEUK_B200_D42, D84 = TEUK_B200_D84,
                                  D105 = TEUK_B200_D105 };
enum class ReductionEvolution { FreeDamped = TEUK_B200_FREE_DAMPED,
                                StageConstrained = TEUK_B200_STAGE_CONSTRAINED };
enum class SecondOrderSourceMode {
  Disabled = TEUK_B200_SOURCE_DISABLED,
  ConstraintAware = TEUK_B200_SOURCE_CONSTRAINT_AWARE,
  Unrestricted = TEUK_B200_SOURCE_UNRESTRICTED
};

// include/teuk/spatial_pipeline.hpp:55-67
struct SecondOrderSourcePolicy {
  SecondOrderSourceMode mode = SecondOrderSourceMode::ConstraintAware;
  double source_start_time = 0.0;
  double normalized_constraint_tolerance = 1.0e-10;
  int required_consecutive_passes = 1;
  static SecondOrderSourcePolicy disabled() {
    return {SecondOrderSourceMode::Disabled, 0.0, 0.0, 1};
  }
  static SecondOrderSourcePolicy unrestricted() {
    return {SecondOrderSourceMode::Unrestricted, 0.0, 0.0, 1};
  }
};

// ModeRegistry lists (include/teuk/modes.hpp:42-80)
struct ModeLists {
  std::vector<int> modes, parents, targets;
  explicit ModeLists(std::vector<int> stored)
      : modes(stored), parents(stored), targets(std::move(stored)) {}
  ModeLists(std::vector<int> stored, std::vector<int> p, std::vector<int> t)
      : modes(std::move(stored)), parents(std::move(p)), targets(std::move(t)) {}
};

struct KerrParameters {
  double mass = 1.0;
  double spin = 0.0;
  double compactification_length = 1.0;
};

struct PipelineAngularBands {
  int ell_max_first = 0;
  int ell_max_second = 0;
};

struct SourceActivationState {
  bool active = false;
  double activation_time = -1.0;
  int consecutive_passes = 0;
  double last_eligibility_time = -1.0;
};

inline void throw_status(const int status) {
  if (status == TEUK_B200_OK) return;
  const std::string message = teuk_b200_last_error();
  if (status == TEUK_B200_ERR_INVALID_ARGUMENT) {
    throw std::invalid_argument(message);
  }
  throw std::runtime_error(message);
}

class SpatialPipeline {
 public:
  SpatialPipeline(const ModeLists& registry, const int radial_points,
                  const PipelineAngularBands bands, const int theta_nodes,
                  const KerrParameters& background,
                  const double reduction_damping = 0.1,
                  const double dissipation = 0.0,
                  const ReductionEvolution reduction =
                      ReductionEvolution::FreeDamped,
                  const SecondOrderSourcePolicy policy = {},
                  const RadialDiscretization discretization =
                      RadialDiscretization::D42)
      : registry_(registry) {
    teuk_b200_config c{};
    c.abi_version = TEUK_B200_ABI_VERSION;
    c.mass = background.mass;
    c.spin = background.spin;
    c.compactification_length = background.compactification_length;
    c.radial_points = radial_points;
    c.theta_nodes = theta_nodes;
    c.ell_max_first = bands.ell_max_first;
    c.ell_max_second = bands.ell_max_second;
    c.mode_count = static_cast<int>(registry_.modes.size());
    c.modes = registry_.modes.data();
    c.parent_count = static_cast<int>(registry_.parents.size());
    c.parents = registry_.parents.data();
    c.target_count = static_cast<int>(registry_.targets.size());
    c.targets = registry_.targets.data();
    c.reduction_damping = reduction_damping;
    c.dissipation = dissipation;
    c.reduction = static_cast<int>(reduction);
    c.discretization = static_cast<int>(discretization);
    c.source_mode = static_cast<int>(policy.mode);
    c.source_start_time = policy.source_start_time;
    c.normalized_constraint_tolerance = policy.normalized_constraint_tolerance;
    c.required_consecutive_passes = policy.required_consecutive_passes;
    throw_status(teuk_b200_create(&c, &handle_));
    size_t s[4];
    throw_status(teuk_b200_shape(handle_, s));
    shape_ = {s[0], s[1], s[2], s[3]};
  }

  SpatialPipeline(const SpatialPipeline&) = delete;
  SpatialPipeline& operator=(const SpatialPipeline&) = delete;
  SpatialPipeline(SpatialPipeline&& other) noexcept
      : registry_(std::move(other.registry_)),
        handle_(std::exchange(other.handle_, nullptr)),
        shape_(other.shape_) {}
  ~SpatialPipeline() {
    if (handle_ != nullptr) teuk_b200_destroy(handle_);
  }

  // extents (mode, field, radial, theta) of storage().state()
  [[nodiscard]] std::vector<size_t> extents() const { return shape_; }
  [[nodiscard]] size_t value_count() const {
    return shape_[0] * shape_[1] * shape_[2] * shape_[3];
  }

  // Host copies of storage().state() in and out.
  void set_state(const std::vector<Complex>& state) {
    require_size(state.size());
    throw_status(teuk_b200_set_state(
        handle_, reinterpret_cast<const double*>(state.data()), state.size(),
        TEUK_B200_HOST));
  }
  [[nodiscard]] std::vector<Complex> state() const {
    std::vector<Complex> out(value_count());
    throw_status(teuk_b200_get_state(handle_, reinterpret_cast<double*>(out.data()),
                                     out.size(), TEUK_B200_HOST));
    return out;
  }
  // Device-pointer variants (complex128 arrays of value_count()).
  void set_state_device(const void* state) {
    throw_status(teuk_b200_set_state(handle_, static_cast<const double*>(state),
                                     value_count(), TEUK_B200_DEVICE));
  }
  void get_state_device(void* state) const {
    throw_status(teuk_b200_get_state(handle_, static_cast<double*>(state),
                                     value_count(), TEUK_B200_DEVICE));
  }

  // SpatialPipeline::evaluate_rhs_at_time on host arrays
  void evaluate_rhs_at_time(const std::vector<Complex>& stage,
                            std::vector<Complex>& output,
                            const double stage_time) {
    require_size(stage.size());
    output.resize(stage.size());
    throw_status(teuk_b200_evaluate_rhs(
        handle_, reinterpret_cast<const double*>(stage.data()),
        reinterpret_cast<double*>(output.data()), stage.size(), stage_time,
        TEUK_B200_HOST));
  }

  // SpatialPipeline::step
  void step(const double time, const double time_step) {
    throw_status(teuk_b200_step(handle_, time, time_step, 1));
  }
  void advance(const double time, const double time_step, const int steps) {
    throw_status(teuk_b200_step(handle_, time, time_step, steps));
  }

  void initialize_gaussian(const double center, const double width,
                           const std::vector<teuk_b200_gaussian_mode>& modes,
                           const bool compact_support = false) {
    teuk_b200_gaussian g{center, width, compact_support ? 1 : 0,
                         static_cast<int>(modes.size()), modes.data()};
    throw_status(teuk_b200_initialize_gaussian(handle_, &g));
  }

  [[nodiscard]] std::vector<teuk_b200_waveform_record> sample_endpoint() {
    std::vector<teuk_b200_waveform_record> records(
        4 * shape_[0] * 64);
    size_t count = 0;
    throw_status(teuk_b200_sample_endpoint(handle_, records.data(),
                                           records.size(), &count));
    records.resize(count);
    return records;
  }

  [[nodiscard]] SourceActivationState source_activation_state() const {
    teuk_b200_activation a{};
    throw_status(teuk_b200_get_activation(handle_, &a));
    return {a.active != 0, a.activation_time, a.consecutive_passes,
            a.last_eligibility_time};
  }
  void restore_source_activation(const SourceActivationState& s) {
    const teuk_b200_activation a{s.active ? 1 : 0, s.activation_time,
                                 s.consecutive_passes, s.last_eligibility_time};
    throw_status(teuk_b200_restore_activation(handle_, &a));
  }
  void reset_source_activation() {
    throw_status(teuk_b200_reset_activation(handle_));
  }
  void fence() { throw_status(teuk_b200_synchronize(handle_)); }

  [[nodiscard]] teuk_b200_pipeline* native_handle() const { return handle_; }

 private:
  void require_size(const size_t n) const {
    if (n != value_count()) {
      throw std::invalid_argument("full pipeline stage extents do not match");
    }
  }

  ModeLists registry_;
  teuk_b200_pipeline* handle_ = nullptr;
  std::vector<size_t> shape_;
};

}  // namespace teuk_b200
