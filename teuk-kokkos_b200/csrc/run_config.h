// Runtime .cfg schema of teuk_solver (include/teuk/config.hpp,
// include/teuk/run_parameters.hpp): parser, validator and resolved text,
// plus the mapping of a validated run onto a pipeline configuration
// (include/teuk/initial_data_factory.hpp, solver_driver.hpp:106-132).
#pragma once

#include <complex>
#include <string>
#include <vector>

#include "engine.h"

namespace teuk_b200 {

struct RunSeed {
  int ell = 2;
  int m = 2;
  std::complex<double> amplitude{1.0e-3, 0.0};
};

// RunParameters with the reference's defaults.
struct RunParameters {
  int config_version = 1;
  double mass = 1.0, spin = 0.0, length = 1.0;
  int nr = 65, ntheta = 7, ell_max_first = 4, ell_max_second = 4;
  std::vector<int> first_order_modes{-2, 2};
  std::vector<int> second_order_modes{-2, 2};
  double final_time = 2.0e-3;
  int steps = 20;
  double cfl = 0.1;
  double reduction_damping = 0.1, dissipation = 0.01;
  int reduction = 0;  // free_damped, stage_constrained
  int disc = kD42;
  int initial_type = 0;  // gaussian, checkpoint
  std::vector<RunSeed> seeds{RunSeed{}};
  bool add_sharp_partner = false, compact_support = false;
  double center_fraction = 0.45, width_fraction = 0.12;
  std::string time_derivative = "zero";
  std::string checkpoint_directory;
  bool second_enabled = false;
  int source_mode = 1;  // constraint_aware, unrestricted (when enabled)
  double source_start_time = 0.0, constraint_tolerance = 1.0e-8;
  int required_passes = 1;
  bool allow_truncated_daughters = false;
  // plus2 companion keys: schema only (the companion is not on this path)
  bool plus2_enabled = false;
  int plus2_mode = 0, plus2_linear_method = 0, plus2_second_method = 0,
      plus2_initial_policy = 0;
  bool plus2_linear_evolve_validation = false;
  std::string plus2_second_checkpoint;
  int plus2_ell_max_first = 4, plus2_ell_max_second = 4;
  bool plus2_regularized = true, plus2_physical = true,
       plus2_source_families = true, plus2_ordered_pairs = false;
  std::string output_directory = "teuk-output";
  int diagnostic_every = 5, checkpoint_every = 0;
};

// parse_run_configuration_text: entries, overrides, resolution, validation.
RunParameters parse_run_configuration(const std::string& text,
                                      const std::vector<std::string>& overrides);
// resolved_configuration_text (config.hpp:697-831), after validation.
std::string resolved_configuration_text(const RunParameters& run);

// Pipeline configuration of a run: registry (union of first- and
// second-order modes), bands, source policy (disabled unless
// second_order.enabled).
Config pipeline_config(const RunParameters& run);
// final_time / steps
double run_time_step(const RunParameters& run);
// Gaussian seeds after the sharp-partner expansion, sorted by (m, ell).
std::vector<RunSeed> expanded_seeds(const RunParameters& run);

}  // namespace teuk_b200
