// Reference-side C ABI: test infrastructure, never linked into the product.
//
// Wraps the unmodified teuk-kokkos headers (compiled against the Kokkos-API
// host shim in oracle/kokkos_shim) behind the same entry points that
// include/teuk_b200.h declares for the B200 engine, with a teuk_ref_ prefix.
// Tests and the CPU baseline of bench.py call both libraries with identical
// arguments. Built by oracle/Makefile into oracle/_ref/libteuk_ref*.so; it
// needs the reference include tree only at build time.
#include <Kokkos_Core.hpp>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "teuk/config.hpp"
#include "teuk/diagnostics.hpp"
#include "teuk/initial_data_factory.hpp"
#include "teuk/pipeline_bands.hpp"
#include "teuk/pipeline_diagnostics.hpp"
#include "teuk/pipeline_checkpoint.hpp"
#include "teuk/pipeline_initial_data.hpp"
#include "teuk/spatial_pipeline.hpp"
#include "teuk/waveform_output.hpp"
#include "teuk_b200.h"

namespace {

thread_local std::string last_error;

int fail(const int code, const std::string& message) {
  last_error = message;
  return code;
}

template <class Body>
int guarded(Body&& body) {
  try {
    body();
    return TEUK_B200_OK;
  } catch (const std::invalid_argument& error) {
    return fail(TEUK_B200_ERR_INVALID_ARGUMENT, error.what());
  } catch (const std::out_of_range& error) {
    return fail(TEUK_B200_ERR_INVALID_ARGUMENT, error.what());
  } catch (const std::exception& error) {
    return fail(TEUK_B200_ERR_RUNTIME, error.what());
  }
}

std::vector<int> list(const int* values, const int count) {
  if (count < 0 || (count > 0 && values == nullptr)) {
    throw std::invalid_argument("mode list pointer/count mismatch");
  }
  return std::vector<int>(values, values + count);
}

teuk::RadialDiscretization discretization(const int value) {
  switch (value) {
    case TEUK_B200_D42: return teuk::RadialDiscretization::D42;
    case TEUK_B200_D84: return teuk::RadialDiscretization::D84;
    case TEUK_B200_D105: return teuk::RadialDiscretization::D105;
  }
  throw std::invalid_argument("unknown radial discretization");
}

teuk::SecondOrderSourcePolicy policy(const teuk_b200_config& c) {
  switch (c.source_mode) {
    case TEUK_B200_SOURCE_DISABLED:
      return teuk::SecondOrderSourcePolicy::disabled();
    case TEUK_B200_SOURCE_CONSTRAINT_AWARE:
      return {teuk::SecondOrderSourceMode::ConstraintAware,
              c.source_start_time, c.normalized_constraint_tolerance,
              c.required_consecutive_passes};
    case TEUK_B200_SOURCE_UNRESTRICTED:
      return {teuk::SecondOrderSourceMode::Unrestricted, c.source_start_time,
              c.normalized_constraint_tolerance,
              c.required_consecutive_passes};
  }
  throw std::invalid_argument("unknown source mode");
}

}  // namespace

struct teuk_ref_pipeline {
  explicit teuk_ref_pipeline(const teuk_b200_config& c)
      : registry(list(c.modes, c.mode_count), list(c.parents, c.parent_count),
                 list(c.targets, c.target_count)),
        horizon(c.compactification_length * c.compactification_length /
                teuk::outer_horizon_radius(c.mass, c.spin)),
        pipeline(execution, registry,
                 teuk::UniformRadialGrid(
                     static_cast<std::size_t>(c.radial_points), 0.0, horizon),
                 teuk::PipelineAngularBands{c.ell_max_first, c.ell_max_second},
                 c.theta_nodes,
                 teuk::KerrParameters{c.mass, c.spin,
                                      c.compactification_length},
                 c.reduction_damping, c.dissipation,
                 c.reduction == TEUK_B200_STAGE_CONSTRAINED
                     ? teuk::ReductionEvolution::StageConstrained
                     : teuk::ReductionEvolution::FreeDamped,
                 "ref_pipeline", policy(c), discretization(c.discretization)),
        sampler(registry, {c.ell_max_first, c.ell_max_second}, c.theta_nodes,
                c.compactification_length, horizon),
        ell_max_first(c.ell_max_first),
        config(c),
        background{c.mass, c.spin, c.compactification_length},
        scratch("ref_scratch_state", registry.size(),
                teuk::point_pipeline_field_count,
                static_cast<std::size_t>(c.radial_points),
                static_cast<std::size_t>(c.theta_nodes)),
        scratch_out("ref_scratch_rhs", registry.size(),
                    teuk::point_pipeline_field_count,
                    static_cast<std::size_t>(c.radial_points),
                    static_cast<std::size_t>(c.theta_nodes)) {}

  teuk::ExecutionSpace execution;
  teuk::ModeRegistry registry;
  double horizon;
  teuk::SpatialPipeline pipeline;
  teuk::EndpointWaveformSampler sampler;
  int ell_max_first;
  teuk_b200_config config;  // scalar fields only (mode pointers not kept)
  teuk::KerrParameters background;
  teuk::FieldView scratch;
  teuk::FieldView scratch_out;
};

namespace {

std::size_t value_count(const teuk_ref_pipeline& p) {
  return p.pipeline.storage().value_count();
}

void check_count(const teuk_ref_pipeline& p, const std::size_t count) {
  if (count != value_count(p)) {
    throw std::invalid_argument("state complex count does not match shape");
  }
}

void copy_in(const teuk::FieldView& view, const double* values) {
  auto* data = view.data();
  for (std::size_t i = 0; i < view.size(); ++i) {
    data[i] = teuk::Complex(values[2 * i], values[2 * i + 1]);
  }
}

void copy_out(const teuk::FieldView& view, double* values) {
  const auto* data = view.data();
  for (std::size_t i = 0; i < view.size(); ++i) {
    values[2 * i] = data[i].real();
    values[2 * i + 1] = data[i].imag();
  }
}

}  // namespace

extern "C" {

const char* teuk_ref_last_error(void) { return last_error.c_str(); }

const char* teuk_ref_backend(void) {
  return teuk::ExecutionSpace::name();
}

int teuk_ref_create(const teuk_b200_config* config, teuk_ref_pipeline** out) {
  if (config == nullptr || out == nullptr) {
    return fail(TEUK_B200_ERR_INVALID_ARGUMENT, "null argument");
  }
  return guarded([&] { *out = new teuk_ref_pipeline(*config); });
}

int teuk_ref_destroy(teuk_ref_pipeline* p) {
  delete p;
  return TEUK_B200_OK;
}

int teuk_ref_shape(const teuk_ref_pipeline* p, size_t shape[4]) {
  const auto s = p->pipeline.storage().snapshot_shape();
  shape[0] = s.modes;
  shape[1] = s.fields;
  shape[2] = s.radial;
  shape[3] = s.theta;
  return TEUK_B200_OK;
}

int teuk_ref_set_state(teuk_ref_pipeline* p, const double* state,
                       size_t count, int) {
  return guarded([&] {
    check_count(*p, count);
    copy_in(p->pipeline.storage().state(), state);
  });
}

int teuk_ref_get_state(teuk_ref_pipeline* p, double* state, size_t count,
                       int) {
  return guarded([&] {
    check_count(*p, count);
    copy_out(p->pipeline.storage().state(), state);
  });
}

int teuk_ref_evaluate_rhs(teuk_ref_pipeline* p, const double* stage,
                          double* output, size_t count, double time, int) {
  return guarded([&] {
    check_count(*p, count);
    copy_in(p->scratch, stage);
    p->pipeline.evaluate_rhs_at_time(p->execution, p->scratch,
                                     p->scratch_out, time);
    copy_out(p->scratch_out, output);
  });
}

int teuk_ref_step(teuk_ref_pipeline* p, double time, double dt, int steps) {
  return guarded([&] {
    for (int i = 0; i < steps; ++i) {
      p->pipeline.step(p->execution, time, dt);
      time += dt;
    }
  });
}

int teuk_ref_initialize_gaussian(teuk_ref_pipeline* p,
                                 const teuk_b200_gaussian* pulse) {
  return guarded([&] {
    teuk::PipelineGaussianPulse gaussian;
    gaussian.center = pulse->center;
    gaussian.width = pulse->width;
    gaussian.compact_support = pulse->compact_support != 0;
    for (int i = 0; i < pulse->mode_count; ++i) {
      gaussian.modes.push_back(
          {pulse->modes[i].ell, pulse->modes[i].m,
           teuk::Complex(pulse->modes[i].amplitude_real,
                         pulse->modes[i].amplitude_imag)});
    }
    teuk::initialize_compactified_gaussian_pulse(
        p->execution, p->pipeline, p->registry, p->ell_max_first,
        p->background, gaussian);
  });
}

int teuk_ref_sample_endpoint(teuk_ref_pipeline* p,
                             teuk_b200_waveform_record* out, size_t capacity,
                             size_t* count) {
  return guarded([&] {
    const auto records =
        p->sampler.sample(p->execution, p->pipeline.storage().state(), 0, 0.0);
    if (records.size() > capacity) {
      throw std::invalid_argument("waveform record capacity is too small");
    }
    for (std::size_t i = 0; i < records.size(); ++i) {
      out[i].boundary = records[i].boundary == teuk::WaveformBoundary::Scri
                            ? TEUK_B200_SCRI
                            : TEUK_B200_HORIZON;
      out[i].order = records[i].perturbative_order;
      out[i].m = records[i].m;
      out[i].ell = records[i].ell;
      out[i].rescaled_real = records[i].rescaled.real();
      out[i].rescaled_imag = records[i].rescaled.imag();
      out[i].endpoint_real = records[i].endpoint_waveform.real();
      out[i].endpoint_imag = records[i].endpoint_waveform.imag();
    }
    *count = records.size();
  });
}

int teuk_ref_get_activation(const teuk_ref_pipeline* p,
                            teuk_b200_activation* out) {
  const auto s = p->pipeline.source_activation_state();
  out->active = s.active ? 1 : 0;
  out->activation_time = s.activation_time;
  out->consecutive_passes = s.consecutive_passes;
  out->last_eligibility_time = s.last_eligibility_time;
  return TEUK_B200_OK;
}

// Project a (modes,13,radial,theta) host state onto the retained bands with
// the reference's own routine (include/teuk/pipeline_bands.hpp).
int teuk_ref_project_to_bands(teuk_ref_pipeline* p, double* state,
                              size_t count) {
  return guarded([&] {
    check_count(*p, count);
    copy_in(p->scratch, state);
    teuk::project_pipeline_state_to_retained_bands(
        p->scratch, p->registry, p->pipeline.angular_bands());
    copy_out(p->scratch, state);
  });
}

// Gauss-Legendre nodes / weights and one fixed-(s,m) synthesis and analysis
// matrix pair exactly as the reference builds them
// (include/teuk/angular.hpp:69-115,329-355), for KAT tests of the product's
// host-side plan builder.
int teuk_ref_gauss_legendre(int nodes, double* x, double* weights) {
  return guarded([&] {
    const auto grid = teuk::angular::gauss_legendre(nodes);
    for (int i = 0; i < nodes; ++i) {
      x[i] = grid.x[static_cast<std::size_t>(i)];
      weights[i] = grid.weights[static_cast<std::size_t>(i)];
    }
  });
}

int teuk_ref_transform_matrices(int spin, int m, int ell_max, int nodes,
                                double* synthesis, double* analysis,
                                int* mode_count) {
  return guarded([&] {
    const teuk::angular::SpinWeightedTransform t(spin, m, ell_max, nodes);
    const std::size_t modes = t.mode_count();
    for (std::size_t j = 0; j < static_cast<std::size_t>(nodes); ++j) {
      for (std::size_t l = 0; l < modes; ++l) {
        synthesis[j * modes + l] = t.synthesis_matrix()(j, l);
        analysis[l * static_cast<std::size_t>(nodes) + j] =
            t.analysis_matrix()(l, j);
      }
    }
    *mode_count = static_cast<int>(modes);
  });
}

// Dense SBP first-derivative matrix h*D and norm weights H/h for n points
// (include/teuk/sbp.hpp, sbp84.hpp, sbp105.hpp).
int teuk_ref_sbp_matrix(int disc, int n, double* derivative, double* norm) {
  return guarded([&] {
    const auto d = discretization(disc);
    const std::size_t count = static_cast<std::size_t>(n);
    std::vector<double> unit(count);
    for (std::size_t column = 0; column < count; ++column) {
      std::fill(unit.begin(), unit.end(), 0.0);
      unit[column] = 1.0;
      for (std::size_t row = 0; row < count; ++row) {
        derivative[row * count + column] =
            teuk::radial_first_derivative_at(d, unit.data(), count, row, 1.0);
      }
    }
    for (std::size_t row = 0; row < count; ++row) {
      norm[row] = teuk::radial_norm_weight(d, count, row);
    }
  });
}

// write_pipeline_checkpoint / load_pipeline_checkpoint_verified
// (include/teuk/pipeline_checkpoint.hpp:782-936) on the reference pipeline.
static teuk::PipelineCheckpointConfiguration checkpoint_configuration(
    const teuk_ref_pipeline& p, const double time_step) {
  teuk::PipelineCheckpointConfiguration c;
  c.background = p.background;
  c.ell_max_first = p.config.ell_max_first;
  c.ell_max_second = p.config.ell_max_second;
  c.theta_nodes = p.config.theta_nodes;
  c.reduction_damping = p.config.reduction_damping;
  c.dissipation = p.config.dissipation;
  c.reduction = p.config.reduction == TEUK_B200_STAGE_CONSTRAINED
                    ? teuk::ReductionEvolution::StageConstrained
                    : teuk::ReductionEvolution::FreeDamped;
  c.time_step = time_step;
  c.source_policy = policy(p.config);
  c.radial_discretization = discretization(p.config.discretization);
  return c;
}

int teuk_ref_checkpoint_write(teuk_ref_pipeline* p, const char* directory,
                              double time_step, double time, uint64_t step) {
  return guarded([&] {
    (void)teuk::write_pipeline_checkpoint(
        p->execution, directory, p->pipeline, p->registry,
        checkpoint_configuration(*p, time_step), {time, step});
  });
}

int teuk_ref_checkpoint_load(teuk_ref_pipeline* p, const char* directory,
                             double time_step, double* time, uint64_t* step) {
  return guarded([&] {
    const auto metadata = teuk::load_pipeline_checkpoint(
        p->execution, directory, p->pipeline, p->registry,
        checkpoint_configuration(*p, time_step));
    if (time != nullptr) *time = metadata.progress.time;
    if (step != nullptr) *step = metadata.progress.step;
  });
}

// parse_run_configuration_text / resolved_configuration_text
// (include/teuk/config.hpp:683-831) and the registry / policy / Gaussian
// mapping of initial_data_factory.hpp:16-79, for parity tests of the
// engine's own parser.
static std::vector<std::string> ref_overrides(const char* const* overrides,
                                              const int count) {
  std::vector<std::string> out;
  for (int i = 0; i < count; ++i) out.emplace_back(overrides[i]);
  return out;
}

int teuk_ref_resolved_config(const char* text, const char* const* overrides,
                             int override_count, char* out, size_t capacity,
                             size_t* length) {
  return guarded([&] {
    const std::string resolved = teuk::resolved_configuration_text(
        teuk::parse_run_configuration_text(
            text, ref_overrides(overrides, override_count)));
    *length = resolved.size();
    if (out != nullptr && capacity > resolved.size()) {
      std::memcpy(out, resolved.c_str(), resolved.size() + 1);
    }
  });
}

int teuk_ref_parse_run_config(const char* text, const char* const* overrides,
                              int override_count, teuk_b200_run_config* out) {
  return guarded([&] {
    const teuk::RunParameters run = teuk::parse_run_configuration_text(
        text, ref_overrides(overrides, override_count));
    const teuk::ModeRegistry registry = teuk::make_run_mode_registry(run);
    const teuk::SecondOrderSourcePolicy policy = teuk::make_source_policy(run);
    teuk_b200_run_config r{};
    r.abi_version = TEUK_B200_ABI_VERSION;
    r.mass = run.background.mass;
    r.spin = run.background.spin;
    r.compactification_length = run.background.compactification_length;
    r.radial_points = run.grid.radial_points;
    r.theta_nodes = run.grid.theta_points;
    r.ell_max_first = run.grid.ell_max_first;
    r.ell_max_second = run.grid.ell_max_second;
    r.mode_count = static_cast<int>(registry.modes().size());
    std::copy(registry.modes().begin(), registry.modes().end(), r.modes);
    r.parent_count = static_cast<int>(registry.parents().size());
    std::copy(registry.parents().begin(), registry.parents().end(), r.parents);
    r.target_count = static_cast<int>(registry.targets().size());
    std::copy(registry.targets().begin(), registry.targets().end(), r.targets);
    r.reduction_damping = run.method.reduction_damping;
    r.dissipation = run.method.dissipation;
    r.reduction = run.method.reduction == teuk::ReductionEvolution::StageConstrained;
    r.discretization = static_cast<int>(run.method.radial_discretization);
    r.source_mode = static_cast<int>(policy.mode);
    r.source_start_time = policy.source_start_time;
    r.normalized_constraint_tolerance = policy.normalized_constraint_tolerance;
    r.required_consecutive_passes = policy.required_consecutive_passes;
    r.final_time = run.time.final_time;
    r.steps = run.time.steps;
    r.cfl = run.time.cfl;
    r.time_step = run.time.final_time / static_cast<double>(run.time.steps);
    r.initial_data_type =
        run.initial_data.type == teuk::InitialDataType::Checkpoint ? 1 : 0;
    const double horizon =
        run.background.compactification_length *
        run.background.compactification_length /
        teuk::outer_horizon_radius(run.background.mass, run.background.spin);
    r.center = run.initial_data.center_fraction * horizon;
    r.width = run.initial_data.width_fraction * horizon;
    r.compact_support = run.initial_data.compact_support ? 1 : 0;
    if (run.initial_data.type == teuk::InitialDataType::Gaussian) {
      const auto seeds = teuk::expanded_gaussian_modes(run.initial_data);
      r.seed_count = static_cast<int>(seeds.size());
      for (std::size_t i = 0; i < seeds.size(); ++i) {
        r.seeds[i] = {seeds[i].ell, seeds[i].m, seeds[i].amplitude.real(),
                      seeds[i].amplitude.imag()};
      }
    }
    std::snprintf(r.checkpoint_directory, sizeof(r.checkpoint_directory), "%s",
                  run.initial_data.checkpoint_directory.c_str());
    std::snprintf(r.output_directory, sizeof(r.output_directory), "%s",
                  run.output.directory.c_str());
    r.diagnostic_every = run.output.diagnostic_interval;
    r.checkpoint_every = run.output.checkpoint_interval;
    *out = r;
  });
}

// PipelineDiagnostics::sample_pipeline (include/teuk/pipeline_diagnostics.hpp)
int teuk_ref_diagnostics(teuk_ref_pipeline* p, teuk_b200_diagnostics* out) {
  return guarded([&] {
    const auto& c = p->config;
    teuk::PipelineDiagnostics diagnostics(
        p->registry.size(),
        teuk::UniformRadialGrid(static_cast<std::size_t>(c.radial_points), 0.0,
                                p->horizon),
        static_cast<std::size_t>(c.theta_nodes), "ref_diagnostics",
        discretization(c.discretization));
    const auto report = diagnostics.sample_pipeline(p->execution, p->pipeline);
    teuk_b200_diagnostics r{};
    for (std::size_t f = 0; f < teuk::point_pipeline_field_count; ++f) {
      r.state[f] = {report.fields[f].state.rms, report.fields[f].state.maximum};
      r.rhs[f] = {report.fields[f].rhs.rms, report.fields[f].rhs.maximum};
    }
    r.first_reduction_constraint = {report.first_reduction_constraint.rms,
                                    report.first_reduction_constraint.maximum};
    r.second_reduction_constraint = {report.second_reduction_constraint.rms,
                                     report.second_reduction_constraint.maximum};
    r.source_over_r3 = {report.source_over_r3.rms, report.source_over_r3.maximum};
    r.forcing = {report.forcing.rms, report.forcing.maximum};
    r.independent_reconstruction_constraint_maximum =
        report.independent_reconstruction_constraint_maximum;
    const teuk::SourceConstraintFamilyNorms* fam[3] = {
        &report.normalized_source_constraints.psi3_bianchi,
        &report.normalized_source_constraints.psi2_bianchi,
        &report.normalized_source_constraints.hll_reality};
    for (int k = 0; k < 3; ++k) {
      r.constraint_absolute_maximum[k] = fam[k]->absolute_maximum;
      r.constraint_normalized_maximum[k] = fam[k]->normalized_maximum;
      r.constraint_weighted_rms[k] = fam[k]->weighted_rms;
      r.constraint_normalized_weighted[k] = fam[k]->normalized_weighted;
    }
    r.constraint_controlling_normalized =
        report.normalized_source_constraints.controlling_normalized;
    r.constraints_finite = report.normalized_source_constraints.all_finite;
    r.activation = {report.source_activation.active ? 1 : 0,
                    report.source_activation.activation_time,
                    report.source_activation.consecutive_passes,
                    report.source_activation.last_eligibility_time};
    r.second_order_source_active = report.second_order_source_active ? 1 : 0;
    r.point_count = report.point_count;
    r.scri_finite = report.scri_finite;
    r.horizon_finite = report.horizon_finite;
    r.all_finite = report.all_finite;
    *out = r;
  });
}

}  // extern "C"
