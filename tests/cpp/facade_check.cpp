// Drives the C++ facade (include/teuk_b200.hpp) the way teuk_solver drives
// teuk::SpatialPipeline.  Exit codes:
//   0  invalid configurations threw std::invalid_argument and, on a GPU
//      host, a valid pipeline stepped and returned a finite state;
//   3  no usable CUDA device: the valid pipeline threw std::runtime_error
//      (the engine has no CPU fallback);
//   1  anything else.
#include <cmath>
#include <cstdio>
#include <stdexcept>

#include "teuk_b200.hpp"

int main() {
  using namespace teuk_b200;
  const ModeLists modes({-2, 2});
  // nr below the D10-5 minimum: rejected before any device work.
  try {
    SpatialPipeline bad(modes, 12, {8, 8}, 13, {1.0, 0.0, 1.0}, 0.1, 0.0,
                        ReductionEvolution::FreeDamped,
                        SecondOrderSourcePolicy::disabled(),
                        RadialDiscretization::D105);
    std::puts("invalid radial grid was accepted");
    return 1;
  } catch (const std::invalid_argument& e) {
    std::printf("invalid_argument: %s\n", e.what());
  }
  // ntheta below the exact-product padding.
  try {
    SpatialPipeline bad(modes, 64, {8, 8}, 9, {1.0, 0.0, 1.0});
    std::puts("invalid theta grid was accepted");
    return 1;
  } catch (const std::invalid_argument& e) {
    std::printf("invalid_argument: %s\n", e.what());
  }
  try {
    SpatialPipeline p(modes, 64, {8, 8}, 13, {1.0, 0.5, 1.0}, 0.1, 0.005,
                      ReductionEvolution::FreeDamped,
                      SecondOrderSourcePolicy::disabled(),
                      RadialDiscretization::D84);
    const double horizon = 1.0 / (1.0 + std::sqrt(1.0 - 0.25));
    p.initialize_gaussian(0.3 * horizon, 0.06 * horizon,
                          {{2, 2, 1e-3, 0.0}, {2, -2, 0.0, 1e-3}});
    p.advance(0.0, 1e-4, 10);
    const auto state = p.state();
    double norm = 0.0;
    for (const auto& v : state) norm += std::norm(v);
    if (!std::isfinite(norm) || norm == 0.0) {
      std::puts("non-finite or empty state");
      return 1;
    }
    const auto records = p.sample_endpoint();
    std::printf("stepped: |state|^2 = %.6e, %zu waveform records\n", norm,
                records.size());
    return 0;
  } catch (const std::runtime_error& e) {
    std::printf("runtime_error: %s\n", e.what());
    return 3;
  }
}
