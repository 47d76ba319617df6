// Pipeline checkpoint format v5 (include/teuk/pipeline_checkpoint.hpp):
// host-side writer and verified reader.  The caller moves the state between
// the device and these host buffers.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "engine.h"

namespace teuk_b200 {

struct CheckpointActivation {
  bool active = false;
  double activation_time = -1.0;
  int consecutive_passes = 0;
  double last_eligibility_time = -1.0;
};

struct CheckpointContents {
  std::vector<double> state;  // interleaved (re, im), (mode, field, r, theta)
  CheckpointActivation activation;
  double time = 0.0;
  std::uint64_t step = 0;
};

// FNV-1a 64 over the little-endian bytes of `count` complex values.
std::uint64_t checkpoint_checksum(const double* values, std::size_t count);

// Publishes directory/{metadata.txt, state.bin} through a sibling temporary
// directory and one rename; an existing destination is an error.
void write_checkpoint(const std::string& directory, const InstancePlan& plan,
                      const CheckpointActivation& activation, double time_step,
                      double time, std::uint64_t step,
                      const std::vector<double>& state);

// Parses and validates a checkpoint against the caller's pipeline plan and
// time step; throws std::runtime_error / std::invalid_argument with the
// reference's messages.
CheckpointContents read_checkpoint(const std::string& directory,
                                   const InstancePlan& plan,
                                   double expected_time_step);

}  // namespace teuk_b200
