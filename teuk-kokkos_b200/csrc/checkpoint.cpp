// Pipeline checkpoint format v5 of teuk-kokkos (a metadata.txt of key=value
// lines plus a state.bin of interleaved binary64 complex values, guarded by
// an FNV-1a 64 checksum), written and read for device-resident pipelines.
// Layout, keys, number formatting, validation order and messages follow
// include/teuk/pipeline_checkpoint.hpp so that checkpoints move between the
// reference and this engine in both directions.
#include "checkpoint.h"

#include <algorithm>
#include <bit>
#include <charconv>
#include <chrono>
#include <cmath>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <limits>
#include <map>
#include <numbers>
#include <set>
#include <sstream>
#include <stdexcept>

namespace teuk_b200 {
namespace {

namespace fs = std::filesystem;

constexpr std::uint64_t kFormatVersion = 5;
constexpr std::uint64_t kLegacyD42Version = 4;
constexpr const char* kMetadataFile = "metadata.txt";
constexpr const char* kStateFile = "state.bin";
constexpr double kRestartBandTolerance = 5.0e-11;
// spin weight of each of the 13 stored fields (include/teuk/pipeline_bands.hpp:25-27)
constexpr int kFieldSpins[kFieldCount] = {-2, -2, -2, -1, -2, 0, -2,
                                          -1, -1, 0,  -2, -2, -2};

const char* reduction_name(const int reduction) {
  if (reduction == 0) return "free_damped";
  if (reduction == 1) return "stage_constrained";
  throw std::invalid_argument("unsupported reduction evolution");
}
const char* source_mode_name(const int mode) {
  switch (mode) {
    case 0: return "disabled";
    case 1: return "constraint_aware";
    case 2: return "unrestricted";
  }
  throw std::invalid_argument("unsupported second-order source mode");
}
const char* discretization_name(const int disc) {
  switch (disc) {
    case kD42: return "d4-2";
    case kD84: return "d8-4";
    case kD105: return "d10-5";
  }
  throw std::invalid_argument("unknown radial discretization");
}
int parse_reduction(const std::string& text) {
  if (text == "free_damped") return 0;
  if (text == "stage_constrained") return 1;
  throw std::runtime_error("unsupported checkpoint reduction evolution");
}
int parse_source_mode(const std::string& text) {
  if (text == "disabled") return 0;
  if (text == "constraint_aware") return 1;
  if (text == "unrestricted") return 2;
  throw std::runtime_error("unsupported checkpoint second-order source mode");
}
int parse_discretization(const std::string& text) {
  if (text == "d4-2") return kD42;
  if (text == "d8-4") return kD84;
  if (text == "d10-5") return kD105;
  throw std::invalid_argument("unknown radial discretization: " + text);
}

// The numerical provenance a checkpoint records and a load must match
// (PipelineCheckpointConfiguration).
struct Provenance {
  double mass, spin, length;
  int ell_max_first, ell_max_second, theta_nodes;
  double damping, dissipation;
  int reduction, disc;
  double time_step;
  int source_mode;
  double source_start_time, tolerance;
  int passes;
  bool operator==(const Provenance&) const = default;
};

Provenance provenance(const InstancePlan& plan, const double time_step) {
  const Config& c = plan.config;
  return {c.mass,          c.spin,        c.length,
          c.ell_max_first, c.ell_max_second, c.ntheta,
          c.damping,       c.dissipation, c.reduction,
          c.disc,          time_step,     c.source_mode,
          c.source_start_time, c.constraint_tolerance, c.required_passes};
}

void require_finite(const double value, const char* name) {
  if (!std::isfinite(value)) {
    throw std::invalid_argument(std::string(name) + " must be finite");
  }
}

// validate_configuration (pipeline_checkpoint.hpp:135-171)
void validate_provenance(const Provenance& p) {
  require_finite(p.mass, "checkpoint mass");
  require_finite(p.spin, "checkpoint spin");
  require_finite(p.length, "checkpoint compactification length");
  require_finite(p.damping, "checkpoint reduction damping");
  require_finite(p.dissipation, "checkpoint dissipation");
  require_finite(p.time_step, "checkpoint time step");
  require_finite(p.source_start_time, "checkpoint source start time");
  require_finite(p.tolerance, "checkpoint source constraint tolerance");
  if (!(p.mass > 0.0) || std::abs(p.spin) > p.mass || !(p.length > 0.0) ||
      p.ell_max_first < 3 || p.ell_max_second < 3 ||
      p.theta_nodes < std::max({p.ell_max_first + 1, p.ell_max_second + 1,
                                (2 * p.ell_max_first + p.ell_max_second + 2) /
                                    2}) ||
      p.damping < 0.0 || p.dissipation < 0.0 || !(p.time_step > 0.0) ||
      p.source_start_time < 0.0 || p.tolerance < 0.0 || p.passes < 1) {
    throw std::invalid_argument("invalid pipeline checkpoint configuration");
  }
  (void)reduction_name(p.reduction);
  (void)source_mode_name(p.source_mode);
  (void)discretization_name(p.disc);
}

std::vector<double> radial_coordinates(const InstancePlan& plan) {
  std::vector<double> r(static_cast<std::size_t>(plan.config.nr));
  for (std::size_t i = 0; i < r.size(); ++i) {
    r[i] = 0.0 + plan.spacing * static_cast<double>(i);
  }
  return r;
}

template <class T>
void write_list(std::ostream& out, const std::vector<T>& values) {
  for (std::size_t i = 0; i < values.size(); ++i) {
    if (i != 0) out << ',';
    out << values[i];
  }
  out << '\n';
}

// serialize_metadata (pipeline_checkpoint.hpp:431-483): key order, the
// max_digits10 default float format and the list syntax are the format.
std::string metadata_text(const InstancePlan& plan, const Provenance& p,
                          const CheckpointActivation& a, const double time,
                          const std::uint64_t step, const std::uint64_t sum) {
  const Config& c = plan.config;
  std::ostringstream out;
  out << std::setprecision(std::numeric_limits<double>::max_digits10)
      << "format=teuk-kokkos-pipeline-checkpoint\n"
      << "version=" << kFormatVersion << '\n'
      << "ordering=mode,field,radial,theta\n"
      << "complex_storage=interleaved_real_imag_float64\n"
      << "byte_order=little\n"
      << "state_file=" << kStateFile << '\n'
      << "modes=" << c.modes.size() << '\n'
      << "fields=" << kFieldCount << '\n'
      << "radial=" << c.nr << '\n'
      << "theta=" << c.ntheta << '\n'
      << "m_values=";
  write_list(out, c.modes);
  out << "target_values=";
  write_list(out, c.targets);
  out << "parent_values=";
  write_list(out, c.parents);
  out << "radial_coordinates=";
  write_list(out, radial_coordinates(plan));
  out << "theta_coordinates=";
  write_list(out, plan.theta);
  out << "mass=" << p.mass << '\n'
      << "spin=" << p.spin << '\n'
      << "compactification_length=" << p.length << '\n'
      << "ell_max_first=" << p.ell_max_first << '\n'
      << "ell_max_second=" << p.ell_max_second << '\n'
      << "theta_nodes=" << p.theta_nodes << '\n'
      << "reduction_damping=" << p.damping << '\n'
      << "dissipation=" << p.dissipation << '\n'
      << "reduction=" << reduction_name(p.reduction) << '\n'
      << "radial_discretization=" << discretization_name(p.disc) << '\n'
      << "time_step=" << p.time_step << '\n'
      << "source_mode=" << source_mode_name(p.source_mode) << '\n'
      << "source_start_time=" << p.source_start_time << '\n'
      << "source_normalized_constraint_tolerance=" << p.tolerance << '\n'
      << "source_required_consecutive_passes=" << p.passes << '\n'
      << "source_active=" << (a.active ? 1 : 0) << '\n'
      << "source_activation_time=" << a.activation_time << '\n'
      << "source_consecutive_passes=" << a.consecutive_passes << '\n'
      << "source_last_eligibility_time=" << a.last_eligibility_time << '\n'
      << "time=" << time << '\n'
      << "step=" << step << '\n'
      << "state_checksum_fnv1a64=" << sum << '\n';
  if (!out) throw std::runtime_error("failed serializing checkpoint metadata");
  return out.str();
}

// read_entries (pipeline_checkpoint.hpp:593-641)
std::map<std::string, std::string> read_entries(const std::string& text) {
  std::map<std::string, std::string> entries;
  std::istringstream in(text);
  std::string line;
  while (std::getline(in, line)) {
    const std::size_t eq = line.find('=');
    if (eq == std::string::npos || eq == 0) {
      throw std::runtime_error("malformed checkpoint metadata line");
    }
    const std::string key = line.substr(0, eq);
    if (!entries.emplace(key, line.substr(eq + 1)).second) {
      throw std::runtime_error("duplicate checkpoint metadata key: " + key);
    }
  }
  std::set<std::string> expected{
      "format", "version", "ordering", "complex_storage", "byte_order",
      "state_file", "modes", "fields", "radial", "theta", "m_values",
      "parent_values", "target_values", "radial_coordinates",
      "theta_coordinates", "mass", "spin", "compactification_length",
      "ell_max_first", "ell_max_second", "theta_nodes", "reduction_damping",
      "dissipation", "reduction", "radial_discretization", "time_step",
      "source_mode", "source_start_time",
      "source_normalized_constraint_tolerance",
      "source_required_consecutive_passes", "source_active",
      "source_activation_time", "source_consecutive_passes",
      "source_last_eligibility_time", "time", "step",
      "state_checksum_fnv1a64"};
  const auto version = entries.find("version");
  if (version == entries.end()) {
    throw std::runtime_error("missing checkpoint key: version");
  }
  if (version->second == std::to_string(kLegacyD42Version)) {
    expected.erase("radial_discretization");
  }
  if (entries.size() != expected.size()) {
    throw std::runtime_error("checkpoint metadata key set does not match format");
  }
  for (const auto& entry : entries) {
    if (!expected.contains(entry.first)) {
      throw std::runtime_error("unknown checkpoint metadata key: " + entry.first);
    }
  }
  return entries;
}

const std::string& text_of(const std::map<std::string, std::string>& e,
                           const char* key) {
  const auto it = e.find(key);
  if (it == e.end()) {
    throw std::runtime_error(std::string("missing checkpoint key: ") + key);
  }
  return it->second;
}

template <class T>
T number_of(const std::map<std::string, std::string>& e, const char* key) {
  const std::string& text = text_of(e, key);
  T value{};
  const auto r = std::from_chars(text.data(), text.data() + text.size(), value);
  if (text.empty() || r.ec != std::errc{} || r.ptr != text.data() + text.size()) {
    throw std::runtime_error(std::string("invalid checkpoint value for ") + key);
  }
  return value;
}

template <class T>
std::vector<T> list_of(const std::map<std::string, std::string>& e,
                       const char* key) {
  const std::string& text = text_of(e, key);
  std::vector<T> values;
  std::size_t begin = 0;
  while (begin < text.size()) {
    const std::size_t comma = text.find(',', begin);
    const std::size_t end = comma == std::string::npos ? text.size() : comma;
    T value{};
    const auto r = std::from_chars(text.data() + begin, text.data() + end, value);
    if (end == begin || r.ec != std::errc{} || r.ptr != text.data() + end) {
      throw std::runtime_error(std::string("invalid checkpoint list: ") + key);
    }
    values.push_back(value);
    if (comma == std::string::npos) break;
    begin = comma + 1;
  }
  return values;
}

bool sorted_unique(const std::vector<int>& v) {
  return !v.empty() && std::is_sorted(v.begin(), v.end()) &&
         std::adjacent_find(v.begin(), v.end()) == v.end();
}

std::string read_bytes(const fs::path& path) {
  std::ifstream in(path, std::ios::binary | std::ios::ate);
  if (!in) throw std::runtime_error("cannot open checkpoint content");
  const auto end = in.tellg();
  if (end < 0) throw std::runtime_error("cannot size checkpoint content");
  std::string bytes(static_cast<std::size_t>(end), '\0');
  in.seekg(0);
  if (!bytes.empty()) in.read(bytes.data(), static_cast<std::streamsize>(bytes.size()));
  if (!in) throw std::runtime_error("failed reading checkpoint content");
  return bytes;
}

void write_bytes(const fs::path& path, const char* data, const std::size_t n) {
  std::ofstream out(path, std::ios::binary | std::ios::trunc);
  if (!out) throw std::runtime_error("cannot open checkpoint byte output");
  out.write(data, static_cast<std::streamsize>(n));
  if (!out) throw std::runtime_error("failed writing checkpoint bytes");
}

fs::path reserve_temporary(const fs::path& destination) {
  static std::uint64_t sequence = 0;
  fs::path parent = destination.parent_path();
  if (parent.empty()) parent = ".";
  fs::create_directories(parent);
  const auto tick = static_cast<std::uint64_t>(
      std::chrono::steady_clock::now().time_since_epoch().count());
  for (int attempt = 0; attempt < 100; ++attempt) {
    const fs::path candidate =
        parent / (destination.filename().string() + ".tmp." +
                  std::to_string(tick) + "." + std::to_string(sequence++));
    std::error_code error;
    if (fs::create_directory(candidate, error)) return candidate;
    if (error && error != std::errc::file_exists) {
      throw std::runtime_error("cannot create temporary checkpoint directory");
    }
  }
  throw std::runtime_error("cannot reserve temporary checkpoint directory");
}

// measure_pipeline_state_off_band (pipeline_bands.hpp:108-196): largest
// relative residual of a radial line after analysis + synthesis on the
// field's retained band (inactive (mode, field) planes must be zero).
double off_band_relative(const InstancePlan& plan, const double* state) {
  const Config& c = plan.config;
  const int nt = c.ntheta;
  const double pi = std::numbers::pi_v<double>;
  double worst = 0.0;
  std::vector<double> A, S;
  for (std::size_t mode = 0; mode < c.modes.size(); ++mode) {
    const int m = c.modes[mode];
    for (int field = 0; field < kFieldCount; ++field) {
      const bool second = field >= 10;
      const int ell_max = second ? c.ell_max_second : c.ell_max_first;
      const std::vector<int>& set = second ? c.targets : c.parents;
      const bool active = std::binary_search(set.begin(), set.end(), m);
      const int spin = kFieldSpins[field];
      const int ell_min = std::max(std::abs(spin), std::abs(m));
      const int ne = active ? ell_max - ell_min + 1 : 0;
      A.assign(static_cast<std::size_t>(std::max(ne, 0) * nt), 0.0);
      S.assign(A.size(), 0.0);
      for (int l = 0; l < ne; ++l) {
        for (int j = 0; j < nt; ++j) {
          const double basis = spin_weighted_harmonic_theta(
              ell_min + l, m, spin, plan.theta[static_cast<std::size_t>(j)]);
          S[static_cast<std::size_t>(j * ne + l)] = basis;
          A[static_cast<std::size_t>(l * nt + j)] =
              2.0 * pi * plan.weights[static_cast<std::size_t>(j)] * basis;
        }
      }
      std::vector<double> modal(2 * static_cast<std::size_t>(std::max(ne, 1)));
      for (int r = 0; r < c.nr; ++r) {
        const double* line =
            state + 2 * (((mode * kFieldCount + static_cast<std::size_t>(field)) *
                              static_cast<std::size_t>(c.nr) +
                          static_cast<std::size_t>(r)) *
                         static_cast<std::size_t>(nt));
        for (int l = 0; l < ne; ++l) {
          double re = 0.0, im = 0.0;
          for (int j = 0; j < nt; ++j) {
            re += A[static_cast<std::size_t>(l * nt + j)] * line[2 * j];
            im += A[static_cast<std::size_t>(l * nt + j)] * line[2 * j + 1];
          }
          modal[2 * l] = re;
          modal[2 * l + 1] = im;
        }
        double norm2 = 0.0, residual2 = 0.0;
        for (int j = 0; j < nt; ++j) {
          double re = 0.0, im = 0.0;
          for (int l = 0; l < ne; ++l) {
            re += S[static_cast<std::size_t>(j * ne + l)] * modal[2 * l];
            im += S[static_cast<std::size_t>(j * ne + l)] * modal[2 * l + 1];
          }
          const double v = std::hypot(line[2 * j], line[2 * j + 1]);
          norm2 += v * v;
          const double d = std::hypot(line[2 * j] - re, line[2 * j + 1] - im);
          residual2 += d * d;
        }
        const double relative =
            std::sqrt(residual2) /
            std::max(std::sqrt(norm2), std::numeric_limits<double>::min());
        worst = std::max(worst, relative);
      }
    }
  }
  return worst;
}

}  // namespace

// checksum (pipeline_checkpoint.hpp:276-296)
std::uint64_t checkpoint_checksum(const double* values, const std::size_t count) {
  std::uint64_t h = 14695981039346656037ULL;
  for (std::size_t i = 0; i < 2 * count; ++i) {
    const std::uint64_t bits = std::bit_cast<std::uint64_t>(values[i]);
    for (int b = 0; b < 8; ++b) {  // little-endian byte order
      h ^= (bits >> (8 * b)) & 0xffULL;
      h *= 1099511628211ULL;
    }
  }
  return h;
}

// write_pipeline_checkpoint (pipeline_checkpoint.hpp:782-857)
void write_checkpoint(const std::string& directory, const InstancePlan& plan,
                      const CheckpointActivation& activation,
                      const double time_step, const double time,
                      const std::uint64_t step, const std::vector<double>& state) {
  static_assert(std::endian::native == std::endian::little,
                "checkpoints are written in little-endian byte order");
  const fs::path dir(directory);
  if (dir.empty() || dir.filename().empty() || dir.filename() == "." ||
      dir.filename() == "..") {
    throw std::invalid_argument("checkpoint destination must name a directory");
  }
  if (fs::exists(dir)) {
    throw std::runtime_error("checkpoint destination already exists");
  }
  const Provenance p = provenance(plan, time_step);
  validate_provenance(p);
  require_finite(time, "checkpoint time");
  if (time < 0.0) throw std::invalid_argument("checkpoint time must be nonnegative");
  const std::size_t count = plan.value_count();
  if (state.size() != 2 * count) {
    throw std::invalid_argument("checkpoint state size does not match the pipeline");
  }
  const std::string meta = metadata_text(plan, p, activation, time, step,
                                         checkpoint_checksum(state.data(), count));
  const fs::path temporary = reserve_temporary(dir);
  try {
    write_bytes(temporary / kStateFile,
                reinterpret_cast<const char*>(state.data()),
                state.size() * sizeof(double));
    write_bytes(temporary / kMetadataFile, meta.data(), meta.size());
    fs::rename(temporary, dir);
  } catch (...) {
    std::error_code ignored;
    fs::remove_all(temporary, ignored);
    throw;
  }
}

// load_pipeline_checkpoint_verified (pipeline_checkpoint.hpp:869-936):
// every check completes before the caller's state changes.
CheckpointContents read_checkpoint(const std::string& directory,
                                   const InstancePlan& plan,
                                   const double expected_time_step) {
  const fs::path dir(directory);
  const auto e = read_entries(read_bytes(dir / kMetadataFile));
  if (text_of(e, "format") != "teuk-kokkos-pipeline-checkpoint" ||
      text_of(e, "ordering") != "mode,field,radial,theta" ||
      text_of(e, "complex_storage") != "interleaved_real_imag_float64" ||
      text_of(e, "byte_order") != "little" ||
      text_of(e, "state_file") != kStateFile) {
    throw std::runtime_error("unsupported pipeline checkpoint format");
  }
  const auto version = number_of<std::uint64_t>(e, "version");
  const auto modes = number_of<std::uint64_t>(e, "modes");
  const auto fields = number_of<std::uint64_t>(e, "fields");
  const auto radial = number_of<std::uint64_t>(e, "radial");
  const auto theta = number_of<std::uint64_t>(e, "theta");
  const auto m_values = list_of<int>(e, "m_values");
  const auto parents = list_of<int>(e, "parent_values");
  const auto targets = list_of<int>(e, "target_values");
  const auto r_coords = list_of<double>(e, "radial_coordinates");
  const auto t_coords = list_of<double>(e, "theta_coordinates");
  Provenance p{};
  p.mass = number_of<double>(e, "mass");
  p.spin = number_of<double>(e, "spin");
  p.length = number_of<double>(e, "compactification_length");
  p.ell_max_first = number_of<int>(e, "ell_max_first");
  p.ell_max_second = number_of<int>(e, "ell_max_second");
  p.theta_nodes = number_of<int>(e, "theta_nodes");
  p.damping = number_of<double>(e, "reduction_damping");
  p.dissipation = number_of<double>(e, "dissipation");
  p.reduction = parse_reduction(text_of(e, "reduction"));
  p.disc = version == kLegacyD42Version
               ? kD42
               : parse_discretization(text_of(e, "radial_discretization"));
  p.time_step = number_of<double>(e, "time_step");
  p.source_mode = parse_source_mode(text_of(e, "source_mode"));
  p.source_start_time = number_of<double>(e, "source_start_time");
  p.tolerance = number_of<double>(e, "source_normalized_constraint_tolerance");
  p.passes = number_of<int>(e, "source_required_consecutive_passes");
  const int active = number_of<int>(e, "source_active");
  if (active != 0 && active != 1) {
    throw std::runtime_error("invalid checkpoint source-active flag");
  }
  CheckpointContents out;
  out.activation.active = active != 0;
  out.activation.activation_time = number_of<double>(e, "source_activation_time");
  out.activation.consecutive_passes = number_of<int>(e, "source_consecutive_passes");
  out.activation.last_eligibility_time =
      number_of<double>(e, "source_last_eligibility_time");
  out.time = number_of<double>(e, "time");
  out.step = number_of<std::uint64_t>(e, "step");
  const auto sum = number_of<std::uint64_t>(e, "state_checksum_fnv1a64");

  // validate_metadata (pipeline_checkpoint.hpp:339-428)
  if ((version != kFormatVersion && version != kLegacyD42Version) ||
      fields != static_cast<std::uint64_t>(kFieldCount) ||
      modes != m_values.size() || radial != r_coords.size() ||
      theta != t_coords.size() ||
      p.theta_nodes != static_cast<int>(theta)) {
    throw std::runtime_error("inconsistent pipeline checkpoint metadata");
  }
  if (!sorted_unique(m_values) || !sorted_unique(parents) ||
      !sorted_unique(targets)) {
    throw std::runtime_error(
        "checkpoint modes and targets must be nonempty, sorted, and unique");
  }
  try {
    validate_provenance(p);
  } catch (const std::invalid_argument&) {
    throw std::runtime_error("invalid pipeline checkpoint configuration");
  }
  require_finite(out.time, "checkpoint time");
  if (out.time < 0.0) throw std::runtime_error("checkpoint time must be nonnegative");
  const CheckpointActivation& a = out.activation;
  if (a.consecutive_passes < 0 || !std::isfinite(a.activation_time) ||
      !std::isfinite(a.last_eligibility_time) ||
      (a.active && (a.activation_time < 0.0 || a.activation_time > out.time)) ||
      (!a.active && a.activation_time != -1.0) ||
      a.last_eligibility_time < -1.0 || a.last_eligibility_time > out.time) {
    throw std::runtime_error("invalid checkpoint source activation state");
  }
  for (const double v : r_coords) require_finite(v, "checkpoint radial coordinate");
  for (const double v : t_coords) require_finite(v, "checkpoint theta coordinate");
  const bool theta_up = std::is_sorted(t_coords.begin(), t_coords.end());
  const bool theta_down = std::is_sorted(t_coords.rbegin(), t_coords.rend());
  const std::size_t min_points =
      static_cast<std::size_t>(disc_info(p.disc).min_points);
  if (r_coords.size() < min_points ||
      !std::is_sorted(r_coords.begin(), r_coords.end()) ||
      std::adjacent_find(r_coords.begin(), r_coords.end()) != r_coords.end() ||
      (!theta_up && !theta_down) ||
      std::adjacent_find(t_coords.begin(), t_coords.end()) != t_coords.end()) {
    throw std::runtime_error("invalid checkpoint spatial geometry");
  }
  const double h = (r_coords.back() - r_coords.front()) /
                   static_cast<double>(r_coords.size() - 1);
  for (std::size_t i = 0; i < r_coords.size(); ++i) {
    double lo = r_coords.front() + h * static_cast<double>(i), hi = lo;
    for (int ulp = 0; ulp < 2; ++ulp) {  // two binary64 ulps either side
      lo = std::nextafter(lo, -std::numeric_limits<double>::infinity());
      hi = std::nextafter(hi, std::numeric_limits<double>::infinity());
    }
    if (r_coords[i] < lo || r_coords[i] > hi) {
      throw std::runtime_error("checkpoint radial grid is not uniform");
    }
  }

  // load-time comparisons with the caller's pipeline
  const Config& c = plan.config;
  const Provenance expected = provenance(plan, expected_time_step);
  validate_provenance(expected);
  if (p.source_mode != expected.source_mode ||
      p.source_start_time != expected.source_start_time ||
      p.tolerance != expected.tolerance || p.passes != expected.passes) {
    throw std::runtime_error(
        "checkpoint source policy does not match the caller pipeline");
  }
  if (p.disc != expected.disc) {
    throw std::runtime_error(
        "checkpoint radial discretization does not match caller pipeline");
  }
  if (m_values != c.modes || parents != c.parents || targets != c.targets) {
    throw std::runtime_error("checkpoint mode registry does not match caller");
  }
  if (!(p == expected)) {
    throw std::runtime_error(
        "checkpoint numerical configuration does not match caller");
  }
  if (modes != c.modes.size() || radial != static_cast<std::uint64_t>(c.nr) ||
      theta != static_cast<std::uint64_t>(c.ntheta)) {
    throw std::runtime_error("checkpoint shape does not match pipeline");
  }
  if (r_coords != radial_coordinates(plan) || t_coords != plan.theta) {
    throw std::runtime_error("checkpoint geometry does not match pipeline");
  }
  const std::string bytes = read_bytes(dir / kStateFile);
  const std::size_t count = plan.value_count();
  if (bytes.size() != count * 2 * sizeof(double)) {
    throw std::runtime_error("binary snapshot size does not match metadata");
  }
  out.state.resize(2 * count);
  std::memcpy(out.state.data(), bytes.data(), bytes.size());
  if (checkpoint_checksum(out.state.data(), count) != sum) {
    throw std::runtime_error("pipeline checkpoint state checksum mismatch");
  }
  if (!(off_band_relative(plan, out.state.data()) <= kRestartBandTolerance)) {
    throw std::runtime_error(
        "pipeline checkpoint contains meaningful off-band angular content");
  }
  return out;
}

}  // namespace teuk_b200
