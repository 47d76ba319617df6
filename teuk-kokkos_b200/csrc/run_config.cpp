// Runtime .cfg schema of teuk_solver: key = value lines with '#' comments,
// command-line overrides, resolution onto RunParameters, validation and the
// resolved_config.cfg text.  Keys, defaults, messages and check order follow
// include/teuk/config.hpp:26-831 so that a configuration is accepted or
// rejected exactly as the reference would and resolves to the same text.
#include "run_config.h"

#include <algorithm>
#include <charconv>
#include <cmath>
#include <iomanip>
#include <limits>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>

namespace teuk_b200 {
namespace {

using Entries = std::map<std::string, std::string>;

std::string trim(const std::string_view text) {
  const auto ws = [](const unsigned char c) {
    return c == ' ' || c == '\t' || c == '\r' || c == '\n';
  };
  std::size_t b = 0, e = text.size();
  while (b < e && ws(static_cast<unsigned char>(text[b]))) ++b;
  while (e > b && ws(static_cast<unsigned char>(text[e - 1]))) --e;
  return std::string(text.substr(b, e - b));
}

std::pair<std::string, std::string> assignment(const std::string_view text,
                                               const std::string& context) {
  const std::size_t eq = text.find('=');
  if (eq == std::string_view::npos ||
      text.find('=', eq + 1) != std::string_view::npos) {
    throw std::invalid_argument(context + ": expected exactly one key = value");
  }
  std::string key = trim(text.substr(0, eq));
  std::string value = trim(text.substr(eq + 1));
  if (key.empty() || value.empty()) {
    throw std::invalid_argument(context + ": empty configuration key or value");
  }
  return {std::move(key), std::move(value)};
}

template <class T>
T number(const std::string& text, const std::string& key) {
  T value{};
  const auto r = std::from_chars(text.data(), text.data() + text.size(), value);
  if (r.ec != std::errc{} || r.ptr != text.data() + text.size()) {
    throw std::invalid_argument("key '" + key + "' has malformed value '" +
                                text + "'");
  }
  return value;
}

bool boolean(const std::string& text, const std::string& key) {
  if (text == "true" || text == "1") return true;
  if (text == "false" || text == "0") return false;
  throw std::invalid_argument("key '" + key + "' requires true, false, 1, or 0");
}

std::vector<int> int_list(const std::string& text, const std::string& key) {
  std::vector<int> values;
  std::size_t begin = 0;
  while (begin < text.size()) {
    const std::size_t comma = text.find(',', begin);
    const std::size_t end = comma == std::string::npos ? text.size() : comma;
    const std::string token = trim(std::string_view(text).substr(begin, end - begin));
    if (token.empty()) {
      throw std::invalid_argument("key '" + key + "' contains an empty item");
    }
    values.push_back(number<int>(token, key));
    if (comma == std::string::npos) break;
    begin = comma + 1;
  }
  if (values.empty()) {
    throw std::invalid_argument("key '" + key + "' requires a nonempty list");
  }
  return values;
}

Entries parse_stream(const std::string& text, const std::string& source) {
  Entries entries;
  std::istringstream in(text);
  std::string line;
  std::size_t number_of_line = 0;
  while (std::getline(in, line)) {
    ++number_of_line;
    const std::size_t hash = line.find('#');
    if (hash != std::string::npos) line.erase(hash);
    if (trim(line).empty()) continue;
    auto [key, value] =
        assignment(line, source + ":" + std::to_string(number_of_line));
    if (!entries.emplace(key, value).second) {
      throw std::invalid_argument(source + ":" + std::to_string(number_of_line) +
                                  ": duplicate key '" + key + "'");
    }
  }
  return entries;
}

void require_finite(const double v, const std::string& key) {
  if (!std::isfinite(v)) throw std::invalid_argument("key '" + key + "' must be finite");
}

const char* disc_name(const int d) {
  switch (d) {
    case kD42: return "d4-2";
    case kD84: return "d8-4";
    case kD105: return "d10-5";
  }
  throw std::invalid_argument("unknown radial discretization");
}
int parse_disc(const std::string& t) {
  if (t == "d4-2") return kD42;
  if (t == "d8-4") return kD84;
  if (t == "d10-5") return kD105;
  throw std::invalid_argument("unknown radial discretization: " + t);
}

constexpr const char* kPlus2Modes[] = {"disabled", "diagnostic_only",
                                       "concurrent", "replay"};
constexpr const char* kPlus2Linear[] = {"metric_curvature", "tsi", "both"};
constexpr const char* kPlus2Policy[] = {"zero", "checkpoint"};
constexpr int kPlus2NormalizationVersion = 2;
constexpr const char* kPlus2NormalizationName =
    "plus2_s0_over_r7_complete_field_factor_v2";

template <std::size_t N>
int parse_name(const char* const (&names)[N], const std::string& text,
               const std::string& what) {
  for (std::size_t i = 0; i < N; ++i) {
    if (text == names[i]) return static_cast<int>(i);
  }
  throw std::invalid_argument("unknown " + what + ": " + text);
}

bool mode_field(const std::string& key, std::size_t& index, std::string& field) {
  constexpr std::string_view prefix = "initial_data.mode.";
  if (!key.starts_with(prefix)) return false;
  const std::size_t dot = key.find('.', prefix.size());
  if (dot == std::string::npos) return false;
  const std::string index_text = key.substr(prefix.size(), dot - prefix.size());
  if (index_text.empty()) return false;
  index = number<std::size_t>(index_text, key);
  field = key.substr(dot + 1);
  return field == "ell" || field == "m" || field == "amplitude_real" ||
         field == "amplitude_imag";
}

// resolve_run_parameters (config.hpp:188-432)
RunParameters resolve(const Entries& entries) {
  RunParameters p;
  std::set<std::string> recognized;
  const auto value = [&](const std::string& key) -> const std::string* {
    const auto it = entries.find(key);
    if (it == entries.end()) return nullptr;
    recognized.insert(key);
    return &it->second;
  };
  const auto set_double = [&](const std::string& k, double& d) {
    if (const auto* t = value(k)) d = number<double>(*t, k);
  };
  const auto set_int = [&](const std::string& k, int& d) {
    if (const auto* t = value(k)) d = number<int>(*t, k);
  };
  const auto set_bool = [&](const std::string& k, bool& d) {
    if (const auto* t = value(k)) d = boolean(*t, k);
  };
  const auto set_string = [&](const std::string& k, std::string& d) {
    if (const auto* t = value(k)) d = *t;
  };
  struct Builder {
    RunSeed seed;
    bool ell = false, m = false, re = false, im = false;
  };
  std::map<std::size_t, Builder> builders;
  builders[0].seed = p.seeds.front();

  set_int("config_version", p.config_version);
  set_double("mass", p.mass);
  set_double("spin", p.spin);
  set_double("compactification_length", p.length);
  set_int("nr", p.nr);
  set_int("ntheta", p.ntheta);
  set_int("ellmax_first", p.ell_max_first);
  const bool second_explicit = entries.contains("ellmax_second");
  set_int("ellmax_second", p.ell_max_second);
  if (!second_explicit) p.ell_max_second = p.ell_max_first;
  if (const auto* t = value("first_order_modes")) {
    p.first_order_modes = int_list(*t, "first_order_modes");
  }
  if (const auto* t = value("second_order_modes")) {
    p.second_order_modes = int_list(*t, "second_order_modes");
  }
  set_double("final_time", p.final_time);
  set_int("steps", p.steps);
  set_double("cfl", p.cfl);
  set_double("reduction_damping", p.reduction_damping);
  set_double("dissipation", p.dissipation);
  if (const auto* t = value("radial_discretization")) p.disc = parse_disc(*t);
  if (const auto* t = value("reduction_mode")) {
    if (*t == "free_damped") {
      p.reduction = 0;
    } else if (*t == "stage_constrained") {
      p.reduction = 1;
    } else {
      throw std::invalid_argument(
          "key 'reduction_mode' requires free_damped or stage_constrained");
    }
  }
  if (const auto* t = value("initial_data.type")) {
    if (*t == "gaussian") {
      p.initial_type = 0;
    } else if (*t == "checkpoint") {
      p.initial_type = 1;
    } else {
      throw std::invalid_argument(
          "key 'initial_data.type' requires gaussian or checkpoint");
    }
  }
  set_bool("initial_data.add_sharp_partner", p.add_sharp_partner);
  set_bool("initial_data.compact_support", p.compact_support);
  set_double("initial_data.center", p.center_fraction);
  set_double("initial_data.width", p.width_fraction);
  set_string("initial_data.time_derivative", p.time_derivative);
  set_string("initial_data.checkpoint_directory", p.checkpoint_directory);
  if (p.checkpoint_directory == "none") p.checkpoint_directory.clear();

  Builder& base = builders[0];
  if (const auto* t = value("initial_data.seed_ell")) {
    base.seed.ell = number<int>(*t, "initial_data.seed_ell");
  }
  if (const auto* t = value("initial_data.seed_m")) {
    base.seed.m = number<int>(*t, "initial_data.seed_m");
  }
  double base_re = base.seed.amplitude.real(), base_im = base.seed.amplitude.imag();
  if (const auto* t = value("initial_data.amplitude_real")) {
    base_re = number<double>(*t, "initial_data.amplitude_real");
  }
  if (const auto* t = value("initial_data.amplitude_imag")) {
    base_im = number<double>(*t, "initial_data.amplitude_imag");
  }
  base.seed.amplitude = {base_re, base_im};
  for (const auto& [key, text] : entries) {
    std::size_t index = 0;
    std::string field;
    if (!mode_field(key, index, field)) continue;
    recognized.insert(key);
    Builder& b = builders[index];
    if (field == "ell") {
      b.seed.ell = number<int>(text, key);
      b.ell = true;
    } else if (field == "m") {
      b.seed.m = number<int>(text, key);
      b.m = true;
    } else if (field == "amplitude_real") {
      b.seed.amplitude = {number<double>(text, key), b.seed.amplitude.imag()};
      b.re = true;
    } else {
      b.seed.amplitude = {b.seed.amplitude.real(), number<double>(text, key)};
      b.im = true;
    }
  }
  p.seeds.clear();
  for (const auto& [index, b] : builders) {
    if (index != 0 && !(b.ell && b.m && b.re && b.im)) {
      throw std::invalid_argument(
          "initial_data.mode." + std::to_string(index) +
          " requires ell, m, amplitude_real, and amplitude_imag");
    }
    p.seeds.push_back(b.seed);
  }

  set_bool("second_order.enabled", p.second_enabled);
  if (const auto* t = value("second_order.source_mode")) {
    if (*t == "constraint_aware") {
      p.source_mode = 1;
    } else if (*t == "unrestricted") {
      p.source_mode = 2;
    } else {
      throw std::invalid_argument(
          "key 'second_order.source_mode' requires constraint_aware or unrestricted");
    }
  }
  set_double("second_order.source_start_time", p.source_start_time);
  set_double("second_order.constraint_tolerance", p.constraint_tolerance);
  set_int("second_order.required_consecutive_passes", p.required_passes);
  set_bool("second_order.allow_truncated_daughter_modes",
           p.allow_truncated_daughters);

  set_bool("plus2.enabled", p.plus2_enabled);
  if (const auto* t = value("plus2.mode")) {
    p.plus2_mode = parse_name(kPlus2Modes, *t, "plus2 run mode");
  }
  if (const auto* t = value("plus2.linear.method")) {
    p.plus2_linear_method = parse_name(kPlus2Linear, *t, "plus2 linear method");
  }
  set_bool("plus2.linear.evolve_validation", p.plus2_linear_evolve_validation);
  if (const auto* t = value("plus2.second.method")) {
    if (*t != "sourced_companion") {
      throw std::invalid_argument("unknown plus2 second method: " + *t);
    }
    p.plus2_second_method = 0;
  }
  if (const auto* t = value("plus2.second.initial_policy")) {
    p.plus2_initial_policy = parse_name(kPlus2Policy, *t, "plus2 initial policy");
  }
  set_string("plus2.second.checkpoint", p.plus2_second_checkpoint);
  if (p.plus2_second_checkpoint == "none") p.plus2_second_checkpoint.clear();
  const bool p2_first = entries.contains("plus2.ell_max_first");
  const bool p2_second = entries.contains("plus2.ell_max_second");
  set_int("plus2.ell_max_first", p.plus2_ell_max_first);
  set_int("plus2.ell_max_second", p.plus2_ell_max_second);
  if (!p2_first) p.plus2_ell_max_first = p.ell_max_first;
  if (!p2_second) p.plus2_ell_max_second = p.ell_max_second;
  set_bool("plus2.output.regularized", p.plus2_regularized);
  set_bool("plus2.output.physical_tetrad_field", p.plus2_physical);
  set_bool("plus2.output.source_families", p.plus2_source_families);
  set_bool("plus2.output.ordered_pairs", p.plus2_ordered_pairs);
  if (const auto* t = value("plus2.source_normalization.version")) {
    if (number<int>(*t, "plus2.source_normalization.version") !=
        kPlus2NormalizationVersion) {
      throw std::invalid_argument(
          "resolved plus2 source-normalization version is incompatible");
    }
  }
  if (const auto* t = value("plus2.source_normalization.name")) {
    if (*t != kPlus2NormalizationName) {
      throw std::invalid_argument(
          "resolved plus2 source-normalization name is incompatible");
    }
  }
  set_string("output.directory", p.output_directory);
  set_int("output.diagnostic_every", p.diagnostic_every);
  set_int("output.checkpoint_every", p.checkpoint_every);
  for (const auto& entry : entries) {
    if (!recognized.contains(entry.first)) {
      throw std::invalid_argument("unknown configuration key '" + entry.first + "'");
    }
  }
  return p;
}

// validate_run_parameters (config.hpp:434-681)
void validate(const RunParameters& p) {
  if (p.config_version != 1) throw std::invalid_argument("config_version must be 1");
  require_finite(p.mass, "mass");
  require_finite(p.spin, "spin");
  require_finite(p.length, "compactification_length");
  if (!(p.mass > 0.0)) throw std::invalid_argument("mass must be positive");
  if (std::abs(p.spin) > p.mass) {
    throw std::invalid_argument("absolute spin must not exceed mass");
  }
  if (!(p.length > 0.0)) {
    throw std::invalid_argument("compactification_length must be positive");
  }
  if (p.nr < disc_info(p.disc).min_points) {
    throw std::invalid_argument("nr is too small for radial_discretization=" +
                                std::string(disc_name(p.disc)));
  }
  if (p.ell_max_first < 3 || p.ell_max_second < 3) {
    throw std::invalid_argument("ellmax_first and ellmax_second must be at least 3");
  }
  const int product = (2 * p.ell_max_first + p.ell_max_second + 2) / 2;
  if (p.ntheta < std::max({p.ell_max_first + 1, p.ell_max_second + 1, product})) {
    throw std::invalid_argument(
        "ntheta is too small for the selected first/second angular bands");
  }
  const auto validate_modes = [](const std::vector<int>& modes, const int ell_max,
                                 const std::string& key) {
    if (modes.empty()) throw std::invalid_argument(key + " must not be empty");
    std::vector<int> sorted = modes;
    std::sort(sorted.begin(), sorted.end());
    if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end()) {
      throw std::invalid_argument(key + " must contain unique signed modes");
    }
    for (const int m : sorted) {
      if (std::abs(m) > ell_max) {
        throw std::invalid_argument(key + " contains |m| above its ellmax");
      }
      if (!std::binary_search(sorted.begin(), sorted.end(), -m)) {
        throw std::invalid_argument(key + " must be closed under m -> -m");
      }
    }
  };
  validate_modes(p.first_order_modes, p.ell_max_first, "first_order_modes");
  validate_modes(p.second_order_modes, p.ell_max_second, "second_order_modes");
  if (p.second_enabled) {
    // validate_quadratic_daughter_modes (modes.hpp:222-264)
    std::set<int> daughters;
    for (const int a : p.first_order_modes) {
      for (const int b : p.first_order_modes) {
        const long long sum = static_cast<long long>(a) + b;
        if (sum < std::numeric_limits<int>::min() ||
            sum > std::numeric_limits<int>::max()) {
          throw std::invalid_argument("quadratic daughter mode overflows int");
        }
        daughters.insert(static_cast<int>(sum));
      }
    }
    std::string missing;
    for (const int d : daughters) {
      if (std::find(p.second_order_modes.begin(), p.second_order_modes.end(), d) ==
          p.second_order_modes.end()) {
        missing += " " + std::to_string(d);
      }
    }
    if (!missing.empty() && !p.allow_truncated_daughters) {
      throw std::invalid_argument("second-order mode set omits quadratic daughters:" +
                                  missing);
    }
  }
  require_finite(p.final_time, "final_time");
  require_finite(p.cfl, "cfl");
  if (!(p.final_time > 0.0) || p.steps <= 0 || !(p.cfl > 0.0)) {
    throw std::invalid_argument("final_time, steps, and cfl must be positive");
  }
  require_finite(p.reduction_damping, "reduction_damping");
  require_finite(p.dissipation, "dissipation");
  if (p.reduction_damping < 0.0 || p.dissipation < 0.0) {
    throw std::invalid_argument(
        "reduction_damping and dissipation must be nonnegative");
  }
  // radial_dissipation_rk4_step_is_admissible (radial_discretization.hpp:20-67)
  const double horizon = p.mass + std::sqrt(p.mass * p.mass - p.spin * p.spin);
  const double compact = p.length * p.length / horizon;
  const double spacing = compact / static_cast<double>(p.nr - 1);
  const double ratio = (p.final_time / static_cast<double>(p.steps)) / spacing;
  const double bounds[3] = {64.0, 1371.0, 5500.0};
  const bool admissible =
      std::isfinite(ratio) && ratio >= 0.0 &&
      (p.dissipation == 0.0 ||
       ratio <= 0.8 * 2.785293563405282 / (p.dissipation * bounds[p.disc]));
  if (!admissible) {
    throw std::invalid_argument(
        "steps are too small for the selected radial dissipation RK4 bound");
  }
  if (p.initial_type == 0) {
    if (p.seeds.empty()) {
      throw std::invalid_argument("Gaussian initial data require a seed mode");
    }
    std::set<std::pair<int, int>> keys;
    for (const RunSeed& s : p.seeds) {
      require_finite(s.amplitude.real(), "initial_data amplitude_real");
      require_finite(s.amplitude.imag(), "initial_data amplitude_imag");
      if (s.ell < std::max(2, std::abs(s.m)) || s.ell > p.ell_max_first) {
        throw std::invalid_argument(
            "initial-data seed ell exceeds ellmax_first or minimum ell");
      }
      if (std::find(p.first_order_modes.begin(), p.first_order_modes.end(), s.m) ==
          p.first_order_modes.end()) {
        throw std::invalid_argument(
            "initial-data seed m is absent from first_order_modes");
      }
      if (!keys.emplace(s.ell, s.m).second) {
        throw std::invalid_argument("duplicate initial-data (ell,m) seed");
      }
      if (p.add_sharp_partner && s.m != 0 && keys.contains({s.ell, -s.m})) {
        throw std::invalid_argument(
            "add_sharp_partner would duplicate an explicit seed");
      }
    }
    require_finite(p.center_fraction, "initial_data.center");
    require_finite(p.width_fraction, "initial_data.width");
    if (p.center_fraction < 0.0 || p.center_fraction > 1.0 ||
        !(p.width_fraction > 0.0)) {
      throw std::invalid_argument(
          "initial_data.center must be in [0,1] and width must be positive");
    }
    if (p.time_derivative != "zero") {
      throw std::invalid_argument(
          "initial_data.time_derivative currently supports only 'zero'");
    }
  } else if (p.checkpoint_directory.empty()) {
    throw std::invalid_argument(
        "checkpoint initial data require initial_data.checkpoint_directory");
  }
  require_finite(p.source_start_time, "second_order.source_start_time");
  require_finite(p.constraint_tolerance, "second_order.constraint_tolerance");
  if (p.source_start_time < 0.0 || p.constraint_tolerance < 0.0 ||
      p.required_passes < 1) {
    throw std::invalid_argument("invalid second-order source activation policy");
  }
  const bool plus2_mode_enabled = p.plus2_mode != 0;
  if (p.plus2_enabled != plus2_mode_enabled) {
    throw std::invalid_argument(
        "plus2.enabled must be true exactly when plus2.mode is not disabled");
  }
  if (p.plus2_ell_max_first < 2 || p.plus2_ell_max_second < 2) {
    throw std::invalid_argument(
        "plus2 ell_max_first and ell_max_second must be at least 2");
  }
  for (const int m : p.first_order_modes) {
    if (std::abs(m) > p.plus2_ell_max_first) {
      throw std::invalid_argument("first_order_modes contains |m| above the plus2 band");
    }
  }
  for (const int m : p.second_order_modes) {
    if (std::abs(m) > p.plus2_ell_max_second) {
      throw std::invalid_argument(
          "second_order_modes contains |m| above the plus2 band");
    }
  }
  const int plus2_product = (2 * p.plus2_ell_max_first + p.plus2_ell_max_second + 2) / 2;
  if (p.plus2_enabled &&
      p.ntheta < std::max({p.plus2_ell_max_first + 1, p.plus2_ell_max_second + 1,
                           plus2_product})) {
    throw std::invalid_argument(
        "ntheta is too small for the selected plus2 angular bands");
  }
  const bool checkpoint_policy = p.plus2_initial_policy == 1;
  if (checkpoint_policy != !p.plus2_second_checkpoint.empty()) {
    throw std::invalid_argument(
        "plus2.second.checkpoint is required exactly for checkpoint initial policy");
  }
  if (!p.plus2_second_checkpoint.empty() &&
      p.plus2_second_checkpoint.find_first_of("\r\n#=") != std::string::npos) {
    throw std::invalid_argument(
        "plus2.second.checkpoint must be a config-safe single-line path");
  }
  if ((p.plus2_mode == 0 || p.plus2_mode == 1) && checkpoint_policy) {
    throw std::invalid_argument(
        "plus2 disabled/diagnostic_only mode cannot load a second-order companion checkpoint");
  }
  if ((p.plus2_mode == 2 || p.plus2_mode == 3) && !p.second_enabled) {
    throw std::invalid_argument(
        "plus2 concurrent/replay requires second_order.enabled=true for four-field evolution");
  }
  if (p.plus2_ordered_pairs && !p.plus2_source_families) {
    throw std::invalid_argument(
        "plus2 ordered-pair output requires source-family output");
  }
  if (p.plus2_enabled && !p.plus2_regularized && !p.plus2_physical) {
    throw std::invalid_argument(
        "enabled plus2 mode must output a regularized or physical tetrad field");
  }
  if (p.output_directory.empty() ||
      p.output_directory.find_first_of("\r\n") != std::string::npos) {
    throw std::invalid_argument("output.directory must be a nonempty single line");
  }
  if (p.diagnostic_every <= 0 || p.checkpoint_every < 0) {
    throw std::invalid_argument(
        "diagnostic cadence must be positive and checkpoint cadence nonnegative");
  }
}

}  // namespace

RunParameters parse_run_configuration(const std::string& text,
                                      const std::vector<std::string>& overrides) {
  Entries entries = parse_stream(text, "<configuration>");
  Entries extra;
  for (std::size_t i = 0; i < overrides.size(); ++i) {
    auto [key, value] =
        assignment(overrides[i], "command-line override " + std::to_string(i + 1));
    if (!extra.emplace(key, value).second) {
      throw std::invalid_argument("duplicate command-line override '" + key + "'");
    }
  }
  for (const auto& [key, value] : extra) entries[key] = value;
  RunParameters run = resolve(entries);
  validate(run);
  return run;
}

std::string resolved_configuration_text(const RunParameters& p) {
  validate(p);
  std::ostringstream out;
  out << std::setprecision(17) << std::boolalpha
      << "config_version = " << p.config_version << '\n'
      << "mass = " << p.mass << '\n'
      << "spin = " << p.spin << '\n'
      << "compactification_length = " << p.length << '\n'
      << "nr = " << p.nr << '\n'
      << "ntheta = " << p.ntheta << '\n'
      << "ellmax_first = " << p.ell_max_first << '\n'
      << "ellmax_second = " << p.ell_max_second << '\n';
  const auto modes = [&](const char* key, const std::vector<int>& v) {
    out << key << " = ";
    for (std::size_t i = 0; i < v.size(); ++i) {
      if (i != 0) out << ',';
      out << v[i];
    }
    out << '\n';
  };
  modes("first_order_modes", p.first_order_modes);
  modes("second_order_modes", p.second_order_modes);
  out << "final_time = " << p.final_time << '\n'
      << "steps = " << p.steps << '\n'
      << "cfl = " << p.cfl << '\n'
      << "reduction_damping = " << p.reduction_damping << '\n'
      << "dissipation = " << p.dissipation << '\n'
      << "radial_discretization = " << disc_name(p.disc) << '\n'
      << "reduction_mode = "
      << (p.reduction == 0 ? "free_damped" : "stage_constrained") << '\n'
      << "initial_data.type = " << (p.initial_type == 0 ? "gaussian" : "checkpoint")
      << '\n'
      << "initial_data.add_sharp_partner = " << p.add_sharp_partner << '\n'
      << "initial_data.compact_support = " << p.compact_support << '\n'
      << "initial_data.center = " << p.center_fraction << '\n'
      << "initial_data.width = " << p.width_fraction << '\n'
      << "initial_data.time_derivative = " << p.time_derivative << '\n'
      << "initial_data.checkpoint_directory = "
      << (p.checkpoint_directory.empty() ? "none" : p.checkpoint_directory) << '\n';
  for (std::size_t i = 0; i < p.seeds.size(); ++i) {
    const RunSeed& s = p.seeds[i];
    out << "initial_data.mode." << i << ".ell = " << s.ell << '\n'
        << "initial_data.mode." << i << ".m = " << s.m << '\n'
        << "initial_data.mode." << i << ".amplitude_real = " << s.amplitude.real()
        << '\n'
        << "initial_data.mode." << i << ".amplitude_imag = " << s.amplitude.imag()
        << '\n';
  }
  out << "second_order.enabled = " << p.second_enabled << '\n'
      << "second_order.source_mode = "
      << (p.source_mode == 2 ? "unrestricted" : "constraint_aware") << '\n'
      << "second_order.source_start_time = " << p.source_start_time << '\n'
      << "second_order.constraint_tolerance = " << p.constraint_tolerance << '\n'
      << "second_order.required_consecutive_passes = " << p.required_passes << '\n'
      << "second_order.allow_truncated_daughter_modes = "
      << p.allow_truncated_daughters << '\n'
      << "plus2.enabled = " << p.plus2_enabled << '\n'
      << "plus2.mode = " << kPlus2Modes[p.plus2_mode] << '\n'
      << "plus2.linear.method = " << kPlus2Linear[p.plus2_linear_method] << '\n'
      << "plus2.linear.evolve_validation = " << p.plus2_linear_evolve_validation
      << '\n'
      << "plus2.second.method = sourced_companion\n"
      << "plus2.second.initial_policy = " << kPlus2Policy[p.plus2_initial_policy]
      << '\n'
      << "plus2.second.checkpoint = "
      << (p.plus2_second_checkpoint.empty() ? "none" : p.plus2_second_checkpoint)
      << '\n'
      << "plus2.ell_max_first = " << p.plus2_ell_max_first << '\n'
      << "plus2.ell_max_second = " << p.plus2_ell_max_second << '\n'
      << "plus2.output.regularized = " << p.plus2_regularized << '\n'
      << "plus2.output.physical_tetrad_field = " << p.plus2_physical << '\n'
      << "plus2.output.source_families = " << p.plus2_source_families << '\n'
      << "plus2.output.ordered_pairs = " << p.plus2_ordered_pairs << '\n'
      << "plus2.source_normalization.version = " << kPlus2NormalizationVersion
      << '\n'
      << "plus2.source_normalization.name = " << kPlus2NormalizationName << '\n'
      << "output.directory = " << p.output_directory << '\n'
      << "output.diagnostic_every = " << p.diagnostic_every << '\n'
      << "output.checkpoint_every = " << p.checkpoint_every << '\n';
  return out.str();
}

// make_run_mode_registry / make_source_policy
// (include/teuk/initial_data_factory.hpp:16-37)
Config pipeline_config(const RunParameters& p) {
  Config c;
  c.mass = p.mass;
  c.spin = p.spin;
  c.length = p.length;
  c.nr = p.nr;
  c.ntheta = p.ntheta;
  c.ell_max_first = p.ell_max_first;
  c.ell_max_second = p.ell_max_second;
  std::vector<int> stored = p.first_order_modes;
  stored.insert(stored.end(), p.second_order_modes.begin(), p.second_order_modes.end());
  std::sort(stored.begin(), stored.end());
  stored.erase(std::unique(stored.begin(), stored.end()), stored.end());
  c.modes = stored;
  c.parents = p.first_order_modes;
  std::sort(c.parents.begin(), c.parents.end());
  c.targets = p.second_order_modes;
  std::sort(c.targets.begin(), c.targets.end());
  c.damping = p.reduction_damping;
  c.dissipation = p.dissipation;
  c.reduction = p.reduction;
  c.disc = p.disc;
  if (p.second_enabled) {
    c.source_mode = p.source_mode;
    c.source_start_time = p.source_start_time;
    c.constraint_tolerance = p.constraint_tolerance;
    c.required_passes = p.required_passes;
  } else {
    c.source_mode = 0;
    c.source_start_time = 0.0;
    c.constraint_tolerance = 0.0;
    c.required_passes = 1;
  }
  return c;
}

double run_time_step(const RunParameters& p) {
  return p.final_time / static_cast<double>(p.steps);
}

// expanded_gaussian_modes (include/teuk/initial_data_factory.hpp:56-79)
std::vector<RunSeed> expanded_seeds(const RunParameters& p) {
  std::vector<RunSeed> out;
  for (const RunSeed& s : p.seeds) {
    out.push_back(s);
    if (p.add_sharp_partner && s.m != 0) {
      out.push_back({s.ell, -s.m, std::conj(s.amplitude)});
    }
  }
  std::sort(out.begin(), out.end(), [](const RunSeed& a, const RunSeed& b) {
    return a.m != b.m ? a.m < b.m : a.ell < b.ell;
  });
  for (std::size_t i = 1; i < out.size(); ++i) {
    if (out[i].m == out[i - 1].m && out[i].ell == out[i - 1].ell) {
      throw std::invalid_argument(
          "expanded Gaussian modes contain duplicate (ell,m) seeds");
    }
  }
  return out;
}

}  // namespace teuk_b200
