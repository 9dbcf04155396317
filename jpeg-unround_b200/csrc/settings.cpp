// The option namespace of docs/cli.md:182-243: names, ranges and defaults as the
// reference's parser has them (cpp/src/settings.cpp:243-453), each option at most once,
// its value after '=' or as the next argument, the data term's options one value for
// every component or a comma-separated list of one for each. Every refusal is collected
// and reported at once.
#include "settings.hpp"

#include <algorithm>
#include <array>
#include <charconv>
#include <cmath>
#include <limits>
#include <map>
#include <string_view>

namespace urb {

namespace {

constexpr std::array<std::string_view, 36> kValued = {
    "method", "alpha", "alpha1", "alpha0", "channel-weights", "channels", "mu", "mu-scale", "mu-power",
    "mu-chroma", "weight-power", "dc-weight", "centres", "slack", "slack-cost", "flat-weight", "flat-levels",
    "flat-dc", "iterations", "tolerance", "relative-tolerance", "partial-tolerance", "partial-radius",
    "step-ratio", "relaxation", "step-product", "norm-squared", "record-every", "free-radius", "threads",
    "subgradient-iterations", "subgradient-step", "subgradient-decay", "subgradient-record-every",
    "max-pixels", "max-scans"};
constexpr std::array<std::string_view, 3> kFlags = {"no-weight-scaling", "no-momentum", "warnings-are-errors"};

bool contains(const auto& list, std::string_view name) {
  return std::find(list.begin(), list.end(), name) != list.end();
}

std::optional<double> parse_real(std::string_view text) {
  if (text.empty()) return std::nullopt;
  double value = 0.0;
  const char* end = text.data() + text.size();
  auto [stop, error] = std::from_chars(text.data(), end, value);
  if (error != std::errc{} || stop != end) return std::nullopt;
  return value;
}

std::optional<std::uint64_t> parse_whole(std::string_view text) {
  if (text.empty()) return std::nullopt;
  std::uint64_t value = 0;
  const char* end = text.data() + text.size();
  auto [stop, error] = std::from_chars(text.data(), end, value);
  if (error != std::errc{} || stop != end) return std::nullopt;
  return value;
}

bool positive(double x) { return x > 0.0 && std::isfinite(x); }
bool nonnegative(double x) { return x >= 0.0 && std::isfinite(x); }

std::vector<std::string_view> split_commas(std::string_view text) {
  std::vector<std::string_view> items;
  std::size_t start = 0;
  for (;;) {
    const std::size_t comma = text.find(',', start);
    if (comma == std::string_view::npos) {
      items.push_back(text.substr(start));
      return items;
    }
    items.push_back(text.substr(start, comma - start));
    start = comma + 1;
  }
}

// The options as given: name -> value ("" for flags), with the refusals of their syntax.
struct Given {
  std::map<std::string, std::string, std::less<>> values;
  std::vector<std::string> errors;

  explicit Given(const std::vector<std::string>& arguments) {
    for (std::size_t i = 0; i < arguments.size(); ++i) {
      const std::string_view argument = arguments[i];
      if (argument.size() < 2 || argument.substr(0, 2) != "--") {
        errors.push_back(std::string(argument) + " is not an option");
        continue;
      }
      const std::size_t equals = argument.find('=');
      const std::string_view name = argument.substr(2, equals == std::string_view::npos ? std::string_view::npos
                                                                                        : equals - 2);
      if (contains(kFlags, name)) {
        if (equals != std::string_view::npos) errors.push_back("--" + std::string(name) + " takes no value");
        if (!values.emplace(std::string(name), std::string()).second) {
          errors.push_back("--" + std::string(name) + " is given twice");
        }
        continue;
      }
      if (!contains(kValued, name)) {
        errors.push_back("--" + std::string(name) + " is not an option");
        const bool next_is_value = equals == std::string_view::npos && i + 1 < arguments.size() &&
                                   std::string_view(arguments[i + 1]).substr(0, 2) != "--";
        if (next_is_value) ++i;
        continue;
      }
      std::string value;
      if (equals != std::string_view::npos) {
        value = std::string(argument.substr(equals + 1));
      } else if (i + 1 < arguments.size()) {
        value = arguments[++i];
      } else {
        errors.push_back("--" + std::string(name) + " needs a value");
        continue;
      }
      if (!values.emplace(std::string(name), value).second) {
        errors.push_back("--" + std::string(name) + " is given twice");
      }
    }
  }

  [[nodiscard]] const std::string* find(std::string_view name) const {
    auto it = values.find(name);
    return it == values.end() ? nullptr : &it->second;
  }
  [[nodiscard]] bool flag(std::string_view name) const { return find(name) != nullptr; }

  void refuse(std::string_view name, std::string_view range, std::string_view value) {
    errors.push_back("--" + std::string(name) + " is " + std::string(range) + ", not " + std::string(value));
  }

  template <typename Check>
  std::optional<double> real(std::string_view name, Check check, std::string_view range) {
    const std::string* text = find(name);
    if (text == nullptr) return std::nullopt;
    auto value = parse_real(*text);
    if (!value || !check(*value)) {
      refuse(name, range, *text);
      return std::nullopt;
    }
    return value;
  }

  std::optional<std::uint64_t> whole(std::string_view name, std::uint64_t least, std::uint64_t most,
                                     std::string_view range) {
    const std::string* text = find(name);
    if (text == nullptr) return std::nullopt;
    auto value = parse_whole(*text);
    if (!value || *value < least || *value > most) {
      refuse(name, range, *text);
      return std::nullopt;
    }
    return value;
  }

  // A list of one value for every component or one for each; each item read by `read`.
  template <typename T, typename Read>
  std::optional<std::vector<T>> list(std::string_view name, Read read, std::string_view range) {
    const std::string* text = find(name);
    if (text == nullptr) return std::nullopt;
    std::vector<T> items;
    for (std::string_view item : split_commas(*text)) {
      std::optional<T> value = read(item);
      if (!value) {
        refuse(name, range, item);
        return std::nullopt;
      }
      items.push_back(*value);
    }
    return items;
  }
};

std::optional<double> nonnegative_item(std::string_view item) {
  auto value = parse_real(item);
  return value && nonnegative(*value) ? value : std::nullopt;
}

}  // namespace

std::string shortest(double value) {
  char buffer[64];
  auto [end, error] = std::to_chars(buffer, buffer + sizeof(buffer), value);
  if (error != std::errc{}) return "nan";
  return std::string(buffer, end);
}

bool parse_settings(const std::vector<std::string>& arguments, Settings& out, std::string& errors) {
  Given given(arguments);
  Settings s;
  if (const std::string* method = given.find("method")) {
    if (*method == "mmse") s.method = Method::mmse;
    else if (*method == "tv") s.method = Method::tv;
    else if (*method == "tgv") s.method = Method::tgv;
    else if (*method == "subgradient") s.method = Method::subgradient;
    else given.errors.push_back("--method is one of mmse, tv, tgv, subgradient, not " + *method);
  }
  constexpr std::string_view above_zero = "above 0 and finite";
  constexpr std::string_view from_zero = "at least 0 and finite";
  if (auto v = given.real("alpha", positive, above_zero)) s.regularizer.alpha = *v;
  if (auto v = given.real("alpha1", positive, above_zero)) s.regularizer.alpha1 = *v;
  if (auto v = given.real("alpha0", positive, above_zero)) s.regularizer.alpha0 = *v;
  if (auto v = given.list<double>(
          "channel-weights",
          [](std::string_view item) -> std::optional<double> {
            auto value = parse_real(item);
            return value && positive(*value) ? value : std::nullopt;
          },
          "a list of numbers above 0 and finite")) {
    s.regularizer.channel_weights = *v;
  }
  if (const std::string* channels = given.find("channels")) {
    if (*channels == "coupled") s.regularizer.coupled = true;
    else if (*channels == "apart") s.regularizer.coupled = false;
    else given.errors.push_back("--channels is one of coupled, apart, not " + *channels);
  }

  auto mu = given.list<std::optional<double>>(
      "mu",
      [](std::string_view item) -> std::optional<std::optional<double>> {
        if (item == "rule") return std::optional<double>{};
        auto value = nonnegative_item(item);
        if (!value) return std::nullopt;
        return std::optional<double>{*value};
      },
      "at least 0 and finite, or rule");
  auto mu_scale = given.list<double>("mu-scale", nonnegative_item, from_zero);
  auto mu_power = given.list<double>(
      "mu-power",
      [](std::string_view item) -> std::optional<double> {
        auto value = parse_real(item);
        return value && std::isfinite(*value) ? value : std::nullopt;
      },
      "finite");
  auto mu_chroma = given.list<double>("mu-chroma", nonnegative_item, from_zero);
  auto power = given.list<double>("weight-power", nonnegative_item, from_zero);
  auto dc_weight = given.list<double>("dc-weight", nonnegative_item, from_zero);
  auto centres = given.list<Centres>(
      "centres",
      [](std::string_view item) -> std::optional<Centres> {
        if (item == "mmse") return Centres::mmse;
        if (item == "midpoint") return Centres::midpoint;
        return std::nullopt;
      },
      "mmse or midpoint");
  auto slack = given.list<double>("slack", nonnegative_item, from_zero);
  auto slack_cost = given.list<double>("slack-cost", nonnegative_item, from_zero);
  auto flat_weight = given.list<double>("flat-weight", nonnegative_item, from_zero);
  auto flat_levels = given.list<std::uint32_t>(
      "flat-levels",
      [](std::string_view item) -> std::optional<std::uint32_t> {
        auto value = parse_whole(item);
        if (!value || *value > 63) return std::nullopt;
        return static_cast<std::uint32_t>(*value);
      },
      "an integer from 0 to 63");
  auto flat_dc = given.list<std::optional<std::uint32_t>>(
      "flat-dc",
      [](std::string_view item) -> std::optional<std::optional<std::uint32_t>> {
        if (item == "any") return std::optional<std::uint32_t>{};
        auto value = parse_whole(item);
        if (!value || *value > std::numeric_limits<std::uint32_t>::max()) return std::nullopt;
        return std::optional<std::uint32_t>{static_cast<std::uint32_t>(*value)};
      },
      "a whole number or any");
  // The lists' length: 1, or one length common to every list longer than 1.
  std::size_t count = 1;
  const std::array<std::pair<std::string_view, std::size_t>, 12> lengths = {{
      {"mu", mu ? mu->size() : 1}, {"mu-scale", mu_scale ? mu_scale->size() : 1},
      {"mu-power", mu_power ? mu_power->size() : 1}, {"mu-chroma", mu_chroma ? mu_chroma->size() : 1},
      {"weight-power", power ? power->size() : 1}, {"dc-weight", dc_weight ? dc_weight->size() : 1},
      {"centres", centres ? centres->size() : 1}, {"slack", slack ? slack->size() : 1},
      {"slack-cost", slack_cost ? slack_cost->size() : 1}, {"flat-weight", flat_weight ? flat_weight->size() : 1},
      {"flat-levels", flat_levels ? flat_levels->size() : 1}, {"flat-dc", flat_dc ? flat_dc->size() : 1},
  }};
  for (const auto& [name, length] : lengths) {
    if (length == 1) continue;
    if (count == 1) {
      count = length;
    } else if (length != count) {
      given.errors.push_back(
          "the options of the data term give one value for every component or one for each, not " +
          std::to_string(length) + " for --" + std::string(name));
    }
  }
  s.data.assign(count, DataTerm{});
  auto pick = [](const auto& values, std::size_t index, auto& into) {
    if (values) into = (*values)[values->size() == 1 ? 0 : index];
  };
  for (std::size_t c = 0; c < count; ++c) {
    DataTerm& term = s.data[c];
    pick(mu, c, term.mu);
    pick(mu_scale, c, term.mu_scale);
    pick(mu_power, c, term.mu_power);
    pick(mu_chroma, c, term.mu_chroma);
    pick(power, c, term.power);
    pick(dc_weight, c, term.dc_weight);
    pick(centres, c, term.centres);
    pick(slack, c, term.slack);
    pick(slack_cost, c, term.slack_cost);
    pick(flat_weight, c, term.flat_weight);
    pick(flat_levels, c, term.flat_levels);
    pick(flat_dc, c, term.flat_dc);
  }

  constexpr std::uint64_t unbounded = std::numeric_limits<std::uint64_t>::max();
  PdhgOptions& pdhg = s.pdhg;
  if (auto v = given.whole("iterations", 0, unbounded, "a whole number")) pdhg.iterations = *v;
  if (auto v = given.real("tolerance", nonnegative, from_zero)) pdhg.tolerance = *v;
  if (auto v = given.real("relative-tolerance", nonnegative, from_zero)) pdhg.relative_tolerance = *v;
  if (auto v = given.real("partial-tolerance", nonnegative, from_zero)) pdhg.partial_tolerance = *v;
  if (auto v = given.real("partial-radius", nonnegative, from_zero)) pdhg.partial_radius = *v;
  if (auto v = given.real("step-ratio", positive, above_zero)) pdhg.step_ratio = *v;
  if (auto v = given.real("relaxation", [](double x) { return x > 0.0 && x < 2.0; }, "between 0 and 2")) {
    pdhg.relaxation = *v;
  }
  if (auto v = given.real("step-product", [](double x) { return x > 0.0 && x < 1.0; }, "between 0 and 1")) {
    pdhg.step_product = *v;
  }
  if (auto v = given.real("norm-squared", positive, above_zero)) pdhg.norm_squared = *v;
  pdhg.weight_scaling = !given.flag("no-weight-scaling");
  if (auto v = given.whole("record-every", 0, unbounded, "a whole number")) pdhg.record_every = *v;
  if (auto v = given.real("free-radius", nonnegative, from_zero)) pdhg.free_radius = *v;
  if (auto v = given.whole("threads", 0, unbounded, "a whole number")) pdhg.threads = *v;

  if (auto v = given.whole("subgradient-iterations", 0, unbounded, "a whole number")) s.subgradient.iterations = *v;
  if (auto v = given.real("subgradient-step", positive, above_zero)) s.subgradient.step = *v;
  if (auto v = given.real("subgradient-decay", nonnegative, from_zero)) s.subgradient.decay = *v;
  s.subgradient.momentum = !given.flag("no-momentum");
  if (auto v = given.whole("subgradient-record-every", 0, unbounded, "a whole number")) {
    s.subgradient.record_every = *v;
  }
  if (auto v = given.whole("max-pixels", 1, unbounded, "a whole number of at least 1")) s.reading.max_pixels = *v;
  constexpr auto most_scans = static_cast<std::uint64_t>(std::numeric_limits<std::int32_t>::max());
  if (auto v = given.whole("max-scans", 1, most_scans, "a whole number of at least 1")) {
    s.reading.max_scans = static_cast<std::int32_t>(*v);
  }
  s.reading.warnings_are_errors = given.flag("warnings-are-errors");

  if (s.method == Method::tv && (pdhg.partial_radius || pdhg.partial_tolerance > 0.0)) {
    given.errors.push_back("the partial gap is TGV's alone, not TV's");
  }
  if (pdhg.partial_tolerance > 0.0 && !pdhg.partial_radius) {
    given.errors.push_back("--partial-tolerance needs --partial-radius");
  }
  if (!given.errors.empty()) {
    errors.clear();
    for (const std::string& e : given.errors) errors += (errors.empty() ? "" : "; ") + e;
    return false;
  }
  out = std::move(s);
  return true;
}

namespace {

template <typename Text>
std::string joined(const std::vector<DataTerm>& data, Text text) {
  const std::string first = text(data.front());
  bool alike = true;
  for (const DataTerm& term : data) alike = alike && text(term) == first;
  if (alike) return first;
  std::string all;
  for (const DataTerm& term : data) all += (all.empty() ? "" : ",") + text(term);
  return all;
}

}  // namespace

std::vector<std::string> options_of(const Settings& s) {
  std::vector<std::string> o;
  auto add = [&o](std::string_view name, const std::string& value) {
    o.push_back("--" + std::string(name) + "=" + value);
  };
  constexpr std::array<const char*, 4> methods = {"mmse", "tv", "tgv", "subgradient"};
  add("method", methods[static_cast<std::size_t>(s.method)]);
  add("alpha", shortest(s.regularizer.alpha));
  add("alpha1", shortest(s.regularizer.alpha1));
  add("alpha0", shortest(s.regularizer.alpha0));
  if (!s.regularizer.channel_weights.empty()) {
    std::string weights;
    for (double w : s.regularizer.channel_weights) weights += (weights.empty() ? "" : ",") + shortest(w);
    add("channel-weights", weights);
  }
  add("channels", s.regularizer.coupled ? "coupled" : "apart");
  const auto& d = s.data;
  add("mu", joined(d, [](const DataTerm& t) { return t.mu ? shortest(*t.mu) : std::string("rule"); }));
  add("mu-scale", joined(d, [](const DataTerm& t) { return shortest(t.mu_scale); }));
  add("mu-power", joined(d, [](const DataTerm& t) { return shortest(t.mu_power); }));
  add("mu-chroma", joined(d, [](const DataTerm& t) { return shortest(t.mu_chroma); }));
  add("weight-power", joined(d, [](const DataTerm& t) { return shortest(t.power); }));
  add("dc-weight", joined(d, [](const DataTerm& t) { return shortest(t.dc_weight); }));
  add("centres", joined(d, [](const DataTerm& t) {
        return std::string(t.centres == Centres::mmse ? "mmse" : "midpoint");
      }));
  add("slack", joined(d, [](const DataTerm& t) { return shortest(t.slack); }));
  add("slack-cost", joined(d, [](const DataTerm& t) { return shortest(t.slack_cost); }));
  add("flat-weight", joined(d, [](const DataTerm& t) { return shortest(t.flat_weight); }));
  add("flat-levels", joined(d, [](const DataTerm& t) { return std::to_string(t.flat_levels); }));
  add("flat-dc", joined(d, [](const DataTerm& t) {
        return t.flat_dc ? std::to_string(*t.flat_dc) : std::string("any");
      }));
  const PdhgOptions& p = s.pdhg;
  if (p.iterations) add("iterations", std::to_string(*p.iterations));
  if (p.tolerance) add("tolerance", shortest(*p.tolerance));
  add("relative-tolerance", shortest(p.relative_tolerance));
  add("partial-tolerance", shortest(p.partial_tolerance));
  if (p.partial_radius) add("partial-radius", shortest(*p.partial_radius));
  if (p.step_ratio) add("step-ratio", shortest(*p.step_ratio));
  add("relaxation", shortest(p.relaxation));
  add("step-product", shortest(p.step_product));
  if (p.norm_squared) add("norm-squared", shortest(*p.norm_squared));
  if (!p.weight_scaling) o.emplace_back("--no-weight-scaling");
  add("record-every", std::to_string(p.record_every));
  add("free-radius", shortest(p.free_radius));
  add("threads", std::to_string(p.threads));
  add("subgradient-iterations", std::to_string(s.subgradient.iterations));
  add("subgradient-step", shortest(s.subgradient.step));
  add("subgradient-decay", shortest(s.subgradient.decay));
  if (!s.subgradient.momentum) o.emplace_back("--no-momentum");
  add("subgradient-record-every", std::to_string(s.subgradient.record_every));
  add("max-pixels", std::to_string(s.reading.max_pixels));
  add("max-scans", std::to_string(s.reading.max_scans));
  if (s.reading.warnings_are_errors) o.emplace_back("--warnings-are-errors");
  return o;
}

}  // namespace urb
