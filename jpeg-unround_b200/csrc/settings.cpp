// The option namespace of the reference's command line (docs/cli.md:182-243 of
// JPEG-Unround), read by one table. Each row names an option, the set of values it accepts
// (its domain, which also gives the wording of a refusal) and its scope: one value, a list
// (the channel weights), or the data term's "one value for every component or a
// comma-separated list of one for each". Reading goes in three passes: the arguments into
// (option, text) pairs, each text into values through its row's domain, then the values
// into a Settings. Every refusal is collected and reported at once, joined by "; ".
//
// Kept as the reference has them, because the same strings must give the same settings
// and a caller matches on the refusals: the names, the domains, the defaults (settings.hpp)
// and the wording of each message.
#include "settings.hpp"

#include <algorithm>
#include <array>
#include <charconv>
#include <cmath>
#include <limits>
#include <span>
#include <string_view>

namespace urb {

namespace {

enum class Domain : std::uint8_t {
  flag,                 // no value
  positive,             // a real above 0, finite
  nonnegative,          // a real at least 0, finite
  finite,               // any finite real
  open_unit,            // a real in (0, 1)
  open_two,             // a real in (0, 2)
  whole,                // a whole number
  whole_from_one,       // a whole number of at least 1
  scans,                // a whole number from 1 to the largest int32
  level,                // a whole number from 0 to 63
  whole_or_any,         // a whole number that fits 32 bits, or "any"
  nonnegative_or_rule,  // a real at least 0, or "rule"
  choice,               // one of the row's words
};

enum class Scope : std::uint8_t { single, list, per_component };

enum class Id : std::uint8_t {
  method, alpha, alpha1, alpha0, channel_weights, channels,
  mu, mu_scale, mu_power, mu_chroma, weight_power, dc_weight, centres, slack, slack_cost,
  flat_weight, flat_levels, flat_dc,
  iterations, tolerance, relative_tolerance, partial_tolerance, partial_radius, step_ratio,
  relaxation, step_product, norm_squared, no_weight_scaling, record_every, free_radius, threads,
  subgradient_iterations, subgradient_step, subgradient_decay, no_momentum, subgradient_record_every,
  max_pixels, max_scans, warnings_are_errors,
};

constexpr std::array<std::string_view, 4> kMethods = {"mmse", "tv", "tgv", "subgradient"};
constexpr std::array<std::string_view, 2> kCouplings = {"coupled", "apart"};
constexpr std::array<std::string_view, 2> kCentres = {"mmse", "midpoint"};

struct Row {
  Id id;
  std::string_view name;
  Domain domain;
  Scope scope;
  std::string_view range;  // what a refusal says the option is
  std::span<const std::string_view> words = {};
};

constexpr std::string_view kAboveZero = "above 0 and finite";
constexpr std::string_view kFromZero = "at least 0 and finite";
constexpr std::string_view kWhole = "a whole number";

// In the order of the reference's documentation, which is also the order of the refusals
// and of the options that give settings back.
constexpr Row kRows[] = {
    {Id::method, "method", Domain::choice, Scope::single, "one of mmse, tv, tgv, subgradient", kMethods},
    {Id::alpha, "alpha", Domain::positive, Scope::single, kAboveZero},
    {Id::alpha1, "alpha1", Domain::positive, Scope::single, kAboveZero},
    {Id::alpha0, "alpha0", Domain::positive, Scope::single, kAboveZero},
    {Id::channel_weights, "channel-weights", Domain::positive, Scope::list, "a list of numbers above 0 and finite"},
    {Id::channels, "channels", Domain::choice, Scope::single, "one of coupled, apart", kCouplings},
    {Id::mu, "mu", Domain::nonnegative_or_rule, Scope::per_component, "at least 0 and finite, or rule"},
    {Id::mu_scale, "mu-scale", Domain::nonnegative, Scope::per_component, kFromZero},
    {Id::mu_power, "mu-power", Domain::finite, Scope::per_component, "finite"},
    {Id::mu_chroma, "mu-chroma", Domain::nonnegative, Scope::per_component, kFromZero},
    {Id::weight_power, "weight-power", Domain::nonnegative, Scope::per_component, kFromZero},
    {Id::dc_weight, "dc-weight", Domain::nonnegative, Scope::per_component, kFromZero},
    {Id::centres, "centres", Domain::choice, Scope::per_component, "mmse or midpoint", kCentres},
    {Id::slack, "slack", Domain::nonnegative, Scope::per_component, kFromZero},
    {Id::slack_cost, "slack-cost", Domain::nonnegative, Scope::per_component, kFromZero},
    {Id::flat_weight, "flat-weight", Domain::nonnegative, Scope::per_component, kFromZero},
    {Id::flat_levels, "flat-levels", Domain::level, Scope::per_component, "an integer from 0 to 63"},
    {Id::flat_dc, "flat-dc", Domain::whole_or_any, Scope::per_component, "a whole number or any"},
    {Id::iterations, "iterations", Domain::whole, Scope::single, kWhole},
    {Id::tolerance, "tolerance", Domain::nonnegative, Scope::single, kFromZero},
    {Id::relative_tolerance, "relative-tolerance", Domain::nonnegative, Scope::single, kFromZero},
    {Id::partial_tolerance, "partial-tolerance", Domain::nonnegative, Scope::single, kFromZero},
    {Id::partial_radius, "partial-radius", Domain::nonnegative, Scope::single, kFromZero},
    {Id::step_ratio, "step-ratio", Domain::positive, Scope::single, kAboveZero},
    {Id::relaxation, "relaxation", Domain::open_two, Scope::single, "between 0 and 2"},
    {Id::step_product, "step-product", Domain::open_unit, Scope::single, "between 0 and 1"},
    {Id::norm_squared, "norm-squared", Domain::positive, Scope::single, kAboveZero},
    {Id::no_weight_scaling, "no-weight-scaling", Domain::flag, Scope::single, ""},
    {Id::record_every, "record-every", Domain::whole, Scope::single, kWhole},
    {Id::free_radius, "free-radius", Domain::nonnegative, Scope::single, kFromZero},
    {Id::threads, "threads", Domain::whole, Scope::single, kWhole},
    {Id::subgradient_iterations, "subgradient-iterations", Domain::whole, Scope::single, kWhole},
    {Id::subgradient_step, "subgradient-step", Domain::positive, Scope::single, kAboveZero},
    {Id::subgradient_decay, "subgradient-decay", Domain::nonnegative, Scope::single, kFromZero},
    {Id::no_momentum, "no-momentum", Domain::flag, Scope::single, ""},
    {Id::subgradient_record_every, "subgradient-record-every", Domain::whole, Scope::single, kWhole},
    {Id::max_pixels, "max-pixels", Domain::whole_from_one, Scope::single, "a whole number of at least 1"},
    {Id::max_scans, "max-scans", Domain::scans, Scope::single, "a whole number of at least 1"},
    {Id::warnings_are_errors, "warnings-are-errors", Domain::flag, Scope::single, ""},
};
constexpr std::size_t kRowCount = std::size(kRows);

const Row* row_named(std::string_view name) {
  for (const Row& row : kRows) {
    if (row.name == name) return &row;
  }
  return nullptr;
}

std::size_t index_of(const Row& row) { return static_cast<std::size_t>(&row - kRows); }

// One value of an option. `keyword` marks "rule" (mu) and "any" (flat-dc), which the
// settings hold as an empty optional; `word` is the index of a choice.
struct Value {
  double real = 0.0;
  std::uint64_t count = 0;
  bool keyword = false;
  std::size_t word = 0;
};

template <typename T>
std::optional<T> number_of(std::string_view text) {
  T value{};
  const char* end = text.data() + text.size();
  const auto [stop, error] = std::from_chars(text.data(), end, value);
  if (text.empty() || error != std::errc{} || stop != end) return std::nullopt;
  return value;
}

// A text read through a domain: the value, or none where the domain refuses it.
std::optional<Value> read(const Row& row, std::string_view text) {
  Value value;
  auto real_within = [&](auto accepts) -> std::optional<Value> {
    const auto x = number_of<double>(text);
    if (!x || !accepts(*x)) return std::nullopt;
    value.real = *x;
    return value;
  };
  auto whole_within = [&](std::uint64_t least, std::uint64_t most) -> std::optional<Value> {
    const auto n = number_of<std::uint64_t>(text);
    if (!n || *n < least || *n > most) return std::nullopt;
    value.count = *n;
    return value;
  };
  constexpr std::uint64_t unbounded = std::numeric_limits<std::uint64_t>::max();
  switch (row.domain) {
    case Domain::flag: return value;
    case Domain::positive: return real_within([](double x) { return x > 0.0 && std::isfinite(x); });
    case Domain::nonnegative: return real_within([](double x) { return x >= 0.0 && std::isfinite(x); });
    case Domain::finite: return real_within([](double x) { return std::isfinite(x); });
    case Domain::open_unit: return real_within([](double x) { return x > 0.0 && x < 1.0; });
    case Domain::open_two: return real_within([](double x) { return x > 0.0 && x < 2.0; });
    case Domain::whole: return whole_within(0, unbounded);
    case Domain::whole_from_one: return whole_within(1, unbounded);
    case Domain::scans: return whole_within(1, static_cast<std::uint64_t>(std::numeric_limits<std::int32_t>::max()));
    case Domain::level: return whole_within(0, 63);
    case Domain::whole_or_any:
      if (text == "any") {
        value.keyword = true;
        return value;
      }
      return whole_within(0, std::numeric_limits<std::uint32_t>::max());
    case Domain::nonnegative_or_rule:
      if (text == "rule") {
        value.keyword = true;
        return value;
      }
      return real_within([](double x) { return x >= 0.0 && std::isfinite(x); });
    case Domain::choice: {
      const auto found = std::find(row.words.begin(), row.words.end(), text);
      if (found == row.words.end()) return std::nullopt;
      value.word = static_cast<std::size_t>(found - row.words.begin());
      return value;
    }
  }
  return std::nullopt;
}

// Pass 1: the arguments as (row, text) pairs, at most one a row.
struct Given {
  std::array<std::optional<std::string>, kRowCount> text;
  std::vector<std::string> errors;

  explicit Given(const std::vector<std::string>& arguments) {
    for (std::size_t i = 0; i < arguments.size(); ++i) {
      const std::string_view argument = arguments[i];
      if (!argument.starts_with("--")) {
        errors.push_back(std::string(argument) + " is not an option");
        continue;
      }
      const std::string_view body = argument.substr(2);
      const std::size_t equals = body.find('=');
      const std::string_view name = body.substr(0, equals);
      const bool inline_value = equals != std::string_view::npos;
      const Row* row = row_named(name);
      if (row == nullptr) {
        errors.push_back("--" + std::string(name) + " is not an option");
        // An unknown option's value, if it has one, is not read as an argument of its own.
        if (!inline_value && i + 1 < arguments.size() && !std::string_view(arguments[i + 1]).starts_with("--")) ++i;
        continue;
      }
      std::string value;
      if (row->domain == Domain::flag) {
        if (inline_value) errors.push_back("--" + std::string(name) + " takes no value");
      } else if (inline_value) {
        value = std::string(body.substr(equals + 1));
      } else if (i + 1 < arguments.size()) {
        value = arguments[++i];
      } else {
        errors.push_back("--" + std::string(name) + " needs a value");
        continue;
      }
      std::optional<std::string>& slot = text[index_of(*row)];
      if (slot) {
        errors.push_back("--" + std::string(name) + " is given twice");
      } else {
        slot = std::move(value);
      }
    }
  }
};

// The items of a list: the text cut at every comma.
std::vector<std::string_view> items_of(std::string_view text) {
  std::vector<std::string_view> items;
  for (std::size_t start = 0;;) {
    const std::size_t comma = text.find(',', start);
    items.push_back(text.substr(start, comma == std::string_view::npos ? comma : comma - start));
    if (comma == std::string_view::npos) return items;
    start = comma + 1;
  }
}

// One option's value into the settings, or, for the data term, into one component's term.
void store(Id id, const Value& v, Settings& s, DataTerm& term) {
  switch (id) {
    case Id::method: s.method = static_cast<Method>(v.word); break;
    case Id::alpha: s.regularizer.alpha = v.real; break;
    case Id::alpha1: s.regularizer.alpha1 = v.real; break;
    case Id::alpha0: s.regularizer.alpha0 = v.real; break;
    case Id::channel_weights: s.regularizer.channel_weights.push_back(v.real); break;
    case Id::channels: s.regularizer.coupled = v.word == 0; break;
    case Id::mu: term.mu = v.keyword ? std::optional<double>{} : std::optional<double>{v.real}; break;
    case Id::mu_scale: term.mu_scale = v.real; break;
    case Id::mu_power: term.mu_power = v.real; break;
    case Id::mu_chroma: term.mu_chroma = v.real; break;
    case Id::weight_power: term.power = v.real; break;
    case Id::dc_weight: term.dc_weight = v.real; break;
    case Id::centres: term.centres = v.word == 0 ? Centres::mmse : Centres::midpoint; break;
    case Id::slack: term.slack = v.real; break;
    case Id::slack_cost: term.slack_cost = v.real; break;
    case Id::flat_weight: term.flat_weight = v.real; break;
    case Id::flat_levels: term.flat_levels = static_cast<std::uint32_t>(v.count); break;
    case Id::flat_dc:
      term.flat_dc = v.keyword ? std::optional<std::uint32_t>{} : std::optional<std::uint32_t>{static_cast<std::uint32_t>(v.count)};
      break;
    case Id::iterations: s.pdhg.iterations = v.count; break;
    case Id::tolerance: s.pdhg.tolerance = v.real; break;
    case Id::relative_tolerance: s.pdhg.relative_tolerance = v.real; break;
    case Id::partial_tolerance: s.pdhg.partial_tolerance = v.real; break;
    case Id::partial_radius: s.pdhg.partial_radius = v.real; break;
    case Id::step_ratio: s.pdhg.step_ratio = v.real; break;
    case Id::relaxation: s.pdhg.relaxation = v.real; break;
    case Id::step_product: s.pdhg.step_product = v.real; break;
    case Id::norm_squared: s.pdhg.norm_squared = v.real; break;
    case Id::no_weight_scaling: s.pdhg.weight_scaling = false; break;
    case Id::record_every: s.pdhg.record_every = v.count; break;
    case Id::free_radius: s.pdhg.free_radius = v.real; break;
    case Id::threads: s.pdhg.threads = v.count; break;
    case Id::subgradient_iterations: s.subgradient.iterations = v.count; break;
    case Id::subgradient_step: s.subgradient.step = v.real; break;
    case Id::subgradient_decay: s.subgradient.decay = v.real; break;
    case Id::no_momentum: s.subgradient.momentum = false; break;
    case Id::subgradient_record_every: s.subgradient.record_every = v.count; break;
    case Id::max_pixels: s.reading.max_pixels = v.count; break;
    case Id::max_scans: s.reading.max_scans = static_cast<std::int32_t>(v.count); break;
    case Id::warnings_are_errors: s.reading.warnings_are_errors = true; break;
  }
}

// One component's value of a data-term option as an option gives it back.
std::string text_of(Id id, const DataTerm& t) {
  switch (id) {
    case Id::mu: return t.mu ? shortest(*t.mu) : std::string("rule");
    case Id::mu_scale: return shortest(t.mu_scale);
    case Id::mu_power: return shortest(t.mu_power);
    case Id::mu_chroma: return shortest(t.mu_chroma);
    case Id::weight_power: return shortest(t.power);
    case Id::dc_weight: return shortest(t.dc_weight);
    case Id::centres: return std::string(kCentres[t.centres == Centres::mmse ? 0 : 1]);
    case Id::slack: return shortest(t.slack);
    case Id::slack_cost: return shortest(t.slack_cost);
    case Id::flat_weight: return shortest(t.flat_weight);
    case Id::flat_levels: return std::to_string(t.flat_levels);
    case Id::flat_dc: return t.flat_dc ? std::to_string(*t.flat_dc) : std::string("any");
    default: return {};
  }
}

// Any other option's value as an option gives it back; none where the settings hold none
// (an unset optional, an empty list, a flag that is off).
std::optional<std::string> text_of(Id id, const Settings& s) {
  const PdhgOptions& p = s.pdhg;
  auto maybe = [](const auto& value) -> std::optional<std::string> {
    if (!value) return std::nullopt;
    if constexpr (std::is_floating_point_v<std::decay_t<decltype(*value)>>) return shortest(*value);
    else return std::to_string(*value);
  };
  switch (id) {
    case Id::method: return std::string(kMethods[static_cast<std::size_t>(s.method)]);
    case Id::alpha: return shortest(s.regularizer.alpha);
    case Id::alpha1: return shortest(s.regularizer.alpha1);
    case Id::alpha0: return shortest(s.regularizer.alpha0);
    case Id::channel_weights: {
      if (s.regularizer.channel_weights.empty()) return std::nullopt;
      std::string all;
      for (double w : s.regularizer.channel_weights) all += (all.empty() ? "" : ",") + shortest(w);
      return all;
    }
    case Id::channels: return std::string(kCouplings[s.regularizer.coupled ? 0 : 1]);
    case Id::iterations: return maybe(p.iterations);
    case Id::tolerance: return maybe(p.tolerance);
    case Id::relative_tolerance: return shortest(p.relative_tolerance);
    case Id::partial_tolerance: return shortest(p.partial_tolerance);
    case Id::partial_radius: return maybe(p.partial_radius);
    case Id::step_ratio: return maybe(p.step_ratio);
    case Id::relaxation: return shortest(p.relaxation);
    case Id::step_product: return shortest(p.step_product);
    case Id::norm_squared: return maybe(p.norm_squared);
    case Id::record_every: return std::to_string(p.record_every);
    case Id::free_radius: return shortest(p.free_radius);
    case Id::threads: return std::to_string(p.threads);
    case Id::subgradient_iterations: return std::to_string(s.subgradient.iterations);
    case Id::subgradient_step: return shortest(s.subgradient.step);
    case Id::subgradient_decay: return shortest(s.subgradient.decay);
    case Id::subgradient_record_every: return std::to_string(s.subgradient.record_every);
    case Id::max_pixels: return std::to_string(s.reading.max_pixels);
    case Id::max_scans: return std::to_string(s.reading.max_scans);
    case Id::no_weight_scaling: return p.weight_scaling ? std::nullopt : std::optional<std::string>("");
    case Id::no_momentum: return s.subgradient.momentum ? std::nullopt : std::optional<std::string>("");
    case Id::warnings_are_errors: return s.reading.warnings_are_errors ? std::optional<std::string>("") : std::nullopt;
    default: return std::nullopt;
  }
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
  std::vector<std::string>& refusals = given.errors;

  // Pass 2: every given text into values, row by row.
  std::array<std::optional<std::vector<Value>>, kRowCount> values;
  for (const Row& row : kRows) {
    const std::optional<std::string>& text = given.text[index_of(row)];
    if (!text) continue;
    std::vector<Value> read_values;
    const std::vector<std::string_view> items =
        row.scope == Scope::single ? std::vector<std::string_view>{*text} : items_of(*text);
    bool refused = false;
    for (std::string_view item : items) {
      std::optional<Value> value = read(row, item);
      if (!value) {
        refusals.push_back("--" + std::string(row.name) + " is " + std::string(row.range) + ", not " + std::string(item));
        refused = true;
        break;
      }
      read_values.push_back(*value);
    }
    if (!refused) values[index_of(row)] = std::move(read_values);
  }

  // The data term's count: 1, or the one length of every list longer than 1.
  std::size_t count = 1;
  for (const Row& row : kRows) {
    const auto& list = values[index_of(row)];
    if (row.scope != Scope::per_component || !list || list->size() == 1) continue;
    if (count == 1) {
      count = list->size();
    } else if (list->size() != count) {
      refusals.push_back("the options of the data term give one value for every component or one for each, not " +
                         std::to_string(list->size()) + " for --" + std::string(row.name));
    }
  }

  // Pass 3: the values into settings.
  Settings s;
  s.data.assign(count, DataTerm{});
  for (const Row& row : kRows) {
    const auto& list = values[index_of(row)];
    if (!list) continue;
    if (row.scope == Scope::per_component) {
      for (std::size_t c = 0; c < count; ++c) store(row.id, (*list)[list->size() == 1 ? 0 : c], s, s.data[c]);
    } else {
      for (const Value& value : *list) store(row.id, value, s, s.data.front());
    }
  }

  if (s.method == Method::tv && (s.pdhg.partial_radius || s.pdhg.partial_tolerance > 0.0)) {
    refusals.emplace_back("the partial gap is TGV's alone, not TV's");
  }
  if (s.pdhg.partial_tolerance > 0.0 && !s.pdhg.partial_radius) {
    refusals.emplace_back("--partial-tolerance needs --partial-radius");
  }
  if (!refusals.empty()) {
    errors.clear();
    for (const std::string& refusal : refusals) errors += (errors.empty() ? "" : "; ") + refusal;
    return false;
  }
  out = std::move(s);
  return true;
}

std::vector<std::string> options_of(const Settings& s) {
  std::vector<std::string> options;
  for (const Row& row : kRows) {
    std::optional<std::string> text;
    if (row.scope == Scope::per_component) {
      // One value where every component's is alike, else one for each.
      std::string all;
      bool alike = true;
      const std::string first = text_of(row.id, s.data.front());
      for (const DataTerm& term : s.data) {
        const std::string one = text_of(row.id, term);
        alike = alike && one == first;
        all += (all.empty() ? "" : ",") + one;
      }
      text = alike ? first : all;
    } else {
      text = text_of(row.id, s);
    }
    if (!text) continue;
    if (row.domain == Domain::flag) {
      options.push_back("--" + std::string(row.name));
    } else {
      options.push_back("--" + std::string(row.name) + "=" + *text);
    }
  }
  return options;
}

}  // namespace urb
