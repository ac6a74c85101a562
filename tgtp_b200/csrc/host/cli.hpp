// Command-line helpers of the drop-in runners (tgtp, benchmark, rw_experiment_saba).
//
// The runners accept and reject exactly the command lines the reference's runners do and print
// the same messages (src/main.cpp:9-31, src/benchmark.cpp:10-28 with src/benchmark_options.h,
// src/rw_experiment_saba.cpp:150-163); the rules are collected here:
//   * a number is what std::stod reads (its own std::invalid_argument / std::out_of_range,
//     message "stod", when the text does not start with a number or overflows), and it must use
//     the whole text and be finite;
//   * a CSV list has no empty item and no trailing comma;
//   * counts are whole numbers in a stated range.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace tgtp_cli {

// The whole of `text` as a finite double; `complaint` is the message when text is left over or
// the value is infinite or NaN.
inline double whole_number(const std::string& text, const std::string& complaint) {
    std::size_t consumed = 0;
    const double x = std::stod(text, &consumed);
    if (consumed != text.size() || !std::isfinite(x)) throw std::invalid_argument(complaint);
    return x;
}

inline bool integral_in(double x, double lo, double hi) {
    return lo <= x && x <= hi && std::floor(x) == x;
}

// Items of a comma-separated list.  An empty item is reported before a trailing comma, which
// is reported like an empty list.
inline std::vector<std::string> csv_items(const std::string& text) {
    if (text.empty()) throw std::invalid_argument("empty CSV list/item");
    std::vector<std::string> items;
    std::size_t from = 0;
    for (;;) {
        const std::size_t comma = text.find(',', from);
        if (comma == std::string::npos) break;
        if (comma == from) throw std::invalid_argument("empty CSV item");
        items.emplace_back(text, from, comma - from);
        from = comma + 1;
    }
    if (from == text.size()) throw std::invalid_argument("empty CSV list/item");
    items.emplace_back(text, from);
    return items;
}

// The benchmark runner's numbers: "invalid number: <text>" and
// "invalid positive integer: <text>" (1 .. INT32_MAX).
inline double bench_number(const std::string& text) {
    return whole_number(text, "invalid number: " + text);
}
inline uint32_t bench_positive(const std::string& text) {
    const double x = bench_number(text);
    if (!integral_in(x, 1, INT32_MAX)) throw std::invalid_argument("invalid positive integer: " + text);
    return static_cast<uint32_t>(x);
}

// A run record printed the reference's way: a results file of "key value" lines and one TSV
// row of the values, both in default ostream formatting (6 significant digits for doubles).
class Record {
  public:
    template <class T>
    Record& add(const char* key, const T& value) {
        std::ostringstream text;
        text << value;
        fields_.emplace_back(key, text.str());
        return *this;
    }
    void write_lines(std::ostream& out) const {
        for (const auto& f : fields_) out << f.first << ' ' << f.second << '\n';
    }
    void write_row(std::ostream& out) const {
        for (std::size_t i = 0; i < fields_.size(); ++i) out << (i ? "\t" : "") << fields_[i].second;
        out << '\n';
    }

  private:
    std::vector<std::pair<std::string, std::string>> fields_;
};

}  // namespace tgtp_cli
