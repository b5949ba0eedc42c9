// icp_cli_options.hpp -- table-driven option parsing for the command-line drop-ins.
//
// Each CLI lists its flags once, as a table of (number of values, handler).  What differs
// between the reference's CLIs -- whether a repeated flag is an error, whether an unknown
// flag is assumed to carry a value, how the errors are worded -- is a Style, so every drop-in
// keeps its reference's exit behaviour and messages.
#pragma once
#include <functional>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

namespace icp::cli {

using Values = std::vector<std::string_view>;

struct Flag {
    unsigned arity;                          // values following the flag
    std::function<void(const Values&)> set;  // receives exactly `arity` values
    bool stops = false;                      // parsing ends after this flag (e.g. --help)
};
using Table = std::map<std::string, Flag, std::less<>>;

struct Style {
    bool unique;              // a repeated flag is an error
    bool unknown_has_value;   // an unknown flag is assumed to carry one value (checked first)
    std::function<std::string(const std::string&)> repeated, missing;
};

// Applies argv[1..] to the table and returns the flags seen; std::invalid_argument on a
// repeated (Style::unique), valueless or unknown flag.  Stops after a Flag::stops flag.
inline std::set<std::string> apply(int argc, char** argv, const Table& table, const Style& style)
{
    std::set<std::string> seen;
    int i = 1;
    while (i < argc) {
        const std::string flag = argv[i++];
        if (!seen.insert(flag).second && style.unique) throw std::invalid_argument(style.repeated(flag));
        const auto it = table.find(flag);
        const unsigned want = it != table.end() ? it->second.arity : (style.unknown_has_value ? 1u : 0u);
        if (argc - i < static_cast<int>(want)) throw std::invalid_argument(style.missing(flag));
        if (it == table.end()) throw std::invalid_argument("Unknown option: " + flag);
        Values values;
        for (unsigned k = 0; k < want; ++k) values.emplace_back(argv[i++]);
        it->second.set(values);
        if (it->second.stops) break;
    }
    return seen;
}

} // namespace icp::cli
