// Test infrastructure only: a silent stand-in for the {fmt} calls in the
// emerald SPH sources. They print diagnostics only (config summaries, frame
// timings); the oracle build drops them. The formatter specializations in
// emerald/util/format.h compile against the declarations below.
#pragma once

#include <stdexcept>
#include <string>

namespace fmt {

struct format_error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

struct format_parse_context {
    char const* b = nullptr;
    char const* e = nullptr;
    constexpr char const* begin() const { return b; }
    constexpr char const* end() const { return e; }
};

template <class T, class Char = char, class Enable = void>
struct formatter {};

template <class... A>
inline void print(A&&...) {}

template <class It, class... A>
inline It format_to(It out, A&&...) {
    return out;
}

template <class... A>
inline std::string format(A&&...) {
    return std::string();
}

}  // namespace fmt
