/* No-op stand-ins for the spdlog/fmt calls in the reference sources compiled
 * for the oracle pin (logging only; no effect on results). */
#pragma once
#include <string>
namespace fmt {
inline const char *runtime(const char *s) { return s; }
inline const std::string &runtime(const std::string &s) { return s; }
template <class... A> std::string format(A &&...) { return std::string(); }
}
namespace spdlog {
template <class... A> void info(A &&...) {}
}
