// Test infrastructure for the oracle build only.
//
// The reference declares `thirdparty/spdlog` as a git submodule that is empty in this
// checkout.  The engine only calls spdlog::info/warn/error with "{}"-style format
// strings, and logging never affects results, so this header provides those three
// functions.  Messages go to stderr only when the environment variable FMREF_LOG is set.
#ifndef FM_ORACLE_SPDLOG_SHIM_H
#define FM_ORACLE_SPDLOG_SHIM_H

#include <cstdio>
#include <cstdlib>
#include <sstream>
#include <string>

namespace spdlog {
namespace detail {

inline void append_rest(std::ostringstream& os, const char* fmt) { os << fmt; }

template <typename A, typename... R>
void append_rest(std::ostringstream& os, const char* fmt, const A& a, const R&... rest)
{
    const char* p = fmt;
    while (*p) {
        if (p[0] == '{') {
            const char* q = p;
            while (*q && *q != '}') ++q;
            if (*q == '}') {
                os << a;
                append_rest(os, q + 1, rest...);
                return;
            }
        }
        os << *p++;
    }
}

template <typename... A>
void emit(const char* level, const char* fmt, const A&... args)
{
    if (std::getenv("FMREF_LOG") == nullptr) return;
    std::ostringstream os;
    append_rest(os, fmt, args...);
    std::fprintf(stderr, "[oracle %s] %s\n", level, os.str().c_str());
}

}  // namespace detail

template <typename... A> void info(const char* fmt, const A&... a) { detail::emit("info", fmt, a...); }
template <typename... A> void warn(const char* fmt, const A&... a) { detail::emit("warn", fmt, a...); }
template <typename... A> void error(const char* fmt, const A&... a) { detail::emit("error", fmt, a...); }

}  // namespace spdlog

#endif
