// Self-written stand-in for fmt::format as the reference sources call it:
// "{}" streams the next argument through std::ostringstream; "{:SPEC}" with
// a printf-style SPEC (".10g", "02d") formats it with snprintf. Only the
// reference sources compiled as test oracles include it.
#pragma once
#include <cstdio>
#include <sstream>
#include <string>
#include <string_view>
#include <type_traits>
namespace fmt {
namespace detail {
template <class T> void put(std::ostringstream& os, std::string_view spec, const T& v) {
    if (spec.empty()) {
        os << v;
        return;
    }
    std::string f = "%" + std::string(spec);
    char buf[128];
    if constexpr (std::is_floating_point_v<T>) {
        std::snprintf(buf, sizeof(buf), f.c_str(), static_cast<double>(v));
    } else if constexpr (std::is_integral_v<T>) {
        f.insert(f.size() - 1, "ll");
        std::snprintf(buf, sizeof(buf), f.c_str(), static_cast<long long>(v));
    } else {
        os << v;
        return;
    }
    os << buf;
}
inline void emit(std::ostringstream& os, std::string_view& f) { os << f; f = {}; }
template <class T, class... R>
void emit(std::ostringstream& os, std::string_view& f, const T& v, const R&... r) {
    const auto pos = f.find('{');
    if (pos == std::string_view::npos) { os << f; f = {}; return; }
    const auto close = f.find('}', pos);
    std::string_view spec = f.substr(pos + 1, close - pos - 1);
    if (!spec.empty() && spec.front() == ':')
        spec.remove_prefix(1);
    os << f.substr(0, pos);
    put(os, spec, v);
    f.remove_prefix(close + 1);
    emit(os, f, r...);
}
} // namespace detail
template <class... A> std::string format(std::string_view f, const A&... a) {
    std::ostringstream os;
    detail::emit(os, f, a...);
    return os.str();
}
} // namespace fmt
