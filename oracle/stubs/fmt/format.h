// Self-written stand-in for fmt::format: replaces each "{}" with the next
// argument streamed through std::ostringstream. Only used for exception
// messages in the reference sources compiled as the test oracle.
#pragma once
#include <sstream>
#include <string>
#include <string_view>
namespace fmt {
namespace detail {
inline void emit(std::ostringstream& os, std::string_view& f) { os << f; f = {}; }
template <class T, class... R>
void emit(std::ostringstream& os, std::string_view& f, const T& v, const R&... r) {
    const auto pos = f.find("{}");
    if (pos == std::string_view::npos) { os << f; f = {}; return; }
    os << f.substr(0, pos) << v;
    f.remove_prefix(pos + 2);
    emit(os, f, r...);
}
} // namespace detail
template <class... A> std::string format(std::string_view f, const A&... a) {
    std::ostringstream os;
    detail::emit(os, f, a...);
    return os.str();
}
} // namespace fmt
