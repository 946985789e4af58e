// Minimal stand-in for the three boost::algorithm string functions that
// zephyr's Limiter(name) uses (TEST INFRASTRUCTURE ONLY).
#pragma once
#include <cctype>
#include <string>

namespace boost {
namespace algorithm {
inline void to_lower(std::string &s) {
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
}
inline void erase_all(std::string &s, const std::string &t) {
    if (t.empty()) return;
    size_t pos;
    while ((pos = s.find(t)) != std::string::npos) s.erase(pos, t.size());
}
inline bool contains(const std::string &s, const std::string &t) { return s.find(t) != std::string::npos; }
}  // namespace algorithm
}  // namespace boost
