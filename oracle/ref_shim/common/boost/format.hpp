// Minimal stand-in for boost::format (TEST INFRASTRUCTURE ONLY): the
// reference uses it only to print states in error messages, so the
// arguments are printed after the format string without substitution.
#pragma once
#include <ostream>
#include <sstream>
#include <string>

namespace boost {
class format {
public:
    explicit format(const std::string &f) : text_(f) {}
    template <class T>
    format &operator%(const T &v) {
        std::ostringstream s;
        s << v;
        text_ += " " + s.str();
        return *this;
    }
    friend std::ostream &operator<<(std::ostream &os, const format &f) { return os << f.text_; }
    std::string str() const { return text_; }

private:
    std::string text_;
};
}  // namespace boost
