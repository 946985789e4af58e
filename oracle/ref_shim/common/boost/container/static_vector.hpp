// Minimal stand-in for boost::container::static_vector (TEST INFRASTRUCTURE
// ONLY): the same interface on a std::vector; capacity is only reserved.
#pragma once
#include <cstddef>
#include <vector>

namespace boost {
namespace container {
template <class T, std::size_t N>
class static_vector : public std::vector<T> {
public:
    using std::vector<T>::vector;
    static_vector() { this->reserve(N); }
    static constexpr std::size_t static_capacity = N;
};
}  // namespace container
}  // namespace boost
