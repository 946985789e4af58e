// Stand-in for zephyr/mesh/storage.h (TEST INFRASTRUCTURE ONLY): a typed
// handle to a named per-cell field.  The checker's mesh keeps each field as
// one contiguous array, like the reference's Storage (one buffer per field).
#pragma once
#include <string>

namespace zephyr::mesh {

template <typename T>
class Storable {
public:
    using type = T;
    Storable() = default;
    explicit Storable(int i) : index(i) {}
    bool operator==(Storable<T> o) const { return index == o.index; }
    bool operator!=(Storable<T> o) const { return index != o.index; }
    int index = -1;
};

}  // namespace zephyr::mesh
