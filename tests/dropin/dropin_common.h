// dropin_common.h -- TEST INFRASTRUCTURE: the final state of a driver run
// and the bit-for-bit comparison of two runs (dropin_smf.cpp, dropin_mmf.cpp).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

namespace dropin {

struct Snapshot {
    std::vector<double> data;  // per cell: centre x, y, level, then the state fields
    std::vector<double> dts;
    size_t cells = 0;
};

// Prints one JSON line; 0 when the two runs agree bit for bit (signed zeros
// aside) in every cell value and every dt.
inline int report(const char *what, const Snapshot &ref, const Snapshot &gpu) {
    const bool same_shape = ref.cells == gpu.cells && ref.data.size() == gpu.data.size() && ref.dts.size() == gpu.dts.size();
    size_t mismatches = 0;
    double max_rel = 0.0;
    if (same_shape) {
        for (size_t k = 0; k < ref.data.size(); ++k) {
            const double a = ref.data[k], b = gpu.data[k];
            // (signed zeros and NaN payloads aside)
            if (std::memcmp(&a, &b, sizeof(double)) != 0 && !(a == 0.0 && b == 0.0) &&
                !(std::isnan(a) && std::isnan(b))) {
                ++mismatches;
                const double d = std::fabs(a - b) / std::max(std::fabs(a), 1e-300);
                if (d > max_rel) max_rel = d;
            }
        }
        for (size_t k = 0; k < ref.dts.size(); ++k)
            if (ref.dts[k] != gpu.dts[k]) ++mismatches;
    }
    const bool equal = same_shape && mismatches == 0;
    std::printf("{\"case\": \"%s\", \"cells_reference\": %zu, \"cells_gpu\": %zu, \"steps\": %zu, "
                "\"mismatches\": %zu, \"max_rel_diff\": %.3e, \"bit_identical\": %s}\n",
                what, ref.cells, gpu.cells, ref.dts.size(), mismatches, max_rel, equal ? "true" : "false");
    return equal ? 0 : 1;
}

}  // namespace dropin
