// vtu_types.h -- packing of zephyr's VTU arrays (io/vtu_file.cpp) from device
// buffers (zg_vtu.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace zg {
namespace vtu {

// The cells to write: a uniform rectangle (ic = i * ny + j, geometry from the
// per-axis tables) or an adaptive mesh (9 map points per cell).
struct MeshSrc {
    int n;     // cells
    int kind;  // 0 rectangle, 1 adaptive
    int ny;
    const double *X, *Y, *cxt, *cyt;  // rectangle: vertex and centre tables
    const double *mvx, *mvy;          // adaptive: map points, 9 per cell
    const double *cx, *cy;            // adaptive: centres
    const int *level, *b_idx, *z_idx; // adaptive
    const int *flag;                  // refinement flags (null: all 0)
};

// Per-cell variables packed on the device.
enum Kind { K_LEVEL = 0, K_INDEX, K_RANK, K_FLAG, K_BIDX, K_ZIDX, K_CENTER, K_VEC3 };

// Points of VtuStructure::fill_adaptive_hex_2D: 4 corners per cell, 3 doubles each.
void launch_points(const MeshSrc &m, double *out, cudaStream_t st);
// connectivity 0..4n-1, offsets 4 (i + 1), types VTK_QUAD.
void launch_cells(int n, uint32_t *conn, uint32_t *offsets, uint8_t *types, cudaStream_t st);
// One variable of kind `kind`; K_VEC3 writes (a, b, 0) as doubles.
void launch_var(const MeshSrc &m, int kind, const double *a, const double *b, void *out, cudaStream_t st);

}  // namespace vtu
}  // namespace zg
