// amr_refine.h -- the GPU refine of a 2-D AMR mesh (amr_refine.cu).
#pragma once

#include <cuda_runtime.h>

#include "amr_core.cuh"

namespace zg {
namespace amr {

struct RefineResult {
    int err = 0;      // 0, -2 CUDA error, -6 capacity too small (n_large cells needed)
    int n = 0;        // cells after the adaptation
    int n_large = 0;  // cells held during it
    int n_coarse = 0, n_refine = 0;
    long long launches = 0;
};

// A Rectangle: nx by ny cells over [x_min, x_max] x [y_min, y_max], boundary
// flags left, right, bottom, top (both sides PERIODIC on a periodic axis).
struct RectSpec {
    int nx, ny;
    double x_min, x_max, y_min, y_max;
    int bc[4];
    bool xper, yper;
};

// The base mesh of the rectangle in the first nx ny cells of m (levels,
// indices, map points, geometry, faces) and its incircle diameters.
int init_rect(const View &m, const RectSpec &r, double *inc, cudaStream_t st);

// Bytes of scratch memory refine() needs for a capacity of `cap` cells.
int scratch_bytes(int cap, size_t *bytes);

// EuMesh::refine of the n-cell mesh in m (flags in m.flag), capacity cap
// cells; fills inc (incircle diameters) of the new cells.  Synchronises the
// stream twice (the counts decide the launch sizes).
RefineResult refine(const View &m, int n, int cap, int max_level, void *scratch, size_t scratch_size, double *inc,
                    cudaStream_t st);

int incircle(const View &m, int n, double *inc, cudaStream_t st);

}  // namespace amr
}  // namespace zg
