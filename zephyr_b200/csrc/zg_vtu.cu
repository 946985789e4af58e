// zg_vtu.cu -- device packing of zephyr's VTU output arrays: the quadrilateral
// corners, connectivity, offsets and types of VtuStructure::
// fill_adaptive_hex_2D (io/vtu_file.cpp:186-201) and the named cell variables
// of io/variable.cpp:11-160, written straight into the layout of the file's
// appended data.
#include "vtu_types.h"

namespace zg {
namespace vtu {
namespace {

constexpr int BLOCK = 256;

__global__ void k_points(MeshSrc m, double *out) {
    const int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= m.n) return;
    double x[4], y[4];
    if (m.kind == 0) {
        const int i = ic / m.ny, j = ic - i * m.ny;
        x[0] = m.X[i];
        y[0] = m.Y[j];
        x[1] = m.X[i + 1];
        y[1] = m.Y[j];
        x[2] = m.X[i + 1];
        y[2] = m.Y[j + 1];
        x[3] = m.X[i];
        y[3] = m.Y[j + 1];
    } else {
        // vs<-1,-1>, vs<+1,-1>, vs<+1,+1>, vs<-1,+1>: map points 0, 2, 8, 6
        const int q[4] = {0, 2, 8, 6};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            x[k] = m.mvx[9 * (size_t)ic + q[k]];
            y[k] = m.mvy[9 * (size_t)ic + q[k]];
        }
    }
    double *o = out + 12 * (size_t)ic;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        o[3 * k] = x[k];
        o[3 * k + 1] = y[k];
        o[3 * k + 2] = 0.0;
    }
}

__global__ void k_cells(int n, uint32_t *conn, uint32_t *offsets, uint8_t *types) {
    const int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= n) return;
#pragma unroll
    for (int k = 0; k < 4; ++k) conn[4 * (size_t)ic + k] = (uint32_t)(4 * ic + k);
    offsets[ic] = (uint32_t)(4 * (ic + 1));
    types[ic] = 9;  // VTK_QUAD
}

__global__ void k_var(MeshSrc m, int kind, const double *a, const double *b, void *out) {
    const int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= m.n) return;
    switch (kind) {
        case K_LEVEL: static_cast<int8_t *>(out)[ic] = (int8_t)(m.kind == 0 ? 0 : m.level[ic]); break;
        case K_INDEX: static_cast<int32_t *>(out)[ic] = ic; break;
        case K_RANK: static_cast<int32_t *>(out)[ic] = 0; break;
        case K_FLAG: static_cast<int8_t *>(out)[ic] = (int8_t)(m.flag ? m.flag[ic] : 0); break;
        case K_BIDX: static_cast<int32_t *>(out)[ic] = m.kind == 0 ? ic : m.b_idx[ic]; break;
        case K_ZIDX: static_cast<int32_t *>(out)[ic] = m.kind == 0 ? 0 : m.z_idx[ic]; break;
        case K_CENTER: {
            double cx, cy;
            if (m.kind == 0) {
                const int i = ic / m.ny, j = ic - i * m.ny;
                cx = m.cxt[i];
                cy = m.cyt[j];
            } else {
                cx = m.cx[ic];
                cy = m.cy[ic];
            }
            float *o = static_cast<float *>(out) + 3 * (size_t)ic;
            o[0] = __double2float_rn(cx);
            o[1] = __double2float_rn(cy);
            o[2] = 0.0f;
            break;
        }
        default: {  // K_VEC3
            double *o = static_cast<double *>(out) + 3 * (size_t)ic;
            o[0] = a[ic];
            o[1] = b[ic];
            o[2] = 0.0;
        }
    }
}

inline unsigned blocks(int n) { return (unsigned)((n + BLOCK - 1) / BLOCK); }

}  // namespace

void launch_points(const MeshSrc &m, double *out, cudaStream_t st) {
    if (m.n > 0) k_points<<<blocks(m.n), BLOCK, 0, st>>>(m, out);
}

void launch_cells(int n, uint32_t *conn, uint32_t *offsets, uint8_t *types, cudaStream_t st) {
    if (n > 0) k_cells<<<blocks(n), BLOCK, 0, st>>>(n, conn, offsets, types);
}

void launch_var(const MeshSrc &m, int kind, const double *a, const double *b, void *out, cudaStream_t st) {
    if (m.n > 0) k_var<<<blocks(m.n), BLOCK, 0, st>>>(m, kind, a, b, out);
}

}  // namespace vtu
}  // namespace zg
