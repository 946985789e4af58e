// smf_slot_order.cu -- a locality order for the FAST step on an adaptive
// rectangle.  The adaptive mesh keeps zephyr's cell order (EuMesh::refine
// appends new cells and fills freed slots from the end, so after many
// adaptations neighbours lie far apart in memory); the gather-form kernels
// then read most neighbour values from scattered cache lines.  Here the
// cells are put in Morton order of their centres (at the finest level's
// spacing) for the duration of the step: the mesh arrays the FAST kernels
// read are copied in that order once per mesh change, the state is gathered
// into it before the step and scattered back after.  Each cell's arithmetic
// (its slots in their own order) is unchanged, and dt is a minimum, so the
// step's results are the same bits as in zephyr's order.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>

#include "smf_struct.cuh"

namespace zg {
namespace slotfast {

constexpr int OBLOCK = 256;
static inline unsigned oblocks(int n) { return (unsigned)((n + OBLOCK - 1) / OBLOCK); }

// Morton key of a cell: its centre's position in units of the finest cell
// (21 bits per axis), the bits of x and y interleaved
__global__ void k_keys(const double *cx, const double *cy, int n, double x0, double y0, double ihx, double ihy,
                       unsigned long long *keys, int *idx) {
    int ic = blockIdx.x * OBLOCK + threadIdx.x;
    if (ic >= n) return;
    const double fx = (cx[ic] - x0) * ihx, fy = (cy[ic] - y0) * ihy;
    const long long ix = fx <= 0.0 ? 0 : (fx >= 2097151.0 ? 2097151 : (long long)fx);
    const long long iy = fy <= 0.0 ? 0 : (fy >= 2097151.0 ? 2097151 : (long long)fy);
    unsigned long long kx = 0, ky = 0;
    for (int b = 0; b < 21; ++b) {
        kx |= (unsigned long long)((ix >> b) & 1) << (2 * b);
        ky |= (unsigned long long)((iy >> b) & 1) << (2 * b + 1);
    }
    keys[ic] = kx | ky;
    idx[ic] = ic;
}

__global__ void k_inverse(const int *perm, int n, int *inv) {
    int p = blockIdx.x * OBLOCK + threadIdx.x;
    if (p < n) inv[perm[p]] = p;
}

// the arrays SlotFastAcc reads, in the new order; neighbour indices renamed
__global__ void k_permute_mesh(SlotMesh m, const int *perm, const int *inv, int n, double *cx, double *cy,
                               double *vol, double *inc, int *level, int *fb, int *fn) {
    int p = blockIdx.x * OBLOCK + threadIdx.x;
    if (p >= n) return;
    const int ic = perm[p];
    cx[p] = m.cx[ic];
    cy[p] = m.cy[ic];
    vol[p] = m.vol[ic];
    inc[p] = m.inc[ic];
    level[p] = m.level[ic];
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        fb[8 * p + s] = m.fb[8 * ic + s];
        const int nb = m.fn[8 * ic + s];
        fn[8 * p + s] = nb >= 0 && nb < n ? inv[nb] : nb;
    }
}

__global__ void k_gather(const int *perm, int n, PrimPtr src, PrimPtr dst, const int *wsrc, int *wdst) {
    int p = blockIdx.x * OBLOCK + threadIdx.x;
    if (p >= n) return;
    const int ic = perm[p];
    dst.r[p] = src.r[ic];
    dst.u[p] = src.u[ic];
    dst.v[p] = src.v[ic];
    dst.p[p] = src.p[ic];
    dst.e[p] = src.e[ic];
    if (wsrc) wdst[p] = wsrc[ic];
}

__global__ void k_scatter(const int *perm, int n, PrimPtr src, PrimPtr dst, const int *wsrc, int *wdst) {
    int p = blockIdx.x * OBLOCK + threadIdx.x;
    if (p >= n) return;
    const int ic = perm[p];
    dst.r[ic] = src.r[p];
    dst.u[ic] = src.u[p];
    dst.v[ic] = src.v[p];
    dst.p[ic] = src.p[p];
    dst.e[ic] = src.e[p];
    if (wsrc) wdst[ic] = wsrc[p];
}

// the face list of the face-once kernels: the slots whose face each cell
// evaluates (computes_face), counted, offset by an exclusive scan, listed
__global__ void k_own_count(SlotMesh m, int n, int *cnt) {
    int p = blockIdx.x * OBLOCK + threadIdx.x;
    if (p > n) return;
    int k = 0;
    if (p < n) {
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            const int flag = m.fb[8 * p + s];
            if (flag != BC_UNDEFINED && computes_face(m, p, s, flag, m.fn[8 * p + s])) ++k;
        }
    }
    cnt[p] = k;  // cnt[n] = 0: the scan's last entry is the total
}

__global__ void k_own_list(SlotMesh m, int n, const int *off, int *list) {
    int p = blockIdx.x * OBLOCK + threadIdx.x;
    if (p >= n) return;
    int o = off[p];
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const int flag = m.fb[8 * p + s];
        if (flag != BC_UNDEFINED && computes_face(m, p, s, flag, m.fn[8 * p + s])) list[o++] = 8 * p + s;
    }
}

// position of slot s among the slots cell p computes (its face list entry
// minus the cell's offset)
__device__ __forceinline__ int own_rank(const SlotMesh &m, int p, int s) {
    int k = 0;
    for (int q = 0; q < s; ++q) {
        const int flag = m.fb[8 * p + q];
        if (flag != BC_UNDEFINED && computes_face(m, p, q, flag, m.fn[8 * p + q])) ++k;
    }
    return k;
}

__global__ void k_face_index(SlotMesh m, int n, const int *off, int *fidx) {
    int p = blockIdx.x * OBLOCK + threadIdx.x;
    if (p >= n) return;
    int o = off[p];
    for (int s = 0; s < 8; ++s) {
        const int flag = m.fb[8 * p + s];
        int x = FACE_NONE;
        if (flag != BC_UNDEFINED) {
            const int nb = m.fn[8 * p + s];
            if (computes_face(m, p, s, flag, nb)) {
                x = o++;
            } else {
                const int q = (s & 3) ^ 1;  // the neighbour's full slot of the opposite side
                x = -(off[nb] + own_rank(m, nb, q)) - 1;
            }
        }
        fidx[8 * p + s] = x;
    }
}

template <bool GATHER>
__global__ void k_permute_mixed(const int *perm, int n, MixedState src, MixedState dst, const int *wsrc, int *wdst) {
    int p = blockIdx.x * OBLOCK + threadIdx.x;
    if (p >= n) return;
    const int ic = perm[p];
    const int from = GATHER ? ic : p, to = GATHER ? p : ic;
#pragma unroll
    for (int k = 0; k < 4; ++k) dst.q[k][to] = src.q[k][from];
#pragma unroll
    for (int k = 0; k < 5; ++k) dst.w[k][to] = src.w[k][from];
    if (wsrc) wdst[to] = wsrc[from];
}

__global__ void k_scatter8(const int *perm, int n, Fields8 src, Fields8 dst) {
    int p = blockIdx.x * OBLOCK + threadIdx.x;
    if (p >= n) return;
    const int ic = perm[p];
#pragma unroll
    for (int k = 0; k < 8; ++k) dst.f[k][ic] = src.f[k][p];
}

size_t order_scratch_bytes(int cap) {
    size_t bytes = 0, scan = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const unsigned long long *)nullptr,
                                    (unsigned long long *)nullptr, (const int *)nullptr, (int *)nullptr, cap, 0, 42);
    cub::DeviceScan::ExclusiveSum(nullptr, scan, (const int *)nullptr, (int *)nullptr, cap + 1);
    return std::max(bytes, scan);
}

int build_order(const SlotMesh &m, int n, double x0, double y0, double hx, double hy, int key_bits,
                OrderBuffers &b, SlotMesh &out, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (n <= 0) return 0;
    k_keys<<<oblocks(n), OBLOCK, 0, st>>>(m.cx, m.cy, n, x0, y0, 1.0 / hx, 1.0 / hy, b.keys, b.idx);
    size_t bytes = b.tmp_bytes;
    // the keys use 2 key_bits bits: one radix pass per 8 of them
    const int end_bit = std::min(42, std::max(2, 2 * key_bits));
    if (cub::DeviceRadixSort::SortPairs(b.tmp, bytes, b.keys, b.keys + b.cap, b.idx, b.perm, n, 0, end_bit, st) !=
        cudaSuccess)
        return -1;
    k_inverse<<<oblocks(n), OBLOCK, 0, st>>>(b.perm, n, b.inv);
    k_permute_mesh<<<oblocks(n), OBLOCK, 0, st>>>(m, b.perm, b.inv, n, b.cx, b.cy, b.vol, b.inc, b.level, b.fb,
                                                   b.fn);
    out = m;
    out.n = n;
    out.cx = b.cx;
    out.cy = b.cy;
    out.vol = b.vol;
    out.inc = b.inc;
    out.level = b.level;
    out.fb = b.fb;
    out.fn = b.fn;
    // the stored per-slot geometry is not read by the FAST kernels
    out.fnx = out.fny = out.fcx = out.fcy = out.fa = nullptr;
    k_own_count<<<oblocks(n + 1), OBLOCK, 0, st>>>(out, n, b.fcnt);
    size_t scan = b.tmp_bytes;
    if (cub::DeviceScan::ExclusiveSum(b.tmp, scan, b.fcnt, b.foff, n + 1, st) != cudaSuccess) return -1;
    k_own_list<<<oblocks(n), OBLOCK, 0, st>>>(out, n, b.foff, b.flist);
    k_face_index<<<oblocks(n), OBLOCK, 0, st>>>(out, n, b.foff, b.fidx);
    // the face count sizes the face kernels' grids (one copy per mesh change)
    if (cudaMemcpyAsync(&b.nfaces, b.foff + n, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return -1;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

void gather_state(const int *perm, int n, PrimPtr src, PrimPtr dst, const int *wsrc, int *wdst, void *stream) {
    if (n > 0) k_gather<<<oblocks(n), OBLOCK, 0, (cudaStream_t)stream>>>(perm, n, src, dst, wsrc, wdst);
}
void gather_mixed(const int *perm, int n, MixedState src, MixedState dst, const int *wsrc, int *wdst, void *stream) {
    if (n > 0) k_permute_mixed<true><<<oblocks(n), OBLOCK, 0, (cudaStream_t)stream>>>(perm, n, src, dst, wsrc, wdst);
}
void scatter_mixed(const int *perm, int n, MixedState src, MixedState dst, const int *wsrc, int *wdst,
                   void *stream) {
    if (n > 0) k_permute_mixed<false><<<oblocks(n), OBLOCK, 0, (cudaStream_t)stream>>>(perm, n, src, dst, wsrc, wdst);
}
void scatter_fields8(const int *perm, int n, Fields8 src, Fields8 dst, void *stream) {
    if (n > 0) k_scatter8<<<oblocks(n), OBLOCK, 0, (cudaStream_t)stream>>>(perm, n, src, dst);
}
void scatter_state(const int *perm, int n, PrimPtr src, PrimPtr dst, const int *wsrc, int *wdst, void *stream) {
    if (n > 0) k_scatter<<<oblocks(n), OBLOCK, 0, (cudaStream_t)stream>>>(perm, n, src, dst, wsrc, wdst);
}

}  // namespace slotfast
}  // namespace zg
