// amr_refine.cu -- EuMesh::refine on the GPU (eu_mesh.cpp:290-359) for a 2-D
// mesh on one rank: flag balancing (balance_flags_fast), the counts and the
// new positions by prefix sums (Statistics, SwapLists, setup_positions), the
// new cells' geometry, connectivity and states (setup_geometry with the
// SmFluid distributor), and the compaction that fills the freed slots
// (move_elements).  The per-cell work is amr_core.cuh; this file orders it
// into kernels.  Compiled with -fmad=false (bit-exact geometry and states).
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include "amr_refine.h"

namespace zg {
namespace amr {

constexpr int BLOCK = 128;

static inline unsigned nb(int n) { return (unsigned)((n + BLOCK - 1) / BLOCK); }

__global__ void k_base(View m, int n, int max_level) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic < n) base_restriction(m, ic, max_level);
}
// the flags after base_restriction decide each cell's list (CellsByLevel)
__global__ void k_copy_flags(View m, int n, int *flag0) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic < n) flag0[ic] = m.flag[ic];
}
// rounds 1-4 of balance_flags_fast for the cells of one level
__global__ void k_round(View m, int n, const int *flag0, int lvl, int max_level, int round) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= n || m.level[ic] != lvl || lvl >= max_level) return;
    const int f0 = flag0[ic];
    if (round == 1) {
        if (f0 == 0) retain_update(m, ic);
    } else if (f0 < 0) {
        if (round == 4) coarse_update_by_sibs(m, ic);
        else coarse_update(m, ic);
    }
}
// counts[0..2] = cells to coarsen, keep, refine (Statistics)
__global__ void k_stats(View m, int n, int *counts) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    int c = 0, r = 0, f = 0;
    if (ic < n) {
        int fl = m.flag[ic];
        c = fl < 0;
        r = fl == 0;
        f = fl > 0;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    r = __reduce_add_sync(0xffffffffu, r);
    f = __reduce_add_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0) {
        if (c) atomicAdd(&counts[0], c);
        if (r) atomicAdd(&counts[1], r);
        if (f) atomicAdd(&counts[2], f);
    }
}
// scan keys: a = changing cell below n_short, b = kept cell, c = refined
// cell, d = first sibling of a coarsened family
__global__ void k_keys(View m, int n, int n_short, int *a, int *b, int *c, int *d) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= n) return;
    int fl = m.flag[ic];
    a[ic] = (ic < n_short && fl != 0) ? 1 : 0;
    b[ic] = fl == 0;
    c[ic] = fl > 0;
    d[ic] = (fl < 0 && m.z_idx[ic] % 4 == 0) ? 1 : 0;
}
// totals of the exclusive scans: counts[3] = changing cells below n_short,
// counts[4] = kept cells
__global__ void k_totals(int n, const int *a, const int *sa, const int *b, const int *sb, int *counts) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        counts[3] = n > 0 ? sa[n - 1] + a[n - 1] : 0;
        counts[4] = n > 0 ? sb[n - 1] + b[n - 1] : 0;
    }
}
// SwapLists (swap_lists.h:17-49): the first changing slots below n_short are
// filled, in increasing order, by the last new cells and then by the last
// kept cells, in decreasing order
__global__ void k_swap_lists(View m, int n, int n_large, int max_swap, int swap_count, int n_retain, const int *a,
                             const int *sa, const int *sb, int *und, int *act) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    const int n_new = n_large - n;
    if (ic < swap_count && ic < n_new) act[ic] = n_large - 1 - ic;
    if (ic >= n) return;
    if (a[ic] && sa[ic] < max_swap) und[sa[ic]] = ic;
    if (m.flag[ic] == 0 && n_new < swap_count) {
        int k = n_new + (n_retain - 1 - sb[ic]);
        if (k < swap_count) act[k] = ic;
    }
}
// setup_positions (setup_positions.h:10-40)
__global__ void k_positions(View m, int n, int n_parents, const int *sc, const int *sd) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= n) return;
    int fl = m.flag[ic];
    if (fl == 0) {
        m.next[ic] = ic;
    } else if (fl > 0) {
        m.next[ic] = n + n_parents + 4 * sc[ic];
    } else if (m.z_idx[ic] % 4 == 0) {
        int sibs[3];
        get_siblings(m, ic, sibs);
        int p = n + sd[ic];
        m.next[ic] = p;
        for (int k = 0; k < 3; ++k) m.next[sibs[k]] = p;
    }
}
__global__ void k_new_positions(View m, int n, int n_large) {
    int ic = n + blockIdx.x * BLOCK + threadIdx.x;
    if (ic < n_large) m.next[ic] = ic;
}
__global__ void k_swap_positions(View m, int swap_count, const int *und, const int *act) {
    int i = blockIdx.x * BLOCK + threadIdx.x;
    if (i < swap_count) m.next[act[i]] = und[i];
}
// setup_geometry (setup_geometry.h:10-35)
__global__ void k_geometry(View m, int n) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= n) return;
    int fl = m.flag[ic];
    if (fl == 0) retain_cell(m, ic);
    else if (fl > 0) refine_cell(m, ic);
    else coarse_cell(m, ic);
}
// move_elements (swap_lists.h:132-143)
__global__ void k_move(View m, int swap_count, const int *und, const int *act) {
    int i = blockIdx.x * BLOCK + threadIdx.x;
    if (i < swap_count) move_cell(m, act[i], und[i]);
}
// incircle diameter of every cell (amr_cells.cpp:107-116, adaptive branch)
__global__ void k_incircle(View m, int n, double *inc) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= n) return;
    P2 a = map_pt(m, ic, vs(1, 0)), b = map_pt(m, ic, vs(-1, 0)), c = map_pt(m, ic, vs(0, 1)), d = map_pt(m, ic, vs(0, -1));
    double dx1 = a.x - b.x, dy1 = a.y - b.y, dx2 = c.x - d.x, dy2 = c.y - d.y, z = 0.0 - 0.0;
    double s1 = dx1 * dx1 + dy1 * dy1 + z * z, s2 = dx2 * dx2 + dy2 * dy2 + z * z;
    inc[ic] = sqrt(s2 < s1 ? s2 : s1);
}

// AmrCells(const Rectangle&) (amr_cells_gen.cpp:128-281): cell ic = i ny + j
// with the map of SqQuad(v00, v01, v10, v11) over its four corners (quad.cpp,
// the four-vertex constructor: mid-edges 0.5 (a + b), centre
// 0.25 (v00 + v01 + v10 + v11)), axis-aligned unit normals, face centres at
// the mid-edges, areas hy, hy, hx, hx; boundary slots name the cell itself.
__global__ void k_init_rect(View m, RectSpec r) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= r.nx * r.ny) return;
    const int i = ic / r.ny, j = ic % r.ny;
    auto X = [&r](int k) { return r.x_min + ((r.x_max - r.x_min) * k) / r.nx; };
    auto Y = [&r](int k) { return r.y_min + ((r.y_max - r.y_min) * k) / r.ny; };
    const double hx = (r.x_max - r.x_min) / r.nx, hy = (r.y_max - r.y_min) / r.ny;
    // the constructor's parameters v00, v01, v10, v11 receive the corners
    // (i, j), (i + 1, j), (i, j + 1), (i + 1, j + 1)
    const P2 a{X(i), Y(j)}, b{X(i + 1), Y(j)}, c{X(i), Y(j + 1)}, d{X(i + 1), Y(j + 1)};
    auto half = [](P2 p, P2 q) { return P2{0.5 * (p.x + q.x), 0.5 * (p.y + q.y)}; };
    const P2 pts[9] = {a, half(a, b), b, half(a, c),
                       P2{0.25 * (a.x + b.x + c.x + d.x), 0.25 * (a.y + b.y + c.y + d.y)},
                       half(b, d), c, half(c, d), d};
    for (int k = 0; k < 9; ++k) {
        m.vx[9 * ic + k] = pts[k].x;
        m.vy[9 * ic + k] = pts[k].y;
    }
    m.next[ic] = ic;
    m.index[ic] = ic;
    m.flag[ic] = 0;
    m.level[ic] = 0;
    m.b_idx[ic] = ic;
    m.z_idx[ic] = 0;
    m.cx[ic] = pts[4].x;
    m.cy[ic] = pts[4].y;
    m.vol[ic] = hx * hy;
    const int nx = r.nx, ny = r.ny;
    auto idx = [ny](int ii, int jj) { return ii * ny + jj; };
    const int neib[4] = {i == 0 && !r.xper ? ic : idx((i - 1 + nx) % nx, j),
                         i == nx - 1 && !r.xper ? ic : idx((i + 1 + nx) % nx, j),
                         j == 0 && !r.yper ? ic : idx(i, (j - 1 + ny) % ny),
                         j == ny - 1 && !r.yper ? ic : idx(i, (j + 1 + ny) % ny)};
    const int bnd[4] = {i > 0 ? BC_INNER : r.bc[0], i < nx - 1 ? BC_INNER : r.bc[1], j > 0 ? BC_INNER : r.bc[2],
                        j < ny - 1 ? BC_INNER : r.bc[3]};
    // -UnitX, UnitX, -UnitY, UnitY (negation keeps the signed zeros)
    const double nxs[4] = {-1.0, 1.0, -0.0, 0.0}, nys[4] = {-0.0, 0.0, -1.0, 1.0};
    const int cpt[4] = {vs(-1, 0), vs(1, 0), vs(0, -1), vs(0, 1)};
    const double area[4] = {hy, hy, hx, hx};
    for (int s = 0; s < 4; ++s) {
        const int f = 8 * ic + s;
        int va, vb;
        sf(s, va, vb);
        m.fb[f] = bnd[s];
        m.fadj[f] = neib[s];
        m.fv[2 * f] = (signed char)va;
        m.fv[2 * f + 1] = (signed char)vb;
        m.fnx[f] = nxs[s];
        m.fny[f] = nys[s];
        m.fcx[f] = pts[cpt[s]].x;
        m.fcy[f] = pts[cpt[s]].y;
        m.fa[f] = area[s];
        const int g = f + 4;  // AmrFaces::set_undefined
        m.fb[g] = BC_UNDEFINED;
        m.fadj[g] = -1;
        m.fv[2 * g] = m.fv[2 * g + 1] = -1;
        m.fnx[g] = m.fny[g] = m.fcx[g] = m.fcy[g] = m.fa[g] = 0.0;
    }
}

int init_rect(const View &m, const RectSpec &r, double *inc, cudaStream_t st) {
    const int n = r.nx * r.ny;
    k_init_rect<<<nb(n), BLOCK, 0, st>>>(m, r);
    k_incircle<<<nb(n), BLOCK, 0, st>>>(m, n, inc);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int scratch_bytes(int cap, size_t *bytes) {
    size_t tb = 0;
    if (cub::DeviceScan::ExclusiveSum(nullptr, tb, (int *)nullptr, (int *)nullptr, cap) != cudaSuccess) return -1;
    *bytes = 8 * (size_t)cap * sizeof(int) + 64 + tb + 256;
    return 0;
}

RefineResult refine(const View &m, int n, int cap, int max_level, void *scratch, size_t scratch_size, double *inc,
                    cudaStream_t st) {
    RefineResult res{};
    res.n = n;
    char *p = static_cast<char *>(scratch);
    int *flag0 = reinterpret_cast<int *>(p);
    int *a = flag0 + cap, *sa = a + cap, *b = sa + cap, *sb = b + cap, *c = sb + cap, *sc = c + cap, *d = sc + cap;
    int *counts = reinterpret_cast<int *>(p + 8 * (size_t)cap * sizeof(int));
    void *cub_tmp = p + 8 * (size_t)cap * sizeof(int) + 64;
    size_t cub_bytes = scratch_size - (8 * (size_t)cap * sizeof(int) + 64);
    int *sd = flag0;  // the flag copy is not needed after balancing

    // balance_flags (balancing_fast.h:330-376)
    k_base<<<nb(n), BLOCK, 0, st>>>(m, n, max_level);
    k_copy_flags<<<nb(n), BLOCK, 0, st>>>(m, n, flag0);
    for (int lvl = max_level - 1; lvl >= 0; --lvl)
        for (int round = 1; round <= 4; ++round) k_round<<<nb(n), BLOCK, 0, st>>>(m, n, flag0, lvl, max_level, round);
    res.launches += 2 + 4 * max_level;

    // Statistics
    cudaMemsetAsync(counts, 0, 64, st);
    k_stats<<<nb(n), BLOCK, 0, st>>>(m, n, counts);
    int hc[8];
    if (cudaMemcpyAsync(hc, counts, sizeof(hc), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        res.err = -2;
        return res;
    }
    res.launches += 1;
    const int n_coarse = hc[0], n_retain = hc[1], n_refine = hc[2];
    const int n_parents = n_coarse / 4, n_children = 4 * n_refine;
    const int n_large = n + n_parents + n_children, n_short = n_retain + n_children + n_parents;
    res.n_coarse = n_coarse;
    res.n_refine = n_refine;
    if (n_large <= n) return res;  // nothing to do (apply_impl)
    if (n_large > cap) {
        res.err = -6;
        res.n_large = n_large;
        return res;
    }

    // prefix sums for SwapLists and setup_positions
    const int max_swap = n_large - n_short;
    k_keys<<<nb(n), BLOCK, 0, st>>>(m, n, n_short, a, b, c, d);
    cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, a, sa, n, st);
    cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, b, sb, n, st);
    cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, c, sc, n, st);
    cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, d, sd, n, st);
    k_totals<<<1, 32, 0, st>>>(n, a, sa, b, sb, counts);
    if (cudaMemcpyAsync(hc, counts, sizeof(hc), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        res.err = -2;
        return res;
    }
    res.launches += 6;
    const int swap_count = hc[3] < max_swap ? hc[3] : max_swap;
    int *und = c, *act = d;  // keys of refined cells and of family heads, no longer needed after their scans
    k_swap_lists<<<nb(n), BLOCK, 0, st>>>(m, n, n_large, max_swap, swap_count, hc[4], a, sa, sb, und, act);
    k_positions<<<nb(n), BLOCK, 0, st>>>(m, n, n_parents, sc, sd);
    k_new_positions<<<nb(n_large - n), BLOCK, 0, st>>>(m, n, n_large);
    k_swap_positions<<<nb(swap_count), BLOCK, 0, st>>>(m, swap_count, und, act);
    k_geometry<<<nb(n), BLOCK, 0, st>>>(m, n);
    k_move<<<nb(swap_count), BLOCK, 0, st>>>(m, swap_count, und, act);
    k_incircle<<<nb(n_short), BLOCK, 0, st>>>(m, n_short, inc);
    res.launches += 7;
    if (cudaGetLastError() != cudaSuccess) {
        res.err = -2;
        return res;
    }
    res.n = n_short;
    res.n_large = n_large;
    return res;
}

int incircle(const View &m, int n, double *inc, cudaStream_t st) {
    k_incircle<<<nb(n), BLOCK, 0, st>>>(m, n, inc);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace amr
}  // namespace zg
