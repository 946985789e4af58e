// zg_api.cu -- the C ABI declared in include/zephyr_gpu.h: context, device
// memory, mesh tables and the orchestration of SmFluid::update on one GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/zephyr_gpu.h"
#include "amr_refine.h"
#include "mmf_types.h"
#include "smf_tiled.cuh"
#include "smf_tiled_launch.h"
#include "smf_types.h"
#include "tr_types.h"
#include "vtu_types.h"

using namespace zg;

// state_mode of a state held in the Morton order of the steps on an
// adaptive rectangle: FP64 primitive in the order buffers (FAST), or the
// MIXED representation in its own double buffers (MIXED)
constexpr int STATE_ORDERED = 100;
constexpr int STATE_ORDERED_MIXED = 101;

struct zg_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    // a second stream for work that overlaps the main stream's (the
    // interface reconstruction and the work list beside dt, the composite
    // Riemann faces beside the pure-stencil cells), with its events; created
    // on first use
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_cleared = nullptr, ev_dt = nullptr;
    std::string err;
    long long launches = 0;

    // mesh (structured rectangle)
    bool have_mesh = false;
    int nx = 0, ny = 0, n = 0;
    double box[4] = {};        // x_min, x_max, y_min, y_max of a rectangle mesh
    StructMesh mesh{};
    bool slots = false;        // mesh given cell by cell (zg_mesh_upload)
    SlotMesh smesh{};
    void *d_slot = nullptr;    // slot-mesh arrays
    void *d_axial = nullptr;   // axisymmetric volume_alt / area_alt of a slot mesh
    double *d_geo = nullptr;  // all geometry tables
    double *d_tgeo = nullptr;  // per-axis tables of the tiled kernels, FP64 then FP32
    tiled::AxisGeo<double> ax64{}, ay64{};
    tiled::AxisGeo<float> ax32{}, ay32{};
    int cap = 0;  // cells every per-cell field holds (n, or the adaptive mesh's capacity)

    // adaptive mesh (AmrCells layout on the device)
    bool amr = false;
    int amr_max_level = 0;
    int amr_distr = ZG_DISTR_SLOPE;
    void *d_amr = nullptr;          // cell and face arrays, `cap` cells
    void *d_amr_scratch = nullptr;  // work space of the refine
    size_t amr_scratch_size = 0;
    amr::View av{};                 // mesh arrays; state pointers set per refine
    zg_amr_stats amr_last{};
    long long mesh_version = 0;     // bumped whenever the cell set changes
    // FAST step on the adaptive mesh: the cells in Morton order for the step
    // (smf_slot_order.cu): order buffers, the reordered mesh arrays, three
    // states and two counter sets in that order (capacity cells)
    void *d_ord = nullptr;
    slotfast::OrderBuffers ord{};
    SlotMesh ord_mesh{};
    PrimPtr oz{}, ozhalf{}, oznext{};
    int *ow[2] = {};
    slotfast::FaceFlux oflux{};  // face-once fluxes, 8 slots per cell
    long long ord_version = -1;
    bool ord_waits = false;  // ow[0] holds the current isolation counters (predictor-corrector)
    bool grad_ordered = false;  // gx / gy hold the last FAST adaptive step's gradients in the cell order

    // solver
    bool configured = false;
    zg_smf_params par{};
    EosD eos{};
    double *d_state = nullptr;  // init/half/next (5 fields each) + 8 gradient fields
    int *d_wait = nullptr;      // two isolation-counter buffers
    unsigned long long *d_dmin = nullptr;
    unsigned int *d_ticket = nullptr;
    double *d_dt = nullptr;     // dt of the last step
    double *d_dt2 = nullptr;    // the other dt slot: the next step's dt when dt_next_ready
    bool dt_next_ready = false; // the FAST adaptive step's cell sums left the next dt in d_dt2
    int *d_flags = nullptr;
    PrimPtr z{}, zhalf{}, znext{};
    double *gx[4] = {}, *gy[4] = {};
    int wait_cur = 0;  // index of the buffer holding the current counters
    bool stepped = false;

    // tiled kernels (FAST / MIXED)
    unsigned long long *d_slots = nullptr;  // three rotating CFL accumulators
    int slot_k = 0;
    bool cfl_valid = false;
    int state_mode = ZG_FP64;  // representation of the current state (zg_precision, or STATE_ORDERED)
    double *d_mq = nullptr;    // MIXED conserved state, two sets of 4 fields
    float *d_mf = nullptr;     // MIXED FP32 fields: two state mirrors (5), stage (5), gradients (8)
    double *mq[2][4] = {};
    float *mw[2][5] = {}, *mh[5] = {}, *mg[8] = {};
    int mcur = 0;

    // multi-material solver (MmFluid)
    bool mm_configured = false;
    zg_mmf_params mpar{};
    double *d_mm = nullptr;        // two states of 6 + 2 NMAT fields, then 3 NMAT interface fields
    unsigned long long *d_mm_scalars = nullptr;  // CFL minimum @0, ticket @8, dt @16, error flag @24
    int *d_mm_flags = nullptr;
    int *d_mm_lists = nullptr;     // 8 counters, then the two work lists of the face loop (n each)
    double *d_mm_qbuf = nullptr;   // conservative states of the closure list
    double *d_mm2 = nullptr;       // second order: half-step state (6 + 2 NMAT fields), then 2 NG gradients
    double *d_mm_grad_a = nullptr;  // CrpMode::MUSCL: volume-fraction gradients, 2 NMAT fields
    bool mm_grad_a_valid = false;
    mmf::MmField mz{}, mznext{};
    double *mnx[mmf::NMAT] = {}, *mny[mmf::NMAT] = {}, *moff[mmf::NMAT] = {};

    // scalar VOF transport (Transfer)
    bool tr_configured = false;
    zg_tr_params tpar{};
    double *d_tr = nullptr;  // u1, n and p (two buffers), face fluxes, then 8 scalar slots
    tr::TrArgs targs{};

    // output: pinned host image of a VTU file's appended data (grown on demand)
    unsigned char *out_img = nullptr;
    size_t out_img_size = 0;

    // per-kernel timing
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, int>> ev_pending;  // (kind, index of the start event)
    size_t ev_used = 0;
};

namespace {

int fail(zg_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(zg_ctx *c, cudaError_t e, const char *what) {
    return fail(c, e == cudaErrorMemoryAllocation ? ZG_ERR_ALLOC : ZG_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

#define ZG_CUDA(ctx, call)                                  \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call); \
    } while (0)

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

void free_mm(zg_ctx *c) {
    cudaFree(c->d_mm2);
    c->d_mm2 = nullptr;
    cudaFree(c->d_mm_grad_a);
    c->d_mm_grad_a = nullptr;
    c->mm_grad_a_valid = false;
    cudaFree(c->d_mm);
    cudaFree(c->d_mm_scalars);
    cudaFree(c->d_mm_flags);
    cudaFree(c->d_mm_lists);
    cudaFree(c->d_mm_qbuf);
    c->d_mm_lists = nullptr;
    c->d_mm_qbuf = nullptr;
    c->d_mm = nullptr;
    c->d_mm_scalars = nullptr;
    c->d_mm_flags = nullptr;
    c->mm_configured = false;
}

void free_tr(zg_ctx *c) {
    cudaFree(c->d_tr);
    c->d_tr = nullptr;
    c->targs = tr::TrArgs{};
    c->tr_configured = false;
}

void free_solver(zg_ctx *c) {
    free_mm(c);
    free_tr(c);
    cudaFree(c->d_mq);
    cudaFree(c->d_mf);
    c->d_mq = nullptr;
    c->d_mf = nullptr;
    cudaFree(c->d_state);
    cudaFree(c->d_wait);
    cudaFree(c->d_dmin);
    cudaFree(c->d_flags);
    c->d_state = nullptr;
    c->d_wait = nullptr;
    c->d_dmin = nullptr;
    c->d_ticket = nullptr;
    c->d_dt = nullptr;
    c->d_dt2 = nullptr;
    c->dt_next_ready = false;
    c->d_flags = nullptr;
    c->configured = false;
    c->stepped = false;
}

void free_mesh(zg_ctx *c) {
    cudaFree(c->d_geo);
    cudaFree(c->d_tgeo);
    cudaFree(c->d_slot);
    cudaFree(c->d_axial);
    c->d_axial = nullptr;
    cudaFree(c->d_amr);
    cudaFree(c->d_amr_scratch);
    cudaFree(c->d_ord);
    c->d_ord = nullptr;
    c->ord = slotfast::OrderBuffers{};
    c->ord_version = -1;
    if (c->state_mode == STATE_ORDERED) c->state_mode = ZG_FP64;  // the state goes with the mesh
    c->grad_ordered = false;
    if (c->state_mode == STATE_ORDERED_MIXED) c->state_mode = ZG_MIXED;
    c->d_geo = nullptr;
    c->d_tgeo = nullptr;
    c->d_slot = nullptr;
    c->d_amr = nullptr;
    c->d_amr_scratch = nullptr;
    c->amr_scratch_size = 0;
    c->amr = false;
    c->av = amr::View{};
    c->amr_last = zg_amr_stats{};
    c->smesh = SlotMesh{};
    c->slots = false;
    c->have_mesh = false;
    c->cap = 0;
}

SmfArgs make_args(const zg_ctx *c) {
    SmfArgs a{};
    a.mesh = c->mesh;
    a.smesh = c->smesh;
    a.eos = c->eos;
    a.flux = c->par.flux;
    a.limiter = c->par.limiter;
    a.CFL = c->par.CFL;
    a.max_dt = c->par.max_dt;
    a.z = c->z;
    a.zhalf = c->zhalf;
    a.znext = c->znext;
    for (int k = 0; k < 4; ++k) {
        a.gx[k] = c->gx[k];
        a.gy[k] = c->gy[k];
    }
    a.wait_in = c->d_wait + (size_t)c->wait_cur * c->cap;
    a.wait_out = c->d_wait + (size_t)(1 - c->wait_cur) * c->cap;
    a.dmin_bits = c->d_dmin;
    a.dt_ticket = c->d_ticket;
    a.dt_out = c->d_dt;
    return a;
}

const unsigned long long *slot_ptr(const zg_ctx *c, int k) { return c->d_slots + ((c->slot_k + k) % 3); }

tiled::Fields<double> fast_fields(const zg_ctx *c) {
    tiled::Fields<double> f{};
    f.gxa = c->ax64;
    f.gya = c->ay64;
    const double *w[5] = {c->z.r, c->z.u, c->z.v, c->z.p, c->z.e};
    double *h[5] = {c->zhalf.r, c->zhalf.u, c->zhalf.v, c->zhalf.p, c->zhalf.e};
    double *wn[5] = {c->znext.r, c->znext.u, c->znext.v, c->znext.p, c->znext.e};
    for (int k = 0; k < 5; ++k) {
        f.w[k] = w[k];
        f.h[k] = h[k];
        f.wn[k] = wn[k];
    }
    for (int k = 0; k < 4; ++k) {
        f.gx[k] = c->gx[k];
        f.gy[k] = c->gy[k];
    }
    f.wait_in = c->d_wait + (size_t)c->wait_cur * c->cap;
    f.wait_out = c->d_wait + (size_t)(1 - c->wait_cur) * c->cap;
    f.slot_cur = const_cast<unsigned long long *>(slot_ptr(c, 0));
    f.slot_nxt = const_cast<unsigned long long *>(slot_ptr(c, 1));
    f.slot_clr = const_cast<unsigned long long *>(slot_ptr(c, 2));
    f.dt_out = c->d_dt;
    return f;
}

tiled::Fields<float> mixed_fields(const zg_ctx *c) {
    tiled::Fields<float> f{};
    f.gxa = c->ax32;
    f.gya = c->ay32;
    int a = c->mcur, b = 1 - c->mcur;
    for (int k = 0; k < 4; ++k) {
        f.q[k] = c->mq[a][k];
        f.qn[k] = c->mq[b][k];
        f.gx[k] = c->mg[k];
        f.gy[k] = c->mg[4 + k];
    }
    for (int k = 0; k < 5; ++k) {
        f.w[k] = c->mw[a][k];
        f.wn[k] = c->mw[b][k];
        f.h[k] = c->mh[k];
    }
    f.wait_in = c->d_wait + (size_t)c->wait_cur * c->cap;
    f.wait_out = c->d_wait + (size_t)(1 - c->wait_cur) * c->cap;
    f.slot_cur = const_cast<unsigned long long *>(slot_ptr(c, 0));
    f.slot_nxt = const_cast<unsigned long long *>(slot_ptr(c, 1));
    f.slot_clr = const_cast<unsigned long long *>(slot_ptr(c, 2));
    f.dt_out = c->d_dt;
    return f;
}

// Bring a state held in the Morton order of the FAST adaptive step back to
// the mesh's own order (FP64 primitive in c->z, counters in the current
// counter buffer); a no-op in the other representations.
slotfast::MixedState mixed_set(const zg_ctx *c, int set) {
    slotfast::MixedState m{};
    for (int k = 0; k < 4; ++k) m.q[k] = c->mq[set][k];
    for (int k = 0; k < 5; ++k) m.w[k] = c->mw[set][k];
    return m;
}

int leave_order(zg_ctx *c) {
    c->dt_next_ready = false;  // the state may change before the next step
    if (c->state_mode == STATE_ORDERED_MIXED) {
        // from the current set (cell order) into the other (mesh order)
        int *wsrc = c->d_wait + (size_t)c->wait_cur * c->cap, *wdst = c->d_wait + (size_t)(1 - c->wait_cur) * c->cap;
        slotfast::scatter_mixed(c->ord.perm, c->n, mixed_set(c, c->mcur), mixed_set(c, 1 - c->mcur), wsrc, wdst,
                                (void *)c->stream);
        ++c->launches;
        c->mcur = 1 - c->mcur;
        c->wait_cur = 1 - c->wait_cur;
        c->state_mode = ZG_MIXED;
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? ZG_OK : cuda_fail(c, e, "state order");
    }
    if (c->state_mode != STATE_ORDERED) return ZG_OK;
    cudaStream_t st = c->stream;
    int *wait = c->d_wait + (size_t)c->wait_cur * c->cap;
    slotfast::scatter_state(c->ord.perm, c->n, c->oz, c->z, c->ord_waits ? c->ow[0] : nullptr, wait, (void *)st);
    ++c->launches;
    c->state_mode = ZG_FP64;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ZG_OK : cuda_fail(c, e, "state order");
}

// The last FAST adaptive step's limited gradients back in the mesh's order,
// for a refine's slope distributor when no gradient computation came between
// (sm_fluid.cpp:372-470 reads the cells' stored gradients): copied into the
// order buffers the state has left, then scattered.  Call after
// leave_order, before the mesh changes.
int unorder_gradients(zg_ctx *c) {
    if (!c->grad_ordered) return ZG_OK;
    cudaStream_t st = c->stream;
    const size_t bytes = (size_t)c->n * sizeof(double);
    double *tmp[8] = {c->oz.r, c->oz.u, c->oz.v, c->oz.p, c->oz.e, c->ozhalf.r, c->ozhalf.u, c->ozhalf.v};
    slotfast::Fields8 src{}, dst{};
    for (int k = 0; k < 8; ++k) {
        double *g = k < 4 ? c->gx[k] : c->gy[k - 4];
        ZG_CUDA(c, cudaMemcpyAsync(tmp[k], g, bytes, cudaMemcpyDeviceToDevice, st));
        src.f[k] = tmp[k];
        dst.f[k] = g;
    }
    slotfast::scatter_fields8(c->ord.perm, c->n, src, dst, (void *)st);
    ++c->launches;
    c->grad_ordered = false;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ZG_OK : cuda_fail(c, e, "gradient order");
}

// Move the current state into the representation `mode` (FP64 primitive or
// MIXED) on the device.
int convert_state(zg_ctx *c, int mode) {
    int rc = leave_order(c);
    if (rc != ZG_OK) return rc;
    if (mode == c->state_mode) return ZG_OK;
    if (mode == ZG_MIXED) {
        tiled::Fields<float> f = mixed_fields(c);
        for (int k = 0; k < 4; ++k) f.qn[k] = c->mq[c->mcur][k];
        for (int k = 0; k < 5; ++k) f.wn[k] = c->mw[c->mcur][k];
        mixed::launch_to_mixed(c->n, c->z, f, (void *)c->stream);
    } else {
        mixed::launch_to_prim(c->n, mixed_fields(c), c->eos, c->z, (void *)c->stream);
    }
    c->launches += 1;
    c->state_mode = mode;
    c->cfl_valid = false;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ZG_OK : cuda_fail(c, e, "state conversion");
}

// Write the FP64 primitive form of the current state into c->z without
// changing the representation the steps use (MIXED keeps its FP64 conserved
// variables, so no conversion round trip enters the solution).
int materialize_prim(zg_ctx *c) {
    int rc = leave_order(c);
    if (rc != ZG_OK) return rc;
    if (c->state_mode != ZG_MIXED) return ZG_OK;
    mixed::launch_to_prim(c->n, mixed_fields(c), c->eos, c->z, (void *)c->stream);
    c->launches += 1;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ZG_OK : cuda_fail(c, e, "state conversion");
}

// Per-axis least-squares geometry of a uniform axis (gradient.h:251-275 for
// axis-aligned faces): V = vertices, C = cell centres, M = mid-edges of the
// other axis' faces, h = face area of this axis' faces, bc_lo / bc_hi the
// boundary flags of the two ends.  Eight tables of n values: wl, wh, rl, rh,
// binv, ol, oh, om.
std::vector<double> axis_tables(const std::vector<double> &V, const std::vector<double> &C,
                                const std::vector<double> &M, double h, int bc_lo, int bc_hi) {
    const int n = (int)C.size();
    std::vector<double> t(8 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        double r[2], w[2];
        for (int side = 0; side < 2; ++side) {
            const bool inner = side == 0 ? i > 0 : i < n - 1;
            const double fc = side == 0 ? V[i] : V[i + 1];
            const double nrm = side == 0 ? -1.0 : 1.0;
            double dr;
            if (inner) {
                dr = (side == 0 ? C[i - 1] : C[i + 1]) - C[i];
            } else {  // mirror of the centre in the face (amr_faces.h:197-199)
                double d = (fc - C[i]) * nrm;
                dr = (C[i] + (2.0 * d) * nrm) - C[i];
            }
            (void)bc_lo;
            (void)bc_hi;
            const double drn = (dr * nrm) * nrm;
            const double ad = std::fabs(drn);
            w[side] = h / (ad * ad * ad);
            r[side] = dr;
            t[(size_t)(0 + side) * n + i] = w[side] * drn;
            t[(size_t)(2 + side) * n + i] = dr;
        }
        double A = t[(size_t)0 * n + i] * r[0] + t[(size_t)1 * n + i] * r[1];
        if (std::fabs(A) < 1e-8) A = 1.0;  // gradient.h:268-273
        t[(size_t)4 * n + i] = 1.0 / A;
        t[(size_t)5 * n + i] = V[i] - C[i];
        t[(size_t)6 * n + i] = V[i + 1] - C[i];
        t[(size_t)7 * n + i] = M[i] - C[i];
    }
    return t;
}

std::string lower_strip(const char *name) {
    std::string s;
    for (const char *p = name; *p; ++p) s.push_back((char)std::tolower((unsigned char)*p));
    auto erase_all = [&s](const std::string &t) {
        size_t pos;
        while ((pos = s.find(t)) != std::string::npos) s.erase(pos, t.size());
    };
    erase_all(" ");
    erase_all("-");
    erase_all("_");
    erase_all("lim");
    erase_all("limiter");
    return s;
}

// Bracket one launch with timing events when timing is on.
template <class F>
void timed(zg_ctx *c, int kind, F &&launch) {
    c->launches += 1;
    if (!c->timing) {
        launch();
        return;
    }
    if (c->ev_used + 2 > c->ev_pool.size()) {
        for (int k = 0; k < 64; ++k) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            c->ev_pool.push_back(e);
        }
    }
    int i0 = (int)c->ev_used;
    c->ev_used += 2;
    cudaEventRecord(c->ev_pool[i0], c->stream);
    launch();
    cudaEventRecord(c->ev_pool[i0 + 1], c->stream);
    c->ev_pending.emplace_back(kind, i0);
}

// timed() for a launch on another stream of the context (its events are
// recorded on that stream).
template <class F>
void timed_on(zg_ctx *c, int kind, cudaStream_t s, F &&launch) {
    c->launches += 1;
    if (!c->timing) {
        launch();
        return;
    }
    if (c->ev_used + 2 > c->ev_pool.size()) {
        for (int k = 0; k < 64; ++k) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            c->ev_pool.push_back(e);
        }
    }
    int i0 = (int)c->ev_used;
    c->ev_used += 2;
    cudaEventRecord(c->ev_pool[i0], s);
    launch();
    cudaEventRecord(c->ev_pool[i0 + 1], s);
    c->ev_pending.emplace_back(kind, i0);
}

// The side stream and its events, created on first use on the context's
// device.  The side stream has the highest priority: its kernels (the
// composite faces: few blocks, long latency chains) are placed first, and
// the pure-stencil kernel fills the rest of the GPU around them (measured
// on the two-material 1024^2 step: 0.267 ms per step against 0.294-0.301
// ms with default priority).
int ensure_side(zg_ctx *c) {
    if (c->side) return ZG_OK;
    int lo = 0, hi = 0;
    ZG_CUDA(c, cudaDeviceGetStreamPriorityRange(&lo, &hi));
    ZG_CUDA(c, cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, hi));
    ZG_CUDA(c, cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    ZG_CUDA(c, cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    ZG_CUDA(c, cudaEventCreateWithFlags(&c->ev_cleared, cudaEventDisableTiming));
    ZG_CUDA(c, cudaEventCreateWithFlags(&c->ev_dt, cudaEventDisableTiming));
    return ZG_OK;
}

// One step of SmFluid::update (sm_fluid.cpp:81-102) as kernel launches.
int enqueue_parity_step(zg_ctx *c) {
    if (c->par.accuracy == 2) c->grad_ordered = false;  // this step's gradients, in the mesh's order
    SmfArgs a = make_args(c);
    void *st = (void *)c->stream;
    timed(c, ZG_K_DT, [&] { parity::launch_dt(a, c->z, c->slots, st); });
    if (c->par.accuracy == 1) {
        timed(c, ZG_K_FLUX1, [&] { parity::launch_flux1(a, c->slots, st); });
    } else if (c->par.scheme == ZG_SCHEME_PREDICTOR_CORRECTOR) {
        timed(c, ZG_K_GRAD, [&] { parity::launch_grad(a, c->z, c->slots, st); });
        timed(c, ZG_K_STAGE1, [&] { parity::launch_stage1(a, c->slots, st); });
        timed(c, ZG_K_STAGE2, [&] { parity::launch_stage2(a, c->slots, st); });
        c->wait_cur = 1 - c->wait_cur;
    } else {
        timed(c, ZG_K_GRAD, [&] { parity::launch_grad(a, c->z, c->slots, st); });
        timed(c, ZG_K_HEUN_A, [&] { parity::launch_heun(a, c->z, c->zhalf, false, c->slots, st); });
        timed(c, ZG_K_GRAD, [&] { parity::launch_grad(a, c->zhalf, c->slots, st); });
        timed(c, ZG_K_HEUN_B, [&] { parity::launch_heun(a, c->zhalf, c->znext, true, c->slots, st); });
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
    std::swap(c->z, c->znext);  // Storage::swap of init and next (sm_fluid.cpp:368-370)
    c->cfl_valid = false;
    c->stepped = true;
    return ZG_OK;
}

// The same step with the tiled kernels: pass A (gradients + predictor),
// pass B (face-once corrector with the next step's CFL minimum).
template <typename R, bool MIXED>
int enqueue_tiled_step(zg_ctx *c) {
    SmfArgs a = make_args(c);
    void *st = (void *)c->stream;
    auto fields = [c]() {
        if constexpr (MIXED) return mixed_fields(c);
        else return fast_fields(c);
    };
    auto L_cfl = [&](const tiled::Fields<R> &f) {
        if constexpr (MIXED) mixed::launch_cfl(a, f, st);
        else fast::launch_cfl(a, f, st);
    };
    auto L_grad = [&](const tiled::Fields<R> &f, bool predict) {
        if constexpr (MIXED) mixed::launch_grad_predict(a, f, predict, st);
        else fast::launch_grad_predict(a, f, predict, st);
    };
    auto L_faces = [&](const tiled::Fields<R> &f, int mode) {
        if constexpr (MIXED) mixed::launch_faces(a, f, mode, st);
        else fast::launch_faces(a, f, mode, st);
    };
    auto L_step = [&](const tiled::Fields<R> &f, int mode) {
        if constexpr (MIXED) mixed::launch_step(a, f, mode, st);
        else fast::launch_step(a, f, mode, st);
    };
    // one kernel per stage (smf_fused.cuh) for HLLC and HLL
    const bool fused = c->par.kernels != ZG_KERNELS_FAST_TWO_PASS &&
                       (c->par.flux == ZG_FLUX_HLLC || c->par.flux == ZG_FLUX_HLL);
    tiled::Fields<R> f = fields();
    if (!c->cfl_valid) {
        // Fresh accumulators for this step's minimum and the next one's
        // (0x7F bytes: a finite double far above any CFL term).
        cudaMemsetAsync(f.slot_cur, 0x7F, sizeof(unsigned long long), c->stream);
        cudaMemsetAsync(f.slot_nxt, 0x7F, sizeof(unsigned long long), c->stream);
        timed(c, ZG_K_DT, [&] { L_cfl(f); });
    }
    if (c->par.accuracy == 1) {
        timed(c, ZG_K_FLUX1, [&] { L_faces(f, 0); });
    } else if (fused && c->par.scheme == ZG_SCHEME_PREDICTOR_CORRECTOR) {
        timed(c, ZG_K_STEP, [&] { L_step(f, 1); });
        c->wait_cur = 1 - c->wait_cur;
    } else if (fused) {
        timed(c, ZG_K_HEUN_A, [&] { L_step(f, 2); });
        timed(c, ZG_K_HEUN_B, [&] { L_step(f, 3); });
    } else if (c->par.scheme == ZG_SCHEME_PREDICTOR_CORRECTOR) {
        timed(c, ZG_K_STAGE1, [&] { L_grad(f, true); });
        timed(c, ZG_K_STAGE2, [&] { L_faces(f, 1); });
        c->wait_cur = 1 - c->wait_cur;
    } else {
        timed(c, ZG_K_GRAD, [&] { L_grad(f, false); });
        timed(c, ZG_K_HEUN_A, [&] { L_faces(f, 2); });
        tiled::Fields<R> fs = f;  // gradients of the stage value z*
        for (int k = 0; k < 5; ++k) fs.w[k] = f.h[k];
        timed(c, ZG_K_GRAD, [&] { L_grad(fs, false); });
        timed(c, ZG_K_HEUN_B, [&] { L_faces(f, 3); });
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
    if constexpr (MIXED) c->mcur = 1 - c->mcur;
    else std::swap(c->z, c->znext);
    c->slot_k = (c->slot_k + 1) % 3;
    c->cfl_valid = true;
    c->stepped = true;
    return ZG_OK;
}

// The buffers of the Morton order (capacity cells), allocated on first use.
int ensure_order(zg_ctx *c) {
    if (c->d_ord) return ZG_OK;
    const size_t cap = (size_t)c->cap;
    const size_t tmp = slotfast::order_scratch_bytes(c->cap);
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t bytes = al(2 * cap * 8) + 3 * al(cap * 4) + al(tmp) + 4 * al(cap * 8) + al(cap * 4) +
                         2 * al(8 * cap * 4) + 15 * al(cap * 8) + 2 * al(cap * 4) + 4 * al(8 * cap * 8) +
                         2 * al((cap + 1) * 4) + 2 * al(8 * cap * 4) + al(8 * cap * 32) + al(cap * 32);
    ZG_CUDA(c, cudaMalloc(&c->d_ord, bytes));
    char *p = static_cast<char *>(c->d_ord);
    auto take = [&p, &al](size_t b) {
        char *q = p;
        p += al(b);
        return q;
    };
    slotfast::OrderBuffers &o = c->ord;
    o.cap = c->cap;
    o.keys = reinterpret_cast<unsigned long long *>(take(2 * cap * 8));
    o.idx = reinterpret_cast<int *>(take(cap * 4));
    o.perm = reinterpret_cast<int *>(take(cap * 4));
    o.inv = reinterpret_cast<int *>(take(cap * 4));
    o.tmp = take(tmp);
    o.tmp_bytes = tmp;
    o.cx = reinterpret_cast<double *>(take(cap * 8));
    o.cy = reinterpret_cast<double *>(take(cap * 8));
    o.vol = reinterpret_cast<double *>(take(cap * 8));
    o.inc = reinterpret_cast<double *>(take(cap * 8));
    o.level = reinterpret_cast<int *>(take(cap * 4));
    o.fb = reinterpret_cast<int *>(take(8 * cap * 4));
    o.fn = reinterpret_cast<int *>(take(8 * cap * 4));
    for (PrimPtr *z : {&c->oz, &c->ozhalf, &c->oznext}) {
        z->r = reinterpret_cast<double *>(take(cap * 8));
        z->u = reinterpret_cast<double *>(take(cap * 8));
        z->v = reinterpret_cast<double *>(take(cap * 8));
        z->p = reinterpret_cast<double *>(take(cap * 8));
        z->e = reinterpret_cast<double *>(take(cap * 8));
    }
    c->ow[0] = reinterpret_cast<int *>(take(cap * 4));
    c->ow[1] = reinterpret_cast<int *>(take(cap * 4));
    c->oflux.f = reinterpret_cast<double4 *>(take(4 * 8 * cap * 8));
    o.fcnt = reinterpret_cast<int *>(take((cap + 1) * 4));
    o.foff = reinterpret_cast<int *>(take((cap + 1) * 4));
    o.flist = reinterpret_cast<int *>(take(8 * cap * 4));
    o.fidx = reinterpret_cast<int *>(take(8 * cap * 4));
    o.sg = reinterpret_cast<double4 *>(take(8 * cap * 32));
    o.bm = reinterpret_cast<double4 *>(take(cap * 32));
    o.nfaces = 0;
    c->ord_version = -1;
    return ZG_OK;
}

// The cell order, the ordered mesh arrays, the face list and the gradient
// geometry of the current mesh (rebuilt after a mesh change).
int order_current(zg_ctx *c) {
    int rc = ensure_order(c);
    if (rc != ZG_OK) return rc;
    if (c->ord_version == c->mesh_version) return ZG_OK;
    void *st = (void *)c->stream;
    const double hx = ldexp(c->smesh.hx0, -c->amr_max_level), hy = ldexp(c->smesh.hy0, -c->amr_max_level);
    // finest cells per axis: the rectangle's extent in cells of the deepest level
    const double finest = std::max((c->box[1] - c->box[0]) / hx, (c->box[3] - c->box[2]) / hy);
    int key_bits = 1;
    while (key_bits < 21 && (double)(1LL << key_bits) <= finest - 0.5) ++key_bits;  // indices < 2^key_bits
    if (slotfast::build_order(c->smesh, c->n, c->box[0], c->box[2], hx, hy, key_bits, c->ord, c->ord_mesh, st) !=
        0)
        return cuda_fail(c, cudaGetLastError(), "cell order");
    SmfArgs ga = make_args(c);
    ga.smesh = c->ord_mesh;
    slotfast::launch_grad_geometry(ga, c->ord.sg, c->ord.bm, st);
    c->launches += 9;
    c->ord_version = c->mesh_version;
    return ZG_OK;
}

// The FAST step on an adaptive rectangle: the kernels of the parity step
// over derived face geometry, with fused multiply-adds, the corrector (and
// the Heun stages) face-once over a face list, run on the cells in Morton
// order.  The state is gathered into that order by the
// first step after it was in the mesh's order and stays there between steps
// (state_mode STATE_ORDERED); every other entry point that reads or writes
// the state, or changes the mesh, first scatters it back (leave_order).  The
// results are the same as in the mesh's own order.
int enqueue_slot_fast_step(zg_ctx *c) {
    void *st = (void *)c->stream;
    int rc = ensure_order(c);
    if (rc != ZG_OK) return rc;
    const bool pc = c->par.accuracy == 2 && c->par.scheme == ZG_SCHEME_PREDICTOR_CORRECTOR;
    if (c->state_mode == STATE_ORDERED && (c->ord_version != c->mesh_version || c->ord_waits != pc)) {
        rc = leave_order(c);  // not reached through the API: the mesh and the scheme change after leave_order
        if (rc != ZG_OK) return rc;
    }
    if (c->state_mode != STATE_ORDERED) {
        rc = convert_state(c, ZG_FP64);
        if (rc != ZG_OK) return rc;
        rc = order_current(c);
        if (rc != ZG_OK) return rc;
        int *wait = c->d_wait + (size_t)c->wait_cur * c->cap;
        slotfast::gather_state(c->ord.perm, c->n, c->z, c->oz, pc ? wait : nullptr, c->ow[0], st);
        ++c->launches;
        c->ord_waits = pc;
        c->state_mode = STATE_ORDERED;
    }
    c->oflux.list = c->ord.flist;
    c->oflux.fidx = c->ord.fidx;
    c->oflux.nfaces = c->ord.nfaces;
    // second order: the corrector's (or the final Heun stage's) cell sums
    // also take the CFL minimum of the state they write, so the next step
    // starts with its dt (in the other dt slot) and launches no dt kernel
    const bool fuse_dt = c->par.accuracy == 2;
    const bool have_dt = c->dt_next_ready;
    if (have_dt) std::swap(c->d_dt, c->d_dt2);
    c->oflux.dt_next = fuse_dt ? c->d_dt2 : nullptr;
    SmfArgs a = make_args(c);
    a.smesh = c->ord_mesh;
    a.z = c->oz;
    a.zhalf = c->ozhalf;
    a.znext = c->oznext;
    a.wait_in = c->ow[0];
    a.wait_out = c->ow[1];
    if (!have_dt) timed(c, ZG_K_DT, [&] { slotfast::launch_dt(a, a.z, st); });
    if (c->par.accuracy == 1) {
        timed(c, ZG_K_FLUX1, [&] { slotfast::launch_flux1(a, st); });
    } else if (pc) {
        // gradients and the predictor in one pass
        timed(c, ZG_K_GRAD, [&] { slotfast::launch_grad_pre(a, a.z, c->ord.sg, c->ord.bm, true, st); });
        // the corrector face-once: the listed faces, then every cell's sum
        timed(c, ZG_K_STAGE2, [&] { slotfast::launch_stage2_faces(a, c->oflux, st); });
        timed(c, ZG_K_STAGE2, [&] { slotfast::launch_stage2_sum(a, c->oflux, st); });
        std::swap(c->ow[0], c->ow[1]);
    } else {
        timed(c, ZG_K_GRAD, [&] { slotfast::launch_grad_pre(a, a.z, c->ord.sg, c->ord.bm, false, st); });
        timed(c, ZG_K_HEUN_A, [&] { slotfast::launch_heun_faces(a, a.z, c->oflux, st); });
        timed(c, ZG_K_HEUN_A, [&] { slotfast::launch_heun_sum(a, a.z, a.zhalf, false, c->oflux, st); });
        timed(c, ZG_K_GRAD, [&] { slotfast::launch_grad_pre(a, a.zhalf, c->ord.sg, c->ord.bm, false, st); });
        timed(c, ZG_K_HEUN_B, [&] { slotfast::launch_heun_faces(a, a.zhalf, c->oflux, st); });
        timed(c, ZG_K_HEUN_B, [&] { slotfast::launch_heun_sum(a, a.zhalf, a.znext, true, c->oflux, st); });
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
    std::swap(c->oz, c->oznext);
    if (c->par.accuracy == 2) c->grad_ordered = true;
    c->dt_next_ready = fuse_dt;
    c->cfl_valid = false;
    c->stepped = true;
    return ZG_OK;
}

// The MIXED step on an adaptive rectangle (FP64 conserved state with an FP32
// primitive mirror, as on a rectangle).
int enqueue_slot_mixed_step(zg_ctx *c) {
    if (c->par.accuracy == 2 && c->par.scheme != ZG_SCHEME_PREDICTOR_CORRECTOR)
        return fail(c, ZG_ERR_STATE,
                    "the MIXED form on an adaptive mesh runs first order or the predictor-corrector scheme");
    // the state in the cell order of the FAST step (smf_slot_order.cu), kept
    // there between steps like the FAST step's: gathered from the current
    // set of the MIXED buffers into the other, with the counters
    void *st = (void *)c->stream;
    int rc = ZG_OK;
    if (c->state_mode == STATE_ORDERED_MIXED && c->ord_version != c->mesh_version) {
        rc = leave_order(c);  // not reached through the API: the mesh changes after leave_order
        if (rc != ZG_OK) return rc;
    }
    if (c->state_mode != STATE_ORDERED_MIXED) {
        rc = convert_state(c, ZG_MIXED);
        if (rc != ZG_OK) return rc;
        rc = order_current(c);
        if (rc != ZG_OK) return rc;
        int *wsrc = c->d_wait + (size_t)c->wait_cur * c->cap, *wdst = c->d_wait + (size_t)(1 - c->wait_cur) * c->cap;
        slotfast::gather_mixed(c->ord.perm, c->n, mixed_set(c, c->mcur), mixed_set(c, 1 - c->mcur), wsrc, wdst, st);
        ++c->launches;
        c->mcur = 1 - c->mcur;
        c->wait_cur = 1 - c->wait_cur;
        c->state_mode = STATE_ORDERED_MIXED;
    }
    // the faces once over the face list, the cell sums taking the next dt
    // (as in the FAST step)
    c->oflux.list = c->ord.flist;
    c->oflux.fidx = c->ord.fidx;
    c->oflux.nfaces = c->ord.nfaces;
    const bool have_dt = c->dt_next_ready;
    if (have_dt) std::swap(c->d_dt, c->d_dt2);
    c->oflux.dt_next = c->d_dt2;
    SmfArgs a = make_args(c);
    a.smesh = c->ord_mesh;
    tiled::Fields<float> f = mixed_fields(c);
    if (!have_dt) timed(c, ZG_K_DT, [&] { slotmixed::launch_dt(a, f, st); });
    if (c->par.accuracy == 1) {
        timed(c, ZG_K_FLUX1, [&] { slotmixed::launch_faces_once(a, f, 0, c->oflux, st); });
        timed(c, ZG_K_FLUX1, [&] { slotmixed::launch_sum(a, f, 0, c->oflux, st); });
    } else {
        timed(c, ZG_K_GRAD, [&] { slotmixed::launch_grad(a, f, c->ord.sg, c->ord.bm, true, st); });
        timed(c, ZG_K_STAGE2, [&] { slotmixed::launch_faces_once(a, f, 1, c->oflux, st); });
        timed(c, ZG_K_STAGE2, [&] { slotmixed::launch_sum(a, f, 1, c->oflux, st); });
        c->wait_cur = 1 - c->wait_cur;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
    c->mcur = 1 - c->mcur;
    c->dt_next_ready = true;
    c->cfl_valid = false;
    c->stepped = true;
    return ZG_OK;
}

int enqueue_step(zg_ctx *c) {
    const bool fast = c->par.kernels != ZG_KERNELS_PARITY;
    if (c->smesh.vol_alt && (fast || c->par.precision != ZG_FP64 || (c->par.accuracy == 2 &&
                                                                        c->par.scheme == ZG_SCHEME_HEUN)))
        return fail(c, ZG_ERR_STATE, "axial symmetry runs with the PARITY kernels and the reference's schemes");
    if (c->amr && c->par.precision == ZG_FP64 && fast) return enqueue_slot_fast_step(c);
    if (c->amr && c->par.precision == ZG_MIXED) return enqueue_slot_mixed_step(c);
    if (c->slots && (c->par.precision == ZG_MIXED || fast))
        return fail(c, ZG_ERR_STATE,
                    "the MIXED kernels need a rectangle mesh; the FAST kernels a rectangle or an adaptive rectangle");
    if (c->par.precision == ZG_MIXED) {
        int rc = convert_state(c, ZG_MIXED);
        if (rc != ZG_OK) return rc;
        return enqueue_tiled_step<float, true>(c);
    }
    int rc = convert_state(c, ZG_FP64);
    if (rc != ZG_OK) return rc;
    if (fast) return enqueue_tiled_step<double, false>(c);
    return enqueue_parity_step(c);
}

}  // namespace

extern "C" {

void zg_smf_default_params(zg_smf_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->eos_kind = ZG_EOS_IDEAL;
    p->gamma = 1.4;
    p->P0 = 0.0;
    p->e0 = 0.0;
    p->flux = ZG_FLUX_HLLC;
    p->limiter = ZG_LIM_MC;
    p->accuracy = 1;
    p->scheme = ZG_SCHEME_PREDICTOR_CORRECTOR;
    p->precision = ZG_FP64;
    p->kernels = ZG_KERNELS_PARITY;
    p->CFL = 0.5;
    p->max_dt = std::numeric_limits<double>::max();
}

int zg_limiter_from_name(const char *name) {
    if (!name) return -1;
    std::string s = lower_strip(name);
    auto has = [&s](const char *t) { return s.find(t) != std::string::npos; };
    if (s.empty() || has("off") || has("none") || has("zero") || has("empty")) return ZG_LIM_NONE;
    if (has("one") || has("unit")) return ZG_LIM_UNIT;
    if (has("minmod")) return ZG_LIM_MINMOD;
    if (has("mc")) return ZG_LIM_MC;
    if (has("leer")) return ZG_LIM_VANLEER;
    if (has("albada")) return has("2") ? ZG_LIM_VANALBADA2 : ZG_LIM_VANALBADA1;
    if (has("charm")) return ZG_LIM_CHARM;
    if (has("hcus")) return ZG_LIM_HCUS;
    if (has("hquick")) return ZG_LIM_HQUICK;
    if (has("koren")) return ZG_LIM_KOREN;
    if (has("smart")) return ZG_LIM_SMART;
    if (has("superbee")) return ZG_LIM_SUPERBEE;
    return -1;
}

int zg_create(zg_ctx **out, int device) {
    if (!out) return ZG_ERR_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return ZG_ERR_CUDA;
    auto *c = new zg_ctx();
    c->device = device;
    DeviceGuard g(device);
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return ZG_ERR_CUDA;
    }
    c->stream = c->own_stream;
    *out = c;
    return ZG_OK;
}

int zg_destroy(zg_ctx *c) {
    if (!c) return ZG_ERR_ARG;
    {
        DeviceGuard g(c->device);
        cudaStreamSynchronize(c->stream);
        free_solver(c);
        free_mesh(c);
        for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
        if (c->out_img) cudaFreeHost(c->out_img);
        if (c->own_stream) cudaStreamDestroy(c->own_stream);
        if (c->side) cudaStreamDestroy(c->side);
        for (cudaEvent_t e : {c->ev_fork, c->ev_join, c->ev_cleared, c->ev_dt})
            if (e) cudaEventDestroy(e);
    }
    delete c;
    return ZG_OK;
}

const char *zg_last_error(const zg_ctx *c) { return c ? c->err.c_str() : "null context"; }

int zg_set_stream(zg_ctx *c, void *stream) {
    if (!c) return ZG_ERR_ARG;
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return ZG_OK;
}

int zg_mesh_rectangle(zg_ctx *c, int nx, int ny, double x_min, double x_max, double y_min, double y_max,
                      const int bounds[4]) {
    if (!c) return ZG_ERR_ARG;
    if (nx < 1 || ny < 1 || !bounds) return fail(c, ZG_ERR_ARG, "zg_mesh_rectangle: nx, ny >= 1 and bounds required");
    if ((long long)nx * ny > (long long)std::numeric_limits<int>::max() / 8)
        return fail(c, ZG_ERR_ARG, "zg_mesh_rectangle: too many cells for 32-bit cell indices");
    if (!(x_max > x_min) || !(y_max > y_min)) return fail(c, ZG_ERR_ARG, "zg_mesh_rectangle: empty box");
    for (int k = 0; k < 4; ++k) {
        if (bounds[k] < ZG_BC_INNER || bounds[k] > ZG_BC_PERIODIC || bounds[k] == ZG_BC_INNER)
            return fail(c, ZG_ERR_ARG, "zg_mesh_rectangle: boundary flags must be WALL, ZOE or PERIODIC");
    }
    DeviceGuard g(c->device);
    cudaStreamSynchronize(c->stream);
    free_solver(c);
    free_mesh(c);

    int bc[4] = {bounds[0], bounds[1], bounds[2], bounds[3]};
    bool xper = bc[0] == ZG_BC_PERIODIC || bc[1] == ZG_BC_PERIODIC;
    bool yper = bc[2] == ZG_BC_PERIODIC || bc[3] == ZG_BC_PERIODIC;
    if (xper) bc[0] = bc[1] = ZG_BC_PERIODIC;
    if (yper) bc[2] = bc[3] = ZG_BC_PERIODIC;

    // Geometry tables with the reference's formulas:
    //   vertices  amr_cells_gen.cpp:155-161  x_min + ((x_max - x_min) * i) / nx
    //   centre    quad.cpp:434               0.25 * (v00 + v01 + v10 + v11)
    //   mid-edges quad.cpp:433-435           0.5 * (a + b)
    //   incircle  amr_cells.cpp:107-116      |vs<+1,0> - vs<-1,0>|^2, |vs<0,+1> - vs<0,-1>|^2
    std::vector<double> X(nx + 1), Y(ny + 1), cx(nx), cy(ny), fxm(nx), fym(ny), i2x(nx), i2y(ny);
    for (int i = 0; i <= nx; ++i) X[i] = x_min + ((x_max - x_min) * i) / nx;
    for (int j = 0; j <= ny; ++j) Y[j] = y_min + ((y_max - y_min) * j) / ny;
    for (int i = 0; i < nx; ++i) {
        cx[i] = 0.25 * (X[i] + X[i + 1] + X[i] + X[i + 1]);
        fxm[i] = 0.5 * (X[i] + X[i + 1]);
        double d = 0.5 * (X[i + 1] + X[i + 1]) - 0.5 * (X[i] + X[i]);
        i2x[i] = d * d + 0.0 * 0.0 + 0.0 * 0.0;
    }
    for (int j = 0; j < ny; ++j) {
        cy[j] = 0.25 * (Y[j] + Y[j] + Y[j + 1] + Y[j + 1]);
        fym[j] = 0.5 * (Y[j] + Y[j + 1]);
        double d = 0.5 * (Y[j + 1] + Y[j + 1]) - 0.5 * (Y[j] + Y[j]);
        i2y[j] = 0.0 * 0.0 + d * d + 0.0 * 0.0;
    }
    size_t total = (size_t)(nx + 1) + (ny + 1) + 3 * (size_t)nx + 3 * (size_t)ny + 2 * (size_t)nx + 2 * (size_t)ny;
    ZG_CUDA(c, cudaMalloc(&c->d_geo, total * sizeof(double)));
    std::vector<double> host;
    host.reserve(total);
    auto put = [&host](const std::vector<double> &v) {
        size_t off = host.size();
        host.insert(host.end(), v.begin(), v.end());
        return off;
    };
    size_t oX = put(X), oY = put(Y), ocx = put(cx), ocy = put(cy), ofx = put(fxm), ofy = put(fym),
           oix = put(i2x), oiy = put(i2y);
    ZG_CUDA(c, cudaMemcpy(c->d_geo, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice));

    // per-axis tables of the tiled kernels (FP64 and FP32 copies)
    {
        std::vector<double> tx = axis_tables(X, cx, fxm, (y_max - y_min) / ny, bc[0], bc[1]);
        std::vector<double> ty = axis_tables(Y, cy, fym, (x_max - x_min) / nx, bc[2], bc[3]);
        size_t nd = tx.size() + ty.size();
        ZG_CUDA(c, cudaMalloc(&c->d_tgeo, nd * (sizeof(double) + sizeof(float))));
        std::vector<double> all(tx);
        all.insert(all.end(), ty.begin(), ty.end());
        std::vector<float> allf(all.begin(), all.end());
        ZG_CUDA(c, cudaMemcpy(c->d_tgeo, all.data(), nd * sizeof(double), cudaMemcpyHostToDevice));
        float *f32 = reinterpret_cast<float *>(c->d_tgeo + nd);
        ZG_CUDA(c, cudaMemcpy(f32, allf.data(), nd * sizeof(float), cudaMemcpyHostToDevice));
        auto fill = [](auto &g, auto *base, int n) {
            g.wl = base;
            g.wh = base + n;
            g.rl = base + 2 * (size_t)n;
            g.rh = base + 3 * (size_t)n;
            g.binv = base + 4 * (size_t)n;
            g.ol = base + 5 * (size_t)n;
            g.oh = base + 6 * (size_t)n;
            g.om = base + 7 * (size_t)n;
        };
        fill(c->ax64, c->d_tgeo, nx);
        fill(c->ay64, c->d_tgeo + tx.size(), ny);
        fill(c->ax32, f32, nx);
        fill(c->ay32, f32 + tx.size(), ny);
    }

    StructMesh &m = c->mesh;
    m.nx = nx;
    m.ny = ny;
    m.n = nx * ny;
    for (int k = 0; k < 4; ++k) m.bc[k] = bc[k];
    m.xper = xper;
    m.yper = yper;
    m.X = c->d_geo + oX;
    m.Y = c->d_geo + oY;
    m.cx = c->d_geo + ocx;
    m.cy = c->d_geo + ocy;
    m.fxm = c->d_geo + ofx;
    m.fym = c->d_geo + ofy;
    m.inc2x = c->d_geo + oix;
    m.inc2y = c->d_geo + oiy;
    c->box[0] = x_min;
    c->box[1] = x_max;
    c->box[2] = y_min;
    c->box[3] = y_max;
    m.hx = (x_max - x_min) / nx;
    m.hy = (y_max - y_min) / ny;
    m.vol = m.hx * m.hy;
    c->nx = nx;
    c->ny = ny;
    c->n = m.n;
    c->cap = m.n;
    c->have_mesh = true;
    return ZG_OK;
}

int zg_mesh_n_cells(const zg_ctx *c, int *n) {
    if (!c || !n) return ZG_ERR_ARG;
    *n = c->have_mesh ? c->n : 0;
    return ZG_OK;
}

int zg_mesh_upload(zg_ctx *c, const zg_mesh_view *v) {
    if (!c || !v) return ZG_ERR_ARG;
    if (v->n_cells < 1) return fail(c, ZG_ERR_ARG, "zg_mesh_upload: n_cells must be positive");
    if ((long long)v->n_cells > (long long)std::numeric_limits<int>::max() / 8)
        return fail(c, ZG_ERR_ARG, "zg_mesh_upload: too many cells for 32-bit indices");
    const void *need[] = {v->center_x, v->center_y, v->volume, v->incircle, v->face_boundary, v->face_neib,
                          v->face_nx, v->face_ny, v->face_cx, v->face_cy, v->face_area};
    for (const void *q : need)
        if (!q) return fail(c, ZG_ERR_ARG, "zg_mesh_upload: null array");
    const int n = v->n_cells;
    for (long long f = 0; f < 8LL * n; ++f) {  // neighbour indices must stay inside the mesh
        int b = v->face_boundary[f], nb = v->face_neib[f];
        if (b != -1 && (nb < 0 || nb >= n))
            return fail(c, ZG_ERR_ARG, "zg_mesh_upload: neighbour index out of range");
        if (b < -1 || b > ZG_BC_PERIODIC) return fail(c, ZG_ERR_ARG, "zg_mesh_upload: unknown boundary flag");
    }
    DeviceGuard g(c->device);
    cudaStreamSynchronize(c->stream);
    free_solver(c);
    free_mesh(c);
    size_t nd = 4 * (size_t)n + 5 * 8 * (size_t)n, ni = 2 * 8 * (size_t)n;
    ZG_CUDA(c, cudaMalloc(&c->d_slot, nd * sizeof(double) + ni * sizeof(int)));
    double *d = static_cast<double *>(c->d_slot);
    int *ip = reinterpret_cast<int *>(d + nd);
    const double *srcd[9] = {v->center_x, v->center_y, v->volume, v->incircle, v->face_nx, v->face_ny,
                             v->face_cx, v->face_cy, v->face_area};
    size_t lens[9] = {(size_t)n, (size_t)n, (size_t)n, (size_t)n, 8 * (size_t)n, 8 * (size_t)n, 8 * (size_t)n,
                      8 * (size_t)n, 8 * (size_t)n};
    const double *dst[9];
    size_t off = 0;
    for (int k = 0; k < 9; ++k) {
        ZG_CUDA(c, cudaMemcpy(d + off, srcd[k], lens[k] * sizeof(double), cudaMemcpyHostToDevice));
        dst[k] = d + off;
        off += lens[k];
    }
    ZG_CUDA(c, cudaMemcpy(ip, v->face_boundary, 8 * (size_t)n * sizeof(int), cudaMemcpyHostToDevice));
    ZG_CUDA(c, cudaMemcpy(ip + 8 * (size_t)n, v->face_neib, 8 * (size_t)n * sizeof(int), cudaMemcpyHostToDevice));
    SlotMesh &m = c->smesh;
    m.n = n;
    m.cx = dst[0];
    m.cy = dst[1];
    m.vol = dst[2];
    m.inc = dst[3];
    m.fnx = dst[4];
    m.fny = dst[5];
    m.fcx = dst[6];
    m.fcy = dst[7];
    m.fa = dst[8];
    m.fb = ip;
    m.fn = ip + 8 * (size_t)n;
    c->mesh = StructMesh{};
    c->mesh.n = n;
    c->n = n;
    c->cap = n;
    c->nx = c->ny = 0;
    c->slots = true;
    c->have_mesh = true;
    return ZG_OK;
}

int zg_mesh_set_axial(zg_ctx *c, const double *volume_alt, const double *face_area_alt) {
    if (!c) return ZG_ERR_ARG;
    if (!c->have_mesh || !c->slots || c->amr)
        return fail(c, ZG_ERR_STATE, "zg_mesh_set_axial: axial symmetry needs a mesh given cell by cell (zg_mesh_upload)");
    if ((volume_alt == nullptr) != (face_area_alt == nullptr))
        return fail(c, ZG_ERR_ARG, "zg_mesh_set_axial: give both arrays, or neither to turn axial symmetry off");
    DeviceGuard g(c->device);
    cudaStreamSynchronize(c->stream);
    cudaFree(c->d_axial);
    c->d_axial = nullptr;
    c->smesh.vol_alt = nullptr;
    c->smesh.fa_alt = nullptr;
    if (!volume_alt) return ZG_OK;
    const size_t n = (size_t)c->n;
    ZG_CUDA(c, cudaMalloc(&c->d_axial, 9 * n * sizeof(double)));
    double *d = static_cast<double *>(c->d_axial);
    ZG_CUDA(c, cudaMemcpy(d, volume_alt, n * sizeof(double), cudaMemcpyHostToDevice));
    ZG_CUDA(c, cudaMemcpy(d + n, face_area_alt, 8 * n * sizeof(double), cudaMemcpyHostToDevice));
    c->smesh.vol_alt = d;
    c->smesh.fa_alt = d + n;
    return ZG_OK;
}

int zg_smf_configure(zg_ctx *c, const zg_smf_params *p) {
    if (!c || !p) return ZG_ERR_ARG;
    if (!c->have_mesh) return fail(c, ZG_ERR_STATE, "zg_smf_configure: no mesh");
    if (p->eos_kind != ZG_EOS_IDEAL && p->eos_kind != ZG_EOS_STIFFENED)
        return fail(c, ZG_ERR_ARG, "zg_smf_configure: unknown EoS");
    if (p->flux < ZG_FLUX_GODUNOV || p->flux > ZG_FLUX_CIR2)
        return fail(c, ZG_ERR_ARG, "zg_smf_configure: unknown numerical flux");
    if (p->flux > ZG_FLUX_HLLC && p->kernels != ZG_KERNELS_PARITY)
        return fail(c, ZG_ERR_ARG, "zg_smf_configure: HLLC_M, HLLC_LM, CIR1 and CIR2 run with the PARITY kernels");
    if (p->limiter < ZG_LIM_NONE || p->limiter > ZG_LIM_SUPERBEE)
        return fail(c, ZG_ERR_ARG, "zg_smf_configure: unknown limiter");
    if (p->scheme != ZG_SCHEME_PREDICTOR_CORRECTOR && p->scheme != ZG_SCHEME_HEUN)
        return fail(c, ZG_ERR_ARG, "zg_smf_configure: unknown scheme");
    if (p->precision != ZG_FP64 && p->precision != ZG_MIXED)
        return fail(c, ZG_ERR_ARG, "zg_smf_configure: unknown precision");
    if (p->kernels != ZG_KERNELS_PARITY && p->kernels != ZG_KERNELS_FAST && p->kernels != ZG_KERNELS_FAST_TWO_PASS)
        return fail(c, ZG_ERR_ARG, "zg_smf_configure: unknown kernel family");
    if (p->precision == ZG_MIXED && p->kernels == ZG_KERNELS_PARITY)
        return fail(c, ZG_ERR_ARG, "zg_smf_configure: the mixed form uses the FAST kernels");
    if (!(p->gamma > 1.0)) return fail(c, ZG_ERR_ARG, "zg_smf_configure: gamma must exceed 1");

    DeviceGuard g(c->device);
    int rc = leave_order(c);  // the new parameters may take the step off the ordered path
    if (rc != ZG_OK) return rc;
    c->par = *p;
    c->par.accuracy = std::min(std::max(1, p->accuracy), 2);        // sm_fluid.cpp:41-43
    c->par.CFL = std::max(0.0, std::min(p->CFL, 1.0));               // sm_fluid.cpp:37-39
    c->eos.kind = p->eos_kind;
    c->eos.gamma = p->gamma;
    c->eos.gm1 = p->gamma - 1.0;
    c->eos.P0 = p->eos_kind == ZG_EOS_IDEAL ? 0.0 : p->P0;
    c->eos.e0 = p->eos_kind == ZG_EOS_IDEAL ? 0.0 : p->e0;
    c->eos.pmin = p->eos_kind == ZG_EOS_IDEAL ? 0.0 : -p->P0;  // min_pressure()
    if (c->configured) return ZG_OK;  // fields exist already: keep the state (setters do not reset data)

    size_t n = (size_t)c->cap;
    size_t nfields = 3 * 5 + 8;
    ZG_CUDA(c, cudaMalloc(&c->d_state, nfields * n * sizeof(double)));
    ZG_CUDA(c, cudaMalloc(&c->d_wait, 2 * n * sizeof(int)));
    ZG_CUDA(c, cudaMalloc(&c->d_flags, n * sizeof(int)));
    ZG_CUDA(c, cudaMemsetAsync(c->d_flags, 0, n * sizeof(int), c->stream));  // cells start unflagged
    ZG_CUDA(c, cudaMalloc(&c->d_dmin, 64));
    c->d_ticket = reinterpret_cast<unsigned int *>(reinterpret_cast<char *>(c->d_dmin) + 8);
    c->d_dt = reinterpret_cast<double *>(reinterpret_cast<char *>(c->d_dmin) + 16);
    c->d_dt2 = reinterpret_cast<double *>(reinterpret_cast<char *>(c->d_dmin) + 48);
    c->dt_next_ready = false;
    c->d_slots = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(c->d_dmin) + 24);
    ZG_CUDA(c, cudaMalloc(&c->d_mq, 8 * n * sizeof(double)));
    ZG_CUDA(c, cudaMalloc(&c->d_mf, 23 * n * sizeof(float)));
    for (int s2 = 0; s2 < 2; ++s2)
        for (int k = 0; k < 4; ++k) c->mq[s2][k] = c->d_mq + (size_t)(4 * s2 + k) * n;
    {
        float *fb = c->d_mf;
        for (int s2 = 0; s2 < 2; ++s2)
            for (int k = 0; k < 5; ++k) c->mw[s2][k] = fb + (size_t)(5 * s2 + k) * n;
        for (int k = 0; k < 5; ++k) c->mh[k] = fb + (size_t)(10 + k) * n;
        for (int k = 0; k < 8; ++k) c->mg[k] = fb + (size_t)(15 + k) * n;
    }
    ZG_CUDA(c, cudaMemsetAsync(c->d_mq, 0, 8 * n * sizeof(double), c->stream));
    ZG_CUDA(c, cudaMemsetAsync(c->d_mf, 0, 23 * n * sizeof(float), c->stream));
    c->state_mode = ZG_FP64;
    c->mcur = 0;
    c->slot_k = 0;
    c->cfl_valid = false;
    double *b = c->d_state;
    auto take = [&b, n]() {
        double *p0 = b;
        b += n;
        return p0;
    };
    PrimPtr *sets[3] = {&c->z, &c->zhalf, &c->znext};
    for (PrimPtr *s : sets) {
        s->r = take();
        s->u = take();
        s->v = take();
        s->p = take();
        s->e = take();
    }
    for (int k = 0; k < 4; ++k) c->gx[k] = take();
    for (int k = 0; k < 4; ++k) c->gy[k] = take();
    ZG_CUDA(c, cudaMemsetAsync(c->d_state, 0, nfields * n * sizeof(double), c->stream));
    ZG_CUDA(c, cudaMemsetAsync(c->d_wait, 0, 2 * n * sizeof(int), c->stream));
    unsigned long long init[3] = {0x7FEFFFFFFFFFFFFFull, 0ull, 0ull};
    double nan = std::numeric_limits<double>::quiet_NaN();
    std::memcpy(&init[2], &nan, sizeof(double));
    ZG_CUDA(c, cudaMemcpyAsync(c->d_dmin, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    c->wait_cur = 0;
    c->configured = true;
    return ZG_OK;
}

int zg_smf_set_max_dt(zg_ctx *c, double max_dt) {
    if (!c) return ZG_ERR_ARG;
    c->par.max_dt = max_dt;
    c->dt_next_ready = false;  // a dt taken with the old cap
    return ZG_OK;
}

int zg_state_upload(zg_ctx *c, const double *rho, const double *vx, const double *vy, const double *p,
                    const double *e) {
    if (!c || !rho || !vx || !vy || !p || !e) return ZG_ERR_ARG;
    if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_state_upload: solver not configured");
    DeviceGuard g(c->device);
    int rc = leave_order(c);  // the counters held in the cell order come back with it
    if (rc != ZG_OK) return rc;
    size_t bytes = (size_t)c->n * sizeof(double);
    const double *src[5] = {rho, vx, vy, p, e};
    double *dst[5] = {c->z.r, c->z.u, c->z.v, c->z.p, c->z.e};
    for (int k = 0; k < 5; ++k)
        ZG_CUDA(c, cudaMemcpyAsync(dst[k], src[k], bytes, cudaMemcpyHostToDevice, c->stream));
    // the uploaded state is FP64 primitive; MIXED steps convert it on use
    c->state_mode = ZG_FP64;
    c->cfl_valid = false;
    return ZG_OK;
}

int zg_state_download(zg_ctx *c, double *rho, double *vx, double *vy, double *p, double *e) {
    if (!c || !rho || !vx || !vy || !p || !e) return ZG_ERR_ARG;
    if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_state_download: solver not configured");
    DeviceGuard g(c->device);
    int rc = materialize_prim(c);
    if (rc != ZG_OK) return rc;
    size_t bytes = (size_t)c->n * sizeof(double);
    double *dst[5] = {rho, vx, vy, p, e};
    const double *src[5] = {c->z.r, c->z.u, c->z.v, c->z.p, c->z.e};
    for (int k = 0; k < 5; ++k)
        ZG_CUDA(c, cudaMemcpyAsync(dst[k], src[k], bytes, cudaMemcpyDeviceToHost, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_wait_upload(zg_ctx *c, const int *wait) {
    if (!c || !wait) return ZG_ERR_ARG;
    if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_wait_upload: solver not configured");
    DeviceGuard g(c->device);
    int rc = leave_order(c);
    if (rc != ZG_OK) return rc;
    ZG_CUDA(c, cudaMemcpyAsync(c->d_wait + (size_t)c->wait_cur * c->cap, wait, (size_t)c->n * sizeof(int),
                               cudaMemcpyHostToDevice, c->stream));
    return ZG_OK;
}

int zg_wait_download(zg_ctx *c, int *wait) {
    if (!c || !wait) return ZG_ERR_ARG;
    if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_wait_download: solver not configured");
    DeviceGuard g(c->device);
    int rc = leave_order(c);
    if (rc != ZG_OK) return rc;
    ZG_CUDA(c, cudaMemcpyAsync(wait, c->d_wait + (size_t)c->wait_cur * c->cap, (size_t)c->n * sizeof(int),
                               cudaMemcpyDeviceToHost, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_smf_update(zg_ctx *c) {
    if (!c) return ZG_ERR_ARG;
    if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_smf_update: solver not configured");
    DeviceGuard g(c->device);
    return enqueue_step(c);
}

int zg_smf_update_n(zg_ctx *c, int n_steps) {
    if (!c || n_steps < 0) return ZG_ERR_ARG;
    if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_smf_update_n: solver not configured");
    DeviceGuard g(c->device);
    for (int k = 0; k < n_steps; ++k) {
        int rc = enqueue_step(c);
        if (rc != ZG_OK) return rc;
    }
    return ZG_OK;
}

int zg_smf_dt(zg_ctx *c, double *dt) {
    if (!c || !dt) return ZG_ERR_ARG;
    if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_smf_dt: solver not configured");
    DeviceGuard g(c->device);
    ZG_CUDA(c, cudaMemcpyAsync(dt, c->d_dt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_smf_set_flags(zg_ctx *c, int *flags) {
    if (!c || (!flags && !c->amr)) return ZG_ERR_ARG;
    if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_smf_set_flags: solver not configured");
    DeviceGuard g(c->device);
    int rc = materialize_prim(c);
    if (rc != ZG_OK) return rc;
    SmfArgs a = make_args(c);
    // on an adaptive mesh the flags go to the mesh's own flag array, where
    // zg_amr_refine reads them (EuCell::set_flag)
    int *dflags = c->amr ? c->av.flag : c->d_flags;
    // an adaptive mesh also keeps the limited gradients of the state, which
    // the slope distributor of the next refine uses (compute_grad,
    // sm_fluid.cpp:521-522)
    if (c->amr) timed(c, ZG_K_GRAD, [&] { parity::launch_grad(a, c->z, true, (void *)c->stream); });
    if (c->amr) c->grad_ordered = false;  // gradients of the current state in the mesh's order
    timed(c, ZG_K_FLAGS, [&] { parity::launch_flags(a, dflags, c->slots, (void *)c->stream); });
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "flags kernel launch");
    if (!flags) return ZG_OK;
    ZG_CUDA(c, cudaMemcpyAsync(flags, dflags, (size_t)c->n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_state_rows(zg_ctx *c, int row0, int nrows, double *fields, int *wait, int put) {
    if (!c || !fields || !wait || nrows < 0) return ZG_ERR_ARG;
    if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_state_rows: solver not configured");
    if (c->nx <= 0 || c->slots) return fail(c, ZG_ERR_STATE, "zg_state_rows: rows of a rectangle mesh");
    if (c->par.precision != ZG_FP64) return fail(c, ZG_ERR_STATE, "zg_state_rows: the FP64 forms");
    if (row0 < 0 || row0 + nrows > c->nx) return fail(c, ZG_ERR_ARG, "zg_state_rows: rows out of range");
    DeviceGuard g(c->device);
    int rc = leave_order(c);
    if (rc != ZG_OK) return rc;
    const size_t off = (size_t)row0 * c->ny, cnt = (size_t)nrows * c->ny;
    double *fld[5] = {c->z.r, c->z.u, c->z.v, c->z.p, c->z.e};
    int *w = c->d_wait + (size_t)c->wait_cur * c->cap;
    // host or device buffers alike (unified addressing)
    for (int k = 0; k < 5; ++k) {
        if (put)
            ZG_CUDA(c, cudaMemcpyAsync(fld[k] + off, fields + k * cnt, cnt * sizeof(double), cudaMemcpyDefault,
                                       c->stream));
        else
            ZG_CUDA(c, cudaMemcpyAsync(fields + k * cnt, fld[k] + off, cnt * sizeof(double), cudaMemcpyDefault,
                                       c->stream));
    }
    if (put)
        ZG_CUDA(c, cudaMemcpyAsync(w + off, wait, cnt * sizeof(int), cudaMemcpyDefault, c->stream));
    else
        ZG_CUDA(c, cudaMemcpyAsync(wait, w + off, cnt * sizeof(int), cudaMemcpyDefault, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    if (put) c->cfl_valid = false;  // the next step takes its CFL minimum from the new rows
    return ZG_OK;
}

int zg_smf_cfl_min(zg_ctx *c, double *dmin) {
    if (!c || !dmin) return ZG_ERR_ARG;
    if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_smf_cfl_min: solver not configured");
    if (c->par.precision != ZG_FP64) return fail(c, ZG_ERR_STATE, "zg_smf_cfl_min: the FP64 forms");
    DeviceGuard g(c->device);
    int rc = leave_order(c);
    if (rc != ZG_OK) return rc;
    void *st = (void *)c->stream;
    if (c->par.kernels != ZG_KERNELS_PARITY && !c->slots) {
        // the FAST kernels' own CFL pass (the one their step runs after an upload)
        tiled::Fields<double> f = fast_fields(c);
        unsigned long long *slot = const_cast<unsigned long long *>(slot_ptr(c, 2));
        f.slot_cur = slot;
        cudaMemsetAsync(slot, 0x7F, sizeof(unsigned long long), c->stream);
        SmfArgs a = make_args(c);
        timed(c, ZG_K_DT, [&] { fast::launch_cfl(a, f, st); });
        unsigned long long bits = 0;
        ZG_CUDA(c, cudaMemcpyAsync(&bits, slot, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
        ZG_CUDA(c, cudaStreamSynchronize(c->stream));
        std::memcpy(dmin, &bits, sizeof(double));
        return ZG_OK;
    }
    // the parity dt kernel with CFL 1 and no cap: dt = 1 * min = min
    SmfArgs a = make_args(c);
    a.CFL = 1.0;
    a.max_dt = std::numeric_limits<double>::max();
    timed(c, ZG_K_DT, [&] { parity::launch_dt(a, c->z, c->slots, st); });
    ZG_CUDA(c, cudaMemcpyAsync(dmin, c->d_dt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_smf_gradients(zg_ctx *c, double *d_dx, double *d_dy) {
    if (!c || !d_dx || !d_dy) return ZG_ERR_ARG;
    if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_smf_gradients: solver not configured");
    DeviceGuard g(c->device);
    int rc = materialize_prim(c);
    if (rc != ZG_OK) return rc;
    SmfArgs a = make_args(c);
    timed(c, ZG_K_GRAD, [&] { parity::launch_grad(a, c->z, c->slots, (void *)c->stream); });
    c->grad_ordered = false;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "gradient kernel launch");
    const size_t n = (size_t)c->n;
    for (int k = 0; k < 4; ++k) {
        ZG_CUDA(c, cudaMemcpyAsync(d_dx + k * n, c->gx[k], n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        ZG_CUDA(c, cudaMemcpyAsync(d_dy + k * n, c->gy[k], n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_launch_count(const zg_ctx *c, long long *count) {
    if (!c || !count) return ZG_ERR_ARG;
    *count = c->launches;
    return ZG_OK;
}

int zg_synchronize(zg_ctx *c) {
    if (!c) return ZG_ERR_ARG;
    DeviceGuard g(c->device);
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_set_timing(zg_ctx *c, int on) {
    if (!c) return ZG_ERR_ARG;
    DeviceGuard g(c->device);
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    c->timing = on != 0;
    c->ev_pending.clear();
    c->ev_used = 0;
    return ZG_OK;
}

int zg_kernel_times(zg_ctx *c, double *ms, long long *launches) {
    if (!c) return ZG_ERR_ARG;
    DeviceGuard g(c->device);
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    if (ms)
        for (int k = 0; k < ZG_K_COUNT; ++k) ms[k] = 0.0;
    if (launches)
        for (int k = 0; k < ZG_K_COUNT; ++k) launches[k] = 0;
    for (auto &pe : c->ev_pending) {
        float t = 0.0f;
        ZG_CUDA(c, cudaEventElapsedTime(&t, c->ev_pool[pe.second], c->ev_pool[pe.second + 1]));
        if (ms) ms[pe.first] += t;
        if (launches) launches[pe.first] += 1;
    }
    c->ev_pending.clear();
    c->ev_used = 0;
    return ZG_OK;
}

const char *zg_kernel_name(int kind) {
    static const char *names[ZG_K_COUNT] = {"dt", "flux1", "grad", "stage1", "stage2", "heun_a", "heun_b",
                                            "flags", "mm_dt", "mm_recover", "mm_flux", "mm_crp",
                                            "mm_closure", "tr_dt", "tr_flux", "tr_update", "tr_normals",
                                            "tr_adjust", "mm_grad", "mm_stage1", "mm_stage2", "step"};
    return (kind >= 0 && kind < ZG_K_COUNT) ? names[kind] : "unknown";
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Multi-material step (MmFluid)

namespace {

// Unit literals of phys/literals.h: the value is double(x * factor) computed
// in long double, x the literal as a long double.
double lit(long double x, double factor) { return double(x * factor); }
double lit_C(long double x) { return double(x + 273.15); }

double ideal_ref_density(double gamma, double Cv, double P, double T) {
    return 1.0 / (((gamma - 1.0) * Cv * T) / P);  // 1 / IdealGas::volume_PT(P, T)
}

mmf::MmArgs make_mm_args(const zg_ctx *c) {
    mmf::MmArgs a{};
    a.mesh = c->mesh;
    for (int i = 0; i < mmf::NMAT; ++i) {
        const zg_material &m = c->mpar.materials[i];
        a.mix.mat[i] = {m.kind == ZG_EOS_STIFFENED ? 1 : 0, m.gamma, m.P0, m.e0, m.Cv, m.T0, m.rho_ref};
        a.nrm_x[i] = c->mnx[i];
        a.nrm_y[i] = c->mny[i];
        a.off[i] = c->moff[i];
    }
    a.crp = c->mpar.crp_mode;
    a.fp32_flux = c->mpar.precision == ZG_MIXED ? 1 : 0;
    a.dir = 0;
    a.dt_scale = 1.0;
    a.CFL = c->mpar.CFL;
    a.max_dt = c->mpar.max_dt;
    a.z = c->mz;
    a.znext = c->mznext;
    a.dmin_bits = c->d_mm_scalars;
    a.dt_ticket = reinterpret_cast<unsigned int *>(c->d_mm_scalars + 1);
    a.dt_out = reinterpret_cast<double *>(c->d_mm_scalars + 2);
    a.err = reinterpret_cast<int *>(c->d_mm_scalars + 3);
    a.counts = c->d_mm_lists;
    a.list_crp = c->d_mm_lists + 8;
    a.list_closure = c->d_mm_lists + 8 + c->n;
    a.qbuf = c->d_mm_qbuf;
    a.fbuf = c->d_mm_qbuf + (4 + mmf::NMAT) * (size_t)c->n;
    a.fsig = a.fbuf + 8 * (4 + mmf::NMAT) * (size_t)c->n;
    a.fflag = reinterpret_cast<int *>(a.fsig + 4 * (size_t)c->n);
    a.acc = c->mpar.accuracy;
    a.limiter = c->mpar.limiter;
    a.grad_a = c->d_mm_grad_a;
    if (c->d_mm2) {
        const size_t n = (size_t)c->n;
        double *b = c->d_mm2;
        auto take = [&b, n]() {
            double *p0 = b;
            b += n;
            return p0;
        };
        mmf::MmField &h = a.zhalf;
        h.rho = take();
        h.vx = take();
        h.vy = take();
        h.P = take();
        h.e = take();
        h.T = take();
        for (int i = 0; i < mmf::NMAT; ++i) h.b[i] = take();
        for (int i = 0; i < mmf::NMAT; ++i) h.r[i] = take();
        for (int k = 0; k < mmf::NG; ++k) a.gx[k] = take();
        for (int k = 0; k < mmf::NG; ++k) a.gy[k] = take();
    }
    return a;
}

int mm_ready(zg_ctx *c, const char *who) {
    if (!c) return ZG_ERR_ARG;
    if (!c->mm_configured) return fail(c, ZG_ERR_STATE, std::string(who) + ": zg_mmf_configure first");
    return ZG_OK;
}

int mm_check_error(zg_ctx *c) {
    int err = 0;
    ZG_CUDA(c, cudaMemcpyAsync(&err, c->d_mm_scalars + 3, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    if (err & 2)
        return fail(c, ZG_ERR_NUMERIC, "MmFluid: CrpMode::MUSCL reached a composite face; the reference has no face "
                                       "fraction for it (alpha_sigma returns NaN, mm_fluid.cpp:245-250, and "
                                       "calc_crp_flux's assert rejects it, mm_fluid.cpp:276)");
    if (err) return fail(c, ZG_ERR_NUMERIC, "MmFluid: negative density, NaN flux or an unsupported composite "
                                            "Riemann configuration (the reference throws here)");
    return ZG_OK;
}

// MmFluid::update (mm_fluid.cpp:112-137): dt once (the dt kernel also
// empties the work lists), then integrate (139-170) over all faces, or over
// the x and y faces in turn with direction splitting.
int enqueue_mm_step(zg_ctx *c) {
    void *st = (void *)c->stream;
    int rc = ensure_side(c);
    if (rc != ZG_OK) return rc;
    const bool first_order = c->mpar.accuracy == 1;
    if (!first_order) {
        mmf::MmArgs a = make_mm_args(c);
        timed(c, ZG_K_MM_DT, [&] { mmf::launch_dt(a, st); });
    }
    int sub = 0;
    auto integrate = [&](int dir, double scale) {
        mmf::MmArgs a = make_mm_args(c);
        a.dir = dir;
        a.dt_scale = scale;
        if (!first_order && sub++ > 0) cudaMemsetAsync(a.counts, 0, 2 * sizeof(int), c->stream);  // empty work lists
        if (c->mpar.accuracy == 2) {
            // MmFluid::integrate, second order (mm_fluid.cpp:152-168)
            timed(c, ZG_K_MM_GRAD, [&] { mmf::launch_grad2(a, st); });
            if (c->mpar.crp_mode == ZG_CRP_MUSCL) timed(c, ZG_K_MM_GRAD, [&] { mmf::launch_grad_a(a, st); });
            if (c->mpar.crp_mode == ZG_CRP_PLIC) timed(c, ZG_K_MM_RECOVER, [&] { mmf::launch_recover(a, st); });
            timed(c, ZG_K_MM_STAGE1, [&] { mmf::launch_stage1(a, st); });
            timed(c, ZG_K_MM_STAGE2, [&] { mmf::launch_stage2(a, st); });
            std::swap(c->mz, c->mznext);
            return;
        }
        // First order, on two streams.  Side: empty the work lists, then
        // MmFluid::integrate's preparation (mm_fluid.cpp:139-150: the
        // volume-fraction gradients for MUSCL, the interface reconstruction
        // for PLIC) and the list of cells next to a mixed state, beside dt
        // (first sub-step; it leaves the lists alone here) on the main
        // stream.  Then the composite faces of the listed cells (side) beside
        // the pure-stencil cells (main); the two write disjoint data, and the
        // cell updates follow on the main stream once both are done.
        a.presorted = 1;
        cudaEventRecord(c->ev_fork, c->stream);
        cudaStreamWaitEvent(c->side, c->ev_fork, 0);
        cudaMemsetAsync(a.counts, 0, 2 * sizeof(int), c->side);
        cudaEventRecord(c->ev_cleared, c->side);
        if (c->mpar.crp_mode == ZG_CRP_MUSCL)
            timed_on(c, ZG_K_MM_GRAD, c->side, [&] { mmf::launch_grad_a(a, (void *)c->side); });
        if (c->mpar.crp_mode == ZG_CRP_PLIC)
            timed_on(c, ZG_K_MM_RECOVER, c->side, [&] { mmf::launch_recover(a, (void *)c->side); });
        timed_on(c, ZG_K_MM_FLUX, c->side, [&] { mmf::launch_classify(a, (void *)c->side); });
        if (sub++ == 0) {
            mmf::MmArgs d = a;
            d.keep_lists = 1;
            timed(c, ZG_K_MM_DT, [&] { mmf::launch_dt(d, st); });
        }
        cudaStreamWaitEvent(c->stream, c->ev_cleared, 0);  // the pure-stencil kernel appends to a list
        cudaEventRecord(c->ev_dt, c->stream);
        cudaStreamWaitEvent(c->side, c->ev_dt, 0);
        timed_on(c, ZG_K_MM_CRP, c->side, [&] { mmf::launch_crp_faces(a, (void *)c->side); });
        timed(c, ZG_K_MM_FLUX, [&] { mmf::launch_flux_pure(a, st); });
        cudaEventRecord(c->ev_join, c->side);
        cudaStreamWaitEvent(c->stream, c->ev_join, 0);
        timed(c, ZG_K_MM_CRP, [&] { mmf::launch_crp_update(a, st); });
        timed(c, ZG_K_MM_CLOSURE, [&] { mmf::launch_closure(a, st); });
        std::swap(c->mz, c->mznext);  // MmFluid::swap (mm_fluid.cpp:682-684)
    };
    if (c->mpar.split == ZG_SPLIT_SIMPLE) {
        integrate(1, 1.0);
        integrate(2, 1.0);
    } else if (c->mpar.split == ZG_SPLIT_STRANG) {
        integrate(1, 0.5);
        integrate(2, 1.0);
        integrate(1, 0.5);
    } else {
        integrate(0, 1.0);
    }
    if (c->mpar.crp_mode == ZG_CRP_MUSCL) c->mm_grad_a_valid = true;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
    return ZG_OK;
}

}  // namespace

extern "C" {

int zg_material_named(int kind, const char *name, zg_material *out) {
    if (!name || !out) return ZG_ERR_ARG;
    std::string n(name);
    zg_material m{};
    if (kind == ZG_EOS_IDEAL) {  // ideal_gas.cpp:14-24
        m.kind = ZG_EOS_IDEAL;
        if (n == "Air") {
            m.gamma = 1.4;
            m.Cv = lit(718.0L, 1.0);
        } else if (n == "SF6") {
            m.gamma = 1.1074;
            m.Cv = lit(567.0L, 1.0);
        } else {
            return ZG_ERR_ARG;
        }
        m.rho_ref = ideal_ref_density(m.gamma, m.Cv, lit(1.0L, 1.0e5), lit_C(0.0L));
        *out = m;
        return ZG_OK;
    }
    if (kind != ZG_EOS_STIFFENED) return ZG_ERR_ARG;
    // stiffened_gas.cpp:13-86: defaults, then the named set
    m.kind = ZG_EOS_STIFFENED;
    m.P0 = 0.0;
    m.e0 = 0.0;
    m.Cv = 1.0;
    m.T0 = 0.0;
    double rho_0 = 1.0;
    if (n == "Air") {
        m.gamma = 1.4;
        m.Cv = lit(718.0L, 1.0);
        rho_0 = lit(1.25L, 1.0);
    } else if (n == "SF6") {
        m.gamma = 1.1074;
        m.Cv = lit(567.0L, 1.0);
        rho_0 = lit(6.17L, 1.0);
    } else if (n == "Water") {
        m.gamma = 4.4;
        m.Cv = lit(4160.0L, 1.0);
        m.P0 = lit(600.0L, 1.0e6);
        m.e0 = 0.0;
        m.T0 = 230.7;
        rho_0 = lit(1.0L, 1.0e3);
    } else if (n == "Water2") {
        m.gamma = 3.0;
        m.Cv = lit(4160.0L, 1.0);
        m.P0 = lit(853.3L, 1.0e6);
        m.e0 = -lit(1.148L, 1.0e6);
        rho_0 = lit(1.0L, 1.0e3);
    } else if (n == "Copper" || n == "Cu") {
        m.gamma = 4.0;
        m.Cv = lit(384.0L, 1.0);
        m.P0 = 341.0;
        m.e0 = 0.0;
        rho_0 = lit(8.96L, 1.0e3);
    } else if (n == "Lead" || n == "Pb") {
        m.gamma = 3.77;
        m.Cv = lit(121.0L, 1.0);
        m.P0 = lit(11.8L, 1.0e9);
        m.e0 = -lit(1.42L, 1.0e6);
        m.T0 = -2832.57;
        rho_0 = lit(11.35L, 1.0e3);
    } else if (n == "Gas") {
        m.gamma = 1.4;
        m.Cv = 2.5;
        rho_0 = 1.0;
    } else if (n == "HeavyGas") {
        m.gamma = 1.1;
        m.Cv = 2.5;
        rho_0 = 4.0;
    } else if (n == "Liquid") {
        m.gamma = 4.4;
        m.Cv = 20.0;
        m.P0 = 6.8e4;
        rho_0 = 1000.0;
    } else if (n == "Solid") {
        m.gamma = 3.8;
        m.Cv = 0.5;
        m.P0 = 1.4e5;
        m.e0 = -15.0;
        m.T0 = -7.0;
        rho_0 = 12500;
    } else {
        return ZG_ERR_ARG;
    }
    m.rho_ref = rho_0;
    *out = m;
    return ZG_OK;
}

void zg_mmf_default_params(zg_mmf_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->n_materials = 0;
    p->crp_mode = ZG_CRP_PLIC;
    p->accuracy = 1;
    p->CFL = 0.7;
    p->max_dt = 1.0e+300;
    p->limiter = ZG_LIM_MC;  // mm_fluid.cpp:20
}

int zg_mmf_configure(zg_ctx *c, const zg_mmf_params *p) {
    if (!c || !p) return ZG_ERR_ARG;
    if (!c->have_mesh || c->slots) return fail(c, ZG_ERR_STATE, "zg_mmf_configure: needs a zg_mesh_rectangle mesh");
    if (p->n_materials != mmf::NMAT)
        return fail(c, ZG_ERR_ARG, "zg_mmf_configure: the kernels are compiled for mixtures of two materials");
    for (int i = 0; i < p->n_materials; ++i) {
        const zg_material &m = p->materials[i];
        if ((m.kind != ZG_EOS_IDEAL && m.kind != ZG_EOS_STIFFENED) || !(m.gamma > 1.0) || !(m.Cv > 0.0))
            return fail(c, ZG_ERR_ARG, "zg_mmf_configure: invalid material");
    }
    if (p->precision != ZG_FP64 && p->precision != ZG_MIXED)
        return fail(c, ZG_ERR_ARG, "zg_mmf_configure: unknown precision");
    if (p->split < ZG_SPLIT_NONE || p->split > ZG_SPLIT_STRANG)
        return fail(c, ZG_ERR_ARG, "zg_mmf_configure: unknown direction splitting");
    if (p->crp_mode < ZG_CRP_NONE || p->crp_mode > ZG_CRP_MUSCL)
        return fail(c, ZG_ERR_ARG, "zg_mmf_configure: unknown CRP mode");
    const int acc = std::min(std::max(1, p->accuracy), 2);  // mm_fluid.cpp:46-48
    if (acc == 2 && p->precision != ZG_FP64 && p->crp_mode == ZG_CRP_NONE)
        return fail(c, ZG_ERR_ARG, "zg_mmf_configure: the mixed second-order form runs with a CRP mode (its "
                                   "FP32 faces are those whose reconstructed states stay pure)");
    if (p->limiter < ZG_LIM_NONE || p->limiter > ZG_LIM_SUPERBEE)
        return fail(c, ZG_ERR_ARG, "zg_mmf_configure: unknown limiter");
    DeviceGuard g(c->device);
    c->mpar = *p;
    c->mpar.accuracy = acc;
    if (acc == 2 && !c->d_mm2) {
        // half-step state and the limited gradients (x, y) of the state
        constexpr int NF = 6 + 2 * mmf::NMAT;
        const size_t n2 = (size_t)c->n;
        ZG_CUDA(c, cudaMalloc(&c->d_mm2, (NF + 2 * mmf::NG) * n2 * sizeof(double)));
        ZG_CUDA(c, cudaMemsetAsync(c->d_mm2, 0, (NF + 2 * mmf::NG) * n2 * sizeof(double), c->stream));
    }
    if (p->crp_mode == ZG_CRP_MUSCL && !c->d_mm_grad_a)
        ZG_CUDA(c, cudaMalloc(&c->d_mm_grad_a, 2 * mmf::NMAT * (size_t)c->n * sizeof(double)));
    c->mpar.CFL = std::max(0.0, std::min(p->CFL, 1.0));  // mm_fluid.cpp:43-45
    if (c->mm_configured) return ZG_OK;
    size_t n = (size_t)c->n;
    constexpr int NF = 6 + 2 * mmf::NMAT;
    ZG_CUDA(c, cudaMalloc(&c->d_mm, (2 * NF + 3 * mmf::NMAT) * n * sizeof(double)));
    ZG_CUDA(c, cudaMalloc(&c->d_mm_scalars, 64));
    ZG_CUDA(c, cudaMalloc(&c->d_mm_flags, n * sizeof(int)));
    ZG_CUDA(c, cudaMalloc(&c->d_mm_lists, (2 * n + 8) * sizeof(int)));
    // closure q; two face parts per face (4 per cell); a_sig and flags per face
    ZG_CUDA(c, cudaMalloc(&c->d_mm_qbuf, (9 * (4 + mmf::NMAT) + 4 + 2) * n * sizeof(double)));
    ZG_CUDA(c, cudaMemsetAsync(c->d_mm_lists, 0, (2 * n + 8) * sizeof(int), c->stream));
    double *b = c->d_mm;
    auto take = [&b, n]() {
        double *p0 = b;
        b += n;
        return p0;
    };
    for (mmf::MmField *f : {&c->mz, &c->mznext}) {
        f->rho = take();
        f->vx = take();
        f->vy = take();
        f->P = take();
        f->e = take();
        f->T = take();
        for (int i = 0; i < mmf::NMAT; ++i) f->b[i] = take();
        for (int i = 0; i < mmf::NMAT; ++i) f->r[i] = take();
    }
    for (int i = 0; i < mmf::NMAT; ++i) {
        c->mnx[i] = take();
        c->mny[i] = take();
        c->moff[i] = take();
    }
    ZG_CUDA(c, cudaMemsetAsync(c->d_mm, 0, (2 * NF + 3 * mmf::NMAT) * n * sizeof(double), c->stream));
    unsigned long long init[4] = {0x7FEFFFFFFFFFFFFFull, 0ull, 0ull, 0ull};
    ZG_CUDA(c, cudaMemcpyAsync(c->d_mm_scalars, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    c->mm_configured = true;
    return ZG_OK;
}

int zg_mmf_state_upload(zg_ctx *c, const double *cells) {
    int rc = mm_ready(c, "zg_mmf_state_upload");
    if (rc != ZG_OK) return rc;
    if (!cells) return fail(c, ZG_ERR_ARG, "zg_mmf_state_upload: null array");
    size_t n = (size_t)c->n;
    constexpr int NF = 6 + 2 * mmf::NMAT;
    std::vector<double> soa(NF * n);
    for (size_t i = 0; i < n; ++i) {
        const double *s = cells + 14 * i;
        for (int k = mmf::NMAT; k < 4; ++k)
            if (s[6 + k] != 0.0) return fail(c, ZG_ERR_ARG, "zg_mmf_state_upload: fraction of an absent material");
        for (int k = 0; k < 6; ++k) soa[k * n + i] = s[k];
        for (int k = 0; k < mmf::NMAT; ++k) {
            soa[(6 + k) * n + i] = s[6 + k];
            soa[(6 + mmf::NMAT + k) * n + i] = s[10 + k];
        }
    }
    DeviceGuard g(c->device);
    ZG_CUDA(c, cudaMemcpyAsync(c->mz.rho, soa.data(), soa.size() * sizeof(double), cudaMemcpyHostToDevice,
                               c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_mmf_state_download(zg_ctx *c, double *cells) {
    int rc = mm_ready(c, "zg_mmf_state_download");
    if (rc != ZG_OK) return rc;
    if (!cells) return fail(c, ZG_ERR_ARG, "zg_mmf_state_download: null array");
    DeviceGuard g(c->device);
    size_t n = (size_t)c->n;
    std::vector<double *> fields = {c->mz.rho, c->mz.vx, c->mz.vy, c->mz.P, c->mz.e, c->mz.T};
    for (int k = 0; k < mmf::NMAT; ++k) fields.push_back(c->mz.b[k]);
    for (int k = 0; k < mmf::NMAT; ++k) fields.push_back(c->mz.r[k]);
    std::vector<double> soa(fields.size() * n);
    for (size_t k = 0; k < fields.size(); ++k)
        ZG_CUDA(c, cudaMemcpyAsync(soa.data() + k * n, fields[k], n * sizeof(double), cudaMemcpyDeviceToHost,
                                   c->stream));
    rc = mm_check_error(c);
    const double nan = std::numeric_limits<double>::quiet_NaN();
    for (size_t i = 0; i < n; ++i) {
        double *s = cells + 14 * i;
        for (int k = 0; k < 6; ++k) s[k] = soa[k * n + i];
        for (int k = 0; k < 4; ++k) {
            s[6 + k] = k < mmf::NMAT ? soa[(6 + k) * n + i] : 0.0;
            s[10 + k] = k < mmf::NMAT ? soa[(6 + mmf::NMAT + k) * n + i] : nan;
        }
    }
    return rc;
}

int zg_mmf_grad_a(zg_ctx *c, double *out) {
    int rc = mm_ready(c, "zg_mmf_grad_a");
    if (rc != ZG_OK) return rc;
    if (!out) return fail(c, ZG_ERR_ARG, "zg_mmf_grad_a: null array");
    if (c->mpar.crp_mode != ZG_CRP_MUSCL || !c->mm_grad_a_valid)
        return fail(c, ZG_ERR_STATE, "zg_mmf_grad_a: computed by the steps of CrpMode::MUSCL only");
    DeviceGuard g(c->device);
    const size_t n = (size_t)c->n;
    std::vector<double> soa(2 * mmf::NMAT * n);
    ZG_CUDA(c, cudaMemcpyAsync(soa.data(), c->d_mm_grad_a, soa.size() * sizeof(double), cudaMemcpyDeviceToHost,
                               c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 2 * mmf::NMAT; ++k) out[2 * mmf::NMAT * i + k] = soa[k * n + i];
    return ZG_OK;
}

int zg_mmf_make_states(zg_ctx *c, const double *rho, const double *vx, const double *vy, const double *p,
                       const double *beta) {
    int rc = mm_ready(c, "zg_mmf_make_states");
    if (rc != ZG_OK) return rc;
    if (!rho || !vx || !vy || !p || !beta) return fail(c, ZG_ERR_ARG, "zg_mmf_make_states: null array");
    DeviceGuard g(c->device);
    size_t n = (size_t)c->n;
    for (size_t i = 0; i < n; ++i)
        for (int k = mmf::NMAT; k < 4; ++k)
            if (beta[4 * i + k] != 0.0) return fail(c, ZG_ERR_ARG, "zg_mmf_make_states: fraction of an absent material");
    // staging: rho, vx, vy, p (n each) and beta (4 n) in the next-state buffer's fields
    double *tmp = nullptr;
    ZG_CUDA(c, cudaMalloc(&tmp, 8 * n * sizeof(double)));
    const double *src[4] = {rho, vx, vy, p};
    for (int k = 0; k < 4; ++k)
        ZG_CUDA(c, cudaMemcpyAsync(tmp + k * n, src[k], n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    ZG_CUDA(c, cudaMemcpyAsync(tmp + 4 * n, beta, 4 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    mmf::MmArgs a = make_mm_args(c);
    mmf::launch_make_states(a, tmp, tmp + n, tmp + 2 * n, tmp + 3 * n, tmp + 4 * n, (void *)c->stream);
    ++c->launches;
    cudaError_t e = cudaGetLastError();
    cudaError_t s = cudaStreamSynchronize(c->stream);
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(c, e, "zg_mmf_make_states launch");
    if (s != cudaSuccess) return cuda_fail(c, s, "zg_mmf_make_states");
    return ZG_OK;
}

int zg_mmf_update(zg_ctx *c) { return zg_mmf_update_n(c, 1); }

int zg_mmf_update_n(zg_ctx *c, int n_steps) {
    int rc = mm_ready(c, "zg_mmf_update");
    if (rc != ZG_OK) return rc;
    if (n_steps < 0) return fail(c, ZG_ERR_ARG, "zg_mmf_update_n: negative step count");
    DeviceGuard g(c->device);
    for (int k = 0; k < n_steps; ++k) {
        rc = enqueue_mm_step(c);
        if (rc != ZG_OK) return rc;
    }
    return ZG_OK;
}

int zg_mmf_dt(zg_ctx *c, double *dt) {
    int rc = mm_ready(c, "zg_mmf_dt");
    if (rc != ZG_OK) return rc;
    if (!dt) return ZG_ERR_ARG;
    DeviceGuard g(c->device);
    ZG_CUDA(c, cudaMemcpyAsync(dt, c->d_mm_scalars + 2, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return mm_check_error(c);
}

int zg_mmf_set_flags(zg_ctx *c, int *flags) {
    int rc = mm_ready(c, "zg_mmf_set_flags");
    if (rc != ZG_OK) return rc;
    if (!flags) return ZG_ERR_ARG;
    DeviceGuard g(c->device);
    mmf::MmArgs a = make_mm_args(c);
    mmf::launch_flags(a, c->d_mm_flags, (void *)c->stream);
    ++c->launches;
    ZG_CUDA(c, cudaGetLastError());
    ZG_CUDA(c, cudaMemcpyAsync(flags, c->d_mm_flags, (size_t)c->n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_mmf_interface(zg_ctx *c, double *normals, double *offsets) {
    int rc = mm_ready(c, "zg_mmf_interface");
    if (rc != ZG_OK) return rc;
    if (!normals || !offsets) return ZG_ERR_ARG;
    DeviceGuard g(c->device);
    mmf::MmArgs a = make_mm_args(c);
    mmf::launch_recover(a, (void *)c->stream);
    ++c->launches;
    ZG_CUDA(c, cudaGetLastError());
    size_t n = (size_t)c->n;
    std::vector<double> buf(3 * mmf::NMAT * n);
    for (int i = 0; i < mmf::NMAT; ++i) {
        ZG_CUDA(c, cudaMemcpyAsync(buf.data() + (3 * i) * n, c->mnx[i], n * sizeof(double), cudaMemcpyDeviceToHost,
                                   c->stream));
        ZG_CUDA(c, cudaMemcpyAsync(buf.data() + (3 * i + 1) * n, c->mny[i], n * sizeof(double),
                                   cudaMemcpyDeviceToHost, c->stream));
        ZG_CUDA(c, cudaMemcpyAsync(buf.data() + (3 * i + 2) * n, c->moff[i], n * sizeof(double),
                                   cudaMemcpyDeviceToHost, c->stream));
    }
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    for (size_t ic = 0; ic < n; ++ic)
        for (int i = 0; i < mmf::NMAT; ++i) {
            normals[(ic * mmf::NMAT + i) * 2] = buf[(3 * i) * n + ic];
            normals[(ic * mmf::NMAT + i) * 2 + 1] = buf[(3 * i + 1) * n + ic];
            offsets[ic * mmf::NMAT + i] = buf[(3 * i + 2) * n + ic];
        }
    return ZG_OK;
}

// ---------------------------------------------------------------------------
// Scalar VOF transport (Transfer, math/solver/transfer.cpp)

void zg_tr_default_params(zg_tr_params *p) {
    if (!p) return;
    *p = zg_tr_params{};
    p->method = ZG_TR_VOF;  // transfer.cpp:44-49
    p->CFL = 0.5;
    p->velocity = ZG_TR_TRANSLATION;  // Transfer::velocity: Vector3d::UnitX() (transfer.cpp:84-86)
    p->vel[0] = 1.0;
}

}  // extern "C"

namespace {

int tr_ready(zg_ctx *c, const char *who) {
    if (!c) return ZG_ERR_ARG;
    if (!c->tr_configured) return fail(c, ZG_ERR_STATE, std::string(who) + ": zg_tr_configure first");
    return ZG_OK;
}

// scalar slots after the fields: dt, time, CFL minimum bits, ticket, error
// counter, the two work-list lengths
enum { TR_DT = 0, TR_TIME = 1, TR_DMIN = 2, TR_TICKET = 3, TR_ERR = 4, TR_COUNT = 5, TR_NSCALAR = 8 };

int tr_check_error(zg_ctx *c) {
    int err = 0;
    ZG_CUDA(c, cudaMemcpyAsync(&err, c->targs.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    if (err) return fail(c, ZG_ERR_NUMERIC, "Transfer: a clipped polygon exceeded the kernels' vertex capacity");
    return ZG_OK;
}

// InterfaceRecovery::update (interface_recovery.cpp:106-113)
void tr_interface(zg_ctx *c, int smoothing) {
    tr::TrArgs &a = c->targs;
    timed(c, ZG_K_TR_NORMALS, [&] { tr::launch_normals(a, c->stream); });
    for (int k = 0; k < smoothing; ++k) {
        timed(c, ZG_K_TR_ADJUST, [&] { tr::launch_adjust(a, c->stream); });
        a.cur = 1 - a.cur;
    }
}

// Transfer::update (transfer.cpp:471-666): the MUSCL slopes, fluxes,
// update (one kernel for WENO), reconstruction (three smoothing passes for
// the VOF, MUSCL and WENO methods, none for CRP).
void tr_update(zg_ctx *c, int dir) {
    const tr::TrArgs &a = c->targs;
    const int m = c->tpar.method;
    if (tr::weno_type(m)) {
        timed(c, ZG_K_TR_FLUX, [&] { tr::launch_weno(a, dir, c->stream); });
    } else {
        if (tr::muscl_type(m)) timed(c, ZG_K_TR_FLUX, [&] { tr::launch_slopes(a, c->stream); });
        timed(c, ZG_K_TR_FLUX, [&] { tr::launch_flux(a, dir, c->stream); });
        timed(c, ZG_K_TR_UPDATE, [&] { tr::launch_apply(a, dir, c->stream); });
    }
    std::swap(c->targs.u, c->targs.u_next);
    tr_interface(c, tr::vof_type(m) || tr::muscl_type(m) || tr::weno_type(m) ? 3 : 0);
}

void tr_dt(zg_ctx *c, bool advance, double t_end) {
    timed(c, ZG_K_TR_DT, [&] { tr::launch_compute_dt(c->targs, advance, t_end, c->stream); });
}

}  // namespace

extern "C" {

int zg_tr_configure(zg_ctx *c, const zg_tr_params *p) {
    if (!c || !p) return ZG_ERR_ARG;
    if (!c->have_mesh || c->slots || c->amr)
        return fail(c, ZG_ERR_STATE, "zg_tr_configure: needs a zg_mesh_rectangle mesh (not adaptive)");
    if (c->mesh.xper || c->mesh.yper)
        return fail(c, ZG_ERR_ARG, "zg_tr_configure: periodic boundaries are not supported (the reference clips "
                                   "the upwind cell's polygon across the domain there)");
    if (p->method < ZG_TR_CRP_V3 || p->method > ZG_TR_WENO_CRP)
        return fail(c, ZG_ERR_ARG, "zg_tr_configure: unknown method");
    if (tr::weno_type(p->method) && (c->mesh.nx < 3 || c->mesh.ny < 3))
        return fail(c, ZG_ERR_ARG, "zg_tr_configure: WENO needs at least 3 cells per axis (its stencil wraps "
                                   "indices once, as EuMesh::operator() does)");
    if (p->velocity != ZG_TR_TRANSLATION && p->velocity != ZG_TR_ROTATION)
        return fail(c, ZG_ERR_ARG, "zg_tr_configure: unknown velocity field");
    DeviceGuard g(c->device);
    c->tpar = *p;
    c->tpar.CFL = std::max(0.0, std::min(p->CFL, 1.0));  // Transfer::set_CFL (transfer.cpp:65-67)
    tr::TrArgs &a = c->targs;
    a.m = tr::TrMesh{c->mesh.nx, c->mesh.ny, c->mesh.X,  c->mesh.Y,  c->mesh.cx, c->mesh.cy,
                     c->mesh.fxm, c->mesh.fym, c->mesh.hx, c->mesh.hy, c->mesh.vol};
    a.vel = tr::TrVel{p->velocity, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (p->velocity == ZG_TR_TRANSLATION) {
        a.vel.vx = p->vel[0];
        a.vel.vy = p->vel[1];
    } else {
        a.vel.cx = p->vel[0];
        a.vel.cy = p->vel[1];
        a.vel.w = p->vel[2];
    }
    a.method = p->method;
    a.CFL = c->tpar.CFL;
    a.limiter = LIM_MC;  // Transfer's m_limiter (transfer.cpp:47)
    if (c->tr_configured) return ZG_OK;

    const size_t n = (size_t)c->n, nx = (size_t)c->mesh.nx, ny = (size_t)c->mesh.ny;
    const size_t nfx = (nx + 1) * ny, nfy = nx * (ny + 1);
    // fields, then the scalars, then the work lists (ints): faces, cells
    const size_t total = 12 * n + 2 * nfx + 2 * nfy + TR_NSCALAR + (nfx + nfy + n + 1) / 2 + 1 + (n + 7) / 8;
    ZG_CUDA(c, cudaMalloc(&c->d_tr, total * sizeof(double)));
    ZG_CUDA(c, cudaMemsetAsync(c->d_tr, 0, total * sizeof(double), c->stream));
    double *b = c->d_tr;
    a.u = b;
    a.u_next = b + n;
    b += 2 * n;
    for (int k = 0; k < 2; ++k) {
        a.nx[k] = b;
        a.ny[k] = b + n;
        a.px[k] = b + 2 * n;
        a.py[k] = b + 3 * n;
        b += 4 * n;
    }
    a.cur = 0;
    a.gx = b;
    a.gy = b + n;
    b += 2 * n;
    a.fxa = b;
    a.fxb = b + nfx;
    b += 2 * nfx;
    a.fya = b;
    a.fyb = b + nfy;
    b += 2 * nfy;
    a.dt = b + TR_DT;
    a.time = b + TR_TIME;
    a.dmin = reinterpret_cast<unsigned long long *>(b + TR_DMIN);
    a.ticket = reinterpret_cast<unsigned int *>(b + TR_TICKET);
    a.err = reinterpret_cast<int *>(b + TR_ERR);
    a.count = reinterpret_cast<int *>(b + TR_COUNT);
    a.flist = reinterpret_cast<int *>(b + TR_NSCALAR);
    a.clist = a.flist + nfx + nfy;
    a.zero_np = reinterpret_cast<unsigned char *>(a.clist + n);
    double init[TR_NSCALAR] = {1.0e+300, 0.0, std::numeric_limits<double>::max(), 0.0, 0.0, 0.0, 0.0, 0.0};
    ZG_CUDA(c, cudaMemcpyAsync(b, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));  // dt 1e300 (transfer.cpp:45)
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    c->tr_configured = true;
    return ZG_OK;
}

int zg_tr_upload(zg_ctx *c, const double *u1) {
    int rc = tr_ready(c, "zg_tr_upload");
    if (rc != ZG_OK) return rc;
    if (!u1) return fail(c, ZG_ERR_ARG, "zg_tr_upload: null array");
    DeviceGuard g(c->device);
    ZG_CUDA(c, cudaMemcpyAsync(c->targs.u, u1, (size_t)c->n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_tr_download(zg_ctx *c, double *u1, double *nrm, double *pt) {
    int rc = tr_ready(c, "zg_tr_download");
    if (rc != ZG_OK) return rc;
    DeviceGuard g(c->device);
    const size_t n = (size_t)c->n;
    const tr::TrArgs &a = c->targs;
    std::vector<double> buf(4 * n);
    if (u1) ZG_CUDA(c, cudaMemcpyAsync(u1, a.u, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    // the current buffers' nx, ny, px, py are contiguous
    if (nrm || pt)
        ZG_CUDA(c, cudaMemcpyAsync(buf.data(), a.nx[a.cur], 4 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < n && (nrm || pt); ++i) {
        if (nrm) {
            nrm[2 * i] = buf[i];
            nrm[2 * i + 1] = buf[n + i];
        }
        if (pt) {
            pt[2 * i] = buf[2 * n + i];
            pt[2 * i + 1] = buf[3 * n + i];
        }
    }
    return tr_check_error(c);
}

int zg_tr_update_interface(zg_ctx *c, int smoothing) {
    int rc = tr_ready(c, "zg_tr_update_interface");
    if (rc != ZG_OK) return rc;
    if (smoothing < 0) return fail(c, ZG_ERR_ARG, "zg_tr_update_interface: negative smoothing");
    DeviceGuard g(c->device);
    tr_interface(c, smoothing);
    ZG_CUDA(c, cudaGetLastError());
    return ZG_OK;
}

int zg_tr_compute_dt(zg_ctx *c, double *dt) {
    int rc = tr_ready(c, "zg_tr_compute_dt");
    if (rc != ZG_OK) return rc;
    DeviceGuard g(c->device);
    tr_dt(c, false, 0.0);
    ZG_CUDA(c, cudaGetLastError());
    if (dt) {
        ZG_CUDA(c, cudaMemcpyAsync(dt, c->targs.dt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    return ZG_OK;
}

int zg_tr_set_dt(zg_ctx *c, double dt) {
    int rc = tr_ready(c, "zg_tr_set_dt");
    if (rc != ZG_OK) return rc;
    DeviceGuard g(c->device);
    ZG_CUDA(c, cudaMemcpyAsync(c->targs.dt, &dt, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_tr_get_dt(zg_ctx *c, double *dt) {
    int rc = tr_ready(c, "zg_tr_get_dt");
    if (rc != ZG_OK) return rc;
    if (!dt) return ZG_ERR_ARG;
    DeviceGuard g(c->device);
    ZG_CUDA(c, cudaMemcpyAsync(dt, c->targs.dt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_tr_update(zg_ctx *c, int dir) {
    int rc = tr_ready(c, "zg_tr_update");
    if (rc != ZG_OK) return rc;
    if (dir < ZG_DIR_ANY || dir > ZG_DIR_Y) return fail(c, ZG_ERR_ARG, "zg_tr_update: unknown direction");
    DeviceGuard g(c->device);
    tr_update(c, dir);
    ZG_CUDA(c, cudaGetLastError());
    return ZG_OK;
}

int zg_tr_advance(zg_ctx *c, int steps, int split, double t_end, double *time) {
    int rc = tr_ready(c, "zg_tr_advance");
    if (rc != ZG_OK) return rc;
    if (steps < 0 || !time) return fail(c, ZG_ERR_ARG, "zg_tr_advance: steps >= 0 and a time required");
    DeviceGuard g(c->device);
    ZG_CUDA(c, cudaMemcpyAsync(c->targs.time, time, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    for (int k = 0; k < steps; ++k) {
        tr_dt(c, true, t_end);
        if (split) {
            tr_update(c, ZG_DIR_X);
            tr_update(c, ZG_DIR_Y);
        } else {
            tr_update(c, ZG_DIR_ANY);
        }
    }
    ZG_CUDA(c, cudaGetLastError());
    ZG_CUDA(c, cudaMemcpyAsync(time, c->targs.time, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_tr_set_flags(zg_ctx *c, int *flags) {
    int rc = tr_ready(c, "zg_tr_set_flags");
    if (rc != ZG_OK) return rc;
    if (!flags) return fail(c, ZG_ERR_ARG, "zg_tr_set_flags: null array");
    DeviceGuard g(c->device);
    int *d = nullptr;
    ZG_CUDA(c, cudaMallocAsync(&d, (size_t)c->n * sizeof(int), c->stream));
    timed(c, ZG_K_FLAGS, [&] { tr::launch_flags(c->targs, d, c->stream); });
    cudaError_t e = cudaMemcpyAsync(flags, d, (size_t)c->n * sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    cudaFreeAsync(d, c->stream);
    if (e != cudaSuccess) return fail(c, ZG_ERR_CUDA, cudaGetErrorString(e));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Output: VTU files and PVD series (io/vtu_file.cpp, io/pvd_file.cpp)

struct zg_pvd {
    std::string filename;  // PvdFile::m_filename (the DataSet file prefix)
    std::string fullname;  // PvdFile::m_fullname (directory / filename)
    std::vector<double> steps;
};

namespace {

struct OutVar {
    std::string name, type;
    int comps = 1;
    size_t elem = 8;  // bytes per component
    int kind = -1;    // vtu::Kind, or -1: a Float64 array copied as is
    const double *a = nullptr, *b = nullptr;  // device fields
    const double *host = nullptr;
};

// The device state field of a source, or null with an error.
int out_field(zg_ctx *c, const zg_out_var &v, OutVar &o) {
    const int k = v.component;
    if (v.source == ZG_OUT_SMF) {
        if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_vtu_write: no SmFluid state (zg_smf_configure)");
        int rc = materialize_prim(c);
        if (rc != ZG_OK) return rc;
        double *f[5] = {c->z.r, c->z.u, c->z.v, c->z.p, c->z.e};
        if (k < 0 || k > 4) return fail(c, ZG_ERR_ARG, "zg_vtu_write: SmFluid component 0..4");
        o.a = f[k];
        return ZG_OK;
    }
    if (v.source == ZG_OUT_MMF) {
        if (!c->mm_configured) return fail(c, ZG_ERR_STATE, "zg_vtu_write: no MmFluid state (zg_mmf_configure)");
        const mmf::MmField &z = c->mz;
        double *f[6 + 2 * mmf::NMAT] = {z.rho, z.vx, z.vy, z.P, z.e, z.T};
        for (int i = 0; i < mmf::NMAT; ++i) {
            f[6 + i] = z.b[i];
            f[6 + mmf::NMAT + i] = z.r[i];
        }
        if (k < 0 || k >= 6 + 2 * mmf::NMAT) return fail(c, ZG_ERR_ARG, "zg_vtu_write: MmFluid component out of range");
        o.a = f[k];
        return ZG_OK;
    }
    if (v.source == ZG_OUT_TR) {
        if (!c->tr_configured) return fail(c, ZG_ERR_STATE, "zg_vtu_write: no Transfer state (zg_tr_configure)");
        const tr::TrArgs &t = c->targs;
        const int q = t.cur;
        if (k == 5 || k == 6) {
            o.kind = vtu::K_VEC3;
            o.comps = 3;
            o.a = k == 5 ? t.nx[q] : t.px[q];
            o.b = k == 5 ? t.ny[q] : t.py[q];
            return ZG_OK;
        }
        double *f[5] = {t.u, t.nx[q], t.ny[q], t.px[q], t.py[q]};
        if (k < 0 || k > 4) return fail(c, ZG_ERR_ARG, "zg_vtu_write: Transfer component 0..6");
        o.a = f[k];
        return ZG_OK;
    }
    return fail(c, ZG_ERR_ARG, "zg_vtu_write: unknown variable source");
}

int out_vars(zg_ctx *c, const zg_out_var *vars, int n_vars, std::vector<OutVar> &out) {
    if (n_vars < 0 || (n_vars > 0 && !vars)) return fail(c, ZG_ERR_ARG, "zg_vtu_write: bad variable list");
    for (int i = 0; i < n_vars; ++i) {
        const zg_out_var &v = vars[i];
        if (!v.name) return fail(c, ZG_ERR_ARG, "zg_vtu_write: variable without a name");
        OutVar o;
        o.name = v.name;
        o.type = "Float64";
        // io::Variable's named variables: types and sizes of io/variable.cpp
        switch (v.source) {
            case ZG_OUT_LEVEL: o.kind = vtu::K_LEVEL; o.type = "Int8"; o.elem = 1; break;
            case ZG_OUT_INDEX: o.kind = vtu::K_INDEX; o.type = "Int32"; o.elem = 4; break;
            case ZG_OUT_RANK: o.kind = vtu::K_RANK; o.type = "Int32"; o.elem = 4; break;
            case ZG_OUT_FLAG: o.kind = vtu::K_FLAG; o.type = "Int8"; o.elem = 1; break;
            case ZG_OUT_B_IDX: o.kind = vtu::K_BIDX; o.type = "Int32"; o.elem = 4; break;
            case ZG_OUT_Z_IDX: o.kind = vtu::K_ZIDX; o.type = "Int32"; o.elem = 4; break;
            case ZG_OUT_CENTER: o.kind = vtu::K_CENTER; o.type = "Float32"; o.elem = 4; o.comps = 3; break;
            case ZG_OUT_HOST:
                if (!v.host) return fail(c, ZG_ERR_ARG, "zg_vtu_write: ZG_OUT_HOST without an array");
                o.host = v.host;
                break;
            default: {
                int rc = out_field(c, v, o);
                if (rc != ZG_OK) return rc;
            }
        }
        out.push_back(o);
    }
    return ZG_OK;
}

// VtuStructure::write_header + write_primitives + write_cells_data
// (vtu_file.cpp:439-530) for quadrilateral cells: the header text, then the
// appended arrays, each behind its uint32 byte count, packed on the device.
int vtu_write(zg_ctx *c, const std::string &filename, const zg_out_var *vars, int n_vars) {
    if (!c->have_mesh || (c->slots && !c->amr))
        return fail(c, ZG_ERR_STATE, "zg_vtu_write: needs a zg_mesh_rectangle mesh (adaptive or not)");
    DeviceGuard g(c->device);
    std::vector<OutVar> vs;
    int rc = out_vars(c, vars, n_vars, vs);
    if (rc != ZG_OK) return rc;
    const size_t n = (size_t)c->n, np = 4 * n;
    if (np > 0xFFFFFFFFull / 24) return fail(c, ZG_ERR_ARG, "zg_vtu_write: mesh too large for 32-bit VTU offsets");

    vtu::MeshSrc m{};
    m.n = (int)n;
    if (c->amr) {
        m.kind = 1;
        m.mvx = c->av.vx;
        m.mvy = c->av.vy;
        m.cx = c->av.cx;
        m.cy = c->av.cy;
        m.level = c->av.level;
        m.b_idx = c->av.b_idx;
        m.z_idx = c->av.z_idx;
        m.flag = c->av.flag;
    } else {
        m.kind = 0;
        m.ny = c->mesh.ny;
        m.X = c->mesh.X;
        m.Y = c->mesh.Y;
        m.cxt = c->mesh.cx;
        m.cyt = c->mesh.cy;
        m.flag = c->configured ? c->d_flags : nullptr;
    }

    // header (byte offsets count each array's uint32 size field)
    std::ostringstream h;
    h << "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
    h << "  <UnstructuredGrid>\n";
    h << "    <Piece NumberOfPoints=\"" << np << "\" NumberOfCells=\"" << n << "\">\n";
    uint64_t off = 0;
    h << "      <Points>\n";
    h << "        <DataArray type=\"Float64\" Name=\"Points\" NumberOfComponents=\"3\" format=\"appended\" offset=\""
      << off << "\"/>\n";
    h << "      </Points>\n";
    const size_t b_pts = 24 * np, b_conn = 4 * np, b_off = 4 * n, b_types = n;
    off += 4 + b_pts;
    h << "      <Cells>\n";
    h << "        <DataArray type=\"UInt32\" Name=\"connectivity\" format=\"appended\" offset=\"" << off << "\"/>\n";
    off += 4 + b_conn;
    h << "        <DataArray type=\"UInt32\" Name=\"offsets\" format=\"appended\" offset=\"" << off << "\"/>\n";
    off += 4 + b_off;
    h << "        <DataArray type=\"UInt8\" Name=\"types\" format=\"appended\" offset=\"" << off << "\"/>\n";
    off += 4 + b_types;
    h << "      </Cells>\n";
    h << "      <CellData>\n";
    for (const OutVar &v : vs) {
        h << "        <DataArray type=\"" << v.type << "\" Name=\"" << v.name;
        if (v.comps >= 2) h << "\" NumberOfComponents=\"" << v.comps;
        h << "\" format=\"appended\" offset=\"" << off << "\"/>\n";
        off += 4 + n * v.comps * v.elem;
    }
    h << "      </CellData>\n";
    h << "    </Piece>\n";
    h << "  </UnstructuredGrid>\n";
    h << "  <AppendedData encoding=\"raw\">\n";
    h << "_";
    if (off > 0xFFFFFFFFull) return fail(c, ZG_ERR_ARG, "zg_vtu_write: file too large for 32-bit VTU offsets");
    const std::string head = h.str();

    // appended data: the device packs each array, one copy each into a
    // pinned host image of the file's tail
    std::vector<size_t> sizes = {b_pts, b_conn, b_off, b_types};
    for (const OutVar &v : vs) sizes.push_back(n * v.comps * v.elem);
    size_t total = 0, dev_total = 0;
    for (size_t sz : sizes) {
        total += 4 + sz;
        dev_total += (sz + 255) / 256 * 256;
    }
    if (c->out_img_size < total) {
        if (c->out_img) cudaFreeHost(c->out_img);
        c->out_img = nullptr;
        c->out_img_size = 0;
        ZG_CUDA(c, cudaMallocHost(&c->out_img, total));
        c->out_img_size = total;
    }
    unsigned char *img = c->out_img, *dev = nullptr;
    cudaError_t e = cudaMallocAsync(&dev, dev_total, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "zg_vtu_write: device scratch");
    std::vector<unsigned char *> dsec;
    size_t doff = 0;
    for (size_t sz : sizes) {
        dsec.push_back(dev + doff);
        doff += (sz + 255) / 256 * 256;
    }
    vtu::launch_points(m, reinterpret_cast<double *>(dsec[0]), c->stream);
    vtu::launch_cells((int)n, reinterpret_cast<uint32_t *>(dsec[1]), reinterpret_cast<uint32_t *>(dsec[2]), dsec[3],
                      c->stream);
    c->launches += 2;
    size_t hoff = 0;
    for (size_t k = 0; k < sizes.size(); ++k) {
        const uint32_t sz32 = (uint32_t)sizes[k];
        std::memcpy(img + hoff, &sz32, 4);
        hoff += 4;
        const unsigned char *src = dsec[k];
        if (k >= 4) {
            const OutVar &v = vs[k - 4];
            if (v.host) {
                std::memcpy(img + hoff, v.host, sizes[k]);
                src = nullptr;
            } else if (v.kind < 0) {
                src = reinterpret_cast<const unsigned char *>(v.a);  // a Float64 field: straight from the state
            } else {
                vtu::launch_var(m, v.kind, v.a, v.b, dsec[k], c->stream);
                ++c->launches;
            }
        }
        if (src && sizes[k]) {
            e = cudaMemcpyAsync(img + hoff, src, sizes[k], cudaMemcpyDeviceToHost, c->stream);
            if (e != cudaSuccess) break;
        }
        hoff += sizes[k];
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFreeAsync(dev, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "zg_vtu_write: packing");
    // create_directories (vtk_type.cpp:13-22), then the file
    std::error_code ec;
    const std::filesystem::path path(filename);
    if (path.has_parent_path()) std::filesystem::create_directories(path.parent_path(), ec);
    FILE *f = std::fopen(filename.c_str(), "wb");
    if (!f) return fail(c, ZG_ERR_ARG, "zg_vtu_write: cannot open '" + filename + "'");
    const bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size() &&
                    std::fwrite(img, 1, total, f) == total;
    std::fclose(f);
    if (!ok) return fail(c, ZG_ERR_ARG, "zg_vtu_write: short write to '" + filename + "'");
    return ZG_OK;
}

// The collection file (pvd_file.cpp:150-211): the datasets saved so far.
bool pvd_rewrite(const zg_pvd *p) {
    FILE *f = std::fopen((p->fullname + ".pvd").c_str(), "wb");
    if (!f) return false;
    std::fputs("<?xml version=\"1.0\"?>\n", f);
    std::fputs("<VTKFile type=\"Collection\" version=\"0.1\" byte_order=\"LittleEndian\">\n", f);
    std::fputs("    <Collection>\n", f);
    for (size_t k = 0; k < p->steps.size(); ++k)
        std::fprintf(f, "        <DataSet timestep=\"%.15e\" part=\"0\" file=\"%s_%zu.vtu\"/>\n", p->steps[k],
                     p->filename.c_str(), k);
    std::fputs("    </Collection>\n", f);
    std::fputs("</VTKFile>\n", f);
    return std::fclose(f) == 0;
}

}  // namespace

extern "C" {

int zg_vtu_write(zg_ctx *c, const char *filename, const zg_out_var *vars, int n_vars) {
    if (!c || !filename) return ZG_ERR_ARG;
    return vtu_write(c, filename, vars, n_vars);
}

int zg_pvd_open(zg_pvd **out, const char *filename, const char *directory) {
    if (!out || !filename) return ZG_ERR_ARG;
    namespace fs = std::filesystem;
    std::error_code ec;
    // PvdFile::open (pvd_file.cpp:89-148)
    fs::path dir = fs::current_path(ec);
    if (directory && *directory) {
        fs::path d = directory;
        dir = d.is_relative() ? dir / d : d;
    }
    if (!fs::exists(dir, ec) || !fs::is_directory(dir, ec)) fs::create_directories(dir, ec);
    auto *p = new zg_pvd();
    std::string name = filename;
    p->filename = name;
    if (name.size() > 4 && name.substr(name.size() - 4) == ".pvd") p->filename = name.substr(name.size() - 4);
    p->fullname = (dir / name).string();
    if (!pvd_rewrite(p)) {
        delete p;
        return ZG_ERR_ARG;
    }
    *out = p;
    return ZG_OK;
}

int zg_pvd_save(zg_pvd *p, zg_ctx *c, const zg_out_var *vars, int n_vars, double timestep) {
    if (!p || !c) return ZG_ERR_ARG;
    const std::string vtu = p->fullname + "_" + std::to_string(p->steps.size()) + ".vtu";
    int rc = vtu_write(c, vtu, vars, n_vars);
    if (rc != ZG_OK) return rc;
    p->steps.push_back(timestep);
    if (!pvd_rewrite(p)) return fail(c, ZG_ERR_ARG, "zg_pvd_save: cannot write '" + p->fullname + ".pvd'");
    return ZG_OK;
}

int zg_pvd_close(zg_pvd *p) {
    delete p;
    return ZG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Adaptive mesh: EuMesh::set_max_level / set_distributor / refine on the GPU

namespace {

// AmrCells arrays of `cap` cells in one allocation: 63 doubles, 22 ints and
// 16 bytes per cell.
size_t amr_bytes(size_t cap) { return cap * (63 * sizeof(double) + 22 * sizeof(int) + 16); }

void amr_carve(zg_ctx *c, size_t cap) {
    double *d = static_cast<double *>(c->d_amr);
    amr::View &v = c->av;
    auto td = [&d](size_t k) {
        double *p = d;
        d += k;
        return p;
    };
    v.vx = td(9 * cap);
    v.vy = td(9 * cap);
    v.cx = td(cap);
    v.cy = td(cap);
    v.vol = td(cap);
    double *inc = td(cap);
    v.fnx = td(8 * cap);
    v.fny = td(8 * cap);
    v.fcx = td(8 * cap);
    v.fcy = td(8 * cap);
    v.fa = td(8 * cap);
    int *ip = reinterpret_cast<int *>(d);
    auto ti = [&ip](size_t k) {
        int *p = ip;
        ip += k;
        return p;
    };
    v.level = ti(cap);
    v.flag = ti(cap);
    v.b_idx = ti(cap);
    v.z_idx = ti(cap);
    v.next = ti(cap);
    v.index = ti(cap);
    v.fb = ti(8 * cap);
    v.fadj = ti(8 * cap);
    v.fv = reinterpret_cast<signed char *>(ip);
    SlotMesh &m = c->smesh;
    m.cx = v.cx;
    m.cy = v.cy;
    m.vol = v.vol;
    m.inc = inc;
    m.level = v.level;
    m.fb = v.fb;
    m.fn = v.fadj;
    m.fnx = v.fnx;
    m.fny = v.fny;
    m.fcx = v.fcx;
    m.fcy = v.fcy;
    m.fa = v.fa;
}

void amr_set_n(zg_ctx *c, int n) {
    ++c->mesh_version;
    c->n = n;
    c->smesh.n = n;
    c->mesh = StructMesh{};
    c->mesh.n = n;
}

// The mesh view with the current state, isolation counters and gradients.
amr::View amr_view(const zg_ctx *c) {
    amr::View v = c->av;
    v.n = c->n;
    v.zr = c->z.r;
    v.zu = c->z.u;
    v.zv = c->z.v;
    v.zp = c->z.p;
    v.ze = c->z.e;
    v.wait = c->d_wait + (size_t)c->wait_cur * c->cap;
    for (int k = 0; k < 4; ++k) {
        v.gx[k] = c->gx[k];
        v.gy[k] = c->gy[k];
    }
    v.slope = c->amr_distr == ZG_DISTR_SLOPE ? 1 : 0;
    v.eos = c->eos;
    return v;
}

}  // namespace

extern "C" {

int zg_amr_enable(zg_ctx *c, int max_level, int capacity) {
    if (!c) return ZG_ERR_ARG;
    if (!c->have_mesh || c->slots || c->nx < 1)
        return fail(c, ZG_ERR_STATE, "zg_amr_enable: needs a mesh from zg_mesh_rectangle");
    if (c->configured || c->mm_configured)
        return fail(c, ZG_ERR_STATE, "zg_amr_enable: call before zg_smf_configure");
    if (c->mesh.xper || c->mesh.yper)
        return fail(c, ZG_ERR_ARG,
                    "zg_amr_enable: periodic boundaries cannot be adaptive (faces across the period have no "
                    "matching vertices; EuMesh::init_amr -> find_rotations fails with 'Invalid rotation')");
    if (capacity < c->n) return fail(c, ZG_ERR_ARG, "zg_amr_enable: capacity below the number of cells");
    if ((long long)capacity > (long long)std::numeric_limits<int>::max() / 16)
        return fail(c, ZG_ERR_ARG, "zg_amr_enable: capacity too large for 32-bit face indices");
    DeviceGuard g(c->device);
    cudaStreamSynchronize(c->stream);
    const size_t cap = (size_t)capacity;
    size_t scratch = 0;
    if (amr::scratch_bytes(capacity, &scratch) != 0) return fail(c, ZG_ERR_CUDA, "zg_amr_enable: scan size query");
    ZG_CUDA(c, cudaMalloc(&c->d_amr, amr_bytes(cap)));
    ZG_CUDA(c, cudaMalloc(&c->d_amr_scratch, scratch));
    c->amr_scratch_size = scratch;
    amr_carve(c, cap);
    amr::RectSpec r{};
    r.nx = c->nx;
    r.ny = c->ny;
    r.x_min = c->box[0];
    r.x_max = c->box[1];
    r.y_min = c->box[2];
    r.y_max = c->box[3];
    for (int k = 0; k < 4; ++k) r.bc[k] = c->mesh.bc[k];
    r.xper = c->mesh.xper;
    r.yper = c->mesh.yper;
    c->smesh.hx0 = (r.x_max - r.x_min) / r.nx;  // amr_cells_gen.cpp:138-139
    c->smesh.hy0 = (r.y_max - r.y_min) / r.ny;
    amr::View v = c->av;
    v.n = c->n;
    if (amr::init_rect(v, r, const_cast<double *>(c->smesh.inc), c->stream) != 0)
        return cuda_fail(c, cudaGetLastError(), "zg_amr_enable: base mesh kernels");
    c->launches += 2;
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    // the rectangle's axis tables are not used on a slot mesh
    cudaFree(c->d_geo);
    cudaFree(c->d_tgeo);
    c->d_geo = nullptr;
    c->d_tgeo = nullptr;
    c->ax64 = c->ay64 = tiled::AxisGeo<double>{};
    c->ax32 = c->ay32 = tiled::AxisGeo<float>{};
    c->cap = capacity;
    c->amr = true;
    c->slots = true;
    c->amr_max_level = std::max(0, std::min(max_level, 15));  // EuMesh::set_max_level
    amr_set_n(c, c->n);
    c->nx = c->ny = 0;
    return ZG_OK;
}

int zg_amr_set_distributor(zg_ctx *c, int kind) {
    if (!c) return ZG_ERR_ARG;
    if (kind != ZG_DISTR_CONST && kind != ZG_DISTR_SLOPE)
        return fail(c, ZG_ERR_ARG, "zg_amr_set_distributor: unknown distributor");  // sm_fluid.cpp:373-375
    c->amr_distr = kind;
    return ZG_OK;
}

int zg_amr_set_flags_gradient(zg_ctx *c, double refine_above, double coarsen_below, int *flags) {
    if (!c || !(refine_above > coarsen_below)) return ZG_ERR_ARG;
    if (!c->amr) return fail(c, ZG_ERR_STATE, "zg_amr_set_flags_gradient: mesh is not adaptive");
    if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_amr_set_flags_gradient: solver not configured");
    DeviceGuard g(c->device);
    int rc = materialize_prim(c);
    if (rc != ZG_OK) return rc;
    SmfArgs a = make_args(c);
    void *st = (void *)c->stream;
    timed(c, ZG_K_GRAD, [&] { slotfast::launch_grad(a, c->z, st); });
    c->grad_ordered = false;
    timed(c, ZG_K_FLAGS, [&] { slotfast::launch_grad_flags(a, c->av.flag, refine_above, coarsen_below, st); });
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "flags kernel launch");
    if (!flags) return ZG_OK;
    ZG_CUDA(c, cudaMemcpyAsync(flags, c->av.flag, (size_t)c->n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

int zg_amr_put_flags(zg_ctx *c, const int *flags) {
    if (!c || !flags) return ZG_ERR_ARG;
    if (!c->amr) return fail(c, ZG_ERR_STATE, "zg_amr_put_flags: mesh is not adaptive");
    DeviceGuard g(c->device);
    ZG_CUDA(c, cudaMemcpyAsync(c->av.flag, flags, (size_t)c->n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    return ZG_OK;
}

int zg_amr_refine(zg_ctx *c) {
    if (!c) return ZG_ERR_ARG;
    if (!c->amr) return fail(c, ZG_ERR_STATE, "zg_amr_refine: mesh is not adaptive (zg_amr_enable)");
    if (!c->configured) return fail(c, ZG_ERR_STATE, "zg_amr_refine: solver not configured");
    if (c->amr_max_level < 1) return ZG_OK;  // EuMesh::refine returns on a non-adaptive mesh
    DeviceGuard g(c->device);
    // the refine moves and splits the FP64 primitive state
    int rc0 = convert_state(c, ZG_FP64);
    if (rc0 == ZG_OK) rc0 = unorder_gradients(c);
    if (rc0 != ZG_OK) return rc0;
    const int n0 = c->n;
    amr::RefineResult res = amr::refine(amr_view(c), c->n, c->cap, c->amr_max_level, c->d_amr_scratch,
                                        c->amr_scratch_size, const_cast<double *>(c->smesh.inc), c->stream);
    c->launches += res.launches;
    if (res.err == -6)
        return fail(c, ZG_ERR_TOO_LARGE,
                    "zg_amr_refine: the adaptation needs " + std::to_string(res.n_large) + " cells, capacity is " +
                        std::to_string(c->cap));
    if (res.err != 0) return cuda_fail(c, cudaGetLastError(), "zg_amr_refine");
    amr_set_n(c, res.n);
    c->cfl_valid = false;
    c->amr_last.n_before = n0;
    c->amr_last.n_after = res.n;
    c->amr_last.n_coarse = res.n_coarse;
    c->amr_last.n_refine = res.n_refine;
    c->amr_last.n_large = res.n_large;
    return ZG_OK;
}

int zg_amr_info(const zg_ctx *c, zg_amr_stats *out) {
    if (!c || !out) return ZG_ERR_ARG;
    *out = c->amr_last;
    out->max_level = c->amr ? c->amr_max_level : 0;
    out->capacity = c->amr ? c->cap : 0;
    return ZG_OK;
}

int zg_amr_download(zg_ctx *c, const zg_amr_cells *out) {
    if (!c || !out) return ZG_ERR_ARG;
    if (!c->amr) return fail(c, ZG_ERR_STATE, "zg_amr_download: mesh is not adaptive");
    DeviceGuard g(c->device);
    const size_t n = (size_t)c->n;
    const amr::View &v = c->av;
    auto cp = [c](void *dst, const void *src, size_t bytes) {
        if (!dst) return cudaSuccess;
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
    };
    const size_t D = sizeof(double), I = sizeof(int);
    struct Item {
        void *dst;
        const void *src;
        size_t bytes;
    } items[] = {{out->center_x, v.cx, n * D},       {out->center_y, v.cy, n * D},
                 {out->volume, v.vol, n * D},        {out->incircle, c->smesh.inc, n * D},
                 {out->map_x, v.vx, 9 * n * D},      {out->map_y, v.vy, 9 * n * D},
                 {out->level, v.level, n * I},       {out->flag, v.flag, n * I},
                 {out->b_idx, v.b_idx, n * I},       {out->z_idx, v.z_idx, n * I},
                 {out->face_boundary, v.fb, 8 * n * I}, {out->face_neib, v.fadj, 8 * n * I},
                 {out->face_nx, v.fnx, 8 * n * D},   {out->face_ny, v.fny, 8 * n * D},
                 {out->face_cx, v.fcx, 8 * n * D},   {out->face_cy, v.fcy, 8 * n * D},
                 {out->face_area, v.fa, 8 * n * D}};
    for (const Item &it : items) ZG_CUDA(c, cp(it.dst, it.src, it.bytes));
    ZG_CUDA(c, cudaStreamSynchronize(c->stream));
    return ZG_OK;
}

}  // extern "C"
