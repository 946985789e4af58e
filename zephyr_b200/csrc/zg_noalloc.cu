// zg_noalloc.cu -- zg_rect_step_noalloc: one first-order step on a rectangle
// that allocates no memory at all.
//
// Some callers cannot let a library call cudaMalloc: a host program that
// owns every byte of device memory through its own pool (a simulation code
// with a fixed memory budget per GPU), or code that runs where an allocation
// would synchronise the device in the middle of its own timed or ordered
// stream work.  zg_smf_update needs a context whose fields are allocated by
// zg_smf_configure; this entry point instead takes the state arrays from the
// caller and keeps everything else it needs -- the CFL accumulator, the
// finishing-block ticket, the step's dt and the mesh's coordinate tables --
// in one fixed-size array of device memory that is part of the library
// image (every GPU that loads the library holds it until the process exits).
//
// The kernels are the parity kernels of zg_smf_update (k_dt, k_flux1 in
// smf_parity.cu), so the result equals a zg_smf_update step bit for bit.
// This file is compiled with -fmad=false so that the coordinate tables it
// builds on the device match the host-built tables of zg_mesh_rectangle.
#include <cuda_runtime.h>

#include <algorithm>
#include <limits>

#include "../../include/zephyr_gpu.h"
#include "smf_types.h"

using namespace zg;

namespace {

// Scratch layout, in doubles from the start of the array:
//   [0]  running CFL minimum (bit image)   [1] finishing-block ticket (low word)
//   [2]  dt of the step                    [3..7] unused
//   [8 ...] X (nx+1), Y (ny+1), cx, fxm, inc2x (nx each), cy, fym, inc2y (ny each)
constexpr int kMaxAxis = ZG_NOALLOC_MAX_AXIS;
constexpr size_t kHeader = 8;
constexpr size_t kScratchDoubles = kHeader + 8 * (size_t)kMaxAxis + 8;

static __device__ __align__(256) double g_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;

// Device address of g_scratch on the current device.  Looked up on every
// call (cheap once the module is loaded), so that a context torn down and
// created again (cudaDeviceReset), which may load the module at another
// address, is followed.  The first lookup on a device may load the library's
// device code there.
int scratch_on(double **out) {
    double *p = nullptr;
    if (cudaGetSymbolAddress((void **)&p, g_scratch) != cudaSuccess || !p) return ZG_ERR_CUDA;
    *out = p;
    return ZG_OK;
}

// Coordinate tables with the formulas of zg_mesh_rectangle (vertices
// amr_cells_gen.cpp:155-161, centres quad.cpp:434, mid-edges quad.cpp:433-435,
// incircle extents amr_cells.cpp:107-116), evaluated in the same order; also
// resets the CFL accumulator and the ticket that k_dt starts from.
__global__ void k_fill_tables(double *s, int nx, int ny, double x_min, double x_max, double y_min,
                              double y_max) {
    double *X = s + kHeader, *Y = X + (nx + 1);
    double *cx = Y + (ny + 1), *fxm = cx + nx, *i2x = fxm + nx;
    double *cy = i2x + nx, *fym = cy + ny, *i2y = fym + ny;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) {
        reinterpret_cast<unsigned long long *>(s)[0] = 0x7FEFFFFFFFFFFFFFull;  // bits of DBL_MAX
        reinterpret_cast<unsigned long long *>(s)[1] = 0ull;
    }
    if (t <= nx) X[t] = x_min + ((x_max - x_min) * t) / nx;
    if (t <= ny) Y[t] = y_min + ((y_max - y_min) * t) / ny;
    if (t < nx) {
        double a = x_min + ((x_max - x_min) * t) / nx, b = x_min + ((x_max - x_min) * (t + 1)) / nx;
        cx[t] = 0.25 * (a + b + a + b);
        fxm[t] = 0.5 * (a + b);
        double d = 0.5 * (b + b) - 0.5 * (a + a);
        i2x[t] = d * d + 0.0 * 0.0 + 0.0 * 0.0;
    }
    if (t < ny) {
        double a = y_min + ((y_max - y_min) * t) / ny, b = y_min + ((y_max - y_min) * (t + 1)) / ny;
        cy[t] = 0.25 * (a + a + b + b);
        fym[t] = 0.5 * (a + b);
        double d = 0.5 * (b + b) - 0.5 * (a + a);
        i2y[t] = 0.0 * 0.0 + d * d + 0.0 * 0.0;
    }
}

struct DeviceSwitch {
    int prev = -1;
    bool ok = true;
    explicit DeviceSwitch(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceSwitch() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" int zg_rect_step_noalloc(int device, int nx, int ny, double x_min, double x_max, double y_min,
                                    double y_max, const int bounds[4], const zg_smf_params *p,
                                    const double *const in[5], double *const out[5], double *dt, void *stream) {
    if (nx > kMaxAxis || ny > kMaxAxis) return ZG_ERR_TOO_LARGE;
    if (nx < 1 || ny < 1 || !bounds || !p || !in || !out) return ZG_ERR_ARG;
    if (!(x_max > x_min) || !(y_max > y_min)) return ZG_ERR_ARG;
    for (int k = 0; k < 4; ++k)
        if (bounds[k] != ZG_BC_WALL && bounds[k] != ZG_BC_ZOE && bounds[k] != ZG_BC_PERIODIC) return ZG_ERR_ARG;
    for (int k = 0; k < 5; ++k) {
        if (!in[k] || !out[k]) return ZG_ERR_ARG;
        for (int j = 0; j < 5; ++j)
            if (out[k] == in[j]) return ZG_ERR_ARG;  // the step reads neighbours of every cell
    }
    if (p->eos_kind != ZG_EOS_IDEAL && p->eos_kind != ZG_EOS_STIFFENED) return ZG_ERR_ARG;
    if (p->flux < ZG_FLUX_GODUNOV || p->flux > ZG_FLUX_CIR2) return ZG_ERR_ARG;
    if (!(p->gamma > 1.0)) return ZG_ERR_ARG;
    if (std::min(std::max(1, p->accuracy), 2) != 1 || p->precision != ZG_FP64 || p->kernels != ZG_KERNELS_PARITY)
        return ZG_ERR_ARG;  // first order, FP64, parity kernels only
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) return ZG_ERR_CUDA;
    if (device < 0 || device >= count || device >= kMaxDevices) return ZG_ERR_ARG;

    DeviceSwitch sw(device);
    if (!sw.ok) return ZG_ERR_CUDA;
    // an error left pending by the caller's own earlier work is not this
    // call's: it is reported, and left pending, before anything is launched
    if (cudaPeekAtLastError() != cudaSuccess) return ZG_ERR_CUDA;
    double *s = nullptr;
    int rc = scratch_on(&s);
    if (rc != ZG_OK) return rc;

    int bc[4] = {bounds[0], bounds[1], bounds[2], bounds[3]};
    bool xper = bc[0] == ZG_BC_PERIODIC || bc[1] == ZG_BC_PERIODIC;
    bool yper = bc[2] == ZG_BC_PERIODIC || bc[3] == ZG_BC_PERIODIC;
    if (xper) bc[0] = bc[1] = ZG_BC_PERIODIC;
    if (yper) bc[2] = bc[3] = ZG_BC_PERIODIC;

    SmfArgs a{};
    StructMesh &m = a.mesh;
    m.nx = nx;
    m.ny = ny;
    m.n = nx * ny;
    for (int k = 0; k < 4; ++k) m.bc[k] = bc[k];
    m.xper = xper;
    m.yper = yper;
    m.X = s + kHeader;
    m.Y = m.X + (nx + 1);
    m.cx = m.Y + (ny + 1);
    m.fxm = m.cx + nx;
    m.inc2x = m.fxm + nx;
    m.cy = m.inc2x + nx;
    m.fym = m.cy + ny;
    m.inc2y = m.fym + ny;
    m.hx = (x_max - x_min) / nx;
    m.hy = (y_max - y_min) / ny;
    m.vol = m.hx * m.hy;
    a.eos.kind = p->eos_kind;
    a.eos.gamma = p->gamma;
    a.eos.gm1 = p->gamma - 1.0;
    a.eos.P0 = p->eos_kind == ZG_EOS_IDEAL ? 0.0 : p->P0;
    a.eos.e0 = p->eos_kind == ZG_EOS_IDEAL ? 0.0 : p->e0;
    a.eos.pmin = p->eos_kind == ZG_EOS_IDEAL ? 0.0 : -p->P0;
    a.flux = p->flux;
    a.limiter = p->limiter;
    a.CFL = std::max(0.0, std::min(p->CFL, 1.0));
    a.max_dt = p->max_dt;
    a.z = PrimPtr{const_cast<double *>(in[0]), const_cast<double *>(in[1]), const_cast<double *>(in[2]),
                  const_cast<double *>(in[3]), const_cast<double *>(in[4])};
    a.znext = PrimPtr{out[0], out[1], out[2], out[3], out[4]};
    a.dmin_bits = reinterpret_cast<unsigned long long *>(s);
    a.dt_ticket = reinterpret_cast<unsigned int *>(s + 1);
    a.dt_out = s + 2;

    cudaStream_t st = (cudaStream_t)stream;
    int span = std::max(nx, ny) + 1;
    k_fill_tables<<<(span + 255) / 256, 256, 0, st>>>(s, nx, ny, x_min, x_max, y_min, y_max);
    if (cudaGetLastError() != cudaSuccess) return ZG_ERR_CUDA;
    parity::launch_dt(a, a.z, false, stream);
    if (cudaGetLastError() != cudaSuccess) return ZG_ERR_CUDA;
    parity::launch_flux1(a, false, stream);
    if (cudaGetLastError() != cudaSuccess) return ZG_ERR_CUDA;
    if (dt && cudaMemcpyAsync(dt, s + 2, sizeof(double), cudaMemcpyDefault, st) != cudaSuccess)
        return ZG_ERR_CUDA;
    return ZG_OK;
}
