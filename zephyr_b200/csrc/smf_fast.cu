// smf_fast.cu -- the tiled FP64 kernels (FAST); multiply-adds may be fused.
#include "smf_fused.cuh"
#include "smf_tiled.cuh"
#include "smf_tiled_launch.h"

namespace zg {
namespace fast {

using tiled::Fields;
// Tile shapes and minimum resident blocks per SM.  The kernels are latency-
// bound, so residency decides their speed: the minimum-block counts cap the
// registers per thread (spilling a few bytes in the gradient pass) and were
// chosen by timing the 2048^2 step over a sweep of these values on a B200.
#ifndef ZG_FAST_TY
#define ZG_FAST_TY 8
#endif
#ifndef ZG_FAST_GY
#define ZG_FAST_GY 4
#endif
#ifndef ZG_FAST_FACES_MINB
#define ZG_FAST_FACES_MINB 4
#endif
#ifndef ZG_FAST_GP_MINB
#define ZG_FAST_GP_MINB 7
#endif
constexpr int BLOCK = 128, TX = 32, TY = ZG_FAST_TY;  // faces: 32 x TY threads, 31 x (TY - 1) interior cells
constexpr int GX = 32, GY = ZG_FAST_GY;               // gradients + predictor: 32 x GY cells
constexpr int FMINB = ZG_FAST_FACES_MINB, GMINB = ZG_FAST_GP_MINB;

static inline unsigned blocks(int n) { return (unsigned)((n + BLOCK - 1) / BLOCK); }

void launch_cfl(const SmfArgs &a, const Fields<double> &f, void *stream) {
    tiled::k_cfl<double, BLOCK><<<blocks(a.mesh.n), BLOCK, 0, (cudaStream_t)stream>>>(a, f);
}

template <int LIM>
static void grad_predict(const SmfArgs &a, const Fields<double> &f, bool predict, cudaStream_t s) {
    dim3 block(GX, GY);
    dim3 grid((a.mesh.ny + GX - 1) / GX, (a.mesh.nx + GY - 1) / GY);
    if (predict)
        tiled::k_grad_predict<double, false, true, LIM, GX, GY, GMINB><<<grid, block, 0, s>>>(a, f);
    else
        tiled::k_grad_predict<double, false, false, LIM, GX, GY, GMINB><<<grid, block, 0, s>>>(a, f);
}

void launch_grad_predict(const SmfArgs &a, const Fields<double> &f, bool predict, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    switch (a.limiter) {  // the common limiters are compiled in; others are selected at run time
        case LIM_VANALBADA1: grad_predict<LIM_VANALBADA1>(a, f, predict, s); break;
        case LIM_MC: grad_predict<LIM_MC>(a, f, predict, s); break;
        case LIM_MINMOD: grad_predict<LIM_MINMOD>(a, f, predict, s); break;
        default: grad_predict<-1>(a, f, predict, s); break;
    }
}

void launch_faces(const SmfArgs &a, const Fields<double> &f, int mode, void *stream) {
    dim3 block(TX, TY);
    dim3 grid((a.mesh.ny + TX - 2) / (TX - 1), (a.mesh.nx + TY - 2) / (TY - 1));
    cudaStream_t s = (cudaStream_t)stream;
    // HLLC and HLL get kernels without the other fluxes' code (registers)
    if (a.flux == FLUX_HLLC || a.flux == FLUX_HLL) {
        switch (mode) {
            case 0: tiled::k_faces<double, false, 0, TX, TY, FMINB, false><<<grid, block, 0, s>>>(a, f); break;
            case 1: tiled::k_faces<double, false, 1, TX, TY, FMINB, false><<<grid, block, 0, s>>>(a, f); break;
            case 2: tiled::k_faces<double, false, 2, TX, TY, FMINB, false><<<grid, block, 0, s>>>(a, f); break;
            default: tiled::k_faces<double, false, 3, TX, TY, FMINB, false><<<grid, block, 0, s>>>(a, f); break;
        }
        return;
    }
    switch (mode) {
        case 0: tiled::k_faces<double, false, 0, TX, TY, FMINB><<<grid, block, 0, s>>>(a, f); break;
        case 1: tiled::k_faces<double, false, 1, TX, TY, FMINB><<<grid, block, 0, s>>>(a, f); break;
        case 2: tiled::k_faces<double, false, 2, TX, TY, FMINB><<<grid, block, 0, s>>>(a, f); break;
        default: tiled::k_faces<double, false, 3, TX, TY, FMINB><<<grid, block, 0, s>>>(a, f); break;
    }
}

// Fused single-pass stages (smf_fused.cuh): 30 x FUSED_TH interior cells per
// block of 32 x (FUSED_TH + 2) threads.
#ifndef ZG_FAST_FUSED_TH
#define ZG_FAST_FUSED_TH 14
#endif
#ifndef ZG_FAST_FUSED_MINB
#define ZG_FAST_FUSED_MINB 2
#endif
void launch_step(const SmfArgs &a, const Fields<double> &f, int mode, void *stream) {
    tiled::fused_dispatch<double, false, ZG_FAST_FUSED_TH, ZG_FAST_FUSED_MINB>(a, f, mode, (cudaStream_t)stream);
}

}  // namespace fast
}  // namespace zg
