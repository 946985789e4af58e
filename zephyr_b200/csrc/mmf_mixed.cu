// mmf_mixed.cu -- the mixed form of the multi-material pure-stencil face
// loop: face states, wave speeds and HLLC fluxes in FP32 (IEEE division and
// square root, no fused multiply-adds), each face flux
// widened to FP64 for the accumulation; the update and the one-material
// closure (EoS pressure recovery) in FP64.  The composite Riemann fluxes,
// the PT-equilibrium closure, PLIC and dt stay in the FP64 kernels of
// mmf_parity.cu.
#include "mmf_pure.cuh"

namespace zg {
namespace mmf {

// minimum resident blocks per SM (register cap; -D overrides for sweeps)
#ifndef ZG_MM_MIXED_MINB
#define ZG_MM_MIXED_MINB 8
#endif

void launch_flux_pure_fp32(const MmArgs &a, void *stream) {
    const unsigned nb = (unsigned)((a.mesh.n + BLOCK - 1) / BLOCK);
    k_flux_pure<float, ZG_MM_MIXED_MINB><<<nb, BLOCK, 0, (cudaStream_t)stream>>>(a);
}

}  // namespace mmf
}  // namespace zg
