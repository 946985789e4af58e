// smf_slot_fast.cu -- the FAST form of the step on an adaptive rectangle: the
// gather-form kernels of smf_struct.cuh over SlotFastAcc (face geometry from
// the cell's centre and level instead of five stored arrays per slot),
// compiled with fused multiply-adds and register caps.  Results match the
// parity form to rounding (not bit for bit).
#include <cuda_runtime.h>

#include "smf_struct.cuh"

namespace zg {
namespace slotfast {

constexpr int BLOCK = 128;
// Minimum resident blocks per SM: register caps chosen by timing the AMR
// blast (512^2, 3 levels) over a sweep on a B200 (-D overrides)
#ifndef ZG_SLOT_GRAD_MINB
#define ZG_SLOT_GRAD_MINB 5
#endif
#ifndef ZG_SLOT_S1_MINB
#define ZG_SLOT_S1_MINB 6
#endif
#ifndef ZG_SLOT_S2_MINB
#define ZG_SLOT_S2_MINB 5
#endif
constexpr int GM = ZG_SLOT_GRAD_MINB, S1M = ZG_SLOT_S1_MINB, S2M = ZG_SLOT_S2_MINB;

static inline unsigned blocks(const SmfArgs &a) { return (unsigned)((a.smesh.n + BLOCK - 1) / BLOCK); }

void launch_dt(const SmfArgs &a, PrimPtr z, void *stream) {
    SmfArgs b = a;
    b.z = z;
    k_dt<SlotFastAcc, BLOCK><<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(b);
}
void launch_flux1(const SmfArgs &a, void *stream) {
    k_flux1<SlotFastAcc, BLOCK, S2M><<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
void launch_grad(const SmfArgs &a, PrimPtr z, void *stream) {
    k_grad<SlotFastAcc, BLOCK, GM><<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a, z);
}
void launch_stage1(const SmfArgs &a, void *stream) {
    k_stage1<SlotFastAcc, BLOCK, S1M><<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
void launch_stage2(const SmfArgs &a, void *stream) {
    k_stage2<SlotFastAcc, BLOCK, S2M><<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
void launch_heun(const SmfArgs &a, PrimPtr zin, PrimPtr zout, bool final, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (final) k_heun<SlotFastAcc, BLOCK, true, S2M><<<blocks(a), BLOCK, 0, st>>>(a, zin, zout);
    else k_heun<SlotFastAcc, BLOCK, false, S2M><<<blocks(a), BLOCK, 0, st>>>(a, zin, zout);
}

}  // namespace slotfast
}  // namespace zg
