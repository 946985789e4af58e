// smf_parity.cu -- instantiates the gather-form FP64 kernels for both mesh
// accessors.  This file is compiled with -fmad=false: no multiply is fused
// into an add, matching the reference's x86-64 build, so results agree bit
// for bit with the oracle and the reference.
#include <cuda_runtime.h>

#include "smf_struct.cuh"

namespace zg {
namespace parity {

constexpr int BLOCK = 128;

static inline unsigned blocks(const SmfArgs &a, bool slots) {
    int n = slots ? a.smesh.n : a.mesh.n;
    return (unsigned)((n + BLOCK - 1) / BLOCK);
}

#define ZG_DISPATCH(KERNEL, ...)                                                                            \
    do {                                                                                                    \
        if (slots)                                                                                          \
            KERNEL<SlotAcc, BLOCK><<<blocks(a, true), BLOCK, 0, (cudaStream_t)stream>>>(__VA_ARGS__);      \
        else                                                                                                \
            KERNEL<StructAcc, BLOCK><<<blocks(a, false), BLOCK, 0, (cudaStream_t)stream>>>(__VA_ARGS__);   \
    } while (0)

void launch_dt(const SmfArgs &a, PrimPtr z, bool slots, void *stream) {
    SmfArgs b = a;
    b.z = z;
    ZG_DISPATCH(k_dt, b);
}
void launch_flux1(const SmfArgs &a, bool slots, void *stream) { ZG_DISPATCH(k_flux1, a); }
void launch_grad(const SmfArgs &a, PrimPtr z, bool slots, void *stream) { ZG_DISPATCH(k_grad, a, z); }
void launch_stage1(const SmfArgs &a, bool slots, void *stream) { ZG_DISPATCH(k_stage1, a); }
void launch_stage2(const SmfArgs &a, bool slots, void *stream) { ZG_DISPATCH(k_stage2, a); }
void launch_heun(const SmfArgs &a, PrimPtr zin, PrimPtr zout, bool final, bool slots, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (slots) {
        if (final) k_heun<SlotAcc, BLOCK, true><<<blocks(a, true), BLOCK, 0, st>>>(a, zin, zout);
        else k_heun<SlotAcc, BLOCK, false><<<blocks(a, true), BLOCK, 0, st>>>(a, zin, zout);
    } else {
        if (final) k_heun<StructAcc, BLOCK, true><<<blocks(a, false), BLOCK, 0, st>>>(a, zin, zout);
        else k_heun<StructAcc, BLOCK, false><<<blocks(a, false), BLOCK, 0, st>>>(a, zin, zout);
    }
}
void launch_flags(const SmfArgs &a, int *flags, bool slots, void *stream) { ZG_DISPATCH(k_flags, a, flags); }

}  // namespace parity
}  // namespace zg
