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
// The kernels that evaluate face fluxes, instantiated per flux family: HLLC
// and HLL without the other fluxes' code (the run-time switch over the
// eight fluxes of NumFlux::create costs registers and spills), the general
// switch for the rest.  The same operations either way.
template <int FX>
static void flux1_fx(const SmfArgs &a, bool slots, void *stream) {
    if (slots) k_flux1<SlotAcc, BLOCK, 1, FX><<<blocks(a, true), BLOCK, 0, (cudaStream_t)stream>>>(a);
    else k_flux1<StructAcc, BLOCK, 1, FX><<<blocks(a, false), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
template <int FX>
static void stage2_fx(const SmfArgs &a, bool slots, void *stream) {
    if (slots) k_stage2<SlotAcc, BLOCK, 1, FX><<<blocks(a, true), BLOCK, 0, (cudaStream_t)stream>>>(a);
    else k_stage2<StructAcc, BLOCK, 1, FX><<<blocks(a, false), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
template <int FX>
static void heun_fx(const SmfArgs &a, PrimPtr zin, PrimPtr zout, bool final, bool slots, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (slots) {
        if (final) k_heun<SlotAcc, BLOCK, true, 1, FX><<<blocks(a, true), BLOCK, 0, st>>>(a, zin, zout);
        else k_heun<SlotAcc, BLOCK, false, 1, FX><<<blocks(a, true), BLOCK, 0, st>>>(a, zin, zout);
    } else {
        if (final) k_heun<StructAcc, BLOCK, true, 1, FX><<<blocks(a, false), BLOCK, 0, st>>>(a, zin, zout);
        else k_heun<StructAcc, BLOCK, false, 1, FX><<<blocks(a, false), BLOCK, 0, st>>>(a, zin, zout);
    }
}
#define ZG_FLUX_FAMILY(FN, ...)                                        \
    do {                                                               \
        if (a.flux == FLUX_HLLC) FN<FLUX_HLLC>(__VA_ARGS__);           \
        else if (a.flux == FLUX_HLL) FN<FLUX_HLL>(__VA_ARGS__);        \
        else FN<-1>(__VA_ARGS__);                                      \
    } while (0)

void launch_flux1(const SmfArgs &a, bool slots, void *stream) { ZG_FLUX_FAMILY(flux1_fx, a, slots, stream); }
void launch_grad(const SmfArgs &a, PrimPtr z, bool slots, void *stream) { ZG_DISPATCH(k_grad, a, z); }
void launch_stage1(const SmfArgs &a, bool slots, void *stream) { ZG_DISPATCH(k_stage1, a); }
void launch_stage2(const SmfArgs &a, bool slots, void *stream) { ZG_FLUX_FAMILY(stage2_fx, a, slots, stream); }
void launch_heun(const SmfArgs &a, PrimPtr zin, PrimPtr zout, bool final, bool slots, void *stream) {
    ZG_FLUX_FAMILY(heun_fx, a, zin, zout, final, slots, stream);
}
void launch_flags(const SmfArgs &a, int *flags, bool slots, void *stream) { ZG_DISPATCH(k_flags, a, flags); }

}  // namespace parity
}  // namespace zg
