// smf_parity.cu -- instantiates the gather-form FP64 kernels.  This file is
// compiled with -fmad=false: no multiply is fused into an add, matching the
// reference's x86-64 build, so results agree bit for bit with the oracle.
#include <cuda_runtime.h>

#include "smf_struct.cuh"

namespace zg {
namespace parity {

constexpr int BLOCK = 128;

static inline unsigned blocks(int n) { return (unsigned)((n + BLOCK - 1) / BLOCK); }

void launch_dt(const SmfArgs &a, PrimPtr z, void *stream) {
    SmfArgs b = a;
    b.z = z;
    k_dt<BLOCK><<<blocks(a.mesh.n), BLOCK, 0, (cudaStream_t)stream>>>(b);
}
void launch_flux1(const SmfArgs &a, void *stream) {
    k_flux1<BLOCK><<<blocks(a.mesh.n), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
void launch_grad(const SmfArgs &a, PrimPtr z, void *stream) {
    k_grad<BLOCK><<<blocks(a.mesh.n), BLOCK, 0, (cudaStream_t)stream>>>(a, z);
}
void launch_stage1(const SmfArgs &a, void *stream) {
    k_stage1<BLOCK><<<blocks(a.mesh.n), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
void launch_stage2(const SmfArgs &a, void *stream) {
    k_stage2<BLOCK><<<blocks(a.mesh.n), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
void launch_heun(const SmfArgs &a, PrimPtr zin, PrimPtr zout, bool final, void *stream) {
    if (final)
        k_heun<BLOCK, true><<<blocks(a.mesh.n), BLOCK, 0, (cudaStream_t)stream>>>(a, zin, zout);
    else
        k_heun<BLOCK, false><<<blocks(a.mesh.n), BLOCK, 0, (cudaStream_t)stream>>>(a, zin, zout);
}
void launch_flags(const SmfArgs &a, int *flags, void *stream) {
    k_flags<BLOCK><<<blocks(a.mesh.n), BLOCK, 0, (cudaStream_t)stream>>>(a, flags);
}

}  // namespace parity
}  // namespace zg
