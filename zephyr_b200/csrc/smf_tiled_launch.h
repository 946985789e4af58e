// smf_tiled_launch.h -- launchers of the tiled kernels (FAST: FP64,
// MIXED: FP32 face arithmetic with FP64 conserved state).
#pragma once

#include "smf_types.h"

namespace zg {
namespace tiled {
template <typename R>
struct Fields;
}

namespace fast {
void launch_cfl(const SmfArgs &a, const tiled::Fields<double> &f, void *stream);
void launch_grad_predict(const SmfArgs &a, const tiled::Fields<double> &f, bool predict, void *stream);
void launch_faces(const SmfArgs &a, const tiled::Fields<double> &f, int mode, void *stream);
// one fused stage: 1 predictor-corrector step, 2 / 3 Heun stage A / B (HLLC, HLL)
void launch_step(const SmfArgs &a, const tiled::Fields<double> &f, int mode, void *stream);
}  // namespace fast

namespace mixed {
void launch_cfl(const SmfArgs &a, const tiled::Fields<float> &f, void *stream);
void launch_grad_predict(const SmfArgs &a, const tiled::Fields<float> &f, bool predict, void *stream);
void launch_faces(const SmfArgs &a, const tiled::Fields<float> &f, int mode, void *stream);
void launch_step(const SmfArgs &a, const tiled::Fields<float> &f, int mode, void *stream);
void launch_to_mixed(int n, PrimPtr z, const tiled::Fields<float> &f, void *stream);
void launch_to_prim(int n, const tiled::Fields<float> &f, EosD eos, PrimPtr z, void *stream);
}  // namespace mixed

// MIXED kernels on an adaptive rectangle (smf_slot_mixed.cu): dt from the FP64
// conserved state, FP32 gradients with the predictor, and the face-once face
// loop (mode 0 first order, 1 corrector).
namespace slotmixed {
void launch_dt(const SmfArgs &a, const tiled::Fields<float> &f, void *stream);
// the gradients over the FAST step's slot geometry (sg, bm); predictor: the
// predictor stage (sm_fluid.cpp:176-253) fused after them
void launch_grad(const SmfArgs &a, const tiled::Fields<float> &f, const double4 *sg, const double4 *bm,
                 bool predictor, void *stream);
// face-once (mode 0 first order, 1 corrector): the listed faces, then the
// cell sums (and the next dt with ff.dt_next)
void launch_faces_once(const SmfArgs &a, const tiled::Fields<float> &f, int mode, const slotfast::FaceFlux &ff,
                       void *stream);
void launch_sum(const SmfArgs &a, const tiled::Fields<float> &f, int mode, const slotfast::FaceFlux &ff,
                void *stream);
}  // namespace slotmixed
}  // namespace zg
