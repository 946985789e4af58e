// ref_mm_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own MmFluid (math/solver/mm_fluid.cpp) with its
// MixturePT closure, mixture HLLC, CRP fluxes and PLIC reconstruction on the
// reference's own EuMesh, all compiled from the reference sources, and
// exposes a C interface so that tests can pin the oracle's multi-material
// restatement (and through it the GPU kernels) to the reference.  Built by
// oracle/ref_build.py into oracle/_ref/libzref_mesh.so.
//
// Cell state exchanged with the caller, 14 doubles per cell in this order:
// density, vx, vy, pressure, energy, temperature, mass fractions [4],
// true densities [4] (the fields of mmf::PState, models.h:167-180).
#include <cmath>
#include <cstring>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include <zephyr/geom/generator/rectangle.h>
#include <zephyr/geom/sections.h>
#include <zephyr/math/cfd/flux/hllc.h>
#include <zephyr/math/solver/mm_fluid.h>
#include <zephyr/mesh/euler/eu_mesh.h>
#include <zephyr/phys/matter/eos/ideal_gas.h>
#include <zephyr/phys/matter/eos/stiffened_gas.h>
#include <zephyr/phys/matter/mixture_pt.h>
#include <zephyr/utils/threads.h>

using namespace zephyr;
using geom::Boundary;
using geom::Vector3d;
using math::MmFluid;
using mesh::EuCell;
using mesh::EuMesh;
using phys::Fractions;
using phys::MixturePT;
using phys::ScalarSet;
namespace mmf = zephyr::math::mmf;

namespace {

struct RefMm {
    std::unique_ptr<EuMesh> mesh;
    MixturePT mixture;
    std::unique_ptr<MmFluid> solver;
    MmFluid::Parts part;
};

// "ideal:Air,stiffened:Water" -> the reference's named materials.
MixturePT make_mixture(const char *spec) {
    MixturePT mix;
    std::stringstream ss(spec);
    std::string item;
    while (std::getline(ss, item, ',')) {
        auto colon = item.find(':');
        std::string kind = item.substr(0, colon), name = item.substr(colon + 1);
        if (kind == "ideal") mix += phys::IdealGas::create(name);
        else mix += phys::StiffenedGas::create(name);
    }
    return mix;
}

void put(const mmf::PState &z, double *o) {
    o[0] = z.density;
    o[1] = z.velocity.x();
    o[2] = z.velocity.y();
    o[3] = z.pressure;
    o[4] = z.energy;
    o[5] = z.temperature;
    for (int k = 0; k < 4; ++k) o[6 + k] = z.mass_frac[k];
    for (int k = 0; k < 4; ++k) o[10 + k] = z.densities[k];
}

mmf::PState get(const double *s) {
    Fractions b = Fractions::Zero();
    ScalarSet r;
    for (int k = 0; k < 4; ++k) {
        b[k] = s[6 + k];
        r[k] = s[10 + k];
    }
    return mmf::PState(s[0], Vector3d(s[1], s[2], 0.0), s[3], s[4], s[5], b, r);
}

}  // namespace

extern "C" {

// MmFluid(mixture) on Rectangle(x_min, x_max, y_min, y_max), nx by ny cells,
// boundary flags {left, right, bottom, top}; crp_mode is the value of the
// reference's CrpMode (0 NONE: plain mixture HLLC, 4 PLIC).
void *zmm_create(int nx, int ny, double x_min, double x_max, double y_min, double y_max, const int *bounds,
                 const char *materials, double CFL, int acc, int crp_mode) {
    auto *r = new RefMm();
    geom::generator::Rectangle gen(x_min, x_max, y_min, y_max);
    gen.set_boundaries({.left = Boundary(bounds[0]), .right = Boundary(bounds[1]),
                        .bottom = Boundary(bounds[2]), .top = Boundary(bounds[3])});
    gen.set_sizes(nx, ny);
    r->mesh = std::make_unique<EuMesh>(gen);
    r->mixture = make_mixture(materials);
    r->solver = std::make_unique<MmFluid>(r->mixture);
    r->solver->set_CFL(CFL);
    r->solver->set_accuracy(acc);
    if (crp_mode == 0) r->solver->set_method(math::Fluxes::HLLC);
    else r->solver->set_crp_mode(math::CrpMode(crp_mode));
    r->part = r->solver->add_types(*r->mesh);
    return r;
}

void zmm_free(void *p) { delete static_cast<RefMm *>(p); }

// MmFluid::set_limiter (mm_fluid.cpp:72-74)
void zmm_set_limiter(void *p, const char *name) { static_cast<RefMm *>(p)->solver->set_limiter(name); }

// MmFluid::set_splitting (mm_fluid.cpp:75-77): 0 NONE, 1 SIMPLE, 2 STRANG
void zmm_set_split(void *p, int split) {
    static_cast<RefMm *>(p)->solver->set_splitting(math::DirSplit(split));
}

int zmm_n_cells(void *p) { return (int)static_cast<RefMm *>(p)->mesh->n_cells(); }

// Initial states through the reference's PState(density, velocity, pressure,
// mass fractions, mixture) constructor (models.cpp:180-188): energy,
// temperature and true densities from the mixture closure.
void zmm_make_states(void *p, const double *rho, const double *vx, const double *vy, const double *P,
                     const double *beta /* 4 per cell */) {
    auto *r = static_cast<RefMm *>(p);
    int n = (int)r->mesh->n_cells();
    for (int i = 0; i < n; ++i) {
        std::array<double, 4> b{beta[4 * i], beta[4 * i + 1], beta[4 * i + 2], beta[4 * i + 3]};
        EuCell cell = (*r->mesh)[i];
        cell[r->part.init] = mmf::PState(rho[i], Vector3d(vx[i], vy[i], 0.0), P[i], Fractions(b), r->mixture);
    }
}

void zmm_set_states(void *p, const double *s) {
    auto *r = static_cast<RefMm *>(p);
    int n = (int)r->mesh->n_cells();
    for (int i = 0; i < n; ++i) {
        EuCell cell = (*r->mesh)[i];
        cell[r->part.init] = get(s + 14 * (size_t)i);
    }
}

void zmm_get_states(void *p, double *s) {
    auto *r = static_cast<RefMm *>(p);
    int n = (int)r->mesh->n_cells();
    for (int i = 0; i < n; ++i) {
        EuCell cell = (*r->mesh)[i];
        put(cell[r->part.init], s + 14 * (size_t)i);
    }
}

// One MmFluid::update; returns its dt.
double zmm_step(void *p) {
    auto *r = static_cast<RefMm *>(p);
    r->solver->update(*r->mesh);
    return r->solver->dt();
}

double zmm_compute_dt(void *p) {
    auto *r = static_cast<RefMm *>(p);
    r->solver->compute_dt(*r->mesh);
    return r->solver->dt();
}

// MmFluid::interface_recovery on the current state; per cell and material:
// the interface normal (x, y) and the plane offset.
void zmm_interface(void *p, double *nrm /* 2 * nmat per cell */, double *off /* nmat per cell */) {
    auto *r = static_cast<RefMm *>(p);
    r->solver->interface_recovery(*r->mesh);
    int n = (int)r->mesh->n_cells(), m = r->mixture.size();
    for (int i = 0; i < n; ++i) {
        EuCell cell = (*r->mesh)[i];
        auto ns = cell[r->part.n];
        auto ps = cell[r->part.p];
        for (int k = 0; k < m; ++k) {
            nrm[(size_t)(i * m + k) * 2] = ns[k].x();
            nrm[(size_t)(i * m + k) * 2 + 1] = ns[k].y();
            off[(size_t)i * m + k] = ps[k];
        }
    }
}

// MmFluid::fractions_grad (mm_fluid.cpp:469-482) on the current state; per
// cell and material the gradient (x, y) of the volume fraction (part.grad_a).
void zmm_fractions_grad(void *p, double *g /* 2 * nmat per cell */) {
    auto *r = static_cast<RefMm *>(p);
    r->solver->fractions_grad(*r->mesh, r->part.init);
    int n = (int)r->mesh->n_cells(), m = r->mixture.size();
    for (int i = 0; i < n; ++i) {
        EuCell cell = (*r->mesh)[i];
        auto ga = cell[r->part.grad_a];
        for (int k = 0; k < m; ++k) {
            g[(size_t)(i * m + k) * 2] = ga[k].x();
            g[(size_t)(i * m + k) * 2 + 1] = ga[k].y();
        }
    }
}

// MmFluid::set_flags: refinement flags per cell.
void zmm_flags(void *p, int *flags) {
    auto *r = static_cast<RefMm *>(p);
    r->solver->set_flags(*r->mesh);
    int n = (int)r->mesh->n_cells();
    for (int i = 0; i < n; ++i) flags[i] = (*r->mesh)[i].flag();
}

// ---- pointwise building blocks, on the mixture of handle p ----

// mmf::PState(QState, mixture, P0, T0, rhos) (models.cpp:190-204): the state
// after an update.  q = density, momentum x, momentum y, total energy,
// partial densities [4]; guess = P0, T0, rhos [4].
void zmm_state_from_q(void *p, const double *q, const double *guess, double *out) {
    auto *r = static_cast<RefMm *>(p);
    ScalarSet mf;
    for (int k = 0; k < 4; ++k) mf[k] = q[4 + k];
    mmf::QState Q(q[0], Vector3d(q[1], q[2], 0.0), q[3], mf);
    double rhos[4] = {guess[2], guess[3], guess[4], guess[5]};
    mmf::PState z(Q, r->mixture, guess[0], guess[1], std::span<const double>(rhos, 4));
    put(z, out);
}

// MixturePT::sound_speed_rP with the options the solver passes (T0, rhos).
double zmm_sound_speed(void *p, const double *s) {
    auto *r = static_cast<RefMm *>(p);
    mmf::PState z = get(s);
    return r->mixture.sound_speed_rP(z.rho(), z.P(), z.beta(), {.T0 = z.T(), .rhos = z.rhos()});
}

// Mixture HLLC flux (hllc.cpp:344-421) of two states already in the face
// frame; out = density, momentum x, y, energy, partial fluxes [4].
void zmm_hllc(void *p, const double *sl, const double *sr, double *out) {
    auto *r = static_cast<RefMm *>(p);
    mmf::Flux f = math::HLLC::calc_flux(get(sl), get(sr), r->mixture);
    out[0] = f.density;
    out[1] = f.momentum.x();
    out[2] = f.momentum.y();
    out[3] = f.energy;
    for (int k = 0; k < 4; ++k) out[4 + k] = f.mass_frac[k];
}

// MmFluid::calc_crp_flux (mm_fluid.cpp:266-345) for states in the face frame.
void zmm_crp_flux(void *p, const double *sl, const double *sr, double hL, double hR, int iA, double a_sig,
                  double dt, double *out) {
    auto *r = static_cast<RefMm *>(p);
    mmf::Flux f = r->solver->calc_crp_flux(get(sl), get(sr), hL, hR, iA, a_sig, dt);
    out[0] = f.density;
    out[1] = f.momentum.x();
    out[2] = f.momentum.y();
    out[3] = f.energy;
    for (int k = 0; k < 4; ++k) out[4 + k] = f.mass_frac[k];
}

// PLIC helpers of geom/sections.cpp.
double zmm_face_fraction(double a1, double a2) { return geom::face_fraction(a1, a2); }
double zmm_quad_find_section(double alpha, double nx, double ny, double A, double B) {
    return geom::quad_find_section(alpha, Vector3d(nx, ny, 0.0), A, B);
}
double zmm_quad_volume_fraction(double p, double nx, double ny, double A, double B) {
    return geom::quad_volume_fraction(p, Vector3d(nx, ny, 0.0), A, B);
}
double zmm_average_flux(double alpha, double cos, double CFL) { return geom::average_flux(alpha, cos, CFL); }

}  // extern "C"
