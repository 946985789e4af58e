// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own SmFluid (math/solver/sm_fluid.cpp, with
// math/cfd/gradient.h, face_extra.h, the HLLC/HLL fluxes, limiters, EoS and
// models.cpp compiled from the reference sources) on a rectangle mesh held by
// the checker's stand-in EuMesh, and exposes a C interface so the tests can
// pin the oracle against it.  Built by oracle/ref_build.py into
// oracle/_ref/libzref.so when the reference sources are present.
//
// Geometry: cell and face centres come from the reference's SqQuad
// (geom/primitives/quad.cpp:429-436, vs<i,j> quad.h:187-198) built on the
// vertices of amr_cells_gen.cpp:155-161; neighbours and boundary flags follow
// amr_cells_gen.cpp:163-184 and 214-228; the incircle diameter follows
// amr_cells.cpp:107-116.
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <zephyr/geom/primitives/quad.h>
#include <zephyr/math/cfd/flux/hll.h>
#include <zephyr/math/cfd/flux/hllc.h>
#include <zephyr/math/cfd/flux/num_flux.h>
#include <zephyr/math/cfd/limiter.h>
#include <zephyr/math/solver/sm_fluid.h>
#include <zephyr/phys/matter/eos/ideal_gas.h>
#include <zephyr/phys/matter/eos/stiffened_gas.h>

using namespace zephyr;
using geom::Boundary;
using geom::SqQuad;
using geom::Vector3d;
using math::SmFluid;
using math::smf::PState;

namespace {

struct Ref {
    mesh::ShimMesh shim;
    std::unique_ptr<mesh::EuMesh> mesh;
    std::unique_ptr<SmFluid> solver;
    phys::Eos::Ptr eos;
};

void build_rectangle(mesh::ShimMesh &m, int nx, int ny, double x_min, double x_max, double y_min, double y_max,
                     const int *bounds_in) {
    int bounds[4] = {bounds_in[0], bounds_in[1], bounds_in[2], bounds_in[3]};
    const int PER = int(Boundary::PERIODIC);
    bool x_period = bounds[0] == PER || bounds[1] == PER;
    bool y_period = bounds[2] == PER || bounds[3] == PER;
    if (x_period) bounds[0] = bounds[1] = PER;
    if (y_period) bounds[2] = bounds[3] = PER;
    const double hx = (x_max - x_min) / nx;
    const double hy = (y_max - y_min) / ny;
    auto idx = [ny](int i, int j) { return i * ny + j; };
    auto vertex = [&](int i, int j) {
        return Vector3d(x_min + ((x_max - x_min) * i) / nx, y_min + ((y_max - y_min) * j) / ny, 0.0);
    };
    auto neib = [&](int i, int j, int side) {
        if (side == 0) return i == 0 && !x_period ? idx(i, j) : idx((i - 1 + nx) % nx, j);
        if (side == 1) return i == nx - 1 && !x_period ? idx(i, j) : idx((i + 1 + nx) % nx, j);
        if (side == 2) return j == 0 && !y_period ? idx(i, j) : idx(i, (j - 1 + ny) % ny);
        return j == ny - 1 && !y_period ? idx(i, j) : idx(i, (j + 1 + ny) % ny);
    };
    int n = nx * ny;
    m.n = n;
    m.center.resize(n);
    m.volume.resize(n);
    m.incircle.resize(n);
    m.flag.assign(n, 0);
    m.boundary.assign(8 * (size_t)n, int(Boundary::UNDEFINED));
    m.adj.assign(8 * (size_t)n, -1);
    m.fnormal.assign(8 * (size_t)n, Vector3d(0.0, 0.0, 0.0));
    m.fcenter.assign(8 * (size_t)n, Vector3d(0.0, 0.0, 0.0));
    m.farea.assign(8 * (size_t)n, 0.0);
    for (int ic = 0; ic < n; ++ic) {
        int i = ic / ny, j = ic % ny;
        SqQuad quad(vertex(i, j), vertex(i + 1, j), vertex(i, j + 1), vertex(i + 1, j + 1));
        m.center[ic] = quad.vs<0, 0>();
        m.volume[ic] = hx * hy;
        m.incircle[ic] = std::sqrt(std::min((quad.vs<+1, 0>() - quad.vs<-1, 0>()).squaredNorm(),
                                            (quad.vs<0, +1>() - quad.vs<0, -1>()).squaredNorm()));
        size_t f = 8 * (size_t)ic;
        m.boundary[f + 0] = i > 0 ? int(Boundary::INNER) : bounds[0];
        m.boundary[f + 1] = i < nx - 1 ? int(Boundary::INNER) : bounds[1];
        m.boundary[f + 2] = j > 0 ? int(Boundary::INNER) : bounds[2];
        m.boundary[f + 3] = j < ny - 1 ? int(Boundary::INNER) : bounds[3];
        for (int s = 0; s < 4; ++s) m.adj[f + s] = neib(i, j, s);
        m.fnormal[f + 0] = -Vector3d::UnitX();
        m.fnormal[f + 1] = Vector3d::UnitX();
        m.fnormal[f + 2] = -Vector3d::UnitY();
        m.fnormal[f + 3] = Vector3d::UnitY();
        m.fcenter[f + 0] = quad.vs<-1, 0>();
        m.fcenter[f + 1] = quad.vs<+1, 0>();
        m.fcenter[f + 2] = quad.vs<0, -1>();
        m.fcenter[f + 3] = quad.vs<0, +1>();
        m.farea[f + 0] = hy;
        m.farea[f + 1] = hy;
        m.farea[f + 2] = hx;
        m.farea[f + 3] = hx;
    }
}

phys::Eos::Ptr make_eos(int kind, double gamma, double P0, double e0) {
    if (kind == 0) return phys::IdealGas::create(gamma);
    return phys::StiffenedGas::create(gamma, P0, e0);
}

}  // namespace

extern "C" {

void *zr_create(int nx, int ny, double x_min, double x_max, double y_min, double y_max, const int *bounds,
                int eos_kind, double gamma, double P0, double e0, int flux, const char *limiter, int acc,
                double CFL) {
    auto *r = new Ref();
    build_rectangle(r->shim, nx, ny, x_min, x_max, y_min, y_max, bounds);
    r->mesh = std::make_unique<mesh::EuMesh>(&r->shim);
    r->eos = make_eos(eos_kind, gamma, P0, e0);
    r->solver = std::make_unique<SmFluid>(r->eos);
    r->solver->set_accuracy(acc);
    r->solver->set_CFL(CFL);
    r->solver->set_limiter(limiter);
    r->solver->set_method(math::Fluxes(flux));
    r->solver->add_types(*r->mesh);
    return r;
}

void zr_free(void *p) { delete static_cast<Ref *>(p); }

void zr_set_threads(void *p, int n) { static_cast<Ref *>(p)->mesh->set_threads(n); }

void zr_set_max_dt(void *p, double dt) { static_cast<Ref *>(p)->solver->set_max_dt(dt); }

void zr_set_state(void *p, const double *rho, const double *u, const double *v, const double *pr,
                  const double *e) {
    auto *r = static_cast<Ref *>(p);
    auto part = r->solver->part;
    for (int ic = 0; ic < r->shim.n; ++ic) {
        mesh::EuCell c(&r->shim, ic);
        c[part.init] = PState(rho[ic], Vector3d(u[ic], v[ic], 0.0), pr[ic], e[ic]);
    }
}

void zr_get_state(void *p, double *rho, double *u, double *v, double *pr, double *e) {
    auto *r = static_cast<Ref *>(p);
    auto part = r->solver->part;
    for (int ic = 0; ic < r->shim.n; ++ic) {
        mesh::EuCell c(&r->shim, ic);
        const PState &z = c[part.init];
        rho[ic] = z.density;
        u[ic] = z.velocity.x();
        v[ic] = z.velocity.y();
        pr[ic] = z.pressure;
        e[ic] = z.energy;
    }
}

void zr_set_wait(void *p, const int *w) {
    auto *r = static_cast<Ref *>(p);
    for (int ic = 0; ic < r->shim.n; ++ic) mesh::EuCell(&r->shim, ic)[r->solver->part.wait] = w[ic];
}

void zr_get_wait(void *p, int *w) {
    auto *r = static_cast<Ref *>(p);
    for (int ic = 0; ic < r->shim.n; ++ic) w[ic] = mesh::EuCell(&r->shim, ic)[r->solver->part.wait];
}

double zr_step(void *p) {
    auto *r = static_cast<Ref *>(p);
    r->solver->update(*r->mesh);
    return r->solver->dt();
}

double zr_steps(void *p, int n) {
    auto *r = static_cast<Ref *>(p);
    for (int k = 0; k < n; ++k) r->solver->update(*r->mesh);
    return r->solver->dt();
}

void zr_set_flags(void *p, int *flags) {
    auto *r = static_cast<Ref *>(p);
    r->solver->set_flags(*r->mesh);
    for (int ic = 0; ic < r->shim.n; ++ic) flags[ic] = r->shim.flag[ic];
}

// Limited gradients (x, y) of density, vx, vy, pressure, energy after
// compute_grad on the current state; arrays of 5 * n, field-major.
void zr_grad(void *p, double *gx, double *gy) {
    auto *r = static_cast<Ref *>(p);
    r->solver->compute_grad(*r->mesh);
    auto part = r->solver->part;
    int n = r->shim.n;
    for (int ic = 0; ic < n; ++ic) {
        mesh::EuCell c(&r->shim, ic);
        const PState &a = c[part.d_dx];
        const PState &b = c[part.d_dy];
        double ax[5] = {a.density, a.velocity.x(), a.velocity.y(), a.pressure, a.energy};
        double by[5] = {b.density, b.velocity.x(), b.velocity.y(), b.pressure, b.energy};
        for (int k = 0; k < 5; ++k) {
            gx[(size_t)k * n + ic] = ax[k];
            gy[(size_t)k * n + ic] = by[k];
        }
    }
}

// Pointwise: numerical flux of two states (6 doubles: rho, vx, vy, vz, p, e)
// in the face frame; out: 5 doubles.
void zr_flux(int kind, const double *zL, const double *zR, int eos_kind, double gamma, double P0, double e0,
             double *out) {
    auto eos = make_eos(eos_kind, gamma, P0, e0);
    PState L(zL[0], Vector3d(zL[1], zL[2], zL[3]), zL[4], zL[5]);
    PState R(zR[0], Vector3d(zR[1], zR[2], zR[3]), zR[4], zR[5]);
    // NumFlux::create (num_flux.cpp:6-40): GODUNOV, RUSANOV, HLL, HLLC, ...
    math::smf::Flux F = math::NumFlux::create(math::Fluxes(kind))->flux(L, R, *eos);
    out[0] = F.density;
    out[1] = F.momentum.x();
    out[2] = F.momentum.y();
    out[3] = F.momentum.z();
    out[4] = F.energy;
}

double zr_limiter(const char *name, double a, double b) { return math::Limiter(name)(a, b); }

}  // extern "C"
