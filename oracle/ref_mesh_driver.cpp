// ref_mesh_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own EuMesh (mesh/euler/*, mesh/amr/*, geom/*) and its
// SmFluid, compiled from the reference sources, and exposes a C interface so
// that tests can check the oracle's AMR restatement, and the GPU, against the
// reference's refine() (flags, balancing, split/merge, hanging faces,
// distributor) and against its step on refined meshes.  Built by
// oracle/ref_build.py into oracle/_ref/libzref_mesh.so.
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <zephyr/geom/generator/rectangle.h>
#include <zephyr/io/pvd_file.h>
#include <zephyr/io/vtu_file.h>
#include <zephyr/math/solver/sm_fluid.h>
#include <zephyr/mesh/euler/eu_mesh.h>
#include <zephyr/phys/matter/eos/ideal_gas.h>
#include <zephyr/phys/matter/eos/stiffened_gas.h>
#include <zephyr/utils/threads.h>

using namespace zephyr;
using geom::Boundary;
using geom::Vector3d;
using math::SmFluid;
using math::smf::PState;
using mesh::EuCell;
using mesh::EuMesh;

namespace {

struct RefMesh {
    std::unique_ptr<EuMesh> mesh;
    std::unique_ptr<SmFluid> solver;
    SmFluid::Parts part;
    phys::Eos::Ptr eos;
};

}  // namespace

extern "C" {

// Mesh of Rectangle(x_min, x_max, y_min, y_max) with nx by ny cells, boundary
// flags {left, right, bottom, top}, an SmFluid with the given settings, and
// AMR up to max_level with the solver's distributor ("slope" or "const").
// With axial != 0 the generator and the solver are axisymmetric
// (Rectangle::set_axial, SmFluid::set_axial: y is the radius).
void *zm_create_ax(int nx, int ny, double x_min, double x_max, double y_min, double y_max, const int *bounds,
                   int eos_kind, double gamma, double P0, double e0, int flux, const char *limiter, int acc,
                   double CFL, int max_level, const char *distributor, int axial) {
    auto *r = new RefMesh();
    geom::generator::Rectangle gen(x_min, x_max, y_min, y_max);
    gen.set_boundaries({.left = Boundary(bounds[0]), .right = Boundary(bounds[1]),
                        .bottom = Boundary(bounds[2]), .top = Boundary(bounds[3])});
    gen.set_sizes(nx, ny);
    if (axial) gen.set_axial(true);
    r->mesh = std::make_unique<EuMesh>(gen);
    r->eos = eos_kind == 0 ? phys::Eos::Ptr(phys::IdealGas::create(gamma))
                           : phys::Eos::Ptr(phys::StiffenedGas::create(gamma, P0, e0));
    r->solver = std::make_unique<SmFluid>(r->eos);
    r->solver->set_accuracy(acc);
    r->solver->set_CFL(CFL);
    r->solver->set_limiter(limiter);
    r->solver->set_method(math::Fluxes(flux));
    r->part = r->solver->add_types(*r->mesh);
    r->mesh->set_max_level(max_level);
    r->mesh->set_distributor(r->solver->distributor(distributor));
    if (axial) r->solver->set_axial(true);
    return r;
}

void *zm_create(int nx, int ny, double x_min, double x_max, double y_min, double y_max, const int *bounds,
                int eos_kind, double gamma, double P0, double e0, int flux, const char *limiter, int acc,
                double CFL, int max_level, const char *distributor) {
    return zm_create_ax(nx, ny, x_min, x_max, y_min, y_max, bounds, eos_kind, gamma, P0, e0, flux, limiter, acc,
                        CFL, max_level, distributor, 0);
}

// The axisymmetric geometry of an axial mesh: per cell volume_alt, per face
// slot (8 per cell) area_alt (AmrCells::volume_alt, AmrFaces::area_alt).
int zm_axial_geometry(void *p, double *vol_alt, double *area_alt) {
    auto &c = static_cast<RefMesh *>(p)->mesh->locals();
    int n = (int)c.size();
    for (int ic = 0; ic < n; ++ic) {
        vol_alt[ic] = c.volume_alt[ic];
        int b = (int)c.face_begin[ic], e = (int)c.face_begin[ic + 1];
        if (e - b != 8) return -1;
        for (int s = 0; s < 8; ++s) area_alt[8 * ic + s] = c.faces.area_alt[b + s];
    }
    return 0;
}

void zm_free(void *p) { delete static_cast<RefMesh *>(p); }

// Worker threads of the reference's threads::for_each (0 or 1: sequential).
void zm_threads(int n) {
    if (n < 2) utils::threads::off();
    else utils::threads::on(n);
}

int zm_n_cells(void *p) { return (int)static_cast<RefMesh *>(p)->mesh->n_cells(); }

// Per cell: centre (x, y), volume, incircle diameter, level, flag, b_idx, z_idx.
void zm_cells(void *p, double *cx, double *cy, double *vol, double *inc, int *level, int *flag, int *b_idx,
              int *z_idx) {
    auto &c = static_cast<RefMesh *>(p)->mesh->locals();
    for (int i = 0; i < (int)c.size(); ++i) {
        cx[i] = c.center[i].x();
        cy[i] = c.center[i].y();
        vol[i] = c.volume[i];
        inc[i] = c.incircle_diameter(i);
        level[i] = c.level[i];
        flag[i] = c.flag[i];
        b_idx[i] = (int)c.b_idx[i];
        z_idx[i] = (int)c.z_idx[i];
    }
}

// Per face slot (8 per cell, slot order of face_begin): boundary flag,
// neighbour index, area, normal (x, y), centre (x, y).
int zm_faces(void *p, int *boundary, int *neib, double *area, double *nx, double *ny, double *fx, double *fy) {
    auto &c = static_cast<RefMesh *>(p)->mesh->locals();
    int n = (int)c.size();
    for (int ic = 0; ic < n; ++ic) {
        int b = (int)c.face_begin[ic], e = (int)c.face_begin[ic + 1];
        if (e - b != 8) return -1;
        for (int s = 0; s < 8; ++s) {
            int f = b + s, k = 8 * ic + s;
            boundary[k] = int(c.faces.boundary[f]);
            neib[k] = (int)c.faces.adjacent.index[f];
            area[k] = c.faces.area[f];
            nx[k] = c.faces.normal[f].x();
            ny[k] = c.faces.normal[f].y();
            fx[k] = c.faces.center[f].x();
            fy[k] = c.faces.center[f].y();
        }
    }
    return 0;
}

// The 9 mapping vertices of every cell (x, y), in SqQuad order.
void zm_verts(void *p, double *vx, double *vy) {
    auto &c = static_cast<RefMesh *>(p)->mesh->locals();
    int n = (int)c.size();
    for (int ic = 0; ic < n; ++ic) {
        int b = (int)c.node_begin[ic];
        for (int k = 0; k < 9; ++k) {
            vx[9 * ic + k] = c.verts[b + k].x();
            vy[9 * ic + k] = c.verts[b + k].y();
        }
    }
}

void zm_set_state(void *p, const double *rho, const double *u, const double *v, const double *pr,
                  const double *e) {
    auto *r = static_cast<RefMesh *>(p);
    int n = (int)r->mesh->n_cells();
    for (int ic = 0; ic < n; ++ic) {
        EuCell cell = (*r->mesh)[ic];
        cell[r->part.init] = PState(rho[ic], Vector3d(u[ic], v[ic], 0.0), pr[ic], e[ic]);
    }
}

void zm_get_state(void *p, double *rho, double *u, double *v, double *pr, double *e) {
    auto *r = static_cast<RefMesh *>(p);
    int n = (int)r->mesh->n_cells();
    for (int ic = 0; ic < n; ++ic) {
        EuCell cell = (*r->mesh)[ic];
        const PState &z = cell[r->part.init];
        rho[ic] = z.density;
        u[ic] = z.velocity.x();
        v[ic] = z.velocity.y();
        pr[ic] = z.pressure;
        e[ic] = z.energy;
    }
}

void zm_set_wait(void *p, const int *w) {
    auto *r = static_cast<RefMesh *>(p);
    int n = (int)r->mesh->n_cells();
    for (int ic = 0; ic < n; ++ic) (*r->mesh)[ic][r->part.wait] = w[ic];
}

void zm_get_wait(void *p, int *w) {
    auto *r = static_cast<RefMesh *>(p);
    int n = (int)r->mesh->n_cells();
    for (int ic = 0; ic < n; ++ic) w[ic] = (*r->mesh)[ic][r->part.wait];
}

void zm_set_max_dt(void *p, double dt) { static_cast<RefMesh *>(p)->solver->set_max_dt(dt); }

double zm_step(void *p) {
    auto *r = static_cast<RefMesh *>(p);
    r->solver->update(*r->mesh);
    return r->solver->dt();
}

// SmFluid::set_flags; the flags are returned in cell order.
void zm_solver_flags(void *p, int *flags) {
    auto *r = static_cast<RefMesh *>(p);
    r->solver->set_flags(*r->mesh);
    auto &c = r->mesh->locals();
    for (int i = 0; i < (int)c.size(); ++i) flags[i] = c.flag[i];
}

// The limited gradients SmFluid::compute_grad left in d_dx, d_dy: density,
// velocity x, velocity y, pressure (4 n each, field-major).
void zm_grad(void *p, double *gx, double *gy) {
    auto *r = static_cast<RefMesh *>(p);
    int n = (int)r->mesh->n_cells();
    for (int ic = 0; ic < n; ++ic) {
        EuCell cell = (*r->mesh)[ic];
        const PState &dx = cell[r->part.d_dx], &dy = cell[r->part.d_dy];
        const double vx[4] = {dx.density, dx.velocity.x(), dx.velocity.y(), dx.pressure};
        const double vy[4] = {dy.density, dy.velocity.x(), dy.velocity.y(), dy.pressure};
        for (int k = 0; k < 4; ++k) {
            gx[(size_t)k * n + ic] = vx[k];
            gy[(size_t)k * n + ic] = vy[k];
        }
    }
}

// Flags chosen by the caller (tests of refine on arbitrary flags).
void zm_put_flags(void *p, const int *flags) {
    auto &c = static_cast<RefMesh *>(p)->mesh->locals();
    for (int i = 0; i < (int)c.size(); ++i) c.flag[i] = flags[i];
}

// EuMesh::refine (eu_mesh.cpp:290-359); returns the new number of cells.
int zm_refine(void *p) {
    auto *r = static_cast<RefMesh *>(p);
    r->mesh->refine();
    return (int)r->mesh->n_cells();
}

// EuMesh::check_base (eu_mesh.cpp:585-679): 0 when the mesh is consistent.
int zm_check(void *p) { return static_cast<RefMesh *>(p)->mesh->check_base() < 0 ? -1 : 0; }

// EuMesh::check_refined (eu_mesh.cpp:681-): 0 when an adapted mesh is
// consistent (hanging faces allowed).
int zm_check_refined(void *p) { return static_cast<RefMesh *>(p)->mesh->check_refined() < 0 ? -1 : 0; }

// ---- output (io/vtu_file.cpp, io/pvd_file.cpp) ----

namespace {
// Variables: the named ones of io/variable.cpp (comma-separated, may be
// empty) and, with `with_state`, the SmFluid state as the single-fluid driver
// writes it (smf_test_2D.cpp:95-99): density, vel.x, vel.y, pressure, energy.
io::Variables out_variables(RefMesh *r, const char *names, int with_state) {
    io::Variables vars;
    std::string list(names ? names : "");
    size_t pos = 0;
    while (pos < list.size()) {
        size_t comma = list.find(',', pos);
        if (comma == std::string::npos) comma = list.size();
        if (comma > pos) vars.append(list.substr(pos, comma - pos));
        pos = comma + 1;
    }
    if (with_state) {
        auto z = r->part.init;
        vars += {"density", [z](EuCell &cell) -> double { return cell[z].density; }};
        vars += {"vel.x", [z](EuCell &cell) -> double { return cell[z].velocity.x(); }};
        vars += {"vel.y", [z](EuCell &cell) -> double { return cell[z].velocity.y(); }};
        vars += {"pressure", [z](EuCell &cell) -> double { return cell[z].pressure; }};
        vars += {"energy", [z](EuCell &cell) -> double { return cell[z].energy; }};
    }
    return vars;
}
}  // namespace

// VtuFile::save of the mesh with the variables above.
void zm_vtu(void *p, const char *filename, const char *names, int with_state) {
    auto *r = static_cast<RefMesh *>(p);
    io::VtuFile::save(filename, *r->mesh, out_variables(r, names, with_state));
}

// PvdFile(filename, directory); save(mesh, timestep) with the variables above.
void *zm_pvd_open(const char *filename, const char *directory) {
    auto *f = new io::PvdFile();
    f->open(filename, directory);
    return f;
}
void zm_pvd_save(void *pvd, void *p, double timestep, const char *names, int with_state) {
    auto *f = static_cast<io::PvdFile *>(pvd);
    f->variables = out_variables(static_cast<RefMesh *>(p), names, with_state);
    f->save(*static_cast<RefMesh *>(p)->mesh, timestep);
}
void zm_pvd_close(void *pvd) { delete static_cast<io::PvdFile *>(pvd); }

}  // extern "C"
