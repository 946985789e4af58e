// mm_fluid_gpu.h -- zephyr's multi-material solver on one B200, as a drop-in
// for zephyr::math::MmFluid (math/solver/mm_fluid.h:45-163).
//
//     MmFluidGPU solver(mixture);           // was: MmFluid solver(mixture);
//     solver.set_CFL(0.4); solver.set_crp_mode(CrpMode::PLIC);
//     auto z = solver.add_types(mesh).init;
//     ... cell[z] = PState(rho, v, p, beta, mixture) ...
//     solver.update(mesh);
//
// The mesh is a rectangle of zephyr's generator (Rectangle, cell order
// ic = i * ny + j, mesh/euler/amr_cells_gen.cpp:145-151) that has not been
// refined: the multi-material kernels of libzephyr_gpu.so run on structured
// rectangles.  Materials in pressure-temperature equilibrium (MixturePT),
// two of them, each IdealGas or StiffenedGas.  update() copies part.init in,
// runs MmFluid::update (mm_fluid.cpp:112-171) with the bit-exact kernels and
// copies the new state back; set_flags() gives MmFluid::set_flags
// (mm_fluid.cpp:836-885).  CrpMode::MUSCL fills part.grad_a as
// fractions_grad does and, like the reference's assert, throws on a step that
// reaches a composite face (the reference defines no face fraction for it).
// Not on the GPU: gravity (set_gravity with g != 0 throws), fluxes other than
// HLLC and CRP, refined meshes.
//
// Errors throw std::runtime_error with the library's message.
#pragma once

#include <cmath>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include <zephyr_gpu.h>

#include <zephyr/math/solver/mm_fluid.h>
#include <zephyr/phys/matter/eos/ideal_gas.h>
#include <zephyr/phys/matter/eos/stiffened_gas.h>

namespace zephyr::math {

class MmFluidGPU {
public:
    using Parts = MmFluid::Parts;

    /// Fields of the solver on the mesh (MmFluid::Parts).
    Parts part;

    /// MmFluid(const MixturePT&) on CUDA device `device` (mm_fluid.cpp:16-26).
    explicit MmFluidGPU(const phys::MixturePT &mixture, int device = 0) : m_host(mixture), m_mix(mixture) {
        if (zg_create(&m_ctx, device) != ZG_OK)
            throw std::runtime_error("MmFluidGPU: cannot create a context on the CUDA device");
        zg_mmf_default_params(&m_par);
        if (m_mix.size() != 2) throw std::runtime_error("MmFluidGPU: the GPU kernels take mixtures of two materials");
        m_par.n_materials = m_mix.size();
        for (int k = 0; k < m_mix.size(); ++k) {
            phys::Eos &e = m_mix[k];
            zg_material &mt = m_par.materials[k];
            mt.rho_ref = e.density();
            if (auto *ig = dynamic_cast<phys::IdealGas *>(&e)) {
                mt.kind = ZG_EOS_IDEAL;
                mt.gamma = ig->gamma;
                mt.P0 = 0.0;
                mt.e0 = 0.0;
                mt.Cv = ig->Cv;
                mt.T0 = 0.0;
            } else if (auto *sg = dynamic_cast<phys::StiffenedGas *>(&e)) {
                mt.kind = ZG_EOS_STIFFENED;
                mt.gamma = sg->gamma;
                mt.P0 = sg->P0;
                mt.e0 = sg->e0;
                mt.Cv = sg->Cv;
                mt.T0 = sg->T0;
            } else {
                throw std::runtime_error("MmFluidGPU: the GPU kernels take IdealGas and StiffenedGas materials");
            }
        }
        m_dt = 1.0e+300;
    }

    ~MmFluidGPU() { zg_destroy(m_ctx); }

    MmFluidGPU(const MmFluidGPU &) = delete;
    MmFluidGPU &operator=(const MmFluidGPU &) = delete;

    /// MmFluid::add_types (mm_fluid.cpp:28-40): the same fields.
    Parts add_types(EuMesh &mesh) {
        part = m_host.add_types(mesh);
        return part;
    }

    void set_CFL(double CFL) { m_par.CFL = std::max(0.0, std::min(CFL, 1.0)); reconfigure(); }
    void set_accuracy(int acc) { m_par.accuracy = std::min(std::max(1, acc), 2); reconfigure(); }
    /// mm_fluid.cpp:50-61: CRP selects the PLIC composite flux over HLLC,
    /// any other method turns the composite flux off.
    void set_method(Fluxes method) {
        if (method == Fluxes::CRP) {
            m_par.crp_mode = ZG_CRP_PLIC;
        } else if (method == Fluxes::HLLC) {
            m_par.crp_mode = ZG_CRP_NONE;
        } else {
            throw std::runtime_error("MmFluidGPU: the GPU kernels use the mixture HLLC flux (HLLC or CRP)");
        }
        reconfigure();
    }
    void set_crp_mode(CrpMode mode) {
        if (mode == CrpMode::NONE) return;  // mm_fluid.cpp:63-70
        m_par.crp_mode = static_cast<int>(mode);
        reconfigure();
    }
    void set_limiter(const std::string &limiter) {
        const int k = zg_limiter_from_name(limiter.c_str());
        if (k < 0) throw std::runtime_error("Unknown limiter '" + limiter + "'");
        m_par.limiter = k;
        reconfigure();
    }
    void set_splitting(DirSplit splitting) { m_par.split = static_cast<int>(splitting); reconfigure(); }
    void set_gravity(double g) {
        if (g != 0.0) throw std::runtime_error("MmFluidGPU: gravity is not implemented on the GPU");
    }
    double CFL() const { return m_par.CFL; }
    double dt() const { return m_dt; }
    void set_max_dt(double dt) { m_par.max_dt = dt; reconfigure(); }

    /// MmFluid::update (mm_fluid.cpp:112-171) on the GPU.
    void update(EuMesh &mesh) {
        sync_mesh(mesh);
        put_state(mesh);
        check(zg_mmf_update(m_ctx));
        get_state(mesh);
        check(zg_mmf_dt(m_ctx, &m_dt));
        if (m_par.crp_mode == ZG_CRP_MUSCL) get_grad_a(mesh);
    }

    /// MmFluid::set_flags (mm_fluid.cpp:836-885).
    void set_flags(EuMesh &mesh) {
        sync_mesh(mesh);
        put_state(mesh);
        const size_t n = mesh.n_cells();
        m_flags.resize(n);
        check(zg_mmf_set_flags(m_ctx, m_flags.data()));
        for (size_t ic = 0; ic < n; ++ic) mesh[ic].set_flag(m_flags[ic]);
    }

    /// MmFluid::distributor: the reference's own host distributor.
    Distributor distributor() const { return m_host.distributor(); }

    /// The library context (for zg_* calls such as zg_mmf_update_n).
    zg_ctx *context() const { return m_ctx; }

private:
    void check(int rc) const {
        if (rc != ZG_OK) throw std::runtime_error(zg_last_error(m_ctx));
    }
    void reconfigure() {
        if (m_configured) check(zg_mmf_configure(m_ctx, &m_par));
    }

    // Upper end of an axis of Rectangle: the generator places vertex i at
    // lo + ((hi - lo) * i) / n and sets the cell size (hi - lo) / n
    // (mesh/euler/amr_cells_gen.cpp:141-163); the mesh keeps these rounded
    // values, so hi itself is the value near the last vertex that reproduces
    // every vertex and the cell size bit for bit.
    static double axis_end(double lo, const std::vector<double> &v, double h) {
        const int n = static_cast<int>(v.size()) - 1;
        double x = v[n];
        for (int k = 0; k < 64; ++k) x = std::nextafter(x, -INFINITY);
        for (int k = 0; k < 129; ++k, x = std::nextafter(x, INFINITY)) {
            if ((x - lo) / n != h) continue;
            bool ok = true;
            for (int i = 0; i <= n && ok; ++i) ok = lo + ((x - lo) * i) / n == v[i];
            if (ok) return x;
        }
        throw std::runtime_error("MmFluidGPU: the mesh is not a uniform Rectangle");
    }

    // The rectangle behind the mesh: ny cells share the first column's x;
    // the vertex coordinates are the centres of the outer faces (slots L, R,
    // B, T = 0..3) of the first row and column, the boundary flags those of
    // the first and the last cell.
    void sync_mesh(EuMesh &mesh) {
        const mesh::AmrCells &c = mesh.locals();
        const size_t n = c.size();
        if (m_configured && n == m_n) return;
        if (n == 0) throw std::runtime_error("MmFluidGPU: empty mesh");
        for (size_t ic = 0; ic < n; ++ic)
            if (c.level[ic] != 0) throw std::runtime_error("MmFluidGPU: the GPU kernels take unrefined rectangles");
        size_t ny = 1;
        while (ny < n && c.center[ny].x() == c.center[0].x()) ++ny;
        const size_t nx = n / ny;
        if (nx * ny != n) throw std::runtime_error("MmFluidGPU: the mesh is not a Rectangle of nx x ny cells");
        const auto b0 = c.face_begin[0], bn = c.face_begin[n - 1];
        std::vector<double> X(nx + 1), Y(ny + 1);
        for (size_t i = 0; i < nx; ++i) X[i] = c.faces.center[c.face_begin[i * ny] + 0].x();
        X[nx] = c.faces.center[c.face_begin[(nx - 1) * ny] + 1].x();
        for (size_t j = 0; j < ny; ++j) Y[j] = c.faces.center[c.face_begin[j] + 2].y();
        Y[ny] = c.faces.center[c.face_begin[ny - 1] + 3].y();
        const double x_min = X[0], y_min = Y[0];
        const double x_max = axis_end(x_min, X, c.faces.area[b0 + 2]);  // bottom face: hx
        const double y_max = axis_end(y_min, Y, c.faces.area[b0 + 0]);  // left face: hy
        const int bounds[4] = {static_cast<int>(c.faces.boundary[b0 + 0]), static_cast<int>(c.faces.boundary[bn + 1]),
                               static_cast<int>(c.faces.boundary[b0 + 2]), static_cast<int>(c.faces.boundary[bn + 3])};
        check(zg_mesh_rectangle(m_ctx, static_cast<int>(nx), static_cast<int>(ny), x_min, x_max, y_min, y_max, bounds));
        check(zg_mmf_configure(m_ctx, &m_par));
        m_configured = true;
        m_n = n;
    }

    // 14 doubles per cell: density, velocity x, y, pressure, energy,
    // temperature, mass fractions [4], true densities [4] (mmf::PState,
    // math/cfd/models.h:167-180)
    void put_state(EuMesh &mesh) {
        const size_t n = mesh.n_cells();
        m_buf.resize(14 * n);
        for (size_t ic = 0; ic < n; ++ic) {
            EuCell cell = mesh[ic];
            const mmf::PState &z = cell[part.init];
            double *s = m_buf.data() + 14 * ic;
            s[0] = z.density;
            s[1] = z.velocity.x();
            s[2] = z.velocity.y();
            s[3] = z.pressure;
            s[4] = z.energy;
            s[5] = z.temperature;
            for (int k = 0; k < 4; ++k) {
                s[6 + k] = z.mass_frac[k];
                s[10 + k] = z.densities[k];
            }
        }
        check(zg_mmf_state_upload(m_ctx, m_buf.data()));
    }

    // part.grad_a (CrpMode::MUSCL): the volume-fraction gradients of the step
    void get_grad_a(EuMesh &mesh) {
        const size_t n = mesh.n_cells();
        const int m = m_mix.size();
        m_buf.resize(2 * m * n);
        check(zg_mmf_grad_a(m_ctx, m_buf.data()));
        for (size_t ic = 0; ic < n; ++ic) {
            EuCell cell = mesh[ic];
            auto ga = cell[part.grad_a];
            for (int k = 0; k < m; ++k)
                ga[k] = Vector3d(m_buf[2 * (m * ic + k)], m_buf[2 * (m * ic + k) + 1], 0.0);
        }
    }

    void get_state(EuMesh &mesh) {
        const size_t n = mesh.n_cells();
        check(zg_mmf_state_download(m_ctx, m_buf.data()));
        for (size_t ic = 0; ic < n; ++ic) {
            EuCell cell = mesh[ic];
            mmf::PState &z = cell[part.init];
            const double *s = m_buf.data() + 14 * ic;
            z.density = s[0];
            z.velocity = Vector3d(s[1], s[2], 0.0);
            z.pressure = s[3];
            z.energy = s[4];
            z.temperature = s[5];
            for (int k = 0; k < 4; ++k) {
                z.mass_frac[k] = s[6 + k];
                z.densities[k] = s[10 + k];
            }
        }
    }

    MmFluid m_host;  // fields and the host-side distributor
    phys::MixturePT m_mix;
    zg_ctx *m_ctx = nullptr;
    zg_mmf_params m_par{};
    double m_dt;
    bool m_configured = false;
    size_t m_n = 0;
    std::vector<double> m_buf;
    std::vector<int> m_flags;
};

}  // namespace zephyr::math
