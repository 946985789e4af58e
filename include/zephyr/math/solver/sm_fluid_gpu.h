// sm_fluid_gpu.h -- zephyr's single-material solver on one B200, as a drop-in
// for zephyr::math::SmFluid (math/solver/sm_fluid.h:22-112).
//
// A driver swaps the solver type and keeps everything else: the constructor
// takes the same Eos::Ptr, add_types() adds the same fields to the EuMesh and
// returns the same Parts, update() / set_flags() take the EuMesh, and
// distributor() plugs into EuMesh::set_distributor as before:
//
//     SmFluidGPU solver(eos);               // was: SmFluid solver(eos);
//     solver.set_accuracy(2); solver.set_CFL(0.5);
//     solver.set_limiter("MC"); solver.set_method(Fluxes::HLLC);
//     auto z = solver.add_types(mesh).init;
//     mesh.set_max_level(3);
//     mesh.set_distributor(solver.distributor());
//     ...
//     solver.update(mesh); solver.set_flags(mesh); mesh.refine();
//
// The EuMesh stays the owner of the cells, as in the reference.  update()
// copies the mesh geometry to the GPU when it has changed since the last
// call (a refine), copies the state (part.init) and the isolation counters
// (part.wait) in, runs SmFluid::update (sm_fluid.cpp:81-102) with the
// bit-exact kernels of libzephyr_gpu.so, and copies the new state back into
// part.init.  set_flags() computes the flags of SmFluid::set_flags
// (sm_fluid.cpp:517-559) and the limited gradients d_dx, d_dy that the slope
// distributor reads on the GPU.  The mesh adaptation itself (EuMesh::refine
// with the distributor) runs on the host EuMesh, as in the reference; the
// distributor is the reference's own (SmFluid::distributor,
// sm_fluid.cpp:372-470).
//
// Errors: a failed call throws std::runtime_error with the library's message,
// as the reference throws.
//
// Build: compile with zephyr's include path and include/ of this repository;
// link zephyr_b200/libzephyr_gpu.so next to zephyr's own libraries.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include <zephyr_gpu.h>

#include <zephyr/math/solver/sm_fluid.h>
#include <zephyr/phys/matter/eos/ideal_gas.h>
#include <zephyr/phys/matter/eos/stiffened_gas.h>

namespace zephyr::math {

class SmFluidGPU {
public:
    using Parts = SmFluid::Parts;

    /// Fields of the solver on the mesh (SmFluid::Parts).
    Parts part;

    /// SmFluid(Eos::Ptr) on CUDA device `device` (sm_fluid.cpp:16-23 defaults).
    explicit SmFluidGPU(Eos::Ptr eos, int device = 0) : m_host(eos) {
        check_rc(zg_create(&m_ctx, device), "SmFluidGPU: cannot create a context on the CUDA device");
        zg_smf_default_params(&m_par);
        if (auto *ig = dynamic_cast<phys::IdealGas *>(eos.get())) {
            m_par.eos_kind = ZG_EOS_IDEAL;
            m_par.gamma = ig->gamma;
        } else if (auto *sg = dynamic_cast<phys::StiffenedGas *>(eos.get())) {
            m_par.eos_kind = ZG_EOS_STIFFENED;
            m_par.gamma = sg->gamma;
            m_par.P0 = sg->P0;
            m_par.e0 = sg->e0;
        } else {
            throw std::runtime_error("SmFluidGPU: the GPU step supports IdealGas and StiffenedGas");
        }
        m_par.max_dt = std::numeric_limits<double>::max();
        m_dt = NAN;
    }

    ~SmFluidGPU() { zg_destroy(m_ctx); }

    SmFluidGPU(const SmFluidGPU &) = delete;
    SmFluidGPU &operator=(const SmFluidGPU &) = delete;

    /// SmFluid::add_types (sm_fluid.cpp:25-36): the same fields, wait = 0.
    Parts add_types(EuMesh &mesh) {
        part = m_host.add_types(mesh);
        return part;
    }

    void set_CFL(double CFL) { m_par.CFL = std::max(0.0, std::min(CFL, 1.0)); reconfigure(); }
    void set_accuracy(int acc) { m_par.accuracy = std::min(std::max(1, acc), 2); reconfigure(); }
    /// SmFluid::set_axial (sm_fluid.cpp:45-47): the mesh must come from an
    /// axisymmetric generator (Rectangle::set_axial), as in the reference.
    void set_axial(bool axial = true) {
        m_axial = axial;
        m_configured = false;  // the next call uploads the geometry again
    }
    void set_method(Fluxes method) {
        const int f = static_cast<int>(method);
        if (f < ZG_FLUX_GODUNOV || f > ZG_FLUX_CIR2)
            throw std::runtime_error("Unknown numerical flux");
        m_par.flux = f;
        reconfigure();
    }
    void set_limiter(const std::string &limiter) {
        const int k = zg_limiter_from_name(limiter.c_str());
        if (k < 0) throw std::runtime_error("Unknown limiter '" + limiter + "'");
        m_par.limiter = k;
        reconfigure();
    }
    double CFL() const { return m_par.CFL; }
    double dt() const { return m_dt; }
    void set_max_dt(double dt) {
        m_par.max_dt = dt;
        if (m_configured) check(zg_smf_set_max_dt(m_ctx, dt));
    }

    /// SmFluid::update (sm_fluid.cpp:81-102) on the GPU.
    void update(EuMesh &mesh) {
        sync_mesh(mesh);
        put_state(mesh);
        check(zg_smf_update(m_ctx));
        get_state(mesh);
        check(zg_smf_dt(m_ctx, &m_dt));
    }

    /// SmFluid::set_flags (sm_fluid.cpp:517-559): flags of every cell and the
    /// limited gradients d_dx, d_dy of part.init for the slope distributor.
    void set_flags(EuMesh &mesh) const {
        if (!mesh.adaptive()) return;
        sync_mesh(mesh);
        put_state(mesh);
        const size_t n = mesh.n_cells();
        m_flags.resize(n);
        m_gx.resize(4 * n);
        m_gy.resize(4 * n);
        check(zg_smf_set_flags(m_ctx, m_flags.data()));
        check(zg_smf_gradients(m_ctx, m_gx.data(), m_gy.data()));
        for (size_t ic = 0; ic < n; ++ic) {
            EuCell cell = mesh[ic];
            cell.set_flag(m_flags[ic]);
            cell[part.d_dx] = grad_state(m_gx, ic, n);
            cell[part.d_dy] = grad_state(m_gy, ic, n);
            cell[part.d_dz] = smf::PState(0.0, Vector3d(0.0, 0.0, 0.0), 0.0, 0.0);
        }
    }

    /// SmFluid::distributor (sm_fluid.cpp:372-470): the reference's own host
    /// distributor, over the same fields.
    Distributor distributor(const std::string &type = "slope") const { return m_host.distributor(type); }

    // -- beyond the reference's interface ---------------------------------
    /// The library context (for zg_* calls such as zg_smf_update_n).
    zg_ctx *context() const { return m_ctx; }

private:
    static void check_rc(int rc, const char *what) {
        if (rc != ZG_OK) throw std::runtime_error(what);
    }
    void check(int rc) const {
        if (rc != ZG_OK) throw std::runtime_error(zg_last_error(m_ctx));
    }

    void reconfigure() {
        if (m_configured) check(zg_smf_configure(m_ctx, &m_par));
    }

    static smf::PState grad_state(const std::vector<double> &g, size_t ic, size_t n) {
        return smf::PState(g[ic], Vector3d(g[n + ic], g[2 * n + ic], 0.0), g[3 * n + ic], 0.0);
    }

    // Copy the geometry of the mesh to the device when it differs from the
    // last copy: per cell centre, volume, incircle diameter; per face slot (8
    // per cell, slot k of cell i at 8 i + k, UNDEFINED slots flagged -1) the
    // boundary code, neighbour, normal, centre and area (AmrCells / AmrFaces,
    // mesh/euler/amr_cells.h:49-104, amr_faces.h:83-154).
    void sync_mesh(EuMesh &mesh) const {
        const mesh::AmrCells &c = mesh.locals();
        const size_t n = c.size();
        if (n == 0) throw std::runtime_error("SmFluidGPU: empty mesh");
        m_cx.resize(n), m_cy.resize(n), m_vol.resize(n), m_inc.resize(n);
        m_fb.resize(8 * n), m_fn.resize(8 * n);
        m_fnx.resize(8 * n), m_fny.resize(8 * n), m_fcx.resize(8 * n), m_fcy.resize(8 * n), m_fa.resize(8 * n);
        for (size_t ic = 0; ic < n; ++ic) {
            m_cx[ic] = c.center[ic].x();
            m_cy[ic] = c.center[ic].y();
            m_vol[ic] = c.volume[ic];
            m_inc[ic] = c.incircle_diameter(ic);
            const auto b = c.face_begin[ic], e = c.face_begin[ic + 1];
            if (e - b != 8) throw std::runtime_error("SmFluidGPU: the GPU step takes 2-D quadrilateral (AMR) cells");
            for (int s = 0; s < 8; ++s) {
                const auto f = b + s;
                const size_t k = 8 * ic + s;
                m_fb[k] = static_cast<int>(c.faces.boundary[f]);
                m_fn[k] = static_cast<int>(c.faces.adjacent.index[f]);
                m_fnx[k] = c.faces.normal[f].x();
                m_fny[k] = c.faces.normal[f].y();
                m_fcx[k] = c.faces.center[f].x();
                m_fcy[k] = c.faces.center[f].y();
                m_fa[k] = c.faces.area[f];
            }
        }
        const std::uint64_t h = fingerprint(n);
        if (m_configured && h == m_hash && n == m_n) return;
        zg_mesh_view v{static_cast<int>(n), m_cx.data(), m_cy.data(), m_vol.data(), m_inc.data(), m_fb.data(),
                       m_fn.data(), m_fnx.data(), m_fny.data(), m_fcx.data(), m_fcy.data(), m_fa.data()};
        check(zg_mesh_upload(m_ctx, &v));
        if (m_axial) {  // AmrCells::volume_alt, AmrFaces::area_alt
            m_vola.resize(n);
            m_faa.resize(8 * n);
            for (size_t ic = 0; ic < n; ++ic) {
                m_vola[ic] = c.volume_alt[ic];
                for (int s = 0; s < 8; ++s) m_faa[8 * ic + s] = c.faces.area_alt[c.face_begin[ic] + s];
            }
            check(zg_mesh_set_axial(m_ctx, m_vola.data(), m_faa.data()));
        }
        check(zg_smf_configure(m_ctx, &m_par));
        m_configured = true;
        m_hash = h;
        m_n = n;
    }

    // FNV-1a over the geometry arrays (a changed mesh changes it)
    std::uint64_t fingerprint(size_t n) const {
        std::uint64_t h = 1469598103934665603ull;
        auto mix = [&h](const void *p, size_t bytes) {
            const unsigned char *b = static_cast<const unsigned char *>(p);
            for (size_t i = 0; i < bytes; ++i) h = (h ^ b[i]) * 1099511628211ull;
        };
        mix(m_cx.data(), n * sizeof(double));
        mix(m_cy.data(), n * sizeof(double));
        mix(m_fb.data(), 8 * n * sizeof(int));
        mix(m_fn.data(), 8 * n * sizeof(int));
        mix(m_fa.data(), 8 * n * sizeof(double));
        return h;
    }

    void put_state(EuMesh &mesh) const {
        const size_t n = mesh.n_cells();
        m_r.resize(n), m_u.resize(n), m_v.resize(n), m_p.resize(n), m_e.resize(n), m_w.resize(n);
        for (size_t ic = 0; ic < n; ++ic) {
            EuCell cell = mesh[ic];
            const smf::PState &z = cell[part.init];
            m_r[ic] = z.density;
            m_u[ic] = z.velocity.x();
            m_v[ic] = z.velocity.y();
            m_p[ic] = z.pressure;
            m_e[ic] = z.energy;
            m_w[ic] = cell[part.wait];
        }
        check(zg_state_upload(m_ctx, m_r.data(), m_u.data(), m_v.data(), m_p.data(), m_e.data()));
        check(zg_wait_upload(m_ctx, m_w.data()));
    }

    void get_state(EuMesh &mesh) const {
        const size_t n = mesh.n_cells();
        check(zg_state_download(m_ctx, m_r.data(), m_u.data(), m_v.data(), m_p.data(), m_e.data()));
        check(zg_wait_download(m_ctx, m_w.data()));
        for (size_t ic = 0; ic < n; ++ic) {
            EuCell cell = mesh[ic];
            smf::PState &z = cell[part.init];
            z.density = m_r[ic];
            z.velocity = Vector3d(m_u[ic], m_v[ic], 0.0);
            z.pressure = m_p[ic];
            z.energy = m_e[ic];
            cell[part.wait] = m_w[ic];
        }
    }

    SmFluid m_host;  // fields and the host-side distributor of EuMesh::refine
    zg_ctx *m_ctx = nullptr;
    zg_smf_params m_par{};
    double m_dt;
    mutable bool m_configured = false;
    mutable std::uint64_t m_hash = 0;
    mutable size_t m_n = 0;
    mutable std::vector<double> m_cx, m_cy, m_vol, m_inc, m_fnx, m_fny, m_fcx, m_fcy, m_fa;
    mutable std::vector<int> m_fb, m_fn, m_flags, m_w;
    mutable std::vector<double> m_r, m_u, m_v, m_p, m_e, m_gx, m_gy, m_vola, m_faa;
    bool m_axial = false;
};

}  // namespace zephyr::math
