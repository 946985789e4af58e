// dropin_smf.cpp -- TEST INFRASTRUCTURE: the time loop of zephyr's
// problems/single-fluid/smf_test_2D.cpp:34-160 (Riemann2D test, sub-sampled
// cell means, the initial adaptation loop, update + set_flags + refine every
// step), minus the output and the MPI load balancing, run for a bounded
// number of steps once with the reference's zephyr::math::SmFluid and once
// with the drop-in zephyr::math::SmFluidGPU
// (include/zephyr/math/solver/sm_fluid_gpu.h), the solver type being the only
// difference.  Every cell of the two final meshes is compared bit for bit.
//
// Usage: dropin_smf <test> <nx> <max_level> <steps> <accuracy> <limiter> <flux> <CFL> [axial]
// Prints one JSON line and exits 0 when the two runs agree bit for bit.
#include <cstdlib>
#include <string>

#include <zephyr/geom/generator/rectangle.h>
#include <zephyr/math/solver/sm_fluid.h>
#include <zephyr/math/solver/sm_fluid_gpu.h>
#include <zephyr/mesh/euler/eu_mesh.h>
#include <zephyr/phys/tests/test_2D.h>

#include "dropin_common.h"

using namespace zephyr;
using dropin::Snapshot;
using geom::Vector3d;
using geom::generator::Rectangle;
using math::Fluxes;
using mesh::EuCell;
using mesh::EuMesh;

namespace {

template <class Solver>
Snapshot run_smf(int test_case, int nx, int max_level, int steps, int acc, const char *lim, int flux, double CFL,
                 bool axial) {
    using math::smf::PState;
    using math::smf::QState;
    phys::Riemann2D test(test_case);
    auto eos = test.get_eos();

    Rectangle gen(test.xmin(), test.xmax(), test.ymin(), test.ymax());
    gen.set_boundaries(test.boundaries());
    gen.set_nx(nx);
    if (axial) gen.set_axial(true);
    EuMesh mesh(gen);

    Solver solver(eos);
    if (axial) solver.set_axial(true);
    solver.set_accuracy(acc);
    solver.set_CFL(CFL);
    solver.set_limiter(lim);
    solver.set_method(Fluxes(flux));
    auto z = solver.add_types(mesh).init;

    if (max_level > 0) {
        mesh.set_max_level(max_level);
        mesh.set_distributor(solver.distributor());
    }
    const int n_sub = 4;
    auto init_cells = [&test, z, eos, n_sub](EuMesh &m) {
        m.for_each([&](EuCell &cell) {
            QState q(test.density_mean(cell, n_sub), test.momentum_mean(cell, n_sub), test.energy_mean(cell, n_sub));
            cell[z] = PState(q, *eos);
        });
    };
    if (max_level > 0) {
        for (int k = 0; k < mesh.max_level() + 3; ++k) {
            init_cells(mesh);
            solver.set_flags(mesh);
            mesh.refine();
        }
    }
    init_cells(mesh);

    Snapshot s;
    double t = 0.0;
    for (int step = 0; step < steps && t < test.max_time(); ++step) {
        solver.set_max_dt(test.max_time() - t);
        solver.update(mesh);
        if (max_level > 0) {
            solver.set_flags(mesh);
            mesh.refine();
        }
        t += solver.dt();
        s.dts.push_back(solver.dt());
    }
    s.cells = mesh.n_cells();
    for (size_t ic = 0; ic < s.cells; ++ic) {
        EuCell cell = mesh[ic];
        const PState &p = cell[z];
        const double row[] = {cell.center().x(), cell.center().y(), double(cell.level()), p.density,
                              p.velocity.x(), p.velocity.y(), p.pressure, p.energy, double(cell[solver.part.wait])};
        s.data.insert(s.data.end(), std::begin(row), std::end(row));
    }
    return s;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 9 && argc != 10) return 2;
    const bool axial = argc == 10 && std::string(argv[9]) == "axial";
    try {
        const int test_case = std::atoi(argv[1]), nx = std::atoi(argv[2]), max_level = std::atoi(argv[3]);
        const int steps = std::atoi(argv[4]), acc = std::atoi(argv[5]), flux = std::atoi(argv[7]);
        const double CFL = std::atof(argv[8]);
        auto ref = run_smf<math::SmFluid>(test_case, nx, max_level, steps, acc, argv[6], flux, CFL, axial);
        auto gpu = run_smf<math::SmFluidGPU>(test_case, nx, max_level, steps, acc, argv[6], flux, CFL, axial);
        return dropin::report("smf", ref, gpu);
    } catch (const std::exception &e) {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 3;
    }
}
