// dropin_mmf.cpp -- TEST INFRASTRUCTURE: a multi-material loop in the
// manner of zephyr's problems/multi-fluid/mmf_air_water.cpp (MixturePT of air
// and water, PState(density, velocity, pressure, fractions, mixture) initial
// states, update per step) on an unrefined rectangle, run once with the
// reference's zephyr::math::MmFluid and once with the drop-in
// zephyr::math::MmFluidGPU (include/zephyr/math/solver/mm_fluid_gpu.h), the
// solver type being the only difference; every cell is compared bit for bit.
//
// Usage: dropin_mmf <nx> <steps> <crp_mode> <accuracy> <CFL>
// Prints one JSON line and exits 0 when the two runs agree bit for bit.
#include <cstdlib>
#include <string>

#include <zephyr/geom/generator/rectangle.h>
#include <zephyr/math/solver/mm_fluid.h>
#include <zephyr/math/solver/mm_fluid_gpu.h>
#include <zephyr/mesh/euler/eu_mesh.h>
#include <zephyr/phys/matter/eos/ideal_gas.h>
#include <zephyr/phys/matter/eos/stiffened_gas.h>

#include "dropin_common.h"

using namespace zephyr;
using dropin::Snapshot;
using geom::Boundary;
using geom::Vector3d;
using geom::generator::Rectangle;
using mesh::EuCell;
using mesh::EuMesh;
using phys::Eos;

namespace {

template <class Solver>
Snapshot run_mmf(int nx, int steps, int crp_mode, int acc, double CFL) {
    using math::mmf::PState;
    using phys::Fractions;
    Eos::Ptr air = phys::IdealGas::create("Air");
    Eos::Ptr water = phys::StiffenedGas::create("Water");
    phys::MixturePT mixture = {air, water};

    // shock in air running into a water column: [0, 0.1]^2 m
    Rectangle gen(0.0, 0.1, 0.0, 0.1);
    gen.set_nx(nx);
    gen.set_boundaries({.left = Boundary::ZOE, .right = Boundary::ZOE, .bottom = Boundary::WALL,
                        .top = Boundary::WALL});
    EuMesh mesh(gen);

    Solver solver(mixture);
    solver.set_CFL(CFL);
    solver.set_accuracy(acc);
    solver.set_crp_mode(math::CrpMode(crp_mode));
    auto z = solver.add_types(mesh).init;

    const PState air0(1.2, Vector3d(0.0, 0.0, 0.0), 1.0e5, Fractions::Pure(0), mixture);
    const PState air1(4.575, Vector3d(744.0, 0.0, 0.0), 1.0e6, Fractions::Pure(0), mixture);
    const PState water0(1000.0, Vector3d(0.0, 0.0, 0.0), 1.0e5, Fractions::Pure(1), mixture);
    for (size_t ic = 0; ic < mesh.n_cells(); ++ic) {
        EuCell cell = mesh[ic];
        const Vector3d c = cell.center();
        const double dx = c.x() - 0.05, dy = c.y() - 0.05;
        if (dx * dx + dy * dy < 0.02 * 0.02) cell[z] = water0;
        else if (c.x() < 0.02) cell[z] = air1;
        else cell[z] = air0;
    }

    Snapshot s;
    for (int step = 0; step < steps; ++step) {
        solver.update(mesh);
        s.dts.push_back(solver.dt());
    }
    s.cells = mesh.n_cells();
    for (size_t ic = 0; ic < s.cells; ++ic) {
        EuCell cell = mesh[ic];
        const PState &p = cell[z];
        const double row[] = {cell.center().x(), cell.center().y(), p.density, p.velocity.x(), p.velocity.y(),
                              p.pressure, p.energy, p.temperature, p.mass_frac[0], p.mass_frac[1],
                              p.densities[0], p.densities[1]};
        s.data.insert(s.data.end(), std::begin(row), std::end(row));
    }
    return s;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 6) return 2;
    try {
        const int nx = std::atoi(argv[1]), steps = std::atoi(argv[2]), crp = std::atoi(argv[3]);
        const int acc = std::atoi(argv[4]);
        const double CFL = std::atof(argv[5]);
        auto ref = run_mmf<math::MmFluid>(nx, steps, crp, acc, CFL);
        auto gpu = run_mmf<math::MmFluidGPU>(nx, steps, crp, acc, CFL);
        return dropin::report("mmf", ref, gpu);
    } catch (const std::exception &e) {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 3;
    }
}
