// Test/benchmark infrastructure only: times the reference's own CPU/OpenMP
// time loop (Solver::advance, cpp/src/solver/solver.cpp:917-963) on a model
// given as an insem_case_desc (the same description the backend's native
// setup takes), built through the reference's C++ API (Simulation,
// MacroMesh, Material, Source, Receiver, TimeConfig).  Linked against the
// oracle build of the reference (libinsem_ref.so); bench.py's reference arm
// and CPU-baseline leg call it through ctypes.
#include <chrono>
#include <cmath>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "insem/core/error.hpp"
#include "insem/sim/simulation.hpp"
#include "insem/solver/solver.hpp"
#include "../../in-house-sem_b200/csrc/host/insem_cases.h"

namespace {
thread_local std::string g_err;
const char* kQuantity[5] = {"displacement", "velocity", "acceleration", "pressure", "particle_velocity"};
}  // namespace

extern "C" {

const char* bench_ref_last_error(void) { return g_err.c_str(); }

// Builds the model, runs `warmup` steps, then times `steps` steps.
// out[0] = seconds of the timed steps, out[1] = setup seconds (forest, dofs,
// geometry, solver incl. the stable-dt power iteration), out[2] = total
// unique global points, out[3] = dt, out[4] = n_elements.
int bench_ref_run(const insem_case_desc* d, double dt, int32_t warmup, int32_t steps, double* out) {
  using namespace insem;
  try {
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<double> nodes(d->nodes, d->nodes + 2 * static_cast<std::size_t>(d->n_nodes));
    const int npc = d->quad9 ? 9 : 4;
    std::vector<index_t> cells(d->cells, d->cells + static_cast<std::size_t>(d->n_cells) * npc);
    std::vector<int> region(d->cell_region, d->cell_region + d->n_cells);
    std::vector<mesh::BoundaryFace> bnd;
    for (int i = 0; i < d->n_boundary; ++i) bnd.push_back({d->boundary[3 * i], d->boundary[3 * i + 1], d->boundary[3 * i + 2]});
    auto macro = std::make_shared<mesh::MacroMesh>(d->quad9 ? mesh::CellType::Quad9 : mesh::CellType::Quad4,
                                                   d->axisymmetric ? mesh::CoordSystem::Axisymmetric
                                                                   : mesh::CoordSystem::Cartesian,
                                                   std::move(nodes), std::move(cells), std::move(region), std::move(bnd));
    Discretization disc;
    disc.order = d->order;
    disc.uniform_level = d->uniform_level;
    disc.f_max = d->f_max;
    disc.points_per_wavelength = d->points_per_wavelength;
    disc.max_level = d->max_level;
    disc.azimuthal_order = d->azimuthal_order;
    for (int i = 0; i < d->n_regions; ++i) {
      const double* r = d->regions + 5 * i;
      disc.regions.push_back({r[0], r[1], r[2], r[3], static_cast<int>(r[4])});
    }
    Simulation sim(macro, disc);
    for (int i = 0; i < d->n_materials; ++i)
      sim.set_material(d->material_region[i], d->material_medium[i] == 0
                                                  ? Material::acoustic(d->material_vp[i], d->material_rho[i])
                                                  : Material::elastic(d->material_vp[i], d->material_vs[i], d->material_rho[i]));
    for (int i = 0; i < d->n_bc; ++i) sim.set_boundary(d->bc_tag[i], static_cast<BoundaryType>(d->bc_type[i]));
    for (int i = 0; i < d->n_sources; ++i) {
      const double* p = d->stf_params + 3 * i;
      SourceTimeFunction stf = d->stf_kind[i] == 1   ? SourceTimeFunction::gaussian(p[0], p[1], p[2])
                               : d->stf_kind[i] == 2 ? SourceTimeFunction::gaussian_derivative(p[0], p[1], p[2])
                                                     : SourceTimeFunction::ricker(p[0], p[1], p[2]);
      const double x = d->source_position[2 * i], z = d->source_position[2 * i + 1];
      const double* c = d->source_components + 3 * i;
      switch (d->source_kind[i]) {
        case 0: sim.add_source(Source::force(x, z, c[0], c[1], stf)); break;
        case 1: sim.add_source(Source::moment_tensor(x, z, c[0], c[1], c[2], stf)); break;
        case 2: sim.add_source(Source::monopole(x, z, stf)); break;
        default: sim.add_source(Source::dipole(x, z, c[0], c[1], stf)); break;
      }
    }
    for (int i = 0; i < d->n_receivers; ++i) {
      Receiver r;
      r.name = "r" + std::to_string(i);
      r.position = {d->receiver_position[2 * i], d->receiver_position[2 * i + 1]};
      for (int q = d->receiver_qoffsets[i]; q < d->receiver_qoffsets[i + 1]; ++q)
        r.quantities.push_back(kQuantity[d->receiver_quantities[q]]);
      if (d->receiver_medium[i] >= 0) r.medium = d->receiver_medium[i] == 0 ? "acoustic" : "elastic";
      sim.add_receiver(r);
    }
    TimeConfig tc;
    tc.dt = dt;
    tc.n_steps = warmup + steps;
    tc.record_every = d->record_every;
    tc.energy_every = d->energy_every;
    sim.set_time(tc);
    solver::Solver& s = sim.solver();
    const auto t1 = std::chrono::steady_clock::now();
    s.advance(warmup);
    const auto t2 = std::chrono::steady_clock::now();
    s.advance(steps);
    const auto t3 = std::chrono::steady_clock::now();
    double points = 0.0;
    index_t elements = 0;
    for (std::size_t i = 0; i < s.n_domains(); ++i) {
      points += s.domain(i).n_global();
      elements += s.domain(i).dofs.n_elements();
    }
    out[0] = std::chrono::duration<double>(t3 - t2).count();
    out[1] = std::chrono::duration<double>(t1 - t0).count();
    out[2] = points;
    out[3] = s.dt();
    out[4] = elements;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

}  // extern "C"
