// Test infrastructure only: the drop-in shim that a maintainer adds to the
// reference behind INSEM_ENABLE_CUDA, compiled against the reference's own
// sources and run end to end.
//
// The reference's Simulation does all of the setup on the CPU (forest,
// geometry, DofMap, Solver construction with its stable time step,
// cpp/src/solver/solver.cpp:91-145).  `cuda_create` below is the shim's
// Solver::cuda_create: it packs exactly the arrays the reference Solver's
// time loop reads into the C ABI structs of include/insem_cuda.h and creates
// the device solver; the time loop is then forwarded (advance, run) and the
// results come back into the reference Solver's own trace, sample-time and
// energy storage, which is what `Solver::traces()` and friends return.  The
// reference keeps those members private (solver.hpp:155-228) and offers no
// hook, so this translation unit reads them with the access specifiers
// opened, as refdump.cpp does; a maintainer's shim would be a member
// function instead.
//
// Python face (pybind11 module `_cudashim`, built into oracle/_ref/float):
//   case(mesh, disc, materials, boundaries, sources, receivers, time) -> Case
//   Case.run_cuda(first)  advance(first) then run() through the backend;
//                         returns {"dt", "n_steps", "times", "traces": {...},
//                         "energy"} from the reference Solver's storage.
//   Case.run_cpu(first)   the same time loop on the reference's CPU path.

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstdint>
#include <map>
#include <memory>
#include <random>
#include <string>
#include <vector>

#define private public
#define protected public
#include "insem/core/error.hpp"
#include "insem/sim/simulation.hpp"
#include "insem/solver/solver.hpp"
#undef private
#undef protected

#include "insem_cuda.h"

namespace py = pybind11;
using namespace insem;

namespace {

void cuda_check(int rc) {
  if (rc != INSEM_CUDA_OK) throw Error(insem_cuda_last_error());
}

int32_t quantity_code(const std::string& q) {
  if (q == "displacement") return INSEM_Q_DISPLACEMENT;
  if (q == "velocity") return INSEM_Q_VELOCITY;
  if (q == "acceleration") return INSEM_Q_ACCELERATION;
  if (q == "pressure") return INSEM_Q_PRESSURE;
  if (q == "particle_velocity") return INSEM_Q_PARTICLE_VELOCITY;
  throw Error("unknown quantity '" + q + "'");
}

// Borrowed views of one reference Solver, kept alive while the device solver is created.
struct Packed {
  std::vector<insem_cuda_domain> domains;
  std::vector<std::vector<insem_cuda_block>> blocks;
  std::vector<std::vector<int32_t>> axis_components;
  std::vector<std::vector<uint8_t>> axial;
  std::vector<insem_cuda_source> sources;
  std::vector<insem_cuda_receiver> receivers;
  std::vector<std::vector<int32_t>> quantities;
  insem_cuda_problem problem{};
};

// Solver::cuda_create of the shim: what the time loop reads, as the C ABI borrows it.
insem_cuda_solver* cuda_create(solver::Solver& s, Packed& pk) {
  const physics::KernelBasis& kb = s.kernel_basis_;
  pk.domains.resize(s.domains_.size());
  pk.blocks.resize(s.domains_.size());
  pk.axis_components.resize(s.domains_.size());
  pk.axial.clear();
  for (std::size_t i = 0; i < s.domains_.size(); ++i) {
    const solver::Domain& d = s.domains_[i];
    for (const ops::ElementBlock& b : d.blocks) {
      pk.axial.emplace_back(b.axial.begin(), b.axial.end());
      pk.blocks[i].push_back({static_cast<int32_t>(b.kind), b.azimuthal_order, static_cast<int32_t>(b.elements.size()),
                              b.elements.data(), b.metric.data(), b.coef0.data(),
                              b.coef1.empty() ? nullptr : b.coef1.data(), b.wr.empty() ? nullptr : b.wr.data(),
                              b.hoop.empty() ? nullptr : b.hoop.data(), b.r.empty() ? nullptr : b.r.data(),
                              pk.axial.back().empty() ? nullptr : pk.axial.back().data()});
    }
    const ops::DofMap& m = d.dofs;
    pk.axis_components[i].assign(d.axis_components.begin(), d.axis_components.end());
    insem_cuda_domain& cd = pk.domains[i];
    cd.medium = static_cast<int32_t>(d.medium);
    cd.ncomp = d.ncomp;
    cd.azimuthal_order = d.azimuthal_order;
    cd.dofs = {m.ngll(), m.n_elements(), m.n_global(), m.l2g_.data(), m.n_rows(), m.row_offsets_.data(),
               m.row_dofs_.data(), m.row_weights_.data(), m.t_offsets_.data(), m.t_slots_.data(),
               m.has_constraints() ? m.t_weights_.data() : nullptr};
    cd.n_blocks = static_cast<int32_t>(pk.blocks[i].size());
    cd.blocks = pk.blocks[i].data();
    cd.mass = d.mass.data();
    cd.inv_mass = d.inv_mass.data();
    cd.n_absorbing = static_cast<int32_t>(d.absorbing_points.size());
    cd.absorbing_points = d.absorbing_points.data();
    cd.absorbing_coef = d.absorbing_coef.data();
    cd.n_dirichlet = static_cast<int32_t>(d.dirichlet_points.size());
    cd.dirichlet_points = d.dirichlet_points.data();
    cd.n_axis = static_cast<int32_t>(d.axis_points.size());
    cd.axis_points = d.axis_points.data();
    cd.n_axis_components = static_cast<int32_t>(pk.axis_components[i].size());
    cd.axis_components = pk.axis_components[i].data();
  }
  for (const auto& t : s.sources_) {
    insem_cuda_stf stf{static_cast<int32_t>(t.stf.kind), t.stf.f0, t.stf.t0, t.stf.amplitude,
                       static_cast<int32_t>(t.stf.samples.size()), t.stf.samples.data(), t.stf.sample_dt};
    pk.sources.push_back({t.domain, static_cast<int32_t>(t.points.size()), t.points.data(), t.coef.data(), stf});
  }
  pk.quantities.clear();
  pk.quantities.reserve(s.receivers_.size());
  for (const auto& r : s.receivers_) {
    pk.quantities.emplace_back();
    for (const std::string& q : r.quantities) pk.quantities.back().push_back(quantity_code(q));
    pk.receivers.push_back({r.domain, static_cast<int32_t>(r.points.size()), r.points.data(), r.value.data(),
                            r.d_dx.data(), r.d_dz.data(), r.rho, static_cast<int32_t>(pk.quantities.back().size()),
                            pk.quantities.back().data()});
  }
  insem_cuda_problem& p = pk.problem;
  p.basis = {kb.ngll, kb.D.data(), kb.Dj.empty() ? nullptr : kb.Dj.data(), kb.w2.data()};
  p.n_domains = static_cast<int32_t>(pk.domains.size());
  p.domains = pk.domains.data();
  p.coupling = {static_cast<int32_t>(s.coupling_.fluid_points.size()), s.coupling_.fluid_points.data(),
                s.coupling_.solid_points.data(), s.coupling_.cx.data(), s.coupling_.cz.data()};
  p.n_sources = static_cast<int32_t>(pk.sources.size());
  p.sources = pk.sources.data();
  p.n_receivers = static_cast<int32_t>(pk.receivers.size());
  p.receivers = pk.receivers.data();
  p.dt = s.dt_;
  p.n_steps = s.n_steps_;
  p.record_every = s.record_every_;
  p.energy_every = s.energy_every_;
  insem_cuda_options o{};
  o.use_graphs = 1;
  o.check_finite = 1;
  insem_cuda_solver* h = nullptr;
  cuda_check(insem_cuda_solver_create(&p, &o, &h));
  return h;
}

// The forwarded results: the reference Solver's own storage filled from the device.
void fetch(solver::Solver& s, insem_cuda_solver* h) {
  s.step_ = insem_cuda_solver_step(h);
  const int32_t ns = insem_cuda_solver_n_samples(h);
  s.sample_times_.assign(static_cast<std::size_t>(ns), 0.0);
  cuda_check(insem_cuda_solver_times(h, s.sample_times_.data()));
  INSEM_CHECK(insem_cuda_solver_n_traces(h) == static_cast<int32_t>(s.traces_.size()), "trace count differs");
  for (std::size_t t = 0; t < s.traces_.size(); ++t) {
    auto& tr = s.traces_[t];
    INSEM_CHECK(insem_cuda_solver_trace_ncomp(h, static_cast<int32_t>(t)) == tr.ncomp, "trace width differs");
    tr.data.assign(static_cast<std::size_t>(ns) * tr.ncomp, 0.0);
    cuda_check(insem_cuda_solver_trace(h, static_cast<int32_t>(t), tr.data.data()));
  }
  std::vector<double> e(3 * static_cast<std::size_t>(s.n_steps_ + 1));
  int32_t ne = 0;
  cuda_check(insem_cuda_solver_energy(h, e.data(), static_cast<int32_t>(e.size() / 3), &ne));
  s.energy_.clear();
  for (int32_t i = 0; i < ne; ++i) s.energy_.push_back({e[3 * i], e[3 * i + 1], e[3 * i + 2]});
}

SourceTimeFunction make_stf(const py::dict& d) {
  const std::string kind = d["kind"].cast<std::string>();
  const double amp = d["amplitude"].cast<double>();
  if (kind == "samples")
    return SourceTimeFunction::sampled(d["samples"].cast<std::vector<double>>(), d["sample_dt"].cast<double>(), amp);
  const double f0 = d["f0"].cast<double>(), t0 = d["t0"].cast<double>();
  if (kind == "ricker") return SourceTimeFunction::ricker(f0, t0, amp);
  if (kind == "gaussian") return SourceTimeFunction::gaussian(f0, t0, amp);
  return SourceTimeFunction::gaussian_derivative(f0, t0, amp);
}

struct Case {
  std::unique_ptr<Simulation> sim;

  py::dict results(solver::Solver& s) {
    py::dict traces;
    for (const auto& t : s.traces_) {
      const std::size_t n = t.data.size() / static_cast<std::size_t>(t.ncomp);
      py::array_t<double> a({n, static_cast<std::size_t>(t.ncomp)});
      std::copy(t.data.begin(), t.data.end(), a.mutable_data());
      traces[py::str(t.receiver + "." + t.quantity)] = a;
    }
    py::array_t<double> times(s.sample_times_.size());
    std::copy(s.sample_times_.begin(), s.sample_times_.end(), times.mutable_data());
    py::array_t<double> energy({s.energy_.size(), std::size_t{3}});
    for (std::size_t i = 0; i < s.energy_.size(); ++i)
      for (int k = 0; k < 3; ++k) energy.mutable_data()[3 * i + k] = s.energy_[i][k];
    py::dict out;
    out["dt"] = s.dt_;
    out["n_steps"] = s.n_steps_;
    out["step"] = s.step_;
    out["times"] = times;
    out["traces"] = traces;
    out["energy"] = energy;
    return out;
  }

  py::dict run_cuda(int first) {
    solver::Solver& s = sim->solver();  // the reference's CPU setup
    Packed pk;
    insem_cuda_solver* h = cuda_create(s, pk);
    try {
      cuda_check(insem_cuda_solver_advance(h, first));
      cuda_check(insem_cuda_solver_run(h));
      fetch(s, h);
    } catch (...) {
      insem_cuda_solver_destroy(h);
      throw;
    }
    insem_cuda_solver_destroy(h);
    return results(s);
  }

  py::dict run_cpu(int first) {
    solver::Solver& s = sim->solver();
    s.advance(first);
    s.run();
    return results(s);
  }
};

Case make_case(const py::dict& mesh, const py::dict& disc, const py::list& materials, const py::list& boundaries,
               const py::list& sources, const py::list& receivers, const py::dict& time) {
  using IArr = py::array_t<int32_t, py::array::c_style | py::array::forcecast>;
  using DArr = py::array_t<double, py::array::c_style | py::array::forcecast>;
  const DArr nodes = mesh["nodes"].cast<DArr>();
  const IArr cells = mesh["cells"].cast<IArr>(), region = mesh["region"].cast<IArr>(),
             bnd = mesh["boundary"].cast<IArr>();
  std::vector<mesh::BoundaryFace> faces;
  for (py::ssize_t i = 0; i < bnd.shape(0); ++i)
    faces.push_back({bnd.at(i, 0), static_cast<int>(bnd.at(i, 1)), static_cast<int>(bnd.at(i, 2))});
  auto macro = std::make_shared<mesh::MacroMesh>(
      mesh["quad9"].cast<bool>() ? mesh::CellType::Quad9 : mesh::CellType::Quad4,
      mesh["axisymmetric"].cast<bool>() ? mesh::CoordSystem::Axisymmetric : mesh::CoordSystem::Cartesian,
      std::vector<double>(nodes.data(), nodes.data() + nodes.size()),
      std::vector<index_t>(cells.data(), cells.data() + cells.size()),
      std::vector<int>(region.data(), region.data() + region.size()), faces);
  Discretization d;
  d.order = disc["order"].cast<int>();
  d.uniform_level = disc["uniform_level"].cast<int>();
  d.f_max = disc["f_max"].cast<double>();
  d.points_per_wavelength = disc["points_per_wavelength"].cast<double>();
  d.max_level = disc["max_level"].cast<int>();
  d.azimuthal_order = disc["azimuthal_order"].cast<int>();
  for (const auto& r : disc["regions"].cast<py::list>()) {
    const auto t = r.cast<std::vector<double>>();
    d.regions.push_back({t[0], t[1], t[2], t[3], static_cast<int>(t[4])});
  }
  Case c;
  c.sim = std::make_unique<Simulation>(macro, d);
  for (const auto& m : materials) {
    const auto t = m.cast<py::tuple>();
    const int reg = t[0].cast<int>();
    const double vp = t[2].cast<double>(), vs = t[3].cast<double>(), rho = t[4].cast<double>();
    c.sim->set_material(reg, t[1].cast<std::string>() == "acoustic" ? Material::acoustic(vp, rho)
                                                                       : Material::elastic(vp, vs, rho));
  }
  for (const auto& b : boundaries) {
    const auto t = b.cast<py::tuple>();
    c.sim->set_boundary(t[0].cast<int>(), boundary_type_from_string(t[1].cast<std::string>()));
  }
  for (const auto& so : sources) {
    const auto s = so.cast<py::dict>();
    const std::string kind = s["kind"].cast<std::string>();
    const double x = s["x"].cast<double>(), z = s["z"].cast<double>();
    const auto cp = s["components"].cast<std::vector<double>>();
    const SourceTimeFunction stf = make_stf(s["stf"].cast<py::dict>());
    if (kind == "monopole") c.sim->add_source(Source::monopole(x, z, stf));
    else if (kind == "dipole") c.sim->add_source(Source::dipole(x, z, cp[0], cp[1], stf));
    else if (kind == "force") c.sim->add_source(Source::force(x, z, cp[0], cp[1], stf));
    else c.sim->add_source(Source::moment_tensor(x, z, cp[0], cp[1], cp[2], stf));
  }
  for (const auto& ro : receivers) {
    const auto r = ro.cast<py::dict>();
    Receiver rec;
    rec.name = r["name"].cast<std::string>();
    rec.position = {r["x"].cast<double>(), r["z"].cast<double>()};
    rec.quantities = r["quantities"].cast<std::vector<std::string>>();
    rec.medium = r["medium"].cast<std::string>();
    c.sim->add_receiver(rec);
  }
  TimeConfig t;
  t.n_steps = time["n_steps"].cast<int>();
  t.duration = time["duration"].cast<double>();
  t.dt = time["dt"].cast<double>();
  t.safety = time["safety"].cast<double>();
  t.record_every = time["record_every"].cast<int>();
  t.energy_every = time["energy_every"].cast<int>();
  c.sim->set_time(t);
  return c;
}

}  // namespace

PYBIND11_MODULE(_cudashim, m) {
  py::register_exception<Error>(m, "InsemError");
  py::class_<Case>(m, "Case")
      .def("run_cuda", &Case::run_cuda, py::arg("first"))
      .def("run_cpu", &Case::run_cpu, py::arg("first"));
  m.def("case", &make_case, py::arg("mesh"), py::arg("disc"), py::arg("materials"), py::arg("boundaries"),
        py::arg("sources"), py::arg("receivers"), py::arg("time"));
}
