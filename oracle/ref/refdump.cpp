// Test infrastructure only: a pybind11 module compiled against the reference
// sources (oracle build) that exports the arrays the reference solver builds
// for its time loop, so that the fixtures under tests/golden carry exactly
// the reference's inputs and outputs.
//
// The reference keeps its source, receiver and coupling terms private
// (cpp/include/insem/solver/solver.hpp:155-211) and offers no accessor; this
// translation unit reads them by compiling the reference headers with their
// access specifiers opened.  Member layout is unchanged by that, so the
// objects built by the reference's own `_core` module are read as they are.
//
// Exposed functions (all take the reference's `insem._core.Solver`):
//   problem(solver)                 -> dict of every per-step input array
//   block_forces(solver, d, b, u)   -> f_local of block b of domain d
//                                      (physics::*_internal_forces, kernels.hpp:32-35)
//   gather(solver, d, u_global)     -> u_local   (DofMap::gather,   dof_map.hpp:95-120)
//   assemble(solver, d, f_local)    -> f_global  (DofMap::assemble, dof_map.hpp:123-141)
//   internal_forces(solver, d, u)   -> f_global  (Solver::internal_forces, solver.cpp:570-581)
//   fields(solver, d)               -> dict u, v, a, f (the domain's current state)

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <array>
#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <optional>
#include <random>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#define private public
#define protected public
#include "insem/core/error.hpp"
#include "insem/solver/solver.hpp"
#undef private
#undef protected

namespace py = pybind11;
using namespace insem;

namespace {

template <class T>
py::array_t<T> arr(const std::vector<T>& v) {
  py::array_t<T> out(static_cast<py::ssize_t>(v.size()));
  std::copy(v.begin(), v.end(), out.mutable_data());
  return out;
}

py::array_t<std::uint8_t> arr_char(const std::vector<char>& v) {
  py::array_t<std::uint8_t> out(static_cast<py::ssize_t>(v.size()));
  for (std::size_t i = 0; i < v.size(); ++i) out.mutable_data()[i] = static_cast<std::uint8_t>(v[i]);
  return out;
}

template <class T>
std::vector<T> vec(const py::array_t<T, py::array::c_style | py::array::forcecast>& a) {
  return std::vector<T>(a.data(), a.data() + a.size());
}

py::dict stf_dict(const SourceTimeFunction& s) {
  py::dict d;
  d["kind"] = static_cast<int>(s.kind);
  d["f0"] = s.f0;
  d["t0"] = s.t0;
  d["amplitude"] = s.amplitude;
  d["samples"] = arr(s.samples);
  d["sample_dt"] = s.sample_dt;
  return d;
}

py::dict problem(solver::Solver& s) {
  py::dict out;
  out["real_bytes"] = static_cast<int>(sizeof(real_t));
  out["dt"] = s.dt_;
  out["stable_dt"] = s.stable_dt_;
  out["n_steps"] = s.n_steps_;
  out["record_every"] = s.record_every_;
  out["energy_every"] = s.energy_every_;
  out["axisym"] = s.axisym_;
  out["azimuthal_order"] = s.azimuthal_order_;
  py::dict kb;
  kb["ngll"] = s.kernel_basis_.ngll;
  kb["D"] = arr(s.kernel_basis_.D);
  kb["Dj"] = arr(s.kernel_basis_.Dj);
  kb["w2"] = arr(s.kernel_basis_.w2);
  out["basis"] = kb;

  py::list domains;
  for (const solver::Domain& d : s.domains_) {
    py::dict dd;
    dd["medium"] = static_cast<int>(d.medium);
    dd["ncomp"] = d.ncomp;
    dd["azimuthal_order"] = d.azimuthal_order;
    dd["n_global"] = d.n_global();
    dd["n_elements"] = d.dofs.n_elements();
    dd["l2g"] = arr(d.dofs.l2g_);
    dd["row_offsets"] = arr(d.dofs.row_offsets_);
    dd["row_dofs"] = arr(d.dofs.row_dofs_);
    dd["row_weights"] = arr(d.dofs.row_weights_);
    dd["t_offsets"] = arr(d.dofs.t_offsets_);
    dd["t_slots"] = arr(d.dofs.t_slots_);
    dd["t_weights"] = arr(d.dofs.t_weights_);
    dd["mass"] = arr(d.mass);
    dd["inv_mass"] = arr(d.inv_mass);
    dd["absorbing_points"] = arr(d.absorbing_points);
    dd["absorbing_coef"] = arr(d.absorbing_coef);
    dd["dirichlet_points"] = arr(d.dirichlet_points);
    dd["axis_points"] = arr(d.axis_points);
    dd["axis_components"] = arr(std::vector<std::int32_t>(d.axis_components.begin(), d.axis_components.end()));
    dd["coords"] = arr(d.coords);
    py::list blocks;
    for (const ops::ElementBlock& b : d.blocks) {
      py::dict bd;
      bd["kind"] = static_cast<int>(b.kind);
      bd["azimuthal_order"] = b.azimuthal_order;
      bd["elements"] = arr(b.elements);
      bd["metric"] = arr(b.metric);
      bd["coef0"] = arr(b.coef0);
      bd["coef1"] = arr(b.coef1);
      bd["wr"] = arr(b.wr);
      bd["hoop"] = arr(b.hoop);
      bd["r"] = arr(b.r);
      bd["axial"] = arr_char(b.axial);
      blocks.append(bd);
    }
    dd["blocks"] = blocks;
    domains.append(dd);
  }
  out["domains"] = domains;

  py::dict cp;
  cp["fluid_points"] = arr(s.coupling_.fluid_points);
  cp["solid_points"] = arr(s.coupling_.solid_points);
  cp["cx"] = arr(s.coupling_.cx);
  cp["cz"] = arr(s.coupling_.cz);
  out["coupling"] = cp;

  py::list sources;
  for (const auto& t : s.sources_) {
    py::dict sd;
    sd["domain"] = t.domain;
    sd["points"] = arr(t.points);
    sd["coef"] = arr(t.coef);
    sd["stf"] = stf_dict(t.stf);
    sources.append(sd);
  }
  out["sources"] = sources;

  py::list receivers;
  for (const auto& r : s.receivers_) {
    py::dict rd;
    rd["name"] = r.name;
    rd["domain"] = r.domain;
    rd["points"] = arr(r.points);
    rd["value"] = arr(r.value);
    rd["d_dx"] = arr(r.d_dx);
    rd["d_dz"] = arr(r.d_dz);
    rd["rho"] = r.rho;
    rd["quantities"] = r.quantities;
    std::vector<std::int64_t> ti(r.trace_index.begin(), r.trace_index.end());
    rd["trace_index"] = arr(ti);
    receivers.append(rd);
  }
  out["receivers"] = receivers;
  return out;
}

using RArray = py::array_t<real_t, py::array::c_style | py::array::forcecast>;

py::array_t<real_t> block_forces(solver::Solver& s, int di, int bi, const RArray& u_local) {
  const solver::Domain& d = s.domains_.at(static_cast<std::size_t>(di));
  const ops::ElementBlock& b = d.blocks.at(static_cast<std::size_t>(bi));
  const std::size_t n = static_cast<std::size_t>(d.ncomp) * d.dofs.n_elements() * d.dofs.points_per_element();
  INSEM_CHECK(static_cast<std::size_t>(u_local.size()) == n, "u_local has the wrong size");
  std::vector<real_t> f(n, real_t(0));
  if (d.medium == Medium::Elastic) {
    physics::elastic_internal_forces(s.kernel_basis_, b, u_local.data(), f.data());
  } else {
    physics::acoustic_internal_forces(s.kernel_basis_, b, u_local.data(), f.data());
  }
  return arr(f);
}

py::array_t<real_t> gather(solver::Solver& s, int di, const RArray& g) {
  const solver::Domain& d = s.domains_.at(static_cast<std::size_t>(di));
  INSEM_CHECK(static_cast<std::size_t>(g.size()) == static_cast<std::size_t>(d.ncomp) * d.n_global(),
              "global field has the wrong size");
  std::vector<real_t> l(static_cast<std::size_t>(d.ncomp) * d.dofs.n_elements() * d.dofs.points_per_element());
  d.dofs.gather(g.data(), l.data(), d.ncomp);
  return arr(l);
}

py::array_t<real_t> assemble(solver::Solver& s, int di, const RArray& l) {
  const solver::Domain& d = s.domains_.at(static_cast<std::size_t>(di));
  INSEM_CHECK(static_cast<std::size_t>(l.size()) ==
                  static_cast<std::size_t>(d.ncomp) * d.dofs.n_elements() * d.dofs.points_per_element(),
              "local field has the wrong size");
  std::vector<real_t> g(static_cast<std::size_t>(d.ncomp) * d.n_global());
  d.dofs.assemble(l.data(), g.data(), d.ncomp);
  return arr(g);
}

py::array_t<real_t> internal_forces(solver::Solver& s, int di, const RArray& u) {
  solver::Domain& d = s.domains_.at(static_cast<std::size_t>(di));
  INSEM_CHECK(static_cast<std::size_t>(u.size()) == d.u.size(), "field has the wrong size");
  std::vector<real_t> x(u.data(), u.data() + u.size());
  const std::vector<real_t> saved = d.f;
  s.internal_forces(d, x, false);
  std::vector<real_t> f = d.f;
  d.f = saved;
  return arr(f);
}

py::dict fields(solver::Solver& s, int di) {
  const solver::Domain& d = s.domains_.at(static_cast<std::size_t>(di));
  py::dict out;
  out["u"] = arr(d.u);
  out["v"] = arr(d.v);
  out["a"] = arr(d.a);
  out["f"] = arr(d.f);
  return out;
}

}  // namespace

PYBIND11_MODULE(_refdump, m) {
  m.doc() = "Oracle-only access to the reference solver's per-step arrays (test infrastructure).";
  m.def("problem", &problem, py::arg("solver"));
  m.def("block_forces", &block_forces, py::arg("solver"), py::arg("domain"), py::arg("block"), py::arg("u_local"));
  m.def("gather", &gather, py::arg("solver"), py::arg("domain"), py::arg("u_global"));
  m.def("assemble", &assemble, py::arg("solver"), py::arg("domain"), py::arg("f_local"));
  m.def("internal_forces", &internal_forces, py::arg("solver"), py::arg("domain"), py::arg("u"));
  m.def("fields", &fields, py::arg("solver"), py::arg("domain"));
}
