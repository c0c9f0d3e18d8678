// Global point numbering of a set of elements, with hanging-node constraints
// (the packed arrays of the DofMap seam, cpp/include/insem/ops/dof_map.hpp).
#pragma once

#include <utility>
#include <vector>

#include "setup_basis.hpp"
#include "setup_mesh.hpp"

namespace insem_setup {

struct PointMap {
  int ngll = 0, npe = 0;
  i32 n_elements = 0, n_global = 0;
  // per element slot (e * npe + j * ngll + i): global point, or -1 - r for a
  // slot constrained by row r
  std::vector<i32> slot;
  std::vector<i32> row_start{0};
  std::vector<i32> row_point;
  std::vector<double> row_weight;
  // transpose, CSR: contributions to global point g, ascending slots
  std::vector<i32> t_start, t_slot;
  std::vector<double> t_weight;  // empty without constraints (all weights 1)
  std::vector<i32> first_slot;   // an unconstrained slot of each global point

  i32 n_rows() const { return static_cast<i32>(row_start.size()) - 1; }
  // (global point, weight) pairs that make up slot s
  std::vector<std::pair<i32, double>> entries(std::size_t s) const;
  template <class Visit>
  void each_entry(std::size_t s, Visit visit) const {
    const i32 m = slot[s];
    if (m >= 0) {
      visit(m, 1.0);
      return;
    }
    for (i32 q = row_start[-1 - m]; q < row_start[-m]; ++q) visit(row_point[q], row_weight[q]);
  }
};

// Numbers the GLL points of `quads` (elements in that order) of a 2:1
// balanced forest: global points in first-touch order along the elements,
// fine points on hanging sides constrained to the coarse side's polynomial.
// `corners` is QuadForest::corner_vertices.  Sides between an element of the
// set and one outside it must be conforming.
PointMap number_points(const QuadForest& forest, int ngll, const std::vector<i32>& quads,
                       const std::vector<i32>& corners, i32 n_vertices, const Interpolant& gll,
                       const Interpolant& glj);

}  // namespace insem_setup
