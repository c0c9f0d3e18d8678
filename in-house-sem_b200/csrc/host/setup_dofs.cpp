// Global point numbering with hanging-node constraints (setup_dofs.hpp).
//
// The numbering is a function of the element order alone, and the solver's
// arrays are laid out by it, so it follows the order in which the reference
// hands out global indices (cpp/src/ops/dof_map.cpp:42-260): walking the
// elements in forest order, an element first claims a block of ngll - 2
// indices for each of its not-yet-seen conforming sides (sides 0..3), then
// numbers its points row by row, a corner vertex at its first touch and each
// interior point in turn.  Constrained points take the coarse side's
// Lagrange interpolant at their position, chained through constrained coarse
// points, and the weights are summed per global point in ascending point
// order (the same floating-point sums).  Everything else -- the element
// classification, the pending-point bookkeeping, the transpose -- is written
// for this library.
#include "setup_dofs.hpp"

#include <cmath>
#include <functional>
#include <limits>
#include <map>
#include <unordered_map>

namespace insem_setup {

std::vector<std::pair<i32, double>> PointMap::entries(std::size_t s) const {
  const i32 m = slot[s];
  if (m >= 0) return {{m, 1.0}};
  std::vector<std::pair<i32, double>> out;
  for (i32 q = row_start[-1 - m]; q < row_start[-m]; ++q) out.push_back({row_point[q], row_weight[q]});
  return out;
}

namespace {

constexpr i32 kUnset = std::numeric_limits<i32>::min();

struct HangingSide {
  i32 coarse = -1;  // element on the coarse side
  int side = -1;    // its side
};

// Slot index of point q (0..n, ascending along the cell axis) of side f.
int slot_on_side(int f, int q, int n, int ngll) {
  switch (f) {
    case 0: return q;
    case 1: return q * ngll + n;
    case 2: return n * ngll + q;
    default: return q * ngll;
  }
}

bool point_on_side(int f, int i, int j, int n) {
  return (f == 0 && j == 0) || (f == 1 && i == n) || (f == 2 && j == n) || (f == 3 && i == 0);
}

}  // namespace

PointMap number_points(const QuadForest& forest, int ngll, const std::vector<i32>& quads,
                       const std::vector<i32>& corners, i32 n_vertices, const Interpolant& gll,
                       const Interpolant& glj) {
  expect(ngll >= 2, "an element needs at least 2 GLL points per direction");
  PointMap pm;
  pm.ngll = ngll;
  pm.npe = ngll * ngll;
  pm.n_elements = static_cast<i32>(quads.size());
  const int n = ngll - 1;
  const std::size_t npe = static_cast<std::size_t>(pm.npe);
  const std::size_t n_slots = npe * quads.size();
  expect(n_slots < static_cast<std::size_t>(std::numeric_limits<i32>::max()),
         "too many element points for 32-bit indices");

  std::vector<i32> element(forest.size(), -1);
  for (std::size_t e = 0; e < quads.size(); ++e) element[quads[e]] = static_cast<i32>(e);

  // Hanging sides (on the fine side) and the vertices hanging in their middle.
  std::vector<std::array<HangingSide, 4>> hanging(quads.size());
  std::vector<char> vertex_hangs(n_vertices, 0);
  for (std::size_t e = 0; e < quads.size(); ++e) {
    for (int f = 0; f < 4; ++f) {
      const Neighbour nb = forest.neighbour(quads[e], f);
      if (nb.quad < 0) continue;
      const i32 ce = element[nb.quad];
      if (ce < 0) {
        expect(nb.jump == 0, "elements of two media meet at different refinement levels");
        continue;
      }
      if (nb.jump >= 0) continue;
      expect(nb.jump == -1, "the forest is not 2:1 balanced");
      hanging[e][f] = {ce, nb.side};
      const i32* coarse_v = &corners[4 * static_cast<std::size_t>(nb.quad)];
      const i32 c0 = coarse_v[kSideCorner[nb.side][0]], c1 = coarse_v[kSideCorner[nb.side][1]];
      for (int k = 0; k < 2; ++k) {
        const i32 v = corners[4 * static_cast<std::size_t>(quads[e]) + kSideCorner[f][k]];
        if (v != c0 && v != c1) vertex_hangs[v] = 1;
      }
    }
  }

  // Unconstrained points, first touch along the elements.
  pm.slot.assign(n_slots, kUnset);
  std::vector<i32> vertex_point(n_vertices, -1);
  struct SideBlock {
    i32 first;
    int users;
  };
  std::unordered_map<uint64_t, SideBlock> side_blocks;
  side_blocks.reserve(2 * quads.size() + 16);
  i32 next = 0;
  for (std::size_t e = 0; e < quads.size(); ++e) {
    const i32* v = &corners[4 * static_cast<std::size_t>(quads[e])];
    i32 block[4];
    bool rising[4];  // the side's counter-clockwise direction runs from its lower to its higher vertex
    for (int f = 0; f < 4; ++f) {
      const i32 p = v[kSideCorner[f][0]], q = v[kSideCorner[f][1]];
      rising[f] = p < q;
      block[f] = -1;
      if (hanging[e][f].coarse >= 0) continue;
      const uint64_t key = (static_cast<uint64_t>(std::min(p, q)) << 32) | static_cast<uint32_t>(std::max(p, q));
      auto it = side_blocks.find(key);
      if (it == side_blocks.end()) {
        it = side_blocks.emplace(key, SideBlock{next, 0}).first;
        next += n - 1;
      }
      expect(++it->second.users <= 2, "an element side is shared by more than two elements");
      block[f] = it->second.first;
    }
    i32* out = &pm.slot[e * npe];
    for (int j = 0; j <= n; ++j) {
      for (int i = 0; i <= n; ++i) {
        const bool i_end = i == 0 || i == n, j_end = j == 0 || j == n;
        i32 g = kUnset;
        if (i_end && j_end) {
          const i32 vx = v[j == 0 ? (i == 0 ? 0 : 1) : (i == n ? 2 : 3)];
          if (!vertex_hangs[vx]) {
            if (vertex_point[vx] < 0) vertex_point[vx] = next++;
            g = vertex_point[vx];
          }
        } else if (i_end || j_end) {
          // side and counter-clockwise position 1..n-1 along it
          const int f = j == 0 ? 0 : i == n ? 1 : j == n ? 2 : 3;
          const int ccw = f == 0 ? i : f == 1 ? j : f == 2 ? n - i : n - j;
          if (block[f] >= 0) g = block[f] + ((rising[f] ? ccw : n - ccw) - 1);
        } else {
          g = next++;
        }
        out[j * ngll + i] = g;
      }
    }
  }
  pm.n_global = next;

  // Constrained points: the coarse side's interpolant at the point, through
  // constrained coarse points where they chain.
  using Row = std::vector<std::pair<i32, double>>;
  auto side_basis = [&](std::size_t e, int f) -> const Interpolant& {
    return (forest.axial(quads[e]) && (f == 0 || f == 2)) ? glj : gll;
  };
  std::map<std::size_t, Row> pending_rows;
  std::function<Row(std::size_t)> row_of = [&](std::size_t s) -> Row {
    const i32 m = pm.slot[s];
    if (m >= 0) return {{m, 1.0}};
    if (m != kUnset) return pm.entries(s);
    const auto known = pending_rows.find(s);
    if (known != pending_rows.end()) return known->second;
    const std::size_t e = s / npe;
    const int k = static_cast<int>(s % npe), i = k % ngll, j = k / ngll;
    int f = 0;
    while (f < 4 && !(hanging[e][f].coarse >= 0 && point_on_side(f, i, j, n))) ++f;
    expect(f < 4, "a constrained point lies on no hanging side");
    const HangingSide h = hanging[e][f];
    const double t = side_basis(e, f).nodes()[(f == 0 || f == 2) ? i : j];
    const double tc = forest.side_coordinate(quads[e], f, t, quads[h.coarse], h.side);
    const std::vector<double> w = side_basis(h.coarse, h.side).at(tc);
    std::map<i32, double> sum;
    for (int q = 0; q <= n; ++q) {
      if (std::abs(w[q]) < 1e-14) continue;
      const std::size_t cs = static_cast<std::size_t>(h.coarse) * npe + slot_on_side(h.side, q, n, ngll);
      for (const auto& [g, wg] : row_of(cs)) sum[g] += w[q] * wg;
    }
    Row row(sum.begin(), sum.end());
    pending_rows.emplace(s, row);
    return row;
  };
  for (std::size_t s = 0; s < n_slots; ++s) {
    if (pm.slot[s] != kUnset) continue;
    const Row row = row_of(s);
    if (row.size() == 1 && std::abs(row[0].second - 1.0) < 1e-12) {
      pm.slot[s] = row[0].first;  // the point coincides with a coarse point
      continue;
    }
    pm.slot[s] = -1 - pm.n_rows();
    for (const auto& [g, w] : row) {
      pm.row_point.push_back(g);
      pm.row_weight.push_back(w);
    }
    pm.row_start.push_back(static_cast<i32>(pm.row_point.size()));
  }

  // Transpose.
  const bool weighted = pm.n_rows() > 0;
  pm.t_start.assign(static_cast<std::size_t>(pm.n_global) + 1, 0);
  for (std::size_t s = 0; s < n_slots; ++s) pm.each_entry(s, [&](i32 g, double) { ++pm.t_start[g + 1]; });
  for (i32 g = 0; g < pm.n_global; ++g) pm.t_start[g + 1] += pm.t_start[g];
  pm.t_slot.resize(pm.t_start.back());
  if (weighted) pm.t_weight.resize(pm.t_start.back());
  std::vector<i32> fill(pm.t_start.begin(), pm.t_start.end() - 1);
  for (std::size_t s = 0; s < n_slots; ++s) {
    pm.each_entry(s, [&](i32 g, double w) {
      const i32 at = fill[g]++;
      pm.t_slot[at] = static_cast<i32>(s);
      if (weighted) pm.t_weight[at] = w;
    });
  }
  pm.first_slot.assign(pm.n_global, -1);
  for (std::size_t s = 0; s < n_slots; ++s) {
    const i32 m = pm.slot[s];
    if (m >= 0 && pm.first_slot[m] < 0) pm.first_slot[m] = static_cast<i32>(s);
  }
  for (i32 g = 0; g < pm.n_global; ++g) expect(pm.first_slot[g] >= 0, "a global point has no unconstrained slot");
  return pm;
}

}  // namespace insem_setup
