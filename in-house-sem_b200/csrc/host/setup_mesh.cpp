// Macro mesh, linear quadtree forest and element geometry (setup_mesh.hpp).
//
// Arithmetic that reaches the packed arrays -- the isoparametric map and its
// Jacobian, quadrant boxes, the chain rule to element coordinates, the side
// coordinates of hanging points -- is evaluated with the same operations, in
// the same order, as the reference (cpp/src/mesh/macro_mesh.cpp:175-230,
// cpp/src/mesh/forest.cpp:167-189 and 243-248, cpp/src/geometry/geometry.cpp:
// 24-109), so that the doubles, and the floats rounded from them, agree bit
// for bit.  The data structures and the search are this library's own.
#include "setup_mesh.hpp"

#include <algorithm>
#include <cmath>
#include <unordered_map>

namespace insem_setup {

// ============================================================ macro mesh
namespace {

// Quad9 node k sits at lattice position (kNineA[k], kNineB[k]) in {0, 1, 2}^2.
constexpr int kNineA[9] = {0, 2, 2, 0, 1, 2, 1, 0, 1};
constexpr int kNineB[9] = {0, 0, 2, 2, 0, 1, 2, 1, 1};
constexpr double kFourXi[4] = {-1.0, 1.0, 1.0, -1.0};
constexpr double kFourEta[4] = {-1.0, -1.0, 1.0, 1.0};

struct Shape {
  int n = 0;
  double v[9], dxi[9], deta[9];
};

void quadratic_1d(double t, double* l, double* dl) {
  l[0] = 0.5 * t * (t - 1.0);
  l[1] = 1.0 - t * t;
  l[2] = 0.5 * t * (t + 1.0);
  dl[0] = t - 0.5;
  dl[1] = -2.0 * t;
  dl[2] = t + 0.5;
}

Shape shape_at(bool quad9, double xi, double eta) {
  Shape s;
  if (!quad9) {
    s.n = 4;
    for (int k = 0; k < 4; ++k) {
      const double fx = 1.0 + kFourXi[k] * xi;
      const double fy = 1.0 + kFourEta[k] * eta;
      s.v[k] = 0.25 * fx * fy;
      s.dxi[k] = 0.25 * kFourXi[k] * fy;
      s.deta[k] = 0.25 * fx * kFourEta[k];
    }
    return s;
  }
  double lx[3], dlx[3], ly[3], dly[3];
  quadratic_1d(xi, lx, dlx);
  quadratic_1d(eta, ly, dly);
  s.n = 9;
  for (int k = 0; k < 9; ++k) {
    s.v[k] = lx[kNineA[k]] * ly[kNineB[k]];
    s.dxi[k] = dlx[kNineA[k]] * ly[kNineB[k]];
    s.deta[k] = lx[kNineA[k]] * dly[kNineB[k]];
  }
  return s;
}

}  // namespace

MacroGrid::MacroGrid(bool quad9, bool axisym, std::vector<double> xy, std::vector<i32> conn, std::vector<i32> region,
                     std::vector<TaggedSide> tagged)
    : quad9_(quad9), axisym_(axisym), xy_(std::move(xy)), conn_(std::move(conn)), region_(std::move(region)),
      tagged_(std::move(tagged)) {
  expect(!region_.empty() && !xy_.empty(), "the macro mesh has no cells or no nodes");
  expect(conn_.size() == region_.size() * static_cast<std::size_t>(nodes_per_cell()),
         "cell connectivity does not match the number of cells");
  const i32 nn = static_cast<i32>(xy_.size() / 2);
  for (i32 v : conn_) expect(v >= 0 && v < nn,
                             [&] { return "a cell names node " + std::to_string(v) + " of " + std::to_string(nn); });
  axis_mask_.assign(region_.size(), 0);
  if (axisym_) turn_axis_sides_to_three();
  connect();
  check();
}

bool MacroGrid::side_touches_axis(i32 c, int f) const {
  if (!axisym_) return false;
  double extent = 0.0;
  for (int k = 0; k < 4; ++k) extent = std::max(extent, std::abs(xy_[2 * node_of(c, k) + 1]));
  for (int k = 0; k < 4; ++k) extent = std::max(extent, std::abs(xy_[2 * node_of(c, k)]));
  const double tol = 1e-10 * std::max(extent, 1e-300);
  return std::abs(xy_[2 * node_of(c, kSideCorner[f][0])]) <= tol &&
         std::abs(xy_[2 * node_of(c, kSideCorner[f][1])]) <= tol;
}

void MacroGrid::turn_axis_sides_to_three() {
  const int npc = nodes_per_cell();
  std::vector<std::vector<std::size_t>> tags_of(region_.size());
  for (std::size_t t = 0; t < tagged_.size(); ++t)
    if (tagged_[t].cell >= 0 && tagged_[t].cell < n_cells()) tags_of[tagged_[t].cell].push_back(t);
  for (i32 c = 0; c < n_cells(); ++c) {
    int on = -1;
    for (int f = 0; f < 4; ++f) {
      if (!side_touches_axis(c, f)) continue;
      expect(on < 0, [&] { return "macro cell " + std::to_string(c) + " touches the symmetry axis with two sides"; });
      on = f;
    }
    if (on < 0 || on == 3) continue;
    const int turn = (on + 1) % 4;  // new corner k = old corner (k + turn) mod 4
    i32* nodes = &conn_[static_cast<std::size_t>(c) * npc];
    const std::vector<i32> was(nodes, nodes + npc);
    for (int k = 0; k < 4; ++k) {
      nodes[k] = was[(k + turn) % 4];
      if (npc == 9) nodes[4 + k] = was[4 + (k + turn) % 4];
    }
    for (std::size_t t : tags_of[c]) tagged_[t].side = (tagged_[t].side - turn + 4) % 4;
  }
  for (i32 c = 0; c < n_cells(); ++c)
    for (int f = 0; f < 4; ++f)
      if (side_touches_axis(c, f)) axis_mask_[c] |= static_cast<uint8_t>(1u << f);
}

void MacroGrid::connect() {
  side_edge_.assign(4 * region_.size(), -1);
  side_sense_.assign(4 * region_.size(), 0);
  std::unordered_map<uint64_t, i32> by_nodes;
  by_nodes.reserve(4 * region_.size());
  for (i32 c = 0; c < n_cells(); ++c) {
    for (int f = 0; f < 4; ++f) {
      const i32 p = node_of(c, kSideCorner[f][0]), q = node_of(c, kSideCorner[f][1]);
      expect(p != q, [&] { return "macro cell " + std::to_string(c) + " has a side of zero length"; });
      const uint64_t key = (static_cast<uint64_t>(std::min(p, q)) << 32) | static_cast<uint32_t>(std::max(p, q));
      const auto found = by_nodes.find(key);
      i32 e;
      if (found == by_nodes.end()) {
        e = static_cast<i32>(edge_cells_.size());
        by_nodes.emplace(key, e);
        edge_cells_.push_back({c, -1});
      } else {
        e = found->second;
        auto& pair = edge_cells_[e];
        expect(pair[1] < 0, "a macro edge is shared by more than two cells");
        // two counter-clockwise cells run along a shared edge in opposite senses
        const i32 first = pair[0];
        expect((p < q) != same_sense(first, side_on(first, e)),
               [&] {
                 return "macro cells " + std::to_string(first) + " and " + std::to_string(c) +
                        " are oriented inconsistently";
               });
        pair[1] = c;
      }
      side_edge_[4 * c + f] = e;
      side_sense_[4 * c + f] = p < q ? 1 : 0;
    }
  }
}

void MacroGrid::check() const {
  for (i32 c = 0; c < n_cells(); ++c) {
    for (double xi : {-1.0, 0.0, 1.0}) {
      for (double eta : {-1.0, 0.0, 1.0}) {
        const auto j = jacobian(c, xi, eta);
        expect(j[0] * j[3] - j[1] * j[2] > 0.0,
               [&] {
                 return "macro cell " + std::to_string(c) +
                        " is inverted or degenerate (cells run counter-clockwise)";
               });
      }
    }
  }
  if (axisym_) {
    double extent = 0.0;
    for (double v : xy_) extent = std::max(extent, std::abs(v));
    for (std::size_t i = 0; i < xy_.size(); i += 2)
      expect(xy_[i] >= -1e-12 * extent, "an axisymmetric mesh has a node at negative radius");
  }
  for (const TaggedSide& t : tagged_) {
    expect(t.cell >= 0 && t.cell < n_cells() && t.side >= 0 && t.side < 4, "a boundary tag names a missing cell side");
    expect(exterior(t.cell, t.side),
           [&] { return "a tagged side of cell " + std::to_string(t.cell) + " is interior"; });
  }
}

i32 MacroGrid::across(i32 c, int f) const {
  const auto& pair = edge_cells_[edge(c, f)];
  return pair[0] == c ? pair[1] : pair[0];
}

int MacroGrid::side_on(i32 c, i32 e) const {
  for (int f = 0; f < 4; ++f)
    if (side_edge_[4 * c + f] == e) return f;
  return -1;
}

std::array<double, 2> MacroGrid::point(i32 c, double xi, double eta) const {
  const Shape s = shape_at(quad9_, xi, eta);
  std::array<double, 2> x{0.0, 0.0};
  for (int k = 0; k < s.n; ++k) {
    const double* node = &xy_[2 * node_of(c, k)];
    x[0] += s.v[k] * node[0];
    x[1] += s.v[k] * node[1];
  }
  return x;
}

std::array<double, 4> MacroGrid::jacobian(i32 c, double xi, double eta) const {
  const Shape s = shape_at(quad9_, xi, eta);
  std::array<double, 4> j{0.0, 0.0, 0.0, 0.0};
  for (int k = 0; k < s.n; ++k) {
    const double* node = &xy_[2 * node_of(c, k)];
    j[0] += s.dxi[k] * node[0];
    j[1] += s.deta[k] * node[0];
    j[2] += s.dxi[k] * node[1];
    j[3] += s.deta[k] * node[1];
  }
  return j;
}

void MacroGrid::point_and_jacobian(i32 c, double xi, double eta, std::array<double, 2>& x,
                                   std::array<double, 4>& j) const {
  const Shape s = shape_at(quad9_, xi, eta);
  x = {0.0, 0.0};
  j = {0.0, 0.0, 0.0, 0.0};
  for (int k = 0; k < s.n; ++k) {
    const double* node = &xy_[2 * node_of(c, k)];
    x[0] += s.v[k] * node[0];
    x[1] += s.v[k] * node[1];
    j[0] += s.dxi[k] * node[0];
    j[1] += s.deta[k] * node[0];
    j[2] += s.dxi[k] * node[1];
    j[3] += s.deta[k] * node[1];
  }
}

// ================================================================= forest
namespace {

uint64_t spread_bits(uint64_t v) {  // bit k of v -> bit 2k
  v &= 0xffffffffULL;
  v = (v | (v << 16)) & 0x0000ffff0000ffffULL;
  v = (v | (v << 8)) & 0x00ff00ff00ff00ffULL;
  v = (v | (v << 4)) & 0x0f0f0f0f0f0f0f0fULL;
  v = (v | (v << 2)) & 0x3333333333333333ULL;
  v = (v | (v << 1)) & 0x5555555555555555ULL;
  return v;
}

// Morton key with i in the even bits: the order of a quadrant's children is
// (i, j) = (0,0), (1,0), (0,1), (1,1).
uint64_t morton(uint64_t i, uint64_t j) { return spread_bits(i) | (spread_bits(j) << 1); }

constexpr int64_t kHalfLattice = int64_t{1} << (kDeepest + 1);

// Counter-clockwise position along side f of a cell of half-lattice point (a, b).
int64_t along_side(int f, int64_t a, int64_t b) {
  switch (f) {
    case 0: return a;
    case 1: return b;
    case 2: return kHalfLattice - a;
    default: return kHalfLattice - b;
  }
}

// The half-lattice point just inside side f of a cell at counter-clockwise position t.
std::array<int64_t, 2> inside_side(int f, int64_t t) {
  switch (f) {
    case 0: return {t, 0};
    case 1: return {kHalfLattice - 1, t};
    case 2: return {kHalfLattice - t, kHalfLattice - 1};
    default: return {0, kHalfLattice - t};
  }
}

}  // namespace

QuadForest::QuadForest(const MacroGrid* grid, int level) : grid_(grid) {
  expect(level >= 0 && level <= kDeepest,
         [&] { return "uniform refinement level must be in 0.." + std::to_string(kDeepest); });
  const uint64_t per_cell = uint64_t{1} << (2 * level);
  expect(per_cell * static_cast<uint64_t>(grid->n_cells()) < (uint64_t{1} << 31),
         [&] { return "uniform refinement to level " + std::to_string(level) + " makes too many elements"; });
  const i32 side = i32{1} << level;
  quads_.reserve(per_cell * grid->n_cells());
  std::vector<std::pair<uint64_t, Quadrant>> cell_quads(per_cell);
  for (i32 c = 0; c < grid->n_cells(); ++c) {
    std::size_t n = 0;
    for (i32 j = 0; j < side; ++j)
      for (i32 i = 0; i < side; ++i) cell_quads[n++] = {morton(i, j), Quadrant{c, level, i, j}};
    std::sort(cell_quads.begin(), cell_quads.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    for (const auto& e : cell_quads) quads_.push_back(e.second);
  }
  index();
}

QuadForest::QuadForest(const MacroGrid* grid, std::vector<Quadrant> quads) : grid_(grid), quads_(std::move(quads)) {
  index();
}

void QuadForest::index() {
  first_.assign(static_cast<std::size_t>(grid_->n_cells()) + 1, 0);
  key_.resize(quads_.size());
  for (std::size_t q = 0; q < quads_.size(); ++q) {
    const Quadrant& d = quads_[q];
    const int shift = kDeepest - d.level;
    key_[q] = morton(static_cast<uint64_t>(d.i) << shift, static_cast<uint64_t>(d.j) << shift);
    ++first_[d.cell + 1];
  }
  for (i32 c = 0; c < grid_->n_cells(); ++c) first_[c + 1] += first_[c];
}

std::array<double, 4> QuadForest::box(i32 q) const {
  const Quadrant& d = quads_[q];
  const double h = 2.0 / static_cast<double>(int64_t{1} << d.level);
  return {-1.0 + d.i * h, -1.0 + (d.i + 1) * h, -1.0 + d.j * h, -1.0 + (d.j + 1) * h};
}

i32 QuadForest::locate(i32 cell, int64_t a, int64_t b) const {
  if (a < 0 || b < 0 || a >= kHalfLattice || b >= kHalfLattice) return -1;
  const uint64_t p = morton(static_cast<uint64_t>(a >> 1), static_cast<uint64_t>(b >> 1));
  const auto lo = key_.begin() + first_[cell], hi = key_.begin() + first_[cell + 1];
  auto it = std::upper_bound(lo, hi, p);
  if (it == lo) return -1;
  const i32 q = static_cast<i32>((it - key_.begin()) - 1);
  const Quadrant& d = quads_[q];
  const int shift = kDeepest + 1 - d.level;
  if ((a >> shift) != d.i || (b >> shift) != d.j) return -1;
  return q;
}

Neighbour QuadForest::neighbour(i32 q, int f) const {
  const Quadrant& d = quads_[q];
  const int64_t s = int64_t{1} << (kDeepest + 1 - d.level);
  const int64_t a0 = d.i * s, b0 = d.j * s;
  // probe the point just outside the side's midpoint
  int64_t a = a0 + s / 2, b = b0 + s / 2;
  switch (f) {
    case 0: b = b0 - 1; break;
    case 1: a = a0 + s; break;
    case 2: b = b0 + s; break;
    default: a = a0 - 1; break;
  }
  Neighbour nb;
  i32 cell = d.cell;
  int side = (f + 2) % 4;
  if (a < 0 || b < 0 || a >= kHalfLattice || b >= kHalfLattice) {
    const i32 other = grid_->across(d.cell, f);
    if (other < 0) return nb;
    const int of = grid_->side_on(other, grid_->edge(d.cell, f));
    // position along the shared edge from its lower node, then along the other side
    const int64_t t = along_side(f, a, b);
    const int64_t from_low = grid_->same_sense(d.cell, f) ? t : kHalfLattice - t;
    const int64_t t2 = grid_->same_sense(other, of) ? from_low : kHalfLattice - from_low;
    const auto p = inside_side(of, t2);
    a = p[0];
    b = p[1];
    cell = other;
    side = of;
  }
  nb.quad = locate(cell, a, b);
  expect(nb.quad >= 0, "the forest does not cover the point across a side");
  nb.side = side;
  nb.jump = quads_[nb.quad].level - d.level;
  return nb;
}

double QuadForest::side_coordinate(i32 from, int f, double t, i32 to, int g) const {
  // extent [u0, u1] of a quadrant along the cell axis its side runs on
  auto extent = [this](i32 q, int side) {
    const Quadrant& d = quads_[q];
    const double n = static_cast<double>(int64_t{1} << d.level);
    const int64_t k = (side == 0 || side == 2) ? d.i : d.j;
    return std::array<double, 2>{k / n, (k + 1) / n};
  };
  auto flip = [](double v, bool yes) { return yes ? 1.0 - v : v; };
  const auto e = extent(from, f);
  double u = e[0] + 0.5 * (t + 1.0) * (e[1] - e[0]);
  const i32 ca = quads_[from].cell, cb = quads_[to].cell;
  if (ca != cb) {
    // cell axis -> counter-clockwise -> from the edge's lower node -> the other cell's axis
    u = flip(u, f >= 2);
    u = flip(u, !grid_->same_sense(ca, f));
    u = flip(u, !grid_->same_sense(cb, g));
    u = flip(u, g >= 2);
  }
  const auto e2 = extent(to, g);
  return -1.0 + 2.0 * (u - e2[0]) / (e2[1] - e2[0]);
}

QuadForest QuadForest::split(const std::vector<char>& flag) const {
  expect(flag.size() == quads_.size(), "split flags do not match the forest");
  std::vector<Quadrant> out;
  out.reserve(quads_.size() + 3 * static_cast<std::size_t>(std::count(flag.begin(), flag.end(), 1)));
  for (std::size_t q = 0; q < quads_.size(); ++q) {
    const Quadrant& d = quads_[q];
    if (!flag[q]) {
      out.push_back(d);
      continue;
    }
    expect(d.level < kDeepest, [&] { return "refinement beyond level " + std::to_string(kDeepest); });
    for (int c = 0; c < 4; ++c) out.push_back({d.cell, d.level + 1, 2 * d.i + (c & 1), 2 * d.j + (c >> 1)});
  }
  return QuadForest(grid_, std::move(out));
}

std::vector<i32> QuadForest::corner_vertices(i32* n_vertices) const {
  // A lattice point's identity independent of the cell it is seen from: a
  // macro node, a macro edge and the distance from its lower node, or a cell
  // and a position inside it.
  constexpr int64_t S = int64_t{1} << kDeepest;
  struct Key {
    uint64_t hi, lo;
    bool operator==(const Key& o) const { return hi == o.hi && lo == o.lo; }
  };
  struct KeyHash {
    std::size_t operator()(const Key& k) const {
      return static_cast<std::size_t>((k.hi * 0x9e3779b97f4a7c15ULL) ^ (k.lo + (k.hi << 7) + 0x7f4a7c15ULL));
    }
  };
  auto identity = [&](i32 cell, int64_t a, int64_t b) -> Key {
    const bool w = a == 0, e = a == S, s = b == 0, n = b == S;
    if ((w || e) && (s || n)) {
      const int corner = s ? (w ? 0 : 1) : (e ? 2 : 3);
      return {0, static_cast<uint64_t>(grid_->node_of(cell, corner))};
    }
    if (w || e || s || n) {
      const int f = s ? 0 : e ? 1 : n ? 2 : 3;
      const int64_t t = f == 0 ? a : f == 1 ? b : f == 2 ? S - a : S - b;
      const int64_t from_low = grid_->same_sense(cell, f) ? t : S - t;
      return {(uint64_t{1} << 62) | static_cast<uint64_t>(grid_->edge(cell, f)), static_cast<uint64_t>(from_low)};
    }
    return {(uint64_t{2} << 62) | static_cast<uint64_t>(cell),
            (static_cast<uint64_t>(a) << 32) | static_cast<uint64_t>(b)};
  };
  constexpr int kDi[4] = {0, 1, 1, 0};
  constexpr int kDj[4] = {0, 0, 1, 1};
  std::vector<i32> out(4 * quads_.size());
  std::unordered_map<Key, i32, KeyHash> ids;
  ids.reserve(2 * quads_.size() + 16);
  for (std::size_t q = 0; q < quads_.size(); ++q) {
    const Quadrant& d = quads_[q];
    const int64_t step = int64_t{1} << (kDeepest - d.level);
    for (int k = 0; k < 4; ++k) {
      const Key key = identity(d.cell, (d.i + kDi[k]) * step, (d.j + kDj[k]) * step);
      const auto ins = ids.emplace(key, static_cast<i32>(ids.size()));
      out[4 * q + k] = ins.first->second;
    }
  }
  *n_vertices = static_cast<i32>(ids.size());
  return out;
}

// =============================================================== geometry
std::array<double, 2> quad_point(const QuadForest& f, i32 q, double xi, double eta) {
  const auto b = f.box(q);
  return f.grid().point(f[q].cell, b[0] + (xi + 1.0) * 0.5 * (b[1] - b[0]), b[2] + (eta + 1.0) * 0.5 * (b[3] - b[2]));
}

std::array<double, 4> quad_jacobian(const QuadForest& f, i32 q, double xi, double eta) {
  const auto b = f.box(q);
  const double hx = 0.5 * (b[1] - b[0]);
  const double hy = 0.5 * (b[3] - b[2]);
  const auto m = f.grid().jacobian(f[q].cell, b[0] + (xi + 1.0) * hx, b[2] + (eta + 1.0) * hy);
  return {m[0] * hx, m[1] * hy, m[2] * hx, m[3] * hy};
}

PointGeometry element_geometry(const QuadForest& f, const std::vector<double>& ref,
                               const std::vector<double>& ref_axial) {
  PointGeometry g;
  const int n = static_cast<int>(ref.size());
  g.ngll = n;
  const std::size_t npe = static_cast<std::size_t>(n) * n;
  const std::size_t total = npe * f.size();
  for (auto* v : {&g.x, &g.z, &g.xi_x, &g.xi_z, &g.eta_x, &g.eta_z, &g.jac}) v->resize(total);
  g.shape.resize(f.size());
  constexpr double kRel = 1e-10;  // a Jacobian varying less than this (relative) is constant
  for (i32 e = 0; e < f.size(); ++e) {
    const i32 cell = f[e].cell;
    const std::vector<double>& rx = f.axial(e) ? ref_axial : ref;
    const auto b = f.box(e);
    const double hx = 0.5 * (b[1] - b[0]);
    const double hy = 0.5 * (b[3] - b[2]);
    double scale = 0.0, spread = 0.0, skew = 0.0;
    std::array<double, 4> first{};
    std::size_t p = static_cast<std::size_t>(e) * npe;
    for (int jq = 0; jq < n; ++jq) {
      for (int iq = 0; iq < n; ++iq, ++p) {
        const double xi = b[0] + (rx[iq] + 1.0) * hx;
        const double eta = b[2] + (ref[jq] + 1.0) * hy;
        std::array<double, 2> pos;
        std::array<double, 4> m;
        f.grid().point_and_jacobian(cell, xi, eta, pos, m);
        const std::array<double, 4> jm{m[0] * hx, m[1] * hy, m[2] * hx, m[3] * hy};
        const double det = jm[0] * jm[3] - jm[1] * jm[2];
        expect(det > 0.0, "an element maps with a non-positive Jacobian");
        g.x[p] = pos[0];
        g.z[p] = pos[1];
        g.jac[p] = det;
        g.xi_x[p] = jm[3] / det;
        g.xi_z[p] = -jm[1] / det;
        g.eta_x[p] = -jm[2] / det;
        g.eta_z[p] = jm[0] / det;
        if (iq == 0 && jq == 0) first = jm;
        for (int k = 0; k < 4; ++k) {
          scale = std::max(scale, std::abs(jm[k]));
          spread = std::max(spread, std::abs(jm[k] - first[k]));
        }
        skew = std::max({skew, std::abs(jm[1]), std::abs(jm[2])});
      }
    }
    g.shape[e] = spread > kRel * scale ? kCurved : skew > kRel * scale ? kAffine : kRect;
  }
  return g;
}

}  // namespace insem_setup
