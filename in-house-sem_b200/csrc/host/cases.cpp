// Native case setup: model description -> packed per-step arrays.
//
// Restates the reference's setup path in one translation unit:
//   quadrature / Lagrange basis ..... cpp/src/basis/quadrature.cpp, lagrange.cpp
//   macro mesh topology, axis faces . cpp/src/mesh/macro_mesh.cpp:72-230
//   quadtree forest, 2:1 balance .... cpp/src/mesh/forest.cpp
//   adaptive refinement ............. cpp/src/sim/simulation.cpp:121-175
//   geometry ........................ cpp/src/geometry/geometry.cpp:44-109
//   DofMap numbering + constraints .. cpp/src/ops/dof_map.cpp:42-260
//   element blocks .................. cpp/src/ops/element_block.cpp
//   point location .................. cpp/src/solver/locate.cpp
//   domains, boundaries, coupling,
//   sources, receivers .............. cpp/src/solver/solver.cpp:147-568
// Deterministic: every ordered container the reference uses for numbering
// (std::map over global points, first-touch numbering in leaf order) is kept,
// so the arrays equal the reference's for the same description.
#include "insem_cases.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

using idx = int32_t;
constexpr double kPi = 3.14159265358979323846;
constexpr double kSqrtHalf = 0.70710678118654752440;
constexpr int kFaceCorners[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
constexpr int kMaxLevel = 20;

struct Fail : std::runtime_error {
  using std::runtime_error::runtime_error;
};
#define REQUIRE(cond, msg)                      \
  do {                                          \
    if (!(cond)) throw Fail(std::string(msg));  \
  } while (0)

thread_local std::string g_error;

// ------------------------------------------------------------- quadrature
double jacobi(int n, double a, double b, double x) {
  if (n == 0) return 1.0;
  double p_prev = 1.0;
  double p = 0.5 * ((a + b + 2.0) * x + (a - b));
  for (int k = 1; k < n; ++k) {
    const double c = 2.0 * k + a + b;
    const double a1 = 2.0 * (k + 1) * (k + a + b + 1) * c;
    const double a2 = (c + 1) * (a * a - b * b);
    const double a3 = (c + 1) * (c + 2) * c;
    const double a4 = 2.0 * (k + a) * (k + b) * (c + 2);
    const double p_next = ((a2 + a3 * x) * p - a4 * p_prev) / a1;
    p_prev = p;
    p = p_next;
  }
  return p;
}

double jacobi_derivative(int n, double a, double b, double x) {
  return n == 0 ? 0.0 : 0.5 * (n + a + b + 1) * jacobi(n - 1, a + 1, b + 1, x);
}

// Roots by Newton with deflation from Chebyshev-like starting points.
std::vector<double> jacobi_roots(int n, double a, double b) {
  std::vector<double> roots(n);
  for (int k = 0; k < n; ++k) {
    double r = -std::cos((2.0 * k + 1.0) * kPi / (2.0 * n));
    if (k > 0) r = 0.5 * (r + roots[k - 1]);
    for (int it = 0; it < 200; ++it) {
      double deflation = 0.0;
      for (int i = 0; i < k; ++i) deflation += 1.0 / (r - roots[i]);
      const double p = jacobi(n, a, b, r);
      const double delta = -p / (jacobi_derivative(n, a, b, r) - deflation * p);
      r += delta;
      if (std::abs(delta) < 1e-16) break;
    }
    roots[k] = r;
  }
  return roots;
}

struct Rule {
  std::vector<double> points, weights;
};

Rule gauss_legendre(int n) {
  Rule r;
  r.points = jacobi_roots(n, 0.0, 0.0);
  r.weights.resize(n);
  for (int i = 0; i < n; ++i) {
    const double x = r.points[i];
    const double dp = jacobi_derivative(n, 0.0, 0.0, x);
    r.weights[i] = 2.0 / ((1.0 - x * x) * dp * dp);
  }
  return r;
}

// Dense solve with partial pivoting (moment system of the Lobatto weights).
std::vector<double> solve_dense(std::vector<double> a, std::vector<double> b, int n) {
  for (int col = 0; col < n; ++col) {
    int pivot = col;
    for (int row = col + 1; row < n; ++row)
      if (std::abs(a[row * n + col]) > std::abs(a[pivot * n + col])) pivot = row;
    REQUIRE(a[pivot * n + col] != 0.0, "singular quadrature moment system");
    if (pivot != col) {
      for (int k = 0; k < n; ++k) std::swap(a[col * n + k], a[pivot * n + k]);
      std::swap(b[col], b[pivot]);
    }
    for (int row = col + 1; row < n; ++row) {
      const double f = a[row * n + col] / a[col * n + col];
      for (int k = col; k < n; ++k) a[row * n + k] -= f * a[col * n + k];
      b[row] -= f * b[col];
    }
  }
  std::vector<double> x(n);
  for (int row = n - 1; row >= 0; --row) {
    double s = b[row];
    for (int k = row + 1; k < n; ++k) s -= a[row * n + k] * x[k];
    x[row] = s / a[row * n + row];
  }
  return x;
}

// Gauss-Lobatto-Jacobi rule with weight (1-x)^alpha (1+x)^beta.
Rule gauss_lobatto_jacobi(int n, int alpha, int beta) {
  Rule r;
  r.points.push_back(-1.0);
  for (double x : jacobi_roots(n - 2, alpha + 1.0, beta + 1.0)) r.points.push_back(x);
  r.points.push_back(1.0);
  const Rule exact = gauss_legendre(n + alpha + beta + 2);
  std::vector<double> moments(n, 0.0);
  for (std::size_t q = 0; q < exact.points.size(); ++q) {
    const double x = exact.points[q];
    const double w = exact.weights[q] * std::pow(1.0 - x, static_cast<double>(alpha)) *
                     std::pow(1.0 + x, static_cast<double>(beta));
    for (int k = 0; k < n; ++k) moments[k] += w * jacobi(k, 0.0, 0.0, x);
  }
  std::vector<double> v(static_cast<std::size_t>(n) * n);
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j) v[k * n + j] = jacobi(k, 0.0, 0.0, r.points[j]);
  r.weights = solve_dense(std::move(v), std::move(moments), n);
  return r;
}

Rule gll(int n) { return gauss_lobatto_jacobi(n, 0, 0); }
Rule glj01(int n) { return gauss_lobatto_jacobi(n, 0, 1); }

// -------------------------------------------------------- Lagrange basis
struct Lagrange {
  std::vector<double> nodes, bary;
  explicit Lagrange(std::vector<double> x) : nodes(std::move(x)) {
    const int n = static_cast<int>(nodes.size());
    bary.assign(n, 1.0);
    for (int j = 0; j < n; ++j)
      for (int k = 0; k < n; ++k)
        if (k != j) bary[j] /= nodes[j] - nodes[k];
  }
  int size() const { return static_cast<int>(nodes.size()); }
  int node_index(double x) const {
    for (int j = 0; j < size(); ++j)
      if (std::abs(x - nodes[j]) <= 1e-14 * (1.0 + std::abs(nodes[j]))) return j;
    return -1;
  }
  std::vector<double> values(double x) const {
    const int n = size();
    std::vector<double> out(n);
    const int at = node_index(x);
    if (at >= 0) {
      for (int j = 0; j < n; ++j) out[j] = j == at ? 1.0 : 0.0;
      return out;
    }
    double denom = 0.0;
    for (int j = 0; j < n; ++j) {
      out[j] = bary[j] / (x - nodes[j]);
      denom += out[j];
    }
    for (int j = 0; j < n; ++j) out[j] /= denom;
    return out;
  }
  std::vector<double> derivatives(double x) const {
    const int n = size();
    std::vector<double> out(n);
    const int at = node_index(x);
    if (at >= 0) {
      double diag = 0.0;
      for (int j = 0; j < n; ++j) {
        if (j == at) continue;
        out[j] = (bary[j] / bary[at]) / (nodes[at] - nodes[j]);
        diag -= out[j];
      }
      out[at] = diag;
      return out;
    }
    out = values(x);
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int k = 0; k < n; ++k)
        if (k != j) s += 1.0 / (x - nodes[k]);
      out[j] *= s;
    }
    return out;
  }
  std::vector<double> derivative_matrix() const {
    const int n = size();
    std::vector<double> d;
    d.reserve(static_cast<std::size_t>(n) * n);
    for (int i = 0; i < n; ++i) {
      const auto r = derivatives(nodes[i]);
      d.insert(d.end(), r.begin(), r.end());
    }
    return d;
  }
};

// -------------------------------------------------------------- macro mesh
struct Macro {
  bool quad9 = false, axisym = false;
  std::vector<double> nodes;
  std::vector<idx> cells;
  std::vector<int> material;
  struct Face {
    idx cell;
    int face;
    int tag;
  };
  std::vector<Face> boundary;
  std::vector<idx> cell_edges;
  std::vector<uint8_t> edge_fwd;
  std::vector<idx> edge_cells;

  int npc() const { return quad9 ? 9 : 4; }
  idx n_cells() const { return static_cast<idx>(material.size()); }
  idx node(idx c, int k) const { return cells[static_cast<std::size_t>(c) * npc() + k]; }
  idx cell_edge(idx c, int f) const { return cell_edges[4 * static_cast<std::size_t>(c) + f]; }
  bool forward(idx c, int f) const { return edge_fwd[4 * static_cast<std::size_t>(c) + f] != 0; }
  bool is_boundary_edge(idx e) const { return edge_cells[2 * static_cast<std::size_t>(e) + 1] < 0; }

  bool is_axis_face(idx c, int f) const {
    if (!axisym) return false;
    double extent = 0.0;
    for (int k = 0; k < 4; ++k) extent = std::max(extent, std::abs(nodes[2 * node(c, k) + 1]));
    for (int k = 0; k < 4; ++k) extent = std::max(extent, std::abs(nodes[2 * node(c, k)]));
    const double tol = 1e-10 * std::max(extent, 1e-300);
    return std::abs(nodes[2 * node(c, kFaceCorners[f][0])]) <= tol &&
           std::abs(nodes[2 * node(c, kFaceCorners[f][1])]) <= tol;
  }
  bool touches_axis(idx c) const { return is_axis_face(c, 3); }

  // Rotates every cell with an axis face so that face becomes face 3.
  void orient_axis_faces() {
    const int n = npc();
    std::vector<std::vector<std::size_t>> faces_of(n_cells());
    for (std::size_t i = 0; i < boundary.size(); ++i) faces_of[boundary[i].cell].push_back(i);
    for (idx c = 0; c < n_cells(); ++c) {
      int af = -1;
      for (int f = 0; f < 4; ++f)
        if (is_axis_face(c, f)) {
          REQUIRE(af < 0, "cell " + std::to_string(c) + " has more than one face on the axis");
          af = f;
        }
      if (af < 0 || af == 3) continue;
      const int k = (af + 1) % 4;
      idx* cell = &cells[static_cast<std::size_t>(c) * n];
      std::vector<idx> old(cell, cell + n);
      for (int i = 0; i < 4; ++i) cell[i] = old[(i + k) % 4];
      if (n == 9)
        for (int i = 0; i < 4; ++i) cell[4 + i] = old[4 + (i + k) % 4];
      for (std::size_t b : faces_of[c]) boundary[b].face = (boundary[b].face - k + 4) % 4;
    }
  }

  void build_topology() {
    const idx nc = n_cells();
    cell_edges.assign(4 * static_cast<std::size_t>(nc), -1);
    edge_fwd.assign(4 * static_cast<std::size_t>(nc), 0);
    edge_cells.clear();
    std::unordered_map<uint64_t, idx> lookup;
    lookup.reserve(4 * static_cast<std::size_t>(nc));
    for (idx c = 0; c < nc; ++c)
      for (int f = 0; f < 4; ++f) {
        const idx a = node(c, kFaceCorners[f][0]), b = node(c, kFaceCorners[f][1]);
        REQUIRE(a != b, "degenerate macro cell face");
        const uint64_t key = (static_cast<uint64_t>(std::min(a, b)) << 32) | static_cast<uint32_t>(std::max(a, b));
        auto [it, inserted] = lookup.try_emplace(key, static_cast<idx>(edge_cells.size() / 2));
        const idx e = it->second;
        if (inserted) {
          edge_cells.push_back(c);
          edge_cells.push_back(-1);
        } else {
          REQUIRE(edge_cells[2 * e + 1] < 0, "macro edge shared by more than two cells");
          edge_cells[2 * e + 1] = c;
        }
        cell_edges[4 * static_cast<std::size_t>(c) + f] = e;
        edge_fwd[4 * static_cast<std::size_t>(c) + f] = a < b ? 1 : 0;
      }
  }

  static void quadratic(double t, double* l, double* dl) {
    l[0] = 0.5 * t * (t - 1.0);
    l[1] = 1.0 - t * t;
    l[2] = 0.5 * t * (t + 1.0);
    dl[0] = t - 0.5;
    dl[1] = -2.0 * t;
    dl[2] = t + 0.5;
  }
  int shape(double xi, double eta, double* n, double* dxi, double* deta) const {
    static constexpr int A[9] = {0, 2, 2, 0, 1, 2, 1, 0, 1};
    static constexpr int B[9] = {0, 0, 2, 2, 0, 1, 2, 1, 1};
    static constexpr double X4[4] = {-1.0, 1.0, 1.0, -1.0};
    static constexpr double E4[4] = {-1.0, -1.0, 1.0, 1.0};
    if (!quad9) {
      for (int k = 0; k < 4; ++k) {
        const double a = 1.0 + X4[k] * xi, b = 1.0 + E4[k] * eta;
        n[k] = 0.25 * a * b;
        dxi[k] = 0.25 * X4[k] * b;
        deta[k] = 0.25 * a * E4[k];
      }
      return 4;
    }
    double lx[3], dlx[3], ly[3], dly[3];
    quadratic(xi, lx, dlx);
    quadratic(eta, ly, dly);
    for (int k = 0; k < 9; ++k) {
      n[k] = lx[A[k]] * ly[B[k]];
      dxi[k] = dlx[A[k]] * ly[B[k]];
      deta[k] = lx[A[k]] * dly[B[k]];
    }
    return 9;
  }
  std::array<double, 2> map(idx c, double xi, double eta) const {
    double n[9], dx[9], de[9];
    const int nk = shape(xi, eta, n, dx, de);
    std::array<double, 2> x{0.0, 0.0};
    for (int k = 0; k < nk; ++k) {
      const idx v = node(c, k);
      x[0] += n[k] * nodes[2 * v];
      x[1] += n[k] * nodes[2 * v + 1];
    }
    return x;
  }
  std::array<double, 4> jacobian(idx c, double xi, double eta) const {
    double n[9], dx[9], de[9];
    const int nk = shape(xi, eta, n, dx, de);
    std::array<double, 4> j{0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < nk; ++k) {
      const idx v = node(c, k);
      j[0] += dx[k] * nodes[2 * v];
      j[1] += de[k] * nodes[2 * v];
      j[2] += dx[k] * nodes[2 * v + 1];
      j[3] += de[k] * nodes[2 * v + 1];
    }
    return j;
  }
};

// -------------------------------------------------------------- forest
struct Leaf {
  idx tree;
  int32_t level, i, j;
};

struct FaceNb {
  idx leaf = -1;
  int face = -1;
  int level_diff = 0;
};

struct LeafKeyHash {
  std::size_t operator()(const std::pair<uint64_t, uint64_t>& k) const {
    return std::hash<uint64_t>()(k.first * 0x9e3779b97f4a7c15ULL ^ (k.second + 0x632be59bd9b4e019ULL));
  }
};

uint32_t compact_bits(uint64_t m) {
  uint64_t x = m & 0x5555555555555555ULL;
  x = (x | (x >> 1)) & 0x3333333333333333ULL;
  x = (x | (x >> 2)) & 0x0f0f0f0f0f0f0f0fULL;
  x = (x | (x >> 4)) & 0x00ff00ff00ff00ffULL;
  x = (x | (x >> 8)) & 0x0000ffff0000ffffULL;
  x = (x | (x >> 16)) & 0x00000000ffffffffULL;
  return static_cast<uint32_t>(x);
}

class Forest {
 public:
  Forest(const Macro* m, std::vector<Leaf> leaves) : m_(m), leaves_(std::move(leaves)) {
    index_.reserve(leaves_.size());
    max_level_ = 0;
    for (std::size_t l = 0; l < leaves_.size(); ++l) {
      const Leaf& lf = leaves_[l];
      index_[key(lf.tree, lf.level, lf.i, lf.j)] = static_cast<idx>(l);
      max_level_ = std::max(max_level_, static_cast<int>(lf.level));
    }
  }
  static Forest uniform(const Macro* m, int level) {
    const uint64_t per = uint64_t{1} << (2 * level);
    REQUIRE(per * static_cast<uint64_t>(m->n_cells()) < (uint64_t{1} << 31), "too many leaves");
    std::vector<Leaf> leaves;
    leaves.reserve(per * m->n_cells());
    for (idx t = 0; t < m->n_cells(); ++t)
      for (uint64_t q = 0; q < per; ++q)
        leaves.push_back({t, level, static_cast<int32_t>(compact_bits(q)), static_cast<int32_t>(compact_bits(q >> 1))});
    return Forest(m, std::move(leaves));
  }
  const Macro& macro() const { return *m_; }
  idx n_leaves() const { return static_cast<idx>(leaves_.size()); }
  const Leaf& leaf(idx l) const { return leaves_[l]; }
  bool is_axial(idx l) const { return leaves_[l].i == 0 && m_->touches_axis(leaves_[l].tree); }
  std::array<double, 4> box(idx l) const {
    const Leaf& lf = leaves_[l];
    const double h = 2.0 / static_cast<double>(int64_t{1} << lf.level);
    return {-1.0 + lf.i * h, -1.0 + (lf.i + 1) * h, -1.0 + lf.j * h, -1.0 + (lf.j + 1) * h};
  }
  std::array<double, 2> leaf_map(idx l, double xi, double eta) const {
    const auto b = box(l);
    return m_->map(leaves_[l].tree, b[0] + (xi + 1.0) * 0.5 * (b[1] - b[0]), b[2] + (eta + 1.0) * 0.5 * (b[3] - b[2]));
  }
  std::array<double, 4> leaf_jacobian(idx l, double xi, double eta) const {
    const auto b = box(l);
    const double hx = 0.5 * (b[1] - b[0]), hy = 0.5 * (b[3] - b[2]);
    const auto j = m_->jacobian(leaves_[l].tree, b[0] + (xi + 1.0) * hx, b[2] + (eta + 1.0) * hy);
    return {j[0] * hx, j[1] * hy, j[2] * hx, j[3] * hy};
  }
  idx find_leaf(idx tree, int64_t a, int64_t b) const {
    constexpr int64_t h = int64_t{1} << (kMaxLevel + 1);
    if (a < 0 || b < 0 || a >= h || b >= h) return -1;
    for (int level = 0; level <= max_level_; ++level) {
      const int shift = kMaxLevel + 1 - level;
      const auto it = index_.find(key(tree, level, a >> shift, b >> shift));
      if (it != index_.end()) return it->second;
    }
    return -1;
  }
  FaceNb face_neighbor(idx l, int f) const {
    constexpr int64_t h = int64_t{1} << (kMaxLevel + 1);
    const Leaf& lf = leaves_[l];
    const int64_t size = int64_t{1} << (kMaxLevel + 1 - lf.level);
    const int64_t a0 = lf.i * size, b0 = lf.j * size, am = a0 + size / 2, bm = b0 + size / 2;
    int64_t a, b;
    switch (f) {
      case 0: a = am; b = b0 - 1; break;
      case 1: a = a0 + size; b = bm; break;
      case 2: a = am; b = b0 + size; break;
      default: a = a0 - 1; b = bm; break;
    }
    FaceNb out;
    idx tree = lf.tree;
    int nface = (f + 2) % 4;
    if (a < 0 || b < 0 || a >= h || b >= h) {
      const idx e = m_->cell_edge(lf.tree, f);
      const idx c0 = m_->edge_cells[2 * e], c1 = m_->edge_cells[2 * e + 1];
      if (c1 < 0) return out;
      const idx other = c0 == lf.tree ? c1 : c0;
      int of = 0;
      while (m_->cell_edge(other, of) != e) ++of;
      const int64_t s_local = (f == 0) ? a : (f == 1) ? b : (f == 2) ? h - a : h - b;
      const int64_t c = m_->forward(lf.tree, f) ? s_local : h - s_local;
      const int64_t s2 = m_->forward(other, of) ? c : h - c;
      switch (of) {
        case 0: a = s2; b = 0; break;
        case 1: a = h - 1; b = s2; break;
        case 2: a = h - s2; b = h - 1; break;
        default: a = 0; b = h - s2; break;
      }
      tree = other;
      nface = of;
    }
    out.leaf = find_leaf(tree, a, b);
    REQUIRE(out.leaf >= 0, "forest has no leaf at a face-neighbour position");
    out.face = nface;
    out.level_diff = leaves_[out.leaf].level - lf.level;
    return out;
  }
  double face_coordinate(idx from, int f, double t, idx to, int to_face) const {
    auto range = [this](idx l, int face) {
      const Leaf& lf = leaves_[l];
      const double n = static_cast<double>(int64_t{1} << lf.level);
      const int64_t i = (face == 0 || face == 2) ? lf.i : lf.j;
      return std::array<double, 2>{i / n, (i + 1) / n};
    };
    const auto r = range(from, f);
    const double u = r[0] + 0.5 * (t + 1.0) * (r[1] - r[0]);
    double u2 = u;
    const Leaf& la = leaves_[from];
    const Leaf& lb = leaves_[to];
    if (la.tree != lb.tree) {
      const double s = (f == 0 || f == 1) ? u : 1.0 - u;
      const double c = m_->forward(la.tree, f) ? s : 1.0 - s;
      const double s2 = m_->forward(lb.tree, to_face) ? c : 1.0 - c;
      u2 = (to_face == 0 || to_face == 1) ? s2 : 1.0 - s2;
    }
    const auto r2 = range(to, to_face);
    return -1.0 + 2.0 * (u2 - r2[0]) / (r2[1] - r2[0]);
  }
  Forest refine(const std::vector<char>& mark) const {
    std::vector<Leaf> out;
    out.reserve(leaves_.size() + 3 * std::count(mark.begin(), mark.end(), 1));
    for (std::size_t l = 0; l < leaves_.size(); ++l) {
      const Leaf& lf = leaves_[l];
      if (!mark[l]) {
        out.push_back(lf);
        continue;
      }
      REQUIRE(lf.level < kMaxLevel, "cannot refine beyond the deepest level");
      for (int c = 0; c < 4; ++c) out.push_back({lf.tree, lf.level + 1, 2 * lf.i + (c & 1), 2 * lf.j + (c >> 1)});
    }
    return Forest(m_, std::move(out));
  }
  Forest balance(const std::function<bool(idx, idx)>& must_match) const {
    Forest cur = *this;
    for (;;) {
      std::vector<char> mark(cur.leaves_.size(), 0);
      bool any = false;
      for (idx l = 0; l < cur.n_leaves(); ++l) {
        const Leaf& lf = cur.leaves_[l];
        for (int f = 0; f < 4; ++f) {
          const FaceNb nb = cur.face_neighbor(l, f);
          if (nb.leaf < 0 || nb.level_diff >= 0) continue;
          const idx ot = cur.leaves_[nb.leaf].tree;
          const bool strict = must_match && ot != lf.tree && must_match(lf.tree, ot);
          if (nb.level_diff < -1 || strict) {
            mark[nb.leaf] = 1;
            any = true;
          }
        }
      }
      if (!any) return cur;
      cur = cur.refine(mark);
    }
  }
  // Unique leaf-corner vertices in first-touch order (forest.cpp:242-261).
  std::vector<idx> leaf_vertices(idx& n_vertices) const {
    struct LK {
      int kind;
      int64_t id, a, b;
      bool operator==(const LK& o) const { return kind == o.kind && id == o.id && a == o.a && b == o.b; }
    };
    struct LKH {
      std::size_t operator()(const LK& k) const {
        uint64_t h = static_cast<uint64_t>(k.kind);
        for (int64_t v : {k.id, k.a, k.b}) h ^= static_cast<uint64_t>(v) + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2);
        return static_cast<std::size_t>(h);
      }
    };
    auto lattice_key = [this](idx cell, int64_t a, int64_t b) -> LK {
      constexpr int64_t s = int64_t{1} << kMaxLevel;
      const bool left = a == 0, right = a == s, bottom = b == 0, top = b == s;
      if ((left || right) && (bottom || top)) {
        const int corner = bottom ? (left ? 0 : 1) : (right ? 2 : 3);
        return {0, m_->node(cell, corner), 0, 0};
      }
      if (bottom || right || top || left) {
        int face;
        int64_t t;
        if (bottom) { face = 0; t = a; }
        else if (right) { face = 1; t = b; }
        else if (top) { face = 2; t = s - a; }
        else { face = 3; t = s - b; }
        const int64_t canonical = m_->forward(cell, face) ? t : s - t;
        return {1, m_->cell_edge(cell, face), canonical, 0};
      }
      return {2, cell, a, b};
    };
    std::vector<idx> corners(4 * leaves_.size());
    std::unordered_map<LK, idx, LKH> ids;
    ids.reserve(leaves_.size() * 2 + 16);
    n_vertices = 0;
    constexpr int di[4] = {0, 1, 1, 0}, dj[4] = {0, 0, 1, 1};
    for (std::size_t l = 0; l < leaves_.size(); ++l) {
      const Leaf& lf = leaves_[l];
      const int64_t step = int64_t{1} << (kMaxLevel - lf.level);
      for (int k = 0; k < 4; ++k) {
        auto [it, ins] = ids.try_emplace(lattice_key(lf.tree, (lf.i + di[k]) * step, (lf.j + dj[k]) * step), n_vertices);
        if (ins) ++n_vertices;
        corners[4 * l + k] = it->second;
      }
    }
    return corners;
  }

 private:
  static std::pair<uint64_t, uint64_t> key(idx tree, int level, int64_t i, int64_t j) {
    return {(static_cast<uint64_t>(tree) << 8) | static_cast<uint64_t>(level),
            (static_cast<uint64_t>(i) << 32) | static_cast<uint64_t>(j)};
  }
  const Macro* m_;
  std::vector<Leaf> leaves_;
  std::unordered_map<std::pair<uint64_t, uint64_t>, idx, LeafKeyHash> index_;
  int max_level_ = 0;
};

// ----------------------------------------------------------- geometry
enum Kind : uint8_t { kRect = 0, kAffine = 1, kCurved = 2, kAxisym = 3 };

struct Geometry {
  int ngll = 0;
  std::vector<double> x, z, xi_x, xi_z, eta_x, eta_z, jac;
  std::vector<uint8_t> kind;
};

Geometry compute_geometry(const Forest& forest, const std::vector<double>& ref, const std::vector<double>& axial_ref) {
  Geometry g;
  g.ngll = static_cast<int>(ref.size());
  const int ng = g.ngll;
  const std::size_t npe = static_cast<std::size_t>(ng) * ng, total = npe * forest.n_leaves();
  for (auto* v : {&g.x, &g.z, &g.xi_x, &g.xi_z, &g.eta_x, &g.eta_z, &g.jac}) v->resize(total);
  g.kind.resize(forest.n_leaves());
  constexpr double kTol = 1e-10;
  for (idx e = 0; e < forest.n_leaves(); ++e) {
    const idx cell = forest.leaf(e).tree;
    const std::vector<double>& rx = forest.is_axial(e) ? axial_ref : ref;
    const auto b = forest.box(e);
    const double hx = 0.5 * (b[1] - b[0]), hy = 0.5 * (b[3] - b[2]);
    double scale = 0.0, deviation = 0.0, off = 0.0;
    std::array<double, 4> j0{};
    for (int jq = 0; jq < ng; ++jq)
      for (int iq = 0; iq < ng; ++iq) {
        const double xi = b[0] + (rx[iq] + 1.0) * hx;
        const double eta = b[2] + (ref[jq] + 1.0) * hy;
        const auto x = forest.macro().map(cell, xi, eta);
        const auto jm = forest.macro().jacobian(cell, xi, eta);
        const std::array<double, 4> j{jm[0] * hx, jm[1] * hy, jm[2] * hx, jm[3] * hy};
        const double det = j[0] * j[3] - j[1] * j[2];
        const std::size_t p = e * npe + static_cast<std::size_t>(jq) * ng + iq;
        g.x[p] = x[0];
        g.z[p] = x[1];
        g.jac[p] = det;
        g.xi_x[p] = j[3] / det;
        g.xi_z[p] = -j[1] / det;
        g.eta_x[p] = -j[2] / det;
        g.eta_z[p] = j[0] / det;
        if (iq == 0 && jq == 0) j0 = j;
        for (int k = 0; k < 4; ++k) {
          scale = std::max(scale, std::abs(j[k]));
          deviation = std::max(deviation, std::abs(j[k] - j0[k]));
        }
        off = std::max({off, std::abs(j[1]), std::abs(j[2])});
      }
    g.kind[e] = deviation > kTol * scale ? kCurved : off > kTol * scale ? kAffine : kRect;
  }
  for (double d : g.jac) REQUIRE(d > 0.0, "leaf mapping has a non-positive Jacobian");
  return g;
}

// -------------------------------------------------------------- DofMap
struct DofMap {
  int ngll = 0, npe = 0;
  idx n_elem = 0, n_global = 0;
  std::vector<idx> l2g, row_offsets{0}, row_dofs, t_offsets, t_slots, primary;
  std::vector<double> row_weights, t_weights;
  idx n_rows() const { return static_cast<idx>(row_offsets.size()) - 1; }
  using Row = std::vector<std::pair<idx, double>>;
  Row slot_entries(idx e, int k) const {
    const idx m = l2g[static_cast<std::size_t>(e) * npe + k];
    if (m >= 0) return {{m, 1.0}};
    Row out;
    const idx r = -1 - m;
    for (idx q = row_offsets[r]; q < row_offsets[r + 1]; ++q) out.push_back({row_dofs[q], row_weights[q]});
    return out;
  }
  idx global_index(idx e, int k) const {
    const idx m = l2g[static_cast<std::size_t>(e) * npe + k];
    REQUIRE(m >= 0, "boundary point lies on a hanging face");
    return m;
  }
};

int face_slot(int f, int m, int n, int ngll) {
  switch (f) {
    case 0: return m;
    case 1: return m * ngll + n;
    case 2: return n * ngll + m;
    default: return m * ngll;
  }
}

DofMap build_dofmap(const Forest& forest, int ngll, const std::vector<idx>& leaves, const std::vector<idx>& corners,
                    idx n_vertices) {
  constexpr idx kPending = std::numeric_limits<idx>::min();
  DofMap d;
  d.ngll = ngll;
  d.npe = ngll * ngll;
  d.n_elem = static_cast<idx>(leaves.size());
  const int n = ngll - 1;
  const std::size_t npe = d.npe, n_slots = static_cast<std::size_t>(d.n_elem) * npe;
  REQUIRE(n_slots < static_cast<std::size_t>(std::numeric_limits<idx>::max()), "too many element points");
  std::vector<idx> element_of_leaf(forest.n_leaves(), -1);
  for (idx e = 0; e < d.n_elem; ++e) element_of_leaf[leaves[e]] = e;
  struct Hang {
    idx coarse = -1;
    int face = -1;
  };
  std::vector<std::array<Hang, 4>> hang(d.n_elem);
  std::vector<char> hanging_vertex(n_vertices, 0);
  for (idx e = 0; e < d.n_elem; ++e) {
    const idx leaf = leaves[e];
    for (int f = 0; f < 4; ++f) {
      const FaceNb nb = forest.face_neighbor(leaf, f);
      if (nb.leaf < 0) continue;
      const idx ce = element_of_leaf[nb.leaf];
      if (ce < 0) {
        REQUIRE(nb.level_diff == 0, "leaves of different domains meet at different refinement levels");
        continue;
      }
      if (nb.level_diff >= 0) continue;
      REQUIRE(nb.level_diff == -1, "forest is not 2:1 balanced");
      hang[e][f] = {ce, nb.face};
      const idx c0 = corners[4 * static_cast<std::size_t>(nb.leaf) + kFaceCorners[nb.face][0]];
      const idx c1 = corners[4 * static_cast<std::size_t>(nb.leaf) + kFaceCorners[nb.face][1]];
      for (int c = 0; c < 2; ++c) {
        const idx v = corners[4 * static_cast<std::size_t>(leaf) + kFaceCorners[f][c]];
        if (v != c0 && v != c1) hanging_vertex[v] = 1;
      }
    }
  }
  // First-touch numbering: per element, its new edges (blocks of n - 1),
  // then its corners and interior points in local order.
  std::vector<idx> vertex_id(n_vertices, -1);
  std::unordered_map<uint64_t, std::pair<idx, int>> edges;
  edges.reserve(2 * static_cast<std::size_t>(d.n_elem) + 16);
  d.l2g.assign(n_slots, -1);
  idx next = 0;
  for (idx e = 0; e < d.n_elem; ++e) {
    const idx* v = &corners[4 * static_cast<std::size_t>(leaves[e])];
    idx base[4];
    bool fwd[4];
    for (int f = 0; f < 4; ++f) {
      const idx a = v[kFaceCorners[f][0]], b = v[kFaceCorners[f][1]];
      fwd[f] = a < b;
      if (hang[e][f].coarse >= 0) {
        base[f] = -1;
        continue;
      }
      const uint64_t key = (static_cast<uint64_t>(std::min(a, b)) << 32) | static_cast<uint32_t>(std::max(a, b));
      auto [it, ins] = edges.try_emplace(key, std::pair<idx, int>{next, 0});
      if (ins) next += n - 1;
      ++it->second.second;
      REQUIRE(it->second.second <= 2, "leaf edge shared by more than two elements");
      base[f] = it->second.first;
    }
    idx* map = &d.l2g[static_cast<std::size_t>(e) * npe];
    for (int j = 0; j <= n; ++j)
      for (int i = 0; i <= n; ++i) {
        const bool xe = i == 0 || i == n, ee = j == 0 || j == n;
        idx g;
        if (xe && ee) {
          const int corner = (j == 0) ? (i == 0 ? 0 : 1) : (i == n ? 2 : 3);
          if (hanging_vertex[v[corner]]) {
            g = kPending;
          } else {
            idx& id = vertex_id[v[corner]];
            if (id < 0) id = next++;
            g = id;
          }
        } else if (xe || ee) {
          int face, p;
          if (j == 0) { face = 0; p = i; }
          else if (i == n) { face = 1; p = j; }
          else if (j == n) { face = 2; p = n - i; }
          else { face = 3; p = n - j; }
          g = base[face] < 0 ? kPending : base[face] + ((fwd[face] ? p : n - p) - 1);
        } else {
          g = next++;
        }
        map[j * ngll + i] = g;
      }
  }
  d.n_global = next;
  // Constraint rows of hanging slots: the coarse face's interpolant, resolved
  // recursively through constrained coarse nodes.
  const Lagrange gll_basis(gll(ngll).points), glj_basis(glj01(ngll).points);
  auto face_basis = [&](idx e, int f) -> const Lagrange& {
    return (forest.is_axial(leaves[e]) && (f == 0 || f == 2)) ? glj_basis : gll_basis;
  };
  std::map<std::size_t, DofMap::Row> memo;
  std::function<DofMap::Row(std::size_t)> resolve = [&](std::size_t slot) -> DofMap::Row {
    const idx m = d.l2g[slot];
    if (m >= 0) return {{m, 1.0}};
    if (m != kPending) {
      DofMap::Row row;
      const idx r = -1 - m;
      for (idx q = d.row_offsets[r]; q < d.row_offsets[r + 1]; ++q) row.push_back({d.row_dofs[q], d.row_weights[q]});
      return row;
    }
    const auto it = memo.find(slot);
    if (it != memo.end()) return it->second;
    const idx e = static_cast<idx>(slot / npe);
    const int k = static_cast<int>(slot % npe), i = k % ngll, j = k / ngll;
    int f = -1;
    for (int c = 0; c < 4 && f < 0; ++c) {
      if (hang[e][c].coarse < 0) continue;
      const bool on = (c == 0 && j == 0) || (c == 1 && i == n) || (c == 2 && j == n) || (c == 3 && i == 0);
      if (on) f = c;
    }
    REQUIRE(f >= 0, "constrained point is not on a hanging face");
    const Hang h = hang[e][f];
    const double t = face_basis(e, f).nodes[(f == 0 || f == 2) ? i : j];
    const double tc = forest.face_coordinate(leaves[e], f, t, leaves[h.coarse], h.face);
    const auto w = face_basis(h.coarse, h.face).values(tc);
    std::map<idx, double> acc;
    for (int q = 0; q <= n; ++q) {
      if (std::abs(w[q]) < 1e-14) continue;
      const std::size_t cs = static_cast<std::size_t>(h.coarse) * npe + face_slot(h.face, q, n, ngll);
      for (const auto& [g, wg] : resolve(cs)) acc[g] += w[q] * wg;
    }
    DofMap::Row row(acc.begin(), acc.end());
    memo[slot] = row;
    return row;
  };
  for (std::size_t slot = 0; slot < n_slots; ++slot) {
    if (d.l2g[slot] != kPending) continue;
    DofMap::Row row = resolve(slot);
    if (row.size() == 1 && std::abs(row[0].second - 1.0) < 1e-12) {
      d.l2g[slot] = row[0].first;
      continue;
    }
    d.l2g[slot] = -1 - d.n_rows();
    for (const auto& [g, w] : row) {
      d.row_dofs.push_back(g);
      d.row_weights.push_back(w);
    }
    d.row_offsets.push_back(static_cast<idx>(d.row_dofs.size()));
  }
  // Transpose, contributions in ascending slot order.
  d.t_offsets.assign(static_cast<std::size_t>(d.n_global) + 1, 0);
  auto each = [&](auto&& fn) {
    for (std::size_t s = 0; s < n_slots; ++s) {
      const idx m = d.l2g[s];
      if (m >= 0) {
        fn(s, m, 1.0);
      } else {
        const idx r = -1 - m;
        for (idx q = d.row_offsets[r]; q < d.row_offsets[r + 1]; ++q) fn(s, d.row_dofs[q], d.row_weights[q]);
      }
    }
  };
  each([&](std::size_t, idx g, double) { ++d.t_offsets[static_cast<std::size_t>(g) + 1]; });
  for (idx g = 0; g < d.n_global; ++g) d.t_offsets[g + 1] += d.t_offsets[g];
  d.t_slots.resize(d.t_offsets.back());
  if (d.n_rows() > 0) d.t_weights.resize(d.t_offsets.back());
  std::vector<idx> fill(d.t_offsets.begin(), d.t_offsets.end() - 1);
  each([&](std::size_t s, idx g, double w) {
    const idx at = fill[g]++;
    d.t_slots[at] = static_cast<idx>(s);
    if (!d.t_weights.empty()) d.t_weights[at] = w;
  });
  d.primary.assign(d.n_global, -1);
  for (std::size_t s = 0; s < n_slots; ++s) {
    const idx m = d.l2g[s];
    if (m >= 0 && d.primary[m] < 0) d.primary[m] = static_cast<idx>(s);
  }
  for (idx g = 0; g < d.n_global; ++g) REQUIRE(d.primary[g] >= 0, "global point without an unconstrained slot");
  return d;
}

// ------------------------------------------------------------ the problem
struct Material {
  int medium = 1;  // 0 acoustic, 1 elastic
  double vp = 0, vs = 0, rho = 0;
};

struct Block {
  int kind = 0, m = 0;
  std::vector<idx> elements;
  std::vector<float> metric, coef0, coef1, wr, hoop, r;
  std::vector<uint8_t> axial;
};

struct Domain {
  int medium = 1, ncomp = 2, m = 0;
  std::vector<idx> leaves, element_of_leaf;
  DofMap dofs;
  std::vector<Block> blocks;
  std::vector<float> mass, inv_mass;
  std::vector<idx> absorbing_points, dirichlet_points, axis_points, axis_components;
  std::vector<float> absorbing_coef;
  std::vector<double> coords;
};

struct SourceTerm {
  int domain;
  std::vector<idx> points;
  std::vector<float> coef;
  int stf_kind;
  double f0, t0, amp;
};

struct ReceiverTerm {
  int domain;
  std::vector<idx> points;
  std::vector<float> value, d_dx, d_dz;
  double rho;
  std::vector<int32_t> quantities;
};

struct Output {
  std::vector<std::string> keys;
  std::vector<insem_case_array> arrays;
  std::vector<std::shared_ptr<void>> owned;

  template <class T>
  void put(const std::string& key, std::vector<T> v, int dtype) {
    auto p = std::make_shared<std::vector<T>>(std::move(v));
    owned.push_back(p);
    keys.push_back(key);
    arrays.push_back({nullptr, dtype, static_cast<int64_t>(p->size()), p->data()});
  }
  void f32(const std::string& k, std::vector<float> v) { put(k, std::move(v), 0); }
  void f64(const std::string& k, std::vector<double> v) { put(k, std::move(v), 1); }
  void i32(const std::string& k, std::vector<idx> v) { put(k, std::move(v), 2); }
  void u8(const std::string& k, std::vector<uint8_t> v) { put(k, std::move(v), 3); }
  void scalar_i(const std::string& k, int64_t v) { i32(k, {static_cast<idx>(v)}); }
  void scalar_d(const std::string& k, double v) { f64(k, {v}); }
  void finish() {
    for (std::size_t i = 0; i < arrays.size(); ++i) arrays[i].key = keys[i].c_str();
  }
};

class Builder {
 public:
  explicit Builder(const insem_case_desc& d) : d_(d) {}

  Output run() {
    make_macro();
    for (int i = 0; i < d_.n_materials; ++i) {
      Material m{d_.material_medium[i], d_.material_vp[i], d_.material_vs[i], d_.material_rho[i]};
      REQUIRE(m.rho > 0 && m.vp > 0, "material with non-positive rho or vp");
      if (m.medium == 1) REQUIRE(m.vs > 0 && m.vp > m.vs, "elastic material needs 0 < vs < vp");
      mats_[d_.material_region[i]] = m;
    }
    for (idx c = 0; c < macro_.n_cells(); ++c)
      REQUIRE(mats_.count(macro_.material[c]), "no material assigned to region " + std::to_string(macro_.material[c]));
    for (int i = 0; i < d_.n_bc; ++i) bcs_[d_.bc_tag[i]] = d_.bc_type[i];
    REQUIRE(d_.order >= 1 && d_.order <= 8, "polynomial order must be in 1..8");
    ngll_ = d_.order + 1;
    axisym_ = macro_.axisym;
    m_ = d_.azimuthal_order;
    REQUIRE(m_ == 0 || (m_ == 1 && axisym_), "azimuthal order 1 needs an axisymmetric mesh");
    rule_ = gll(ngll_);
    glj_ = glj01(ngll_);
    forest_ = std::make_unique<Forest>(build_forest());
    geom_ = compute_geometry(*forest_, rule_.points, glj_.points);
    corners_ = forest_->leaf_vertices(n_vertices_);
    build_domains();
    for (Domain& dom : domains_) build_boundaries(dom);
    build_coupling();
    build_sources();
    build_receivers();
    return pack();
  }

 private:
  const Material& material_of_leaf(idx leaf) const { return mats_.at(macro_.material[forest_->leaf(leaf).tree]); }

  void make_macro() {
    macro_.quad9 = d_.quad9 != 0;
    macro_.axisym = d_.axisymmetric != 0;
    REQUIRE(d_.n_nodes > 0 && d_.n_cells > 0, "empty macro mesh");
    macro_.nodes.assign(d_.nodes, d_.nodes + 2 * static_cast<std::size_t>(d_.n_nodes));
    macro_.cells.assign(d_.cells, d_.cells + static_cast<std::size_t>(d_.n_cells) * macro_.npc());
    for (idx v : macro_.cells) REQUIRE(v >= 0 && v < d_.n_nodes, "cell references a missing node");
    macro_.material.assign(d_.cell_region, d_.cell_region + d_.n_cells);
    for (int i = 0; i < d_.n_boundary; ++i)
      macro_.boundary.push_back({d_.boundary[3 * i], d_.boundary[3 * i + 1], d_.boundary[3 * i + 2]});
    if (macro_.axisym) macro_.orient_axis_faces();
    macro_.build_topology();
  }

  Forest build_forest() {
    Forest forest = Forest::uniform(&macro_, d_.uniform_level);
    for (;;) {
      std::vector<char> mark(forest.n_leaves(), 0);
      bool any = false;
      for (idx l = 0; l < forest.n_leaves(); ++l) {
        const Leaf& lf = forest.leaf(l);
        if (lf.level >= d_.max_level) continue;
        std::array<std::array<double, 2>, 4> c;
        const double ref[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
        for (int k = 0; k < 4; ++k) c[k] = forest.leaf_map(l, ref[k][0], ref[k][1]);
        bool refine = false;
        if (d_.f_max > 0.0) {
          double h = 0.0;
          for (int k = 0; k < 4; ++k)
            h = std::max(h, std::hypot(c[(k + 1) % 4][0] - c[k][0], c[(k + 1) % 4][1] - c[k][1]));
          const Material& m = mats_.at(macro_.material[lf.tree]);
          const double v_min = m.medium == 1 ? m.vs : m.vp;
          refine = h > d_.order * (v_min / d_.f_max) / d_.points_per_wavelength;
        }
        if (!refine) {
          double x0 = c[0][0], x1 = c[0][0], z0 = c[0][1], z1 = c[0][1];
          for (const auto& p : c) {
            x0 = std::min(x0, p[0]);
            x1 = std::max(x1, p[0]);
            z0 = std::min(z0, p[1]);
            z1 = std::max(z1, p[1]);
          }
          for (int r = 0; r < d_.n_regions; ++r) {
            const double* g = d_.regions + 5 * r;
            if (lf.level < static_cast<int>(g[4]) && x0 <= g[1] && x1 >= g[0] && z0 <= g[3] && z1 >= g[2]) refine = true;
          }
        }
        if (refine) {
          mark[l] = 1;
          any = true;
        }
      }
      if (!any) break;
      forest = forest.refine(mark);
    }
    return forest.balance([this](idx a, idx b) {
      return mats_.at(macro_.material[a]).medium != mats_.at(macro_.material[b]).medium;
    });
  }

  // solver.cpp:147-254
  void build_domains() {
    const std::size_t npe = static_cast<std::size_t>(ngll_) * ngll_;
    for (int medium : {0, 1}) {
      Domain dom;
      dom.medium = medium;
      dom.m = m_;
      dom.ncomp = medium == 1 ? (m_ == 1 ? 3 : 2) : 1;
      if (axisym_) {
        if (medium == 1) dom.axis_components = m_ == 1 ? std::vector<idx>{0, 2} : std::vector<idx>{0};
        else if (m_ == 1) dom.axis_components = {0};
      }
      dom.element_of_leaf.assign(forest_->n_leaves(), -1);
      for (idx l = 0; l < forest_->n_leaves(); ++l)
        if (material_of_leaf(l).medium == medium) {
          dom.element_of_leaf[l] = static_cast<idx>(dom.leaves.size());
          dom.leaves.push_back(l);
        }
      if (dom.leaves.empty()) continue;
      dom.dofs = build_dofmap(*forest_, ngll_, dom.leaves, corners_, n_vertices_);
      const std::size_t nl = dom.leaves.size() * npe;
      std::vector<double> wr(nl), hoop(nl, 0.0);
      std::vector<char> axial(dom.leaves.size(), 0);
      for (std::size_t e = 0; e < dom.leaves.size(); ++e) {
        const idx leaf = dom.leaves[e];
        axial[e] = axisym_ && forest_->is_axial(leaf) ? 1 : 0;
        for (std::size_t k = 0; k < npe; ++k) {
          const int i = static_cast<int>(k % ngll_), j = static_cast<int>(k / ngll_);
          const std::size_t pt = static_cast<std::size_t>(leaf) * npe + k;
          const double jac = geom_.jac[pt];
          if (!axisym_) {
            wr[e * npe + k] = rule_.weights[i] * rule_.weights[j] * jac;
          } else if (!axial[e]) {
            hoop[e * npe + k] = rule_.weights[i] * rule_.weights[j] * jac;
            wr[e * npe + k] = hoop[e * npe + k] * std::max(geom_.x[pt], 0.0);
          } else {
            const double x_xi = geom_.eta_z[pt] * jac;
            const double rt = i == 0 ? x_xi : geom_.x[pt] / (1.0 + glj_.points[i]);
            wr[e * npe + k] = glj_.weights[i] * rule_.weights[j] * jac * rt;
            hoop[e * npe + k] = i == 0 ? 0.0 : wr[e * npe + k] / geom_.x[pt];
          }
        }
      }
      std::vector<double> coef0(nl), coef1(nl), local_mass(nl);
      for (std::size_t e = 0; e < dom.leaves.size(); ++e) {
        const Material& m = material_of_leaf(dom.leaves[e]);
        for (std::size_t k = 0; k < npe; ++k) {
          const std::size_t q = e * npe + k;
          if (medium == 1) {
            coef0[q] = m.rho * (m.vp * m.vp - 2.0 * m.vs * m.vs);
            coef1[q] = m.rho * m.vs * m.vs;
            local_mass[q] = wr[q] * m.rho;
          } else {
            coef0[q] = 1.0 / m.rho;
            coef1[q] = 0.0;
            local_mass[q] = wr[q] / (m.rho * m.vp * m.vp);
          }
        }
      }
      if (axisym_) dom.blocks = {axisym_block(dom, coef0, coef1, wr, hoop, axial)};
      else dom.blocks = cartesian_blocks(dom, coef0, coef1);
      // Lumped mass: assemble of the local masses (dof_map.hpp:123-141, double).
      std::vector<double> mass(dom.dofs.n_global);
      const bool weighted = !dom.dofs.t_weights.empty();
      for (idx g = 0; g < dom.dofs.n_global; ++g) {
        double s = 0.0;
        for (idx q = dom.dofs.t_offsets[g]; q < dom.dofs.t_offsets[g + 1]; ++q) {
          const double v = local_mass[dom.dofs.t_slots[q]];
          s += weighted ? dom.dofs.t_weights[q] * v : v;
        }
        mass[g] = s;
      }
      dom.mass.assign(mass.begin(), mass.end());
      dom.inv_mass.resize(mass.size());
      for (std::size_t g = 0; g < mass.size(); ++g) {
        REQUIRE(mass[g] > 0.0, "non-positive lumped mass at a global point (degenerate element?)");
        dom.inv_mass[g] = static_cast<float>(1.0 / mass[g]);
      }
      const std::size_t ng = dom.dofs.n_global;
      dom.coords.resize(2 * ng);
      for (std::size_t g = 0; g < ng; ++g) {
        const std::size_t s = dom.dofs.primary[g];
        const std::size_t q = static_cast<std::size_t>(dom.leaves[s / npe]) * npe + s % npe;
        dom.coords[g] = geom_.x[q];
        dom.coords[ng + g] = geom_.z[q];
        if (!dom.axis_components.empty() && geom_.x[q] <= 0.0) dom.axis_points.push_back(static_cast<idx>(g));
      }
      domains_.push_back(std::move(dom));
    }
  }

  Block axisym_block(const Domain& dom, const std::vector<double>& coef0, const std::vector<double>& coef1,
                     const std::vector<double>& wr, const std::vector<double>& hoop, const std::vector<char>& axial) {
    const std::size_t npe = static_cast<std::size_t>(ngll_) * ngll_;
    Block b;
    b.kind = kAxisym;
    b.m = m_;
    b.axial.assign(axial.begin(), axial.end());
    const std::size_t n = dom.leaves.size();
    b.elements.resize(n);
    b.metric.reserve(n * npe * 5);
    for (std::size_t e = 0; e < n; ++e) {
      b.elements[e] = static_cast<idx>(e);
      const std::size_t p0 = static_cast<std::size_t>(dom.leaves[e]) * npe;
      for (std::size_t k = 0; k < npe; ++k) {
        const std::size_t p = p0 + k, q = e * npe + k;
        for (double v : {geom_.xi_x[p], geom_.xi_z[p], geom_.eta_x[p], geom_.eta_z[p], geom_.jac[p]})
          b.metric.push_back(static_cast<float>(v));
        b.coef0.push_back(static_cast<float>(coef0[q]));
        b.coef1.push_back(static_cast<float>(coef1[q]));
        b.wr.push_back(static_cast<float>(wr[q]));
        b.hoop.push_back(static_cast<float>(hoop[q]));
        b.r.push_back(static_cast<float>(geom_.x[p] <= 0.0 ? 0.0 : geom_.x[p]));
      }
    }
    return b;
  }

  std::vector<Block> cartesian_blocks(const Domain& dom, const std::vector<double>& coef0,
                                      const std::vector<double>& coef1) {
    const std::size_t npe = static_cast<std::size_t>(ngll_) * ngll_;
    std::vector<Block> out;
    for (int kind : {kRect, kAffine, kCurved}) {
      Block b;
      b.kind = kind;
      for (std::size_t e = 0; e < dom.leaves.size(); ++e) {
        const idx leaf = dom.leaves[e];
        if (geom_.kind[leaf] != kind) continue;
        b.elements.push_back(static_cast<idx>(e));
        const std::size_t p0 = static_cast<std::size_t>(leaf) * npe;
        if (kind == kRect) {
          for (double v : {geom_.xi_x[p0], geom_.eta_z[p0], geom_.jac[p0]}) b.metric.push_back(static_cast<float>(v));
        } else if (kind == kAffine) {
          for (double v : {geom_.xi_x[p0], geom_.xi_z[p0], geom_.eta_x[p0], geom_.eta_z[p0], geom_.jac[p0]})
            b.metric.push_back(static_cast<float>(v));
        } else {
          for (std::size_t k = 0; k < npe; ++k) {
            const std::size_t p = p0 + k;
            for (double v : {geom_.xi_x[p], geom_.xi_z[p], geom_.eta_x[p], geom_.eta_z[p], geom_.jac[p]})
              b.metric.push_back(static_cast<float>(v));
          }
        }
        for (std::size_t k = 0; k < npe; ++k) {
          b.coef0.push_back(static_cast<float>(coef0[e * npe + k]));
          b.coef1.push_back(static_cast<float>(coef1[e * npe + k]));
        }
      }
      if (!b.elements.empty()) out.push_back(std::move(b));
    }
    return out;
  }

  static void face_point(int f, int q, int n, int& i, int& j) {
    switch (f) {
      case 0: i = q; j = 0; break;
      case 1: i = n; j = q; break;
      case 2: i = n - q; j = n; break;
      default: i = 0; j = n - q; break;
    }
  }

  // Quadrature weight x surface Jacobian (x r) and outward normal (solver.cpp:39-60, 338-355).
  void face_weight(idx leaf, int f, int i, int j, double& w, double& nx, double& nz) const {
    const std::size_t pt = static_cast<std::size_t>(leaf) * ngll_ * ngll_ + j * ngll_ + i;
    const double jac = geom_.jac[pt];
    double tx, tz;
    if (f == 0 || f == 2) {
      tx = geom_.eta_z[pt] * jac;
      tz = -geom_.eta_x[pt] * jac;
    } else {
      tx = -geom_.xi_z[pt] * jac;
      tz = geom_.xi_x[pt] * jac;
    }
    if (f >= 2) {
      tx = -tx;
      tz = -tz;
    }
    const double ds = std::hypot(tx, tz);
    nx = tz / ds;
    nz = -tx / ds;
    const bool along_xi = f == 0 || f == 2;
    if (!axisym_) {
      w = rule_.weights[along_xi ? i : j] * ds;
    } else if (along_xi && forest_->is_axial(leaf)) {
      const double x_xi = geom_.eta_z[pt] * geom_.jac[pt];
      const double rt = i == 0 ? x_xi : geom_.x[pt] / (1.0 + glj_.points[i]);
      w = glj_.weights[i] * ds * rt;
    } else {
      w = rule_.weights[along_xi ? i : j] * ds * std::max(geom_.x[pt], 0.0);
    }
  }

  // solver.cpp:256-336
  void build_boundaries(Domain& dom) {
    std::map<int64_t, int> face_tag;
    for (const auto& bf : macro_.boundary) face_tag[static_cast<int64_t>(bf.cell) * 4 + bf.face] = bf.tag;
    const int n = ngll_ - 1, nc = dom.ncomp;
    std::map<idx, std::array<double, 9>> absorbing;
    std::set<idx> dirichlet;
    for (std::size_t e = 0; e < dom.leaves.size(); ++e) {
      const idx leaf = dom.leaves[e];
      const Leaf& lf = forest_->leaf(leaf);
      const int last = (1 << lf.level) - 1;
      const bool on_face[4] = {lf.j == 0, lf.i == last, lf.j == last, lf.i == 0};
      const Material& mat = material_of_leaf(leaf);
      for (int f = 0; f < 4; ++f) {
        if (!on_face[f] || !macro_.is_boundary_edge(macro_.cell_edge(lf.tree, f))) continue;
        int type = dom.medium == 1 ? 0 : 1;  // natural: free (elastic), rigid (acoustic)
        const auto tag = face_tag.find(static_cast<int64_t>(lf.tree) * 4 + f);
        if (tag != face_tag.end()) {
          const auto bc = bcs_.find(tag->second);
          if (bc != bcs_.end()) type = bc->second;
          REQUIRE(!(macro_.is_axis_face(lf.tree, f) && bc != bcs_.end()),
                  "boundary tag " + std::to_string(tag->second) + " is on the symmetry axis, which takes no boundary condition");
        }
        if (macro_.is_axis_face(lf.tree, f)) continue;
        const bool is_dirichlet = (dom.medium == 1 && type == 1) || (dom.medium == 0 && type == 0);
        if (type != 2 && !is_dirichlet) continue;
        for (int q = 0; q <= n; ++q) {
          int i, j;
          face_point(f, q, n, i, j);
          const idx g = dom.dofs.global_index(static_cast<idx>(e), j * ngll_ + i);
          if (is_dirichlet) {
            dirichlet.insert(g);
            continue;
          }
          double w, nx, nz;
          face_weight(leaf, f, i, j, w, nx, nz);
          auto& acc = absorbing.try_emplace(g, std::array<double, 9>{}).first->second;
          if (dom.medium == 0) {
            acc[0] += w / (mat.rho * mat.vp);
            continue;
          }
          const double a = w * mat.rho * mat.vp, b = w * mat.rho * mat.vs;
          const double cxx = a * nx * nx + b * (1.0 - nx * nx);
          const double czz = a * nz * nz + b * (1.0 - nz * nz);
          const double cxz = (a - b) * nx * nz;
          if (nc == 2) {
            acc[0] += cxx;
            acc[1] += cxz;
            acc[2] += cxz;
            acc[3] += czz;
          } else {
            const double ct = w * mat.rho * mat.vs;
            const double cpp = 0.5 * (cxx + ct), cpm = 0.5 * (cxx - ct), cpz = kSqrtHalf * cxz;
            const double c[9] = {cpp, cpm, cpz, cpm, cpp, cpz, cpz, cpz, czz};
            for (int s = 0; s < 9; ++s) acc[s] += c[s];
          }
        }
      }
    }
    const std::set<idx> axis(dom.axis_points.begin(), dom.axis_points.end());
    for (auto [g, c] : absorbing) {
      if (dirichlet.count(g)) continue;
      if (axis.count(g))
        for (idx ac : dom.axis_components)
          for (int s = 0; s < nc; ++s) c[ac * nc + s] = c[s * nc + ac] = 0.0;
      dom.absorbing_points.push_back(g);
      for (int s = 0; s < nc * nc; ++s) dom.absorbing_coef.push_back(static_cast<float>(c[s]));
    }
    dom.dirichlet_points.assign(dirichlet.begin(), dirichlet.end());
  }

  int domain_index(int medium) const {
    for (std::size_t i = 0; i < domains_.size(); ++i)
      if (domains_[i].medium == medium) return static_cast<int>(i);
    return -1;
  }

  // solver.cpp:357-418
  void build_coupling() {
    const int fi = domain_index(0), si = domain_index(1);
    if (fi < 0 || si < 0) return;
    const Domain& fluid = domains_[fi];
    const Domain& solid = domains_[si];
    const int n = ngll_ - 1;
    auto edge_key = [](idx a, idx b) {
      return (static_cast<uint64_t>(std::min(a, b)) << 32) | static_cast<uint32_t>(std::max(a, b));
    };
    std::unordered_map<uint64_t, std::pair<idx, int>> solid_faces;
    solid_faces.reserve(4 * solid.leaves.size());
    for (std::size_t e = 0; e < solid.leaves.size(); ++e) {
      const idx* v = &corners_[4 * static_cast<std::size_t>(solid.leaves[e])];
      for (int f = 0; f < 4; ++f)
        solid_faces[edge_key(v[kFaceCorners[f][0]], v[kFaceCorners[f][1]])] = {static_cast<idx>(e), f};
    }
    struct Entry {
      idx solid_point;
      double cx, cz;
    };
    std::map<idx, Entry> entries;
    for (std::size_t e = 0; e < fluid.leaves.size(); ++e) {
      const idx leaf = fluid.leaves[e];
      const idx* v = &corners_[4 * static_cast<std::size_t>(leaf)];
      for (int f = 0; f < 4; ++f) {
        const idx a = v[kFaceCorners[f][0]], b = v[kFaceCorners[f][1]];
        const auto it = solid_faces.find(edge_key(a, b));
        if (it == solid_faces.end()) continue;
        const auto [es, fs] = it->second;
        const idx* vs = &corners_[4 * static_cast<std::size_t>(solid.leaves[es])];
        const bool sfwd = vs[kFaceCorners[fs][0]] < vs[kFaceCorners[fs][1]];
        for (int q = 0; q <= n; ++q) {
          int i, j, is, js;
          face_point(f, q, n, i, j);
          const int pos = a < b ? q : n - q;
          face_point(fs, sfwd ? pos : n - pos, n, is, js);
          const idx gf = fluid.dofs.global_index(static_cast<idx>(e), j * ngll_ + i);
          const idx gs = solid.dofs.global_index(es, js * ngll_ + is);
          double w, nx, nz;
          face_weight(leaf, f, i, j, w, nx, nz);
          auto [en, ins] = entries.try_emplace(gf, Entry{gs, 0.0, 0.0});
          REQUIRE(en->second.solid_point == gs, "inconsistent fluid-solid interface point");
          en->second.cx += w * nx;
          en->second.cz += w * nz;
        }
      }
    }
    for (const auto& [gf, en] : entries) {
      cpl_fluid_.push_back(gf);
      cpl_solid_.push_back(en.solid_point);
      cpl_cx_.push_back(static_cast<float>(en.cx));
      cpl_cz_.push_back(static_cast<float>(en.cz));
    }
  }

  // Spatial index of leaf bounding boxes (padded like locate.cpp) over a
  // uniform grid; candidates are tested in ascending leaf order so the first
  // containing leaf is the one the reference's linear scan finds.
  struct LeafGrid {
    double x0 = 0, z0 = 0, hx = 1, hz = 1;
    int nx = 1, nz = 1;
    std::vector<std::vector<idx>> cells;
  };
  LeafGrid make_grid(const std::vector<idx>& leaves) const {
    LeafGrid g;
    const std::size_t npe = static_cast<std::size_t>(ngll_) * ngll_;
    double X0 = 1e300, X1 = -1e300, Z0 = 1e300, Z1 = -1e300;
    std::vector<std::array<double, 4>> boxes(leaves.size());
    for (std::size_t q = 0; q < leaves.size(); ++q) {
      const std::size_t p0 = static_cast<std::size_t>(leaves[q]) * npe;
      const auto [xa, xb] = std::minmax_element(geom_.x.begin() + p0, geom_.x.begin() + p0 + npe);
      const auto [za, zb] = std::minmax_element(geom_.z.begin() + p0, geom_.z.begin() + p0 + npe);
      const double pad = 0.25 * std::max(*xb - *xa, *zb - *za);
      boxes[q] = {*xa - pad, *xb + pad, *za - pad, *zb + pad};
      X0 = std::min(X0, boxes[q][0]);
      X1 = std::max(X1, boxes[q][1]);
      Z0 = std::min(Z0, boxes[q][2]);
      Z1 = std::max(Z1, boxes[q][3]);
    }
    const int side = std::max(1, static_cast<int>(std::sqrt(static_cast<double>(leaves.size()))));
    g.nx = g.nz = side;
    g.x0 = X0;
    g.z0 = Z0;
    g.hx = std::max((X1 - X0) / side, 1e-300);
    g.hz = std::max((Z1 - Z0) / side, 1e-300);
    g.cells.assign(static_cast<std::size_t>(side) * side, {});
    for (std::size_t q = 0; q < leaves.size(); ++q) {
      const int i0 = std::clamp(static_cast<int>((boxes[q][0] - g.x0) / g.hx), 0, side - 1);
      const int i1 = std::clamp(static_cast<int>((boxes[q][1] - g.x0) / g.hx), 0, side - 1);
      const int j0 = std::clamp(static_cast<int>((boxes[q][2] - g.z0) / g.hz), 0, side - 1);
      const int j1 = std::clamp(static_cast<int>((boxes[q][3] - g.z0) / g.hz), 0, side - 1);
      for (int j = j0; j <= j1; ++j)
        for (int i = i0; i <= i1; ++i) g.cells[static_cast<std::size_t>(j) * side + i].push_back(static_cast<idx>(q));
    }
    return g;
  }

  struct Location {
    idx leaf = -1;
    double xi = 0, eta = 0;
  };

  // locate.cpp:7-48 over the candidates of the grid cell containing x.
  Location locate(const std::array<double, 2>& x, int di) {
    const Domain& dom = domains_[di];
    auto it = grids_.find(di);
    if (it == grids_.end()) it = grids_.emplace(di, make_grid(dom.leaves)).first;
    const LeafGrid& g = it->second;
    const std::size_t npe = static_cast<std::size_t>(ngll_) * ngll_;
    const int i = static_cast<int>(std::floor((x[0] - g.x0) / g.hx)), j = static_cast<int>(std::floor((x[1] - g.z0) / g.hz));
    if (i < 0 || j < 0 || i >= g.nx || j >= g.nz) {
      // outside every padded box unless the point sits on the grid's upper edge
      if (!(i == g.nx && j >= 0 && j < g.nz) && !(j == g.nz && i >= 0 && i <= g.nx)) return {};
    }
    const int ci = std::min(i, g.nx - 1), cj = std::min(j, g.nz - 1);
    std::vector<idx> cand = g.cells[static_cast<std::size_t>(cj) * g.nx + ci];
    std::sort(cand.begin(), cand.end());
    for (idx q : cand) {
      const idx leaf = dom.leaves[q];
      const std::size_t p0 = static_cast<std::size_t>(leaf) * npe;
      const auto [xa, xb] = std::minmax_element(geom_.x.begin() + p0, geom_.x.begin() + p0 + npe);
      const auto [za, zb] = std::minmax_element(geom_.z.begin() + p0, geom_.z.begin() + p0 + npe);
      const double pad = 0.25 * std::max(*xb - *xa, *zb - *za);
      if (x[0] < *xa - pad || x[0] > *xb + pad || x[1] < *za - pad || x[1] > *zb + pad) continue;
      double xi = 0.0, eta = 0.0;
      bool converged = false;
      for (int itn = 0; itn < 30; ++itn) {
        const auto y = forest_->leaf_map(leaf, xi, eta);
        const auto jm = forest_->leaf_jacobian(leaf, xi, eta);
        const double rx = y[0] - x[0], rz = y[1] - x[1];
        const double det = jm[0] * jm[3] - jm[1] * jm[2];
        const double dxi = (jm[3] * rx - jm[1] * rz) / det;
        const double deta = (-jm[2] * rx + jm[0] * rz) / det;
        xi = std::clamp(xi - dxi, -2.0, 2.0);
        eta = std::clamp(eta - deta, -2.0, 2.0);
        if (std::abs(dxi) + std::abs(deta) < 1e-12) {
          converged = true;
          break;
        }
      }
      constexpr double kTol = 1e-9;
      if (converged && std::abs(xi) <= 1.0 + kTol && std::abs(eta) <= 1.0 + kTol)
        return {leaf, std::clamp(xi, -1.0, 1.0), std::clamp(eta, -1.0, 1.0)};
    }
    return {};
  }

  struct Weights {
    std::vector<double> value, d_dx, d_dz;
  };
  Weights point_weights(const Location& loc) const {
    const bool axial = axisym_ && forest_->is_axial(loc.leaf);
    const Lagrange bx(axial ? glj_.points : rule_.points), by(rule_.points);
    const int n = bx.size();
    const auto lx = bx.values(loc.xi), ly = by.values(loc.eta), dlx = bx.derivatives(loc.xi), dly = by.derivatives(loc.eta);
    const auto j = forest_->leaf_jacobian(loc.leaf, loc.xi, loc.eta);
    const double det = j[0] * j[3] - j[1] * j[2];
    const double xi_x = j[3] / det, xi_z = -j[1] / det, eta_x = -j[2] / det, eta_z = j[0] / det;
    Weights w;
    w.value.resize(static_cast<std::size_t>(n) * n);
    w.d_dx.resize(w.value.size());
    w.d_dz.resize(w.value.size());
    for (int jj = 0; jj < n; ++jj)
      for (int ii = 0; ii < n; ++ii) {
        const std::size_t k = static_cast<std::size_t>(jj) * n + ii;
        const double d_xi = dlx[ii] * ly[jj], d_eta = lx[ii] * dly[jj];
        w.value[k] = lx[ii] * ly[jj];
        w.d_dx[k] = d_xi * xi_x + d_eta * eta_x;
        w.d_dz[k] = d_xi * xi_z + d_eta * eta_z;
      }
    return w;
  }

  // solver.cpp:427-520
  void build_sources() {
    for (int si = 0; si < d_.n_sources; ++si) {
      const int kind = d_.source_kind[si];
      const int medium = (kind == 2 || kind == 3) ? 0 : 1;
      const int di = domain_index(medium);
      REQUIRE(di >= 0, "source " + std::to_string(si) + " needs a medium the model does not have");
      const Domain& dom = domains_[di];
      const std::array<double, 2> pos{d_.source_position[2 * si], d_.source_position[2 * si + 1]};
      const Location loc = locate(pos, di);
      REQUIRE(loc.leaf >= 0, "source " + std::to_string(si) + " is not inside its medium");
      const Weights w = point_weights(loc);
      const idx e = dom.element_of_leaf[loc.leaf];
      const int npe = ngll_ * ngll_;
      const double scale = !axisym_ ? 1.0 : m_ == 1 ? 1.0 / kPi : 1.0 / (2.0 * kPi);
      const double rs = pos[0];
      const double* c = d_.source_components + 3 * si;
      const bool directional = kind == 0 || kind == 3;
      if (axisym_) {
        const bool on_axis = std::abs(rs) <= 1e-12 * (1.0 + std::abs(pos[1]));
        if (m_ == 0) {
          REQUIRE(!(on_axis && directional && c[0] != 0.0), "a radial force or dipole on the axis is not axisymmetric");
          REQUIRE(!(on_axis && kind == 1 && c[2] != 0.0), "an M_rz moment on the axis is not axisymmetric");
        } else {
          REQUIRE(directional, "azimuthal order 1 takes force and dipole sources only");
          REQUIRE(!(on_axis && c[1] != 0.0), "a vertical force or dipole on the axis is axisymmetric");
        }
      }
      const double rho = material_of_leaf(loc.leaf).rho;
      const bool pm = dom.medium == 1 && dom.m == 1;
      std::map<idx, std::array<double, 3>> acc;
      for (int k = 0; k < npe; ++k) {
        double fc[3] = {0.0, 0.0, 0.0};
        switch (kind) {
          case 0:
            if (pm) {
              fc[0] = fc[1] = kSqrtHalf * c[0] * w.value[k];
              fc[2] = c[1] * w.value[k];
            } else {
              fc[0] = c[0] * w.value[k];
              fc[1] = c[1] * w.value[k];
            }
            break;
          case 1:
            fc[0] = c[0] * w.d_dx[k] + c[2] * w.d_dz[k];
            fc[1] = c[2] * w.d_dx[k] + c[1] * w.d_dz[k];
            if (axisym_) fc[0] += c[0] * (rs > 0.0 ? w.value[k] / rs : w.d_dx[k]);
            break;
          case 2:
            fc[0] = w.value[k];
            break;
          case 3:
            fc[0] = (c[0] * w.d_dx[k] + c[1] * w.d_dz[k]) / rho;
            break;
        }
        for (const auto& [g, wt] : dom.dofs.slot_entries(e, k)) {
          auto& a = acc.try_emplace(g, std::array<double, 3>{}).first->second;
          for (int comp = 0; comp < dom.ncomp; ++comp) a[comp] += wt * fc[comp] * scale;
        }
      }
      SourceTerm t;
      t.domain = di;
      t.stf_kind = d_.stf_kind[si];
      t.f0 = d_.stf_params[3 * si];
      t.t0 = d_.stf_params[3 * si + 1];
      t.amp = d_.stf_params[3 * si + 2];
      for (const auto& [g, f] : acc) t.points.push_back(g);
      t.coef.resize(static_cast<std::size_t>(dom.ncomp) * acc.size());
      std::size_t i = 0;
      for (const auto& [g, f] : acc) {
        for (int comp = 0; comp < dom.ncomp; ++comp) t.coef[comp * acc.size() + i] = static_cast<float>(f[comp]);
        ++i;
      }
      sources_.push_back(std::move(t));
    }
  }

  // solver.cpp:522-568
  void build_receivers() {
    for (int ri = 0; ri < d_.n_receivers; ++ri) {
      const std::array<double, 2> pos{d_.receiver_position[2 * ri], d_.receiver_position[2 * ri + 1]};
      Location loc;
      int di = -1;
      for (std::size_t q = 0; q < domains_.size() && loc.leaf < 0; ++q) {
        if (d_.receiver_medium[ri] >= 0 && domains_[q].medium != d_.receiver_medium[ri]) continue;
        loc = locate(pos, static_cast<int>(q));
        if (loc.leaf >= 0) di = static_cast<int>(q);
      }
      REQUIRE(loc.leaf >= 0, "receiver " + std::to_string(ri) + " is outside the model");
      const Domain& dom = domains_[di];
      const Weights w = point_weights(loc);
      const idx e = dom.element_of_leaf[loc.leaf];
      std::map<idx, std::array<double, 3>> acc;
      for (int k = 0; k < ngll_ * ngll_; ++k)
        for (const auto& [g, wt] : dom.dofs.slot_entries(e, k)) {
          auto& a = acc.try_emplace(g, std::array<double, 3>{}).first->second;
          a[0] += wt * w.value[k];
          a[1] += wt * w.d_dx[k];
          a[2] += wt * w.d_dz[k];
        }
      ReceiverTerm t;
      t.domain = di;
      for (const auto& [g, c] : acc) {
        t.points.push_back(g);
        t.value.push_back(static_cast<float>(c[0]));
        t.d_dx.push_back(static_cast<float>(c[1]));
        t.d_dz.push_back(static_cast<float>(c[2]));
      }
      t.rho = material_of_leaf(loc.leaf).rho;
      for (int q = d_.receiver_qoffsets[ri]; q < d_.receiver_qoffsets[ri + 1]; ++q) {
        const int quantity = d_.receiver_quantities[q];
        const bool elastic_q = quantity <= 2;
        REQUIRE(elastic_q == (dom.medium == 1) && (elastic_q || quantity == 3 || quantity == 4),
                "receiver " + std::to_string(ri) + " records a quantity its medium does not have");
        t.quantities.push_back(quantity);
      }
      REQUIRE(!t.quantities.empty(), "receiver records no quantities");
      receivers_.push_back(std::move(t));
    }
  }

  Output pack() {
    Output o;
    const std::string P = "problem.";
    const Lagrange basis(rule_.points);
    const auto D = basis.derivative_matrix();
    const auto Dj = Lagrange(glj_.points).derivative_matrix();
    std::vector<float> w2(static_cast<std::size_t>(ngll_) * ngll_);
    for (int j = 0; j < ngll_; ++j)
      for (int i = 0; i < ngll_; ++i) w2[j * ngll_ + i] = static_cast<float>(rule_.weights[i] * rule_.weights[j]);
    o.scalar_i(P + "basis.ngll", ngll_);
    o.f32(P + "basis.D", std::vector<float>(D.begin(), D.end()));
    o.f32(P + "basis.Dj", std::vector<float>(Dj.begin(), Dj.end()));
    o.f32(P + "basis.w2", std::move(w2));
    o.f64("gll.points", rule_.points);
    o.f64("gll.weights", rule_.weights);
    o.scalar_i(P + "axisym", axisym_ ? 1 : 0);
    o.scalar_i(P + "azimuthal_order", m_);
    o.scalar_i(P + "record_every", d_.record_every);
    o.scalar_i(P + "energy_every", d_.energy_every);
    o.scalar_i(P + "domains.count", static_cast<int64_t>(domains_.size()));
    for (std::size_t di = 0; di < domains_.size(); ++di) {
      Domain& d = domains_[di];
      const std::string p = P + "domains." + std::to_string(di) + ".";
      o.scalar_i(p + "medium", d.medium);
      o.scalar_i(p + "ncomp", d.ncomp);
      o.scalar_i(p + "azimuthal_order", d.m);
      o.scalar_i(p + "n_global", d.dofs.n_global);
      o.scalar_i(p + "n_elements", d.dofs.n_elem);
      o.i32(p + "l2g", std::move(d.dofs.l2g));
      o.i32(p + "row_offsets", std::move(d.dofs.row_offsets));
      o.i32(p + "row_dofs", std::move(d.dofs.row_dofs));
      o.f64(p + "row_weights", std::move(d.dofs.row_weights));
      o.i32(p + "t_offsets", std::move(d.dofs.t_offsets));
      o.i32(p + "t_slots", std::move(d.dofs.t_slots));
      o.f64(p + "t_weights", std::move(d.dofs.t_weights));
      o.f32(p + "mass", std::move(d.mass));
      o.f32(p + "inv_mass", std::move(d.inv_mass));
      o.i32(p + "absorbing_points", std::move(d.absorbing_points));
      o.f32(p + "absorbing_coef", std::move(d.absorbing_coef));
      o.i32(p + "dirichlet_points", std::move(d.dirichlet_points));
      o.i32(p + "axis_points", std::move(d.axis_points));
      o.i32(p + "axis_components", std::move(d.axis_components));
      o.f64(p + "coords", std::move(d.coords));
      o.scalar_i(p + "blocks.count", static_cast<int64_t>(d.blocks.size()));
      for (std::size_t bi = 0; bi < d.blocks.size(); ++bi) {
        Block& b = d.blocks[bi];
        const std::string q = p + "blocks." + std::to_string(bi) + ".";
        o.scalar_i(q + "kind", b.kind);
        o.scalar_i(q + "azimuthal_order", b.m);
        o.i32(q + "elements", std::move(b.elements));
        o.f32(q + "metric", std::move(b.metric));
        o.f32(q + "coef0", std::move(b.coef0));
        o.f32(q + "coef1", std::move(b.coef1));
        o.f32(q + "wr", std::move(b.wr));
        o.f32(q + "hoop", std::move(b.hoop));
        o.f32(q + "r", std::move(b.r));
        o.u8(q + "axial", std::move(b.axial));
      }
    }
    o.i32(P + "coupling.fluid_points", std::move(cpl_fluid_));
    o.i32(P + "coupling.solid_points", std::move(cpl_solid_));
    o.f32(P + "coupling.cx", std::move(cpl_cx_));
    o.f32(P + "coupling.cz", std::move(cpl_cz_));
    o.scalar_i(P + "sources.count", static_cast<int64_t>(sources_.size()));
    for (std::size_t si = 0; si < sources_.size(); ++si) {
      SourceTerm& s = sources_[si];
      const std::string p = P + "sources." + std::to_string(si) + ".";
      o.scalar_i(p + "domain", s.domain);
      o.i32(p + "points", std::move(s.points));
      o.f32(p + "coef", std::move(s.coef));
      o.scalar_i(p + "stf.kind", s.stf_kind);
      o.scalar_d(p + "stf.f0", s.f0);
      o.scalar_d(p + "stf.t0", s.t0);
      o.scalar_d(p + "stf.amplitude", s.amp);
    }
    o.scalar_i(P + "receivers.count", static_cast<int64_t>(receivers_.size()));
    for (std::size_t ri = 0; ri < receivers_.size(); ++ri) {
      ReceiverTerm& r = receivers_[ri];
      const std::string p = P + "receivers." + std::to_string(ri) + ".";
      o.scalar_i(p + "domain", r.domain);
      o.i32(p + "points", std::move(r.points));
      o.f32(p + "value", std::move(r.value));
      o.f32(p + "d_dx", std::move(r.d_dx));
      o.f32(p + "d_dz", std::move(r.d_dz));
      o.scalar_d(p + "rho", r.rho);
      o.i32(p + "quantities", std::move(r.quantities));
    }
    std::vector<uint8_t> kinds(geom_.kind.begin(), geom_.kind.end());
    o.u8("geometry.kind", std::move(kinds));
    o.finish();
    return o;
  }

  const insem_case_desc& d_;
  Macro macro_;
  std::map<int, Material> mats_;
  std::map<int, int> bcs_;
  int ngll_ = 0, m_ = 0;
  bool axisym_ = false;
  Rule rule_, glj_;
  std::unique_ptr<Forest> forest_;
  Geometry geom_;
  std::vector<idx> corners_;
  idx n_vertices_ = 0;
  std::vector<Domain> domains_;
  std::vector<idx> cpl_fluid_, cpl_solid_;
  std::vector<float> cpl_cx_, cpl_cz_;
  std::vector<SourceTerm> sources_;
  std::vector<ReceiverTerm> receivers_;
  std::map<int, LeafGrid> grids_;
};

}  // namespace

struct insem_case_out {
  Output o;
};

extern "C" {

int insem_case_build(const insem_case_desc* desc, insem_case_out** out) {
  try {
    if (!desc || !out) throw Fail("null argument");
    Builder b(*desc);
    auto h = std::make_unique<insem_case_out>();
    h->o = b.run();
    h->o.finish();
    *out = h.release();
    g_error.clear();
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

int32_t insem_case_n_arrays(const insem_case_out* out) { return out ? static_cast<int32_t>(out->o.arrays.size()) : 0; }

const insem_case_array* insem_case_array_at(const insem_case_out* out, int32_t i) {
  if (!out || i < 0 || i >= static_cast<int32_t>(out->o.arrays.size())) return nullptr;
  return &out->o.arrays[i];
}

void insem_case_free(insem_case_out* out) { delete out; }

const char* insem_case_last_error(void) { return g_error.c_str(); }

}  // extern "C"
