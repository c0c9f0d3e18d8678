// Macro mesh, linear quadtree forest and element geometry of the native case
// setup.
//
// The forest is stored as one Morton-ordered list of quadrants per macro
// cell (a linear quadtree): a point is located by a binary search over the
// Morton keys of the quadrants' lower-left corners.  Elements are the
// quadrants in (macro cell, Morton) order, the order the reference's
// numbering walks (cpp/include/insem/mesh/forest.hpp:35-40), and refinement
// keeps that order because a quadrant's four children take its place in
// Morton order.
#pragma once

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace insem_setup {

using i32 = int32_t;

struct SetupError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

[[noreturn]] inline void fail(const std::string& what) { throw SetupError(what); }
inline void expect(bool ok, const char* what) {
  if (!ok) fail(what);
}
// Checks whose message is formatted: the message is built only on failure.
template <class Message>
inline void expect(bool ok, Message&& message) {
  if (!ok) fail(message());
}

// Corners of local face f, counter-clockwise: face 0 is eta = -1, 1 is
// xi = +1, 2 is eta = +1, 3 is xi = -1.
constexpr int kSideCorner[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};

// ------------------------------------------------------------- macro mesh
struct TaggedSide {
  i32 cell;
  int side;
  int tag;
};

class MacroGrid {
 public:
  MacroGrid(bool quad9, bool axisym, std::vector<double> xy, std::vector<i32> conn, std::vector<i32> region,
            std::vector<TaggedSide> tagged);

  bool quad9() const { return quad9_; }
  bool axisymmetric() const { return axisym_; }
  int nodes_per_cell() const { return quad9_ ? 9 : 4; }
  i32 n_cells() const { return static_cast<i32>(region_.size()); }
  i32 node_of(i32 c, int k) const { return conn_[static_cast<std::size_t>(c) * nodes_per_cell() + k]; }
  int region(i32 c) const { return region_[c]; }
  const std::vector<TaggedSide>& tagged() const { return tagged_; }

  // Macro edge of side f of cell c; whether the side's counter-clockwise
  // direction runs from the edge's lower to its higher node; the cell across.
  i32 edge(i32 c, int f) const { return side_edge_[4 * c + f]; }
  bool same_sense(i32 c, int f) const { return side_sense_[4 * c + f] != 0; }
  i32 across(i32 c, int f) const;
  bool exterior(i32 c, int f) const { return across(c, f) < 0; }
  // Local side of cell c that lies on macro edge e.
  int side_on(i32 c, i32 e) const;

  // Axisymmetric meshes: side f of c lies on r = 0.  Cells with such a side
  // are renumbered at construction so that it is side 3 (xi = -1), where
  // axial elements carry their GLJ points.
  bool axis_side(i32 c, int f) const { return (axis_mask_[c] >> f) & 1; }
  bool on_axis(i32 c) const { return axis_side(c, 3); }

  // Isoparametric map of cell c and its Jacobian {x_xi, x_eta, z_xi, z_eta}.
  std::array<double, 2> point(i32 c, double xi, double eta) const;
  std::array<double, 4> jacobian(i32 c, double xi, double eta) const;
  // Both from one evaluation of the shape functions (same values as the two calls).
  void point_and_jacobian(i32 c, double xi, double eta, std::array<double, 2>& x, std::array<double, 4>& j) const;

 private:
  bool side_touches_axis(i32 c, int f) const;
  void turn_axis_sides_to_three();
  void connect();
  void check() const;

  bool quad9_, axisym_;
  std::vector<double> xy_;
  std::vector<i32> conn_;
  std::vector<i32> region_;
  std::vector<TaggedSide> tagged_;
  std::vector<i32> side_edge_;
  std::vector<uint8_t> side_sense_;
  std::vector<std::array<i32, 2>> edge_cells_;
  std::vector<uint8_t> axis_mask_;
};

// ----------------------------------------------------------------- forest
constexpr int kDeepest = 20;  // finest quadrant level; lattice 2^20 per cell side

struct Quadrant {
  i32 cell;
  int level;
  i32 i, j;  // position among the 2^level x 2^level quadrants of the cell
};

struct Neighbour {
  i32 quad = -1;   // -1: the side lies on the domain boundary
  int side = -1;   // the neighbour's side that touches ours
  int jump = 0;    // neighbour level - our level
};

class QuadForest {
 public:
  QuadForest(const MacroGrid* grid, int level);
  QuadForest(const MacroGrid* grid, std::vector<Quadrant> quads);

  const MacroGrid& grid() const { return *grid_; }
  i32 size() const { return static_cast<i32>(quads_.size()); }
  const Quadrant& operator[](i32 q) const { return quads_[q]; }

  // Reference sub-square of quadrant q inside its cell: {xi0, xi1, eta0, eta1}.
  std::array<double, 4> box(i32 q) const;
  bool axial(i32 q) const { return quads_[q].i == 0 && grid_->on_axis(quads_[q].cell); }

  // The quadrant containing lattice point (a, b) of a cell, in half-lattice
  // units (a 2^21 grid per side; cells half-open), or -1.
  i32 locate(i32 cell, int64_t a, int64_t b) const;
  Neighbour neighbour(i32 q, int f) const;

  // Maps t in [-1, 1] along side f of quadrant `from` to the coordinate
  // along side g of quadrant `to` (the same physical point of a shared side).
  double side_coordinate(i32 from, int f, double t, i32 to, int g) const;

  // Quadrants with flag[q] set split into four.
  QuadForest split(const std::vector<char>& flag) const;
  // 2:1 across every side, and equal levels across sides of cells for which
  // `same_level(cell_a, cell_b)` holds.
  template <class SameLevel>
  QuadForest balanced(SameLevel same_level) const;

  // Corner vertices shared across quadrants and cells: vertex[4 q + k] is
  // corner k (counter-clockwise from (-1, -1)) of quadrant q; ids in
  // first-touch order over (quadrant, corner).
  std::vector<i32> corner_vertices(i32* n_vertices) const;

 private:
  void index();

  const MacroGrid* grid_;
  std::vector<Quadrant> quads_;
  std::vector<i32> first_;     // per cell: first quadrant
  std::vector<uint64_t> key_;  // Morton key of each quadrant's lower-left corner at kDeepest
};

template <class SameLevel>
QuadForest QuadForest::balanced(SameLevel same_level) const {
  QuadForest f = *this;
  for (;;) {
    std::vector<char> flag(f.size(), 0);
    bool any = false;
    for (i32 q = 0; q < f.size(); ++q) {
      for (int s = 0; s < 4; ++s) {
        const Neighbour nb = f.neighbour(q, s);
        if (nb.quad < 0 || nb.jump >= 0) continue;
        const i32 cq = f[q].cell, cn = f[nb.quad].cell;
        if (nb.jump < -1 || (cq != cn && same_level(cq, cn))) {
          flag[nb.quad] = 1;
          any = true;
        }
      }
    }
    if (!any) return f;
    f = f.split(flag);
  }
}

// --------------------------------------------------------------- geometry
enum ElementShape : uint8_t { kRect = 0, kAffine = 1, kCurved = 2 };

// Per element point (element-major, then j * ngll + i): physical position
// and inverse metric, plus each element's shape class.
struct PointGeometry {
  int ngll = 0;
  std::vector<double> x, z, xi_x, xi_z, eta_x, eta_z, jac;
  std::vector<uint8_t> shape;
};

// Axial elements use `ref_axial` along xi (GLJ points), all others `ref`.
PointGeometry element_geometry(const QuadForest& f, const std::vector<double>& ref,
                               const std::vector<double>& ref_axial);

// Map and Jacobian of quadrant q from its own reference square.
std::array<double, 2> quad_point(const QuadForest& f, i32 q, double xi, double eta);
std::array<double, 4> quad_jacobian(const QuadForest& f, i32 q, double xi, double eta);

}  // namespace insem_setup
