// Native case setup: a model description (insem_cases.h) -> the packed
// per-step arrays of include/insem_cuda.h.
//
// Stages, each in its own function of CaseSetup:
//   refine       quadtree refinement to the wavelength and region criteria,
//                then 2:1 balance with equal levels across fluid-solid sides
//                (the reference's Simulation::build_forest,
//                cpp/src/sim/simulation.cpp:121-175);
//   media        per medium: elements, point numbering, quadrature weights
//                (GLJ on the axis), material coefficients, lumped mass,
//                element blocks (solver.cpp:147-254, element_block.cpp);
//   edges        Stacey coefficients, Dirichlet and axis points (solver.cpp:256-336);
//   interface    fluid-solid coupling weights (solver.cpp:357-418);
//   point terms  source and receiver interpolation (solver.cpp:427-568,
//                locate.cpp).
// Every number that reaches an array is computed with the reference's
// operations in the reference's order -- products left to right, sums over
// points and sides in the same sequence, std::map-ordered accumulation per
// global point -- because the backend's results are compared with the
// reference bit for bit.  Which numbers are formed is fixed by that; how the
// stages, searches and containers are organised is this library's own.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "insem_cases.h"
#include "setup_basis.hpp"
#include "setup_dofs.hpp"
#include "setup_mesh.hpp"

namespace insem_setup {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kSqrtHalf = 0.70710678118654752440;
enum Medium { kAcoustic = 0, kElastic = 1 };
enum Condition { kFree = 0, kRigid = 1, kAbsorbing = 2 };
enum SourceKind { kForce = 0, kMoment = 1, kMonopole = 2, kDipole = 3 };
enum Quantity { kDisplacement = 0, kVelocity = 1, kAcceleration = 2, kPressure = 3, kParticleVelocity = 4 };
enum BlockKind { kBlockRect = 0, kBlockAffine = 1, kBlockCurved = 2, kBlockAxisym = 3 };

thread_local std::string t_message;

std::string fmt(double v) {
  char b[32];
  std::snprintf(b, sizeof b, "%g", v);
  return b;
}

struct MaterialSpec {
  int medium = kElastic;
  double vp = 0.0, vs = 0.0, rho = 0.0;
};

// Point of an element in reference coordinates.
struct Located {
  i32 quad = -1;
  double xi = 0.0, eta = 0.0;
};

// Lagrange values and physical gradients of an element's nodal basis at a point.
struct Stencil {
  std::vector<double> value, ddx, ddz;
};

struct Block {
  int kind = kBlockRect, m = 0;
  std::vector<i32> elements;
  std::vector<float> metric, coef0, coef1, wr, hoop, r;
  std::vector<uint8_t> axial;
};

struct MediumPart {
  int medium = kElastic, ncomp = 2, m = 0;
  std::vector<i32> quads;          // element e -> forest quadrant
  std::vector<i32> element_of;     // quadrant -> element, or -1
  PointMap points;
  std::vector<Block> blocks;
  std::vector<float> mass, inv_mass;
  std::vector<i32> axis_components, axis_points, dirichlet, absorbing;
  std::vector<float> absorbing_coef;
  std::vector<double> coords;
};

struct PointSource {
  int domain = 0, stf_kind = 0;
  double f0 = 0, t0 = 0, amplitude = 1;
  std::vector<i32> points;
  std::vector<float> coef;
};

struct PointReceiver {
  int domain = 0;
  double rho = 0;
  std::vector<i32> points, quantities;
  std::vector<float> value, ddx, ddz;
};

// Flat output arrays keyed like the problem layout ("problem.domains.0.l2g").
class Packed {
 public:
  template <class T>
  void put(std::string key, std::vector<T> v, int32_t dtype) {
    auto hold = std::make_shared<std::vector<T>>(std::move(v));
    keys_.push_back(std::move(key));
    items_.push_back({nullptr, dtype, static_cast<int64_t>(hold->size()), hold->data()});
    hold_.push_back(std::move(hold));
  }
  void f32(std::string k, std::vector<float> v) { put(std::move(k), std::move(v), 0); }
  void f64(std::string k, std::vector<double> v) { put(std::move(k), std::move(v), 1); }
  void i32s(std::string k, std::vector<i32> v) { put(std::move(k), std::move(v), 2); }
  void u8(std::string k, std::vector<uint8_t> v) { put(std::move(k), std::move(v), 3); }
  void one(std::string k, int64_t v) { i32s(std::move(k), {static_cast<i32>(v)}); }
  void real(std::string k, double v) { f64(std::move(k), {v}); }
  void seal() {
    for (std::size_t i = 0; i < items_.size(); ++i) items_[i].key = keys_[i].c_str();
  }
  std::size_t size() const { return items_.size(); }
  const insem_case_array* at(std::size_t i) const { return &items_[i]; }

 private:
  std::vector<std::string> keys_;
  std::vector<insem_case_array> items_;
  std::vector<std::shared_ptr<void>> hold_;
};

class CaseSetup {
 public:
  explicit CaseSetup(const insem_case_desc& d) : in_(d) {}

  Packed run() {
    read_description();
    refine();
    geom_ = element_geometry(*forest_, gll_.x, glj_.x);
    corners_ = forest_->corner_vertices(&n_vertices_);
    for (int medium : {kAcoustic, kElastic}) media(medium);
    for (MediumPart& part : parts_) edges(part);
    interface();
    for (int s = 0; s < in_.n_sources; ++s) source(s);
    for (int r = 0; r < in_.n_receivers; ++r) receiver(r);
    return pack();
  }

 private:
  // ------------------------------------------------------------ inputs
  void read_description() {
    expect(in_.n_nodes > 0 && in_.n_cells > 0 && in_.nodes && in_.cells && in_.cell_region,
           "the model has no macro mesh");
    const int npc = in_.quad9 ? 9 : 4;
    std::vector<TaggedSide> tagged;
    for (int t = 0; t < in_.n_boundary; ++t)
      tagged.push_back({in_.boundary[3 * t], in_.boundary[3 * t + 1], in_.boundary[3 * t + 2]});
    grid_ = std::make_unique<MacroGrid>(
        in_.quad9 != 0, in_.axisymmetric != 0, std::vector<double>(in_.nodes, in_.nodes + 2 * in_.n_nodes),
        std::vector<i32>(in_.cells, in_.cells + static_cast<std::size_t>(in_.n_cells) * npc),
        std::vector<i32>(in_.cell_region, in_.cell_region + in_.n_cells), std::move(tagged));
    for (int i = 0; i < in_.n_materials; ++i)
      material_[in_.material_region[i]] =
          MaterialSpec{in_.material_medium[i], in_.material_vp[i], in_.material_vs[i], in_.material_rho[i]};
    std::set<int> used;
    for (i32 c = 0; c < grid_->n_cells(); ++c) {
      const int region = grid_->region(c);
      if (!used.insert(region).second) continue;
      const auto it = material_.find(region);
      expect(it != material_.end(), [&] { return "region " + std::to_string(region) + " has no material"; });
      const MaterialSpec& m = it->second;
      expect(m.rho > 0.0 && std::isfinite(m.rho) && m.vp > 0.0 && std::isfinite(m.vp),
             [&] {
               return "material of region " + std::to_string(region) + ": density and P velocity must be positive";
             });
      if (m.medium == kElastic)
        expect(m.vs > 0.0 && m.vp > m.vs,
               [&] { return "material of region " + std::to_string(region) + ": an elastic solid needs 0 < vs < vp"; });
    }
    for (int i = 0; i < in_.n_bc; ++i) condition_[in_.bc_tag[i]] = in_.bc_type[i];
    expect(in_.order >= 1 && in_.order <= 8,
           [&] { return "the GLL order must be 1..8, got " + std::to_string(in_.order); });
    ngll_ = in_.order + 1;
    axisym_ = grid_->axisymmetric();
    m_ = in_.azimuthal_order;
    expect(m_ == 0 || (m_ == 1 && axisym_), [&] { return "azimuthal order " + std::to_string(m_) +
                                                 " needs an axisymmetric mesh (orders 0 and 1 exist)"; });
    expect(in_.record_every >= 1 && in_.energy_every >= 0, "record_every must be >= 1 and energy_every >= 0");
    gll_ = gll_rule(ngll_);
    glj_ = glj_rule(ngll_);
    gll_basis_ = std::make_unique<Interpolant>(gll_.x);
    glj_basis_ = std::make_unique<Interpolant>(glj_.x);
  }

  const MaterialSpec& material_of(i32 quad) const { return material_.at(grid_->region((*forest_)[quad].cell)); }

  // ------------------------------------------------------------ refine
  void refine() {
    QuadForest f(grid_.get(), in_.uniform_level);
    const double ref[4][2] = {{-1.0, -1.0}, {1.0, -1.0}, {1.0, 1.0}, {-1.0, 1.0}};
    for (;;) {
      std::vector<char> split(f.size(), 0);
      bool any = false;
      for (i32 q = 0; q < f.size(); ++q) {
        if (f[q].level >= in_.max_level) continue;
        std::array<std::array<double, 2>, 4> c;
        for (int k = 0; k < 4; ++k) c[k] = quad_point(f, q, ref[k][0], ref[k][1]);
        bool go = false;
        if (in_.f_max > 0.0) {
          double longest = 0.0;
          for (int k = 0; k < 4; ++k)
            longest = std::max(longest, std::hypot(c[(k + 1) % 4][0] - c[k][0], c[(k + 1) % 4][1] - c[k][1]));
          const MaterialSpec& m = material_.at(grid_->region(f[q].cell));
          const double slowest = m.medium == kElastic ? m.vs : m.vp;
          go = longest > in_.order * (slowest / in_.f_max) / in_.points_per_wavelength;
        }
        if (!go) {
          double x0 = c[0][0], x1 = c[0][0], z0 = c[0][1], z1 = c[0][1];
          for (const auto& p : c) {
            x0 = std::min(x0, p[0]);
            x1 = std::max(x1, p[0]);
            z0 = std::min(z0, p[1]);
            z1 = std::max(z1, p[1]);
          }
          for (int r = 0; r < in_.n_regions && !go; ++r) {
            const double* b = in_.regions + 5 * r;
            go = f[q].level < static_cast<int>(b[4]) && x0 <= b[1] && x1 >= b[0] && z0 <= b[3] && z1 >= b[2];
          }
        }
        if (go) {
          split[q] = 1;
          any = true;
        }
      }
      if (!any) break;
      f = f.split(split);
    }
    // fluid and solid elements meet at equal levels (conforming interface)
    const MacroGrid& g = *grid_;
    const auto& mats = material_;
    forest_ = std::make_unique<QuadForest>(f.balanced([&g, &mats](i32 a, i32 b) {
      const auto ma = mats.find(g.region(a)), mb = mats.find(g.region(b));
      return ma != mats.end() && mb != mats.end() && ma->second.medium != mb->second.medium;
    }));
  }

  // ------------------------------------------------------------- media
  void media(int medium) {
    MediumPart d;
    d.medium = medium;
    d.m = m_;
    d.ncomp = medium == kElastic ? (m_ == 1 ? 3 : 2) : 1;
    if (axisym_) {
      if (medium == kElastic) d.axis_components = m_ == 1 ? std::vector<i32>{0, 2} : std::vector<i32>{0};
      else if (m_ == 1) d.axis_components = {0};
    }
    d.element_of.assign(forest_->size(), -1);
    for (i32 q = 0; q < forest_->size(); ++q) {
      if (material_of(q).medium != medium) continue;
      d.element_of[q] = static_cast<i32>(d.quads.size());
      d.quads.push_back(q);
    }
    if (d.quads.empty()) return;
    d.points = number_points(*forest_, ngll_, d.quads, corners_, n_vertices_, *gll_basis_, *glj_basis_);

    const std::size_t npe = static_cast<std::size_t>(ngll_) * ngll_;
    const std::size_t nl = d.quads.size() * npe;
    // quadrature weight per point: w_i w_j J, times r on axisymmetric meshes
    // (GLJ along xi on the axis, where the integrand r / (1 + xi) -> dr/dxi)
    std::vector<double> wr(nl), hoop(nl, 0.0);
    std::vector<uint8_t> axial(d.quads.size(), 0);
    for (std::size_t e = 0; e < d.quads.size(); ++e) {
      const i32 q = d.quads[e];
      axial[e] = axisym_ && forest_->axial(q) ? 1 : 0;
      for (std::size_t k = 0; k < npe; ++k) {
        const int i = static_cast<int>(k % ngll_), j = static_cast<int>(k / ngll_);
        const std::size_t pt = static_cast<std::size_t>(q) * npe + k, at = e * npe + k;
        const double jac = geom_.jac[pt];
        if (!axisym_) {
          wr[at] = gll_.w[i] * gll_.w[j] * jac;
        } else if (!axial[e]) {
          hoop[at] = gll_.w[i] * gll_.w[j] * jac;
          wr[at] = hoop[at] * std::max(geom_.x[pt], 0.0);
        } else {
          const double dr_dxi = geom_.eta_z[pt] * jac;
          const double radius_factor = i == 0 ? dr_dxi : geom_.x[pt] / (1.0 + glj_.x[i]);
          wr[at] = glj_.w[i] * gll_.w[j] * jac * radius_factor;
          hoop[at] = i == 0 ? 0.0 : wr[at] / geom_.x[pt];
        }
      }
    }
    std::vector<double> coef0(nl), coef1(nl), lumped(nl);
    for (std::size_t e = 0; e < d.quads.size(); ++e) {
      const MaterialSpec& m = material_of(d.quads[e]);
      for (std::size_t k = 0; k < npe; ++k) {
        const std::size_t at = e * npe + k;
        if (medium == kElastic) {
          coef0[at] = m.rho * (m.vp * m.vp - 2.0 * m.vs * m.vs);  // lambda
          coef1[at] = m.rho * m.vs * m.vs;                        // mu
          lumped[at] = wr[at] * m.rho;
        } else {
          coef0[at] = 1.0 / m.rho;
          coef1[at] = 0.0;
          lumped[at] = wr[at] / (m.rho * m.vp * m.vp);
        }
      }
    }
    if (axisym_) d.blocks.push_back(axisym_block(d, coef0, coef1, wr, hoop, axial));
    else cartesian_blocks(d, coef0, coef1);

    // lumped mass: the element masses summed per global point in slot order
    const PointMap& pm = d.points;
    d.mass.resize(pm.n_global);
    d.inv_mass.resize(pm.n_global);
    const bool weighted = !pm.t_weight.empty();
    for (i32 g = 0; g < pm.n_global; ++g) {
      double sum = 0.0;
      for (i32 s = pm.t_start[g]; s < pm.t_start[g + 1]; ++s)
        sum += weighted ? pm.t_weight[s] * lumped[pm.t_slot[s]] : lumped[pm.t_slot[s]];
      expect(sum > 0.0, "a global point has no positive mass (degenerate element?)");
      d.mass[g] = static_cast<float>(sum);
      d.inv_mass[g] = static_cast<float>(1.0 / sum);
    }
    const std::size_t ng = static_cast<std::size_t>(pm.n_global);
    d.coords.resize(2 * ng);
    for (std::size_t g = 0; g < ng; ++g) {
      const std::size_t s = static_cast<std::size_t>(pm.first_slot[g]);
      const std::size_t pt = static_cast<std::size_t>(d.quads[s / npe]) * npe + s % npe;
      d.coords[g] = geom_.x[pt];
      d.coords[ng + g] = geom_.z[pt];
      if (!d.axis_components.empty() && geom_.x[pt] <= 0.0) d.axis_points.push_back(static_cast<i32>(g));
    }
    parts_.push_back(std::move(d));
  }

  Block axisym_block(const MediumPart& d, const std::vector<double>& coef0, const std::vector<double>& coef1,
                     const std::vector<double>& wr, const std::vector<double>& hoop,
                     const std::vector<uint8_t>& axial) {
    const std::size_t npe = static_cast<std::size_t>(ngll_) * ngll_;
    Block b;
    b.kind = kBlockAxisym;
    b.m = m_;
    b.axial = axial;
    for (std::size_t e = 0; e < d.quads.size(); ++e) {
      b.elements.push_back(static_cast<i32>(e));
      const std::size_t p0 = static_cast<std::size_t>(d.quads[e]) * npe;
      for (std::size_t k = 0; k < npe; ++k) {
        const std::size_t pt = p0 + k, at = e * npe + k;
        push_metric(b, pt);
        b.coef0.push_back(static_cast<float>(coef0[at]));
        b.coef1.push_back(static_cast<float>(coef1[at]));
        b.wr.push_back(static_cast<float>(wr[at]));
        b.hoop.push_back(static_cast<float>(hoop[at]));
        b.r.push_back(static_cast<float>(geom_.x[pt] <= 0.0 ? 0.0 : geom_.x[pt]));  // exactly 0 on the axis
      }
    }
    return b;
  }

  void push_metric(Block& b, std::size_t pt) const {
    for (const std::vector<double>* v : {&geom_.xi_x, &geom_.xi_z, &geom_.eta_x, &geom_.eta_z, &geom_.jac})
      b.metric.push_back(static_cast<float>((*v)[pt]));
  }

  void cartesian_blocks(MediumPart& d, const std::vector<double>& coef0, const std::vector<double>& coef1) {
    const std::size_t npe = static_cast<std::size_t>(ngll_) * ngll_;
    for (int kind : {kBlockRect, kBlockAffine, kBlockCurved}) {
      Block b;
      b.kind = kind;
      for (std::size_t e = 0; e < d.quads.size(); ++e) {
        const i32 q = d.quads[e];
        if (geom_.shape[q] != kind) continue;
        b.elements.push_back(static_cast<i32>(e));
        const std::size_t p0 = static_cast<std::size_t>(q) * npe;
        if (kind == kBlockRect) {
          for (const std::vector<double>* v : {&geom_.xi_x, &geom_.eta_z, &geom_.jac})
            b.metric.push_back(static_cast<float>((*v)[p0]));
        } else if (kind == kBlockAffine) {
          push_metric(b, p0);
        } else {
          for (std::size_t k = 0; k < npe; ++k) push_metric(b, p0 + k);
        }
        for (std::size_t k = 0; k < npe; ++k) {
          b.coef0.push_back(static_cast<float>(coef0[e * npe + k]));
          b.coef1.push_back(static_cast<float>(coef1[e * npe + k]));
        }
      }
      if (!b.elements.empty()) d.blocks.push_back(std::move(b));
    }
  }

  // Quadrature weight times surface element of a side point, with the unit
  // outward normal; axisymmetric weights carry r (GLJ on sides leaving the axis).
  void side_weight(i32 quad, int f, int i, int j, double& w, double& nx, double& nz) const {
    const std::size_t pt = static_cast<std::size_t>(quad) * ngll_ * ngll_ + j * ngll_ + i;
    const double jac = geom_.jac[pt];
    // counter-clockwise tangent from the inverse metric
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
      w = gll_.w[along_xi ? i : j] * ds;
    } else if (along_xi && forest_->axial(quad)) {
      const double dr_dxi = geom_.eta_z[pt] * geom_.jac[pt];
      const double radius_factor = i == 0 ? dr_dxi : geom_.x[pt] / (1.0 + glj_.x[i]);
      w = glj_.w[i] * ds * radius_factor;
    } else {
      w = gll_.w[along_xi ? i : j] * ds * std::max(geom_.x[pt], 0.0);
    }
  }

  // Element point q (0..n) of side f in counter-clockwise order.
  static void side_point(int f, int q, int n, int& i, int& j) {
    switch (f) {
      case 0: i = q; j = 0; break;
      case 1: i = n; j = q; break;
      case 2: i = n - q; j = n; break;
      default: i = 0; j = n - q; break;
    }
  }

  static i32 unconstrained(const PointMap& pm, std::size_t s) {
    expect(pm.slot[s] >= 0, "a boundary or interface point is constrained by a hanging side");
    return pm.slot[s];
  }

  // ------------------------------------------------------------- edges
  void edges(MediumPart& d) {
    std::map<int64_t, int> tag_of;  // cell * 4 + side -> tag
    for (const TaggedSide& t : grid_->tagged()) tag_of[static_cast<int64_t>(t.cell) * 4 + t.side] = t.tag;
    const int n = ngll_ - 1, nc = d.ncomp;
    std::map<i32, std::array<double, 9>> damping;  // by global point, ascending
    std::set<i32> fixed;
    for (std::size_t e = 0; e < d.quads.size(); ++e) {
      const i32 q = d.quads[e];
      const Quadrant& qd = (*forest_)[q];
      const i32 last = (i32{1} << qd.level) - 1;
      const bool outer[4] = {qd.j == 0, qd.i == last, qd.j == last, qd.i == 0};
      const MaterialSpec& mat = material_of(q);
      for (int f = 0; f < 4; ++f) {
        if (!outer[f] || !grid_->exterior(qd.cell, f)) continue;
        int kind = d.medium == kElastic ? kFree : kRigid;  // the medium's natural condition
        const bool on_axis = grid_->axis_side(qd.cell, f);
        const auto tag = tag_of.find(static_cast<int64_t>(qd.cell) * 4 + f);
        if (tag != tag_of.end()) {
          const auto bc = condition_.find(tag->second);
          if (bc != condition_.end()) {
            expect(!on_axis, [&] { return "boundary tag " + std::to_string(tag->second) +
                                 " lies on the symmetry axis, which takes no boundary condition"; });
            kind = bc->second;
          }
        }
        if (on_axis) continue;
        const bool dirichlet = (d.medium == kElastic && kind == kRigid) || (d.medium == kAcoustic && kind == kFree);
        if (kind != kAbsorbing && !dirichlet) continue;
        for (int p = 0; p <= n; ++p) {
          int i, j;
          side_point(f, p, n, i, j);
          const i32 g = unconstrained(d.points, e * d.points.npe + j * ngll_ + i);
          if (dirichlet) {
            fixed.insert(g);
            continue;
          }
          double w, nx, nz;
          side_weight(q, f, i, j, w, nx, nz);
          auto& acc = damping.try_emplace(g, std::array<double, 9>{}).first->second;
          if (d.medium == kAcoustic) {
            acc[0] += w / (mat.rho * mat.vp);
            continue;
          }
          // traction -C v, C = w rho [vp n n^T + vs (I - n n^T)]
          const double a = w * mat.rho * mat.vp;
          const double b = w * mat.rho * mat.vs;
          const double cxx = a * nx * nx + b * (1.0 - nx * nx);
          const double czz = a * nz * nz + b * (1.0 - nz * nz);
          const double cxz = (a - b) * nx * nz;
          if (nc == 2) {
            acc[0] += cxx;
            acc[1] += cxz;
            acc[2] += cxz;
            acc[3] += czz;
          } else {
            // (r, theta, z) with theta tangential, in the (U+, U-, U_z) basis
            const double ct = w * mat.rho * mat.vs;
            const double pp = 0.5 * (cxx + ct), pm = 0.5 * (cxx - ct), pz = kSqrtHalf * cxz;
            const double c[9] = {pp, pm, pz, pm, pp, pz, pz, pz, czz};
            for (int s = 0; s < 9; ++s) acc[s] += c[s];
          }
        }
      }
    }
    const std::set<i32> axis(d.axis_points.begin(), d.axis_points.end());
    for (auto& [g, c] : damping) {
      if (fixed.count(g)) continue;  // a Dirichlet condition wins at shared corners
      if (axis.count(g))
        for (i32 ac : d.axis_components)
          for (int s = 0; s < nc; ++s) c[ac * nc + s] = c[s * nc + ac] = 0.0;
      d.absorbing.push_back(g);
      for (int s = 0; s < nc * nc; ++s) d.absorbing_coef.push_back(static_cast<float>(c[s]));
    }
    d.dirichlet.assign(fixed.begin(), fixed.end());
  }

  MediumPart* part(int medium) {
    for (MediumPart& d : parts_)
      if (d.medium == medium) return &d;
    return nullptr;
  }
  int part_index(int medium) const {
    for (std::size_t i = 0; i < parts_.size(); ++i)
      if (parts_[i].medium == medium) return static_cast<int>(i);
    return -1;
  }

  // --------------------------------------------------------- interface
  void interface() {
    const MediumPart* fluid = part(kAcoustic);
    const MediumPart* solid = part(kElastic);
    if (!fluid || !solid) return;
    const int n = ngll_ - 1;
    auto side_key = [](i32 a, i32 b) {
      return (static_cast<uint64_t>(std::min(a, b)) << 32) | static_cast<uint32_t>(std::max(a, b));
    };
    std::map<uint64_t, std::pair<i32, int>> solid_side;  // element side by its vertex pair
    for (std::size_t e = 0; e < solid->quads.size(); ++e) {
      const i32* v = &corners_[4 * static_cast<std::size_t>(solid->quads[e])];
      for (int f = 0; f < 4; ++f)
        solid_side[side_key(v[kSideCorner[f][0]], v[kSideCorner[f][1]])] = {static_cast<i32>(e), f};
    }
    struct Pair {
      i32 solid;
      double cx, cz;
    };
    std::map<i32, Pair> by_fluid_point;
    for (std::size_t e = 0; e < fluid->quads.size(); ++e) {
      const i32 q = fluid->quads[e];
      const i32* v = &corners_[4 * static_cast<std::size_t>(q)];
      for (int f = 0; f < 4; ++f) {
        const i32 a = v[kSideCorner[f][0]], b = v[kSideCorner[f][1]];
        const auto hit = solid_side.find(side_key(a, b));
        if (hit == solid_side.end()) continue;
        const auto [es, fs] = hit->second;
        const i32* vs = &corners_[4 * static_cast<std::size_t>(solid->quads[es])];
        const bool solid_rising = vs[kSideCorner[fs][0]] < vs[kSideCorner[fs][1]];
        for (int p = 0; p <= n; ++p) {
          int i, j, is, js;
          side_point(f, p, n, i, j);
          const int from_low = a < b ? p : n - p;
          side_point(fs, solid_rising ? from_low : n - from_low, n, is, js);
          const i32 gf = unconstrained(fluid->points, e * fluid->points.npe + j * ngll_ + i);
          const std::size_t solid_slot = static_cast<std::size_t>(es) * solid->points.npe + js * ngll_ + is;
          const i32 gs = unconstrained(solid->points, solid_slot);
          double w, nx, nz;
          side_weight(q, f, i, j, w, nx, nz);
          Pair& pr = by_fluid_point.try_emplace(gf, Pair{gs, 0.0, 0.0}).first->second;
          expect(pr.solid == gs, "a fluid interface point faces two solid points");
          pr.cx += w * nx;
          pr.cz += w * nz;
        }
      }
    }
    for (const auto& [gf, pr] : by_fluid_point) {
      cpl_fluid_.push_back(gf);
      cpl_solid_.push_back(pr.solid);
      cpl_cx_.push_back(static_cast<float>(pr.cx));
      cpl_cz_.push_back(static_cast<float>(pr.cz));
    }
  }

  // -------------------------------------------------------- point terms
  // Bins over the padded bounding boxes of a medium's elements, for locate().
  struct Bins {
    double x0 = 0, z0 = 0, hx = 1, hz = 1;
    int nx = 1, nz = 1;
    std::vector<std::vector<i32>> members;  // element indices, ascending
  };

  std::array<double, 4> padded_box(i32 q) const {
    const std::size_t npe = static_cast<std::size_t>(ngll_) * ngll_, p0 = static_cast<std::size_t>(q) * npe;
    const auto [xa, xb] = std::minmax_element(geom_.x.begin() + p0, geom_.x.begin() + p0 + npe);
    const auto [za, zb] = std::minmax_element(geom_.z.begin() + p0, geom_.z.begin() + p0 + npe);
    const double pad = 0.25 * std::max(*xb - *xa, *zb - *za);  // curved elements bulge past their points
    return {*xa - pad, *xb + pad, *za - pad, *zb + pad};
  }

  const Bins& bins_of(int di) {
    auto found = bins_.find(di);
    if (found != bins_.end()) return found->second;
    const MediumPart& d = parts_[di];
    Bins b;
    std::vector<std::array<double, 4>> boxes(d.quads.size());
    double X0 = 1e300, X1 = -1e300, Z0 = 1e300, Z1 = -1e300;
    for (std::size_t e = 0; e < d.quads.size(); ++e) {
      boxes[e] = padded_box(d.quads[e]);
      X0 = std::min(X0, boxes[e][0]);
      X1 = std::max(X1, boxes[e][1]);
      Z0 = std::min(Z0, boxes[e][2]);
      Z1 = std::max(Z1, boxes[e][3]);
    }
    b.nx = b.nz = std::max(1, static_cast<int>(std::sqrt(static_cast<double>(d.quads.size()))));
    b.x0 = X0;
    b.z0 = Z0;
    b.hx = std::max((X1 - X0) / b.nx, 1e-300);
    b.hz = std::max((Z1 - Z0) / b.nz, 1e-300);
    b.members.assign(static_cast<std::size_t>(b.nx) * b.nz, {});
    auto cell = [](double v, double v0, double h, int nmax) {
      return std::clamp(static_cast<int>(std::floor((v - v0) / h)), 0, nmax - 1);
    };
    for (std::size_t e = 0; e < d.quads.size(); ++e) {
      const int i0 = cell(boxes[e][0], b.x0, b.hx, b.nx), i1 = cell(boxes[e][1], b.x0, b.hx, b.nx);
      const int j0 = cell(boxes[e][2], b.z0, b.hz, b.nz), j1 = cell(boxes[e][3], b.z0, b.hz, b.nz);
      for (int j = j0; j <= j1; ++j)
        for (int i = i0; i <= i1; ++i) b.members[static_cast<std::size_t>(j) * b.nx + i].push_back(static_cast<i32>(e));
    }
    return bins_.emplace(di, std::move(b)).first->second;
  }

  // The first element of medium part di, in element order, whose map reaches
  // x by Newton's method inside its reference square (locate.cpp:8-49).
  Located locate(int di, std::array<double, 2> x) {
    const Bins& b = bins_of(di);
    const int bi = static_cast<int>(std::floor((x[0] - b.x0) / b.hx));
    const int bj = static_cast<int>(std::floor((x[1] - b.z0) / b.hz));
    if (bi < 0 || bj < 0 || bi > b.nx || bj > b.nz) return {};
    const std::size_t bin = static_cast<std::size_t>(std::min(bj, b.nz - 1)) * b.nx + std::min(bi, b.nx - 1);
    const std::vector<i32>& cand = b.members[bin];
    for (i32 e : cand) {
      const i32 q = parts_[di].quads[e];
      const auto box = padded_box(q);
      if (x[0] < box[0] || x[0] > box[1] || x[1] < box[2] || x[1] > box[3]) continue;
      double xi = 0.0, eta = 0.0;
      bool settled = false;
      for (int it = 0; it < 30 && !settled; ++it) {
        const auto y = quad_point(*forest_, q, xi, eta);
        const auto j = quad_jacobian(*forest_, q, xi, eta);
        const double rx = y[0] - x[0];
        const double rz = y[1] - x[1];
        const double det = j[0] * j[3] - j[1] * j[2];
        const double dxi = (j[3] * rx - j[1] * rz) / det;
        const double deta = (-j[2] * rx + j[0] * rz) / det;
        xi = std::clamp(xi - dxi, -2.0, 2.0);
        eta = std::clamp(eta - deta, -2.0, 2.0);
        settled = std::abs(dxi) + std::abs(deta) < 1e-12;
      }
      constexpr double kSlack = 1e-9;
      if (settled && std::abs(xi) <= 1.0 + kSlack && std::abs(eta) <= 1.0 + kSlack)
        return {q, std::clamp(xi, -1.0, 1.0), std::clamp(eta, -1.0, 1.0)};
    }
    return {};
  }

  Stencil stencil(const Located& at) const {
    const Interpolant& bx = axisym_ && forest_->axial(at.quad) ? *glj_basis_ : *gll_basis_;
    const Interpolant& by = *gll_basis_;
    const auto lx = bx.at(at.xi), ly = by.at(at.eta), dlx = bx.slope_at(at.xi), dly = by.slope_at(at.eta);
    const auto j = quad_jacobian(*forest_, at.quad, at.xi, at.eta);
    const double det = j[0] * j[3] - j[1] * j[2];
    const double xi_x = j[3] / det, xi_z = -j[1] / det, eta_x = -j[2] / det, eta_z = j[0] / det;
    const int n = ngll_;
    Stencil s;
    s.value.resize(static_cast<std::size_t>(n) * n);
    s.ddx.resize(s.value.size());
    s.ddz.resize(s.value.size());
    for (int jj = 0; jj < n; ++jj) {
      for (int ii = 0; ii < n; ++ii) {
        const std::size_t k = static_cast<std::size_t>(jj) * n + ii;
        const double d_xi = dlx[ii] * ly[jj];
        const double d_eta = lx[ii] * dly[jj];
        s.value[k] = lx[ii] * ly[jj];
        s.ddx[k] = d_xi * xi_x + d_eta * eta_x;
        s.ddz[k] = d_xi * xi_z + d_eta * eta_z;
      }
    }
    return s;
  }

  void source(int si) {
    const int kind = in_.source_kind[si];
    const int medium = (kind == kMonopole || kind == kDipole) ? kAcoustic : kElastic;
    const char* kind_name[] = {"force", "moment tensor", "monopole", "dipole"};
    const int di = part_index(medium);
    const std::string label = "source " + std::to_string(si) + " (" + kind_name[kind & 3] + ")";
    expect(di >= 0, [&] { return label + " acts in the " + (medium == kElastic ? "elastic" : "acoustic") +
                        " medium, which the model does not have"; });
    const MediumPart& d = parts_[di];
    const std::array<double, 2> x{in_.source_position[2 * si], in_.source_position[2 * si + 1]};
    const Located at = locate(di, x);
    expect(at.quad >= 0, [&] { return label + " at (" + fmt(x[0]) + ", " + fmt(x[1]) + ") is not inside the " +
                             (medium == kElastic ? "elastic" : "acoustic") + " medium"; });
    const Stencil w = stencil(at);
    const double* c = in_.source_components + 3 * si;
    const bool directional = kind == kForce || kind == kDipole;
    // the weak form is per radian (m = 0) or per pi (m = 1) on axisymmetric meshes
    const double scale = !axisym_ ? 1.0 : m_ == 1 ? 1.0 / kPi : 1.0 / (2.0 * kPi);
    const double rs = x[0];
    if (axisym_) {
      const bool on_axis = std::abs(rs) <= 1e-12 * (1.0 + std::abs(x[1]));
      if (m_ == 0) {
        expect(!(on_axis && directional && c[0] != 0.0),
               [&] {
                 return label + ": a radial force or dipole on the axis is not axisymmetric (use azimuthal order 1)";
               });
        expect(!(on_axis && kind == kMoment && c[2] != 0.0),
               [&] { return label + ": an M_rz moment on the axis is not axisymmetric"; });
      } else {
        expect(directional, [&] { return label + ": azimuthal order 1 takes force and dipole sources only"; });
        expect(!(on_axis && c[1] != 0.0),
               [&] {
                 return label + ": a vertical force or dipole on the axis is axisymmetric (use azimuthal order 0)";
               });
      }
    }
    const double rho = material_of(at.quad).rho;
    const bool plus_minus = d.medium == kElastic && m_ == 1;
    const i32 e = d.element_of[at.quad];
    std::map<i32, std::array<double, 3>> acc;
    for (int k = 0; k < d.points.npe; ++k) {
      double fc[3] = {0.0, 0.0, 0.0};
      switch (kind) {
        case kForce:
          if (plus_minus) {
            fc[0] = fc[1] = kSqrtHalf * c[0] * w.value[k];
            fc[2] = c[1] * w.value[k];
          } else {
            fc[0] = c[0] * w.value[k];
            fc[1] = c[1] * w.value[k];
          }
          break;
        case kMoment:
          fc[0] = c[0] * w.ddx[k] + c[2] * w.ddz[k];
          fc[1] = c[2] * w.ddx[k] + c[1] * w.ddz[k];
          if (axisym_) fc[0] += c[0] * (rs > 0.0 ? w.value[k] / rs : w.ddx[k]);  // hoop part
          break;
        case kMonopole:
          fc[0] = w.value[k];
          break;
        default:
          fc[0] = (c[0] * w.ddx[k] + c[1] * w.ddz[k]) / rho;
          break;
      }
      for (const auto& [g, wt] : d.points.entries(static_cast<std::size_t>(e) * d.points.npe + k)) {
        auto& a = acc.try_emplace(g, std::array<double, 3>{}).first->second;
        for (int comp = 0; comp < d.ncomp; ++comp) a[comp] += wt * fc[comp] * scale;
      }
    }
    PointSource ps;
    ps.domain = di;
    ps.stf_kind = in_.stf_kind[si];
    ps.f0 = in_.stf_params[3 * si];
    ps.t0 = in_.stf_params[3 * si + 1];
    ps.amplitude = in_.stf_params[3 * si + 2];
    for (const auto& kv : acc) ps.points.push_back(kv.first);
    ps.coef.resize(static_cast<std::size_t>(d.ncomp) * acc.size());
    std::size_t i = 0;
    for (const auto& kv : acc) {
      for (int comp = 0; comp < d.ncomp; ++comp) ps.coef[comp * acc.size() + i] = static_cast<float>(kv.second[comp]);
      ++i;
    }
    sources_.push_back(std::move(ps));
  }

  void receiver(int ri) {
    const std::array<double, 2> x{in_.receiver_position[2 * ri], in_.receiver_position[2 * ri + 1]};
    const int want = in_.receiver_medium ? in_.receiver_medium[ri] : -1;
    Located at;
    int di = -1;
    for (std::size_t i = 0; i < parts_.size() && at.quad < 0; ++i) {
      if (want >= 0 && parts_[i].medium != want) continue;
      at = locate(static_cast<int>(i), x);
      if (at.quad >= 0) di = static_cast<int>(i);
    }
    expect(at.quad >= 0, [&] {
      const std::string where = want < 0 ? "model" : want == kElastic ? "elastic medium" : "acoustic medium";
      return "receiver " + std::to_string(ri) + " at (" + fmt(x[0]) + ", " + fmt(x[1]) + ") is not inside the " + where;
    });
    const MediumPart& d = parts_[di];
    const Stencil w = stencil(at);
    const i32 e = d.element_of[at.quad];
    std::map<i32, std::array<double, 3>> acc;
    for (int k = 0; k < d.points.npe; ++k) {
      for (const auto& [g, wt] : d.points.entries(static_cast<std::size_t>(e) * d.points.npe + k)) {
        auto& a = acc.try_emplace(g, std::array<double, 3>{}).first->second;
        a[0] += wt * w.value[k];
        a[1] += wt * w.ddx[k];
        a[2] += wt * w.ddz[k];
      }
    }
    PointReceiver pr;
    pr.domain = di;
    for (const auto& [g, a] : acc) {
      pr.points.push_back(g);
      pr.value.push_back(static_cast<float>(a[0]));
      pr.ddx.push_back(static_cast<float>(a[1]));
      pr.ddz.push_back(static_cast<float>(a[2]));
    }
    pr.rho = material_of(at.quad).rho;
    for (int q = in_.receiver_qoffsets[ri]; q < in_.receiver_qoffsets[ri + 1]; ++q) {
      const int quantity = in_.receiver_quantities[q];
      const bool solid_quantity = quantity == kDisplacement || quantity == kVelocity || quantity == kAcceleration;
      const bool fluid_quantity = quantity == kPressure || quantity == kParticleVelocity;
      expect(d.medium == kElastic ? solid_quantity : fluid_quantity,
             [&] { return "receiver " + std::to_string(ri) + " records a quantity its medium does not have"; });
      pr.quantities.push_back(quantity);
    }
    expect(!pr.quantities.empty(), [&] { return "receiver " + std::to_string(ri) + " records nothing"; });
    receivers_.push_back(std::move(pr));
  }

  // -------------------------------------------------------------- pack
  Packed pack() {
    Packed o;
    const std::string P = "problem.";
    const auto D = gll_basis_->derivative_matrix();
    const auto Dj = glj_basis_->derivative_matrix();
    std::vector<float> w2(static_cast<std::size_t>(ngll_) * ngll_);
    for (int j = 0; j < ngll_; ++j)
      for (int i = 0; i < ngll_; ++i) w2[j * ngll_ + i] = static_cast<float>(gll_.w[i] * gll_.w[j]);
    o.one(P + "basis.ngll", ngll_);
    o.f32(P + "basis.D", std::vector<float>(D.begin(), D.end()));
    o.f32(P + "basis.Dj", std::vector<float>(Dj.begin(), Dj.end()));
    o.f32(P + "basis.w2", std::move(w2));
    o.one(P + "axisym", axisym_ ? 1 : 0);
    o.one(P + "azimuthal_order", m_);
    o.one(P + "record_every", in_.record_every);
    o.one(P + "energy_every", in_.energy_every);
    o.one(P + "domains.count", static_cast<int64_t>(parts_.size()));
    for (std::size_t di = 0; di < parts_.size(); ++di) {
      MediumPart& d = parts_[di];
      PointMap& pm = d.points;
      const std::string p = P + "domains." + std::to_string(di) + ".";
      o.one(p + "medium", d.medium);
      o.one(p + "ncomp", d.ncomp);
      o.one(p + "azimuthal_order", d.m);
      o.one(p + "n_global", pm.n_global);
      o.one(p + "n_elements", pm.n_elements);
      o.i32s(p + "l2g", std::move(pm.slot));
      o.i32s(p + "row_offsets", std::move(pm.row_start));
      o.i32s(p + "row_dofs", std::move(pm.row_point));
      o.f64(p + "row_weights", std::move(pm.row_weight));
      o.i32s(p + "t_offsets", std::move(pm.t_start));
      o.i32s(p + "t_slots", std::move(pm.t_slot));
      o.f64(p + "t_weights", std::move(pm.t_weight));
      o.f32(p + "mass", std::move(d.mass));
      o.f32(p + "inv_mass", std::move(d.inv_mass));
      o.i32s(p + "absorbing_points", std::move(d.absorbing));
      o.f32(p + "absorbing_coef", std::move(d.absorbing_coef));
      o.i32s(p + "dirichlet_points", std::move(d.dirichlet));
      o.i32s(p + "axis_points", std::move(d.axis_points));
      o.i32s(p + "axis_components", std::move(d.axis_components));
      o.f64(p + "coords", std::move(d.coords));
      o.one(p + "blocks.count", static_cast<int64_t>(d.blocks.size()));
      for (std::size_t bi = 0; bi < d.blocks.size(); ++bi) {
        Block& b = d.blocks[bi];
        const std::string q = p + "blocks." + std::to_string(bi) + ".";
        o.one(q + "kind", b.kind);
        o.one(q + "azimuthal_order", b.m);
        o.i32s(q + "elements", std::move(b.elements));
        o.f32(q + "metric", std::move(b.metric));
        o.f32(q + "coef0", std::move(b.coef0));
        o.f32(q + "coef1", std::move(b.coef1));
        o.f32(q + "wr", std::move(b.wr));
        o.f32(q + "hoop", std::move(b.hoop));
        o.f32(q + "r", std::move(b.r));
        o.u8(q + "axial", std::move(b.axial));
      }
    }
    o.i32s(P + "coupling.fluid_points", std::move(cpl_fluid_));
    o.i32s(P + "coupling.solid_points", std::move(cpl_solid_));
    o.f32(P + "coupling.cx", std::move(cpl_cx_));
    o.f32(P + "coupling.cz", std::move(cpl_cz_));
    o.one(P + "sources.count", static_cast<int64_t>(sources_.size()));
    for (std::size_t si = 0; si < sources_.size(); ++si) {
      PointSource& s = sources_[si];
      const std::string p = P + "sources." + std::to_string(si) + ".";
      o.one(p + "domain", s.domain);
      o.i32s(p + "points", std::move(s.points));
      o.f32(p + "coef", std::move(s.coef));
      o.one(p + "stf.kind", s.stf_kind);
      o.real(p + "stf.f0", s.f0);
      o.real(p + "stf.t0", s.t0);
      o.real(p + "stf.amplitude", s.amplitude);
    }
    o.one(P + "receivers.count", static_cast<int64_t>(receivers_.size()));
    for (std::size_t ri = 0; ri < receivers_.size(); ++ri) {
      PointReceiver& r = receivers_[ri];
      const std::string p = P + "receivers." + std::to_string(ri) + ".";
      o.one(p + "domain", r.domain);
      o.i32s(p + "points", std::move(r.points));
      o.f32(p + "value", std::move(r.value));
      o.f32(p + "d_dx", std::move(r.ddx));
      o.f32(p + "d_dz", std::move(r.ddz));
      o.real(p + "rho", r.rho);
      o.i32s(p + "quantities", std::move(r.quantities));
    }
    o.seal();
    return o;
  }

  const insem_case_desc& in_;
  std::unique_ptr<MacroGrid> grid_;
  std::unique_ptr<QuadForest> forest_;
  std::map<int, MaterialSpec> material_;
  std::map<int, int> condition_;
  int ngll_ = 0, m_ = 0;
  bool axisym_ = false;
  Rule1D gll_, glj_;
  std::unique_ptr<Interpolant> gll_basis_, glj_basis_;
  PointGeometry geom_;
  std::vector<i32> corners_;
  i32 n_vertices_ = 0;
  std::vector<MediumPart> parts_;
  std::map<int, Bins> bins_;
  std::vector<i32> cpl_fluid_, cpl_solid_;
  std::vector<float> cpl_cx_, cpl_cz_;
  std::vector<PointSource> sources_;
  std::vector<PointReceiver> receivers_;
};

}  // namespace
}  // namespace insem_setup

struct insem_case_out {
  insem_setup::Packed arrays;
};

extern "C" {

int insem_case_build(const insem_case_desc* desc, insem_case_out** out) {
  try {
    insem_setup::expect(desc != nullptr && out != nullptr, "null argument");
    auto h = std::make_unique<insem_case_out>();
    h->arrays = insem_setup::CaseSetup(*desc).run();
    *out = h.release();
    insem_setup::t_message.clear();
    return 0;
  } catch (const std::exception& e) {
    insem_setup::t_message = e.what();
    return 1;
  }
}

int32_t insem_case_n_arrays(const insem_case_out* out) { return out ? static_cast<int32_t>(out->arrays.size()) : 0; }

const insem_case_array* insem_case_array_at(const insem_case_out* out, int32_t i) {
  if (!out || i < 0 || static_cast<std::size_t>(i) >= out->arrays.size()) return nullptr;
  return out->arrays.at(static_cast<std::size_t>(i));
}

void insem_case_free(insem_case_out* out) { delete out; }

const char* insem_case_last_error(void) { return insem_setup::t_message.c_str(); }

}  // extern "C"
