// Host-side check of the tile kernels' shared-memory layout (TileLayout::make).
//
// The layout reuses the element-data region (metric .. descriptors) for
// data that is only live after the fluxes: the xi-flux rows (phases 3b-4),
// then the assembly target with v and 1/M (phases 5-7).  For every ngll,
// geometry kind, medium, azimuthal order and tile size this checks:
//   - every region starts on a 16-byte boundary (bulk copies need it);
//   - regions that are live in the same phase never overlap;
//   - a region placed in the element-data region lies inside it;
//   - everything lies inside [0, total).
// Prints "ok" and exits 0, or prints the first violation and exits 1.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "tiled.cuh"

using insem_b200::TileCfg;
using insem_b200::TileLayout;
using insem_b200::rows_elem_stride;

namespace {

struct Region {
  const char* name;
  uint32_t beg, end;
};

bool disjoint(const Region& a, const Region& b) { return a.end <= b.beg || b.end <= a.beg; }

int fail(const std::string& what) {
  std::printf("FAIL %s\n", what.c_str());
  return 1;
}

int te_max(int ng) {
  switch (ng) {
    case 2: return TileCfg<2>::TE;
    case 3: return TileCfg<3>::TE;
    case 4: return TileCfg<4>::TE;
    case 5: return TileCfg<5>::TE;
    case 6: return TileCfg<6>::TE;
    case 7: return TileCfg<7>::TE;
    case 8: return TileCfg<8>::TE;
    default: return TileCfg<9>::TE;
  }
}

}  // namespace

int main() {
  long cases = 0;
  for (int ng = 2; ng <= 9; ++ng) {
    const int npe = ng * ng, q = ng - 1;
    for (int kind = 0; kind <= 3; ++kind)
      for (int elastic = 0; elastic <= 1; ++elastic)
        for (int m = 0; m <= (kind == 3 ? 1 : 0); ++m) {
          const int nc = elastic ? (m == 1 ? 3 : 2) : 1;
          for (int te = 1; te <= te_max(ng); ++te)
          for (int rs = 1; rs <= 8; rs += 3) {
            // capacities as the tile builder bounds them: complete points plus a perimeter of halo points
            int side = 1;
            while (side * side < te) ++side;
            const int ncp = te * q * q, tp = ncp + 4 * side * q + 4;
            const int tp_cap = (tp + 3) & ~3, nc_cap = (ncp + 3) & ~3;
            const TileLayout L = TileLayout::make(ng, nc, kind, elastic != 0, te, tp_cap, nc_cap, rs);
            ++cases;
            const std::string id = "ng " + std::to_string(ng) + " kind " + std::to_string(kind) + " elastic " +
                                   std::to_string(elastic) + " m " + std::to_string(m) + " te " + std::to_string(te) +
                                   " rs " + std::to_string(rs);
            const uint32_t offs[] = {L.bar, L.metric, L.wr, L.hoop, L.r,  L.u,  L.v,
                                     L.im,  L.pl,     L.su, L.sfx,  L.ax, L.total};
            if (te * nc * npe > 32768) return fail(id + ": staging places do not fit the point lists' 15 bits");
            for (uint32_t o : offs)
              if (o % 16u) return fail(id + ": offset " + std::to_string(o) + " not 16-byte aligned");
            const uint32_t rows = static_cast<uint32_t>(rows_elem_stride(ng, nc));
            const uint32_t su_floats = rows > static_cast<uint32_t>(nc * npe) ? rows : static_cast<uint32_t>(nc * npe);
            const uint32_t elem_end = L.u;  // the element data runs up to the u region
            const Region bar{"barriers", L.bar, L.bar + 16};
            const Region elem{"element data", L.metric, elem_end};
            const Region u{"u", L.u, L.u + 4u * nc * tp_cap};
            const Region su{"field rows / staging", L.su, L.su + 4u * te * su_floats};
            const Region sfx{"xi-flux rows", L.sfx, L.sfx + 4u * te * rows};
            const Region pl{"point lists", L.pl, L.pl + 2u * rs * nc_cap};
            const Region v{"v", L.v, L.v + 4u * nc * nc_cap};
            const Region im{"1/M", L.im, L.im + 4u * nc_cap};
            const Region ax{"axis terms", L.ax, L.ax + (kind == 3 ? 4u * te * 4 * ((ng + 3) & ~3) : 0u)};
            // phases 1-3a: copies land, rows are built, fluxes read the element data
            std::vector<Region> p1 = {bar, elem, u, su, ax};
            if (insem_b200::early_flux_rows(ng, nc)) p1.push_back(sfx);  // f_xi rows written during the fluxes
            // phases 3b-4: flux rows written and read; the element data is dead, and
            // v and 1/M arrive (late copies) or are held
            std::vector<Region> p2 = {bar, u, su, ax, sfx, v, im};
            // phases 5-7: staging (in su), point lists, completion of the points
            std::vector<Region> p3 = {bar, u, su, pl, v, im};
            if (!L.late) {
              p1.push_back(v);
              p1.push_back(im);
            }
            for (const auto* set : {&p1, &p2, &p3})
              for (std::size_t a = 0; a < set->size(); ++a) {
                if ((*set)[a].end > L.total) return fail(id + ": " + (*set)[a].name + " ends past the total");
                for (std::size_t b = a + 1; b < set->size(); ++b)
                  if ((*set)[a].end > (*set)[a].beg && (*set)[b].end > (*set)[b].beg && !disjoint((*set)[a], (*set)[b]))
                    return fail(id + ": " + (*set)[a].name + " overlaps " + (*set)[b].name);
              }
            auto inside = [&](const Region& r) { return r.beg >= elem.beg && r.end <= elem.end; };
            if (L.sfx == L.metric && !inside(sfx)) return fail(id + ": xi-flux rows overrun the element data");
            if (L.late && !(inside(pl) && inside(v) && inside(im)))
              return fail(id + ": late regions overrun the element data");
          }
        }
  }
  std::printf("ok %ld layouts\n", cases);
  return 0;
}
