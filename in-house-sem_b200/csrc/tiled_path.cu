// Tiling and device numbering of the tiled fused step (host side).
//
// Per domain:
//   1. elements of each block are grown into compact tiles of <= TE elements
//      (breadth-first over elements that share a global point);
//   2. a point is "complete" when every contribution to it is an
//      unconstrained slot of one tile and it carries no boundary, coupling,
//      source, receiver, Dirichlet or axis term; all other points are halo
//      points;
//   3. device numbering: complete points tile by tile, then halo points
//      (both in ascending reference order inside their group);
//   4. slot descriptors give each slot its tile point and, for complete
//      points, its rank in the point's ascending slot list (the order of
//      DofMap::assemble, dof_map.hpp:123-141);
//   5. halo slots write to a halo buffer whose entries each halo point sums
//      through a CSR in ascending slot order (weights of constrained maps kept).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>

#include "tiled_path.cuh"

namespace insem_b200 {

void set_constant_basis_ng2(const float*, const float*, const float*);
void set_constant_basis_ng3(const float*, const float*, const float*);
void set_constant_basis_ng4(const float*, const float*, const float*);
void set_constant_basis_ng5(const float*, const float*, const float*);
void set_constant_basis_ng6(const float*, const float*, const float*);
void set_constant_basis_ng7(const float*, const float*, const float*);
void set_constant_basis_ng8(const float*, const float*, const float*);
void set_constant_basis_ng9(const float*, const float*, const float*);
int tile_elements_ng2();
int tile_elements_ng3();
int tile_elements_ng4();
int tile_elements_ng5();
int tile_elements_ng6();
int tile_elements_ng7();
int tile_elements_ng8();
int tile_elements_ng9();

namespace {
// What each device's constant basis holds per ngll.  Solves of one ngll share
// the bank: D and w2 are written by the first solve and must agree after; the
// GLJ matrix is written by the first solve that has axial elements and never
// cleared (a solve without it does not read it).  So a bank is written at most
// once per part, never while kernels of that ngll that read the part run.
struct BasisBank {
  std::vector<float> D, Dj, w2;
};
std::mutex g_basis_mutex;
std::map<std::pair<int, int>, BasisBank> g_basis;  // (device, ngll)

void write_basis(int ngll, const float* D, const float* Dj, const float* w2) {
  switch (ngll) {
    case 2: set_constant_basis_ng2(D, Dj, w2); break;
    case 3: set_constant_basis_ng3(D, Dj, w2); break;
    case 4: set_constant_basis_ng4(D, Dj, w2); break;
    case 5: set_constant_basis_ng5(D, Dj, w2); break;
    case 6: set_constant_basis_ng6(D, Dj, w2); break;
    case 7: set_constant_basis_ng7(D, Dj, w2); break;
    case 8: set_constant_basis_ng8(D, Dj, w2); break;
    case 9: set_constant_basis_ng9(D, Dj, w2); break;
    default: check_ngll(ngll);
  }
}
}  // namespace

void set_constant_basis(int ngll, const std::vector<float>& D, const std::vector<float>& Dj,
                        const std::vector<float>& w2) {
  check_ngll(ngll);
  int device = 0;
  CUDA_CHECK(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lk(g_basis_mutex);
  BasisBank& bank = g_basis[{device, ngll}];
  if (bank.D.empty()) {
    write_basis(ngll, D.data(), nullptr, w2.data());
    bank.D = D;
    bank.w2 = w2;
  } else {
    INSEM_REQUIRE(bank.D == D && bank.w2 == w2, INSEM_CUDA_ERR_INVALID,
                  "solves of one ngll must share the GLL basis (D, w_i w_j)");
  }
  if (!Dj.empty()) {
    if (bank.Dj.empty()) {
      write_basis(ngll, nullptr, Dj.data(), nullptr);
      bank.Dj = Dj;
    } else {
      INSEM_REQUIRE(bank.Dj == Dj, INSEM_CUDA_ERR_INVALID, "solves of one ngll must share the GLJ derivative matrix");
    }
  }
}

int tile_elements(int ngll) {
  switch (ngll) {
    case 2: return tile_elements_ng2();
    case 3: return tile_elements_ng3();
    case 4: return tile_elements_ng4();
    case 5: return tile_elements_ng5();
    case 6: return tile_elements_ng6();
    case 7: return tile_elements_ng7();
    case 8: return tile_elements_ng8();
    case 9: return tile_elements_ng9();
    default: check_ngll(ngll);
  }
  return 0;
}

void launch_tiles(int ngll, const TileLaunch& a) {
  switch (ngll) {
    case 2: launch_tiles_ng2(a); break;
    case 3: launch_tiles_ng3(a); break;
    case 4: launch_tiles_ng4(a); break;
    case 5: launch_tiles_ng5(a); break;
    case 6: launch_tiles_ng6(a); break;
    case 7: launch_tiles_ng7(a); break;
    case 8: launch_tiles_ng8(a); break;
    case 9: launch_tiles_ng9(a); break;
    default: check_ngll(ngll);
  }
}

namespace {
std::mutex g_tile_mutex;
std::map<int, int> g_tile_table;  // key (ngll, kind, elastic, m) -> elements per tile
int tile_key(int ngll, int kind, bool elastic, int m) { return ((ngll * 4 + kind) * 2 + (elastic ? 1 : 0)) * 2 + m; }
}  // namespace

void set_tile_elements(int ngll, int kind, bool elastic, int m, int te) {
  check_ngll(ngll);
  INSEM_REQUIRE(te <= tile_elements(ngll), INSEM_CUDA_ERR_INVALID, "more tile elements than the kernel takes");
  std::lock_guard<std::mutex> lk(g_tile_mutex);
  if (te <= 0) g_tile_table.erase(tile_key(ngll, kind, elastic, m));
  else g_tile_table[tile_key(ngll, kind, elastic, m)] = te;
}

int tile_step_occupancy(int ngll, int kind, bool elastic, int m, int te, uint32_t smem) {
  switch (ngll) {
    case 2: return tile_step_occupancy_ng2(kind, elastic, m, te, smem);
    case 3: return tile_step_occupancy_ng3(kind, elastic, m, te, smem);
    case 4: return tile_step_occupancy_ng4(kind, elastic, m, te, smem);
    case 5: return tile_step_occupancy_ng5(kind, elastic, m, te, smem);
    case 6: return tile_step_occupancy_ng6(kind, elastic, m, te, smem);
    case 7: return tile_step_occupancy_ng7(kind, elastic, m, te, smem);
    case 8: return tile_step_occupancy_ng8(kind, elastic, m, te, smem);
    case 9: return tile_step_occupancy_ng9(kind, elastic, m, te, smem);
    default: return -1;
  }
}

int analytic_tile_elements(int ngll, int kind, bool elastic, int m, int ncomp) {
  // one answer per class and device (the occupancy queries below ask the device)
  static std::mutex mu;
  static std::map<std::pair<int, int>, int> cache;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    dev = -1;
  }
  const int key = ((((ngll * 4 + kind) * 2 + (elastic ? 1 : 0)) * 2 + m) * 4 + ncomp);
  {
    std::lock_guard<std::mutex> lk(mu);
    const auto it = cache.find({dev, key});
    if (it != cache.end()) return it->second;
  }
  const int te_max = tile_elements(ngll);
  const int q = ngll - 1;
  double best = -1.0;
  int best_te = te_max;
  for (int te = te_max; te >= 1; --te) {
    if (tile_threads(te, ngll) < 64 && te < te_max) break;
    // tile points: interior (q^2 per element) plus the patch's perimeter
    const int side = static_cast<int>(std::ceil(std::sqrt(static_cast<double>(te))));
    const int nc = te * q * q;
    const int tp = nc + 4 * side * q + 4;
    const TileLayout L = TileLayout::make(ngll, ncomp, kind, elastic, te, (tp + 3) & ~3, (nc + 3) & ~3, 4);
    // CTAs per SM: the device's answer for the kernel (its registers count
    // too), else shared memory alone with 2 KB per CTA for the reserved and
    // static parts
    const int occ = dev >= 0 ? tile_step_occupancy(ngll, kind, elastic, m, te, L.total) : -1;
    const int by_smem = (228 * 1024) / (static_cast<int>(L.total) + 2048);
    const int ctas = std::min({occ >= 0 ? occ : by_smem, 2048 / tile_threads(te, ngll), 32});
    if (ctas < 1) continue;
    const double halo = static_cast<double>(tp - nc) / tp;                 // points shared with other tiles
    const double overlap = ctas >= 3 ? 1.0 : ctas == 2 ? 0.9 : 0.6;       // copies of one tile under another's math
    const double lanes = static_cast<double>(te * ngll) / tile_threads(te, ngll);  // threads with an element column
    const double score = ctas * te * (1.0 - 0.5 * halo) * overlap * lanes;
    if (score > best + 1e-9) {
      best = score;
      best_te = te;
    }
  }
  {
    std::lock_guard<std::mutex> lk(mu);
    cache[{dev, key}] = best_te;
  }
  return best_te;
}

int choose_tile_elements(int ngll, int kind, bool elastic, int m, int ncomp, int requested) {
  const int te_max = tile_elements(ngll);
  if (requested > 0) return std::min(requested, te_max);
  {
    std::lock_guard<std::mutex> lk(g_tile_mutex);
    const auto it = g_tile_table.find(tile_key(ngll, kind, elastic, m));
    if (it != g_tile_table.end()) return std::min(it->second, te_max);
  }
  return analytic_tile_elements(ngll, kind, elastic, m, ncomp);
}

int tile_batch(int ngll, const TileBatchLaunch& a, bool launch) {
  switch (ngll) {
    case 2: return tile_batch_ng2(a, launch);
    case 3: return tile_batch_ng3(a, launch);
    case 4: return tile_batch_ng4(a, launch);
    case 5: return tile_batch_ng5(a, launch);
    case 6: return tile_batch_ng6(a, launch);
    case 7: return tile_batch_ng7(a, launch);
    case 8: return tile_batch_ng8(a, launch);
    case 9: return tile_batch_ng9(a, launch);
    default: check_ngll(ngll);
  }
  return 0;
}

namespace {
uint32_t bits_of(float v) {
  uint32_t b;
  std::memcpy(&b, &v, sizeof b);
  return b;
}
}  // namespace

BlockDev TiledDomain::BlockTiles::view() const {
  BlockDev v;
  v.kind = kind;
  v.m = m;
  v.n = n;
  v.metric = metric.get();
  v.coef0 = coef0.get();
  v.coef1 = coef1.get();
  v.wr = wr.get();
  v.hoop = hoop.get();
  v.r = r.get();
  v.axial = axial.get();
  return v;
}

TiledDev TiledDomain::view(int parity) const {
  TiledDev t;
  t.ng = ng;
  t.n_complete = n_complete;
  t.n_hbuf = n_hbuf;
  t.n_cslots = n_cslots;
  t.inv_mass = inv_mass.get();
  t.mass = mass.get();
  t.u_cur = parity ? u1.get() : u0.get();
  t.u_nxt = const_cast<float*>(parity ? u0.get() : u1.get());
  t.v = const_cast<float*>(v.get());
  t.a = const_cast<float*>(a.get());
  t.vn = const_cast<float*>(vn.get());
  t.sdesc = sdesc.get();
  t.tiles = tiles.get();
  t.halo_tp = halo_tp.get();
  t.hs_slot = hs_slot.get();
  t.hs_dst = hs_dst.get();
  t.mdst_off = mdst_off.get();
  t.mdst = mdst.get();
  t.cs_slot = cs_slot.get();
  t.cs_idx = cs_idx.get();
  t.cval = cval.get();
  t.hbuf = const_cast<float*>(hbuf.get());
  return t;
}

HaloDev TiledDomain::halo_view() const {
  HaloDev h;
  h.n = n_halo;
  h.off = h_off.get();
  h.w = weighted ? h_w.get() : nullptr;
  h.spec = h_spec.get();
  h.src_off = src_off.get();
  h.src_which = src_which.get();
  h.src_coef = src_coef.get();
  h.cpl_off = cpl_off.get();
  h.cpl_idx = cpl_idx.get();
  h.abs_idx = abs_idx.get();
  h.abs_coef = abs_coef_d.get();
  h.zero = zero.get();
  return h;
}

void TiledDomain::build(const insem_cuda_domain& d, int ngll, int te, const SpecialTerms& sp,
                        const std::vector<float>& abs_coef_host) {
  medium = d.medium;
  ncomp = d.ncomp;
  m = d.azimuthal_order;
  this->te = te;
  ng = d.dofs.n_global;  // reference count while building; the padded stride at the end
  ng_ref = ng;
  npe = ngll * ngll;
  n_elements = d.dofs.n_elements;
  const std::size_t n_slots = static_cast<std::size_t>(n_elements) * npe;
  const auto l2g = host_vec(d.dofs.l2g, n_slots);
  const auto t_off = host_vec(d.dofs.t_offsets, static_cast<std::size_t>(ng) + 1);
  const auto t_slots = host_vec(d.dofs.t_slots, static_cast<std::size_t>(t_off.back()));
  weighted = d.dofs.n_rows > 0 && d.dofs.t_weights != nullptr;
  const auto t_w = weighted ? host_vec(d.dofs.t_weights, static_cast<std::size_t>(t_off.back())) : std::vector<double>{};

  // special points
  std::vector<char> special(ng, 0);
  for (const auto& kv : sp.sources) special[kv.first] = 1;
  for (const auto& kv : sp.coupling) special[kv.first] = 1;
  for (const auto& kv : sp.absorbing) special[kv.first] = 1;
  for (const auto& kv : sp.zero) special[kv.first] = 1;
  for (int32_t g : sp.receivers) special[g] = 1;

  // 1. tiles per block
  std::vector<int32_t> eblock(n_elements, -1), epos(n_elements, -1);
  for (int b = 0; b < d.n_blocks; ++b)
    for (int q = 0; q < d.blocks[b].n_elements; ++q) {
      const int32_t e = d.blocks[b].elements[q];
      INSEM_REQUIRE(e >= 0 && e < n_elements && eblock[e] < 0, INSEM_CUDA_ERR_INVALID, "block elements overlap");
      eblock[e] = b;
      epos[e] = q;
    }
  std::vector<int32_t> tile_of(n_elements, -1), stamp(n_elements, -1);
  std::vector<std::vector<int32_t>> tile_elems;
  std::vector<int32_t> tile_block;
  blocks.clear();
  blocks.resize(d.n_blocks);
  std::vector<int32_t> queue;
  for (int b = 0; b < d.n_blocks; ++b) {
    blocks[b].kind = d.blocks[b].kind;
    blocks[b].m = d.blocks[b].azimuthal_order;
    blocks[b].n = d.blocks[b].n_elements;
    blocks[b].tile0 = static_cast<int>(tile_elems.size());
    for (int q = 0; q < d.blocks[b].n_elements; ++q) {
      const int32_t seed = d.blocks[b].elements[q];
      if (tile_of[seed] >= 0) continue;
      const int32_t t = static_cast<int32_t>(tile_elems.size());
      tile_elems.emplace_back();
      tile_block.push_back(b);
      auto& te_list = tile_elems.back();
      queue.clear();
      queue.push_back(seed);
      stamp[seed] = t;
      std::size_t head = 0;
      while (head < queue.size() && static_cast<int>(te_list.size()) < te) {
        const int32_t e = queue[head++];
        tile_of[e] = t;
        te_list.push_back(e);
        for (int k = 0; k < npe; ++k) {
          const int32_t g = l2g[static_cast<std::size_t>(e) * npe + k];
          if (g < 0) continue;
          for (int32_t s = t_off[g]; s < t_off[g + 1]; ++s) {
            const int32_t e2 = t_slots[s] / npe;
            if (eblock[e2] == b && tile_of[e2] < 0 && stamp[e2] != t) {
              stamp[e2] = t;
              queue.push_back(e2);
            }
          }
        }
      }
      std::sort(te_list.begin(), te_list.end());
    }
    blocks[b].ntiles = static_cast<int>(tile_elems.size()) - blocks[b].tile0;
  }
  n_tiles = static_cast<int>(tile_elems.size());

  // 2. point classification
  std::vector<int32_t> owner(ng, -1);
  for (int32_t g = 0; g < ng; ++g) {
    if (special[g]) continue;
    int32_t t = -2;
    bool ok = true;
    for (int32_t s = t_off[g]; s < t_off[g + 1] && ok; ++s) {
      const int32_t slot = t_slots[s];
      if (l2g[slot] != g) ok = false;
      const int32_t tt = tile_of[slot / npe];
      if (t == -2) t = tt;
      else if (tt != t) ok = false;
    }
    if (ok && t >= 0) owner[g] = t;
  }
  // 3. device numbering
  std::vector<int32_t> count(n_tiles + 1, 0);
  for (int32_t g = 0; g < ng; ++g)
    if (owner[g] >= 0) ++count[owner[g] + 1];
  // every tile's complete range starts on a multiple of 4 points (16 bytes)
  // so it can be moved by bulk copies; the gaps are unused padding points
  auto up4 = [](int32_t x) { return (x + 3) & ~3; };
  std::vector<int32_t> cbeg(n_tiles + 1, 0);
  for (int t = 0; t < n_tiles; ++t) cbeg[t + 1] = up4(cbeg[t] + count[t + 1]);
  n_complete = cbeg[n_tiles];
  perm.assign(ng, -1);
  int32_t n_halo_pts = 0;
  {
    std::vector<int32_t> fill(cbeg.begin(), cbeg.end() - 1);
    int32_t h = n_complete;
    for (int32_t g = 0; g < ng; ++g) {
      if (owner[g] >= 0) perm[g] = fill[owner[g]]++;
      else {
        perm[g] = h++;
        ++n_halo_pts;
      }
    }
  }
  n_halo = n_halo_pts;
  const int32_t ng_dev = std::max(up4(n_complete + n_halo), 4);
  const int cs = point_stride_rt(npe);

  // 4. ranks of complete points' slots
  std::vector<uint8_t> rank_of(n_slots, 0xff);
  for (int32_t g = 0; g < ng; ++g) {
    if (owner[g] < 0) continue;
    const int32_t nsl = t_off[g + 1] - t_off[g];
    INSEM_REQUIRE(nsl < 255, INSEM_CUDA_ERR_UNSUPPORTED, "too many contributions to one point");
    for (int32_t s = t_off[g]; s < t_off[g + 1]; ++s) rank_of[t_slots[s]] = static_cast<uint8_t>(s - t_off[g]);
  }

  // 5. per tile: tile points, descriptors, halo and constrained slots
  std::vector<TileHdr> hdr(n_tiles);
  std::vector<uint32_t> desc(static_cast<std::size_t>(n_elements) * cs, 0u);
  std::vector<int32_t> htp, hslot, cslot, cidx, crow;
  std::vector<int32_t> hpos_of_slot(n_slots, -1);
  std::vector<int32_t> tpi(ng_dev, -1), tpi_stamp(ng, -1);
  std::vector<int32_t> block_elem_count(d.n_blocks, 0);
  for (int b = 0; b < d.n_blocks; ++b) blocks[b].e_off = 0;
  int32_t e_running = 0, hb = 0;
  for (int b = 0; b < d.n_blocks; ++b) {
    blocks[b].e_off = e_running;
    int32_t be = 0;
    for (int t = blocks[b].tile0; t < blocks[b].tile0 + blocks[b].ntiles; ++t) {
      TileHdr& th = hdr[t];
      th.be0 = be;
      th.ne = static_cast<int32_t>(tile_elems[t].size());
      th.cbeg = cbeg[t];
      th.nc = count[t + 1];  // owned points; [cbeg + nc, cbeg[t + 1]) is padding
      th.hl_off = static_cast<int32_t>(htp.size());
      th.hs_off = static_cast<int32_t>(hslot.size());
      th.cs_off = static_cast<int32_t>(cslot.size());
      th.hb = hb;
      th.maxrank = 0;
      // halo points read by the tile
      std::vector<int32_t> hp;
      for (int32_t e : tile_elems[t])
        for (int k = 0; k < npe; ++k) {
          const int32_t g = l2g[static_cast<std::size_t>(e) * npe + k];
          if (g >= 0 && owner[g] != t && tpi_stamp[g] != t) {
            tpi_stamp[g] = t;
            hp.push_back(perm[g]);
          }
        }
      std::sort(hp.begin(), hp.end());
      for (std::size_t q = 0; q < hp.size(); ++q) htp.push_back(hp[q]);
      th.ntp = th.nc + static_cast<int32_t>(hp.size());
      // tile point index of every point the tile touches
      // halo tile points follow the complete points' padded range
      for (std::size_t q = 0; q < hp.size(); ++q) tpi[hp[q]] = up4(th.nc) + static_cast<int32_t>(q);
      int32_t nh = 0;
      for (int el = 0; el < th.ne; ++el) {
        const int32_t e = tile_elems[t][el];
        for (int k = 0; k < npe; ++k) {
          const std::size_t s = static_cast<std::size_t>(e) * npe + k;
          const int32_t g = l2g[s];
          const int32_t ls = el * npe + k;
          uint32_t dsc;
          if (g >= 0) {
            const int32_t pg = perm[g];
            const int32_t p = owner[g] == t ? pg - th.cbeg : tpi[pg];
            INSEM_REQUIRE(p >= 0 && p < 65536, INSEM_CUDA_ERR_UNSUPPORTED, "tile has too many points");
            const uint32_t rank = owner[g] == t ? rank_of[s] : kSlotRankNone;
            dsc = static_cast<uint32_t>(p) | (rank << kSlotRankShift);
            if (owner[g] == t && static_cast<int32_t>(rank) == t_off[g + 1] - t_off[g] - 1) dsc |= kSlotLast;
            if (owner[g] == t) {
              th.maxrank = std::max<int32_t>(th.maxrank, static_cast<int32_t>(rank));
            } else {
              hpos_of_slot[s] = hb + nh++;
              hslot.push_back(ls);
            }
          } else {
            dsc = kSlotConstrained | (kSlotRankNone << kSlotRankShift);
            cslot.push_back(ls);
            cidx.push_back(static_cast<int32_t>(crow.size()));
            crow.push_back(-1 - g);
            hpos_of_slot[s] = hb + nh++;
            hslot.push_back(ls);
          }
          desc[(static_cast<std::size_t>(e_running) + be + el) * cs + k] = dsc;
        }
      }
      th.nhs = nh;
      th.ncs = static_cast<int32_t>(cslot.size()) - th.cs_off;
      hb += nh;
      be += th.ne;
    }
    e_running += be;
  }
  const int32_t n_entries = hb;
  n_cslots = static_cast<int32_t>(crow.size());
  tp_cap = 4;
  nc_cap = 4;
  rank_cap = 1;
  for (const auto& th : hdr) {
    tp_cap = std::max(tp_cap, up4(th.nc) + th.ntp - th.nc);
    nc_cap = std::max(nc_cap, up4(th.nc));
    rank_cap = std::max(rank_cap, th.maxrank + 1);
  }
  tp_cap = up4(tp_cap);  // keeps every component row of the staged u 16-byte aligned

  // 6. halo CSR and special records (device order of halo points)
  std::vector<int32_t> hoff{0}, hpos, hspec(n_halo, -1), soff{0}, swhich, coff{0}, cidx2, aidx;
  std::vector<float> hw, scoef;
  std::vector<uint8_t> zm;
  std::vector<int32_t> halo_orig(n_halo);
  for (int32_t g = 0; g < ng; ++g)
    if (owner[g] < 0) halo_orig[perm[g] - n_complete] = g;
  for (int32_t h = 0; h < n_halo; ++h) {
    const int32_t g = halo_orig[h];
    for (int32_t s = t_off[g]; s < t_off[g + 1]; ++s) {
      const int32_t pos = hpos_of_slot[t_slots[s]];
      INSEM_REQUIRE(pos >= 0, INSEM_CUDA_ERR_INVALID, "halo contribution without a halo-buffer entry");
      hpos.push_back(pos);
      if (weighted) hw.push_back(static_cast<float>(t_w[s]));
    }
    hoff.push_back(static_cast<int32_t>(hpos.size()));
    if (!special[g]) continue;
    const int32_t rec = static_cast<int32_t>(aidx.size());
    hspec[h] = rec;
    if (auto it = sp.sources.find(g); it != sp.sources.end())
      for (const auto& [s, cs] : it->second) {
        swhich.push_back(s);
        scoef.insert(scoef.end(), cs.begin(), cs.end());
      }
    soff.push_back(static_cast<int32_t>(swhich.size()));
    if (auto it = sp.coupling.find(g); it != sp.coupling.end())
      for (int32_t ci : it->second) cidx2.push_back(ci);
    coff.push_back(static_cast<int32_t>(cidx2.size()));
    auto ia = sp.absorbing.find(g);
    aidx.push_back(ia == sp.absorbing.end() ? -1 : ia->second);
    auto iz = sp.zero.find(g);
    zm.push_back(iz == sp.zero.end() ? 0 : iz->second);
  }

  // Places of the halo-buffer entries in hbuf: hbuf holds each halo point's
  // contributions in its ascending slot order, point after point (the list
  // hoff indexes), so the halo kernel reads them contiguously.  An entry has
  // one place, unless it is a constrained slot feeding several parent
  // points; those entries keep a list of places.
  n_hbuf = static_cast<int32_t>(hpos.size());
  std::vector<int32_t> ecount(n_entries, 0);
  for (int32_t e : hpos) ++ecount[e];
  std::vector<int32_t> hdst(n_entries, 0), moff{0}, mlist;
  {
    std::vector<std::vector<int32_t>> multi(n_entries);
    for (int32_t q = 0; q < n_hbuf; ++q) {
      const int32_t e = hpos[q];
      if (ecount[e] == 1) hdst[e] = q;
      else multi[e].push_back(q);
    }
    for (int32_t e = 0; e < n_entries; ++e) {
      if (ecount[e] == 1) continue;
      hdst[e] = -1 - (static_cast<int32_t>(moff.size()) - 1);
      mlist.insert(mlist.end(), multi[e].begin(), multi[e].end());
      moff.push_back(static_cast<int32_t>(mlist.size()));
    }
  }

  // 7. uploads
  sdesc.upload(desc);
  tiles.upload(hdr);
  host_tiles = std::move(hdr);
  halo_tp.upload(htp.empty() ? std::vector<int32_t>{0} : htp);
  hs_slot.upload(hslot.empty() ? std::vector<int32_t>{0} : hslot);
  hs_dst.upload(hdst.empty() ? std::vector<int32_t>{0} : hdst);
  mdst_off.upload(moff);
  mdst.upload(mlist.empty() ? std::vector<int32_t>{0} : mlist);
  cs_slot.upload(cslot.empty() ? std::vector<int32_t>{0} : cslot);
  cs_idx.upload(cidx.empty() ? std::vector<int32_t>{0} : cidx);
  cs_row.upload(crow.empty() ? std::vector<int32_t>{0} : crow);
  cval.resize(static_cast<std::size_t>(ncomp) * std::max(n_cslots, 1));
  hbuf.resize(static_cast<std::size_t>(ncomp) * std::max(n_hbuf, 1));
  h_off.upload(hoff);
  if (weighted) h_w.upload(hw.empty() ? std::vector<float>{0.0f} : hw);
  h_spec.upload(hspec.empty() ? std::vector<int32_t>{0} : hspec);
  src_off.upload(soff);
  src_which.upload(swhich.empty() ? std::vector<int32_t>{0} : swhich);
  src_coef.upload(scoef.empty() ? std::vector<float>{0.0f} : scoef);
  cpl_off.upload(coff);
  cpl_idx.upload(cidx2.empty() ? std::vector<int32_t>{0} : cidx2);
  abs_idx.upload(aidx.empty() ? std::vector<int32_t>{0} : aidx);
  zero.upload(zm.empty() ? std::vector<uint8_t>{0} : zm);
  abs_coef_d.upload(abs_coef_host.empty() ? std::vector<float>{0.0f} : abs_coef_host);
  // constraint rows with device-numbered dofs (weights rounded as the gather does)
  {
    const auto ro = host_vec(d.dofs.row_offsets, static_cast<std::size_t>(d.dofs.n_rows) + 1);
    const std::size_t nrd = ro.empty() ? 0 : static_cast<std::size_t>(ro.back());
    auto rd = host_vec(d.dofs.row_dofs, nrd);
    const auto rw = host_vec(d.dofs.row_weights, nrd);
    for (auto& g : rd) g = perm[g];
    rows_off.upload(ro.empty() ? std::vector<int32_t>{0} : ro);
    rows_dofs.upload(rd.empty() ? std::vector<int32_t>{0} : rd);
    rows_w.upload(rw.empty() ? std::vector<float>{0.0f} : std::vector<float>(rw.begin(), rw.end()));
  }
  // mass in device numbering
  const auto mh = host_vec(d.mass, ng), imh = host_vec(d.inv_mass, ng);
  host_mass.assign(ng_dev, 0.0f);
  std::vector<float> im(ng_dev, 0.0f);
  for (int32_t g = 0; g < ng; ++g) {
    host_mass[perm[g]] = mh[g];
    im[perm[g]] = imh[g];
  }
  mass.upload(host_mass);
  inv_mass.upload(im);
  const std::size_t nf = static_cast<std::size_t>(ncomp) * ng_dev;
  for (auto* buf : {&u0, &u1, &v, &a, &vn}) {
    buf->resize(nf);
    buf->zero();
  }
  // element data of every block in tile order, padded layout
  for (int b = 0; b < d.n_blocks; ++b) {
    std::vector<int32_t> order;  // block-local positions in tile order
    for (int t = blocks[b].tile0; t < blocks[b].tile0 + blocks[b].ntiles; ++t)
      for (int32_t e : tile_elems[t]) order.push_back(epos[e]);
    PackedBlock pk = pack_block(d.blocks[b], npe, medium, order);
    blocks[b].metric.upload(pk.metric);
    // One material per element: the tile kernels read one coefficient pair
    // per element instead of one per point.
    const std::size_t cs = point_stride_rt(npe);
    std::vector<float> c0(order.size()), c1(medium == INSEM_ELASTIC ? order.size() : 0);
    for (std::size_t q = 0; q < order.size(); ++q) {
      c0[q] = pk.coef0[q * cs];
      if (!c1.empty()) c1[q] = pk.coef1[q * cs];
      for (int k = 1; k < npe; ++k) {
        const bool same = bits_of(pk.coef0[q * cs + k]) == bits_of(c0[q]) &&
                          (c1.empty() || bits_of(pk.coef1[q * cs + k]) == bits_of(c1[q]));
        INSEM_REQUIRE(same, INSEM_CUDA_ERR_UNSUPPORTED,
                      "material coefficients vary inside an element; the tiled path takes one material per "
                      "element (options.path = 1 takes per-point coefficients)");
      }
    }
    blocks[b].coef0.upload(c0);
    if (medium == INSEM_ELASTIC) blocks[b].coef1.upload(c1);
    if (d.blocks[b].kind == INSEM_AXISYM) {
      blocks[b].wr.upload(pk.wr);
      blocks[b].hoop.upload(pk.hoop);
      blocks[b].r.upload(pk.r);
      blocks[b].axial.upload(pk.axial);
    }
  }
  ng = ng_dev;  // from here on the component stride of the device arrays
}

}  // namespace insem_b200
