// Tiled fused time step.
//
// Elements of each block are grouped into compact tiles (one CTA each).  A
// tile kernel stages the field of the tile's points in shared memory,
// computes every element's force vector, assembles the points whose
// contributions all come from the tile ("complete" points) in shared memory,
// and finishes them in the same pass: a = f / M, corrector, and the next
// step's predictor, writing u^{n+1} to the other field buffer.  Contributions
// to points shared with other tiles, constrained (hanging) slots and every
// point carrying a boundary, coupling, source or receiver term go to a halo
// buffer; a halo kernel finishes those points with the full reference logic.
//
// Bitwise parity with the reference: each point's contributions are summed
// in ascending slot order (DofMap::assemble, dof_map.hpp:123-141).  Inside a
// tile, slot s of point p carries its rank (position of s in p's ascending
// slot list); ranks are accumulated phase by phase (rank 0 stores 0 + f,
// rank r adds), so the sum is the reference's.  Halo points sum their halo
// buffer entries in the reference's slot order from a CSR list.
//
// Element math: one thread per element column i (NG threads per element).
// A column thread holds its column of the field, its f_eta column and the
// xi-row / xi-column of the basis derivative matrix in registers; rows of the
// field and of f_xi come from shared memory as broadcasts within an
// element; D entries indexed by the unrolled loop counters come from the
// constant bank.  Every sum keeps the reference's operand order.
#pragma once

#include <cstddef>


#include "element_ops.cuh"
#include "step_kernels.cuh"

namespace insem_b200 {

// GLL derivative matrix, GLJ derivative matrix and w_i w_j per ngll (2..9).
static __constant__ float c_basis[8][3][81];

// Both components of an interleaved pair in one 64-bit shared-memory load.
__device__ __forceinline__ float2 pair_load(const float* p) { return *reinterpret_cast<const float2*>(p); }

// Two-lane FP32 arithmetic on a component pair (sm_100 add/fma .f32x2).  Each
// lane rounds exactly like the scalar instruction.  The assembler fuses a
// two-lane multiply that feeds a two-lane add into one fused multiply-add,
// which rounds once where the reference rounds the product and the sum
// separately; so a product is formed as fma(a, b, z) with z = -0 read from
// constant memory at run time, which is exactly the rounded product (for
// every a, b, including signed zeros) and is not fused further.
static __constant__ float c_neg_zero;  // -0.0f, written with the basis
using f2x = unsigned long long;        // two packed floats (lane 0 low)
__device__ __forceinline__ f2x pk2(float x, float y) {
  f2x r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
  return r;
}
__device__ __forceinline__ float2 upk2(f2x r) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return v;
}
__device__ __forceinline__ f2x add2(f2x a, f2x b) {
  f2x d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
// a * b rounded once per lane (nz = pk2(-0, -0) from c_neg_zero)
__device__ __forceinline__ f2x mul2(f2x a, f2x b, f2x nz) {
  f2x d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(nz));
  return d;
}
__device__ __forceinline__ f2x pair_load2(const float* p) { return *reinterpret_cast<const f2x*>(p); }

// Element stride (floats) of the field / xi-flux rows in shared memory.
// Two components are stored interleaved, row j of element e at
// e * stride + j * 2 * ngll, (l, c) at + 2 l + c, so one 64-bit load gives
// both; the stride is padded so that the elements one warp reads fall on
// distinct 64-bit bank pairs.  Other component counts keep
// [component][row][ROW].
__host__ __device__ constexpr int rows_elem_stride(int ng, int nc) {
  if (nc != 2) return nc * ng * ((ng + 1) & ~1);
  const int base = 2 * ng * ng;
  const int per_warp = 32 / ng + 2;
  for (int s = base; s < base + 64; s += 2) {
    bool ok = true;
    for (int a = 0; a < per_warp && ok; ++a)
      for (int b = a + 1; b < per_warp && ok; ++b) {
        const int da = (a * s) % 32, db = (b * s) % 32;
        if (da == db || (da + 1) % 32 == db || (db + 1) % 32 == da) ok = false;
      }
    if (ok) return s;
  }
  return base;
}

// kModeIdle: a batched solve past its last step (the batch's kernels skip it).
enum StepMode : int32_t { kModeNormal = 0, kModeFinal = 1, kModeInit = 2, kModeIdle = 3 };

// Slot descriptor bits.
constexpr uint32_t kSlotPointMask = 0xffffu;      // tile point index
constexpr int kSlotRankShift = 16;                // local assembly rank (0..254)
constexpr uint32_t kSlotRankNone = 0xffu;          // not assembled in the tile
constexpr uint32_t kSlotConstrained = 1u << 24;   // value from the constrained-slot list
constexpr uint32_t kSlotLast = 1u << 25;          // the highest rank of its (complete) point

struct TileHdr {
  int32_t be0;     // first element of the tile (block-local, tile order)
  int32_t ne;      // elements
  int32_t cbeg;    // first complete point (device numbering)
  int32_t nc;      // complete points
  int32_t ntp;     // tile points: nc complete + halo points the tile reads
  int32_t hl_off;  // offset of the halo tile points in halo_tp
  int32_t hb;      // first halo-buffer entry of the tile
  int32_t nhs;     // halo slots (entries written to the halo buffer)
  int32_t hs_off;  // offset into hs_slot
  int32_t ncs;     // constrained slots of the tile
  int32_t cs_off;  // offset into cs_slot / cs_idx
  int32_t maxrank; // highest local rank
};

// One domain of the tiled path, in device numbering.
struct TiledDev {
  int32_t ng = 0;          // points
  int32_t n_complete = 0;  // complete points are [0, n_complete)
  int32_t n_hbuf = 0;      // halo contributions (per component): the halo points' lists, point by point
  int32_t n_cslots = 0;    // constrained slots of the domain
  const float* inv_mass = nullptr;
  const float* mass = nullptr;
  const float* u_cur = nullptr;
  float* u_nxt = nullptr;
  float* v = nullptr;
  float* a = nullptr;
  float* vn = nullptr;     // v^n at halo points (receivers)
  const uint32_t* sdesc = nullptr;  // [n_el_tiles * npe] slot descriptors, tile order
  const TileHdr* tiles = nullptr;
  const int32_t* halo_tp = nullptr; // device point of each halo tile point
  const int32_t* hs_slot = nullptr; // tile-local slot (e * npe + k) of each halo entry
  const int32_t* hs_dst = nullptr;  // its place in hbuf, or -1 - m: the places mdst[mdst_off[m] ..)
  const int32_t* mdst_off = nullptr;  // entries with several places (constrained slots feeding several points)
  const int32_t* mdst = nullptr;
  const int32_t* cs_slot = nullptr; // tile-local slot of each constrained slot
  const int32_t* cs_idx = nullptr;  // its index into cval
  const float* cval = nullptr;      // [ncomp][n_cslots] gathered constrained-slot values
  float* hbuf = nullptr;            // [ncomp][n_hbuf], each halo point's contributions in its slot order
};

struct StepScalars {
  float rdt, half_dt, half_dt2;
  int32_t energy_every;
};

// Tile elements are chosen per domain at run time (te <= TE, one thread per
// element column).  CTAs are whole warps: te x NG threads rounded up to a
// multiple of 32 (the extra threads have no element and only take part in the
// strided loops, the barriers and the warp reductions).
template <int NG>
struct TileCfg {
  static constexpr int NPE = NG * NG;
  static constexpr int TE = (256 / NG) > 64 ? 64 : (256 / NG);  // elements per tile (max)
  static constexpr int THREADS = (TE * NG + 31) / 32 * 32;       // threads per CTA (max)
  static constexpr int ROW = (NG + 1) & ~1;                      // padded row stride (floats)
};
__host__ __device__ constexpr int tile_threads(int te, int ng) { return (te * ng + 31) / 32 * 32; }

__device__ __forceinline__ float cbasis(int ng, int which, int idx) { return c_basis[ng - 2][which][idx]; }


// ------------------------------------------------------- bulk-copy helpers
// Two mbarriers per CTA track the tile's bulk copies (cp.async.bulk, the
// non-tensor TMA path), one for the copies at the start of a tile and one
// for the late copies: thread 0 announces the byte count and issues the
// copies; every thread waits on the barrier's phase 0 (one tile per CTA).
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Orders this thread's earlier generic-proxy accesses to shared memory (made
// visible to it by a block barrier) before bulk copies that overwrite them.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after `limit` polls (each poll may suspend the
// thread for a hardware-defined interval) and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
constexpr uint32_t kBulkWaitLimit = 1u << 22;

// Whether a class writes its f_xi rows as the fluxes are formed (into a
// region of their own, fewer registers held across the barrier) instead of
// after the barrier into the dead element data (less shared memory).  Only
// three-component classes, and of the benchmarked orders only ngll 6, gain
// from it under their register budgets (256-model batch, per class: ngll 6
// m=1 0.147 vs 0.154 ms early vs late; ngll 5 0.106 vs 0.103; ngll 7 0.229
// vs 0.224).
__host__ __device__ constexpr bool early_flux_rows(int ng, int nc) { return nc == 3 && ng != 5 && ng != 7; }

// Shared-memory layout of one tile CTA, byte offsets (16-byte aligned).
// Per-tile data arrives by bulk copies: element data (metric, axisymmetric
// weights), slot descriptors, and the complete points' u, v and inverse mass
// (v and 1/M later, when `late`); halo tile points are gathered by the
// threads into the u region after the complete points (at index
// roundup(nc, 4) on).  The material coefficients (one pair per element) and
// the slot descriptors (which each column thread keeps in registers) are read
// from global memory by the threads that use them.  `pl` holds, for every
// complete point, the staging places of its contributions in rank order
// (`rs` entries per point, uint16).
struct TileLayout {
  uint32_t bar, metric, wr, hoop, r, u, v, im, pl, su, sfx, ax, total;
  int32_t tp_cap, nc_cap, ms, cs, row, rs;
  int32_t late;  // 1: v and 1/M arrive by a second copy into the element-data region

  __host__ __device__ static uint32_t up16(uint32_t x) { return (x + 15u) & ~15u; }
  // rs: the most contributions one complete point of the class's tiles has
  __host__ __device__ static TileLayout make(int ng, int nc, int kind, bool elastic, int te, int tp_cap, int nc_cap,
                                            int rs) {
    TileLayout L{};
    L.rs = (rs + 3) & ~3;  // a point's list is read four entries (8 bytes) at a time
    const int npe = ng * ng;
    L.cs = (npe + 3) & ~3;
    L.ms = kind == INSEM_RECT ? 4 : kind == INSEM_AFFINE ? 8 : (kind == INSEM_AXISYM ? 4 : 5) * L.cs;
    L.row = (ng + 1) & ~1;
    L.tp_cap = tp_cap;
    L.nc_cap = nc_cap;
    const bool axi = kind == INSEM_AXISYM;
    uint32_t o = 0;
    L.bar = o;  // two mbarriers: the tile's copies, the late v and 1/M copies
    o = up16(o + 16);
    L.metric = o;
    o = up16(o + 4u * te * L.ms);
    L.wr = o;
    if (axi) o = up16(o + 4u * te * L.cs);
    L.hoop = o;
    if (axi) o = up16(o + 4u * te * L.cs);
    L.r = o;
    if (axi) o = up16(o + 4u * te * L.cs);
    // The element data [metric, elem_end) is last read by the fluxes.  Then
    // that region takes, when it is large enough, the f_xi rows (written
    // after the fluxes, read by the divergence) and beside them v and 1/M
    // (copied in after the fluxes); the point lists (written after the
    // divergence) take the place of the f_xi rows.
    const uint32_t elem = o - L.metric;
    L.u = o;
    o = up16(o + 4u * nc * tp_cap);
    L.su = o;
    const uint32_t rows = static_cast<uint32_t>(rows_elem_stride(ng, nc));
    // su doubles as the halo staging area: [te][nc][npe]
    o = up16(o + 4u * te * (rows > static_cast<uint32_t>(nc * npe) ? rows : static_cast<uint32_t>(nc * npe)));
    const uint32_t sfx_b = up16(4u * te * rows);
    // classes that write their f_xi rows as the fluxes are formed
    // (early_flux_rows) cannot keep them in the element data the fluxes
    // still read
    if (sfx_b <= elem && !early_flux_rows(ng, nc)) {
      L.sfx = L.metric;
    } else {
      L.sfx = o;
      o += sfx_b;
    }
    const uint32_t pl_b = up16(2u * L.rs * nc_cap), v_b = up16(4u * nc * nc_cap), im_b = up16(4u * nc_cap);
    const uint32_t sfx_in = L.sfx == L.metric ? sfx_b : 0u;  // f_xi rows inside the element data
    const uint32_t head = pl_b > sfx_in ? pl_b : sfx_in;
    L.late = head + v_b + im_b <= elem ? 1 : 0;
    uint32_t p = L.late ? L.metric : o;
    L.pl = p;
    L.v = p + (L.late ? head : pl_b);
    L.im = L.v + v_b;
    if (!L.late) o += pl_b + v_b + im_b;
    L.ax = o;
    if (axi) o = up16(o + 4u * te * 4 * ((ng + 3) & ~3));
    L.total = o;
    return L;
  }
};

// Mode-dependent completion of a point (solver.cpp:924-944 fused):
//   normal: v = v_half + dt/2 a; u' = u + dt v + dt^2/2 a; v' = v + dt/2 a
//   final:  v = v_half + dt/2 a; u' = u                      (state complete)
//   init:   v unchanged;         u' = u                      (step 0)
__device__ __forceinline__ void complete_point(int mode, const StepScalars& sc, float u, float vh, float a, float& u_out,
                                               float& v_state, float& v_n) {
  if (mode == kModeInit) {
    v_n = vh;
    v_state = vh;
    u_out = u;
    return;
  }
  const float vn = fadd(vh, fmul(sc.half_dt, a));
  v_n = vn;
  if (mode == kModeFinal) {
    v_state = vn;
    u_out = u;
  } else {
    u_out = fadd(u, fadd(fmul(sc.rdt, vn), fmul(sc.half_dt2, a)));
    v_state = fadd(vn, fmul(sc.half_dt, a));
  }
}

// Gathers the values of constrained slots (DofMap::gather rows, dof_map.hpp:110-115).
__device__ __forceinline__ void constrained_gather_body(int32_t n, const int32_t* __restrict__ row_of, const RowsDev& rows,
                                                        const float* __restrict__ u, int32_t ng, int32_t ncomp,
                                                        float* __restrict__ cval, int32_t i) {
  if (i >= n) return;
  const int32_t r = row_of[i];
  for (int c = 0; c < ncomp; ++c) {
    float s = 0.0f;
    for (int32_t q = rows.offsets[r]; q < rows.offsets[r + 1]; ++q)
      s = fadd(s, fmul(rows.weights[q], u[static_cast<size_t>(c) * ng + rows.dofs[q]]));
    cval[static_cast<size_t>(c) * n + i] = s;
  }
}

static __global__ void constrained_gather_kernel(int32_t n, const int32_t* __restrict__ row_of, RowsDev rows,
                                                 const float* __restrict__ u, int32_t ng, int32_t ncomp,
                                                 float* __restrict__ cval) {
  constrained_gather_body(n, row_of, rows, u, ng, ncomp, cval, blockIdx.x * blockDim.x + threadIdx.x);
}

// Predictor on the whole field, in place (start of an advance() after a final step).
static __global__ void predictor_inplace_kernel(float* __restrict__ u, float* __restrict__ v, const float* __restrict__ a,
                                         int64_t n, float rdt, float half_dt, float half_dt2) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float vi = v[i], ai = a[i];
    u[i] = fadd(u[i], fadd(fmul(rdt, vi), fmul(half_dt2, ai)));
    v[i] = fadd(vi, fmul(half_dt, ai));
  }
}

// One tile of the fused step (the whole CTA).  `thp` is the tile's header
// (entry `tile` of the domain's tile table, or a copy of it).  `g_first`, if
// not negative, is this thread's first halo tile point (halo_tp entry
// blockDim.x - 1 - threadIdx.x), already loaded.  `bar` is an
// initialised mbarrier whose next phase to complete has parity `phase`.
// Returns false (after recording the error) if the tile's bulk copies did
// not arrive within the wait limit.
template <int NG, int KIND, bool EL, int M>
__device__ __forceinline__ bool tile_step_body(const BlockDev& blk, const TiledDev& td, const StepScalars& sc,
                                               StepState* __restrict__ st, double* __restrict__ epartial,
                                               int32_t tile, const TileHdr* thp, const TileLayout& L,
                                               unsigned char* smem_raw, uint64_t* bar, uint32_t phase,
                                               int32_t g_first = -1) {
  using Cfg = TileCfg<NG>;
  using CE = ElemCfg<NG, KIND, EL, M>;
  constexpr int NC = CE::NC;
  constexpr int NPE = NG * NG;
  constexpr int CS = point_stride<NPE>();
  constexpr int ROW = Cfg::ROW;
  constexpr bool AXI = KIND == INSEM_AXISYM;
  constexpr int MS = KIND == INSEM_RECT ? 4 : KIND == INSEM_AFFINE ? 8 : (AXI ? 4 : 5) * CS;
  float* s_metric = reinterpret_cast<float*>(smem_raw + L.metric);
  float* s_wr = reinterpret_cast<float*>(smem_raw + L.wr);
  float* s_hoop = reinterpret_cast<float*>(smem_raw + L.hoop);
  float* s_r = reinterpret_cast<float*>(smem_raw + L.r);
  float* tu = reinterpret_cast<float*>(smem_raw + L.u);    // [NC][tp_cap]
  float* s_v = reinterpret_cast<float*>(smem_raw + L.v);   // [NC][nc_cap]
  float* s_im = reinterpret_cast<float*>(smem_raw + L.im); // [nc_cap]
  uint16_t* pl = reinterpret_cast<uint16_t*>(smem_raw + L.pl);  // [nc_cap][rs] staging places, rank order
  float* su = reinterpret_cast<float*>(smem_raw + L.su);   // [TE][NC][NG][ROW] field rows, later staging
  float* sfx = reinterpret_cast<float*>(smem_raw + L.sfx); // [TE][NC][NG][ROW] f_xi rows
  float* sax = reinterpret_cast<float*>(smem_raw + L.ax);  // [TE][4][AXS] axis terms
  const int tp_cap = L.tp_cap, nc_cap = L.nc_cap;

  const TileHdr th = *thp;
  const int tid = threadIdx.x;
  const int nthreads = blockDim.x;  // (tile elements) x NG
  // thread 0 issues the bulk copies; the halo tile points are gathered from
  // the last thread down, so thread 0 has the fewest of them
  const int issuer = 0;
  const int tg = nthreads - 1 - tid;
  const int mode = st->mode;
  const int32_t step = st->step;
  const bool energy = (mode == kModeInit) ? (sc.energy_every > 0) : (sc.energy_every > 0 && step % sc.energy_every == 0);
  const int nc4 = (th.nc + 3) & ~3;

  // 1. bulk copies of the tile's element data, slot descriptors and complete
  //    points (u; v and 1/M too unless they come late)
  if (tid == issuer) {
    const uint32_t eb = 4u * th.ne;
    uint32_t total = eb * MS + eb * CS * (AXI ? 3 : 0);
    if (nc4 > 0) total += 4u * nc4 * (L.late ? NC : 2 * NC + 1);
    fence_proxy_async_smem();
    mbar_expect_tx(bar, total);
    bulk_load(s_metric, blk.metric + static_cast<size_t>(th.be0) * MS, eb * MS, bar);
    if constexpr (AXI) {
      bulk_load(s_wr, blk.wr + static_cast<size_t>(th.be0) * CS, eb * CS, bar);
      bulk_load(s_hoop, blk.hoop + static_cast<size_t>(th.be0) * CS, eb * CS, bar);
      bulk_load(s_r, blk.r + static_cast<size_t>(th.be0) * CS, eb * CS, bar);
    }
    if (nc4 > 0) {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        bulk_load(tu + c * tp_cap, td.u_cur + static_cast<size_t>(c) * td.ng + th.cbeg, 4u * nc4, bar);
        if (!L.late) bulk_load(s_v + c * nc_cap, td.v + static_cast<size_t>(c) * td.ng + th.cbeg, 4u * nc4, bar);
      }
      if (!L.late) bulk_load(s_im, td.inv_mass + th.cbeg, 4u * nc4, bar);
    }
  }
  // this column's slot descriptors, loaded while the bulk copies are in flight
  const int el = tid / NG;
  const int i = tid - el * NG;
  const bool active = el < th.ne;
  uint32_t dsc[NG];
  float ec0 = 0.0f, ec1 = 0.0f;  // the element's material coefficients
  bool axial = false;             // axisymmetric element on the axis (GLJ basis in xi)
  if (active) {
    const uint32_t* gdesc = td.sdesc + static_cast<size_t>(th.be0 + el) * CS + i;
#pragma unroll
    for (int j = 0; j < NG; ++j) dsc[j] = gdesc[j * NG];
    ec0 = blk.coef0[th.be0 + el];
    if constexpr (EL) ec1 = blk.coef1[th.be0 + el];
    if constexpr (AXI) axial = blk.axial[th.be0 + el] != 0;
  }
  // halo tile points, gathered while the bulk copies are in flight
  for (int t = tg; t < th.ntp - th.nc; t += nthreads) {
    const int32_t g = (t == tg && g_first >= 0) ? g_first : td.halo_tp[th.hl_off + t];
#pragma unroll
    for (int c = 0; c < NC; ++c) tu[c * tp_cap + nc4 + t] = td.u_cur[static_cast<size_t>(c) * td.ng + g];
  }
  const bool arrived = mbar_wait_bounded(bar, phase, kBulkWaitLimit);
  if (__syncthreads_or(!arrived)) {
    if (tid == 0) atomicExch(&st->error, 1);
    // give copies still in flight a second bounded wait before the shared memory is left
    mbar_wait_bounded(bar, phase, kBulkWaitLimit);
    return false;
  }

  // element data now in shared memory, indexed by the tile-local element
  BlockDev lb = blk;
  lb.metric = s_metric;
  lb.coef0 = nullptr;  // one pair per element: ec0 / ec1
  lb.coef1 = nullptr;
  lb.wr = s_wr;
  lb.hoop = s_hoop;
  lb.r = s_r;

  constexpr int ES = rows_elem_stride(NG, NC);  // element stride of the rows
  constexpr bool PAIR = NC == 2;                 // interleaved components, two-lane sums
  // position of (component c, row j, column l) in an element's rows
  auto ridx = [](int c, int j, int l) { return PAIR ? j * 2 * NG + 2 * l + c : (c * NG + j) * ROW + l; };
  float* urow = su + el * ES;
  float* frow = sfx + el * ES;
  constexpr int AXS = (NG + 3) & ~3;  // one axis-term array (gx0, gy0, gx1, gy1) of an element
  float* ax = sax + el * 4 * AXS;

  // 2. element field rows (slots through their tile point or the constrained list)
  if (active) {
#pragma unroll
    for (int j = 0; j < NG; ++j) {
      if (!(dsc[j] & kSlotConstrained)) {
        const int p = dsc[j] & kSlotPointMask;
        if constexpr (PAIR) {
          *reinterpret_cast<float2*>(urow + ridx(0, j, i)) = make_float2(tu[p], tu[tp_cap + p]);
        } else {
#pragma unroll
          for (int c = 0; c < NC; ++c) urow[ridx(c, j, i)] = tu[c * tp_cap + p];
        }
      }
    }
  }
  for (int q = tid; q < th.ncs; q += nthreads) {
    const int32_t ls = td.cs_slot[th.cs_off + q];
    const int32_t ci = td.cs_idx[th.cs_off + q];
    const int e = ls / NPE, k = ls - e * NPE;
    const int jj = k / NG, ii = k - jj * NG;
#pragma unroll
    for (int c = 0; c < NC; ++c)
      su[e * ES + ridx(c, jj, ii)] = td.cval[static_cast<size_t>(c) * td.n_cslots + ci];
  }
  __syncthreads();

  // 3. derivatives and fluxes, one column per thread
  float dxr[NG], dxc[NG], w2c[NG];  // Dx row i, Dx column i, w_i w_j
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    dxr[l] = cbasis(NG, axial ? 1 : 0, i * NG + l);
    dxc[l] = cbasis(NG, axial ? 1 : 0, l * NG + i);
    w2c[l] = cbasis(NG, 2, l * NG + i);
  }
  float ucol[NC][NG], fe[NC][NG], fx[NC][NG], dir[2][NG];  // fx: f_xi column, stored after the barrier
  if (active) {
    if constexpr (PAIR) {
      // column i of both components, one 64-bit load per row; both
      // components' sums in two-lane instructions
      const float nzs = c_neg_zero;
      const f2x nz = pk2(nzs, nzs);
      f2x uc[NG];
#pragma unroll
      for (int l = 0; l < NG; ++l) {
        uc[l] = pair_load2(urow + ridx(0, l, i));
        const float2 v = upk2(uc[l]);
        ucol[0][l] = v.x;
        ucol[1][l] = v.y;
      }
#pragma unroll
      for (int j = 0; j < NG; ++j) {
        const int k = j * NG + i;
        const float* row = urow + ridx(0, j, 0);
        f2x a = 0ull, b = 0ull;  // (+0, +0)
#pragma unroll
        for (int l = 0; l < NG; ++l) {
          const float d = cbasis(NG, 0, j * NG + l);
          a = add2(a, mul2(pk2(dxr[l], dxr[l]), pair_load2(row + 2 * l), nz));
          b = add2(b, mul2(pk2(d, d), uc[l], nz));
        }
        const float2 av = upk2(a), bv = upk2(b);
        float uxi[NC] = {av.x, av.y}, ueta[NC] = {bv.x, bv.y}, upt[NC] = {ucol[0][j], ucol[1][j]};
        float fxp[NC], fy[NC], dr[2] = {0.0f, 0.0f};
        point_flux<NG, KIND, EL, M, true>(lb, el, k, i, j, axial, uxi, ueta, upt, fxp, fy, dr, ax, ax + AXS, ax + 2 * AXS,
                                    ax + 3 * AXS, w2c[j], ec0, ec1);
        fx[0][j] = fxp[0];
        fx[1][j] = fxp[1];
        fe[0][j] = fy[0];
        fe[1][j] = fy[1];
        dir[0][j] = dr[0];
        dir[1][j] = dr[1];
      }
    } else {
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < NG; ++j) ucol[c][j] = urow[ridx(c, j, i)];
#pragma unroll
      for (int j = 0; j < NG; ++j) {
        const int k = j * NG + i;
        float uxi[NC], ueta[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          // the row two entries per 8-byte load (rows are ROW = even floats
          // long and start on 8-byte boundaries; the pad entry is never used)
          const float* row = urow + ridx(c, j, 0);
          float a = 0.0f, b = 0.0f;
#pragma unroll
          for (int l = 0; l < NG; l += 2) {
            const float2 r2 = *reinterpret_cast<const float2*>(row + l);
            a = fadd(a, fmul(dxr[l], r2.x));
            b = fadd(b, fmul(cbasis(NG, 0, j * NG + l), ucol[c][l]));
            if (l + 1 < NG) {
              a = fadd(a, fmul(dxr[l + 1], r2.y));
              b = fadd(b, fmul(cbasis(NG, 0, j * NG + l + 1), ucol[c][l + 1]));
            }
          }
          uxi[c] = a;
          ueta[c] = b;
        }
        float fxp[NC], fy[NC], dr[2] = {0.0f, 0.0f}, upt[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) upt[c] = ucol[c][j];
        point_flux<NG, KIND, EL, M, true>(lb, el, k, i, j, axial, uxi, ueta, upt, fxp, fy, dr, ax, ax + AXS, ax + 2 * AXS,
                                    ax + 3 * AXS, w2c[j], ec0, ec1);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          if constexpr (early_flux_rows(NG, NC)) frow[ridx(c, j, i)] = fxp[c];  // own region: store now
          else fx[c][j] = fxp[c];
          fe[c][j] = fy[c];
        }
        dir[0][j] = dr[0];
        dir[1][j] = dr[1];
      }
    }
  }
  __syncthreads();  // the element data is dead: the f_xi rows may overwrite it
  // v and 1/M of the complete points, into the element-data region beside
  // the f_xi rows, while the divergence runs
  if (L.late && tid == issuer) {
    fence_proxy_async_smem();
    mbar_expect_tx(bar + 1, nc4 > 0 ? 4u * nc4 * (NC + 1) : 0u);
    if (nc4 > 0) {
#pragma unroll
      for (int c = 0; c < NC; ++c)
        bulk_load(s_v + c * nc_cap, td.v + static_cast<size_t>(c) * td.ng + th.cbeg, 4u * nc4, bar + 1);
      bulk_load(s_im, td.inv_mass + th.cbeg, 4u * nc4, bar + 1);
    }
  }
  if (active && !early_flux_rows(NG, NC)) {
#pragma unroll
    for (int j = 0; j < NG; ++j) {
      if constexpr (PAIR) {
        *reinterpret_cast<float2*>(frow + ridx(0, j, i)) = make_float2(fx[0][j], fx[1][j]);
      } else {
#pragma unroll
        for (int c = 0; c < NC; ++c) frow[ridx(c, j, i)] = fx[c][j];
      }
    }
  }
  __syncthreads();

  // 4. weak divergence (interleaved xi / eta terms), hoop and axis terms
  float fo[NC][NG];
  if (active) {
#pragma unroll
    for (int j = 0; j < NG; ++j) {
      float s[NC];
      if constexpr (PAIR) {
        const float nzs = c_neg_zero;
        const f2x nz = pk2(nzs, nzs);
        const float* row = frow + ridx(0, j, 0);
        f2x acc = 0ull;  // (+0, +0)
#pragma unroll
        for (int l = 0; l < NG; ++l) {
          const float d = cbasis(NG, 0, l * NG + j);
          acc = add2(acc, mul2(pk2(dxc[l], dxc[l]), pair_load2(row + 2 * l), nz));
          acc = add2(acc, mul2(pk2(d, d), pk2(fe[0][l], fe[1][l]), nz));
        }
        const float2 sv = upk2(acc);
        s[0] = sv.x;
        s[1] = sv.y;
      } else {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const float* row = frow + ridx(c, j, 0);
          float acc = 0.0f;
#pragma unroll
          for (int l = 0; l < NG; l += 2) {
            const float2 r2 = *reinterpret_cast<const float2*>(row + l);
            acc = fadd(acc, fmul(dxc[l], r2.x));
            acc = fadd(acc, fmul(cbasis(NG, 0, l * NG + j), fe[c][l]));
            if (l + 1 < NG) {
              acc = fadd(acc, fmul(dxc[l + 1], r2.y));
              acc = fadd(acc, fmul(cbasis(NG, 0, (l + 1) * NG + j), fe[c][l + 1]));
            }
          }
          s[c] = acc;
        }
      }
      const float drj[2] = {dir[0][j], dir[1][j]};
      float out[NC];
      point_divergence<NG, KIND, EL, M>(i, j, axial, s, drj, dxc[0], [](int q) { return cbasis(NG, 0, q); }, ax,
                                        ax + AXS, ax + 2 * AXS, ax + 3 * AXS, out);
#pragma unroll
      for (int c = 0; c < NC; ++c) fo[c][j] = out[c];
    }
  }
  __syncthreads();  // su is reused below as halo staging; the f_xi rows are dead

  // 5. every slot's contribution to the staging area; each complete point's
  //    slots listed by rank (their sum is formed in step 7, in rank order,
  //    which is the reference's ascending slot order).  This thread's first
  //    halo entry (step 6) is fetched now, so that its index loads complete
  //    meanwhile.
  int32_t hs_first = 0, hd_first = 0;
  if (tid < th.nhs) {
    hs_first = td.hs_slot[th.hs_off + tid];
    hd_first = td.hs_dst[th.hs_off + tid];
  }
  float* stage = su;  // [te][NPE][NC]: a slot's components side by side
  const int rs = L.rs;
  if (active) {
#pragma unroll
    for (int j = 0; j < NG; ++j) {
      const int base = (el * NPE + j * NG + i) * NC;
      if constexpr (NC == 2) {
        *reinterpret_cast<float2*>(stage + base) = make_float2(fo[0][j], fo[1][j]);
      } else {
#pragma unroll
        for (int c = 0; c < NC; ++c) stage[base + c] = fo[c][j];
      }
      const uint32_t rank = (dsc[j] >> kSlotRankShift) & 0xffu;
      if (rank != kSlotRankNone)
        pl[(dsc[j] & kSlotPointMask) * rs + rank] = static_cast<uint16_t>(base | ((dsc[j] & kSlotLast) ? 0x8000 : 0));
    }
  }
  __syncthreads();

  // 6. halo contributions out, each to its place in its halo point's list
  for (int q = tid; q < th.nhs; q += nthreads) {
    const int32_t ls = q == tid ? hs_first : td.hs_slot[th.hs_off + q];
    const int32_t dst = q == tid ? hd_first : td.hs_dst[th.hs_off + q];
    const int e = ls / NPE, k = ls - e * NPE;
    float val[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) val[c] = stage[(e * NPE + k) * NC + c];
    if (dst >= 0) {
#pragma unroll
      for (int c = 0; c < NC; ++c) td.hbuf[static_cast<size_t>(c) * td.n_hbuf + dst] = val[c];
    } else {
      const int32_t mi = -1 - dst;
      for (int32_t d = td.mdst_off[mi]; d < td.mdst_off[mi + 1]; ++d) {
        const int32_t p = td.mdst[d];
#pragma unroll
        for (int c = 0; c < NC; ++c) td.hbuf[static_cast<size_t>(c) * td.n_hbuf + p] = val[c];
      }
    }
  }

  if (L.late) {
    const bool late_arrived = mbar_wait_bounded(bar + 1, phase, kBulkWaitLimit);
    if (__syncthreads_or(!late_arrived)) {
      if (tid == 0) atomicExch(&st->error, 1);
      mbar_wait_bounded(bar + 1, phase, kBulkWaitLimit);
      return false;
    }
  }

  // 7. complete points: a = f / M, corrector, predictor; energy partials
  double kin = 0.0, pot = 0.0;
  for (int t = tid; t < th.nc; t += nthreads) {
    const int32_t g = th.cbeg + t;
    const float im = s_im[t];
    // the point's force: its contributions added in rank order, 0 + f_0
    // first.  Four list entries come in one load; the values of the valid
    // ones (up to the entry flagged last) load together, then add in order.
    float fsum[NC] = {};
    bool more = true;
    for (int r0 = 0; more && r0 < rs; r0 += 4) {
      const uint2 w = *reinterpret_cast<const uint2*>(pl + t * rs + r0);
      const uint32_t e[4] = {w.x & 0xffffu, w.x >> 16, w.y & 0xffffu, w.y >> 16};
      bool valid[4];
      valid[0] = true;
#pragma unroll
      for (int k = 1; k < 4; ++k) valid[k] = valid[k - 1] && !(e[k - 1] & 0x8000u);
      float x[4][NC];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float* sp = stage + (e[k] & 0x7fffu);
        if constexpr (NC == 2) {
          const float2 q = valid[k] ? *reinterpret_cast<const float2*>(sp) : make_float2(0.0f, 0.0f);
          x[k][0] = q.x;
          x[k][1] = q.y;
        } else {
#pragma unroll
          for (int c = 0; c < NC; ++c) x[k][c] = valid[k] ? sp[c] : 0.0f;
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int c = 0; c < NC; ++c)
          if (valid[k]) fsum[c] = (r0 + k == 0) ? fadd(0.0f, x[k][c]) : fadd(fsum[c], x[k][c]);
      more = valid[3] && !(e[3] & 0x8000u);
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const size_t gi = static_cast<size_t>(c) * td.ng + g;
      const float f = fsum[c];
      const float a = fmul(f, im);
      const float u = tu[c * tp_cap + t];
      float u_out, v_state, v_n;
      complete_point(mode, sc, u, s_v[c * nc_cap + t], a, u_out, v_state, v_n);
      td.u_nxt[gi] = u_out;
      td.v[gi] = v_state;
      if (mode != kModeNormal) td.a[gi] = a;
      if (energy) {
        pot = dadd(pot, dmul(static_cast<double>(u), static_cast<double>(f)));
        const double vv = v_n, aa = a;
        const double m = td.mass[g];
        kin = dadd(kin, dmul(m, dsub(dmul(dmul(0.5, vv), vv), dmul(dmul(st->kin_c, aa), aa))));
      }
    }
  }
  if (energy) {
    // deterministic CTA reduction: warp shuffles in a fixed tree, then warps in order
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      kin = dadd(kin, __shfl_down_sync(0xffffffffu, kin, off));
      pot = dadd(pot, __shfl_down_sync(0xffffffffu, pot, off));
    }
    __shared__ double wk[16], wp[16];
    const int w = tid >> 5;
    if ((tid & 31) == 0) {
      wk[w] = kin;
      wp[w] = pot;
    }
    __syncthreads();
    if (tid == 0) {
      double k2 = 0.0, p2 = 0.0;
      for (int q = 0; q < (nthreads + 31) / 32; ++q) {
        k2 = dadd(k2, wk[q]);
        p2 = dadd(p2, wp[q]);
      }
      epartial[2 * tile] = k2;
      epartial[2 * tile + 1] = p2;
    }
  }
  return true;
}

template <int NG, int KIND, bool EL, int M>
__device__ __forceinline__ void tile_step_run(const BlockDev& blk, const TiledDev& td, const StepScalars& sc,
                                              StepState* __restrict__ st, double* __restrict__ epartial,
                                              int32_t tile0, const TileLayout& L) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + L.bar);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
  }
  __syncthreads();
  const int32_t tile = tile0 + blockIdx.x;
  tile_step_body<NG, KIND, EL, M>(blk, td, sc, st, epartial, tile, td.tiles + tile, L, smem_raw, bar, 0u);
}
template <int NG, int KIND, bool EL, int M>
static __global__ void __launch_bounds__(TileCfg<NG>::THREADS)
    tile_step_kernel(BlockDev blk, TiledDev td, StepScalars sc, StepState* __restrict__ st,
                     double* __restrict__ epartial, int32_t tile0, TileLayout L) {
  tile_step_run<NG, KIND, EL, M>(blk, td, sc, st, epartial, tile0, L);
}

// Tiles of many solves in one launch.  A segment is one block of one
// domain of one solve; its field buffers are chosen by that solve's parity.
struct TileSeg {
  BlockDev blk;
  TiledDev td;          // parity-0 view (u_cur = u0, u_nxt = u1)
  StepScalars sc;
  StepState* st;
  double* epartial;     // the domain's tile partials
};

// One work item of a batched tile launch: a tile of one segment, with a copy
// of its header, its solve's step state and its halo point list, so that a
// CTA needs one load of its item before it can read the segment, the state
// and its first halo tile points (in parallel) and issue the tile's bulk
// copies.
struct __align__(16) TileItem {
  TileHdr th;               // the tile's header (entry `tile` of the domain's table)
  const StepState* st;      // the segment's solve
  int32_t seg;              // segment index
  int32_t tile;             // tile index in the domain's table (energy partials)
  const int32_t* halo_tp;   // the tile's halo tile points (domain halo_tp + th.hl_off)
  int64_t pad;
};
static_assert(sizeof(TileItem) == 80, "TileItem is loaded as 20 words");

// One CTA per work item (CTA b takes item b).  Items of solves past their
// last step (idle) are skipped: the CTA exits.  (CTAs that loop over items
// measured slower: the loop keeps about 40 more registers per thread live,
// which costs resident CTAs per SM.)  One shared memory layout serves the
// class (sized for its largest tile).
template <int NG, int KIND, bool EL, int M>
__device__ __forceinline__ void tile_batch_run(const TileSeg* __restrict__ segs, const TileItem* __restrict__ items,
                                               const TileLayout& L) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ __align__(16) TileSeg s_seg;   // the item's segment, read by the body from shared memory
  __shared__ __align__(16) TileItem s_it;
  __shared__ int32_t s_idle;
  static_assert(sizeof(TileSeg) % 4 == 0, "TileSeg is copied as 32-bit words");
  if (threadIdx.x < 20)
    reinterpret_cast<uint32_t*>(&s_it)[threadIdx.x] = reinterpret_cast<const uint32_t*>(items + blockIdx.x)[threadIdx.x];
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
  }
  __syncthreads();
  // this thread's first halo tile point, loaded beside the segment and the state
  const int tg = static_cast<int>(blockDim.x - 1 - threadIdx.x);
  const int32_t g_first = tg < s_it.th.ntp - s_it.th.nc ? s_it.halo_tp[tg] : -1;
  {
    // the segment's words; on the solve's odd steps the words of u_cur and
    // u_nxt are exchanged (both candidates and the parity load together)
    constexpr int kUc = static_cast<int>((offsetof(TileSeg, td) + offsetof(TiledDev, u_cur)) / 4);
    constexpr int kUn = static_cast<int>((offsetof(TileSeg, td) + offsetof(TiledDev, u_nxt)) / 4);
    static_assert(kUn == kUc + 2, "u_cur and u_nxt are adjacent pointers");
    const uint32_t* src = reinterpret_cast<const uint32_t*>(segs + s_it.seg);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&s_seg);
    for (int q = threadIdx.x; q < static_cast<int>(sizeof(TileSeg) / 4); q += blockDim.x) {
      if (q >= kUc && q < kUc + 4) {
        const uint32_t own = src[q], other = src[q < kUn ? q + 2 : q - 2];
        dst[q] = s_it.st->parity ? other : own;
      } else {
        dst[q] = src[q];
      }
    }
  }
  if (threadIdx.x == blockDim.x - 1) s_idle = s_it.st->mode == kModeIdle;
  __syncthreads();
  if (s_idle) return;
  tile_step_body<NG, KIND, EL, M>(s_seg.blk, s_seg.td, s_seg.sc, s_seg.st, s_seg.epartial, s_it.tile, &s_it.th, L,
                                  smem_raw, bar, 0u, g_first);
}
template <int NG, int KIND, bool EL, int M>
static __global__ void __launch_bounds__(TileCfg<NG>::THREADS)
    tile_batch_kernel(const TileSeg* __restrict__ segs, const TileItem* __restrict__ items, TileLayout L) {
  tile_batch_run<NG, KIND, EL, M>(segs, items, L);
}
// Register budgets for the elastic axisymmetric batch classes whose CTAs
// per SM shared memory or the launch's thread count limit anyway: the
// budget is what those CTAs can use.  Uncapped, the compiler gives the ngll
// 7 kernels 99-128 registers (2-3 CTAs per SM where 4 fit) and the ngll 5
// and 6 m=1 kernels 80 with 44-60 bytes of spills although their shared
// memory allows only 3 CTAs.  0: no cap (the kernel's launch bounds apply).
template <int NG, int M>
constexpr int kBatchRegs = NG == 7 ? (M == 1 ? 128 : 96) : (M == 1 ? (NG == 6 ? 112 : NG == 5 ? 96 : 0) : 0);
template <int NG, int KIND, bool EL, int M, int REGS>
static __global__ void __maxnreg__(REGS)
    tile_batch_kernel_capped(const TileSeg* __restrict__ segs, const TileItem* __restrict__ items, TileLayout L) {
  tile_batch_run<NG, KIND, EL, M>(segs, items, L);
}

// ------------------------------------------------------------ halo kernel
// Special-point records of a domain's halo points.
struct HaloDev {
  int32_t n = 0;                     // halo points: device points [n_complete, n_complete + n)
  const int32_t* off = nullptr;      // [n+1] each point's contributions in hbuf, ascending slot order
  const float* w = nullptr;          // its weight (constrained maps), nullptr when all are 1
  const int32_t* spec = nullptr;     // [n] special record or -1
  const int32_t* src_off = nullptr;  // [n_spec+1] source contributions of each record
  const int32_t* src_which = nullptr;// source index of each contribution (row of the amplitude table)
  const float* src_coef = nullptr;   // [contributions][ncomp]
  const int32_t* cpl_off = nullptr;  // [n_spec+1] coupling entries of each record
  const int32_t* cpl_idx = nullptr;
  const int32_t* abs_idx = nullptr;  // [n_spec] Stacey index or -1
  const float* abs_coef = nullptr;   // [n_abs][ncomp*ncomp]
  const uint8_t* zero = nullptr;     // [n_spec] components set to zero (Dirichlet, axis)
};

// Fluid-solid interface in device numbering of both domains.
struct CouplingDev {
  const int32_t* fluid = nullptr;
  const int32_t* solid = nullptr;
  const float* cx = nullptr;
  const float* cz = nullptr;
};

// Finishes the halo points of one domain: the assembled force from the halo
// buffer, then (solver.cpp:669-762) sources, coupling, a = f / M or the
// implicit Stacey solve, Dirichlet / axis zeros, and the mode's update.
// `other` is the fluid's current pressure (solid domain) or the solid's new
// acceleration (fluid domain), in that domain's device numbering.
// One halo point per thread; CTAs of 256 threads, `part` = the CTA's energy partial.
template <int NC, bool ELASTIC>
__device__ __forceinline__ void halo_step_body(const TiledDev& td, const HaloDev& hd, const CouplingDev& cp,
                                               const float* __restrict__ other, int32_t other_ng, bool pm,
                                               const float* __restrict__ amp, int32_t n_amp, const StepScalars& sc,
                                               double h_damp, const StepState* __restrict__ st,
                                               double* __restrict__ epartial, int32_t part, int32_t h) {
  const int mode = st->mode;
  const int32_t step = st->step;
  const bool energy = (mode == kModeInit) ? (sc.energy_every > 0) : (sc.energy_every > 0 && step % sc.energy_every == 0);
  double kin = 0.0, pot = 0.0;
  if (h < hd.n) {
    const int32_t g = td.n_complete + h;
    // the point's own values first, all loads in flight together (the
    // stores below may alias them for the compiler)
    float uc[NC], vc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      uc[c] = td.u_cur[static_cast<size_t>(c) * td.ng + g];
      vc[c] = td.v[static_cast<size_t>(c) * td.ng + g];
    }
    const float im = td.inv_mass[g];
    const int32_t sp = hd.spec[h];
    float f[NC], a[NC];
    const int32_t b = hd.off[h], e = hd.off[h + 1];
    constexpr int K = 4;  // contributions gathered at once (conforming 2D points have at most 4)
    if (e - b <= K) {
      float vq[NC][K];
#pragma unroll
      for (int q = 0; q < K; ++q)
#pragma unroll
        for (int c = 0; c < NC; ++c) vq[c][q] = b + q < e ? td.hbuf[static_cast<size_t>(c) * td.n_hbuf + b + q] : 0.0f;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        float s = 0.0f;
#pragma unroll
        for (int q = 0; q < K; ++q)
          if (b + q < e) s = fadd(s, hd.w ? fmul(hd.w[b + q], vq[c][q]) : vq[c][q]);
        f[c] = s;
      }
    } else {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        float s = 0.0f;
        for (int32_t q = b; q < e; ++q) {
          const float v = td.hbuf[static_cast<size_t>(c) * td.n_hbuf + q];
          s = fadd(s, hd.w ? fmul(hd.w[q], v) : v);
        }
        f[c] = s;
      }
    }
    if (energy) {
#pragma unroll
      for (int c = 0; c < NC; ++c) pot = dadd(pot, dmul(static_cast<double>(uc[c]), static_cast<double>(f[c])));
    }
    int32_t ai = -1;
    uint8_t zmask = 0;
    if (sp >= 0) {
      for (int32_t q = hd.src_off[sp]; q < hd.src_off[sp + 1]; ++q) {
        const float am = amp[static_cast<size_t>(hd.src_which[q]) * n_amp + step];
#pragma unroll
        for (int c = 0; c < NC; ++c) f[c] = fadd(f[c], fmul(hd.src_coef[static_cast<size_t>(q) * NC + c], am));
      }
      const float hs = static_cast<float>(kSqrtHalf);
      for (int32_t q = hd.cpl_off[sp]; q < hd.cpl_off[sp + 1]; ++q) {
        const int32_t ci = hd.cpl_idx[q];
        if constexpr (ELASTIC) {
          const float p = other[cp.fluid[ci]];
          if (pm) {
            const float t = fmul(fmul(hs, cp.cx[ci]), p);
            f[0] = fadd(f[0], t);
            f[1] = fadd(f[1], t);
          } else {
            f[0] = fadd(f[0], fmul(cp.cx[ci], p));
          }
          f[NC - 1] = fadd(f[NC - 1], fmul(cp.cz[ci], p));
        } else {
          const int32_t gs = cp.solid[ci];
          const float ar = pm ? fmul(hs, fadd(other[gs], other[static_cast<size_t>(other_ng) + gs])) : other[gs];
          const float az = other[static_cast<size_t>(pm ? 2 : 1) * other_ng + gs];
          f[0] = fsub(f[0], fadd(fmul(cp.cx[ci], ar), fmul(cp.cz[ci], az)));
        }
      }
      ai = hd.abs_idx[sp];
      zmask = hd.zero[sp];
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) a[c] = fmul(f[c], im);
    if (ai >= 0) {
      const float* cc = hd.abs_coef + static_cast<size_t>(ai) * NC * NC;
      double A[NC * NC], rhs[NC];
      const double mass = td.mass[g];
#pragma unroll
      for (int r = 0; r < NC; ++r) {
        rhs[r] = static_cast<double>(f[r]);
#pragma unroll
        for (int s2 = 0; s2 < NC; ++s2) {
          rhs[r] = dsub(rhs[r], dmul(static_cast<double>(cc[r * NC + s2]), static_cast<double>(vc[s2])));
          A[r * NC + s2] = dadd(dmul(h_damp, static_cast<double>(cc[r * NC + s2])), r == s2 ? mass : 0.0);
        }
      }
      solve_spd_dev(NC, A, rhs);
#pragma unroll
      for (int r = 0; r < NC; ++r) a[r] = static_cast<float>(rhs[r]);
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      if (zmask & (1u << c)) a[c] = 0.0f;
      const size_t gi = static_cast<size_t>(c) * td.ng + g;
      float u_out, v_state, v_n;
      complete_point(mode, sc, uc[c], vc[c], a[c], u_out, v_state, v_n);
      td.u_nxt[gi] = u_out;
      td.v[gi] = v_state;
      td.a[gi] = a[c];
      td.vn[gi] = v_n;
      if (energy) {
        const double vv = v_n, aa = a[c];
        kin = dadd(kin, dmul(static_cast<double>(td.mass[g]), dsub(dmul(dmul(0.5, vv), vv), dmul(dmul(st->kin_c, aa), aa))));
      }
    }
  }
  if (energy) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      kin = dadd(kin, __shfl_down_sync(0xffffffffu, kin, off));
      pot = dadd(pot, __shfl_down_sync(0xffffffffu, pot, off));
    }
    __shared__ double wk[8], wp[8];
    if ((threadIdx.x & 31) == 0) {
      wk[threadIdx.x >> 5] = kin;
      wp[threadIdx.x >> 5] = pot;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double k2 = 0.0, p2 = 0.0;
      for (int q = 0; q < 8; ++q) {
        k2 = dadd(k2, wk[q]);
        p2 = dadd(p2, wp[q]);
      }
      epartial[2 * part] = k2;
      epartial[2 * part + 1] = p2;
    }
  }
}

// Register budgets of the halo kernels (256 threads per CTA): two-component
// points fit in 48 registers without spills (5 CTAs per SM instead of 4);
// three-component ones in 64 with 40 bytes of spills in the rarely taken
// Stacey solve (4 CTAs instead of 3).
template <int NC>
constexpr int kHaloRegs = NC == 2 ? 48 : 64;
template <int NC, bool ELASTIC>
static __global__ void __maxnreg__(kHaloRegs<NC>)
    halo_step_kernel(TiledDev td, HaloDev hd, CouplingDev cp, const float* __restrict__ other, int32_t other_ng,
                     bool pm, const float* __restrict__ amp, int32_t n_amp, StepScalars sc, double h_damp,
                     const StepState* __restrict__ st, double* __restrict__ epartial, int32_t epart0) {
  halo_step_body<NC, ELASTIC>(td, hd, cp, other, other_ng, pm, amp, n_amp, sc, h_damp, st, epartial,
                              epart0 + blockIdx.x, blockIdx.x * blockDim.x + threadIdx.x);
}

// energy[sample] = (time, kinetic, potential) from the per-CTA partials of
// the tiled step: kinetic sums all sets, potential = -0.5 x each domain's
// u . f_int, elastic first (solver.cpp:673-678).  Partials of set d are
// [start_d, start_d + count_d).
__device__ __forceinline__ void tiled_energy_body(const double* __restrict__ epartial, int n_dom, int4 sets0, int4 sets1,
                                                  const StepState* __restrict__ st, int32_t energy_every, double dt,
                                                  double* __restrict__ energy, int32_t max_samples) {
  __shared__ double sh[kReduceThreads];
  const int mode = st->mode;
  const int32_t step = st->step;
  const bool on = (mode == kModeInit) ? (energy_every > 0) : (energy_every > 0 && step % energy_every == 0);
  if (!on) return;
  const int starts[4] = {sets0.x, sets0.z, sets1.x, sets1.z};
  const int counts[4] = {sets0.y, sets0.w, sets1.y, sets1.w};
  double kin = 0.0, pot = 0.0;
  for (int d = 0; d < n_dom; ++d) {
    double pk = 0.0, pp = 0.0;
    // two partial sets per domain: tiles (set 2d) and halo (set 2d + 1)
    for (int part = 0; part < 2; ++part) {
      const int q = 2 * d + part;
      double sk = 0.0, spp = 0.0;
      for (int i = threadIdx.x; i < counts[q]; i += blockDim.x) {
        sk = dadd(sk, epartial[2 * (starts[q] + i)]);
        spp = dadd(spp, epartial[2 * (starts[q] + i) + 1]);
      }
      const double bk = block_reduce(sk, sh);
      __syncthreads();
      const double bp = block_reduce(spp, sh);
      __syncthreads();
      pk = dadd(pk, bk);
      pp = dadd(pp, bp);
    }
    kin = dadd(kin, pk);
    pot = dsub(pot, dmul(0.5, pp));
  }
  if (threadIdx.x == 0) {
    const int32_t sample = energy_every > 0 ? step / energy_every : 0;
    if (sample < max_samples) {
      energy[sample * 3 + 0] = dmul(static_cast<double>(step), dt);
      energy[sample * 3 + 1] = kin;
      energy[sample * 3 + 2] = pot;
    }
  }
}

static __global__ void tiled_energy_kernel(const double* __restrict__ epartial, int n_dom, int4 sets0, int4 sets1,
                                           const StepState* __restrict__ st, int32_t energy_every, double dt,
                                           double* __restrict__ energy, int32_t max_samples) {
  tiled_energy_body(epartial, n_dom, sets0, sets1, st, energy_every, dt, energy, max_samples);
}

// ------------------------------------------------------- batched step kernels
// The point-wise kernels of many solves in one launch each: one CTA per work
// item (segment, chunk); the segment carries one solve's pointers and
// scalars, the solve's StepState its step, mode and buffer parity.
constexpr int kHaloChunk = 256;
constexpr int kConsChunk = 128;
constexpr int kRecChunk = 64;

struct HaloSeg {
  TiledDev td;          // parity-0 view
  HaloDev hd;
  CouplingDev cp;
  const float* other0;  // coupling input at parity 0 / 1 (fluid u, or the solid's a at both)
  const float* other1;
  int32_t other_ng;
  int32_t pm;
  const float* amp;
  int32_t n_amp;
  StepScalars sc;
  double h_damp;
  const StepState* st;
  double* epartial;
  int32_t epart0;
};

template <int NC, bool ELASTIC>
static __global__ void __maxnreg__(kHaloRegs<NC>) halo_batch_kernel(const HaloSeg* __restrict__ segs,
                                                                         const int2* __restrict__ items) {
  const int2 it = items[blockIdx.x];
  const HaloSeg& sg = segs[it.x];
  if (sg.st->mode == kModeIdle) return;
  const int par = sg.st->parity;
  TiledDev td = sg.td;
  if (par) {
    const float* cur = td.u_cur;
    td.u_cur = td.u_nxt;
    td.u_nxt = const_cast<float*>(cur);
  }
  halo_step_body<NC, ELASTIC>(td, sg.hd, sg.cp, par ? sg.other1 : sg.other0, sg.other_ng, sg.pm != 0, sg.amp,
                              sg.n_amp, sg.sc, sg.h_damp, sg.st, sg.epartial, sg.epart0 + it.y,
                              it.y * kHaloChunk + static_cast<int32_t>(threadIdx.x));
}

struct ConsSeg {
  int32_t n;
  const int32_t* row_of;
  RowsDev rows;
  const float* u0;
  const float* u1;
  int32_t ng, ncomp;
  float* cval;
  const StepState* st;
};

static __global__ void __launch_bounds__(kConsChunk) constrained_batch_kernel(const ConsSeg* __restrict__ segs,
                                                                               const int2* __restrict__ items) {
  const int2 it = items[blockIdx.x];
  const ConsSeg& sg = segs[it.x];
  if (sg.st->mode == kModeIdle) return;
  constrained_gather_body(sg.n, sg.row_of, sg.rows, sg.st->parity ? sg.u1 : sg.u0, sg.ng, sg.ncomp, sg.cval,
                          it.y * kConsChunk + static_cast<int32_t>(threadIdx.x));
}

struct RecSeg {
  ReceiversDev rv;
  AllFields f0, f1;     // fields at parity 0 / 1
  const int32_t* acoustic_recv;
  int32_t n_acoustic;
  double dt;
  const RecordColumn* cols;
  int32_t n_cols;
  const StepState* st;
  int32_t record_every;
  double* traces;
  int32_t max_samples;
};

static __global__ void __launch_bounds__(kRecChunk) particle_velocity_batch_kernel(const RecSeg* __restrict__ segs,
                                                                                   const int2* __restrict__ items) {
  const int2 it = items[blockIdx.x];
  const RecSeg& sg = segs[it.x];
  if (sg.st->mode == kModeIdle) return;
  particle_velocity_body(sg.rv, sg.st->parity ? sg.f1 : sg.f0, sg.acoustic_recv, sg.n_acoustic, sg.dt, 0,
                         it.y * kRecChunk + static_cast<int32_t>(threadIdx.x));
}

static __global__ void __launch_bounds__(kRecChunk) record_batch_kernel(const RecSeg* __restrict__ segs,
                                                                        const int2* __restrict__ items) {
  const int2 it = items[blockIdx.x];
  const RecSeg& sg = segs[it.x];
  if (sg.st->mode == kModeIdle) return;
  record_body(sg.rv, sg.st->parity ? sg.f1 : sg.f0, sg.cols, sg.n_cols, sg.st->step, sg.record_every, sg.traces,
              sg.max_samples, it.y * kRecChunk + static_cast<int32_t>(threadIdx.x));
}

struct EnergySeg {
  const double* epartial;
  int32_t n_dom;
  int4 s0, s1;
  const StepState* st;
  int32_t energy_every;
  double dt;
  double* energy;
  int32_t max_samples;
};

static __global__ void __launch_bounds__(kReduceThreads) energy_batch_kernel(const EnergySeg* __restrict__ segs) {
  const EnergySeg& sg = segs[blockIdx.x];
  if (sg.st->mode == kModeIdle) return;
  tiled_energy_body(sg.epartial, sg.n_dom, sg.s0, sg.s1, sg.st, sg.energy_every, sg.dt, sg.energy, sg.max_samples);
}

// First kernel of a batched step: every solve's step counter, buffer parity
// and mode (final on its last step, idle after it).
static __global__ void batch_begin_kernel(StepState* const* __restrict__ sts, int32_t n) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    StepState* s = sts[i];
    if (s->step >= s->last_step) {
      s->mode = kModeIdle;
    } else {
      s->step += 1;
      s->parity ^= 1;
      s->mode = s->step == s->last_step ? kModeFinal : kModeNormal;
    }
  }
}

}  // namespace insem_b200
