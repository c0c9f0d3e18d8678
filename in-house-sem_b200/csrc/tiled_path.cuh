// Host side of the tiled fused step: tiling, device numbering and launches.
#pragma once

#include <map>
#include <vector>

#include "device_data.cuh"
#include "tiled.cuh"

namespace insem_b200 {

// Per-point special terms of one domain, in the reference's point numbering.
struct SpecialTerms {
  std::map<int32_t, std::vector<std::pair<int32_t, std::vector<float>>>> sources;  // point -> (source, coef[ncomp])
  std::map<int32_t, std::vector<int32_t>> coupling;                               // point -> coupling entries
  std::map<int32_t, int32_t> absorbing;                                           // point -> Stacey index
  std::map<int32_t, uint8_t> zero;                                                // point -> zeroed components
  std::vector<int32_t> receivers;                                                 // points read by receivers
};

// One domain of the tiled path.
class TiledDomain {
 public:
  // Builds tiles of at most `te` elements per block and the device numbering.
  void build(const insem_cuda_domain& d, int ngll, int te, const SpecialTerms& sp, const std::vector<float>& abs_coef);

  // ng: component stride of the device arrays (points padded so that every
  // tile's complete range starts on a 16-byte boundary); ng_ref: the
  // reference's point count.  Halo points are [n_complete, n_complete + n_halo).
  int medium = 0, ncomp = 1, m = 0, ng = 0, ng_ref = 0, npe = 0, n_elements = 0;
  int n_complete = 0, n_halo = 0, n_tiles = 0, tp_cap = 0, nc_cap = 0, n_hbuf = 0, n_cslots = 0;
  int rank_cap = 1;  // the most contributions one complete point of a tile has
  int te = 0;  // elements per tile (CTAs of tile_threads(te, ngll) threads)
  bool weighted = false;
  std::vector<int32_t> perm;  // reference point -> device point
  struct BlockTiles {
    int kind = 0, m = 0, tile0 = 0, ntiles = 0, n = 0, e_off = 0;
    DeviceBuffer<float> metric, coef0, coef1, wr, hoop, r;
    DeviceBuffer<uint8_t> axial;
    BlockDev view() const;
  };
  std::vector<BlockTiles> blocks;
  // device data
  DeviceBuffer<uint32_t> sdesc;
  DeviceBuffer<TileHdr> tiles;
  std::vector<TileHdr> host_tiles;  // the same headers on the host (the batched tile items copy them)
  DeviceBuffer<int32_t> halo_tp, hs_slot, hs_dst, mdst_off, mdst, cs_slot, cs_idx, cs_row;
  DeviceBuffer<float> cval, hbuf, mass, inv_mass;
  DeviceBuffer<float> u0, u1, v, a, vn;
  DeviceBuffer<int32_t> h_off, h_spec, src_off, src_which, cpl_off, cpl_idx, abs_idx;
  DeviceBuffer<float> h_w, src_coef, abs_coef_d;
  DeviceBuffer<uint8_t> zero;
  DeviceBuffer<int32_t> rows_off, rows_dofs;  // constraint rows in device numbering
  DeviceBuffer<float> rows_w;
  RowsDev rows() const { return {rows_off.get(), rows_dofs.get(), rows_w.get()}; }
  std::vector<float> host_mass;

  TiledDev view(int parity) const;  // parity 0: u0 current, u1 next
  HaloDev halo_view() const;
  float* u_cur(int parity) { return parity ? u1.get() : u0.get(); }
};

// Launchers, instantiated per ngll in tiled_ng.cu.
struct TileLaunch {
  const TiledDomain* dom = nullptr;
  int block = 0;
  int parity = 0;
  StepScalars sc{};
  StepState* st = nullptr;
  double* epartial = nullptr;
  bool elastic = false;
  cudaStream_t stream = nullptr;
};
void launch_tiles_ng2(const TileLaunch&);
void launch_tiles_ng3(const TileLaunch&);
void launch_tiles_ng4(const TileLaunch&);
void launch_tiles_ng5(const TileLaunch&);
void launch_tiles_ng6(const TileLaunch&);
void launch_tiles_ng7(const TileLaunch&);
void launch_tiles_ng8(const TileLaunch&);
void launch_tiles_ng9(const TileLaunch&);
void launch_tiles(int ngll, const TileLaunch& a);
int tile_elements(int ngll);  // TileCfg<NG>::TE (the largest tile)
// Elements per tile of a domain: `requested` if > 0, else a registered entry
// (set_tile_elements, e.g. from the autotuner), else the analytic choice that
// keeps the most elements resident per SM with several CTAs per SM.
int choose_tile_elements(int ngll, int kind, bool elastic, int m, int ncomp, int requested);
void set_tile_elements(int ngll, int kind, bool elastic, int m, int te);  // te <= 0 clears the entry
int analytic_tile_elements(int ngll, int kind, bool elastic, int m, int ncomp);
// CTAs per SM of the plain tile kernel of a class at te elements and smem
// bytes of dynamic shared memory (registers, shared memory and threads as
// the current device counts them); -1 if the device cannot be asked.
int tile_step_occupancy(int ngll, int kind, bool elastic, int m, int te, uint32_t smem);
int tile_step_occupancy_ng2(int kind, bool elastic, int m, int te, uint32_t smem);
int tile_step_occupancy_ng3(int kind, bool elastic, int m, int te, uint32_t smem);
int tile_step_occupancy_ng4(int kind, bool elastic, int m, int te, uint32_t smem);
int tile_step_occupancy_ng5(int kind, bool elastic, int m, int te, uint32_t smem);
int tile_step_occupancy_ng6(int kind, bool elastic, int m, int te, uint32_t smem);
int tile_step_occupancy_ng7(int kind, bool elastic, int m, int te, uint32_t smem);
int tile_step_occupancy_ng8(int kind, bool elastic, int m, int te, uint32_t smem);
int tile_step_occupancy_ng9(int kind, bool elastic, int m, int te, uint32_t smem);

template <int NG>
int tile_step_occupancy_cfg(int kind, bool elastic, int m, int te, uint32_t smem) {
  auto ask = [&](auto kernel) -> int {
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess) {
      cudaGetLastError();
      return -1;
    }
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, tile_threads(te, NG), smem) != cudaSuccess) {
      cudaGetLastError();
      return -1;
    }
    return nb;
  };
  if (kind == INSEM_AXISYM) {
    if (m == 1) return elastic ? ask(tile_step_kernel<NG, INSEM_AXISYM, true, 1>) : ask(tile_step_kernel<NG, INSEM_AXISYM, false, 1>);
    return elastic ? ask(tile_step_kernel<NG, INSEM_AXISYM, true, 0>) : ask(tile_step_kernel<NG, INSEM_AXISYM, false, 0>);
  }
  switch (kind) {
    case INSEM_RECT:
      return elastic ? ask(tile_step_kernel<NG, INSEM_RECT, true, 0>) : ask(tile_step_kernel<NG, INSEM_RECT, false, 0>);
    case INSEM_AFFINE:
      return elastic ? ask(tile_step_kernel<NG, INSEM_AFFINE, true, 0>) : ask(tile_step_kernel<NG, INSEM_AFFINE, false, 0>);
    default:
      return elastic ? ask(tile_step_kernel<NG, INSEM_CURVED, true, 0>) : ask(tile_step_kernel<NG, INSEM_CURVED, false, 0>);
  }
}
// Uploads the GLL / GLJ basis of one ngll to constant memory (must agree with earlier uploads).
void set_constant_basis(int ngll, const std::vector<float>& D, const std::vector<float>& Dj,
                        const std::vector<float>& w2);

// Batched tile launches: one launch per tile class (ngll, kind, medium,
// order) over the work items of many solves, one CTA per item.
struct TileBatchLaunch {
  int kind = 0, m = 0;
  bool elastic = false;
  const TileSeg* segs = nullptr;
  const TileItem* items = nullptr;
  int te = 0;      // elements per tile of the class (CTA size tile_threads(te, ngll))
  TileLayout L{};  // the class layout; its total is the dynamic shared memory
  uint32_t smem = 0;
  int grid = 0;
  cudaStream_t stream = nullptr;
};
// launch == false: sets the class kernel's dynamic shared memory (outside
// stream capture) and returns its resident CTAs per SM; true: launches.
int tile_batch_ng2(const TileBatchLaunch&, bool launch);
int tile_batch_ng3(const TileBatchLaunch&, bool launch);
int tile_batch_ng4(const TileBatchLaunch&, bool launch);
int tile_batch_ng5(const TileBatchLaunch&, bool launch);
int tile_batch_ng6(const TileBatchLaunch&, bool launch);
int tile_batch_ng7(const TileBatchLaunch&, bool launch);
int tile_batch_ng8(const TileBatchLaunch&, bool launch);
int tile_batch_ng9(const TileBatchLaunch&, bool launch);
int tile_batch(int ngll, const TileBatchLaunch& a, bool launch);

template <int NG>
int tile_batch_cfg(const TileBatchLaunch& a, bool launch) {
  INSEM_REQUIRE(a.smem <= 227u * 1024u, INSEM_CUDA_ERR_UNSUPPORTED, "tile needs too much shared memory");
  auto go = [&](auto kernel) -> int {
    if (!launch) {
      CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(a.smem)));
      int nb = 0;
      CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, tile_threads(a.te, NG), a.smem));
      return nb;
    }
    INSEM_REQUIRE(a.te >= 1 && a.te <= TileCfg<NG>::TE, INSEM_CUDA_ERR_INVALID, "tile elements out of range");
    kernel<<<a.grid, tile_threads(a.te, NG), a.smem, a.stream>>>(a.segs, a.items, a.L);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess)
      throw Error(INSEM_CUDA_ERR_CUDA, "batched tile kernel launch (ngll " + std::to_string(NG) + ", kind " +
                                           std::to_string(a.kind) + ", grid " + std::to_string(a.grid) + ", smem " +
                                           std::to_string(a.smem) + "): " + cudaGetErrorString(err));
    return 0;
  };
  if (a.kind == INSEM_AXISYM) {
    if (a.elastic) {
      if constexpr (kBatchRegs<NG, 1> > 0)
        if (a.m == 1) return go(tile_batch_kernel_capped<NG, INSEM_AXISYM, true, 1, kBatchRegs<NG, 1>>);
      if constexpr (kBatchRegs<NG, 0> > 0)
        if (a.m == 0) return go(tile_batch_kernel_capped<NG, INSEM_AXISYM, true, 0, kBatchRegs<NG, 0>>);
    }
    if (a.m == 1) return a.elastic ? go(tile_batch_kernel<NG, INSEM_AXISYM, true, 1>)
                                   : go(tile_batch_kernel<NG, INSEM_AXISYM, false, 1>);
    return a.elastic ? go(tile_batch_kernel<NG, INSEM_AXISYM, true, 0>) : go(tile_batch_kernel<NG, INSEM_AXISYM, false, 0>);
  }
  switch (a.kind) {
    case INSEM_RECT:
      return a.elastic ? go(tile_batch_kernel<NG, INSEM_RECT, true, 0>) : go(tile_batch_kernel<NG, INSEM_RECT, false, 0>);
    case INSEM_AFFINE:
      return a.elastic ? go(tile_batch_kernel<NG, INSEM_AFFINE, true, 0>)
                       : go(tile_batch_kernel<NG, INSEM_AFFINE, false, 0>);
    default:
      return a.elastic ? go(tile_batch_kernel<NG, INSEM_CURVED, true, 0>)
                       : go(tile_batch_kernel<NG, INSEM_CURVED, false, 0>);
  }
}

template <int NG>
void launch_tiles_cfg(const TileLaunch& a) {
  const TiledDomain& d = *a.dom;
  const auto& b = d.blocks[a.block];
  if (b.ntiles == 0) return;
  auto go = [&](auto kernel, int nc) {
    INSEM_REQUIRE(d.te >= 1 && d.te <= TileCfg<NG>::TE, INSEM_CUDA_ERR_INVALID, "tile elements out of range");
    const TileLayout L = TileLayout::make(NG, nc, b.kind, a.elastic, d.te, d.tp_cap, d.nc_cap, d.rank_cap);
    const size_t smem = L.total;
    // Opt in to this launch's dynamic shared memory (outside stream capture;
    // the first launch of every tile kernel happens in the uncaptured initial step).
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CUDA_CHECK(cudaStreamIsCapturing(a.stream, &cap));
    if (cap == cudaStreamCaptureStatusNone)
      CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    INSEM_REQUIRE(smem <= 227 * 1024, INSEM_CUDA_ERR_UNSUPPORTED, "tile needs too much shared memory");
    TiledDev td = d.view(a.parity);
    td.sdesc += static_cast<size_t>(b.e_off) * point_stride<NG * NG>();
    kernel<<<b.ntiles, tile_threads(d.te, NG), smem, a.stream>>>(b.view(), td, a.sc, a.st, a.epartial, b.tile0, L);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess)
      throw Error(INSEM_CUDA_ERR_CUDA, "tile kernel launch (ngll " + std::to_string(NG) + ", kind " +
                                           std::to_string(b.kind) + ", tiles " + std::to_string(b.ntiles) +
                                           ", threads " + std::to_string(tile_threads(d.te, NG)) + ", smem " +
                                           std::to_string(smem) + "): " + cudaGetErrorString(err));
  };
  if (b.kind == INSEM_AXISYM) {
    if (b.m == 1) {
      if (a.elastic) go(tile_step_kernel<NG, INSEM_AXISYM, true, 1>, 3);
      else go(tile_step_kernel<NG, INSEM_AXISYM, false, 1>, 1);
    } else {
      if (a.elastic) go(tile_step_kernel<NG, INSEM_AXISYM, true, 0>, 2);
      else go(tile_step_kernel<NG, INSEM_AXISYM, false, 0>, 1);
    }
    return;
  }
  switch (b.kind) {
    case INSEM_RECT:
      if (a.elastic) go(tile_step_kernel<NG, INSEM_RECT, true, 0>, 2);
      else go(tile_step_kernel<NG, INSEM_RECT, false, 0>, 1);
      break;
    case INSEM_AFFINE:
      if (a.elastic) go(tile_step_kernel<NG, INSEM_AFFINE, true, 0>, 2);
      else go(tile_step_kernel<NG, INSEM_AFFINE, false, 0>, 1);
      break;
    default:
      if (a.elastic) go(tile_step_kernel<NG, INSEM_CURVED, true, 0>, 2);
      else go(tile_step_kernel<NG, INSEM_CURVED, false, 0>, 1);
      break;
  }
}

}  // namespace insem_b200
