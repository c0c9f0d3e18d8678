// Tile-kernel launchers and the constant-memory basis for one number of GLL
// points, selected with -DINSEM_NG=<2..9> (one object per value).  Every
// object has its own copy of c_basis; the host writes the entry of this
// object's ngll through set_constant_basis_ng<N>, once per device and part.
#include "tiled_path.cuh"

#ifndef INSEM_NG
#error "compile with -DINSEM_NG=<number of GLL points>"
#endif

#define INSEM_CAT2(a, b) a##b
#define INSEM_CAT(a, b) INSEM_CAT2(a, b)

namespace insem_b200 {

void INSEM_CAT(launch_tiles_ng, INSEM_NG)(const TileLaunch& a) { launch_tiles_cfg<INSEM_NG>(a); }

// Writes the given parts of this ngll's constant basis (a null part is left as it is).
void INSEM_CAT(set_constant_basis_ng, INSEM_NG)(const float* D, const float* Dj, const float* w2) {
  constexpr int n = INSEM_NG * INSEM_NG;
  const float* parts[3] = {D, Dj, w2};
  for (int which = 0; which < 3; ++which) {
    if (!parts[which]) continue;
    float buf[81] = {};
    for (int q = 0; q < n; ++q) buf[q] = parts[which][q];
    CUDA_CHECK(cudaMemcpyToSymbol(c_basis, buf, sizeof(buf), sizeof(float) * 81 * (3 * (INSEM_NG - 2) + which)));
  }
  const float neg_zero = -0.0f;
  CUDA_CHECK(cudaMemcpyToSymbol(c_neg_zero, &neg_zero, sizeof(float)));
}

int INSEM_CAT(tile_elements_ng, INSEM_NG)() { return TileCfg<INSEM_NG>::TE; }

int INSEM_CAT(tile_step_occupancy_ng, INSEM_NG)(int kind, bool elastic, int m, int te, uint32_t smem) {
  return tile_step_occupancy_cfg<INSEM_NG>(kind, elastic, m, te, smem);
}

int INSEM_CAT(tile_batch_ng, INSEM_NG)(const TileBatchLaunch& a, bool launch) {
  return tile_batch_cfg<INSEM_NG>(a, launch);
}

}  // namespace insem_b200
