// Element-forces kernel templates and their per-ngll launchers.
//
// One CTA stages EPB elements (EPB * npe threads, one per element point):
//   1. the element field into shared memory -- from an element-local array
//      (the per-block seam) or gathered from the global field through the
//      local-to-global map and the constraint rows (fused DofMap::gather);
//   2. fluxes and hoop/axis terms per point (element_fluxes);
//   3. the weak divergence per point (element_divergence), written to the
//      element-local force array.
// The launchers are compiled once per ngll (element_ng.cu with
// INSEM_NG = 2..9) so the 160 instantiations build in parallel.
#pragma once

#include "element_ops.cuh"

namespace insem_b200 {

// Value of slot k of element e, component c, of a global field
// (DofMap::gather, dof_map.hpp:95-120): direct, or the constraint row's
// weighted sum in row order starting from zero.
__device__ __forceinline__ float gather_slot(const float* __restrict__ g, int32_t m, const RowsDev& rows) {
  if (m >= 0) return __ldg(g + m);
  const int32_t r = -1 - m;
  float s = 0.0f;
  for (int32_t q = rows.offsets[r]; q < rows.offsets[r + 1]; ++q) s = fadd(s, fmul(rows.weights[q], __ldg(g + rows.dofs[q])));
  return s;
}

template <int NG, int KIND, bool ELASTIC, int M, bool GATHER>
__global__ void __launch_bounds__(ElemCfg<NG, KIND, ELASTIC, M>::THREADS)
    element_forces_kernel(BasisDev basis, BlockDev blk, const float* __restrict__ u_in,
                          const int32_t* __restrict__ l2g, RowsDev rows, int32_t n_global,
                          float* __restrict__ f_local) {
  using C = ElemCfg<NG, KIND, ELASTIC, M>;
  __shared__ ElemSmem<C> sm;
  const int tid = threadIdx.x;
  for (int t = tid; t < C::NPE; t += C::THREADS) {
    sm.D[t] = basis.D[t];
    sm.w2[t] = basis.w2[t];
    if constexpr (C::AXI) sm.Dj[t] = basis.Dj ? basis.Dj[t] : 0.0f;
  }
  const int el = tid / C::NPE;
  const int kpt = tid - el * C::NPE;
  const int bb = blockIdx.x * C::EPB + el;
  const bool active = bb < blk.n;
  int e = 0;
  bool axial = false;
  if (active) {
    e = blk.elements[bb];
    if constexpr (C::AXI) axial = blk.axial[bb] != 0;
    if constexpr (GATHER) {
      const int32_t m = l2g[static_cast<size_t>(e) * C::NPE + kpt];
#pragma unroll
      for (int c = 0; c < C::NC; ++c) sm.u[el][c][kpt] = gather_slot(u_in + static_cast<size_t>(c) * n_global, m, rows);
    } else {
#pragma unroll
      for (int c = 0; c < C::NC; ++c) sm.u[el][c][kpt] = u_in[(static_cast<size_t>(e) * C::NC + c) * C::NPE + kpt];
    }
  }
  __syncthreads();
  float direct[2] = {0.0f, 0.0f};
  const float* Dx = (C::AXI && axial) ? sm.Dj : sm.D;
  if (active) {
    element_fluxes<NG, KIND, ELASTIC, M>(blk, bb, kpt, axial, Dx, sm.D, sm.w2, sm.u[el], sm.f1[el], sm.f2[el],
                                         sm.gx[el][0], sm.gy[el][0], sm.gx[el][C::NAX - 1],
                                         sm.gy[el][C::NAX - 1], direct);
  }
  __syncthreads();
  if (active) {
    float out[C::NC];
    element_divergence<NG, KIND, ELASTIC, M>(kpt, axial, Dx, sm.D, sm.f1[el], sm.f2[el], sm.gx[el][0],
                                             sm.gy[el][0], sm.gx[el][C::NAX - 1], sm.gy[el][C::NAX - 1],
                                             direct, out);
#pragma unroll
    for (int c = 0; c < C::NC; ++c) f_local[(static_cast<size_t>(e) * C::NC + c) * C::NPE + kpt] = out[c];
  }
}

// Arguments of one element-forces launch.
struct ElementLaunch {
  BasisDev basis;
  BlockDev blk;
  const float* u_in = nullptr;     // element-local field, or global field when gathering
  const int32_t* l2g = nullptr;    // gathering only
  RowsDev rows;                    // gathering only
  int32_t n_global = 0;            // gathering only
  float* f_local = nullptr;
  bool gather = false;
  bool elastic = false;
  // load the kernel this launch would run (its module, under lazy loading)
  // without launching it
  bool preload = false;
  cudaStream_t stream = nullptr;
};

template <int NG, int KIND, bool ELASTIC, int M>
void launch_element_cfg(const ElementLaunch& a) {
  using C = ElemCfg<NG, KIND, ELASTIC, M>;
  if (a.blk.n <= 0) return;
  if (a.preload) {
    cudaFuncAttributes fa;
    if (a.gather) CUDA_CHECK(cudaFuncGetAttributes(&fa, element_forces_kernel<NG, KIND, ELASTIC, M, true>));
    else CUDA_CHECK(cudaFuncGetAttributes(&fa, element_forces_kernel<NG, KIND, ELASTIC, M, false>));
    return;
  }
  const int grid = ceil_div(a.blk.n, C::EPB);
  if (a.gather) {
    element_forces_kernel<NG, KIND, ELASTIC, M, true>
        <<<grid, C::THREADS, 0, a.stream>>>(a.basis, a.blk, a.u_in, a.l2g, a.rows, a.n_global, a.f_local);
  } else {
    element_forces_kernel<NG, KIND, ELASTIC, M, false>
        <<<grid, C::THREADS, 0, a.stream>>>(a.basis, a.blk, a.u_in, a.l2g, a.rows, a.n_global, a.f_local);
  }
  CUDA_LAUNCH_CHECK();
}

template <int NG>
void launch_element_ng(const ElementLaunch& a) {
  const int kind = a.blk.kind, m = a.blk.m;
  if (kind == INSEM_AXISYM) {
    if (m == 1) {
      a.elastic ? launch_element_cfg<NG, INSEM_AXISYM, true, 1>(a) : launch_element_cfg<NG, INSEM_AXISYM, false, 1>(a);
    } else {
      a.elastic ? launch_element_cfg<NG, INSEM_AXISYM, true, 0>(a) : launch_element_cfg<NG, INSEM_AXISYM, false, 0>(a);
    }
    return;
  }
  switch (kind) {
    case INSEM_RECT:
      a.elastic ? launch_element_cfg<NG, INSEM_RECT, true, 0>(a) : launch_element_cfg<NG, INSEM_RECT, false, 0>(a);
      break;
    case INSEM_AFFINE:
      a.elastic ? launch_element_cfg<NG, INSEM_AFFINE, true, 0>(a) : launch_element_cfg<NG, INSEM_AFFINE, false, 0>(a);
      break;
    case INSEM_CURVED:
      a.elastic ? launch_element_cfg<NG, INSEM_CURVED, true, 0>(a) : launch_element_cfg<NG, INSEM_CURVED, false, 0>(a);
      break;
    default:
      throw Error(INSEM_CUDA_ERR_UNSUPPORTED, "unknown geometry kind " + std::to_string(kind));
  }
}

// Per-ngll launchers (defined in element_ng.cu, one object per ngll).
void launch_element_ng2(const ElementLaunch&);
void launch_element_ng3(const ElementLaunch&);
void launch_element_ng4(const ElementLaunch&);
void launch_element_ng5(const ElementLaunch&);
void launch_element_ng6(const ElementLaunch&);
void launch_element_ng7(const ElementLaunch&);
void launch_element_ng8(const ElementLaunch&);
void launch_element_ng9(const ElementLaunch&);

// Dispatch on the number of GLL points; unsupported values fail like
// physics::select (kernels.cpp:451-468).
void launch_element_forces(int ngll, const ElementLaunch& a);

}  // namespace insem_b200
