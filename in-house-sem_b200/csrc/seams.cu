// C-ABI entry points of the per-block kernel seam and the DofMap seam, the
// gather / assemble kernels, and the library-wide error state.
//
//   insem_cuda_block_*   <-> physics::{elastic,acoustic}_internal_forces (kernels.hpp:32-35)
//   insem_cuda_dofmap_*  <-> ops::DofMap::gather / assemble             (dof_map.hpp:73-77)
#include "device_data.cuh"

namespace insem_b200 {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

void launch_element_forces(int ngll, const ElementLaunch& a) {
  switch (ngll) {
    case 2: launch_element_ng2(a); break;
    case 3: launch_element_ng3(a); break;
    case 4: launch_element_ng4(a); break;
    case 5: launch_element_ng5(a); break;
    case 6: launch_element_ng6(a); break;
    case 7: launch_element_ng7(a); break;
    case 8: launch_element_ng8(a); break;
    case 9: launch_element_ng9(a); break;
    default: check_ngll(ngll);
  }
}

// ------------------------------------------------------- gather / assemble
// DofMap::gather (dof_map.hpp:95-120): one thread per element slot.
__global__ void gather_kernel(const int32_t* __restrict__ l2g, RowsDev rows, int32_t n_slots, int32_t npe,
                              int32_t ncomp, int32_t n_global, const float* __restrict__ global,
                              float* __restrict__ local) {
  const int32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots) return;
  const int32_t e = s / npe, k = s - e * npe;
  const int32_t m = l2g[s];
  for (int c = 0; c < ncomp; ++c)
    local[(static_cast<size_t>(e) * ncomp + c) * npe + k] =
        gather_slot(global + static_cast<size_t>(c) * n_global, m, rows);
}

// DofMap::assemble (dof_map.hpp:123-141): one thread per global point, its
// contributions summed in ascending slot order from zero.
template <bool WEIGHTED>
__global__ void assemble_kernel(const int32_t* __restrict__ t_offsets, const int32_t* __restrict__ t_slots,
                                const float* __restrict__ t_weights, int32_t n_global, int32_t npe,
                                int32_t ncomp, const float* __restrict__ local, float* __restrict__ global) {
  const int32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_global) return;
  const int32_t b = t_offsets[g], en = t_offsets[g + 1];
  for (int c = 0; c < ncomp; ++c) {
    float sum = 0.0f;
    for (int32_t q = b; q < en; ++q) {
      const int32_t slot = t_slots[q];
      const int32_t e = slot / npe, k = slot - e * npe;
      const float v = local[(static_cast<size_t>(e) * ncomp + c) * npe + k];
      sum = fadd(sum, WEIGHTED ? fmul(t_weights[q], v) : v);
    }
    global[static_cast<size_t>(c) * n_global + g] = sum;
  }
}

void launch_gather(const DeviceDofMap& d, int ncomp, const float* global, float* local, cudaStream_t s) {
  const int32_t n_slots = d.n_elements * d.npe;
  if (n_slots == 0) return;
  gather_kernel<<<ceil_div(n_slots, 256), 256, 0, s>>>(d.l2g.get(), d.rows(), n_slots, d.npe, ncomp, d.n_global,
                                                         global, local);
  CUDA_LAUNCH_CHECK();
}

void preload_assemble(bool weighted) {
  cudaFuncAttributes fa;
  if (weighted) CUDA_CHECK(cudaFuncGetAttributes(&fa, assemble_kernel<true>));
  else CUDA_CHECK(cudaFuncGetAttributes(&fa, assemble_kernel<false>));
}

void launch_assemble(const DeviceDofMap& d, int ncomp, const float* local, float* global, cudaStream_t s) {
  if (d.n_global == 0) return;
  if (d.weighted) {
    assemble_kernel<true><<<ceil_div(d.n_global, 256), 256, 0, s>>>(
        d.t_offsets.get(), d.t_slots.get(), d.t_weights.get(), d.n_global, d.npe, ncomp, local, global);
  } else {
    assemble_kernel<false><<<ceil_div(d.n_global, 256), 256, 0, s>>>(
        d.t_offsets.get(), d.t_slots.get(), nullptr, d.n_global, d.npe, ncomp, local, global);
  }
  CUDA_LAUNCH_CHECK();
}

}  // namespace insem_b200

using namespace insem_b200;

// ------------------------------------------------------------------ C ABI
struct insem_cuda_block_h {
  int device = 0;
  int medium = 0;
  int ncomp = 0;
  DeviceBasis basis;
  DeviceBlock block;
};

struct insem_cuda_dofmap_h {
  int device = 0;
  DeviceDofMap dofs;
};

extern "C" {

const char* insem_cuda_last_error(void) { return last_error(); }
const char* insem_cuda_version(void) { return "insem-b200 0.1.0"; }

int insem_cuda_mem_info(int32_t device, int64_t* free_bytes, int64_t* total_bytes) {
  return guarded([&] {
    DeviceGuard dg(device);
    std::size_t f = 0, t = 0;
    CUDA_CHECK(cudaMemGetInfo(&f, &t));
    if (free_bytes) *free_bytes = static_cast<int64_t>(f);
    if (total_bytes) *total_bytes = static_cast<int64_t>(t);
  });
}

int insem_cuda_block_create(const insem_cuda_basis* basis, const insem_cuda_block* block, int32_t medium,
                            int32_t device, insem_cuda_block_h** out) {
  return guarded([&] {
    INSEM_REQUIRE(basis && block && out, INSEM_CUDA_ERR_INVALID, "null argument");
    INSEM_REQUIRE(medium == INSEM_ACOUSTIC || medium == INSEM_ELASTIC, INSEM_CUDA_ERR_INVALID, "unknown medium");
    DeviceGuard dg(device);
    auto h = std::make_unique<insem_cuda_block_h>();
    h->device = device;
    h->medium = medium;
    h->ncomp = ncomp_of(medium, block->azimuthal_order);
    h->block.upload(*block, basis->ngll, medium);
    h->basis.upload(*basis, h->block.any_axial);
    *out = h.release();
  });
}

void insem_cuda_block_destroy(insem_cuda_block_h* h) {
  if (!h) return;
  DeviceGuard dg(h->device);
  delete h;
}

int insem_cuda_block_forces(insem_cuda_block_h* h, int32_t n_local_elements, const float* u_local,
                            float* f_local, void* stream) {
  return guarded([&] {
    INSEM_REQUIRE(h && u_local && f_local, INSEM_CUDA_ERR_INVALID, "null argument");
    for (int32_t e : h->block.host_elements)
      INSEM_REQUIRE(e >= 0 && e < n_local_elements, INSEM_CUDA_ERR_INVALID, "block element outside the local array");
    DeviceGuard dg(h->device);
    ElementLaunch a;
    a.basis = h->basis.view();
    a.blk = h->block.view();
    a.u_in = u_local;
    a.f_local = f_local;
    a.elastic = h->medium == INSEM_ELASTIC;
    a.stream = static_cast<cudaStream_t>(stream);
    launch_element_forces(h->basis.ngll, a);
  });
}

int insem_cuda_block_forces_host(insem_cuda_block_h* h, int32_t n_local_elements, const float* u_local,
                                 float* f_local) {
  return guarded([&] {
    INSEM_REQUIRE(h && u_local && f_local, INSEM_CUDA_ERR_INVALID, "null argument");
    DeviceGuard dg(h->device);
    const std::size_t n = static_cast<std::size_t>(n_local_elements) * h->ncomp * h->basis.ngll * h->basis.ngll;
    DeviceBuffer<float> du, df;
    du.upload(u_local, n);
    df.upload(f_local, n);  // elements outside the block keep their values
    const int rc = insem_cuda_block_forces(h, n_local_elements, du.get(), df.get(), nullptr);
    if (rc != INSEM_CUDA_OK) throw Error(rc, last_error());
    CUDA_CHECK(cudaMemcpy(f_local, df.get(), n * sizeof(float), cudaMemcpyDeviceToHost));
  });
}

int insem_cuda_dofmap_create(const insem_cuda_dofmap* dofs, int32_t device, insem_cuda_dofmap_h** out) {
  return guarded([&] {
    INSEM_REQUIRE(dofs && out, INSEM_CUDA_ERR_INVALID, "null argument");
    DeviceGuard dg(device);
    auto h = std::make_unique<insem_cuda_dofmap_h>();
    h->device = device;
    h->dofs.upload(*dofs);
    *out = h.release();
  });
}

void insem_cuda_dofmap_destroy(insem_cuda_dofmap_h* h) {
  if (!h) return;
  DeviceGuard dg(h->device);
  delete h;
}

int insem_cuda_gather(insem_cuda_dofmap_h* h, int32_t ncomp, const float* global, float* local, void* stream) {
  return guarded([&] {
    INSEM_REQUIRE(h && global && local && ncomp >= 1 && ncomp <= 3, INSEM_CUDA_ERR_INVALID, "invalid argument");
    DeviceGuard dg(h->device);
    launch_gather(h->dofs, ncomp, global, local, static_cast<cudaStream_t>(stream));
  });
}

int insem_cuda_assemble(insem_cuda_dofmap_h* h, int32_t ncomp, const float* local, float* global, void* stream) {
  return guarded([&] {
    INSEM_REQUIRE(h && global && local && ncomp >= 1 && ncomp <= 3, INSEM_CUDA_ERR_INVALID, "invalid argument");
    DeviceGuard dg(h->device);
    launch_assemble(h->dofs, ncomp, local, global, static_cast<cudaStream_t>(stream));
  });
}

}  // extern "C"
