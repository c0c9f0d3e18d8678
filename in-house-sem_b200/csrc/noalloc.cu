// Internal forces of one domain without any device allocation.
//
// insem_cuda_solver_internal_forces takes host arrays. It copies them through
// device buffers it allocates, and on first use it allocates the two-pass
// path's field buffers. Some callers cannot let a library allocate device
// memory on its own:
// - applications whose device memory is owned by another allocator (a
//   framework's caching pool that has reserved the GPU), where a cudaMalloc
//   fails or fragments that pool;
// - latency-sensitive loops sharing the GPU with other work, where
//   cudaFree's wait for the whole device would stall everything else.
// For them, insem_cuda_solver_internal_forces_noalloc takes the field and
// the result as device arrays the caller owns. Its one piece of scratch, the
// element-local force vectors between the element kernels and the assembly,
// lives in a fixed array compiled into this file.
//
// Under lazy module loading (the CUDA default since 12.2) the driver loads a
// module, and reserves its device memory, the first time something in it is
// used. Creating a solver therefore loads this file's array and the kernels
// the entry point runs, on the solver's device (prepare_noalloc); from then
// on that GPU holds the array until the process exits, and the entry point's
// calls load nothing.
#include "solver.cuh"

namespace insem_b200 {
namespace {

// Element-local forces: ncomp x elements x ngll^2 floats, at most 16 MiB.
constexpr std::size_t kNoAllocScratchFloats = std::size_t{1} << 22;
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];

// In host code g_noalloc_scratch names a host-side stand-in, not device
// memory: kernels get the device address, looked up on the current device at
// every call (a host-side lookup; nothing is cached, so a context that was
// torn down and created again is addressed afresh).
float* scratch_on_current_device() {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(INSEM_CUDA_ERR_CUDA, std::string("cannot address the scratch array: ") + cudaGetErrorString(e));
  }
  return static_cast<float*>(p);
}

}  // namespace

void Solver::prepare_noalloc() {
  scratch_on_current_device();
  for (const DeviceDomainData& d : domains) {
    for (const DeviceBlock& b : d.blocks) {
      ElementLaunch a;
      a.blk = b.view();
      a.gather = true;
      a.elastic = d.medium == INSEM_ELASTIC;
      a.preload = true;
      launch_element_forces(ngll, a);
    }
    preload_assemble(d.dofs.weighted);
  }
}

void Solver::internal_forces_noalloc(int32_t di, const float* u_global, float* f_global, cudaStream_t s) {
  INSEM_REQUIRE(di >= 0 && di < static_cast<int32_t>(domains.size()), INSEM_CUDA_ERR_INVALID, "domain out of range");
  DeviceDomainData& d = domains[di];
  const std::size_t need = static_cast<std::size_t>(d.ncomp) * d.n_elements * d.npe;
  INSEM_REQUIRE(need <= kNoAllocScratchFloats, INSEM_CUDA_ERR_UNSUPPORTED,
                "the domain's element-local forces need " + std::to_string(need) +
                    " floats; the allocation-free entry point holds at most " +
                    std::to_string(kNoAllocScratchFloats) + " (use insem_cuda_solver_internal_forces)");
  float* scratch = scratch_on_current_device();
  // the array keeps the previous call's values: start from zeros
  CUDA_CHECK(cudaMemsetAsync(scratch, 0, need * sizeof(float), s));
  for (const DeviceBlock& b : d.blocks) {
    ElementLaunch a;
    a.basis = basis.view();
    a.blk = b.view();
    a.u_in = u_global;
    a.l2g = d.dofs.l2g.get();
    a.rows = d.dofs.rows();
    a.n_global = d.ng;
    a.f_local = scratch;
    a.gather = true;
    a.elastic = d.medium == INSEM_ELASTIC;
    a.stream = s;
    launch_element_forces(ngll, a);
  }
  launch_assemble(d.dofs, d.ncomp, scratch, f_global, s);
}

}  // namespace insem_b200

using namespace insem_b200;

extern "C" int insem_cuda_solver_internal_forces_noalloc(insem_cuda_solver* h, int32_t domain, const float* u,
                                                         float* f, void* stream) {
  return guarded([&] {
    INSEM_REQUIRE(h && u && f, INSEM_CUDA_ERR_INVALID, "null argument");
    Solver& s = *h->s;
    DeviceGuard dg(s.device);
    s.internal_forces_noalloc(domain, u, f, static_cast<cudaStream_t>(stream));
  });
}
