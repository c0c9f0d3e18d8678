// Wavefield snapshots on the device (Solver::record_snapshot,
// cpp/src/solver/solver.cpp:813-839).
//
// At a snapshot step the solver's state is complete (the tiled path ends its
// span with a final-mode step), and one kernel per recorded field gathers it
// to element points: every element slot takes its point's value, or its
// hanging-node row summed in row order (DofMap::gather), and the azimuthal
// order 1 elastic pair (U+, U-) becomes (U_r, U_theta) in double, rounded to
// float, as the reference does.  The layout is the reference's:
// [component][element][ngll^2] per snapshot, in the reference's element
// order.  Each snapshot is copied to the host when it is taken, so device
// memory holds one snapshot at a time however many are recorded.
#include <algorithm>

#include "solver.cuh"

namespace insem_b200 {
namespace {

// One thread per element slot: `field` in the solver's point numbering
// (component stride ng), `l2g` the slot's point or -1 - its constraint row.
__global__ void snapshot_gather_kernel(const int32_t* __restrict__ l2g, RowsDev rows, const float* __restrict__ field,
                                       int64_t ng, int32_t ncomp, int64_t n_slots, int32_t rotate_pm,
                                       float* __restrict__ out) {
  const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (s >= n_slots) return;
  const int32_t m = l2g[s];
  float val[3];
  for (int c = 0; c < ncomp && c < 3; ++c) val[c] = gather_slot(field + c * ng, m, rows);
  if (rotate_pm) {
    constexpr double kSqrtHalf = 0.70710678118654752440;
    const double up = val[0], um = val[1];
    val[0] = static_cast<float>(__dmul_rn(kSqrtHalf, __dadd_rn(up, um)));
    val[1] = static_cast<float>(__dmul_rn(kSqrtHalf, __dsub_rn(up, um)));
  }
  for (int c = 0; c < ncomp && c < 3; ++c) out[c * n_slots + s] = val[c];
}

}  // namespace

void Solver::set_snapshots(int32_t every, int32_t n_quantities, const int32_t* quantities) {
  DeviceGuard dg(device);
  INSEM_REQUIRE(!initialized, INSEM_CUDA_ERR_STATE, "snapshots must be set before the first time step");
  INSEM_REQUIRE(!in_batch, INSEM_CUDA_ERR_STATE, "a solve that records snapshots is stepped on its own");
  INSEM_REQUIRE(every >= 0 && n_quantities >= 0 && (n_quantities == 0 || quantities), INSEM_CUDA_ERR_INVALID,
                "snapshot_every must be >= 0");
  snap_fields.clear();
  snap_times.clear();
  snap_every = 0;
  if (every == 0 || n_quantities == 0) return;
  // per quantity, every medium that has it, in domain order (the reference's Solver constructor)
  for (int32_t q = 0; q < n_quantities; ++q) {
    const int32_t qu = quantities[q];
    INSEM_REQUIRE(qu == INSEM_Q_DISPLACEMENT || qu == INSEM_Q_VELOCITY || qu == INSEM_Q_ACCELERATION ||
                      qu == INSEM_Q_PRESSURE,
                  INSEM_CUDA_ERR_INVALID, "unknown snapshot quantity (displacement, velocity, acceleration, pressure)");
    for (std::size_t di = 0; di < domains.size(); ++di) {
      const bool elastic = domains[di].medium == INSEM_ELASTIC;
      if (elastic ? qu == INSEM_Q_PRESSURE : qu != INSEM_Q_PRESSURE) continue;
      SnapField f;
      f.domain = static_cast<int32_t>(di);
      f.quantity = qu;
      f.ncomp = domains[di].ncomp;
      snap_fields.push_back(std::move(f));
    }
  }
  // element slot -> point of the field arrays (the tiled path renumbers points)
  snap_l2g.clear();
  std::size_t stage = 0;
  for (std::size_t di = 0; di < domains.size(); ++di) {
    DeviceDomainData& d = domains[di];
    std::vector<int32_t> l2g = d.dofs.l2g.download();
    if (tiled)
      for (int32_t& m : l2g)
        if (m >= 0) m = tdom[di].perm[m];
    snap_l2g.emplace_back();
    snap_l2g.back().upload(l2g);
    stage = std::max(stage, static_cast<std::size_t>(d.ncomp) * l2g.size());
  }
  snap_stage.resize(stage);
  snap_every = every;
}

void Solver::record_snapshot() {
  snap_times.push_back(step * dt);
  for (SnapField& f : snap_fields) {
    DeviceDomainData& d = domains[f.domain];
    const float* field;
    int64_t ng;
    RowsDev rows;
    if (tiled) {
      TiledDomain& t = tdom[f.domain];
      field = f.quantity == INSEM_Q_VELOCITY ? t.v.get() : f.quantity == INSEM_Q_ACCELERATION ? t.a.get()
                                                                                             : t.u_cur(parity);
      ng = t.ng;
      rows = t.rows();
    } else {
      field = f.quantity == INSEM_Q_VELOCITY ? d.v.get() : f.quantity == INSEM_Q_ACCELERATION ? d.a.get() : d.u.get();
      ng = d.ng;
      rows = d.dofs.rows();
    }
    const int64_t n_slots = static_cast<int64_t>(d.n_elements) * d.npe;
    const int32_t rotate = d.medium == INSEM_ELASTIC && d.m == 1 ? 1 : 0;
    snapshot_gather_kernel<<<grid_for(n_slots), 256, 0, stream>>>(snap_l2g[f.domain].get(), rows, field, ng, d.ncomp,
                                                                  n_slots, rotate, snap_stage.get());
    CUDA_LAUNCH_CHECK();
    const std::size_t n = static_cast<std::size_t>(d.ncomp) * n_slots;
    const std::size_t base = f.data.size();
    f.data.resize(base + n);
    CUDA_CHECK(cudaMemcpyAsync(f.data.data() + base, snap_stage.get(), n * sizeof(float), cudaMemcpyDeviceToHost,
                               stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
  }
}

}  // namespace insem_b200

using namespace insem_b200;

extern "C" {

int insem_cuda_solver_set_snapshots(insem_cuda_solver* h, int32_t every, int32_t n_quantities,
                                    const int32_t* quantities) {
  return guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    h->s->set_snapshots(every, n_quantities, quantities);
  });
}

int32_t insem_cuda_solver_n_snapshots(const insem_cuda_solver* h) {
  return h ? static_cast<int32_t>(h->s->snap_times.size()) : 0;
}

int32_t insem_cuda_solver_n_snapshot_fields(const insem_cuda_solver* h) {
  return h ? static_cast<int32_t>(h->s->snap_fields.size()) : 0;
}

int insem_cuda_solver_snapshot_field(const insem_cuda_solver* h, int32_t field, int32_t* medium, int32_t* quantity,
                                     int32_t* ncomp, int64_t* n_points) {
  return guarded([&] {
    INSEM_REQUIRE(h && field >= 0 && field < static_cast<int32_t>(h->s->snap_fields.size()), INSEM_CUDA_ERR_INVALID,
                  "snapshot field out of range");
    const Solver::SnapField& f = h->s->snap_fields[field];
    const DeviceDomainData& d = h->s->domains[f.domain];
    if (medium) *medium = d.medium;
    if (quantity) *quantity = f.quantity;
    if (ncomp) *ncomp = f.ncomp;
    if (n_points) *n_points = static_cast<int64_t>(d.n_elements) * d.npe;
  });
}

int insem_cuda_solver_snapshot(const insem_cuda_solver* h, int32_t field, float* out) {
  return guarded([&] {
    INSEM_REQUIRE(h && out && field >= 0 && field < static_cast<int32_t>(h->s->snap_fields.size()),
                  INSEM_CUDA_ERR_INVALID, "snapshot field out of range");
    const auto& data = h->s->snap_fields[field].data;
    std::copy(data.begin(), data.end(), out);
  });
}

int insem_cuda_solver_snapshot_times(const insem_cuda_solver* h, double* out) {
  return guarded([&] {
    INSEM_REQUIRE(h && out, INSEM_CUDA_ERR_INVALID, "null argument");
    std::copy(h->s->snap_times.begin(), h->s->snap_times.end(), out);
  });
}

}  // extern "C"
