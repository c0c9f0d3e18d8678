// Owning device copies of the reference's per-step descriptions (basis,
// element blocks, DofMap), converted to the device layouts the kernels read.
#pragma once

#include <memory>

#include "element_kernels.cuh"

namespace insem_b200 {

inline bool kernel_supported(int ngll) { return ngll >= 2 && ngll <= 9; }

inline int ncomp_of(int medium, int m) { return medium == INSEM_ELASTIC ? (m == 1 ? 3 : 2) : 1; }

inline void check_ngll(int ngll) {
  INSEM_REQUIRE(kernel_supported(ngll), INSEM_CUDA_ERR_UNSUPPORTED,
                "no kernel for " + std::to_string(ngll) + " GLL points (supported: 2..9)");
}

struct DeviceBasis {
  int ngll = 0;
  DeviceBuffer<float> D, Dj, w2;

  void upload(const insem_cuda_basis& b, bool need_dj) {
    check_ngll(b.ngll);
    ngll = b.ngll;
    const std::size_t n = static_cast<std::size_t>(ngll) * ngll;
    D.upload(host_vec(b.D, n));
    w2.upload(host_vec(b.w2, n));
    INSEM_REQUIRE(!need_dj || b.Dj != nullptr, INSEM_CUDA_ERR_INVALID,
                  "axial elements need the GLJ derivative matrix (basis.Dj)");
    if (b.Dj) Dj.upload(host_vec(b.Dj, n));
  }
  BasisDev view() const { return {D.get(), Dj.get(), w2.get()}; }
};

// A block's element data in the padded device layout (element_ops.cuh),
// elements taken in `order` (block-local positions): metric Rect 4 / Affine 8
// floats per element, per-point arrays CS = npe rounded up to 4 per element,
// per-point metric [element][component][CS] (transposed from the reference's
// [element][point][5]; axisymmetric blocks keep the first 4 components).
struct PackedBlock {
  std::vector<float> metric, coef0, coef1, wr, hoop, r;
  std::vector<uint8_t> axial;
};

inline PackedBlock pack_block(const insem_cuda_block& b, int npe, int medium, const std::vector<int32_t>& order) {
  PackedBlock pk;
  const std::size_t n = order.size(), cs = point_stride_rt(npe);
  const std::size_t ms = metric_stride_rt(b.kind, npe);
  pk.metric.assign(n * ms, 0.0f);
  pk.coef0.assign(n * cs, 0.0f);
  const bool el = medium == INSEM_ELASTIC, axi = b.kind == INSEM_AXISYM;
  if (el) pk.coef1.assign(n * cs, 0.0f);
  if (axi) {
    pk.wr.assign(n * cs, 0.0f);
    pk.hoop.assign(n * cs, 0.0f);
    pk.r.assign(n * cs, 0.0f);
    pk.axial.assign(n, 0);
  }
  INSEM_REQUIRE(b.n_elements == 0 || (b.metric && b.coef0), INSEM_CUDA_ERR_INVALID, "block arrays missing");
  INSEM_REQUIRE(!el || b.n_elements == 0 || b.coef1, INSEM_CUDA_ERR_INVALID, "elastic block needs coef1");
  INSEM_REQUIRE(!axi || b.n_elements == 0 || (b.wr && b.hoop && b.r && b.axial), INSEM_CUDA_ERR_INVALID,
                "axisymmetric block needs wr, hoop, r and axial");
  for (std::size_t q = 0; q < n; ++q) {
    const std::size_t o = static_cast<std::size_t>(order[q]);
    INSEM_REQUIRE(o < static_cast<std::size_t>(b.n_elements), INSEM_CUDA_ERR_INVALID, "element order out of range");
    if (b.kind == INSEM_RECT || b.kind == INSEM_AFFINE) {
      const int src = b.kind == INSEM_RECT ? 3 : 5;
      for (int k = 0; k < src; ++k) pk.metric[q * ms + k] = b.metric[o * src + k];
    } else {
      const int rows = axi ? 4 : 5;
      for (int k = 0; k < npe; ++k)
        for (int c = 0; c < rows; ++c) pk.metric[(q * rows + c) * cs + k] = b.metric[(o * npe + k) * 5 + c];
    }
    for (int k = 0; k < npe; ++k) {
      pk.coef0[q * cs + k] = b.coef0[o * npe + k];
      if (el) pk.coef1[q * cs + k] = b.coef1[o * npe + k];
      if (axi) {
        pk.wr[q * cs + k] = b.wr[o * npe + k];
        pk.hoop[q * cs + k] = b.hoop[o * npe + k];
        pk.r[q * cs + k] = b.r[o * npe + k];
      }
    }
    if (axi) pk.axial[q] = b.axial[o];
  }
  return pk;
}

struct DeviceBlock {
  int kind = 0, m = 0, n = 0;
  DeviceBuffer<int32_t> elements;
  DeviceBuffer<float> metric, coef0, coef1, wr, hoop, r;
  DeviceBuffer<uint8_t> axial;
  std::vector<int32_t> host_elements;
  bool any_axial = false;

  void upload(const insem_cuda_block& b, int ngll, int medium) {
    kind = b.kind;
    m = b.azimuthal_order;
    n = b.n_elements;
    INSEM_REQUIRE(kind >= INSEM_RECT && kind <= INSEM_AXISYM, INSEM_CUDA_ERR_UNSUPPORTED,
                  "unknown geometry kind " + std::to_string(kind));
    INSEM_REQUIRE(m == 0 || (m == 1 && kind == INSEM_AXISYM), INSEM_CUDA_ERR_UNSUPPORTED,
                  "no kernel for azimuthal order " + std::to_string(m) + " on non-axisymmetric elements");
    INSEM_REQUIRE(n >= 0, INSEM_CUDA_ERR_INVALID, "negative block size");
    const int npe = ngll * ngll;
    host_elements = host_vec(b.elements, n);
    elements.upload(host_elements);
    std::vector<int32_t> order(n);
    for (int q = 0; q < n; ++q) order[q] = q;
    PackedBlock pk = pack_block(b, npe, medium, order);
    metric.upload(pk.metric);
    coef0.upload(pk.coef0);
    if (medium == INSEM_ELASTIC) coef1.upload(pk.coef1);
    if (kind == INSEM_AXISYM) {
      wr.upload(pk.wr);
      hoop.upload(pk.hoop);
      r.upload(pk.r);
      for (auto a : pk.axial) any_axial |= a != 0;
      axial.upload(pk.axial);
    }
  }
  BlockDev view() const {
    BlockDev v;
    v.kind = kind;
    v.m = m;
    v.n = n;
    v.elements = elements.get();
    v.metric = metric.get();
    v.coef0 = coef0.get();
    v.coef1 = coef1.get();
    v.wr = wr.get();
    v.hoop = hoop.get();
    v.r = r.get();
    v.axial = axial.get();
    return v;
  }
};

struct DeviceDofMap {
  int ngll = 0, npe = 0, n_elements = 0, n_global = 0, n_rows = 0;
  DeviceBuffer<int32_t> l2g, row_offsets, row_dofs, t_offsets, t_slots;
  DeviceBuffer<float> row_weights, t_weights;  // rounded to float as the reference's gather/assemble do
  bool weighted = false;

  void upload(const insem_cuda_dofmap& d) {
    check_ngll(d.ngll);
    ngll = d.ngll;
    npe = ngll * ngll;
    n_elements = d.n_elements;
    n_global = d.n_global;
    n_rows = d.n_rows;
    INSEM_REQUIRE(n_elements >= 0 && n_global >= 0 && n_rows >= 0, INSEM_CUDA_ERR_INVALID, "negative DofMap size");
    const std::size_t ns = static_cast<std::size_t>(n_elements) * npe;
    const auto l = host_vec(d.l2g, ns);
    for (int32_t m : l)
      INSEM_REQUIRE(m < n_global && (m >= 0 || -1 - m < n_rows), INSEM_CUDA_ERR_INVALID, "l2g entry out of range");
    l2g.upload(l);
    const auto ro = host_vec(d.row_offsets, static_cast<std::size_t>(n_rows) + 1);
    row_offsets.upload(ro.empty() ? std::vector<int32_t>{0} : ro);
    const std::size_t nrd = ro.empty() ? 0 : static_cast<std::size_t>(ro.back());
    const auto rd = host_vec(d.row_dofs, nrd);
    for (int32_t g : rd) INSEM_REQUIRE(g >= 0 && g < n_global, INSEM_CUDA_ERR_INVALID, "row dof out of range");
    row_dofs.upload(rd);
    const auto rw = host_vec(d.row_weights, nrd);
    row_weights.upload(std::vector<float>(rw.begin(), rw.end()));
    const auto to = host_vec(d.t_offsets, static_cast<std::size_t>(n_global) + 1);
    t_offsets.upload(to);
    const std::size_t nt = to.empty() ? 0 : static_cast<std::size_t>(to.back());
    const auto ts = host_vec(d.t_slots, nt);
    for (int32_t s : ts) INSEM_REQUIRE(s >= 0 && static_cast<std::size_t>(s) < ns, INSEM_CUDA_ERR_INVALID, "t_slot out of range");
    t_slots.upload(ts);
    weighted = d.t_weights != nullptr && n_rows > 0;
    if (weighted) {
      const auto tw = host_vec(d.t_weights, nt);
      t_weights.upload(std::vector<float>(tw.begin(), tw.end()));
    }
  }
  RowsDev rows() const { return {row_offsets.get(), row_dofs.get(), row_weights.get()}; }
};

// Element-local gather and CSR assemble (DofMap seam), in dofmap_kernels.cu.
void launch_gather(const DeviceDofMap& d, int ncomp, const float* global, float* local, cudaStream_t s);
void launch_assemble(const DeviceDofMap& d, int ncomp, const float* local, float* global, cudaStream_t s);
// Loads assemble_kernel<weighted> (its module, under lazy loading) without launching it.
void preload_assemble(bool weighted);

}  // namespace insem_b200
