// Per-element stiffness operators f = -K u of the six reference kernels
// (cpp/src/cpu/kernels.cpp:64-431), written for one thread per element GLL
// point with the element's field, fluxes and axis terms staged in shared
// memory.
//
// Every floating-point expression keeps the reference's association and
// operand order (left-to-right sums over l, the interleaved xi/eta order of
// the weak divergence, the hoop and axis terms), using never-fused
// __fmul_rn/__fadd_rn, so that force vectors are bit-identical to the
// reference CPU build.
//
// Device layouts (chosen for coalesced loads; uploaded by the host code):
//   metric  Rect   [n][3]          (xi_x, eta_z, jac)     per element
//           Affine [n][5]          (xi_x, xi_z, eta_x, eta_z, jac)
//           Curved [n][5][npe]     metric component major inside an element
//           Axisym [n][5][npe]
//   coef0/coef1/wr/hoop/r [n][npe]; axial [n]
#pragma once

#include "common.cuh"

namespace insem_b200 {

// Block of elements of one kind, in device memory.
struct BlockDev {
  int32_t kind = 0;
  int32_t m = 0;          // azimuthal order
  int32_t n = 0;          // elements
  const int32_t* elements = nullptr;
  const float* metric = nullptr;
  const float* coef0 = nullptr;
  const float* coef1 = nullptr;
  const float* wr = nullptr;
  const float* hoop = nullptr;
  const float* r = nullptr;
  const uint8_t* axial = nullptr;
};

// Basis matrices in device memory ([ngll*ngll] each).
struct BasisDev {
  const float* D = nullptr;
  const float* Dj = nullptr;
  const float* w2 = nullptr;
};

// Constraint rows of a DofMap in device memory (weights rounded to float as
// the reference's gather does: static_cast<T>(rw[q]), dof_map.hpp:114).
struct RowsDev {
  const int32_t* offsets = nullptr;
  const int32_t* dofs = nullptr;
  const float* weights = nullptr;
};

template <int NG, int KIND, bool ELASTIC, int M>
struct ElemCfg {
  static constexpr int NPE = NG * NG;
  static constexpr int NC = ELASTIC ? (M == 1 ? 3 : 2) : 1;
  static constexpr bool AXI = KIND == INSEM_AXISYM;
  static constexpr int EPB = (256 / NPE) > 0 ? (256 / NPE) : 1;  // elements per CTA
  static constexpr int THREADS = EPB * NPE;
  static constexpr int NAX = (AXI && (M == 1) && ELASTIC) ? 2 : 1;  // axis spreads per element
};

// Shared memory of one CTA of the element kernel.
template <class C>
struct ElemSmem {
  float D[C::NPE];
  float Dj[C::NPE];
  float w2[C::NPE];
  float u[C::EPB][C::NC][C::NPE];
  float f1[C::EPB][C::NC][C::NPE];
  float f2[C::EPB][C::NC][C::NPE];
  float gx[C::EPB][C::NAX][C::AXI ? 16 : 1];  // axis term x xi_r at (0, jq)
  float gy[C::EPB][C::NAX][C::AXI ? 16 : 1];  // axis term x eta_r at (0, jq)
};

// ---------------------------------------------------------------- helpers
// reference_derivatives(_xy) (kernels.cpp:42-51, 170-179): sequential l.
template <int NG>
__device__ __forceinline__ void ref_derivs(const float* Dx, const float* Dy, const float* u, int i, int j,
                                           float& u_xi, float& u_eta) {
  float a = 0.0f, b = 0.0f;
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    a = fadd(a, fmul(Dx[i * NG + l], u[j * NG + l]));
    b = fadd(b, fmul(Dy[j * NG + l], u[l * NG + i]));
  }
  u_xi = a;
  u_eta = b;
}

// weak_divergence(_xy) (kernels.cpp:55-62, 182-190): interleaved xi/eta terms.
template <int NG>
__device__ __forceinline__ float weak_div(const float* Dx, const float* Dy, const float* f_xi,
                                          const float* f_eta, int i, int j) {
  float s = 0.0f;
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    s = fadd(s, fmul(Dx[l * NG + i], f_xi[j * NG + l]));
    s = fadd(s, fmul(Dy[l * NG + j], f_eta[l * NG + i]));
  }
  return s;
}

// physical_gradient (pointwise.hpp:30-35).
__device__ __forceinline__ void phys_grad(float a_xi, float a_eta, float xi_x, float xi_z, float eta_x,
                                          float eta_z, float& a_x, float& a_z) {
  a_x = fadd(fmul(a_xi, xi_x), fmul(a_eta, eta_x));
  a_z = fadd(fmul(a_xi, xi_z), fmul(a_eta, eta_z));
}

// reference_flux (pointwise.hpp:40-45).
__device__ __forceinline__ void ref_flux(float wj, float qx, float qz, float xi_x, float xi_z, float eta_x,
                                         float eta_z, float& f_xi, float& f_eta) {
  f_xi = fmul(wj, fadd(fmul(qx, xi_x), fmul(qz, xi_z)));
  f_eta = fmul(wj, fadd(fmul(qx, eta_x), fmul(qz, eta_z)));
}

// elastic_stress (pointwise.hpp:12-19).
__device__ __forceinline__ void el_stress(float lambda, float mu, float ux_x, float ux_z, float uz_x, float uz_z,
                                          float& sxx, float& szz, float& sxz) {
  const float div = fadd(ux_x, uz_z);
  const float two_mu = fmul(2.0f, mu);
  sxx = fadd(fmul(lambda, div), fmul(two_mu, ux_x));
  szz = fadd(fmul(lambda, div), fmul(two_mu, uz_z));
  sxz = fmul(mu, fadd(ux_z, uz_x));
}

// Padded strides of the device layout (16-byte multiples, so that every
// element's data can be moved with bulk copies):
//   per-point arrays: CS = npe rounded up to 4 floats per element (and per
//                     metric component);
//   metric: Rect 4 floats, Affine 8 floats, Curved 5 * CS floats (xi_x,
//           xi_z, eta_x, eta_z, jac), Axisym 4 * CS (xi_r, xi_z, eta_r, eta_z:
//           the axisymmetric fluxes use the Jacobian only through wr).
template <int NPE>
constexpr int point_stride() {
  return (NPE + 3) & ~3;
}
inline int point_stride_rt(int npe) { return (npe + 3) & ~3; }
inline int metric_stride_rt(int kind, int npe) {
  return kind == INSEM_RECT ? 4 : kind == INSEM_AFFINE ? 8 : (kind == INSEM_AXISYM ? 4 : 5) * point_stride_rt(npe);
}

// Metric of block element b at point k in the device layout.
template <int KIND, int NPE>
__device__ __forceinline__ void load_metric(const float* metric, int b, int k, float& xi_x, float& xi_z,
                                            float& eta_x, float& eta_z, float& jac) {
  constexpr int CS = point_stride<NPE>();
  if constexpr (KIND == INSEM_RECT) {
    const float* m = metric + static_cast<size_t>(b) * 4;
    xi_x = m[0];
    xi_z = 0.0f;
    eta_x = 0.0f;
    eta_z = m[1];
    jac = m[2];
  } else if constexpr (KIND == INSEM_AFFINE) {
    const float* m = metric + static_cast<size_t>(b) * 8;
    xi_x = m[0];
    xi_z = m[1];
    eta_x = m[2];
    eta_z = m[3];
    jac = m[4];
  } else {
    const float* m = metric + static_cast<size_t>(b) * 5 * CS + k;
    xi_x = m[0];
    xi_z = m[CS];
    eta_x = m[2 * CS];
    eta_z = m[3 * CS];
    jac = m[4 * CS];
  }
}

// ------------------------------------------------------------- point math
// Fluxes of one element point from its reference derivatives u_xi / u_eta
// (per component), the point's own field values upt (hoop terms), and the
// block data: f_xi / f_eta per component, the direct (hoop) terms, and for
// axis points of axial elements the axis terms g xi_r, g eta_r (stored at
// row j of gx*/gy*).  The body of each reference kernel's first loop.
// ECOEF: the element's coefficients come in as ec0 / ec1 (the material is
// one per element, so every point of it carries the same coefficients; the
// caller reads them once) instead of from blk.coef0 / coef1 per point.
template <int NG, int KIND, bool ELASTIC, int M, bool ECOEF = false>
__device__ __forceinline__ void point_flux(const BlockDev& blk, int bb, int kpt, int i, int j, bool axial,
                                           const float* uxi, const float* ueta, const float* upt, float* fx,
                                           float* fy, float* direct, float* gx0, float* gy0, float* gx1,
                                           float* gy1, float w2k, float ec0 = 0.0f, float ec1 = 0.0f) {
  constexpr int NPE = NG * NG;
  constexpr int CS = point_stride<NPE>();
  if constexpr (KIND != INSEM_AXISYM) {
    float xi_x, xi_z, eta_x, eta_z, jac;
    load_metric<KIND, NPE>(blk.metric, bb, kpt, xi_x, xi_z, eta_x, eta_z, jac);
    const size_t p = static_cast<size_t>(bb) * CS + kpt;
    if constexpr (ELASTIC) {
      // elastic_kernel (kernels.cpp:64-120)
      float ux_x, ux_z, uz_x, uz_z;
      if constexpr (KIND == INSEM_RECT) {
        ux_x = fmul(uxi[0], xi_x);
        ux_z = fmul(ueta[0], eta_z);
        uz_x = fmul(uxi[1], xi_x);
        uz_z = fmul(ueta[1], eta_z);
      } else {
        phys_grad(uxi[0], ueta[0], xi_x, xi_z, eta_x, eta_z, ux_x, ux_z);
        phys_grad(uxi[1], ueta[1], xi_x, xi_z, eta_x, eta_z, uz_x, uz_z);
      }
      float sxx, szz, sxz;
      el_stress((ECOEF ? ec0 : blk.coef0[p]), (ECOEF ? ec1 : blk.coef1[p]), ux_x, ux_z, uz_x, uz_z, sxx, szz, sxz);
      const float wj = fmul(w2k, jac);
      if constexpr (KIND == INSEM_RECT) {
        fx[0] = fmul(fmul(wj, sxx), xi_x);
        fx[1] = fmul(fmul(wj, sxz), xi_x);
        fy[0] = fmul(fmul(wj, sxz), eta_z);
        fy[1] = fmul(fmul(wj, szz), eta_z);
      } else {
        ref_flux(wj, sxx, sxz, xi_x, xi_z, eta_x, eta_z, fx[0], fy[0]);
        ref_flux(wj, sxz, szz, xi_x, xi_z, eta_x, eta_z, fx[1], fy[1]);
      }
    } else {
      // acoustic_kernel (kernels.cpp:122-158)
      const float c = fmul(fmul(w2k, jac), (ECOEF ? ec0 : blk.coef0[p]));
      if constexpr (KIND == INSEM_RECT) {
        fx[0] = fmul(fmul(fmul(c, uxi[0]), xi_x), xi_x);
        fy[0] = fmul(fmul(fmul(c, ueta[0]), eta_z), eta_z);
      } else {
        float p_x, p_z;
        phys_grad(uxi[0], ueta[0], xi_x, xi_z, eta_x, eta_z, p_x, p_z);
        ref_flux(c, p_x, p_z, xi_x, xi_z, eta_x, eta_z, fx[0], fy[0]);
      }
    }
  } else {
    const size_t p = static_cast<size_t>(bb) * CS + kpt;
    const float* mt = blk.metric + static_cast<size_t>(bb) * 4 * CS + kpt;
    const float xi_r = mt[0], xi_z = mt[CS], eta_r = mt[2 * CS], eta_z = mt[3 * CS];
    const bool axis_pt = axial && i == 0;
    if constexpr (ELASTIC && M == 0) {
      // elastic_axisym_kernel (kernels.cpp:206-263)
      float ur_r, ur_z, uz_r, uz_z;
      phys_grad(uxi[0], ueta[0], xi_r, xi_z, eta_r, eta_z, ur_r, ur_z);
      phys_grad(uxi[1], ueta[1], xi_r, xi_z, eta_r, eta_z, uz_r, uz_z);
      const float r = blk.r[p];
      const float e_tt = r == 0.0f ? ur_r : __fdiv_rn(upt[0], r);
      const float lambda = (ECOEF ? ec0 : blk.coef0[p]), mu = (ECOEF ? ec1 : blk.coef1[p]);
      const float tr = fadd(fadd(ur_r, uz_z), e_tt);
      const float two_mu = fmul(2.0f, mu);
      const float ltr = fmul(lambda, tr);
      const float srr = fadd(ltr, fmul(two_mu, ur_r));
      const float szz = fadd(ltr, fmul(two_mu, uz_z));
      const float stt = fadd(ltr, fmul(two_mu, e_tt));
      const float srz = fmul(mu, fadd(ur_z, uz_r));
      const float w = blk.wr[p];
      ref_flux(w, srr, srz, xi_r, xi_z, eta_r, eta_z, fx[0], fy[0]);
      ref_flux(w, srz, szz, xi_r, xi_z, eta_r, eta_z, fx[1], fy[1]);
      if (axis_pt) {
        direct[0] = 0.0f;
        const float g = fmul(w, stt);
        gx0[j] = fmul(g, xi_r);
        gy0[j] = fmul(g, eta_r);
      } else {
        direct[0] = fmul(blk.hoop[p], stt);
      }
    } else if constexpr (!ELASTIC && M == 0) {
      // acoustic_axisym_kernel (kernels.cpp:265-294)
      float p_r, p_z;
      phys_grad(uxi[0], ueta[0], xi_r, xi_z, eta_r, eta_z, p_r, p_z);
      ref_flux(fmul(blk.wr[p], (ECOEF ? ec0 : blk.coef0[p])), p_r, p_z, xi_r, xi_z, eta_r, eta_z, fx[0], fy[0]);
    } else if constexpr (ELASTIC && M == 1) {
      // elastic_axisym1_kernel (kernels.cpp:305-385)
      const float s2 = 1.41421356237309504880f;
      const float is2 = 0.70710678118654752440f;
      float up_r, up_z, um_r, um_z, uz_r, uz_z;
      phys_grad(uxi[0], ueta[0], xi_r, xi_z, eta_r, eta_z, up_r, up_z);
      phys_grad(uxi[1], ueta[1], xi_r, xi_z, eta_r, eta_z, um_r, um_z);
      phys_grad(uxi[2], ueta[2], xi_r, xi_z, eta_r, eta_z, uz_r, uz_z);
      const float r = blk.r[p];
      const bool on_axis = r == 0.0f;
      const float up_over_r = on_axis ? up_r : __fdiv_rn(upt[0], r);
      const float uz_over_r = on_axis ? uz_r : __fdiv_rn(upt[2], r);
      const float ur_r = fmul(fadd(up_r, um_r), is2), ur_z = fmul(fadd(up_z, um_z), is2);
      const float ut_r = fmul(fsub(up_r, um_r), is2), ut_z = fmul(fsub(up_z, um_z), is2);
      const float e_tt = fmul(s2, up_over_r);
      const float lambda = (ECOEF ? ec0 : blk.coef0[p]), mu = (ECOEF ? ec1 : blk.coef1[p]);
      const float tr = fadd(fadd(ur_r, uz_z), e_tt);
      const float two_mu = fmul(2.0f, mu);
      const float ltr = fmul(lambda, tr);
      const float srr = fadd(ltr, fmul(two_mu, ur_r));
      const float szz = fadd(ltr, fmul(two_mu, uz_z));
      const float stt = fadd(ltr, fmul(two_mu, e_tt));
      const float srz = fmul(mu, fadd(ur_z, uz_r));
      const float srt = fmul(mu, fsub(ut_r, fmul(s2, up_over_r)));
      const float stz = fmul(mu, fsub(ut_z, uz_over_r));
      const float w = blk.wr[p];
      ref_flux(w, fmul(fadd(srr, srt), is2), fmul(fadd(srz, stz), is2), xi_r, xi_z, eta_r, eta_z, fx[0], fy[0]);
      ref_flux(w, fmul(fsub(srr, srt), is2), fmul(fsub(srz, stz), is2), xi_r, xi_z, eta_r, eta_z, fx[1], fy[1]);
      ref_flux(w, srz, szz, xi_r, xi_z, eta_r, eta_z, fx[2], fy[2]);
      const float cp = fmul(s2, fsub(stt, srt));
      const float cz = -stz;
      if (axis_pt) {
        direct[0] = 0.0f;
        direct[1] = 0.0f;
        const float gp = fmul(w, cp), gz = fmul(w, cz);
        gx0[j] = fmul(gp, xi_r);
        gy0[j] = fmul(gp, eta_r);
        gx1[j] = fmul(gz, xi_r);
        gy1[j] = fmul(gz, eta_r);
      } else {
        direct[0] = fmul(blk.hoop[p], cp);
        direct[1] = fmul(blk.hoop[p], cz);
      }
    } else {
      // acoustic_axisym1_kernel (kernels.cpp:389-431)
      float p_r, p_z;
      phys_grad(uxi[0], ueta[0], xi_r, xi_z, eta_r, eta_z, p_r, p_z);
      const float inv_rho = (ECOEF ? ec0 : blk.coef0[p]);
      const float wri = fmul(blk.wr[p], inv_rho);
      ref_flux(wri, p_r, p_z, xi_r, xi_z, eta_r, eta_z, fx[0], fy[0]);
      if (axis_pt) {
        direct[0] = 0.0f;
        const float g = fmul(wri, p_r);
        gx0[j] = fmul(g, xi_r);
        gy0[j] = fmul(g, eta_r);
      } else {
        direct[0] = __fdiv_rn(fmul(fmul(blk.hoop[p], inv_rho), upt[0]), blk.r[p]);
      }
    }
  }
}

// spread_axis_term (kernels.cpp:195-204) as seen from point (ia, ja): the
// row-jq update (f -= g_jq xi_r Dx[ia]) reaches the points of row ja; the
// column update (f -= g_jq eta_r Dy[jq][ja]) reaches column 0 for every jq,
// after that jq's row update.  dx_row0 = Dx[ia] (row 0 of Dx); dy(q) =
// Dy[q] with q = jq * NG + ja.
template <int NG, class DyFn>
__device__ __forceinline__ float axis_spread(float f, int ia, int ja, float dx_row0, DyFn dy, const float* gx,
                                             const float* gy) {
  if (ia != 0) return fsub(f, fmul(gx[ja], dx_row0));
#pragma unroll
  for (int jq = 0; jq < NG; ++jq) {
    if (jq == ja) f = fsub(f, fmul(gx[jq], dx_row0));
    f = fsub(f, fmul(gy[jq], dy(jq * NG + ja)));
  }
  return f;
}

// Force of one element point from its weak divergence sums s[c] (the second
// loop of each reference kernel): negation, hoop term, axis spread.
template <int NG, int KIND, bool ELASTIC, int M, class DyFn>
__device__ __forceinline__ void point_divergence(int i, int j, bool axial, const float* s, const float* direct,
                                                 float dx_row0, DyFn dy, const float* gx0, const float* gy0,
                                                 const float* gx1, const float* gy1, float* out) {
  using C = ElemCfg<NG, KIND, ELASTIC, M>;
  if constexpr (KIND != INSEM_AXISYM) {
#pragma unroll
    for (int c = 0; c < C::NC; ++c) out[c] = -s[c];
  } else if constexpr (ELASTIC && M == 0) {
    out[0] = -fadd(s[0], direct[0]);
    out[1] = -s[1];
    if (axial) out[0] = axis_spread<NG>(out[0], i, j, dx_row0, dy, gx0, gy0);
  } else if constexpr (!ELASTIC && M == 0) {
    out[0] = -s[0];
  } else if constexpr (ELASTIC && M == 1) {
    out[0] = -fadd(s[0], direct[0]);
    out[1] = -s[1];
    out[2] = -fadd(s[2], direct[1]);
    if (axial) {
      out[0] = axis_spread<NG>(out[0], i, j, dx_row0, dy, gx0, gy0);
      out[2] = axis_spread<NG>(out[2], i, j, dx_row0, dy, gx1, gy1);
    }
  } else {
    out[0] = -fadd(s[0], direct[0]);
    if (axial) out[0] = axis_spread<NG>(out[0], i, j, dx_row0, dy, gx0, gy0);
  }
}

// ------------------------------------------- one-thread-per-point phases
// Phase 1 of an element (point threads): derivatives from the staged field
// su[c][k], then point_flux; fluxes to shared memory f1/f2[c][k].
template <int NG, int KIND, bool ELASTIC, int M>
__device__ __forceinline__ void element_fluxes(const BlockDev& blk, int bb, int kpt, bool axial,
                                               const float* Dx, const float* Dy, const float* w2,
                                               const float (*su)[NG * NG], float (*f1)[NG * NG],
                                               float (*f2)[NG * NG], float* gx0, float* gy0, float* gx1,
                                               float* gy1, float* direct) {
  using C = ElemCfg<NG, KIND, ELASTIC, M>;
  const int i = kpt % NG, j = kpt / NG;
  float uxi[C::NC], ueta[C::NC], upt[C::NC], fx[C::NC], fy[C::NC];
#pragma unroll
  for (int c = 0; c < C::NC; ++c) {
    ref_derivs<NG>(Dx, Dy, su[c], i, j, uxi[c], ueta[c]);
    upt[c] = su[c][kpt];
  }
  point_flux<NG, KIND, ELASTIC, M>(blk, bb, kpt, i, j, axial, uxi, ueta, upt, fx, fy, direct, gx0, gy0, gx1, gy1,
                                   w2[kpt]);
#pragma unroll
  for (int c = 0; c < C::NC; ++c) {
    f1[c][kpt] = fx[c];
    f2[c][kpt] = fy[c];
  }
}

// Phase 2 of an element (point threads): f[c] at point kpt from the staged fluxes.
template <int NG, int KIND, bool ELASTIC, int M>
__device__ __forceinline__ void element_divergence(int kpt, bool axial, const float* Dx, const float* Dy,
                                                   const float (*f1)[NG * NG], const float (*f2)[NG * NG],
                                                   const float* gx0, const float* gy0, const float* gx1,
                                                   const float* gy1, const float* direct, float* out) {
  using C = ElemCfg<NG, KIND, ELASTIC, M>;
  const int i = kpt % NG, j = kpt / NG;
  float s[C::NC];
#pragma unroll
  for (int c = 0; c < C::NC; ++c) s[c] = weak_div<NG>(Dx, Dy, f1[c], f2[c], i, j);
  point_divergence<NG, KIND, ELASTIC, M>(i, j, axial, s, direct, Dx[i], [Dy](int q) { return Dy[q]; }, gx0, gy0, gx1,
                                         gy1, out);
}

}  // namespace insem_b200
