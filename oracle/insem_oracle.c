/*
 * insem_oracle.c -- CPU restatement of insem's per-time-step path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA backend is compared
 * with; nothing in the product links or calls it.  It follows the reference
 * (nmutovkin/in-house-sem) function by function, with sequential loops in the
 * reference's summation order, compiled without FMA contraction
 * (-ffp-contract=off), so on x86-64 it reproduces the reference float build
 * bit for bit.  Its inputs are the packed problem of include/insem_cuda.h.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks every function here
 * against outputs of the reference itself (tests/golden/<case>.npz, generated by
 * tests/golden/make_golden.py from the reference build in oracle/ref).
 *
 * Reference map:
 *   ref_derivatives / weak_divergence ..... cpp/src/cpu/kernels.cpp:40-62, 168-190
 *   element kernels ....................... kernels.cpp:64-158 (Cartesian),
 *                                           206-294 (axisym m=0), 305-431 (m=1)
 *   spread_axis_term ...................... kernels.cpp:195-204
 *   gather / assemble ..................... cpp/include/insem/ops/dof_map.hpp:95-141
 *   internal_forces ....................... cpp/src/solver/solver.cpp:570-581
 *   compute_acceleration .................. solver.cpp:669-691
 *   add_coupling_forces ................... solver.cpp:693-727
 *   solve_acceleration / solve_spd ........ solver.cpp:729-762, 67-80
 *   apply_dirichlet ....................... cpp/include/insem/solver/solver.hpp:57-65
 *   record / initialize / kinetic_energy .. solver.cpp:780-811, 878-915
 *   advance ............................... solver.cpp:917-963
 *   SourceTimeFunction ................... cpp/src/sim/description.cpp:88-113
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/insem_cuda.h"

#define MAXNG 9
#define MAXNPE (MAXNG * MAXNG)

/* ------------------------------------------------------------ element ops */
static void ref_derivs(int ng, const float* Dx, const float* Dy, const float* u, int i, int j, float* u_xi,
                       float* u_eta) {
  float a = 0, b = 0;
  for (int l = 0; l < ng; ++l) {
    a += Dx[i * ng + l] * u[j * ng + l];
    b += Dy[j * ng + l] * u[l * ng + i];
  }
  *u_xi = a;
  *u_eta = b;
}

static float weak_div(int ng, const float* Dx, const float* Dy, const float* fx, const float* fe, int i, int j) {
  float s = 0;
  for (int l = 0; l < ng; ++l) {
    s += Dx[l * ng + i] * fx[j * ng + l];
    s += Dy[l * ng + j] * fe[l * ng + i];
  }
  return s;
}

static void phys_grad(float a_xi, float a_eta, float xi_x, float xi_z, float eta_x, float eta_z, float* a_x,
                      float* a_z) {
  *a_x = a_xi * xi_x + a_eta * eta_x;
  *a_z = a_xi * xi_z + a_eta * eta_z;
}

static void ref_flux(float wj, float qx, float qz, float xi_x, float xi_z, float eta_x, float eta_z, float* f_xi,
                     float* f_eta) {
  *f_xi = wj * (qx * xi_x + qz * xi_z);
  *f_eta = wj * (qx * eta_x + qz * eta_z);
}

static void el_stress(float lambda, float mu, float ux_x, float ux_z, float uz_x, float uz_z, float* sxx,
                      float* szz, float* sxz) {
  const float div = ux_x + uz_z;
  *sxx = lambda * div + 2.0f * mu * ux_x;
  *szz = lambda * div + 2.0f * mu * uz_z;
  *sxz = mu * (ux_z + uz_x);
}

static void spread_axis(int ng, const float* Dx, const float* Dy, const float* m, const float* g, float* f) {
  for (int jq = 0; jq < ng; ++jq) {
    const int kq = jq * ng;
    const float xi_r = m[5 * kq], eta_r = m[5 * kq + 2];
    for (int ia = 0; ia < ng; ++ia) f[jq * ng + ia] -= g[jq] * xi_r * Dx[ia];
    for (int ja = 0; ja < ng; ++ja) f[ja * ng] -= g[jq] * eta_r * Dy[jq * ng + ja];
  }
}

static void cartesian_element(const insem_cuda_basis* kb, const insem_cuda_block* blk, int elastic, int b,
                              const float* u, float* f) {
  const int ng = kb->ngll, npe = ng * ng, K = blk->kind;
  const float* D = kb->D;
  float f1[3][MAXNPE], f2[3][MAXNPE];
  for (int j = 0; j < ng; ++j)
    for (int i = 0; i < ng; ++i) {
      const int k = j * ng + i;
      float xi_x, xi_z, eta_x, eta_z, jac;
      if (K == INSEM_RECT) {
        const float* m = blk->metric + (size_t)b * 3;
        xi_x = m[0]; xi_z = 0; eta_x = 0; eta_z = m[1]; jac = m[2];
      } else {
        const float* m = blk->metric + (K == INSEM_AFFINE ? (size_t)b * 5 : ((size_t)b * npe + k) * 5);
        xi_x = m[0]; xi_z = m[1]; eta_x = m[2]; eta_z = m[3]; jac = m[4];
      }
      const size_t p = (size_t)b * npe + k;
      if (elastic) {
        float ux_xi, ux_eta, uz_xi, uz_eta, ux_x, ux_z, uz_x, uz_z, sxx, szz, sxz;
        ref_derivs(ng, D, D, u, i, j, &ux_xi, &ux_eta);
        ref_derivs(ng, D, D, u + npe, i, j, &uz_xi, &uz_eta);
        if (K == INSEM_RECT) {
          ux_x = ux_xi * xi_x; ux_z = ux_eta * eta_z; uz_x = uz_xi * xi_x; uz_z = uz_eta * eta_z;
        } else {
          phys_grad(ux_xi, ux_eta, xi_x, xi_z, eta_x, eta_z, &ux_x, &ux_z);
          phys_grad(uz_xi, uz_eta, xi_x, xi_z, eta_x, eta_z, &uz_x, &uz_z);
        }
        el_stress(blk->coef0[p], blk->coef1[p], ux_x, ux_z, uz_x, uz_z, &sxx, &szz, &sxz);
        const float wj = kb->w2[k] * jac;
        if (K == INSEM_RECT) {
          f1[0][k] = wj * sxx * xi_x; f1[1][k] = wj * sxz * xi_x;
          f2[0][k] = wj * sxz * eta_z; f2[1][k] = wj * szz * eta_z;
        } else {
          ref_flux(wj, sxx, sxz, xi_x, xi_z, eta_x, eta_z, &f1[0][k], &f2[0][k]);
          ref_flux(wj, sxz, szz, xi_x, xi_z, eta_x, eta_z, &f1[1][k], &f2[1][k]);
        }
      } else {
        float p_xi, p_eta;
        ref_derivs(ng, D, D, u, i, j, &p_xi, &p_eta);
        const float c = kb->w2[k] * jac * blk->coef0[p];
        if (K == INSEM_RECT) {
          f1[0][k] = c * p_xi * xi_x * xi_x;
          f2[0][k] = c * p_eta * eta_z * eta_z;
        } else {
          float p_x, p_z;
          phys_grad(p_xi, p_eta, xi_x, xi_z, eta_x, eta_z, &p_x, &p_z);
          ref_flux(c, p_x, p_z, xi_x, xi_z, eta_x, eta_z, &f1[0][k], &f2[0][k]);
        }
      }
    }
  const int nc = elastic ? 2 : 1;
  for (int c = 0; c < nc; ++c)
    for (int j = 0; j < ng; ++j)
      for (int i = 0; i < ng; ++i) f[c * npe + j * ng + i] = -weak_div(ng, D, D, f1[c], f2[c], i, j);
}

static void axisym_element(const insem_cuda_basis* kb, const insem_cuda_block* blk, int elastic, int b,
                           const float* u, float* f) {
  const int ng = kb->ngll, npe = ng * ng, M = blk->azimuthal_order;
  const int axial = blk->axial[b] != 0;
  const float* Dx = axial ? kb->Dj : kb->D;
  const float* Dy = kb->D;
  const size_t p0 = (size_t)b * npe;
  const float* m = blk->metric + p0 * 5;
  const float s2 = 1.41421356237309504880f, is2 = 0.70710678118654752440f;
  float f1[3][MAXNPE], f2[3][MAXNPE], direct[2][MAXNPE], axis_g[2][MAXNG];
  for (int j = 0; j < ng; ++j)
    for (int i = 0; i < ng; ++i) {
      const int k = j * ng + i;
      const size_t p = p0 + k;
      const float xi_r = m[5 * k], xi_z = m[5 * k + 1], eta_r = m[5 * k + 2], eta_z = m[5 * k + 3];
      const int axis_pt = axial && i == 0;
      if (elastic && M == 0) {
        float ur_xi, ur_eta, uz_xi, uz_eta, ur_r, ur_z, uz_r, uz_z;
        ref_derivs(ng, Dx, Dy, u, i, j, &ur_xi, &ur_eta);
        ref_derivs(ng, Dx, Dy, u + npe, i, j, &uz_xi, &uz_eta);
        phys_grad(ur_xi, ur_eta, xi_r, xi_z, eta_r, eta_z, &ur_r, &ur_z);
        phys_grad(uz_xi, uz_eta, xi_r, xi_z, eta_r, eta_z, &uz_r, &uz_z);
        const float r = blk->r[p];
        const float e_tt = r == 0.0f ? ur_r : u[k] / r;
        const float lambda = blk->coef0[p], mu = blk->coef1[p];
        const float tr = ur_r + uz_z + e_tt;
        const float srr = lambda * tr + 2.0f * mu * ur_r;
        const float szz = lambda * tr + 2.0f * mu * uz_z;
        const float stt = lambda * tr + 2.0f * mu * e_tt;
        const float srz = mu * (ur_z + uz_r);
        const float w = blk->wr[p];
        ref_flux(w, srr, srz, xi_r, xi_z, eta_r, eta_z, &f1[0][k], &f2[0][k]);
        ref_flux(w, srz, szz, xi_r, xi_z, eta_r, eta_z, &f1[1][k], &f2[1][k]);
        if (axis_pt) { direct[0][k] = 0; axis_g[0][j] = w * stt; }
        else direct[0][k] = blk->hoop[p] * stt;
      } else if (!elastic && M == 0) {
        float p_xi, p_eta, p_r, p_z;
        ref_derivs(ng, Dx, Dy, u, i, j, &p_xi, &p_eta);
        phys_grad(p_xi, p_eta, xi_r, xi_z, eta_r, eta_z, &p_r, &p_z);
        ref_flux(blk->wr[p] * blk->coef0[p], p_r, p_z, xi_r, xi_z, eta_r, eta_z, &f1[0][k], &f2[0][k]);
      } else if (elastic) {
        float up_xi, up_eta, um_xi, um_eta, uz_xi, uz_eta, up_r, up_z, um_r, um_z, uz_r, uz_z;
        ref_derivs(ng, Dx, Dy, u, i, j, &up_xi, &up_eta);
        ref_derivs(ng, Dx, Dy, u + npe, i, j, &um_xi, &um_eta);
        ref_derivs(ng, Dx, Dy, u + 2 * npe, i, j, &uz_xi, &uz_eta);
        phys_grad(up_xi, up_eta, xi_r, xi_z, eta_r, eta_z, &up_r, &up_z);
        phys_grad(um_xi, um_eta, xi_r, xi_z, eta_r, eta_z, &um_r, &um_z);
        phys_grad(uz_xi, uz_eta, xi_r, xi_z, eta_r, eta_z, &uz_r, &uz_z);
        const float r = blk->r[p];
        const int on_axis = r == 0.0f;
        const float up_over_r = on_axis ? up_r : u[k] / r;
        const float uz_over_r = on_axis ? uz_r : u[2 * npe + k] / r;
        const float ur_r = (up_r + um_r) * is2, ur_z = (up_z + um_z) * is2;
        const float ut_r = (up_r - um_r) * is2, ut_z = (up_z - um_z) * is2;
        const float e_tt = s2 * up_over_r;
        const float lambda = blk->coef0[p], mu = blk->coef1[p];
        const float tr = ur_r + uz_z + e_tt;
        const float srr = lambda * tr + 2.0f * mu * ur_r;
        const float szz = lambda * tr + 2.0f * mu * uz_z;
        const float stt = lambda * tr + 2.0f * mu * e_tt;
        const float srz = mu * (ur_z + uz_r);
        const float srt = mu * (ut_r - s2 * up_over_r);
        const float stz = mu * (ut_z - uz_over_r);
        const float w = blk->wr[p];
        ref_flux(w, (srr + srt) * is2, (srz + stz) * is2, xi_r, xi_z, eta_r, eta_z, &f1[0][k], &f2[0][k]);
        ref_flux(w, (srr - srt) * is2, (srz - stz) * is2, xi_r, xi_z, eta_r, eta_z, &f1[1][k], &f2[1][k]);
        ref_flux(w, srz, szz, xi_r, xi_z, eta_r, eta_z, &f1[2][k], &f2[2][k]);
        const float cp = s2 * (stt - srt), cz = -stz;
        if (axis_pt) {
          direct[0][k] = direct[1][k] = 0;
          axis_g[0][j] = w * cp;
          axis_g[1][j] = w * cz;
        } else {
          direct[0][k] = blk->hoop[p] * cp;
          direct[1][k] = blk->hoop[p] * cz;
        }
      } else {
        float p_xi, p_eta, p_r, p_z;
        ref_derivs(ng, Dx, Dy, u, i, j, &p_xi, &p_eta);
        phys_grad(p_xi, p_eta, xi_r, xi_z, eta_r, eta_z, &p_r, &p_z);
        const float inv_rho = blk->coef0[p];
        ref_flux(blk->wr[p] * inv_rho, p_r, p_z, xi_r, xi_z, eta_r, eta_z, &f1[0][k], &f2[0][k]);
        if (axis_pt) { direct[0][k] = 0; axis_g[0][j] = blk->wr[p] * inv_rho * p_r; }
        else direct[0][k] = blk->hoop[p] * inv_rho * u[k] / blk->r[p];
      }
    }
  for (int j = 0; j < ng; ++j)
    for (int i = 0; i < ng; ++i) {
      const int k = j * ng + i;
      if (elastic && M == 0) {
        f[k] = -(weak_div(ng, Dx, Dy, f1[0], f2[0], i, j) + direct[0][k]);
        f[npe + k] = -weak_div(ng, Dx, Dy, f1[1], f2[1], i, j);
      } else if (!elastic && M == 0) {
        f[k] = -weak_div(ng, Dx, Dy, f1[0], f2[0], i, j);
      } else if (elastic) {
        f[k] = -(weak_div(ng, Dx, Dy, f1[0], f2[0], i, j) + direct[0][k]);
        f[npe + k] = -weak_div(ng, Dx, Dy, f1[1], f2[1], i, j);
        f[2 * npe + k] = -(weak_div(ng, Dx, Dy, f1[2], f2[2], i, j) + direct[1][k]);
      } else {
        f[k] = -(weak_div(ng, Dx, Dy, f1[0], f2[0], i, j) + direct[0][k]);
      }
    }
  if (axial) {
    if (elastic && M == 0) spread_axis(ng, Dx, Dy, m, axis_g[0], f);
    else if (!elastic && M == 1) spread_axis(ng, Dx, Dy, m, axis_g[0], f);
    else if (elastic && M == 1) {
      spread_axis(ng, Dx, Dy, m, axis_g[0], f);
      spread_axis(ng, Dx, Dy, m, axis_g[1], f + 2 * npe);
    }
  }
}

/* physics::*_internal_forces (kernels.hpp:32-35) for one block. */
int oracle_block_forces(const insem_cuda_basis* kb, const insem_cuda_block* blk, int32_t medium,
                        const float* u_local, float* f_local) {
  const int ng = kb->ngll, npe = ng * ng;
  if (ng < 2 || ng > MAXNG) return INSEM_CUDA_ERR_UNSUPPORTED;
  if (!(blk->azimuthal_order == 0 || (blk->azimuthal_order == 1 && blk->kind == INSEM_AXISYM)))
    return INSEM_CUDA_ERR_UNSUPPORTED;
  const int elastic = medium == INSEM_ELASTIC;
  const int nc = elastic ? (blk->azimuthal_order == 1 ? 3 : 2) : 1;
  for (int b = 0; b < blk->n_elements; ++b) {
    const size_t e = (size_t)blk->elements[b];
    const float* u = u_local + e * nc * npe;
    float* f = f_local + e * nc * npe;
    if (blk->kind == INSEM_AXISYM) axisym_element(kb, blk, elastic, b, u, f);
    else cartesian_element(kb, blk, elastic, b, u, f);
  }
  return INSEM_CUDA_OK;
}

/* DofMap::gather (dof_map.hpp:95-120). */
void oracle_gather(const insem_cuda_dofmap* d, int32_t ncomp, const float* global, float* local) {
  const size_t ng = (size_t)d->n_global, npe = (size_t)d->ngll * d->ngll;
  for (int32_t e = 0; e < d->n_elements; ++e) {
    const int32_t* map = d->l2g + (size_t)e * npe;
    for (int c = 0; c < ncomp; ++c) {
      const float* g = global + c * ng;
      float* l = local + ((size_t)e * ncomp + c) * npe;
      for (size_t k = 0; k < npe; ++k) {
        const int32_t m = map[k];
        if (m >= 0) {
          l[k] = g[m];
        } else {
          const int32_t r = -1 - m;
          float s = 0;
          for (int32_t q = d->row_offsets[r]; q < d->row_offsets[r + 1]; ++q)
            s += (float)d->row_weights[q] * g[d->row_dofs[q]];
          l[k] = s;
        }
      }
    }
  }
}

/* DofMap::assemble (dof_map.hpp:123-141). */
void oracle_assemble(const insem_cuda_dofmap* d, int32_t ncomp, const float* local, float* global) {
  const size_t ng = (size_t)d->n_global, npe = (size_t)d->ngll * d->ngll;
  const int weighted = d->t_weights != NULL && d->n_rows > 0;
  for (int32_t g = 0; g < d->n_global; ++g)
    for (int c = 0; c < ncomp; ++c) {
      float sum = 0;
      for (int32_t s = d->t_offsets[g]; s < d->t_offsets[g + 1]; ++s) {
        const size_t slot = (size_t)d->t_slots[s];
        const size_t e = slot / npe, k = slot - e * npe;
        const float v = local[(e * ncomp + c) * npe + k];
        sum += weighted ? (float)d->t_weights[s] * v : v;
      }
      global[c * ng + g] = sum;
    }
}

/* SourceTimeFunction::operator() (description.cpp:88-113). */
static double stf_value(const insem_cuda_stf* s, double t) {
  const double kPi = 3.14159265358979323846;
  switch (s->kind) {
    case INSEM_STF_RICKER: {
      const double x = kPi * s->f0 * (t - s->t0);
      const double a = x * x;
      return s->amplitude * (1.0 - 2.0 * a) * exp(-a);
    }
    case INSEM_STF_GAUSSIAN: {
      const double x = kPi * s->f0 * (t - s->t0);
      return s->amplitude * exp(-(x * x));
    }
    case INSEM_STF_GAUSSIAN_DERIVATIVE: {
      const double tau = t - s->t0;
      const double y = kPi * s->f0;
      const double c = y * y;
      return s->amplitude * (-2.0 * c * tau) * exp(-c * tau * tau);
    }
    case INSEM_STF_SAMPLES: {
      if (s->n_samples <= 0) return 0.0;
      const double x = t / s->sample_dt;
      if (x < 0.0 || x > (double)(s->n_samples - 1)) return 0.0;
      const size_t i = (size_t)x;
      if (i + 1 >= (size_t)s->n_samples) return s->amplitude * s->samples[s->n_samples - 1];
      const double w = x - (double)i;
      return s->amplitude * ((1.0 - w) * s->samples[i] + w * s->samples[i + 1]);
    }
  }
  return 0.0;
}

/* ----------------------------------------------------------------- solver */
typedef struct {
  const insem_cuda_domain* d;
  size_t ng, nl;
  float *u, *v, *a, *f, *u_local, *f_local;
} odomain;

typedef struct oracle_solver {
  const insem_cuda_problem* p;
  odomain dom[2];
  int nd, solid, fluid;
  int step, initialized;
  double potential;
  double* pv;         /* [n_receivers][4] prev_ax, prev_az, vel_x, vel_z */
  int n_cols, max_samples;
  double* traces;     /* [max_samples][n_cols] */
  double* energy;     /* [n_energy][3] */
  int n_energy_cap;
} oracle_solver;

static void apply_dirichlet(const odomain* o, float* x) {
  const insem_cuda_domain* d = o->d;
  for (int c = 0; c < d->ncomp; ++c)
    for (int i = 0; i < d->n_dirichlet; ++i) x[c * o->ng + d->dirichlet_points[i]] = 0;
  for (int q = 0; q < d->n_axis_components; ++q)
    for (int i = 0; i < d->n_axis; ++i) x[d->axis_components[q] * o->ng + d->axis_points[i]] = 0;
}

static double dotf(const float* a, const float* b, size_t n) {
  double s = 0.0;
  for (size_t i = 0; i < n; ++i) s += (double)a[i] * (double)b[i];
  return s;
}

/* Solver::internal_forces (solver.cpp:570-581); returns u . f when asked. */
static double internal_forces(oracle_solver* s, odomain* o, const float* u, int energy) {
  const insem_cuda_domain* d = o->d;
  oracle_gather(&d->dofs, d->ncomp, u, o->u_local);
  for (int b = 0; b < d->n_blocks; ++b) oracle_block_forces(&s->p->basis, &d->blocks[b], d->medium, o->u_local, o->f_local);
  oracle_assemble(&d->dofs, d->ncomp, o->f_local, o->f);
  return energy ? dotf(u, o->f, d->ncomp * o->ng) : 0.0;
}

static void add_coupling_forces(oracle_solver* s, odomain* o) {
  const insem_cuda_coupling* cp = &s->p->coupling;
  if (cp->n == 0) return;
  const int pm = o->d->azimuthal_order == 1;
  const float h = (float)0.70710678118654752440;
  if (o->d->medium == INSEM_ELASTIC) {
    const odomain* fl = &s->dom[s->fluid];
    const size_t ng = o->ng, zc = pm ? 2 * ng : ng;
    for (int i = 0; i < cp->n; ++i) {
      const float p = fl->u[cp->fluid_points[i]];
      const size_t g = cp->solid_points[i];
      if (pm) {
        o->f[g] += h * cp->cx[i] * p;
        o->f[ng + g] += h * cp->cx[i] * p;
      } else {
        o->f[g] += cp->cx[i] * p;
      }
      o->f[zc + g] += cp->cz[i] * p;
    }
  } else {
    const odomain* so = &s->dom[s->solid];
    const size_t ngs = so->ng, zc = pm ? 2 * ngs : ngs;
    for (int i = 0; i < cp->n; ++i) {
      const size_t gs = cp->solid_points[i];
      const float ar = pm ? h * (so->a[gs] + so->a[ngs + gs]) : so->a[gs];
      o->f[cp->fluid_points[i]] -= cp->cx[i] * ar + cp->cz[i] * so->a[zc + gs];
    }
  }
}

static void solve_spd(int n, double* A, double* b) {
  for (int k = 0; k < n; ++k)
    for (int i = k + 1; i < n; ++i) {
      const double l = A[i * n + k] / A[k * n + k];
      for (int j = k; j < n; ++j) A[i * n + j] -= l * A[k * n + j];
      b[i] -= l * b[k];
    }
  for (int k = n - 1; k >= 0; --k) {
    double sum = b[k];
    for (int j = k + 1; j < n; ++j) sum -= A[k * n + j] * b[j];
    b[k] = sum / A[k * n + k];
  }
}

static void solve_acceleration(oracle_solver* s, odomain* o, int implicit) {
  const insem_cuda_domain* d = o->d;
  const size_t ng = o->ng;
  const int nc = d->ncomp;
  for (size_t g = 0; g < ng; ++g)
    for (int c = 0; c < nc; ++c) o->a[c * ng + g] = o->f[c * ng + g] * d->inv_mass[g];
  const double h = implicit ? 0.5 * s->p->dt : 0.0;
  for (int i = 0; i < d->n_absorbing; ++i) {
    const size_t g = d->absorbing_points[i];
    const float* c = d->absorbing_coef + (size_t)nc * nc * i;
    double A[9], rhs[3];
    for (int r = 0; r < nc; ++r) {
      rhs[r] = o->f[r * ng + g];
      for (int q = 0; q < nc; ++q) {
        rhs[r] -= (double)c[r * nc + q] * o->v[q * ng + g];
        A[r * nc + q] = h * c[r * nc + q] + (r == q ? (double)d->mass[g] : 0.0);
      }
    }
    solve_spd(nc, A, rhs);
    for (int r = 0; r < nc; ++r) o->a[r * ng + g] = (float)rhs[r];
  }
  apply_dirichlet(o, o->a);
}

static void compute_acceleration(oracle_solver* s, double t, int energy, int implicit) {
  s->potential = 0.0;
  const int order[2] = {s->solid, s->fluid};
  for (int q = 0; q < 2; ++q) {
    const int di = order[q];
    if (di < 0) continue;
    odomain* o = &s->dom[di];
    s->potential -= 0.5 * internal_forces(s, o, o->u, energy);
    for (int k = 0; k < s->p->n_sources; ++k) {
      const insem_cuda_source* src = &s->p->sources[k];
      if (src->domain != di) continue;
      const float amp = (float)stf_value(&src->stf, t);
      const size_t np = src->n_points;
      for (int c = 0; c < o->d->ncomp; ++c)
        for (size_t i = 0; i < np; ++i) o->f[c * o->ng + src->points[i]] += src->coef[c * np + i] * amp;
    }
    add_coupling_forces(s, o);
    solve_acceleration(s, o, implicit);
  }
}

static double interp(const insem_cuda_receiver* r, const float* field, size_t ng, int c) {
  double sum = 0.0;
  for (int i = 0; i < r->n_points; ++i) sum += (double)r->value[i] * field[c * ng + r->points[i]];
  return sum;
}

static void record(oracle_solver* s) {
  const int sample = s->step / s->p->record_every;
  if (sample >= s->max_samples) return;
  double* row = s->traces + (size_t)sample * s->n_cols;
  int col = 0;
  for (int ri = 0; ri < s->p->n_receivers; ++ri) {
    const insem_cuda_receiver* r = &s->p->receivers[ri];
    const odomain* o = &s->dom[r->domain];
    for (int qi = 0; qi < r->n_quantities; ++qi) {
      const int q = r->quantities[qi];
      if (q == INSEM_Q_PARTICLE_VELOCITY) {
        row[col++] = s->pv[4 * ri + 2];
        row[col++] = s->pv[4 * ri + 3];
        continue;
      }
      const float* field = q == INSEM_Q_VELOCITY ? o->v : q == INSEM_Q_ACCELERATION ? o->a : o->u;
      if (o->d->medium == INSEM_ELASTIC && o->d->azimuthal_order == 1) {
        const double up = interp(r, field, o->ng, 0), um = interp(r, field, o->ng, 1);
        row[col++] = 0.70710678118654752440 * (up + um);
        row[col++] = 0.70710678118654752440 * (up - um);
        row[col++] = interp(r, field, o->ng, 2);
        continue;
      }
      for (int c = 0; c < o->d->ncomp; ++c) row[col++] = interp(r, field, o->ng, c);
    }
  }
}

static double kinetic_energy(oracle_solver* s) {
  const double c = s->p->dt * s->p->dt / 8.0;
  double kin = 0.0;
  for (int di = 0; di < s->nd; ++di) {
    const odomain* o = &s->dom[di];
    for (int comp = 0; comp < o->d->ncomp; ++comp)
      for (size_t g = 0; g < o->ng; ++g) {
        const double v = o->v[comp * o->ng + g], a = o->a[comp * o->ng + g];
        kin += o->d->mass[g] * (0.5 * v * v - c * a * a);
      }
  }
  return kin;
}

static void push_energy(oracle_solver* s) {
  const int k = s->step / s->p->energy_every;
  if (k >= s->n_energy_cap) return;
  s->energy[3 * k] = s->step * s->p->dt;
  s->energy[3 * k + 1] = kinetic_energy(s);
  s->energy[3 * k + 2] = s->potential;
}

static void receiver_accel(oracle_solver* s, int ri, double* ax, double* az) {
  const insem_cuda_receiver* r = &s->p->receivers[ri];
  const odomain* o = &s->dom[r->domain];
  double gx = 0.0, gz = 0.0;
  for (int i = 0; i < r->n_points; ++i) {
    gx += (double)r->d_dx[i] * o->u[r->points[i]];
    gz += (double)r->d_dz[i] * o->u[r->points[i]];
  }
  *ax = -gx / r->rho;
  *az = -gz / r->rho;
}

static void initialize(oracle_solver* s) {
  const int energy = s->p->energy_every > 0;
  compute_acceleration(s, 0.0, energy, 0);
  for (int ri = 0; ri < s->p->n_receivers; ++ri) {
    if (s->dom[s->p->receivers[ri].domain].d->medium != INSEM_ACOUSTIC) continue;
    receiver_accel(s, ri, &s->pv[4 * ri], &s->pv[4 * ri + 1]);
  }
  s->initialized = 1;
  record(s);
  if (energy) push_energy(s);
}

oracle_solver* oracle_solver_create(const insem_cuda_problem* p) {
  oracle_solver* s = (oracle_solver*)calloc(1, sizeof(oracle_solver));
  s->p = p;
  s->nd = p->n_domains;
  s->solid = s->fluid = -1;
  for (int i = 0; i < p->n_domains; ++i) {
    odomain* o = &s->dom[i];
    o->d = &p->domains[i];
    o->ng = (size_t)o->d->dofs.n_global;
    o->nl = (size_t)o->d->dofs.n_elements * p->basis.ngll * p->basis.ngll;
    const size_t nf = o->d->ncomp * o->ng, nlf = o->d->ncomp * o->nl;
    o->u = (float*)calloc(nf, sizeof(float));
    o->v = (float*)calloc(nf, sizeof(float));
    o->a = (float*)calloc(nf, sizeof(float));
    o->f = (float*)calloc(nf, sizeof(float));
    o->u_local = (float*)calloc(nlf, sizeof(float));
    o->f_local = (float*)calloc(nlf, sizeof(float));
    if (o->d->medium == INSEM_ELASTIC) s->solid = i;
    else s->fluid = i;
  }
  s->pv = (double*)calloc(4 * (size_t)(p->n_receivers + 1), sizeof(double));
  int cols = 0;
  for (int ri = 0; ri < p->n_receivers; ++ri) {
    const insem_cuda_receiver* r = &p->receivers[ri];
    const insem_cuda_domain* d = &p->domains[r->domain];
    for (int q = 0; q < r->n_quantities; ++q)
      cols += r->quantities[q] == INSEM_Q_PARTICLE_VELOCITY ? 2 : d->ncomp;
  }
  s->n_cols = cols;
  s->max_samples = p->n_steps / p->record_every + 1;
  s->traces = (double*)calloc((size_t)s->max_samples * (cols > 0 ? cols : 1), sizeof(double));
  s->n_energy_cap = p->energy_every > 0 ? p->n_steps / p->energy_every + 1 : 0;
  s->energy = (double*)calloc(3 * (size_t)(s->n_energy_cap + 1), sizeof(double));
  return s;
}

void oracle_solver_destroy(oracle_solver* s) {
  if (!s) return;
  for (int i = 0; i < s->nd; ++i) {
    odomain* o = &s->dom[i];
    free(o->u); free(o->v); free(o->a); free(o->f); free(o->u_local); free(o->f_local);
  }
  free(s->pv);
  free(s->traces);
  free(s->energy);
  free(s);
}

int oracle_solver_set_state(oracle_solver* s, int32_t medium, const double* u, const double* v) {
  if (s->initialized) return INSEM_CUDA_ERR_STATE;
  for (int i = 0; i < s->nd; ++i) {
    odomain* o = &s->dom[i];
    if (o->d->medium != medium) continue;
    const size_t n = o->d->ncomp * o->ng;
    for (size_t k = 0; k < n; ++k) {
      o->u[k] = (float)u[k];
      o->v[k] = (float)v[k];
    }
    apply_dirichlet(o, o->u);
    apply_dirichlet(o, o->v);
    return INSEM_CUDA_OK;
  }
  return INSEM_CUDA_ERR_INVALID;
}

/* Solver::advance (solver.cpp:917-963). */
void oracle_solver_advance(oracle_solver* s, int32_t n) {
  if (!s->initialized) initialize(s);
  const double dt = s->p->dt;
  const float rdt = (float)dt, half_dt = (float)(0.5 * dt), half_dt2 = (float)(0.5 * dt * dt);
  for (int k = 0; k < n && s->step < s->p->n_steps; ++k) {
    for (int di = 0; di < s->nd; ++di) {
      odomain* o = &s->dom[di];
      const size_t len = o->d->ncomp * o->ng;
      for (size_t i = 0; i < len; ++i) {
        o->u[i] += rdt * o->v[i] + half_dt2 * o->a[i];
        o->v[i] += half_dt * o->a[i];
      }
    }
    ++s->step;
    const int energy = s->p->energy_every > 0 && s->step % s->p->energy_every == 0;
    compute_acceleration(s, s->step * dt, energy, 1);
    for (int di = 0; di < s->nd; ++di) {
      odomain* o = &s->dom[di];
      const size_t len = o->d->ncomp * o->ng;
      for (size_t i = 0; i < len; ++i) o->v[i] += half_dt * o->a[i];
    }
    for (int ri = 0; ri < s->p->n_receivers; ++ri) {
      if (s->dom[s->p->receivers[ri].domain].d->medium != INSEM_ACOUSTIC) continue;
      double ax, az;
      receiver_accel(s, ri, &ax, &az);
      double* pv = &s->pv[4 * ri];
      pv[2] += 0.5 * dt * (pv[0] + ax);
      pv[3] += 0.5 * dt * (pv[1] + az);
      pv[0] = ax;
      pv[1] = az;
    }
    if (s->step % s->p->record_every == 0) record(s);
    if (energy) push_energy(s);
  }
}

int32_t oracle_solver_step(const oracle_solver* s) { return s->step; }
int32_t oracle_solver_n_cols(const oracle_solver* s) { return s->n_cols; }
int32_t oracle_solver_n_samples(const oracle_solver* s) {
  return s->initialized ? s->step / s->p->record_every + 1 : 0;
}
/* Copies samples [n_samples][n_cols]. */
void oracle_solver_samples(const oracle_solver* s, double* out) {
  memcpy(out, s->traces, sizeof(double) * (size_t)oracle_solver_n_samples(s) * s->n_cols);
}
int32_t oracle_solver_n_energy(const oracle_solver* s) {
  return (s->initialized && s->p->energy_every > 0) ? s->step / s->p->energy_every + 1 : 0;
}
void oracle_solver_energy(const oracle_solver* s, double* out) {
  memcpy(out, s->energy, sizeof(double) * 3 * (size_t)oracle_solver_n_energy(s));
}
void oracle_solver_state(const oracle_solver* s, int32_t di, float* u, float* v, float* a) {
  const odomain* o = &s->dom[di];
  const size_t n = o->d->ncomp * o->ng;
  memcpy(u, o->u, n * sizeof(float));
  memcpy(v, o->v, n * sizeof(float));
  memcpy(a, o->a, n * sizeof(float));
}
/* f = -K u of a domain (internal_forces without energy). */
void oracle_internal_forces(oracle_solver* s, int32_t di, const float* u, float* f) {
  odomain* o = &s->dom[di];
  internal_forces(s, o, u, 0);
  memcpy(f, o->f, sizeof(float) * o->d->ncomp * o->ng);
}
