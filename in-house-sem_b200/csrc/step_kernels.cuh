// Point-wise kernels of the time step (cpp/src/solver/solver.cpp:669-963):
// predictor/corrector, sources, fluid-solid coupling, the lumped-mass /
// implicit-Stacey acceleration solve, Dirichlet and axis conditions,
// receivers, energy reductions.  Every kernel reproduces the reference's
// expression order (float or double as the reference has it), so a step is
// bit-identical to the reference float build.
#pragma once

#include "common.cuh"

namespace insem_b200 {

constexpr double kSqrtHalf = 0.70710678118654752440;
constexpr int kReduceBlocks = 512;  // fixed grid of the deterministic reductions
constexpr int kReduceThreads = 256;

// Device-resident counters shared by the kernels of a captured step.
struct StepState {
  int32_t step;           // current step index (after the predictor's increment)
  int32_t nonfinite;      // set when a NaN/Inf was found
  int32_t mode;           // tiled path: 0 normal, 1 final (state complete), 2 initial
  int32_t error;          // a bounded device-side wait gave up
  int32_t parity;         // batched steps: field buffer parity of the current step
  int32_t last_step;      // batched steps: the step that runs in final mode
  double kin_c;           // dt^2 / 8 of the kinetic energy (solver.cpp:903)
};

// u += dt v + dt^2/2 a; v += dt/2 a   (solver.cpp:929-933)
static __global__ void predictor_kernel(float* __restrict__ u, float* __restrict__ v, const float* __restrict__ a,
                                 int64_t n, float rdt, float half_dt, float half_dt2) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float vi = v[i], ai = a[i];
    u[i] = fadd(u[i], fadd(fmul(rdt, vi), fmul(half_dt2, ai)));
    v[i] = fadd(vi, fmul(half_dt, ai));
  }
}

// v += dt/2 a   (solver.cpp:942-943)
static __global__ void corrector_kernel(float* __restrict__ v, const float* __restrict__ a, int64_t n, float half_dt) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    v[i] = fadd(v[i], fmul(half_dt, a[i]));
}

static __global__ void advance_step_kernel(StepState* st) { st->step += 1; }

// Sources (solver.cpp:679-687), merged per global point: every point's
// contributions are applied in source order, f += coef * amp.
struct SourcesDev {
  int32_t n_points = 0;
  const int32_t* points = nullptr;   // [n_points]
  const int32_t* offsets = nullptr;  // [n_points+1] into entries
  const int32_t* source = nullptr;   // [n_entries] source index (row of amp)
  const float* coef = nullptr;       // [n_entries][ncomp]
  const float* amp = nullptr;        // [n_sources][n_amp] (real_t) stf(step * dt)
  int32_t n_amp = 0;
};

static __global__ void sources_kernel(SourcesDev s, const StepState* st, int step_override, float* __restrict__ f,
                               int32_t n_global, int32_t ncomp) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n_points) return;
  const int32_t step = step_override >= 0 ? step_override : st->step;
  const int32_t g = s.points[i];
  for (int32_t q = s.offsets[i]; q < s.offsets[i + 1]; ++q) {
    const float amp = s.amp[static_cast<size_t>(s.source[q]) * s.n_amp + step];
    for (int32_t c = 0; c < ncomp; ++c) {
      float* fc = f + static_cast<size_t>(c) * n_global + g;
      *fc = fadd(*fc, fmul(s.coef[static_cast<size_t>(q) * ncomp + c], amp));
    }
  }
}

// add_coupling_forces, solid side (solver.cpp:700-715): traction p n_f.
static __global__ void coupling_solid_kernel(int32_t n, const int32_t* __restrict__ fluid_points,
                                      const int32_t* __restrict__ solid_points, const float* __restrict__ cx,
                                      const float* __restrict__ cz, const float* __restrict__ p_fluid,
                                      float* __restrict__ f, int32_t ng, bool pm, bool serial) {
  const int32_t first = serial ? 0 : blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t last = serial ? n : first + 1;
  if (serial && (blockIdx.x != 0 || threadIdx.x != 0)) return;
  const float h = static_cast<float>(kSqrtHalf);
  const size_t zc = pm ? 2 * static_cast<size_t>(ng) : static_cast<size_t>(ng);
  for (int32_t i = first; i < last && i < n; ++i) {
    const float p = p_fluid[fluid_points[i]];
    const int32_t g = solid_points[i];
    if (pm) {
      const float t = fmul(fmul(h, cx[i]), p);
      f[g] = fadd(f[g], t);
      f[ng + g] = fadd(f[ng + g], t);
    } else {
      f[g] = fadd(f[g], fmul(cx[i], p));
    }
    f[zc + g] = fadd(f[zc + g], fmul(cz[i], p));
  }
}

// add_coupling_forces, fluid side (solver.cpp:716-726): -n_f . a_s.
static __global__ void coupling_fluid_kernel(int32_t n, const int32_t* __restrict__ fluid_points,
                                      const int32_t* __restrict__ solid_points, const float* __restrict__ cx,
                                      const float* __restrict__ cz, const float* __restrict__ a_solid,
                                      int32_t ngs, float* __restrict__ f, bool pm, bool serial) {
  const int32_t first = serial ? 0 : blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t last = serial ? n : first + 1;
  if (serial && (blockIdx.x != 0 || threadIdx.x != 0)) return;
  const float h = static_cast<float>(kSqrtHalf);
  const size_t zc = pm ? 2 * static_cast<size_t>(ngs) : static_cast<size_t>(ngs);
  for (int32_t i = first; i < last && i < n; ++i) {
    const int32_t gs = solid_points[i];
    const float ar = pm ? fmul(h, fadd(a_solid[gs], a_solid[ngs + gs])) : a_solid[gs];
    const int32_t gf = fluid_points[i];
    f[gf] = fsub(f[gf], fadd(fmul(cx[i], ar), fmul(cz[i], a_solid[zc + gs])));
  }
}

// a = f * inv_mass   (solver.cpp:735-738)
static __global__ void inv_mass_kernel(const float* __restrict__ f, const float* __restrict__ inv_mass,
                                float* __restrict__ a, int32_t ng, int32_t ncomp) {
  const int64_t total = static_cast<int64_t>(ng) * ncomp;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t g = static_cast<int32_t>(i % ng);
    a[i] = fmul(f[i], inv_mass[g]);
  }
}

// solve_spd (solver.cpp:67-80): Gaussian elimination without pivoting, n <= 3.
__device__ __forceinline__ void solve_spd_dev(int n, double* A, double* b) {
  for (int k = 0; k < n; ++k) {
    for (int i = k + 1; i < n; ++i) {
      const double l = __ddiv_rn(A[i * n + k], A[k * n + k]);
      for (int j = k; j < n; ++j) A[i * n + j] = dsub(A[i * n + j], dmul(l, A[k * n + j]));
      b[i] = dsub(b[i], dmul(l, b[k]));
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    double s = b[k];
    for (int j = k + 1; j < n; ++j) s = dsub(s, dmul(A[k * n + j], b[j]));
    b[k] = __ddiv_rn(s, A[k * n + k]);
  }
}

// Stacey points (solver.cpp:740-760): (M + h C) a = f - C v per point, in double.
static __global__ void stacey_kernel(int32_t n_abs, const int32_t* __restrict__ points, const float* __restrict__ coef,
                              const float* __restrict__ mass, const float* __restrict__ f,
                              const float* __restrict__ v, float* __restrict__ a, int32_t ng, int32_t ncomp,
                              double h) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_abs) return;
  const int32_t g = points[i];
  const float* c = coef + static_cast<size_t>(i) * ncomp * ncomp;
  double A[9], rhs[3];
  for (int r = 0; r < ncomp; ++r) {
    rhs[r] = static_cast<double>(f[static_cast<size_t>(r) * ng + g]);
    for (int s = 0; s < ncomp; ++s) {
      rhs[r] = dsub(rhs[r], dmul(static_cast<double>(c[r * ncomp + s]),
                                 static_cast<double>(v[static_cast<size_t>(s) * ng + g])));
      A[r * ncomp + s] =
          dadd(dmul(h, static_cast<double>(c[r * ncomp + s])), r == s ? static_cast<double>(mass[g]) : 0.0);
    }
  }
  solve_spd_dev(ncomp, A, rhs);
  for (int r = 0; r < ncomp; ++r) a[static_cast<size_t>(r) * ng + g] = static_cast<float>(rhs[r]);
}

// apply_dirichlet (solver.hpp:57-65) on a flat list of component*n_global+point indices.
static __global__ void zero_kernel(int32_t n, const int64_t* __restrict__ idx, float* __restrict__ x) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[idx[i]] = 0.0f;
}

// Receivers (solver.cpp:780-811, 945-958).  One record column per thread.
struct ReceiversDev {
  int32_t n = 0;
  const int32_t* offsets = nullptr;  // [n+1] into points/value/d_dx/d_dz
  const int32_t* points = nullptr;
  const float* value = nullptr;
  const float* d_dx = nullptr;
  const float* d_dz = nullptr;
  const double* rho = nullptr;       // [n]
  const int32_t* domain = nullptr;   // [n]
  double* pv = nullptr;              // [n][4] prev_ax, prev_az, vel_x, vel_z
};

// One column of a recorded sample.
struct RecordColumn {
  int32_t receiver;
  int32_t field;  // 0 u, 1 v, 2 a, 3 particle velocity
  int32_t mode;   // 0 component `comp`; 1 (U+ + U-)/sqrt2; 2 (U+ - U-)/sqrt2; 3 vel_x; 4 vel_z
  int32_t comp;
};

// Per-domain field pointers for receivers and energy.
struct DomainFields {
  const float* u;
  const float* v;
  const float* a;
  int32_t ng;
};

struct AllFields {
  DomainFields d[2];
};

// sum over q = beg .. end-1 of (double)coef[q] * (double)field[pts[q]], added
// in ascending q (the reference's order); the loads of four terms are issued
// before their four additions, so their latencies overlap.
__device__ __forceinline__ double ordered_dot(const float* __restrict__ coef, const int32_t* __restrict__ pts,
                                              int32_t beg, int32_t end, const float* __restrict__ field) {
  double s = 0.0;
  int32_t q = beg;
  for (; q + 4 <= end; q += 4) {
    int32_t p[4];
    float c[4], f[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) p[k] = pts[q + k];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      c[k] = coef[q + k];
      f[k] = field[p[k]];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) s = dadd(s, dmul(static_cast<double>(c[k]), static_cast<double>(f[k])));
  }
  for (; q < end; ++q) s = dadd(s, dmul(static_cast<double>(coef[q]), static_cast<double>(field[pts[q]])));
  return s;
}

__device__ __forceinline__ double interp(const ReceiversDev& r, int32_t rec, const float* field, int32_t ng, int c) {
  return ordered_dot(r.value, r.points, r.offsets[rec], r.offsets[rec + 1], field + static_cast<size_t>(c) * ng);
}

// Particle velocity of acoustic receivers: trapezoid of -grad(p)/rho.  With
// init != 0 only prev_a is set (Solver::initialize, solver.cpp:883-893).
__device__ __forceinline__ void particle_velocity_body(const ReceiversDev& r, const AllFields& fl,
                                                       const int32_t* __restrict__ acoustic_recv, int32_t n_acoustic,
                                                       double dt, int init, int32_t t) {
  if (t >= n_acoustic) return;
  const int32_t rec = acoustic_recv[t];
  const DomainFields& d = fl.d[r.domain[rec]];
  // two independent sums, each in ascending point order
  const double gx = ordered_dot(r.d_dx, r.points, r.offsets[rec], r.offsets[rec + 1], d.u);
  const double gz = ordered_dot(r.d_dz, r.points, r.offsets[rec], r.offsets[rec + 1], d.u);
  const double ax = __ddiv_rn(-gx, r.rho[rec]), az = __ddiv_rn(-gz, r.rho[rec]);
  double* pv = r.pv + static_cast<size_t>(rec) * 4;
  if (!init) {
    const double hdt = dmul(0.5, dt);
    pv[2] = dadd(pv[2], dmul(hdt, dadd(pv[0], ax)));
    pv[3] = dadd(pv[3], dmul(hdt, dadd(pv[1], az)));
  }
  pv[0] = ax;
  pv[1] = az;
}

static __global__ void particle_velocity_kernel(ReceiversDev r, AllFields fl, const int32_t* __restrict__ acoustic_recv,
                                         int32_t n_acoustic, double dt, int init) {
  particle_velocity_body(r, fl, acoustic_recv, n_acoustic, dt, init, blockIdx.x * blockDim.x + threadIdx.x);
}

__device__ __forceinline__ void record_body(const ReceiversDev& r, const AllFields& fl,
                                            const RecordColumn* __restrict__ cols, int32_t n_cols, int32_t step,
                                            int32_t record_every, double* __restrict__ traces, int32_t max_samples,
                                            int32_t t) {
  if (t >= n_cols || step % record_every != 0) return;
  const int32_t sample = step / record_every;
  if (sample >= max_samples) return;
  const RecordColumn col = cols[t];
  double out;
  if (col.field == 3) {
    out = r.pv[static_cast<size_t>(col.receiver) * 4 + (col.mode == 3 ? 2 : 3)];
  } else {
    const DomainFields& d = fl.d[r.domain[col.receiver]];
    const float* field = col.field == 0 ? d.u : col.field == 1 ? d.v : d.a;
    if (col.mode == 0) {
      out = interp(r, col.receiver, field, d.ng, col.comp);
    } else {
      const double up = interp(r, col.receiver, field, d.ng, 0), um = interp(r, col.receiver, field, d.ng, 1);
      out = dmul(kSqrtHalf, col.mode == 1 ? dadd(up, um) : dsub(up, um));
    }
  }
  traces[static_cast<size_t>(sample) * n_cols + t] = out;
}

static __global__ void record_kernel(ReceiversDev r, AllFields fl, const RecordColumn* __restrict__ cols, int32_t n_cols,
                              const StepState* st, int32_t record_every, double* __restrict__ traces,
                              int32_t max_samples) {
  record_body(r, fl, cols, n_cols, st->step, record_every, traces, max_samples, blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------- energy
// Deterministic two-level reductions: kReduceBlocks partial sums over a
// grid-stride loop, then one block adds the partials in a fixed tree order.
__device__ __forceinline__ double block_reduce(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] = dadd(sh[threadIdx.x], sh[threadIdx.x + s]);
    __syncthreads();
  }
  return sh[0];
}

// partial[blockIdx] = sum_i (double)x[i] * (double)y[i], gated on energy steps.
static __global__ void dot_partial_kernel(const float* __restrict__ x, const float* __restrict__ y, int64_t n,
                                   const StepState* st, int32_t energy_every, int force, double* partial) {
  __shared__ double sh[kReduceThreads];
  if (!force && (energy_every <= 0 || st->step % energy_every != 0)) return;
  double s = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    s = dadd(s, dmul(static_cast<double>(x[i]), static_cast<double>(y[i])));
  const double b = block_reduce(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = b;
}

// partial[blockIdx] = sum mass[g] (0.5 v v - c a a)   (kinetic_energy, solver.cpp:900-915)
static __global__ void kinetic_partial_kernel(const float* __restrict__ v, const float* __restrict__ a,
                                       const float* __restrict__ mass, int32_t ng, int32_t ncomp, double c,
                                       const StepState* st, int32_t energy_every, int force, double* partial) {
  __shared__ double sh[kReduceThreads];
  if (!force && (energy_every <= 0 || st->step % energy_every != 0)) return;
  const int64_t n = static_cast<int64_t>(ng) * ncomp;
  double s = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double vv = v[i], aa = a[i];
    s = dadd(s, dmul(static_cast<double>(mass[i % ng]), dsub(dmul(dmul(0.5, vv), vv), dmul(dmul(c, aa), aa))));
  }
  const double b = block_reduce(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = b;
}

// energy[sample] = (time, kinetic, potential): kinetic = sum of the n_kin
// partial sets 0..n_kin-1 (domain order), potential = -0.5 * each of the
// n_pot dot sets stored from set 2 on (elastic first, solver.cpp:673-678).
static __global__ void energy_finalize_kernel(const double* partial, int n_kin, int n_pot, const StepState* st,
                                       int32_t energy_every, int force, double dt, double* energy,
                                       int32_t max_samples) {
  __shared__ double sh[kReduceThreads];
  const int32_t step = st->step;
  if (!force && (energy_every <= 0 || step % energy_every != 0)) return;
  const int32_t sample = energy_every > 0 ? step / energy_every : 0;
  double kin = 0.0, pot = 0.0;
  for (int q = 0; q < n_kin + n_pot; ++q) {
    const int set = q < n_kin ? q : 2 + (q - n_kin);
    double s = 0.0;
    for (int i = threadIdx.x; i < kReduceBlocks; i += blockDim.x) s = dadd(s, partial[set * kReduceBlocks + i]);
    const double b = block_reduce(s, sh);
    __syncthreads();
    if (q < n_kin) kin = dadd(kin, b);
    else pot = dsub(pot, dmul(0.5, b));
  }
  if (threadIdx.x == 0 && sample < max_samples) {
    energy[sample * 3 + 0] = dmul(static_cast<double>(step), dt);
    energy[sample * 3 + 1] = kin;
    energy[sample * 3 + 2] = pot;
  }
}

// ------------------------------------------------------- power iteration
// partial[blockIdx] = sum mass[g] x x over [ncomp][ng]   (solver.cpp:597-601, 631-638)
static __global__ void mass_norm_partial_kernel(const float* __restrict__ x, const float* __restrict__ mass, int32_t ng,
                                         int32_t ncomp, double* partial) {
  __shared__ double sh[kReduceThreads];
  const int64_t n = static_cast<int64_t>(ng) * ncomp;
  double s = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double xi = x[i];
    s = dadd(s, dmul(dmul(static_cast<double>(mass[i % ng]), xi), xi));
  }
  const double b = block_reduce(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = b;
}

// x = (float)(-f * inv_mass); partial = sum y^2   (solver.cpp:603-609)
static __global__ void power_update_kernel(const float* __restrict__ f, const float* __restrict__ inv_mass,
                                    float* __restrict__ x, int32_t ng, int32_t ncomp, double* partial) {
  __shared__ double sh[kReduceThreads];
  const int64_t n = static_cast<int64_t>(ng) * ncomp;
  double s = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double y = dmul(-static_cast<double>(f[i]), static_cast<double>(inv_mass[i % ng]));
    x[i] = static_cast<float>(y);
    s = dadd(s, dmul(y, y));
  }
  const double b = block_reduce(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = b;
}

// x = (float)(src * scale)
static __global__ void scale_kernel(const float* __restrict__ src, float* __restrict__ x, int64_t n, double scale) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    x[i] = static_cast<float>(dmul(static_cast<double>(src[i]), scale));
}

// Power-iteration scalars kept on the device, so an iteration needs no host
// round trip: the partial sums, their reductions and the scalar logic of
// estimate_stable_dt / coupled_lambda_max (solver.cpp:583-667) all run in
// stream order; the host reads the result once.
enum PowerSlot : int {
  kPwLambda = 0,   // running max of the Rayleigh quotients (uncoupled domains)
  kPwA = 1,        // reduction results
  kPwB = 2,
  kPwNorm = 3,
  kPwDone = 4,     // the loop has stopped (the reference's break)
  kPwScale = 5,    // factor of the next scaling
  kPwNx = 6,
  kPwNy = 7,
  kPwCoupled = 8,  // running max of sqrt(ny / nx) (coupled operator)
  kPwCount = 9
};

// pw[slot] = sign x (sum of partial[0..n) in index order, as the host loop
// adds them).  One CTA of kReduceBlocks threads stages the partials in shared
// memory with parallel loads; thread 0 then adds them in order.
static __global__ void __launch_bounds__(kReduceBlocks) sum_partials_kernel(const double* __restrict__ partial, int n,
                                                                          double sign, double* pw, int slot) {
  __shared__ double sh[kReduceBlocks];
  for (int i = threadIdx.x; i < n && i < kReduceBlocks; i += blockDim.x) sh[i] = partial[i];
  __syncthreads();
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (int i = 0; i < n && i < kReduceBlocks; ++i) s = dadd(s, sh[i]);
  pw[slot] = sign < 0.0 ? -s : s;
}

// pw[dst] = pw[kPwA] + pw[kPwB]
static __global__ void sum_ab_kernel(double* pw, int dst) {
  if (blockIdx.x == 0 && threadIdx.x == 0) pw[dst] = dadd(pw[kPwA], pw[kPwB]);
}

// One uncoupled power iteration's scalars (solver.cpp:597-612): lambda from
// x.Kx / x.Mx, then stop on a zero norm or set the scale 1 / sqrt(norm).
static __global__ void power_step_kernel(double* pw) {
  if (blockIdx.x != 0 || threadIdx.x != 0 || pw[kPwDone] != 0.0) return;
  const double xmx = pw[kPwB];
  if (xmx > 0.0) {
    const double q = pw[kPwA] / xmx;
    if (pw[kPwLambda] < q) pw[kPwLambda] = q;
  }
  const double norm = pw[kPwNorm];
  if (norm == 0.0) {
    pw[kPwDone] = 1.0;
    return;
  }
  pw[kPwScale] = 1.0 / sqrt(norm);
}

// One coupled iteration's scalars (solver.cpp:641-662): stop on a zero norm,
// sqrt(ny / nx) from iteration 60 on, scale -1 / sqrt(ny).
static __global__ void coupled_step_kernel(double* pw, int it) {
  if (blockIdx.x != 0 || threadIdx.x != 0 || pw[kPwDone] != 0.0) return;
  const double nx = pw[kPwNx], ny = pw[kPwNy];
  if (nx <= 0.0 || ny <= 0.0) {
    pw[kPwDone] = 1.0;
    return;
  }
  if (it >= 60) {
    const double q = sqrt(ny / nx);
    if (pw[kPwCoupled] < q) pw[kPwCoupled] = q;
  }
  pw[kPwScale] = -1.0 / sqrt(ny);
}

// x = (float)(src * pw[kPwScale]) unless the loop has stopped.
static __global__ void scale_dev_kernel(const float* __restrict__ src, float* __restrict__ x, int64_t n,
                                        const double* __restrict__ pw) {
  if (pw[kPwDone] != 0.0) return;
  const double scale = pw[kPwScale];
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    x[i] = static_cast<float>(dmul(static_cast<double>(src[i]), scale));
}

// Sets st->nonfinite if any entry of x is NaN or Inf.
static __global__ void finite_check_kernel(const float* __restrict__ x, int64_t n, StepState* st) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    if (!isfinite(x[i])) {
      st->nonfinite = 1;
      return;
    }
}

}  // namespace insem_b200
