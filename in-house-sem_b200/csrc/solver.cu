// Device-resident twin of solver::Solver (cpp/include/insem/solver/solver.hpp:91-228)
// and its C ABI.  Fields, boundary data, sources and receivers live in HBM;
// the host only launches the step (a CUDA graph per step) and copies traces,
// energy and state back on request.
//
// Step order per solver.cpp:917-963:
//   predictor (all domains) -> step += 1 ->
//   for elastic, acoustic:  element forces (gather fused) -> assemble (CSR, ascending slots)
//                           -> potential energy dot -> sources -> coupling
//                           -> a = f / M, Stacey solve, Dirichlet/axis
//   -> corrector -> acoustic particle velocity -> record -> energy.
#include <algorithm>
#include <map>
#include <memory>
#include <set>

#include "device_data.cuh"
#include "solver.cuh"
#include "stf.hpp"

namespace insem_b200 {

int32_t* pinned_modes();

void DeviceDomainData::upload(const insem_cuda_domain& d, const insem_cuda_basis& basis) {
  medium = d.medium;
  INSEM_REQUIRE(medium == INSEM_ACOUSTIC || medium == INSEM_ELASTIC, INSEM_CUDA_ERR_INVALID, "unknown medium");
  m = d.azimuthal_order;
  ncomp = d.ncomp;
  INSEM_REQUIRE(ncomp == ncomp_of(medium, m), INSEM_CUDA_ERR_INVALID, "ncomp does not match medium and order");
  INSEM_REQUIRE(d.dofs.ngll == basis.ngll, INSEM_CUDA_ERR_INVALID, "DofMap and basis differ in ngll");
  dofs.upload(d.dofs);
  ng = dofs.n_global;
  npe = dofs.npe;
  n_elements = dofs.n_elements;
  INSEM_REQUIRE(static_cast<int64_t>(ng) * ncomp < (int64_t{1} << 31), INSEM_CUDA_ERR_INVALID, "domain too large");
  blocks.clear();
  blocks.resize(d.n_blocks);
  for (int b = 0; b < d.n_blocks; ++b) {
    blocks[b].upload(d.blocks[b], basis.ngll, medium);
    for (int32_t e : blocks[b].host_elements)
      INSEM_REQUIRE(e >= 0 && e < n_elements, INSEM_CUDA_ERR_INVALID, "block element out of range");
    any_axial |= blocks[b].any_axial;
  }
  host_mass = host_vec(d.mass, ng);
  mass.upload(host_mass);
  inv_mass.upload(host_vec(d.inv_mass, ng));
  n_abs = d.n_absorbing;
  const auto ap = host_vec(d.absorbing_points, n_abs);
  for (int32_t g : ap) INSEM_REQUIRE(g >= 0 && g < ng, INSEM_CUDA_ERR_INVALID, "absorbing point out of range");
  absorbing_points.upload(ap);
  absorbing_coef.upload(host_vec(d.absorbing_coef, static_cast<std::size_t>(n_abs) * ncomp * ncomp));
  std::vector<int64_t> z;
  const auto dp = host_vec(d.dirichlet_points, d.n_dirichlet);
  for (int c = 0; c < ncomp; ++c)
    for (int32_t g : dp) {
      INSEM_REQUIRE(g >= 0 && g < ng, INSEM_CUDA_ERR_INVALID, "Dirichlet point out of range");
      z.push_back(static_cast<int64_t>(c) * ng + g);
    }
  const auto axp = host_vec(d.axis_points, d.n_axis);
  const auto axc = host_vec(d.axis_components, d.n_axis_components);
  for (int32_t c : axc) {
    INSEM_REQUIRE(c >= 0 && c < ncomp, INSEM_CUDA_ERR_INVALID, "axis component out of range");
    for (int32_t g : axp) {
      INSEM_REQUIRE(g >= 0 && g < ng, INSEM_CUDA_ERR_INVALID, "axis point out of range");
      z.push_back(static_cast<int64_t>(c) * ng + g);
    }
  }
  host_zero = z;
  zero_idx.upload(z);
}

void DeviceDomainData::alloc_fields(cudaStream_t s) {
  if (fields_ready) return;
  const std::size_t nf = static_cast<std::size_t>(ncomp) * ng;
  u.resize(nf);
  v.resize(nf);
  a.resize(nf);
  f.resize(nf);
  f_local.resize(static_cast<std::size_t>(ncomp) * n_elements * npe);
  // zeroed in the order of the stream that uses them next (a memset on the
  // default stream is not ordered with the solver's non-blocking streams)
  u.zero(s);
  v.zero(s);
  a.zero(s);
  f.zero(s);
  f_local.zero(s);
  fields_ready = true;
}

void DeviceDomainData::free_fields() {
  u.resize(0);
  v.resize(0);
  a.resize(0);
  f.resize(0);
  f_local.resize(0);
  fields_ready = false;
}

Solver::Solver(const insem_cuda_problem& p, const insem_cuda_options* opt, bool setup_only,
               const insem_cuda_time* time) {
  if (opt) opts = *opt;
  else {
    opts = insem_cuda_options{};
    opts.use_graphs = 1;
    opts.check_finite = 1;
  }
  device = opts.device;
  DeviceGuard dg(device);
  CUDA_CHECK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  CUDA_CHECK(cudaEventCreate(&ev0));
  CUDA_CHECK(cudaEventCreate(&ev1));
  CUDA_CHECK(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
  CUDA_CHECK(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
  CUDA_CHECK(cudaEventCreateWithFlags(&join_ev, cudaEventDisableTiming));
  check_ngll(p.basis.ngll);
  ngll = p.basis.ngll;
  INSEM_REQUIRE(p.n_domains >= 1 && p.n_domains <= 2, INSEM_CUDA_ERR_INVALID, "a problem has 1 or 2 domains");
  INSEM_REQUIRE(p.record_every >= 1, INSEM_CUDA_ERR_INVALID, "record_every must be >= 1");
  INSEM_REQUIRE(p.energy_every >= 0, INSEM_CUDA_ERR_INVALID, "energy_every must be >= 0");
  INSEM_REQUIRE((setup_only || time || p.dt > 0.0) && (time || p.n_steps >= 0), INSEM_CUDA_ERR_INVALID,
                "dt must be positive and n_steps >= 0");
  dt = p.dt;
  n_steps = p.n_steps;
  record_every = p.record_every;
  energy_every = p.energy_every;
  domains.resize(p.n_domains);
  bool need_dj = false;
  for (int i = 0; i < p.n_domains; ++i) {
    domains[i].upload(p.domains[i], p.basis);
    need_dj |= domains[i].any_axial;
  }
  basis.upload(p.basis, need_dj);
  for (int i = 0; i < p.n_domains; ++i) {
    if (domains[i].medium == INSEM_ELASTIC) solid = i;
    else fluid = i;
  }
  INSEM_REQUIRE(p.n_domains == 1 || (solid >= 0 && fluid >= 0), INSEM_CUDA_ERR_INVALID,
                "two domains must be one acoustic and one elastic");
  build_coupling(p.coupling);
  st = static_cast<StepState*>(device_alloc(sizeof(StepState)));
  CUDA_CHECK(cudaMemset(st, 0, sizeof(StepState)));
  partial.resize(static_cast<std::size_t>(kReduceBlocks) * 4);
  if (time) {
    // Solver::Solver (solver.cpp:131-144)
    stable_dt_estimate = stable_dt();
    if (time->dt > 0.0) {
      INSEM_REQUIRE(time->dt <= stable_dt_estimate, INSEM_CUDA_ERR_INVALID,
                    "time step " + std::to_string(time->dt) + " s exceeds the estimated stability limit " +
                        std::to_string(stable_dt_estimate) + " s");
      dt = time->dt;
    } else {
      INSEM_REQUIRE(time->safety > 0.0 && time->safety <= 1.0, INSEM_CUDA_ERR_INVALID,
                    "time step safety factor must be in (0, 1]");
      dt = time->safety * stable_dt_estimate;
    }
    if (time->n_steps > 0) n_steps = time->n_steps;
    else if (time->duration > 0.0) n_steps = static_cast<int32_t>(std::ceil(time->duration / dt - 1e-9));
    else n_steps = 0;
    // the power iteration's two-pass fields; the path chosen below allocates what it uses
    for (auto& d : domains) d.free_fields();
  }
  build_sources(p);
  build_receivers(p);
  const int32_t n_energy = energy_every > 0 ? n_steps / energy_every + 1 : 0;
  energy.resize(static_cast<std::size_t>(std::max(n_energy, 1)) * 3);
  energy.zero();
  {
    StepState hs{};
    hs.kin_c = dt * dt / 8.0;
    CUDA_CHECK(cudaMemcpy(st, &hs, sizeof(hs), cudaMemcpyHostToDevice));
  }
  // the two-pass path's global fields and element-local forces; the tiled
  // path keeps its own fields and allocates these only for internal_forces()
  if (setup_only || opts.path == 1)
    for (auto& d : domains) d.alloc_fields();
  if (!setup_only && opts.path != 1) build_tiled(p);
  if (!setup_only) prepare_noalloc();
  // uploads and zeroing ran on the legacy stream and this solver's stream;
  // other streams (other solvers, batches) are not waited for
  CUDA_CHECK(cudaStreamSynchronize(nullptr));
  CUDA_CHECK(cudaStreamSynchronize(stream));
}

Solver::~Solver() {
  DeviceGuard dg(device);
  // buffers go back to the pool below: both streams must be done with them
  if (stream) cudaStreamSynchronize(stream);
  if (side) cudaStreamSynchronize(side);
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  for (auto& g : tgraph)
    if (g) cudaGraphExecDestroy(g);
  device_free(st);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (fork_ev) cudaEventDestroy(fork_ev);
  if (join_ev) cudaEventDestroy(join_ev);
  if (side) cudaStreamDestroy(side);
  if (stream) cudaStreamDestroy(stream);
}

void Solver::build_coupling(const insem_cuda_coupling& c) {
  n_cpl = c.n;
  if (n_cpl == 0) return;
  INSEM_REQUIRE(solid >= 0 && fluid >= 0, INSEM_CUDA_ERR_INVALID, "coupling needs both media");
  const auto fp = host_vec(c.fluid_points, n_cpl), sp = host_vec(c.solid_points, n_cpl);
  std::set<int32_t> fs, ss;
  for (int i = 0; i < n_cpl; ++i) {
    INSEM_REQUIRE(fp[i] >= 0 && fp[i] < domains[fluid].ng && sp[i] >= 0 && sp[i] < domains[solid].ng,
                  INSEM_CUDA_ERR_INVALID, "coupling point out of range");
    fs.insert(fp[i]);
    ss.insert(sp[i]);
  }
  // Repeated points make the per-point updates order-dependent: keep the
  // reference's sequential order then.
  cpl_serial_fluid = static_cast<int>(fs.size()) != n_cpl;
  cpl_serial_solid = static_cast<int>(ss.size()) != n_cpl;
  cpl_fluid.upload(fp);
  cpl_solid.upload(sp);
  cpl_cx.upload(host_vec(c.cx, n_cpl));
  cpl_cz.upload(host_vec(c.cz, n_cpl));
}

void Solver::build_sources(const insem_cuda_problem& p) {
  n_sources = p.n_sources;
  n_amp = n_steps + 1;
  std::vector<float> amp(static_cast<std::size_t>(std::max(n_sources, 1)) * n_amp, 0.0f);
  // Per domain: point -> ordered (source, coef) contributions.
  std::vector<std::map<int32_t, std::vector<std::pair<int32_t, std::vector<float>>>>> per(domains.size());
  for (int s = 0; s < n_sources; ++s) {
    const insem_cuda_source& so = p.sources[s];
    INSEM_REQUIRE(so.domain >= 0 && so.domain < static_cast<int>(domains.size()), INSEM_CUDA_ERR_INVALID,
                  "source domain out of range");
    const auto& d = domains[so.domain];
    const auto pts = host_vec(so.points, so.n_points);
    const auto coef = host_vec(so.coef, static_cast<std::size_t>(so.n_points) * d.ncomp);
    for (int i = 0; i < so.n_points; ++i) {
      INSEM_REQUIRE(pts[i] >= 0 && pts[i] < d.ng, INSEM_CUDA_ERR_INVALID, "source point out of range");
      std::vector<float> cs(d.ncomp);
      for (int c = 0; c < d.ncomp; ++c) cs[c] = coef[static_cast<std::size_t>(c) * so.n_points + i];
      per[so.domain][pts[i]].push_back({s, cs});
    }
    for (int k = 0; k < n_amp; ++k)
      amp[static_cast<std::size_t>(s) * n_amp + k] = static_cast<float>(stf_value(so.stf, k * dt));
  }
  src_amp.upload(amp);
  src_per_point = per;
  src.resize(domains.size());
  for (std::size_t di = 0; di < domains.size(); ++di) {
    std::vector<int32_t> points, offsets{0}, which;
    std::vector<float> coefs;
    for (const auto& [g, list] : per[di]) {
      points.push_back(g);
      for (const auto& [s, cs] : list) {
        which.push_back(s);
        coefs.insert(coefs.end(), cs.begin(), cs.end());
      }
      offsets.push_back(static_cast<int32_t>(which.size()));
    }
    auto& sd = src[di];
    sd.n_points = static_cast<int32_t>(points.size());
    sd.points.upload(points);
    sd.offsets.upload(offsets);
    sd.source.upload(which);
    sd.coef.upload(coefs);
  }
}

void Solver::build_receivers(const insem_cuda_problem& p) {
  n_receivers = p.n_receivers;
  std::vector<int32_t> offsets{0}, points, dom, acoustic;
  std::vector<float> value, ddx, ddz;
  std::vector<double> rho;
  std::vector<RecordColumn> cols;
  for (int r = 0; r < n_receivers; ++r) {
    const insem_cuda_receiver& rc = p.receivers[r];
    INSEM_REQUIRE(rc.domain >= 0 && rc.domain < static_cast<int>(domains.size()), INSEM_CUDA_ERR_INVALID,
                  "receiver domain out of range");
    const auto& d = domains[rc.domain];
    const auto pts = host_vec(rc.points, rc.n_points);
    for (int32_t g : pts) INSEM_REQUIRE(g >= 0 && g < d.ng, INSEM_CUDA_ERR_INVALID, "receiver point out of range");
    points.insert(points.end(), pts.begin(), pts.end());
    const auto vv = host_vec(rc.value, rc.n_points), dx = host_vec(rc.d_dx, rc.n_points),
               dz = host_vec(rc.d_dz, rc.n_points);
    value.insert(value.end(), vv.begin(), vv.end());
    ddx.insert(ddx.end(), dx.begin(), dx.end());
    ddz.insert(ddz.end(), dz.begin(), dz.end());
    offsets.push_back(static_cast<int32_t>(points.size()));
    dom.push_back(rc.domain);
    rho.push_back(rc.rho);
    if (d.medium == INSEM_ACOUSTIC) acoustic.push_back(r);
    const auto qs = host_vec(rc.quantities, rc.n_quantities);
    for (int32_t q : qs) {
      TraceInfo ti;
      ti.first_col = static_cast<int32_t>(cols.size());
      if (q == INSEM_Q_PARTICLE_VELOCITY) {
        INSEM_REQUIRE(d.medium == INSEM_ACOUSTIC, INSEM_CUDA_ERR_INVALID, "particle_velocity needs an acoustic receiver");
        cols.push_back({r, 3, 3, 0});
        cols.push_back({r, 3, 4, 0});
      } else {
        const bool elastic_q = q == INSEM_Q_DISPLACEMENT || q == INSEM_Q_VELOCITY || q == INSEM_Q_ACCELERATION;
        INSEM_REQUIRE(elastic_q == (d.medium == INSEM_ELASTIC) && (elastic_q || q == INSEM_Q_PRESSURE),
                      INSEM_CUDA_ERR_INVALID, "quantity does not exist in the receiver's medium");
        const int32_t field = q == INSEM_Q_VELOCITY ? 1 : q == INSEM_Q_ACCELERATION ? 2 : 0;
        if (d.medium == INSEM_ELASTIC && d.m == 1) {
          cols.push_back({r, field, 1, 0});
          cols.push_back({r, field, 2, 0});
          cols.push_back({r, field, 0, 2});
        } else {
          for (int c = 0; c < d.ncomp; ++c) cols.push_back({r, field, 0, c});
        }
      }
      ti.ncomp = static_cast<int32_t>(cols.size()) - ti.first_col;
      traces.push_back(ti);
    }
  }
  n_cols = static_cast<int32_t>(cols.size());
  rec_offsets.upload(offsets);
  rec_points.upload(points);
  rec_value.upload(value);
  rec_ddx.upload(ddx);
  rec_ddz.upload(ddz);
  rec_rho.upload(rho);
  rec_domain.upload(dom);
  rec_acoustic.upload(acoustic);
  n_acoustic_rec = static_cast<int32_t>(acoustic.size());
  rec_pv.resize(static_cast<std::size_t>(std::max(n_receivers, 1)) * 4);
  rec_pv.zero();
  rec_cols.upload(cols);
  max_samples = n_steps / record_every + 1;
  trace_buf.resize(static_cast<std::size_t>(std::max(n_cols, 1)) * max_samples);
  trace_buf.zero();
}

ReceiversDev Solver::receivers_view() {
  ReceiversDev r;
  r.n = n_receivers;
  r.offsets = rec_offsets.get();
  r.points = rec_points.get();
  r.value = rec_value.get();
  r.d_dx = rec_ddx.get();
  r.d_dz = rec_ddz.get();
  r.rho = rec_rho.get();
  r.domain = rec_domain.get();
  r.pv = rec_pv.get();
  return r;
}

AllFields Solver::fields_view() {
  AllFields f{};
  for (std::size_t i = 0; i < domains.size() && i < 2; ++i)
    f.d[i] = {domains[i].u.get(), domains[i].v.get(), domains[i].a.get(), domains[i].ng};
  return f;
}

void Solver::internal_forces(DeviceDomainData& d, const float* u_global, float* f_global) {
  d.alloc_fields(stream);
  for (const DeviceBlock& b : d.blocks) {
    ElementLaunch a;
    a.basis = basis.view();
    a.blk = b.view();
    a.u_in = u_global;
    a.l2g = d.dofs.l2g.get();
    a.rows = d.dofs.rows();
    a.n_global = d.ng;
    a.f_local = d.f_local.get();
    a.gather = true;
    a.elastic = d.medium == INSEM_ELASTIC;
    a.stream = stream;
    launch_element_forces(ngll, a);
  }
  launch_assemble(d.dofs, d.ncomp, d.f_local.get(), f_global, stream);
}

// compute_acceleration (solver.cpp:669-691) for one domain.
void Solver::domain_acceleration(int di, int pot_set, int force_energy, double h, int step_override) {
  DeviceDomainData& d = domains[di];
  internal_forces(d, d.u.get(), d.f.get());
  dot_partial_kernel<<<kReduceBlocks, kReduceThreads, 0, stream>>>(
      d.u.get(), d.f.get(), static_cast<int64_t>(d.ncomp) * d.ng, st, energy_every, force_energy,
      partial.get() + static_cast<std::size_t>(pot_set) * kReduceBlocks);
  CUDA_LAUNCH_CHECK();
  const auto& sd = src[di];
  if (sd.n_points > 0) {
    SourcesDev s;
    s.n_points = sd.n_points;
    s.points = sd.points.get();
    s.offsets = sd.offsets.get();
    s.source = sd.source.get();
    s.coef = sd.coef.get();
    s.amp = src_amp.get();
    s.n_amp = n_amp;
    sources_kernel<<<ceil_div(sd.n_points, 128), 128, 0, stream>>>(s, st, step_override, d.f.get(), d.ng, d.ncomp);
    CUDA_LAUNCH_CHECK();
  }
  coupling_forces(di);
  inv_mass_kernel<<<grid_for(static_cast<int64_t>(d.ng) * d.ncomp), 256, 0, stream>>>(
      d.f.get(), d.inv_mass.get(), d.a.get(), d.ng, d.ncomp);
  CUDA_LAUNCH_CHECK();
  if (d.n_abs > 0) {
    stacey_kernel<<<ceil_div(d.n_abs, 128), 128, 0, stream>>>(d.n_abs, d.absorbing_points.get(),
                                                               d.absorbing_coef.get(), d.mass.get(), d.f.get(),
                                                               d.v.get(), d.a.get(), d.ng, d.ncomp, h);
    CUDA_LAUNCH_CHECK();
  }
  zero_constrained(d, d.a.get());
}

void Solver::zero_constrained(DeviceDomainData& d, float* x) {
  if (d.host_zero.empty()) return;
  zero_kernel<<<ceil_div(static_cast<int64_t>(d.host_zero.size()), 256), 256, 0, stream>>>(
      static_cast<int32_t>(d.host_zero.size()), d.zero_idx.get(), x);
  CUDA_LAUNCH_CHECK();
}

// add_coupling_forces (solver.cpp:693-727) into domains[di].f.
void Solver::coupling_forces(int di) {
  if (n_cpl == 0) return;
  DeviceDomainData& d = domains[di];
  const bool pm = d.m == 1;
  if (d.medium == INSEM_ELASTIC) {
    coupling_solid_kernel<<<cpl_serial_solid ? 1 : ceil_div(n_cpl, 128), 128, 0, stream>>>(
        n_cpl, cpl_fluid.get(), cpl_solid.get(), cpl_cx.get(), cpl_cz.get(), domains[fluid].u.get(), d.f.get(),
        d.ng, pm, cpl_serial_solid);
  } else {
    const auto& s = domains[solid];
    coupling_fluid_kernel<<<cpl_serial_fluid ? 1 : ceil_div(n_cpl, 128), 128, 0, stream>>>(
        n_cpl, cpl_fluid.get(), cpl_solid.get(), cpl_cx.get(), cpl_cz.get(), s.a.get(), s.ng, d.f.get(),
        s.m == 1, cpl_serial_fluid);
  }
  CUDA_LAUNCH_CHECK();
}

// Sum of the kReduceBlocks partials of set 0, in a fixed order on the host.
double Solver::reduce_partials() {
  std::vector<double> h(kReduceBlocks);
  CUDA_CHECK(cudaMemcpyAsync(h.data(), partial.get(), kReduceBlocks * sizeof(double), cudaMemcpyDeviceToHost, stream));
  CUDA_CHECK(cudaStreamSynchronize(stream));
  double s = 0.0;
  for (double v : h) s += v;
  return s;
}

void Solver::replay(int n, const std::function<void()>& body) {
  if (n <= 0) return;
  cudaGraph_t g = nullptr;
  CUDA_CHECK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  try {
    body();
  } catch (...) {
    // leave capture mode before the error propagates
    if (cudaStreamEndCapture(stream, &g) == cudaSuccess && g) cudaGraphDestroy(g);
    cudaGetLastError();
    throw;
  }
  CUDA_CHECK(cudaStreamEndCapture(stream, &g));
  cudaGraphExec_t ge = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  CUDA_CHECK(e);
  cudaError_t le = cudaSuccess;
  for (int i = 0; i < n && le == cudaSuccess; ++i) le = cudaGraphLaunch(ge, stream);
  const cudaError_t se = cudaStreamSynchronize(stream);
  cudaGraphExecDestroy(ge);
  CUDA_CHECK(le);
  CUDA_CHECK(se);
}

// estimate_stable_dt (solver.cpp:583-619): 100 power iterations per domain
// with x ~ U(-1, 1) from mt19937(12345), Rayleigh quotients in double.
double Solver::stable_dt() {
  DeviceGuard dg(device);
  for (auto& d : domains) d.alloc_fields(stream);
  std::mt19937 rng(12345);
  std::uniform_real_distribution<double> dist(-1.0, 1.0);
  DeviceBuffer<double> pw(kPwCount);
  pw.zero(stream);
  auto reduce_into = [&](int slot, double sign) {
    sum_partials_kernel<<<1, kReduceBlocks, 0, stream>>>(partial.get(), kReduceBlocks, sign, pw.get(), slot);
    CUDA_LAUNCH_CHECK();
  };
  for (auto& d : domains) {
    const int64_t n = static_cast<int64_t>(d.ncomp) * d.ng;
    std::vector<float> x(n);
    for (auto& v : x) v = static_cast<float>(dist(rng));
    DeviceBuffer<float> dx(n);
    CUDA_CHECK(cudaMemcpyAsync(dx.get(), x.data(), n * sizeof(float), cudaMemcpyHostToDevice, stream));
    CUDA_CHECK(cudaMemsetAsync(pw.get() + kPwDone, 0, sizeof(double), stream));
    replay(100, [&] {
      zero_constrained(d, dx.get());
      internal_forces(d, dx.get(), d.f.get());
      dot_partial_kernel<<<kReduceBlocks, kReduceThreads, 0, stream>>>(dx.get(), d.f.get(), n, st, 0, 1,
                                                                       partial.get());
      CUDA_LAUNCH_CHECK();
      reduce_into(kPwA, -1.0);  // x.Kx = -(x . f_int)
      mass_norm_partial_kernel<<<kReduceBlocks, kReduceThreads, 0, stream>>>(dx.get(), d.mass.get(), d.ng,
                                                                             d.ncomp, partial.get());
      CUDA_LAUNCH_CHECK();
      reduce_into(kPwB, 1.0);
      power_update_kernel<<<kReduceBlocks, kReduceThreads, 0, stream>>>(d.f.get(), d.inv_mass.get(), dx.get(),
                                                                        d.ng, d.ncomp, partial.get());
      CUDA_LAUNCH_CHECK();
      reduce_into(kPwNorm, 1.0);
      power_step_kernel<<<1, 1, 0, stream>>>(pw.get());
      CUDA_LAUNCH_CHECK();
      scale_dev_kernel<<<grid_for(n), 256, 0, stream>>>(dx.get(), dx.get(), n, pw.get());
      CUDA_LAUNCH_CHECK();
    });
    d.f.zero(stream);
    // dx is released below: its last kernels must have run
    CUDA_CHECK(cudaStreamSynchronize(stream));
  }
  if (n_cpl > 0) coupled_lambda_max(rng, pw.get());
  double h[kPwCount];
  CUDA_CHECK(cudaMemcpyAsync(h, pw.get(), sizeof(h), cudaMemcpyDeviceToHost, stream));
  CUDA_CHECK(cudaStreamSynchronize(stream));
  double lambda = h[kPwLambda];
  if (n_cpl > 0) lambda = std::max(lambda, h[kPwCoupled]);
  INSEM_REQUIRE(lambda > 0.0, INSEM_CUDA_ERR_INVALID, "could not estimate the stable time step (empty or rigid model?)");
  return 2.0 / std::sqrt(lambda);
}

// coupled_lambda_max (solver.cpp:621-667): growth of the mass norm under the
// coupled operator, 120 iterations, sqrt(ny / nx) from iteration 60 on; the
// result lands in pw[kPwCoupled].
void Solver::coupled_lambda_max(std::mt19937& rng, double* pw) {
  DeviceDomainData& sd = domains[solid];
  DeviceDomainData& fd = domains[fluid];
  std::uniform_real_distribution<double> dist(-1.0, 1.0);
  std::vector<std::vector<float>> x0(2);
  int q = 0;
  for (DeviceDomainData* d : {&sd, &fd}) {
    auto& x = x0[q++];
    x.resize(static_cast<std::size_t>(d->ncomp) * d->ng);
    for (auto& v : x) v = static_cast<float>(dist(rng));
    CUDA_CHECK(cudaMemcpyAsync(d->u.get(), x.data(), x.size() * sizeof(float), cudaMemcpyHostToDevice, stream));
  }
  CUDA_CHECK(cudaMemsetAsync(pw + kPwDone, 0, sizeof(double), stream));
  CUDA_CHECK(cudaMemsetAsync(pw + kPwCoupled, 0, sizeof(double), stream));
  auto mass_norm = [&](DeviceDomainData& d, const float* x, int slot) {
    mass_norm_partial_kernel<<<kReduceBlocks, kReduceThreads, 0, stream>>>(x, d.mass.get(), d.ng, d.ncomp,
                                                                           partial.get());
    CUDA_LAUNCH_CHECK();
    sum_partials_kernel<<<1, kReduceBlocks, 0, stream>>>(partial.get(), kReduceBlocks, 1.0, pw, slot);
    CUDA_LAUNCH_CHECK();
  };
  // iterations 0..59 and 60..119 differ only in coupled_step_kernel's test it >= 60
  auto iteration = [&](int it) {
    zero_constrained(sd, sd.u.get());
    zero_constrained(fd, fd.u.get());
    mass_norm(sd, sd.u.get(), kPwA);
    mass_norm(fd, fd.u.get(), kPwB);
    sum_ab_kernel<<<1, 1, 0, stream>>>(pw, kPwNx);
    CUDA_LAUNCH_CHECK();
    for (int di : {solid, fluid}) {
      DeviceDomainData& d = domains[di];
      internal_forces(d, d.u.get(), d.f.get());
      coupling_forces(di);
      inv_mass_kernel<<<grid_for(static_cast<int64_t>(d.ng) * d.ncomp), 256, 0, stream>>>(
          d.f.get(), d.inv_mass.get(), d.a.get(), d.ng, d.ncomp);
      CUDA_LAUNCH_CHECK();
      zero_constrained(d, d.a.get());
    }
    mass_norm(sd, sd.a.get(), kPwA);
    mass_norm(fd, fd.a.get(), kPwB);
    sum_ab_kernel<<<1, 1, 0, stream>>>(pw, kPwNy);
    CUDA_LAUNCH_CHECK();
    coupled_step_kernel<<<1, 1, 0, stream>>>(pw, it);
    CUDA_LAUNCH_CHECK();
    for (DeviceDomainData* d : {&sd, &fd}) {
      const int64_t n = static_cast<int64_t>(d->ncomp) * d->ng;
      scale_dev_kernel<<<grid_for(n), 256, 0, stream>>>(d->a.get(), d->u.get(), n, pw);
      CUDA_LAUNCH_CHECK();
    }
  };
  replay(60, [&] { iteration(0); });
  replay(60, [&] { iteration(60); });
  for (DeviceDomainData* d : {&sd, &fd}) {
    d->u.zero(stream);
    d->a.zero(stream);
    d->f.zero(stream);
  }
  CUDA_CHECK(cudaStreamSynchronize(stream));  // the host start vectors are read until here
}

// Kernels of the whole acceleration solve, elastic first (solver.cpp:674).
void Solver::compute_acceleration(int force_energy, double h, int step_override) {
  int set = 0;
  n_pot_sets = 0;
  if (solid >= 0) domain_acceleration(solid, 2 + set++, force_energy, h, step_override);
  if (fluid >= 0) domain_acceleration(fluid, 2 + set++, force_energy, h, step_override);
  n_pot_sets = set;
}

void Solver::observers(int force_energy, int init) {
  if (n_acoustic_rec > 0) {
    particle_velocity_kernel<<<ceil_div(n_acoustic_rec, 64), 64, 0, stream>>>(
        receivers_view(), fields_view(), rec_acoustic.get(), n_acoustic_rec, dt, init);
    CUDA_LAUNCH_CHECK();
  }
  if (n_cols > 0) {
    record_kernel<<<ceil_div(n_cols, 64), 64, 0, stream>>>(receivers_view(), fields_view(), rec_cols.get(), n_cols,
                                                            st, record_every, trace_buf.get(), max_samples);
    CUDA_LAUNCH_CHECK();
  }
  if (energy_every > 0 || force_energy) {
    const double c = dt * dt / 8.0;
    int set = 0;
    for (auto& d : domains) {
      kinetic_partial_kernel<<<kReduceBlocks, kReduceThreads, 0, stream>>>(
          d.v.get(), d.a.get(), d.mass.get(), d.ng, d.ncomp, c, st, energy_every, force_energy,
          partial.get() + static_cast<std::size_t>(set++) * kReduceBlocks);
      CUDA_LAUNCH_CHECK();
    }
    energy_finalize_kernel<<<1, kReduceThreads, 0, stream>>>(partial.get(), set, n_pot_sets, st, energy_every,
                                                              force_energy, dt, energy.get(),
                                                              static_cast<int32_t>(energy.size() / 3));
    CUDA_LAUNCH_CHECK();
  }
}

void Solver::enqueue_step() {
  const float rdt = static_cast<float>(dt);
  const float half_dt = static_cast<float>(0.5 * dt);
  const float half_dt2 = static_cast<float>(0.5 * dt * dt);
  for (auto& d : domains) {
    const int64_t n = static_cast<int64_t>(d.ncomp) * d.ng;
    predictor_kernel<<<grid_for(n), 256, 0, stream>>>(d.u.get(), d.v.get(), d.a.get(), n, rdt, half_dt, half_dt2);
    CUDA_LAUNCH_CHECK();
  }
  advance_step_kernel<<<1, 1, 0, stream>>>(st);
  CUDA_LAUNCH_CHECK();
  compute_acceleration(0, 0.5 * dt, -1);
  for (auto& d : domains) {
    const int64_t n = static_cast<int64_t>(d.ncomp) * d.ng;
    corrector_kernel<<<grid_for(n), 256, 0, stream>>>(d.v.get(), d.a.get(), n, half_dt);
    CUDA_LAUNCH_CHECK();
  }
  observers(0, 0);
}

void Solver::initialize() {
  // compute_acceleration(0, energy, explicit damping) then observers at t = 0
  // (Solver::initialize, solver.cpp:878-898).
  const int force = energy_every > 0 ? 1 : 0;
  compute_acceleration(force, 0.0, 0);
  observers(force, 1);
  initialized = true;
}

void Solver::set_state(int32_t medium, const double* u_in, const double* v_in) {
  INSEM_REQUIRE(!initialized, INSEM_CUDA_ERR_STATE, "initial conditions must be set before the first time step");
  int di = -1;
  for (std::size_t i = 0; i < domains.size(); ++i)
    if (domains[i].medium == medium) di = static_cast<int>(i);
  INSEM_REQUIRE(di >= 0, INSEM_CUDA_ERR_INVALID, "the model has no such medium");
  auto& d = domains[di];
  const std::size_t n = static_cast<std::size_t>(d.ncomp) * d.ng;
  INSEM_REQUIRE(u_in && v_in, INSEM_CUDA_ERR_INVALID, "null state array");
  std::vector<float> fu(n), fv(n);
  for (std::size_t i = 0; i < n; ++i) {
    fu[i] = static_cast<float>(u_in[i]);
    fv[i] = static_cast<float>(v_in[i]);
  }
  for (int64_t z : d.host_zero) fu[z] = fv[z] = 0.0f;
  if (!tiled) {
    CUDA_CHECK(cudaMemcpy(d.u.get(), fu.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d.v.get(), fv.data(), n * sizeof(float), cudaMemcpyHostToDevice));
  } else {
    TiledDomain& t = tdom[di];
    const std::size_t nd = static_cast<std::size_t>(d.ncomp) * t.ng;
    std::vector<float> pu(nd, 0.0f), pv(nd, 0.0f);
    for (int c = 0; c < d.ncomp; ++c)
      for (int32_t g = 0; g < d.ng; ++g) {
        pu[static_cast<std::size_t>(c) * t.ng + t.perm[g]] = fu[static_cast<std::size_t>(c) * d.ng + g];
        pv[static_cast<std::size_t>(c) * t.ng + t.perm[g]] = fv[static_cast<std::size_t>(c) * d.ng + g];
      }
    CUDA_CHECK(cudaMemcpy(t.u_cur(parity), pu.data(), nd * sizeof(float), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(t.v.get(), pv.data(), nd * sizeof(float), cudaMemcpyHostToDevice));
  }
}

void Solver::advance(int32_t n) {
  DeviceGuard dg(device);
  INSEM_REQUIRE(n >= 0, INSEM_CUDA_ERR_INVALID, "negative step count");
  INSEM_REQUIRE(!in_batch, INSEM_CUDA_ERR_STATE, "this solve is stepped by a batch");
  if (snap_every <= 0) {
    advance_span(n);
    return;
  }
  // spans that end on snapshot steps, where the state is complete
  double ms = 0.0;
  if (!initialized) {
    advance_span(0);
    ms += last_ms;
    record_snapshot();
  }
  int32_t left = std::min<int32_t>(n, n_steps - step);
  while (left > 0) {
    const int32_t k = std::min<int32_t>(left, snap_every - step % snap_every);
    advance_span(k);
    ms += last_ms;
    left -= k;
    if (step % snap_every == 0) record_snapshot();
  }
  last_ms = ms;
}

void Solver::advance_span(int32_t n) {
  if (tiled) {
    int32_t dummy = 0;
    advance_tiled(n, nullptr, nullptr, &dummy);
    return;
  }
  CUDA_CHECK(cudaEventRecord(ev0, stream));
  if (!initialized) initialize();
  const int32_t todo = std::min<int32_t>(n, n_steps - step);
  if (todo > 0) {
    if (opts.use_graphs) {
      ensure_graph();
      for (int32_t s = 0; s < todo; ++s) CUDA_CHECK(cudaGraphLaunch(graph_exec, stream));
    } else {
      for (int32_t s = 0; s < todo; ++s) enqueue_step();
    }
    step += todo;
  }
  CUDA_CHECK(cudaEventRecord(ev1, stream));
  if (opts.check_finite) {
    for (auto& d : domains) {
      const int64_t nn = static_cast<int64_t>(d.ncomp) * d.ng;
      finite_check_kernel<<<grid_for(nn), 256, 0, stream>>>(d.u.get(), nn, st);
      CUDA_LAUNCH_CHECK();
    }
  }
  CUDA_CHECK(cudaStreamSynchronize(stream));
  float ms = 0.0f;
  CUDA_CHECK(cudaEventElapsedTime(&ms, ev0, ev1));
  last_ms = ms;
  if (opts.check_finite) {
    StepState hs;
    CUDA_CHECK(cudaMemcpy(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost));
    if (hs.nonfinite) nonfinite_seen = true;
    INSEM_REQUIRE(!hs.nonfinite, INSEM_CUDA_ERR_NONFINITE, "the solution contains NaN or Inf (unstable time step?)");
  }
}

// Captures one step into a CUDA graph (once) and counts its kernel nodes.
void Solver::ensure_graph() {
  if (graph_exec) return;
  cudaGraph_t g = nullptr;
  CUDA_CHECK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue_step();
  } catch (...) {
    cudaStreamEndCapture(stream, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  CUDA_CHECK(cudaStreamEndCapture(stream, &g));
  std::size_t n_nodes = 0;
  CUDA_CHECK(cudaGraphGetNodes(g, nullptr, &n_nodes));
  std::vector<cudaGraphNode_t> nodes(n_nodes);
  if (n_nodes) CUDA_CHECK(cudaGraphGetNodes(g, nodes.data(), &n_nodes));
  kernels_per_step = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    CUDA_CHECK(cudaGraphNodeGetType(nd, &t));
    if (t == cudaGraphNodeTypeKernel) ++kernels_per_step;
  }
  CUDA_CHECK(cudaGraphInstantiate(&graph_exec, g, 0));
  CUDA_CHECK(cudaGraphDestroy(g));
}

// Per step: source amplitudes in (H2D), the step's graph, the record row out (D2H).
void Solver::advance_streamed(int32_t n, const float* amp_in, double* rows_out, int32_t* n_rows) {
  INSEM_REQUIRE(!in_batch, INSEM_CUDA_ERR_STATE, "this solve is stepped by a batch");
  INSEM_REQUIRE(snap_every <= 0, INSEM_CUDA_ERR_STATE, "snapshots are recorded by advance(), not the streamed form");
  DeviceGuard dg(device);
  INSEM_REQUIRE(n >= 0 && n_rows, INSEM_CUDA_ERR_INVALID, "invalid streamed advance");
  INSEM_REQUIRE(n_sources == 0 || amp_in, INSEM_CUDA_ERR_INVALID, "missing source amplitudes");
  if (tiled) {
    advance_tiled(n, amp_in, rows_out, n_rows);
    return;
  }
  if (!initialized) initialize();
  ensure_graph();
  const int32_t todo = std::min<int32_t>(n, n_steps - step);
  int32_t rows = 0;
  CUDA_CHECK(cudaEventRecord(ev0, stream));
  for (int32_t k = 0; k < todo; ++k) {
    const int32_t s = step + 1 + k;
    for (int q = 0; q < n_sources; ++q)
      CUDA_CHECK(cudaMemcpyAsync(src_amp.get() + static_cast<std::size_t>(q) * n_amp + s,
                                 amp_in + static_cast<std::size_t>(k) * n_sources + q, sizeof(float),
                                 cudaMemcpyHostToDevice, stream));
    CUDA_CHECK(cudaGraphLaunch(graph_exec, stream));
    if (s % record_every == 0 && rows_out && n_cols > 0) {
      CUDA_CHECK(cudaMemcpyAsync(rows_out + static_cast<std::size_t>(rows) * n_cols,
                                 trace_buf.get() + static_cast<std::size_t>(s / record_every) * n_cols,
                                 n_cols * sizeof(double), cudaMemcpyDeviceToHost, stream));
      ++rows;
    }
  }
  CUDA_CHECK(cudaEventRecord(ev1, stream));
  CUDA_CHECK(cudaStreamSynchronize(stream));
  step += todo;
  float ms = 0.0f;
  CUDA_CHECK(cudaEventElapsedTime(&ms, ev0, ev1));
  last_ms = ms;
  *n_rows = rows;
}

int32_t Solver::n_samples() const { return initialized ? step / record_every + 1 : 0; }

void Solver::copy_trace(int32_t t, double* out) {
  INSEM_REQUIRE(t >= 0 && t < static_cast<int32_t>(traces.size()), INSEM_CUDA_ERR_INVALID, "trace index out of range");
  const int32_t ns = n_samples();
  if (ns == 0) return;
  std::vector<double> buf(static_cast<std::size_t>(ns) * n_cols);
  CUDA_CHECK(cudaMemcpy(buf.data(), trace_buf.get(), buf.size() * sizeof(double), cudaMemcpyDeviceToHost));
  const TraceInfo& ti = traces[t];
  for (int32_t s = 0; s < ns; ++s)
    for (int32_t c = 0; c < ti.ncomp; ++c)
      out[static_cast<std::size_t>(s) * ti.ncomp + c] = buf[static_cast<std::size_t>(s) * n_cols + ti.first_col + c];
}

int32_t Solver::n_energy() const {
  if (!initialized || energy_every <= 0) return 0;
  return step / energy_every + 1;
}

void Solver::copy_state(int32_t di, double* u_out, double* v_out, double* a_out) {
  INSEM_REQUIRE(di >= 0 && di < static_cast<int32_t>(domains.size()), INSEM_CUDA_ERR_INVALID, "domain out of range");
  auto& d = domains[di];
  CUDA_CHECK(cudaStreamSynchronize(stream));
  if (tiled) {  // before the first step: the set state, a = 0
    TiledDomain& t = tdom[di];
    auto conv = [&](const float* dev, double* out) {
      if (!out) return;
      std::vector<float> h(static_cast<std::size_t>(d.ncomp) * t.ng);
      CUDA_CHECK(cudaMemcpy(h.data(), dev, h.size() * sizeof(float), cudaMemcpyDeviceToHost));
      for (int c = 0; c < d.ncomp; ++c)
        for (int32_t g = 0; g < d.ng; ++g)
          out[static_cast<std::size_t>(c) * d.ng + g] = h[static_cast<std::size_t>(c) * t.ng + t.perm[g]];
    };
    conv(t.u_cur(parity), u_out);
    conv(t.v.get(), v_out);
    conv(t.a.get(), a_out);
    return;
  }
  auto conv = [&](DeviceBuffer<float>& b, double* out) {
    if (!out) return;
    const auto h = b.download();
    for (std::size_t i = 0; i < h.size(); ++i) out[i] = h[i];
  };
  conv(d.u, u_out);
  conv(d.v, v_out);
  conv(d.a, a_out);
}

// ------------------------------------------------------------ tiled path
void Solver::build_tiled(const insem_cuda_problem& p) {
  const std::size_t npe = static_cast<std::size_t>(ngll) * ngll;
  set_constant_basis(ngll, host_vec(p.basis.D, npe), p.basis.Dj ? host_vec(p.basis.Dj, npe) : std::vector<float>{},
                     host_vec(p.basis.w2, npe));
  const auto fp = host_vec(p.coupling.fluid_points, n_cpl), sp = host_vec(p.coupling.solid_points, n_cpl);
  tdom.resize(domains.size());
  for (std::size_t di = 0; di < domains.size(); ++di) {
    const insem_cuda_domain& d = p.domains[di];
    SpecialTerms terms;
    terms.sources = src_per_point[di];
    for (int32_t i = 0; i < n_cpl; ++i) {
      if (static_cast<int>(di) == fluid) terms.coupling[fp[i]].push_back(i);
      if (static_cast<int>(di) == solid) terms.coupling[sp[i]].push_back(i);
    }
    const auto ap = host_vec(d.absorbing_points, d.n_absorbing);
    for (int32_t i = 0; i < d.n_absorbing; ++i) terms.absorbing[ap[i]] = i;
    const uint8_t all = static_cast<uint8_t>((1u << d.ncomp) - 1u);
    for (int32_t g : host_vec(d.dirichlet_points, d.n_dirichlet)) terms.zero[g] |= all;
    const auto axc = host_vec(d.axis_components, d.n_axis_components);
    uint8_t axm = 0;
    for (int32_t c : axc) axm |= static_cast<uint8_t>(1u << c);
    if (axm)
      for (int32_t g : host_vec(d.axis_points, d.n_axis)) terms.zero[g] |= axm;
    for (int r = 0; r < p.n_receivers; ++r)
      if (p.receivers[r].domain == static_cast<int>(di))
        for (int32_t g : host_vec(p.receivers[r].points, p.receivers[r].n_points)) terms.receivers.push_back(g);
    // tile size by the domain's dominant element kind
    std::map<int, int64_t> per_kind;
    for (int b = 0; b < d.n_blocks; ++b) per_kind[d.blocks[b].kind] += d.blocks[b].n_elements;
    int kind = INSEM_RECT;
    int64_t most = -1;
    for (const auto& kv : per_kind)
      if (kv.second > most) {
        most = kv.second;
        kind = kv.first;
      }
    const int te = choose_tile_elements(ngll, kind, d.medium == INSEM_ELASTIC, kind == INSEM_AXISYM ? d.azimuthal_order : 0,
                                        d.ncomp, opts.tile_elements);
    tdom[di].build(d, ngll, te, terms,
                   host_vec(d.absorbing_coef, static_cast<std::size_t>(d.n_absorbing) * d.ncomp * d.ncomp));
  }
  if (n_cpl > 0) {
    std::vector<int32_t> f(n_cpl), s(n_cpl);
    for (int32_t i = 0; i < n_cpl; ++i) {
      f[i] = tdom[fluid].perm[fp[i]];
      s[i] = tdom[solid].perm[sp[i]];
    }
    tcpl_fluid.upload(f);
    tcpl_solid.upload(s);
  }
  std::vector<int32_t> rp;
  for (int r = 0; r < p.n_receivers; ++r)
    for (int32_t g : host_vec(p.receivers[r].points, p.receivers[r].n_points))
      rp.push_back(tdom[p.receivers[r].domain].perm[g]);
  trec_points.upload(rp.empty() ? std::vector<int32_t>{0} : rp);
  int base = 0;
  for (std::size_t di = 0; di < tdom.size(); ++di) {
    ep_tile[di] = base;
    ep_ntile[di] = tdom[di].n_tiles;
    base += tdom[di].n_tiles;
    ep_halo[di] = base;
    ep_nhalo[di] = ceil_div(std::max(tdom[di].n_halo, 1), 256);
    base += ep_nhalo[di];
  }
  epart.resize(2 * static_cast<std::size_t>(std::max(base, 1)));
  epart.zero();
  mode_host = pinned_modes();
  tiled = true;
}

AllFields Solver::tiled_fields(int par) {
  AllFields f{};
  for (std::size_t i = 0; i < tdom.size() && i < 2; ++i)
    f.d[i] = {tdom[i].u_cur(par), tdom[i].vn.get(), tdom[i].a.get(), tdom[i].ng};
  return f;
}

// Pinned {normal, final, init} shared by every solver for the whole process
// (a per-solver pinned buffer would cost a device-wide wait when freed).
int32_t* pinned_modes() {
  static std::once_flag once;
  static int32_t* modes = nullptr;
  std::call_once(once, [] {
    CUDA_CHECK(cudaMallocHost(&modes, 4 * sizeof(int32_t)));
    modes[0] = kModeNormal;
    modes[1] = kModeFinal;
    modes[2] = kModeInit;
    modes[3] = kModeIdle;
  });
  return modes;
}

void Solver::set_mode(int mode) {
  if (mode == cur_mode) return;
  CUDA_CHECK(cudaMemcpyAsync(&st->mode, mode_host + mode, sizeof(int32_t), cudaMemcpyHostToDevice, stream));
  cur_mode = mode;
}

// One step of the tiled path on the field buffers of `par` (init: step 0,
// explicit damping, no step increment).
void Solver::enqueue_tiled(int par, bool init) {
  if (!init) {
    advance_step_kernel<<<1, 1, 0, stream>>>(st);
    CUDA_LAUNCH_CHECK();
  }
  StepScalars sc{static_cast<float>(dt), static_cast<float>(0.5 * dt), static_cast<float>(0.5 * dt * dt),
                 energy_every};
  for (std::size_t di = 0; di < tdom.size(); ++di) {
    TiledDomain& t = tdom[di];
    if (t.n_cslots > 0) {
      constrained_gather_kernel<<<ceil_div(t.n_cslots, 128), 128, 0, stream>>>(
          t.n_cslots, t.cs_row.get(), t.rows(), t.u_cur(par), t.ng, t.ncomp, t.cval.get());
      CUDA_LAUNCH_CHECK();
    }
  }
  // the fluid's tiles beside the solid's: neither reads what the other
  // writes (the solid's halo kernel reads the fluid's current field only)
  const bool split = solid >= 0 && fluid >= 0;
  if (split) {
    CUDA_CHECK(cudaEventRecord(fork_ev, stream));
    CUDA_CHECK(cudaStreamWaitEvent(side, fork_ev, 0));
  }
  for (int di : {solid, fluid}) {
    if (di < 0) continue;
    TiledDomain& t = tdom[di];
    for (std::size_t b = 0; b < t.blocks.size(); ++b) {
      TileLaunch a;
      a.dom = &t;
      a.block = static_cast<int>(b);
      a.parity = par;
      a.sc = sc;
      a.st = st;
      a.epartial = epart.get() + 2 * static_cast<std::size_t>(ep_tile[di]);
      a.elastic = t.medium == INSEM_ELASTIC;
      a.stream = split && di == fluid ? side : stream;
      launch_tiles(ngll, a);
    }
  }
  if (split) {
    CUDA_CHECK(cudaEventRecord(join_ev, side));
    CUDA_CHECK(cudaStreamWaitEvent(stream, join_ev, 0));
  }
  const double h_damp = init ? 0.0 : 0.5 * dt;
  CouplingDev cp{tcpl_fluid.get(), tcpl_solid.get(), cpl_cx.get(), cpl_cz.get()};
  for (int di : {solid, fluid}) {
    if (di < 0) continue;
    TiledDomain& t = tdom[di];
    if (t.n_halo == 0) continue;
    const bool el = t.medium == INSEM_ELASTIC;
    const float* other = nullptr;
    int32_t other_ng = 0;
    bool pm = false;
    if (n_cpl > 0) {
      if (el) {
        other = tdom[fluid].u_cur(par);
        other_ng = tdom[fluid].ng;
        pm = t.m == 1;
      } else {
        other = tdom[solid].a.get();
        other_ng = tdom[solid].ng;
        pm = tdom[solid].m == 1;
      }
    }
    const int grid = ceil_div(t.n_halo, 256);
    double* ep = epart.get();
    const int e0 = ep_halo[di];
    const TiledDev tv = t.view(par);
    const HaloDev hv = t.halo_view();
    if (!el) {
      halo_step_kernel<1, false><<<grid, 256, 0, stream>>>(tv, hv, cp, other, other_ng, pm, src_amp.get(), n_amp, sc,
                                                           h_damp, st, ep, e0);
    } else if (t.ncomp == 2) {
      halo_step_kernel<2, true><<<grid, 256, 0, stream>>>(tv, hv, cp, other, other_ng, pm, src_amp.get(), n_amp, sc,
                                                          h_damp, st, ep, e0);
    } else {
      halo_step_kernel<3, true><<<grid, 256, 0, stream>>>(tv, hv, cp, other, other_ng, pm, src_amp.get(), n_amp, sc,
                                                          h_damp, st, ep, e0);
    }
    CUDA_LAUNCH_CHECK();
  }
  ReceiversDev rv = receivers_view();
  rv.points = trec_points.get();
  if (n_acoustic_rec > 0) {
    particle_velocity_kernel<<<ceil_div(n_acoustic_rec, 64), 64, 0, stream>>>(rv, tiled_fields(par),
                                                                              rec_acoustic.get(), n_acoustic_rec, dt,
                                                                              init ? 1 : 0);
    CUDA_LAUNCH_CHECK();
  }
  if (n_cols > 0) {
    record_kernel<<<ceil_div(n_cols, 64), 64, 0, stream>>>(rv, tiled_fields(par), rec_cols.get(), n_cols, st,
                                                            record_every, trace_buf.get(), max_samples);
    CUDA_LAUNCH_CHECK();
  }
  if (energy_every > 0) {
    // potential order: elastic first
    const int d0 = solid >= 0 ? solid : fluid;
    const int d1 = solid >= 0 ? fluid : -1;
    const int n_dom = d1 >= 0 ? 2 : 1;
    int4 s0{ep_tile[d0], ep_ntile[d0], ep_halo[d0], tdom[d0].n_halo > 0 ? ep_nhalo[d0] : 0};
    int4 s1{0, 0, 0, 0};
    if (d1 >= 0) s1 = int4{ep_tile[d1], ep_ntile[d1], ep_halo[d1], tdom[d1].n_halo > 0 ? ep_nhalo[d1] : 0};
    tiled_energy_kernel<<<1, kReduceThreads, 0, stream>>>(epart.get(), n_dom, s0, s1, st, energy_every, dt,
                                                          energy.get(), static_cast<int32_t>(energy.size() / 3));
    CUDA_LAUNCH_CHECK();
  }
}

void Solver::tiled_begin_steps() {
  if (!complete) return;
  for (auto& t : tdom) {
    const int64_t n = static_cast<int64_t>(t.ncomp) * t.ng;
    predictor_inplace_kernel<<<grid_for(n), 256, 0, stream>>>(t.u_cur(parity), t.v.get(), t.a.get(), n,
                                                             static_cast<float>(dt), static_cast<float>(0.5 * dt),
                                                             static_cast<float>(0.5 * dt * dt));
    CUDA_LAUNCH_CHECK();
  }
  complete = false;
}

// advance(n) on the tiled path; with rows_out, the streamed variant (amplitudes
// in, recorded rows out, per step).
void Solver::advance_tiled(int32_t n, const float* amp_in, double* rows_out, int32_t* n_rows) {
  const bool streamed = rows_out != nullptr || amp_in != nullptr;
  CUDA_CHECK(cudaEventRecord(ev0, stream));
  if (!initialized) {
    set_mode(kModeInit);
    enqueue_tiled(parity, true);
    parity ^= 1;
    complete = true;
    initialized = true;
  }
  const int32_t todo = std::min<int32_t>(n, n_steps - step);
  if (todo > 0 && opts.use_graphs && !tgraph[0]) {
    for (int par = 0; par < 2; ++par) {
      cudaGraph_t g = nullptr;
      CUDA_CHECK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      try {
        enqueue_tiled(par, false);
      } catch (...) {
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      CUDA_CHECK(cudaStreamEndCapture(stream, &g));
      if (par == 0) {
        std::size_t nn = 0;
        CUDA_CHECK(cudaGraphGetNodes(g, nullptr, &nn));
        std::vector<cudaGraphNode_t> nodes(nn);
        if (nn) CUDA_CHECK(cudaGraphGetNodes(g, nodes.data(), &nn));
        kernels_per_step = 0;
        for (auto nd : nodes) {
          cudaGraphNodeType ty;
          CUDA_CHECK(cudaGraphNodeGetType(nd, &ty));
          if (ty == cudaGraphNodeTypeKernel) ++kernels_per_step;
        }
      }
      CUDA_CHECK(cudaGraphInstantiate(&tgraph[par], g, 0));
      CUDA_CHECK(cudaGraphDestroy(g));
    }
  }
  int32_t rows = 0;
  for (int32_t k = 0; k < todo; ++k) {
    tiled_begin_steps();
    set_mode(k == todo - 1 ? kModeFinal : kModeNormal);
    const int32_t s = step + 1 + k;
    if (amp_in)
      for (int q = 0; q < n_sources; ++q)
        CUDA_CHECK(cudaMemcpyAsync(src_amp.get() + static_cast<std::size_t>(q) * n_amp + s,
                                   amp_in + static_cast<std::size_t>(k) * n_sources + q, sizeof(float),
                                   cudaMemcpyHostToDevice, stream));
    if (opts.use_graphs) CUDA_CHECK(cudaGraphLaunch(tgraph[parity], stream));
    else enqueue_tiled(parity, false);
    parity ^= 1;
    if (rows_out && s % record_every == 0 && n_cols > 0) {
      CUDA_CHECK(cudaMemcpyAsync(rows_out + static_cast<std::size_t>(rows) * n_cols,
                                 trace_buf.get() + static_cast<std::size_t>(s / record_every) * n_cols,
                                 n_cols * sizeof(double), cudaMemcpyDeviceToHost, stream));
      ++rows;
    }
  }
  if (todo > 0) complete = true;
  step += todo;
  CUDA_CHECK(cudaEventRecord(ev1, stream));
  if (opts.check_finite && !streamed) {
    for (auto& t : tdom) {
      const int64_t nn = static_cast<int64_t>(t.ncomp) * t.ng;
      finite_check_kernel<<<grid_for(nn), 256, 0, stream>>>(t.u_cur(parity), nn, st);
      CUDA_LAUNCH_CHECK();
    }
  }
  CUDA_CHECK(cudaStreamSynchronize(stream));
  float ms = 0.0f;
  CUDA_CHECK(cudaEventElapsedTime(&ms, ev0, ev1));
  last_ms = ms;
  *n_rows = rows;
  StepState hs;
  CUDA_CHECK(cudaMemcpy(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost));
  INSEM_REQUIRE(!hs.error, INSEM_CUDA_ERR_TIMEOUT, "a tile's bulk copies did not arrive within the wait limit");
  if (hs.nonfinite) nonfinite_seen = true;
  if (opts.check_finite && !streamed)
    INSEM_REQUIRE(!hs.nonfinite, INSEM_CUDA_ERR_NONFINITE, "the solution contains NaN or Inf (unstable time step?)");
}

}  // namespace insem_b200

using namespace insem_b200;

extern "C" {

int insem_cuda_solver_create(const insem_cuda_problem* problem, const insem_cuda_options* options,
                             insem_cuda_solver** out) {
  return guarded([&] {
    INSEM_REQUIRE(problem && out, INSEM_CUDA_ERR_INVALID, "null argument");
    auto h = std::make_unique<insem_cuda_solver>();
    h->s = std::make_unique<Solver>(*problem, options);
    *out = h.release();
  });
}

int insem_cuda_solver_create_timed(const insem_cuda_problem* problem, const insem_cuda_time* time,
                                   const insem_cuda_options* options, insem_cuda_solver** out) {
  return guarded([&] {
    INSEM_REQUIRE(problem && time && out, INSEM_CUDA_ERR_INVALID, "null argument");
    auto h = std::make_unique<insem_cuda_solver>();
    h->s = std::make_unique<Solver>(*problem, options, false, time);
    *out = h.release();
  });
}

double insem_cuda_solver_stable_dt(const insem_cuda_solver* h) { return h ? h->s->stable_dt_estimate : 0.0; }

void insem_cuda_solver_destroy(insem_cuda_solver* h) { delete h; }

int insem_cuda_solver_set_state(insem_cuda_solver* h, int32_t medium, const double* u, const double* v) {
  return guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    DeviceGuard dg(h->s->device);
    h->s->set_state(medium, u, v);
  });
}

int insem_cuda_solver_advance(insem_cuda_solver* h, int32_t n) {
  return guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    h->s->advance(n);
  });
}

int insem_cuda_solver_run(insem_cuda_solver* h) {
  return guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    h->s->advance(h->s->n_steps - h->s->step);
  });
}

int32_t insem_cuda_solver_step(const insem_cuda_solver* h) { return h ? h->s->step : -1; }
int32_t insem_cuda_solver_status(const insem_cuda_solver* h) {
  if (!h) return INSEM_CUDA_ERR_INVALID;
  return h->s->nonfinite_seen ? INSEM_CUDA_ERR_NONFINITE : INSEM_CUDA_OK;
}
int32_t insem_cuda_solver_n_steps(const insem_cuda_solver* h) { return h ? h->s->n_steps : -1; }
double insem_cuda_solver_dt(const insem_cuda_solver* h) { return h ? h->s->dt : 0.0; }
int32_t insem_cuda_solver_n_samples(const insem_cuda_solver* h) { return h ? h->s->n_samples() : -1; }
int32_t insem_cuda_solver_n_traces(const insem_cuda_solver* h) {
  return h ? static_cast<int32_t>(h->s->traces.size()) : -1;
}
int32_t insem_cuda_solver_trace_ncomp(const insem_cuda_solver* h, int32_t t) {
  if (!h || t < 0 || t >= static_cast<int32_t>(h->s->traces.size())) return -1;
  return h->s->traces[t].ncomp;
}

int insem_cuda_solver_trace(insem_cuda_solver* h, int32_t trace, double* out) {
  return guarded([&] {
    INSEM_REQUIRE(h && out, INSEM_CUDA_ERR_INVALID, "null argument");
    DeviceGuard dg(h->s->device);
    h->s->copy_trace(trace, out);
  });
}

int insem_cuda_solver_times(insem_cuda_solver* h, double* out) {
  return guarded([&] {
    INSEM_REQUIRE(h && out, INSEM_CUDA_ERR_INVALID, "null argument");
    const int32_t ns = h->s->n_samples();
    for (int32_t s = 0; s < ns; ++s) out[s] = static_cast<double>(s * h->s->record_every) * h->s->dt;
  });
}

int insem_cuda_solver_energy(insem_cuda_solver* h, double* out, int32_t capacity, int32_t* n_out) {
  return guarded([&] {
    INSEM_REQUIRE(h && n_out, INSEM_CUDA_ERR_INVALID, "null argument");
    DeviceGuard dg(h->s->device);
    const int32_t n = h->s->n_energy();
    *n_out = n;
    if (!out || n == 0) return;
    INSEM_REQUIRE(capacity >= n, INSEM_CUDA_ERR_INVALID, "energy buffer too small");
    CUDA_CHECK(cudaMemcpy(out, h->s->energy.get(), static_cast<std::size_t>(n) * 3 * sizeof(double),
                          cudaMemcpyDeviceToHost));
  });
}

int insem_cuda_solver_state(insem_cuda_solver* h, int32_t domain, double* u, double* v, double* a) {
  return guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    DeviceGuard dg(h->s->device);
    h->s->copy_state(domain, u, v, a);
  });
}

double insem_cuda_solver_last_advance_ms(const insem_cuda_solver* h) { return h ? h->s->last_ms : 0.0; }

int insem_cuda_solver_internal_forces(insem_cuda_solver* h, int32_t domain, const float* u, float* f) {
  return guarded([&] {
    INSEM_REQUIRE(h && u && f, INSEM_CUDA_ERR_INVALID, "null argument");
    Solver& s = *h->s;
    DeviceGuard dg(s.device);
    INSEM_REQUIRE(domain >= 0 && domain < static_cast<int32_t>(s.domains.size()), INSEM_CUDA_ERR_INVALID,
                  "domain out of range");
    auto& d = s.domains[domain];
    const std::size_t n = static_cast<std::size_t>(d.ncomp) * d.ng;
    DeviceBuffer<float> du, df(n);
    du.upload(u, n);
    s.internal_forces(d, du.get(), df.get());
    CUDA_CHECK(cudaStreamSynchronize(s.stream));
    CUDA_CHECK(cudaMemcpy(f, df.get(), n * sizeof(float), cudaMemcpyDeviceToHost));
  });
}

int insem_cuda_set_tile_elements(int32_t ngll, int32_t kind, int32_t medium, int32_t azimuthal_order,
                                 int32_t tile_elements) {
  return guarded([&] {
    INSEM_REQUIRE(kind >= INSEM_RECT && kind <= INSEM_AXISYM, INSEM_CUDA_ERR_INVALID, "unknown geometry kind");
    INSEM_REQUIRE(azimuthal_order == 0 || (azimuthal_order == 1 && kind == INSEM_AXISYM), INSEM_CUDA_ERR_INVALID,
                  "azimuthal order 1 needs the axisymmetric kind");
    set_tile_elements(ngll, kind, medium == INSEM_ELASTIC, azimuthal_order, tile_elements);
  });
}

int32_t insem_cuda_tile_elements(int32_t ngll, int32_t kind, int32_t medium, int32_t azimuthal_order, int32_t ncomp) {
  int32_t out = 0;
  guarded([&] {
    out = choose_tile_elements(ngll, kind, medium == INSEM_ELASTIC, kind == INSEM_AXISYM ? azimuthal_order : 0, ncomp, 0);
  });
  return out;
}

int32_t insem_cuda_solver_tile_elements(const insem_cuda_solver* h, int32_t domain) {
  if (!h || !h->s->tiled || domain < 0 || domain >= static_cast<int32_t>(h->s->domains.size())) return 0;
  return h->s->tiled_tile_elements(domain);
}

int insem_cuda_solver_point_classes(const insem_cuda_solver* h, int32_t domain, int32_t* n_tile_points,
                                    int32_t* n_halo_points) {
  return guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    const Solver& s = *h->s;
    INSEM_REQUIRE(domain >= 0 && domain < static_cast<int32_t>(s.domains.size()), INSEM_CUDA_ERR_INVALID,
                  "domain out of range");
    int32_t nt = 0, nh = 0;
    if (s.tiled) {
      nh = s.tiled_halo_points(domain);
      nt = s.domains[domain].ng - nh;
    } else {
      nh = s.domains[domain].ng;
    }
    if (n_tile_points) *n_tile_points = nt;
    if (n_halo_points) *n_halo_points = nh;
  });
}

int insem_cuda_solver_advance_streamed(insem_cuda_solver* h, int32_t n, const float* amp_in, double* rows_out,
                                       int32_t* n_rows) {
  return guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    h->s->advance_streamed(n, amp_in, rows_out, n_rows);
  });
}

int32_t insem_cuda_solver_n_columns(const insem_cuda_solver* h) { return h ? h->s->n_columns() : -1; }

int32_t insem_cuda_solver_kernels_per_step(insem_cuda_solver* h) {
  if (!h) return -1;
  if (h->s->tiled) return h->s->kernels_per_step;  // counted when the step graphs are captured
  const int rc = guarded([&] {
    DeviceGuard dg(h->s->device);
    h->s->ensure_graph();
  });
  return rc == INSEM_CUDA_OK ? h->s->kernels_per_step : -1;
}

int insem_cuda_stable_dt(const insem_cuda_problem* problem, int32_t device, double* stable_dt) {
  return guarded([&] {
    INSEM_REQUIRE(problem && stable_dt, INSEM_CUDA_ERR_INVALID, "null argument");
    insem_cuda_options o{};
    o.device = device;
    o.use_graphs = 0;
    Solver s(*problem, &o, true);
    *stable_dt = s.stable_dt();
  });
}

}  // extern "C"
