// Device-resident solver state (the twin of solver::Solver).
#pragma once

#include <functional>

#include <memory>
#include <random>
#include <vector>

#include "device_data.cuh"
#include "step_kernels.cuh"
#include "tiled_path.cuh"

namespace insem_b200 {

// One medium's fields and per-step arrays in HBM (solver::Domain, solver.hpp:25-66).
struct DeviceDomainData {
  int medium = 0, m = 0, ncomp = 1, ng = 0, npe = 0, n_elements = 0;
  DeviceDofMap dofs;
  std::vector<DeviceBlock> blocks;
  bool any_axial = false;
  std::vector<float> host_mass;
  DeviceBuffer<float> mass, inv_mass;
  int32_t n_abs = 0;
  DeviceBuffer<int32_t> absorbing_points;
  DeviceBuffer<float> absorbing_coef;
  std::vector<int64_t> host_zero;   // Dirichlet and axis entries (component * ng + point)
  DeviceBuffer<int64_t> zero_idx;
  DeviceBuffer<float> u, v, a, f, f_local;  // two-pass path only (alloc_fields)
  bool fields_ready = false;
  void alloc_fields(cudaStream_t s = nullptr);
  void free_fields();

  void upload(const insem_cuda_domain& d, const insem_cuda_basis& basis);
};

struct DomainSources {
  int32_t n_points = 0;
  DeviceBuffer<int32_t> points, offsets, source;
  DeviceBuffer<float> coef;
};

struct TraceInfo {
  int32_t first_col = 0;
  int32_t ncomp = 0;
};

struct BatchTables;

class Solver {
 public:
  // setup_only: dt may be 0 (the problem is used to estimate the stable time step).
  // time: dt and n_steps come from the stable time step estimated here
  // (solver.cpp:131-144) instead of from the problem.
  Solver(const insem_cuda_problem& p, const insem_cuda_options* opt, bool setup_only = false,
         const insem_cuda_time* time = nullptr);
  ~Solver();
  Solver(const Solver&) = delete;
  Solver& operator=(const Solver&) = delete;

  void set_state(int32_t medium, const double* u, const double* v);
  void advance(int32_t n);
  // Wavefield snapshots (Solver::record_snapshot, solver.cpp:813-839): every
  // `every` steps (and at step 0) the listed quantities of every medium that
  // has them, gathered to element points.  Before the first step only.
  void set_snapshots(int32_t every, int32_t n_quantities, const int32_t* quantities);
  struct SnapField {
    int32_t domain = 0, quantity = 0, ncomp = 0;
    std::vector<float> data;  // [snapshot][component][element * npe + k]
  };
  int32_t snap_every = 0;
  std::vector<SnapField> snap_fields;
  std::vector<double> snap_times;
  void advance_streamed(int32_t n, const float* amp_in, double* rows_out, int32_t* n_rows);
  void ensure_graph();
  int32_t kernels_per_step = 0;
  int32_t n_columns() const { return n_cols; }
  int32_t n_samples() const;
  int32_t n_energy() const;
  void copy_trace(int32_t t, double* out);
  void copy_state(int32_t di, double* u, double* v, double* a);
  // f = -K u for a domain: gather-fused element kernels + CSR assemble.
  void internal_forces(DeviceDomainData& d, const float* u_global, float* f_global);
  // Power iteration for lambda_max(M^-1 K) (solver.cpp:583-667); returns 2/sqrt(lambda).
  double stable_dt();
  // f = -K u of domain di on the caller's device arrays, without allocating
  // (the element-local forces use a fixed array, see noalloc.cu).
  void internal_forces_noalloc(int32_t di, const float* u_global, float* f_global, cudaStream_t s);
  // Run by the constructor on the solver's device: loads the fixed scratch
  // array and the kernels internal_forces_noalloc launches, so that under lazy
  // module loading none of them is loaded (allocated) by a later call.
  void prepare_noalloc();

  insem_cuda_options opts{};
  int device = 0;
  int ngll = 0;
  double dt = 0.0;
  double stable_dt_estimate = 0.0;  // set by the timed constructor
  int32_t n_steps = 0, step = 0, record_every = 1, energy_every = 0;
  bool initialized = false;
  std::vector<DeviceBuffer<int32_t>> snap_l2g;  // per domain: element slot -> field point, or -1 - constraint row
  DeviceBuffer<float> snap_stage;
  void record_snapshot();
  void advance_span(int32_t n);
  bool nonfinite_seen = false;  // a finite check found NaN or Inf in the fields
  double last_ms = 0.0;
  cudaStream_t stream = nullptr;
  std::vector<DeviceDomainData> domains;
  std::vector<TraceInfo> traces;
  DeviceBuffer<double> energy;  // [n_energy][3]

 private:
  void build_coupling(const insem_cuda_coupling& c);
  void build_sources(const insem_cuda_problem& p);
  void build_receivers(const insem_cuda_problem& p);
  ReceiversDev receivers_view();
  AllFields fields_view();
  void domain_acceleration(int di, int pot_set, int force_energy, double h, int step_override);
  void compute_acceleration(int force_energy, double h, int step_override);
  void observers(int force_energy, int init);
  void enqueue_step();
  void initialize();
  double reduce_partials();
  void zero_constrained(DeviceDomainData& d, float* x);
  void coupling_forces(int di);
  void coupled_lambda_max(std::mt19937& rng, double* pw);
  // Runs `body` (launches on `stream` only) n times: captured once as a CUDA
  // graph and replayed; returns after the stream has drained.
  void replay(int n, const std::function<void()>& body);

  DeviceBasis basis;
  int solid = -1, fluid = -1;
  // coupling
  int32_t n_cpl = 0;
  bool cpl_serial_fluid = false, cpl_serial_solid = false;
  DeviceBuffer<int32_t> cpl_fluid, cpl_solid;
  DeviceBuffer<float> cpl_cx, cpl_cz;
  // sources
  int32_t n_sources = 0, n_amp = 0;
  DeviceBuffer<float> src_amp;
  std::vector<DomainSources> src;
  // receivers
  int32_t n_receivers = 0, n_cols = 0, n_acoustic_rec = 0, max_samples = 0;
  DeviceBuffer<int32_t> rec_offsets, rec_points, rec_domain, rec_acoustic;
  DeviceBuffer<float> rec_value, rec_ddx, rec_ddz;
  DeviceBuffer<double> rec_rho, rec_pv, trace_buf;
  DeviceBuffer<RecordColumn> rec_cols;
  // energy
  DeviceBuffer<double> partial;
  int n_pot_sets = 0;
  // step state and graph
  StepState* st = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // Coupled models: the fluid's tile launches run on `side`, beside the
  // solid's (neither reads what the other writes), forked after the step's
  // first kernels and joined before the halo kernels.
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;

  // ------------------------------------------------------ tiled fused path
 public:
  bool tiled = false;  // the default path: tiles + halo kernel per step
 private:
  void build_tiled(const insem_cuda_problem& p);
  void enqueue_tiled(int parity, bool init);
  void tiled_begin_steps();      // predictor after a complete state
  void set_mode(int mode);
  void advance_tiled(int32_t n, const float* amp_in, double* rows_out, int32_t* n_rows);
  AllFields tiled_fields(int parity);
  std::vector<TiledDomain> tdom;
  std::vector<std::map<int32_t, std::vector<std::pair<int32_t, std::vector<float>>>>> src_per_point;
  DeviceBuffer<int32_t> tcpl_fluid, tcpl_solid, trec_points;
  DeviceBuffer<double> epart;
  int ep_tile[2] = {0, 0}, ep_halo[2] = {0, 0}, ep_ntile[2] = {0, 0}, ep_nhalo[2] = {0, 0};
  cudaGraphExec_t tgraph[2] = {nullptr, nullptr};
  int parity = 0;
  bool complete = false;  // u, v, a hold step `step` (after an init or final step)
  int cur_mode = -1;
  int32_t* mode_host = nullptr;  // pinned {normal, final, init}

  // ------------------------------------------------------ batched stepping
 public:
  bool in_batch = false;        // prepared for batched steps; advance() refuses
  const void* batch_owner = nullptr;  // the Batch that owns this solve
  int32_t remaining() const { return n_steps - step; }
  // Runs the initial step (if not yet run) and the predictor, leaving the
  // fields ready for a normal step; primes the StepState's parity and last step.
  void batch_prepare();
  // Appends this solve's segments and work items.
  void batch_collect(BatchTables& t);
  // Host bookkeeping after k batched steps.
  void batch_advanced(int32_t k);
  // NaN/Inf check of the current fields (throws INSEM_CUDA_ERR_NONFINITE).
  void check_fields();
  // Points of a domain finished by the halo kernel (the rest by their tile).
  int32_t tiled_halo_points(int di) const { return tdom[di].n_halo; }
  int32_t tiled_tile_elements(int di) const { return tdom[di].te; }
};

}  // namespace insem_b200

// Opaque handle of the C ABI.
struct insem_cuda_solver {
  std::unique_ptr<insem_b200::Solver> s;
};
