/*
 * insem_cuda.h -- C ABI of the B200 backend for insem's per-time-step path.
 *
 * The reference (nmutovkin/in-house-sem, "insem") reserves a CUDA backend
 * behind the INSEM_ENABLE_CUDA switch (CMakeLists.txt:5,18-20) but ships no
 * GPU code and no backend interface.  This header is the boundary a CUDA
 * build of the reference binds: plain structs of pointers and sizes, int
 * status codes, a thread-local error message, opaque handles.  No C++ or
 * torch types cross it.
 *
 * The entry points replace, one for one, the seams of the reference path:
 *   insem_cuda_block_*     physics::{elastic,acoustic}_internal_forces
 *                          (cpp/include/insem/physics/kernels.hpp:32-35)
 *   insem_cuda_dofmap_*    ops::DofMap::gather / ::assemble
 *                          (cpp/include/insem/ops/dof_map.hpp:73-77, 95-141)
 *   insem_cuda_solver_*    solver::Solver (cpp/include/insem/solver/solver.hpp:91-228):
 *                          advance / run / set_state / traces / energy / state
 *   insem_cuda_stable_dt   Solver::estimate_stable_dt + coupled_lambda_max
 *                          (cpp/src/solver/solver.cpp:583-667), FP64 reductions
 *   insem_cuda_solver_create_timed  Solver::Solver's stable-dt and dt / n_steps
 *                          rule (cpp/src/solver/solver.cpp:131-144)
 *   insem_cuda_batch_*     many independent solves advanced by shared launches
 *                          (the serving loop admits and retires solves through it)
 *
 * Conventions follow the reference:
 *   - real_t is float: every field, metric and coefficient array is float;
 *     constraint weights, source time functions and traces are double.
 *   - global fields are [component][global point]; element-local fields are
 *     [element][component][j * ngll + i], i along xi (r), j along eta (z)
 *     (dof_map.hpp:15-18).
 *   - indices are int32 (index_t, core/config.hpp:26).
 *   - enums keep the reference's numeric values (Medium, GeometryKind,
 *     SourceTimeFunction::Kind).
 *
 * Errors: every function returns INSEM_CUDA_OK (0) or a positive code; the
 * message of the last failure on the calling thread is returned by
 * insem_cuda_last_error().  A C++ shim rethrows it as insem::Error, so Python
 * callers of the reference bindings still see InsemError.
 *
 * Threading: handles are independent; one handle is used by one thread at a
 * time (the reference drives a Solver from one thread, bindings.cpp:336-337).
 *
 * Streams: a `stream` argument of NULL means the calling thread's default
 * stream (the library is built with per-thread default streams), which CUDA
 * keeps ordered with the legacy default stream in both directions.
 */
#ifndef INSEM_CUDA_H
#define INSEM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define INSEM_CUDA_OK 0
#define INSEM_CUDA_ERR_INVALID 1     /* invalid argument or inconsistent problem  */
#define INSEM_CUDA_ERR_UNSUPPORTED 2 /* no kernel for this ngll / kind / order     */
#define INSEM_CUDA_ERR_CUDA 3        /* CUDA runtime error                         */
#define INSEM_CUDA_ERR_STATE 4       /* call not allowed in the handle's state     */
#define INSEM_CUDA_ERR_NOMEM 5       /* device memory budget exceeded              */
#define INSEM_CUDA_ERR_NONFINITE 6   /* a solve produced NaN or Inf                */
#define INSEM_CUDA_ERR_TIMEOUT 7     /* a bounded device-side wait gave up         */

/* Message of the last failed call on this thread ("" if none). */
const char* insem_cuda_last_error(void);
/* Library version string. */
const char* insem_cuda_version(void);
/* Free and total device memory (bytes) of a device: the serving loop's HBM admission. */
int insem_cuda_mem_info(int32_t device, int64_t* free_bytes, int64_t* total_bytes);

/* ------------------------------------------------------------------- enums */
enum insem_cuda_medium { INSEM_ACOUSTIC = 0, INSEM_ELASTIC = 1 }; /* description.hpp:17 */
enum insem_cuda_kind {                                            /* geometry.hpp:17-22 */
  INSEM_RECT = 0,
  INSEM_AFFINE = 1,
  INSEM_CURVED = 2,
  INSEM_AXISYM = 3
};
enum insem_cuda_stf_kind { /* description.hpp, SourceTimeFunction::Kind */
  INSEM_STF_RICKER = 0,
  INSEM_STF_GAUSSIAN = 1,
  INSEM_STF_GAUSSIAN_DERIVATIVE = 2,
  INSEM_STF_SAMPLES = 3
};
enum insem_cuda_quantity { /* recorded quantities, description.hpp Receiver */
  INSEM_Q_DISPLACEMENT = 0,
  INSEM_Q_VELOCITY = 1,
  INSEM_Q_ACCELERATION = 2,
  INSEM_Q_PRESSURE = 3,
  INSEM_Q_PARTICLE_VELOCITY = 4
};

/* ----------------------------------------------------------- descriptions */
/* 1D basis data of the element kernels (physics::KernelBasis, kernels.hpp:12-21). */
typedef struct insem_cuda_basis {
  int32_t ngll;     /* GLL points per direction, 2..9 */
  const float* D;   /* [ngll*ngll] D[i*ngll+l] = l_l'(x_i) */
  const float* Dj;  /* [ngll*ngll] derivative matrix on the GLJ(0,1) points; NULL without axial elements */
  const float* w2;  /* [ngll*ngll] w2[j*ngll+i] = w_i w_j */
} insem_cuda_basis;

/* One element block (ops::ElementBlock, element_block.hpp:31-46). */
typedef struct insem_cuda_block {
  int32_t kind;             /* insem_cuda_kind */
  int32_t azimuthal_order;  /* 0 or 1 (1 only with INSEM_AXISYM) */
  int32_t n_elements;       /* elements in the block */
  const int32_t* elements;  /* [n_elements] domain-local element index */
  const float* metric;      /* Rect 3/elem, Affine 5/elem, Curved/Axisym 5/point (xi_x, xi_z, eta_x, eta_z, jac) */
  const float* coef0;       /* [n_elements*npe] lambda (elastic) or 1/rho (acoustic) */
  const float* coef1;       /* [n_elements*npe] mu (elastic); unused (may be NULL) for acoustic */
  const float* wr;          /* Axisym: [n_elements*npe] weight x J x r */
  const float* hoop;        /* Axisym: [n_elements*npe] wr / r */
  const float* r;           /* Axisym: [n_elements*npe] radius, exactly 0 on the axis */
  const uint8_t* axial;     /* Axisym: [n_elements] 1 if the xi = -1 face is on the axis */
} insem_cuda_block;

/* Local/global numbering with hanging-node constraints (ops::DofMap, dof_map.hpp:30-92). */
typedef struct insem_cuda_dofmap {
  int32_t ngll;
  int32_t n_elements;
  int32_t n_global;
  const int32_t* l2g;          /* [n_elements*npe] global index, or -1-r for constraint row r */
  int32_t n_rows;              /* constraint rows */
  const int32_t* row_offsets;  /* [n_rows+1] */
  const int32_t* row_dofs;     /* [row_offsets[n_rows]] */
  const double* row_weights;   /* [row_offsets[n_rows]] */
  const int32_t* t_offsets;    /* [n_global+1] transpose CSR, contributions in ascending slot order */
  const int32_t* t_slots;      /* [t_offsets[n_global]] slot = element*npe + k */
  const double* t_weights;     /* [t_offsets[n_global]] or NULL when n_rows == 0 (all weights 1) */
} insem_cuda_dofmap;

/* One medium's domain (solver::Domain, solver.hpp:25-66). */
typedef struct insem_cuda_domain {
  int32_t medium;               /* insem_cuda_medium */
  int32_t ncomp;                /* 1 acoustic, 2 elastic (m=0), 3 elastic (m=1) */
  int32_t azimuthal_order;
  insem_cuda_dofmap dofs;
  int32_t n_blocks;
  const insem_cuda_block* blocks;
  const float* mass;            /* [n_global] lumped mass */
  const float* inv_mass;        /* [n_global] (real_t)(1 / mass) */
  int32_t n_absorbing;          /* Stacey points */
  const int32_t* absorbing_points;
  const float* absorbing_coef;  /* [n_absorbing*ncomp*ncomp] row-major damping matrices */
  int32_t n_dirichlet;
  const int32_t* dirichlet_points;
  int32_t n_axis;
  const int32_t* axis_points;
  int32_t n_axis_components;
  const int32_t* axis_components;
} insem_cuda_domain;

/* Fluid-solid interface (Solver::coupling_, solver.hpp:208-211). */
typedef struct insem_cuda_coupling {
  int32_t n;
  const int32_t* fluid_points;
  const int32_t* solid_points;
  const float* cx;
  const float* cz;
} insem_cuda_coupling;

/* Source time function (SourceTimeFunction, description.hpp). */
typedef struct insem_cuda_stf {
  int32_t kind;         /* insem_cuda_stf_kind */
  double f0, t0, amplitude;
  int32_t n_samples;    /* INSEM_STF_SAMPLES only */
  const double* samples;
  double sample_dt;
} insem_cuda_stf;

/* Point source expanded onto global points (Solver::SourceTerm, solver.hpp:155-160). */
typedef struct insem_cuda_source {
  int32_t domain;       /* index into problem.domains */
  int32_t n_points;
  const int32_t* points;
  const float* coef;    /* [ncomp][n_points] */
  insem_cuda_stf stf;
} insem_cuda_source;

/* Receiver interpolation weights (Solver::ReceiverTerm, solver.hpp:161-172). */
typedef struct insem_cuda_receiver {
  int32_t domain;
  int32_t n_points;
  const int32_t* points;
  const float* value;   /* [n_points] */
  const float* d_dx;    /* [n_points] */
  const float* d_dz;    /* [n_points] */
  double rho;
  int32_t n_quantities;
  const int32_t* quantities; /* insem_cuda_quantity; one trace per quantity, in order */
} insem_cuda_receiver;

/* Everything the time loop reads (what Solver(Problem) builds, solver.cpp:91-145). */
typedef struct insem_cuda_problem {
  insem_cuda_basis basis;
  int32_t n_domains;    /* domains in the reference's order (acoustic first) */
  const insem_cuda_domain* domains;
  insem_cuda_coupling coupling;
  int32_t n_sources;
  const insem_cuda_source* sources;
  int32_t n_receivers;
  const insem_cuda_receiver* receivers;
  double dt;            /* time step in use (Solver::dt) */
  int32_t n_steps;
  int32_t record_every; /* >= 1 */
  int32_t energy_every; /* 0 = off */
} insem_cuda_problem;

/* Options of a solver handle (0-initialised = defaults). */
typedef struct insem_cuda_options {
  int32_t device;          /* CUDA device ordinal */
  int32_t use_graphs;      /* 1: capture the step loop in CUDA graphs (default 1; 0 = plain launches) */
  int32_t path;            /* 0 default; 1 plain two-pass (element forces -> CSR assemble); 2 tiled fused */
  int32_t tile_elements;   /* tiled path: elements per tile (0 = autotuned) */
  int32_t check_finite;    /* 1: check fields for NaN/Inf at every advance() end (default 1) */
  int32_t tile_streams;    /* batches: streams the tile launches of a step spread over (0 = default 2, at most 8) */
} insem_cuda_options;

/* ------------------------------------------------- per-block kernel seam */
typedef struct insem_cuda_block_h insem_cuda_block_h;

/* Uploads one block (and its basis).  `medium` selects the elastic or the
 * acoustic operator; ncomp follows from medium and azimuthal order.
 * Unsupported ngll / kind / order return INSEM_CUDA_ERR_UNSUPPORTED like
 * physics::select (kernels.cpp:451-468). */
int insem_cuda_block_create(const insem_cuda_basis* basis, const insem_cuda_block* block, int32_t medium,
                            int32_t device, insem_cuda_block_h** out);
void insem_cuda_block_destroy(insem_cuda_block_h* h);
/* f_local = -K u_local on the block's elements (device pointers, element-local
 * layout of the whole domain, n_local_elements elements); only the block's
 * elements of f_local are written.  Asynchronous on `stream` (cudaStream_t or
 * NULL). Bitwise equal to the reference CPU build (no FMA contraction). */
int insem_cuda_block_forces(insem_cuda_block_h* h, int32_t n_local_elements, const float* u_local,
                            float* f_local, void* stream);
/* Same with host pointers, synchronous: the reference's per-block call as is. */
int insem_cuda_block_forces_host(insem_cuda_block_h* h, int32_t n_local_elements, const float* u_local,
                                 float* f_local);

/* ---------------------------------------------------- gather / assemble */
typedef struct insem_cuda_dofmap_h insem_cuda_dofmap_h;
int insem_cuda_dofmap_create(const insem_cuda_dofmap* dofs, int32_t device, insem_cuda_dofmap_h** out);
void insem_cuda_dofmap_destroy(insem_cuda_dofmap_h* h);
/* local = C global (DofMap::gather); device pointers, asynchronous on stream. */
int insem_cuda_gather(insem_cuda_dofmap_h* h, int32_t ncomp, const float* global, float* local, void* stream);
/* global = C^T local (DofMap::assemble): every global point written once, its
 * contributions summed in ascending slot order, as the reference. */
int insem_cuda_assemble(insem_cuda_dofmap_h* h, int32_t ncomp, const float* local, float* global, void* stream);

/* --------------------------------------------------------------- solver */
typedef struct insem_cuda_solver insem_cuda_solver;

/* Uploads a problem; fields start at zero.  `options` may be NULL. */
int insem_cuda_solver_create(const insem_cuda_problem* problem, const insem_cuda_options* options,
                             insem_cuda_solver** out);

/* Time settings (TimeConfig, cpp/include/insem/sim/description.hpp:128-135). */
typedef struct insem_cuda_time {
  double dt;        /* > 0: this step (it must not exceed the stability limit); 0: safety x stable dt */
  double safety;    /* share of the stability limit used when dt = 0, in (0, 1] */
  int32_t n_steps;  /* > 0: this many steps; 0: ceil(duration / dt - 1e-9) */
  double duration;  /* simulated seconds, used when n_steps = 0 */
} insem_cuda_time;

/* The reference Solver constructor's time handling (solver.cpp:131-144): the
 * problem's dt and n_steps are ignored; the solver estimates the stable time
 * step on the device from the arrays it has just uploaded (as
 * insem_cuda_stable_dt does) and derives dt and n_steps from `time`.  Same
 * result as insem_cuda_stable_dt followed by insem_cuda_solver_create with
 * the derived dt and n_steps, with one upload of the problem instead of two.
 * A dt above the stability limit or a safety outside (0, 1] is
 * INSEM_CUDA_ERR_INVALID, as in the reference. */
int insem_cuda_solver_create_timed(const insem_cuda_problem* problem, const insem_cuda_time* time,
                                   const insem_cuda_options* options, insem_cuda_solver** out);
/* The stable time step estimated by insem_cuda_solver_create_timed (0 for a
 * solver made by insem_cuda_solver_create). */
double insem_cuda_solver_stable_dt(const insem_cuda_solver* h);
void insem_cuda_solver_destroy(insem_cuda_solver* h);
/* Initial conditions of one medium ([ncomp][n_global], host doubles), before
 * the first step only (Solver::set_state, solver.cpp:764-778). */
int insem_cuda_solver_set_state(insem_cuda_solver* h, int32_t medium, const double* u, const double* v);
/* Advances n steps or up to n_steps (Solver::advance, solver.cpp:917-963). */
int insem_cuda_solver_advance(insem_cuda_solver* h, int32_t n);
/* Advances to the end (Solver::run). */
int insem_cuda_solver_run(insem_cuda_solver* h);
int32_t insem_cuda_solver_step(const insem_cuda_solver* h);
/* INSEM_CUDA_ERR_NONFINITE once a finite check of this solve (the end of an
 * advance, or a batch member's last step) found NaN or Inf in its fields,
 * else INSEM_CUDA_OK.  A batch advance that fails this way names the members
 * in its message; this tells a server which of them to evict.  No reference
 * counterpart (the reference raises from Solver::advance). */
int32_t insem_cuda_solver_status(const insem_cuda_solver* h);
int32_t insem_cuda_solver_n_steps(const insem_cuda_solver* h);
double insem_cuda_solver_dt(const insem_cuda_solver* h);
/* Number of recorded samples so far, traces and their component counts. */
int32_t insem_cuda_solver_n_samples(const insem_cuda_solver* h);
int32_t insem_cuda_solver_n_traces(const insem_cuda_solver* h);
int32_t insem_cuda_solver_trace_ncomp(const insem_cuda_solver* h, int32_t trace);
/* Copies trace `trace` ([n_samples][ncomp] doubles) to host memory. */
int insem_cuda_solver_trace(insem_cuda_solver* h, int32_t trace, double* out);
/* Sample times ([n_samples] doubles). */
int insem_cuda_solver_times(insem_cuda_solver* h, double* out);
/* Energy samples ([n][3]: time, kinetic, potential); *n_out receives n. */
int insem_cuda_solver_energy(insem_cuda_solver* h, double* out, int32_t capacity, int32_t* n_out);
/* Wavefield snapshots (Solver::record_snapshot, cpp/src/solver/solver.cpp:813-839;
 * TimeConfig::snapshot_every / snapshot_quantities).  Set before the first
 * step: every `every` steps, and at step 0, advance() records each of the
 * `quantities` (insem_cuda_quantity: displacement, velocity, acceleration,
 * pressure) of every medium that has it -- per quantity, media in domain
 * order -- gathered to element points ([component][element][ngll^2], hanging
 * points interpolated, azimuthal order 1 elastic as (U_r, U_theta, U_z)).
 * every = 0 turns snapshots off.  Solves with snapshots step on their own
 * (not streamed, not in a batch). */
int insem_cuda_solver_set_snapshots(insem_cuda_solver* h, int32_t every, int32_t n_quantities,
                                    const int32_t* quantities);
int32_t insem_cuda_solver_n_snapshots(const insem_cuda_solver* h);        /* snapshots taken so far */
int32_t insem_cuda_solver_n_snapshot_fields(const insem_cuda_solver* h);  /* recorded (medium, quantity) pairs */
/* Medium, quantity, components and element points (elements x ngll^2) of a recorded field. */
int insem_cuda_solver_snapshot_field(const insem_cuda_solver* h, int32_t field, int32_t* medium, int32_t* quantity,
                                     int32_t* ncomp, int64_t* n_points);
/* A field's snapshots: [n_snapshots][ncomp][n_points] floats. */
int insem_cuda_solver_snapshot(const insem_cuda_solver* h, int32_t field, float* out);
/* Times of the snapshots taken ([n_snapshots] doubles: step x dt). */
int insem_cuda_solver_snapshot_times(const insem_cuda_solver* h, double* out);
/* Current u, v, a of domain `domain` ([ncomp][n_global] host doubles; any may be NULL). */
int insem_cuda_solver_state(insem_cuda_solver* h, int32_t domain, double* u, double* v, double* a);
/* Device time of the last advance() call in milliseconds (CUDA events). */
double insem_cuda_solver_last_advance_ms(const insem_cuda_solver* h);
/* Internal forces f = -K u of a domain for a host field (Solver::internal_forces). */
int insem_cuda_solver_internal_forces(insem_cuda_solver* h, int32_t domain, const float* u, float* f);
/* Streamed advance: n steps where every step first copies that step's source
 * amplitudes amp_in[s * n_sources + k] (host, pinned for best speed) to the
 * device and, on record steps, copies the recorded sample row back to
 * rows_out[r * n_columns ...] (host); *n_rows receives the rows written.
 * Amplitudes given here replace the ones computed from the source time
 * functions for those steps.  One synchronisation at the end. */
int insem_cuda_solver_advance_streamed(insem_cuda_solver* h, int32_t n, const float* amp_in, double* rows_out,
                                       int32_t* n_rows);
/* Columns of a recorded sample row (all traces side by side, in trace order). */
int32_t insem_cuda_solver_n_columns(const insem_cuda_solver* h);
/* Kernel launches of one captured step (the step graph's kernel nodes). */
int32_t insem_cuda_solver_kernels_per_step(insem_cuda_solver* h);
/* Elements per tile (one CTA) of the tiled path.  A solver takes
 * options.tile_elements when > 0, else the entry set here for its domain's
 * class (ngll, dominant geometry kind, medium, azimuthal order), else an
 * occupancy-based default.  The autotuner (insem_b200.autotune) times
 * candidates and sets the entries; tile_elements <= 0 clears one.  Applies to
 * solvers created afterwards; process-wide. */
int insem_cuda_set_tile_elements(int32_t ngll, int32_t kind, int32_t medium, int32_t azimuthal_order,
                                 int32_t tile_elements);
/* The choice a new solver would make for that class (ncomp: field components). */
int32_t insem_cuda_tile_elements(int32_t ngll, int32_t kind, int32_t medium, int32_t azimuthal_order, int32_t ncomp);
/* Elements per tile a solver's domain was built with (0 on the two-pass path). */
int32_t insem_cuda_solver_tile_elements(const insem_cuda_solver* h, int32_t domain);
/* Internal forces f = -K u of one domain, like insem_cuda_solver_internal_forces,
 * for callers that cannot have the library allocate device memory: u and f
 * are device arrays the caller owns ([ncomp][n_global], the reference's
 * numbering), the work is enqueued on `stream` (a cudaStream_t; NULL is the
 * legacy default stream) and the call returns without waiting for it.  No
 * counterpart in the reference: it adds an allocation-free form of the
 * internal_forces seam (solver.cpp:570-581).
 *   - Nothing is allocated or freed: the element-local force vectors go to a
 *     fixed 16 MiB device array inside the library (4,194,304 floats).  A
 *     domain needing more (ncomp x elements x ngll^2 floats) is rejected with
 *     INSEM_CUDA_ERR_UNSUPPORTED before anything is enqueued.
 *   - Under lazy module loading (the CUDA default) the driver reserves a
 *     module's device memory when the module is first used.  Creating a
 *     solver (insem_cuda_solver_create*) therefore loads the array and the
 *     kernels this entry point runs, on the solver's device: the 16 MiB are
 *     reserved then and held until the process exits, and calls here load
 *     nothing.  Create the solver while device memory is still free.
 *   - Each call looks up the array's device address on the current device
 *     (a host-side lookup, nothing cached).
 *   - All calls share the array: calls whose work overlaps on the GPU (other
 *     streams, other threads, other handles) race on it.  Each call clears
 *     the part it uses before use. */
int insem_cuda_solver_internal_forces_noalloc(insem_cuda_solver* h, int32_t domain, const float* u, float* f,
                                              void* stream);
/* Points of a domain finished inside their tile's kernel and by the halo
 * kernel (the roofline's split of the step's bytes). */
int insem_cuda_solver_point_classes(const insem_cuda_solver* h, int32_t domain, int32_t* n_tile_points,
                                    int32_t* n_halo_points);

/* ------------------------------------------------------------ stable dt */
/* Power iteration for lambda_max(M^-1 K) with the reference's seeds and
 * iteration counts, FP64 reductions on the device; returns 2/sqrt(lambda). */
int insem_cuda_stable_dt(const insem_cuda_problem* problem, int32_t device, double* stable_dt);

/* ---------------------------------------------------------- batched solves */
/* Many independent solves (models, shots) of any ngll, geometry kind, medium
 * and azimuthal order, advanced together: every batched step is one CUDA
 * graph of a fixed number of launches (one tile launch per tile class, its
 * CTAs fed by a device work queue, then the point-wise kernels of all
 * solves).  Each solve keeps its own time step and step count and gets the
 * results it gets alone, bit for bit.  The reference has no batch API; its
 * nearest form is one Simulation per thread (bindings.cpp:336-337).
 * Members are insem_cuda_solver handles owned by the batch: read them with
 * the insem_cuda_solver_* accessors (set_state before the first batched
 * step), never destroy them and never advance them directly. */
typedef struct insem_cuda_batch insem_cuda_batch;
int insem_cuda_batch_create(const insem_cuda_options* options, insem_cuda_batch** out);
void insem_cuda_batch_destroy(insem_cuda_batch* h);
/* Builds a solve (device upload) and appends it; *index (may be NULL) is its index. */
int insem_cuda_batch_add(insem_cuda_batch* h, const insem_cuda_problem* problem, int32_t* index);
/* Runs what joining a batch needs (the initial step and the predictor) now,
 * on the solver's own stream, so that a later add to a batch costs nothing on
 * the batch's stream.  Afterwards only a batch steps the solver. */
int insem_cuda_solver_prepare_for_batch(insem_cuda_solver* h);
/* Takes ownership of a solver handle that no batch owns (prepared or not). */
int insem_cuda_batch_adopt(insem_cuda_batch* h, insem_cuda_solver* solver, int32_t* index);
/* n batched steps (fewer if every member ends sooner); a member with fewer
 * steps left runs its last step in final mode and then idles: the batch's
 * kernels skip it until the next composition leaves it out. */
int insem_cuda_batch_advance(insem_cuda_batch* h, int32_t n);
/* Steps until every member is complete. */
int insem_cuda_batch_run(insem_cuda_batch* h);
/* Frees a member (indices of the others are unchanged). */
int insem_cuda_batch_remove(insem_cuda_batch* h, int32_t index);
/* Borrowed handle of member `index` (NULL and an error message if there is none). */
insem_cuda_solver* insem_cuda_batch_member(insem_cuda_batch* h, int32_t index);
/* Streamed batched steps (end-to-end serving form): n steps (fewer if every
 * member ends sooner); *n_done is the number done.  A member with r < n steps
 * left has valid rows for its first r steps.  Per step it takes
 * amp_in[step][amp_cols], the source amplitudes of the members running at
 * the call
 * (index order, each member's sources in order, FP32 as the reference casts
 * them), and writes rows_out[step][row_cols], each active member's latest
 * sample row (its columns as insem_cuda_solver_n_columns lays them out); one
 * host-to-device and one device-to-host copy per step.  amp_in NULL: the
 * solves' own source time functions (resident tables); rows_out may be NULL. */
int insem_cuda_batch_advance_streamed(insem_cuda_batch* h, int32_t n, const float* amp_in, double* rows_out,
                                      int32_t* n_done);
/* n steps with plain launches and CUDA events around each step's tile
 * launches (as insem_cuda_batch_advance): device ms of the tile launches
 * and of the whole steps. */
int insem_cuda_batch_profile(insem_cuda_batch* h, int32_t n, double* tile_ms, double* step_ms);
/* amp_cols and row_cols of the members running now (0 when none is). */
int insem_cuda_batch_stream_layout(insem_cuda_batch* h, int32_t* amp_cols, int32_t* row_cols);
int32_t insem_cuda_batch_size(const insem_cuda_batch* h);
int32_t insem_cuda_batch_active(const insem_cuda_batch* h);
/* Steps until the next member completes, and until all are (0 when none is running). */
int32_t insem_cuda_batch_steps_to_next_completion(const insem_cuda_batch* h);
int32_t insem_cuda_batch_steps_to_completion(const insem_cuda_batch* h);
/* Device time of the last advance / run segment, ms; points x steps it did. */
double insem_cuda_batch_last_advance_ms(const insem_cuda_batch* h);
int64_t insem_cuda_batch_point_updates(const insem_cuda_batch* h);
/* Kernel nodes of the current batched-step graph. */
int32_t insem_cuda_batch_kernels_per_step(const insem_cuda_batch* h);

#ifdef __cplusplus
}
#endif

#endif /* INSEM_CUDA_H */
