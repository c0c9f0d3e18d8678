// Batched solves: many independent solves (models, shots) of any ngll,
// geometry kind, medium and azimuthal order advance together, one step of
// every unfinished solve per batched step.
//
// A batched step is one CUDA graph of a fixed number of launches whatever
// the number of solves:
//   begin (step counters, buffer parities, modes; tile queues reset)
//   constrained-slot gathers of every solve
//   one tile launch per tile class (ngll, kind, medium, order): one CTA
//     per (segment, tile) item
//   halo points of every solve (elastic classes, then acoustic: the fluid's
//     coupling term reads the solid's new acceleration)
//   receivers (particle velocity, then recording) and energy of every solve
// Each solve keeps its own device data, time step, parity and step count,
// so its results are the ones it gets alone, bit for bit.  Solves that
// reach their last step run it in final mode and idle (every batched kernel
// skips them) until the tables are rebuilt without them: membership changes
// re-capture the graph at the next advance.
#pragma once

#include <map>
#include <memory>
#include <vector>

#include "solver.cuh"

namespace insem_b200 {

// Streamed batched steps: where each solve's amplitudes and sample columns sit
// in the per-step host rows.
struct StreamSeg {
  float* src_amp;        // [n_sources][n_amp] amplitude table of the solve
  int32_t n_amp, n_sources, amp_off;
  const double* traces;  // [max_samples][n_cols]
  int32_t n_cols, col_off, record_every, max_samples;
  const StepState* st;
};

struct TileClass {
  int ngll = 0, kind = 0, m = 0, ncomp = 0;
  bool elastic = false;
  int tp_cap = 0, nc_cap = 0, te = 0, rank_cap = 1;  // largest tile of the class
  std::vector<TileSeg> segs;
  std::vector<TileItem> items;
};

// Host-side segment tables of one batch composition.
struct BatchTables {
  std::map<int, TileClass> tiles;  // key: ((ngll * 4 + kind) * 2 + elastic) * 2 + m
  std::vector<HaloSeg> halo_segs[3];  // 1 component (acoustic), 2 and 3 components (elastic)
  std::vector<int2> halo_items[3];
  std::vector<ConsSeg> cons_segs;
  std::vector<int2> cons_items;
  std::vector<RecSeg> rec_segs;
  std::vector<int2> pv_items, rec_items;
  std::vector<EnergySeg> energy_segs;
  std::vector<StepState*> states;
  std::vector<StreamSeg> stream_segs;
  int32_t amp_cols = 0, row_cols = 0;
};

class Batch {
 public:
  explicit Batch(const insem_cuda_options* opt);
  ~Batch();
  Batch(const Batch&) = delete;
  Batch& operator=(const Batch&) = delete;

  // Builds a solve on the batch's device; returns its index.
  int32_t add(const insem_cuda_problem& p);
  // Takes ownership of an existing solve that no batch has stepped.
  int32_t adopt(insem_cuda_solver* h);
  // n batched steps; a solve with fewer steps left idles after its last one.
  void advance(int32_t n);
  // Steps until every solve is complete.
  void run();
  // n steps (fewer if every solve ends sooner) with per-step host I/O:
  // amp_in[step][amp_cols] are the active solves' source amplitudes (in index
  // order, each solve's sources in order), rows_out[step][row_cols] their
  // latest sample rows.  Returns the steps done.
  int32_t advance_streamed(int32_t n, const float* amp_in, double* rows_out);
  // Column counts of the streamed rows for the current composition.
  void stream_layout(int32_t* amp_cols, int32_t* row_cols);
  // n steps with plain launches and CUDA events around the tile launches of
  // every step: device ms of the tile launches and of the whole steps.
  void profile(int32_t n, double* tile_ms, double* step_ms);
  // Frees a solve (its index stays unused).
  void remove(int32_t index);
  insem_cuda_solver* member(int32_t index);
  int32_t size() const { return static_cast<int32_t>(members.size()); }
  int32_t active() const;
  int32_t steps_to_next_completion() const;
  int32_t max_remaining() const;  // steps until every member is complete

  insem_cuda_options opts{};
  double last_ms = 0.0;           // device time of the last advance()
  int32_t kernels_per_step = 0;   // kernel nodes of the step graph
  int64_t point_updates = 0;      // sum of points x steps of the last advance()

 private:
  void rebuild();
  void finish_steps();       // error flags of the steps just enqueued; waits for them
  void credit(int32_t k);    // host bookkeeping after k batched steps
  void enqueue(cudaEvent_t tiles_begin = nullptr, cudaEvent_t tiles_end = nullptr);

  struct DevClass {
    int ngll = 0, kind = 0, m = 0, ncomp = 1;
    bool elastic = false;
    DeviceBuffer<TileSeg> segs;
    DeviceBuffer<TileItem> items;
    int32_t n_items = 0;
    int lane = 0;
    int te = 0;
    TileLayout L{};
    int grid = 0;
  };

  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // The tile classes of a step run side by side on `n_lanes` streams (lane 0
  // is `stream`, lane k > 0 is lanes[k - 1]): no tile writes what another
  // tile reads (complete points belong to one tile, halo contributions have
  // their own places), so classes need no order among them.  The lanes fork
  // after the constrained gathers.  Elastic classes of two components go to
  // lane 0 and those of three to lane 1, and each lane then runs the halo
  // kernel of its component count, which reads only those tiles' output;
  // acoustic classes go to the least loaded lane.  The lanes join before the
  // acoustic halo kernel, whose coupling term reads the solid's new
  // acceleration.
  static constexpr int kMaxLanes = 8;
  int n_lanes = 1;
  int lane3() const { return n_lanes > 1 ? 1 : 0; }  // the lane of three-component elastic classes
  cudaStream_t lanes[kMaxLanes - 1] = {};
  cudaEvent_t fork_ev = nullptr;
  cudaEvent_t join_ev[kMaxLanes - 1] = {};
  int n_sms = 0;
  std::vector<std::unique_ptr<insem_cuda_solver>> members;  // null after remove()
  std::vector<char> prepared;
  bool dirty = true;
  cudaGraphExec_t graph = nullptr;
  // device tables of the current composition
  std::vector<DevClass> dclasses;
  DeviceBuffer<HaloSeg> dhalo_segs[3];
  DeviceBuffer<int2> dhalo_items[3];
  int32_t n_halo_items[3] = {0, 0, 0};
  DeviceBuffer<ConsSeg> dcons_segs;
  DeviceBuffer<int2> dcons_items;
  int32_t n_cons_items = 0;
  DeviceBuffer<RecSeg> drec_segs;
  DeviceBuffer<int2> dpv_items, drec_items;
  int32_t n_pv_items = 0, n_rec_items = 0;
  DeviceBuffer<EnergySeg> denergy;
  int32_t n_energy = 0;
  DeviceBuffer<StepState*> dstates;
  int32_t n_states = 0;
  DeviceBuffer<StreamSeg> dstream;
  int32_t n_stream = 0, amp_cols = 0, row_cols = 0;
  DeviceBuffer<float> amp_stage;
  DeviceBuffer<double> row_stage;
  DeviceBuffer<int32_t> derr;
  int32_t* herr = nullptr;  // pinned
  std::vector<int64_t> member_points;
};

}  // namespace insem_b200
