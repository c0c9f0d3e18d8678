// Batched solves (see batch.cuh) and the Solver hooks they use.
#include <algorithm>
#include <cstddef>

#include "batch.cuh"

namespace insem_b200 {

// Error flags of every batched solve into out[0] (bounded-wait timeouts).
static __global__ void batch_error_kernel(StepState* const* __restrict__ sts, int32_t n, int32_t* __restrict__ out) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && sts[i]->error) atomicOr(out, 1);
}

// Streamed steps: this step's amplitudes from the staged host row into each
// solve's amplitude table (the step about to run is st->step + 1).
static __global__ void batch_amp_scatter_kernel(const StreamSeg* __restrict__ segs, const float* __restrict__ stage) {
  const StreamSeg& sg = segs[blockIdx.x];
  const int32_t s = sg.st->step + 1;
  if (s >= sg.n_amp) return;
  for (int32_t q = threadIdx.x; q < sg.n_sources; q += blockDim.x)
    sg.src_amp[static_cast<size_t>(q) * sg.n_amp + s] = stage[sg.amp_off + q];
}

// Streamed steps: each solve's latest sample row into the staged host row.
static __global__ void batch_row_gather_kernel(const StreamSeg* __restrict__ segs, double* __restrict__ stage) {
  const StreamSeg& sg = segs[blockIdx.x];
  const int32_t sample = sg.st->step / sg.record_every;
  for (int32_t c = threadIdx.x; c < sg.n_cols; c += blockDim.x)
    stage[sg.col_off + c] = sample < sg.max_samples ? sg.traces[static_cast<size_t>(sample) * sg.n_cols + c] : 0.0;
}

// ------------------------------------------------------------ Solver hooks
void Solver::batch_prepare() {
  DeviceGuard dg(device);
  INSEM_REQUIRE(tiled, INSEM_CUDA_ERR_STATE, "batched solves run on the tiled path");
  INSEM_REQUIRE(snap_every <= 0, INSEM_CUDA_ERR_STATE, "a solve that records snapshots is stepped on its own");
  if (in_batch) return;  // prepared already
  if (!initialized) {
    set_mode(kModeInit);
    enqueue_tiled(parity, true);
    parity ^= 1;
    complete = true;
    initialized = true;
  }
  tiled_begin_steps();
  // the begin kernel flips the parity before each step; the first batched
  // step must use the host's current parity
  const int32_t vals[2] = {parity ^ 1, n_steps};
  static_assert(offsetof(StepState, last_step) == offsetof(StepState, parity) + sizeof(int32_t), "StepState layout");
  CUDA_CHECK(cudaMemcpyAsync(&st->parity, vals, sizeof(vals), cudaMemcpyHostToDevice, stream));
  CUDA_CHECK(cudaStreamSynchronize(stream));
  cur_mode = -1;
  in_batch = true;
}

void Solver::batch_collect(BatchTables& T) {
  T.states.push_back(st);
  T.stream_segs.push_back(StreamSeg{src_amp.get(), n_amp, n_sources, T.amp_cols, trace_buf.get(), n_cols, T.row_cols,
                                    record_every, max_samples, st});
  T.amp_cols += n_sources;
  T.row_cols += n_cols;
  const StepScalars sc{static_cast<float>(dt), static_cast<float>(0.5 * dt), static_cast<float>(0.5 * dt * dt),
                       energy_every};
  for (auto& t : tdom) {
    if (t.n_cslots <= 0) continue;
    const int32_t seg = static_cast<int32_t>(T.cons_segs.size());
    T.cons_segs.push_back(ConsSeg{t.n_cslots, t.cs_row.get(), t.rows(), t.u0.get(), t.u1.get(), t.ng, t.ncomp,
                                  t.cval.get(), st});
    for (int k = 0; k < ceil_div(t.n_cslots, kConsChunk); ++k) T.cons_items.push_back(int2{seg, k});
  }
  for (int di : {solid, fluid}) {
    if (di < 0) continue;
    TiledDomain& t = tdom[di];
    const bool el = t.medium == INSEM_ELASTIC;
    for (const auto& bt : t.blocks) {
      if (bt.ntiles == 0) continue;
      TileSeg sg{};
      sg.blk = bt.view();
      sg.td = t.view(0);
      sg.td.sdesc += static_cast<size_t>(bt.e_off) * point_stride_rt(ngll * ngll);
      sg.sc = sc;
      sg.st = st;
      sg.epartial = epart.get() + 2 * static_cast<std::size_t>(ep_tile[di]);
      const int m = bt.kind == INSEM_AXISYM ? bt.m : 0;
      const int key = ((ngll * 4 + bt.kind) * 2 + (el ? 1 : 0)) * 2 + m;
      TileClass& c = T.tiles[key];
      c.ngll = ngll;
      c.kind = bt.kind;
      c.m = m;
      c.ncomp = t.ncomp;
      c.elastic = el;
      c.te = std::max(c.te, t.te);
      c.tp_cap = std::max(c.tp_cap, t.tp_cap);
      c.nc_cap = std::max(c.nc_cap, t.nc_cap);
      c.rank_cap = std::max(c.rank_cap, t.rank_cap);
      const int32_t seg = static_cast<int32_t>(c.segs.size());
      c.segs.push_back(sg);
      for (int k = 0; k < bt.ntiles; ++k) {
        TileItem it{};
        it.th = t.host_tiles[bt.tile0 + k];
        it.halo_tp = sg.td.halo_tp + it.th.hl_off;
        it.st = st;
        it.seg = seg;
        it.tile = bt.tile0 + k;
        c.items.push_back(it);
      }
    }
  }
  CouplingDev cp{tcpl_fluid.get(), tcpl_solid.get(), cpl_cx.get(), cpl_cz.get()};
  for (int di : {solid, fluid}) {
    if (di < 0) continue;
    TiledDomain& t = tdom[di];
    if (t.n_halo == 0) continue;
    const bool el = t.medium == INSEM_ELASTIC;
    HaloSeg h{};
    h.td = t.view(0);
    h.hd = t.halo_view();
    h.cp = cp;
    if (n_cpl > 0) {
      if (el) {
        h.other0 = tdom[fluid].u0.get();
        h.other1 = tdom[fluid].u1.get();
        h.other_ng = tdom[fluid].ng;
        h.pm = t.m == 1;
      } else {
        h.other0 = h.other1 = tdom[solid].a.get();
        h.other_ng = tdom[solid].ng;
        h.pm = tdom[solid].m == 1;
      }
    }
    h.amp = src_amp.get();
    h.n_amp = n_amp;
    h.sc = sc;
    h.h_damp = 0.5 * dt;
    h.st = st;
    h.epartial = epart.get();
    h.epart0 = ep_halo[di];
    const int cls = !el ? 0 : (t.ncomp == 2 ? 1 : 2);
    const int32_t seg = static_cast<int32_t>(T.halo_segs[cls].size());
    T.halo_segs[cls].push_back(h);
    for (int k = 0; k < ceil_div(t.n_halo, kHaloChunk); ++k) T.halo_items[cls].push_back(int2{seg, k});
  }
  if (n_acoustic_rec > 0 || n_cols > 0) {
    RecSeg r{};
    r.rv = receivers_view();
    r.rv.points = trec_points.get();
    r.f0 = tiled_fields(0);
    r.f1 = tiled_fields(1);
    r.acoustic_recv = rec_acoustic.get();
    r.n_acoustic = n_acoustic_rec;
    r.dt = dt;
    r.cols = rec_cols.get();
    r.n_cols = n_cols;
    r.st = st;
    r.record_every = record_every;
    r.traces = trace_buf.get();
    r.max_samples = max_samples;
    const int32_t seg = static_cast<int32_t>(T.rec_segs.size());
    T.rec_segs.push_back(r);
    for (int k = 0; k < ceil_div(n_acoustic_rec, kRecChunk); ++k) T.pv_items.push_back(int2{seg, k});
    for (int k = 0; k < ceil_div(n_cols, kRecChunk); ++k) T.rec_items.push_back(int2{seg, k});
  }
  if (energy_every > 0) {
    const int d0 = solid >= 0 ? solid : fluid;
    const int d1 = solid >= 0 ? fluid : -1;
    EnergySeg e{};
    e.epartial = epart.get();
    e.n_dom = d1 >= 0 ? 2 : 1;
    e.s0 = int4{ep_tile[d0], ep_ntile[d0], ep_halo[d0], tdom[d0].n_halo > 0 ? ep_nhalo[d0] : 0};
    if (d1 >= 0) e.s1 = int4{ep_tile[d1], ep_ntile[d1], ep_halo[d1], tdom[d1].n_halo > 0 ? ep_nhalo[d1] : 0};
    e.st = st;
    e.energy_every = energy_every;
    e.dt = dt;
    e.energy = energy.get();
    e.max_samples = static_cast<int32_t>(energy.size() / 3);
    T.energy_segs.push_back(e);
  }
}

void Solver::batch_advanced(int32_t k) {
  step += k;
  if (k & 1) parity ^= 1;
  complete = step == n_steps;  // the last step ran in final mode
  cur_mode = -1;
}

void Solver::check_fields() {
  DeviceGuard dg(device);
  for (auto& t : tdom) {
    const int64_t nn = static_cast<int64_t>(t.ncomp) * t.ng;
    finite_check_kernel<<<grid_for(nn), 256, 0, stream>>>(t.u_cur(parity), nn, st);
    CUDA_LAUNCH_CHECK();
  }
  StepState hs;
  CUDA_CHECK(cudaMemcpyAsync(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost, stream));
  CUDA_CHECK(cudaStreamSynchronize(stream));
  if (hs.nonfinite) nonfinite_seen = true;
  INSEM_REQUIRE(!hs.nonfinite, INSEM_CUDA_ERR_NONFINITE, "the solution contains NaN or Inf (unstable time step?)");
}

// ------------------------------------------------------------------ Batch
Batch::Batch(const insem_cuda_options* opt) {
  if (opt) opts = *opt;
  else {
    opts = insem_cuda_options{};
    opts.use_graphs = 1;
    opts.check_finite = 1;
  }
  INSEM_REQUIRE(opts.path != 1, INSEM_CUDA_ERR_INVALID, "batched solves run on the tiled path");
  DeviceGuard dg(opts.device);
  CUDA_CHECK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  CUDA_CHECK(cudaEventCreate(&ev0));
  CUDA_CHECK(cudaEventCreate(&ev1));
  INSEM_REQUIRE(opts.tile_streams >= 0 && opts.tile_streams <= kMaxLanes, INSEM_CUDA_ERR_INVALID,
                "tile_streams must be 0..8");
  n_lanes = opts.tile_streams > 0 ? opts.tile_streams : 2;
  CUDA_CHECK(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
  for (int k = 0; k + 1 < n_lanes; ++k) {
    CUDA_CHECK(cudaStreamCreateWithFlags(&lanes[k], cudaStreamNonBlocking));
    CUDA_CHECK(cudaEventCreateWithFlags(&join_ev[k], cudaEventDisableTiming));
  }
  CUDA_CHECK(cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, opts.device));
  CUDA_CHECK(cudaMallocHost(&herr, sizeof(int32_t)));
  derr.resize(1);
}

Batch::~Batch() {
  DeviceGuard dg(opts.device);
  // members' buffers are released below: both streams must be done with them
  if (stream) cudaStreamSynchronize(stream);
  for (cudaStream_t l : lanes)
    if (l) cudaStreamSynchronize(l);
  if (graph) cudaGraphExecDestroy(graph);
  members.clear();
  if (herr) cudaFreeHost(herr);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (fork_ev) cudaEventDestroy(fork_ev);
  for (cudaEvent_t e : join_ev)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t l : lanes)
    if (l) cudaStreamDestroy(l);
  if (stream) cudaStreamDestroy(stream);
}

int32_t Batch::add(const insem_cuda_problem& p) {
  DeviceGuard dg(opts.device);
  auto h = std::make_unique<insem_cuda_solver>();
  h->s = std::make_unique<Solver>(p, &opts);
  const int32_t i = adopt(h.get());
  h.release();
  return i;
}

int32_t Batch::adopt(insem_cuda_solver* h) {
  INSEM_REQUIRE(h && h->s, INSEM_CUDA_ERR_INVALID, "null solve");
  INSEM_REQUIRE(h->s->tiled, INSEM_CUDA_ERR_INVALID, "batched solves run on the tiled path");
  INSEM_REQUIRE(h->s->device == opts.device, INSEM_CUDA_ERR_INVALID, "the solve lives on another device");
  INSEM_REQUIRE(!h->s->batch_owner, INSEM_CUDA_ERR_STATE, "the solve belongs to a batch");
  for (const auto& m : members) INSEM_REQUIRE(m.get() != h, INSEM_CUDA_ERR_STATE, "the solve belongs to this batch");
  int64_t pts = 0;
  for (const auto& d : h->s->domains) pts += d.ng;
  members.emplace_back(h);
  h->s->batch_owner = this;
  prepared.push_back(0);
  member_points.push_back(pts);
  dirty = true;
  return static_cast<int32_t>(members.size()) - 1;
}

void Batch::remove(int32_t index) {
  INSEM_REQUIRE(index >= 0 && index < size() && members[index], INSEM_CUDA_ERR_INVALID, "no such batch member");
  DeviceGuard dg(opts.device);
  CUDA_CHECK(cudaStreamSynchronize(stream));
  if (graph) {
    CUDA_CHECK(cudaGraphExecDestroy(graph));
    graph = nullptr;
  }
  members[index].reset();
  dirty = true;
}

insem_cuda_solver* Batch::member(int32_t index) {
  INSEM_REQUIRE(index >= 0 && index < size() && members[index], INSEM_CUDA_ERR_INVALID, "no such batch member");
  return members[index].get();
}

int32_t Batch::active() const {
  int32_t n = 0;
  for (const auto& m : members)
    if (m && m->s->remaining() > 0) ++n;
  return n;
}

int32_t Batch::steps_to_next_completion() const {
  int32_t k = 0;
  for (const auto& m : members)
    if (m && m->s->remaining() > 0) k = k == 0 ? m->s->remaining() : std::min(k, m->s->remaining());
  return k;
}

void Batch::rebuild() {
  CUDA_CHECK(cudaStreamSynchronize(stream));
  if (graph) {
    CUDA_CHECK(cudaGraphExecDestroy(graph));
    graph = nullptr;
  }
  BatchTables T;
  for (std::size_t i = 0; i < members.size(); ++i) {
    if (!members[i] || members[i]->s->remaining() <= 0) continue;
    Solver& s = *members[i]->s;
    if (!prepared[i]) {
      s.batch_prepare();
      prepared[i] = 1;
    }
    s.batch_collect(T);
  }
  dclasses.clear();
  std::vector<std::pair<double, std::size_t>> work;  // (elements x points per element x components, class)
  for (auto& kv : T.tiles) {
    TileClass& c = kv.second;
    DevClass d;
    d.ngll = c.ngll;
    d.kind = c.kind;
    d.m = c.m;
    d.ncomp = c.ncomp;
    d.elastic = c.elastic;
    d.segs.upload_async(c.segs, stream);
    d.items.upload_async(c.items, stream);
    d.n_items = static_cast<int32_t>(c.items.size());
    d.te = c.te;
    d.L = TileLayout::make(c.ngll, c.ncomp, c.kind, c.elastic, c.te, c.tp_cap, c.nc_cap, c.rank_cap);
    TileBatchLaunch a;
    a.te = c.te;
    a.kind = c.kind;
    a.m = c.m;
    a.elastic = c.elastic;
    a.L = d.L;
    a.smem = d.L.total;
    const int per_sm = std::max(1, tile_batch(c.ngll, a, false));
    // one CTA per item (the call above also sets the kernel's shared memory size)
    (void)per_sm;
    d.grid = d.n_items;  // CTA b reads item b: no launch without items
    double w = 0.0;
    for (const TileItem& it : c.items) w += static_cast<double>(it.th.ne);
    work.emplace_back(w * c.ngll * c.ngll * c.ncomp, dclasses.size());
    dclasses.push_back(std::move(d));
  }
  {
    // lanes: elastic classes by component count, then the acoustic classes
    // by work, largest first, each to the least loaded lane
    std::sort(work.begin(), work.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<double> load(n_lanes, 0.0);
    for (const auto& w : work) {
      DevClass& d = dclasses[w.second];
      if (!d.elastic) continue;
      d.lane = d.ncomp == 3 ? lane3() : 0;
      load[d.lane] += w.first;
    }
    for (const auto& w : work) {
      DevClass& d = dclasses[w.second];
      if (d.elastic) continue;
      d.lane = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
      load[d.lane] += w.first;
    }
  }
  for (int c = 0; c < 3; ++c) {
    dhalo_segs[c].upload_async(T.halo_segs[c], stream);
    dhalo_items[c].upload_async(T.halo_items[c], stream);
    n_halo_items[c] = static_cast<int32_t>(T.halo_items[c].size());
  }
  dcons_segs.upload_async(T.cons_segs, stream);
  dcons_items.upload_async(T.cons_items, stream);
  n_cons_items = static_cast<int32_t>(T.cons_items.size());
  drec_segs.upload_async(T.rec_segs, stream);
  dpv_items.upload_async(T.pv_items, stream);
  drec_items.upload_async(T.rec_items, stream);
  n_pv_items = static_cast<int32_t>(T.pv_items.size());
  n_rec_items = static_cast<int32_t>(T.rec_items.size());
  denergy.upload_async(T.energy_segs, stream);
  n_energy = static_cast<int32_t>(T.energy_segs.size());
  dstates.upload_async(T.states, stream);
  n_states = static_cast<int32_t>(T.states.size());
  dstream.upload_async(T.stream_segs, stream);
  n_stream = static_cast<int32_t>(T.stream_segs.size());
  amp_cols = T.amp_cols;
  row_cols = T.row_cols;
  if (amp_stage.size() < static_cast<std::size_t>(std::max(amp_cols, 1))) amp_stage.resize(std::max(amp_cols, 1));
  if (row_stage.size() < static_cast<std::size_t>(std::max(row_cols, 1))) row_stage.resize(std::max(row_cols, 1));
  CUDA_CHECK(cudaStreamSynchronize(stream));
  if (opts.use_graphs && n_states > 0) {
    cudaGraph_t g = nullptr;
    CUDA_CHECK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue();
    } catch (...) {
      cudaStreamEndCapture(stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    CUDA_CHECK(cudaStreamEndCapture(stream, &g));
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
    CUDA_CHECK(cudaGraphInstantiate(&graph, g, 0));
    CUDA_CHECK(cudaGraphDestroy(g));
  }
  dirty = false;
}

void Batch::enqueue(cudaEvent_t tiles_begin, cudaEvent_t tiles_end) {
  const int32_t nq = static_cast<int32_t>(dclasses.size());
  batch_begin_kernel<<<ceil_div(std::max(n_states, 1), 256), 256, 0, stream>>>(dstates.get(), n_states);
  CUDA_LAUNCH_CHECK();
  if (n_cons_items > 0) {
    constrained_batch_kernel<<<n_cons_items, kConsChunk, 0, stream>>>(dcons_segs.get(), dcons_items.get());
    CUDA_LAUNCH_CHECK();
  }
  if (tiles_begin) CUDA_CHECK(cudaEventRecord(tiles_begin, stream));
  int used = 1;  // lanes in use: 0 .. used-1
  for (const DevClass& d : dclasses) used = std::max(used, d.lane + 1);
  if (n_halo_items[2] > 0) used = std::max(used, lane3() + 1);
  if (used > 1) {
    CUDA_CHECK(cudaEventRecord(fork_ev, stream));
    for (int k = 1; k < used; ++k) CUDA_CHECK(cudaStreamWaitEvent(lanes[k - 1], fork_ev, 0));
  }
  for (int32_t q = 0; q < nq; ++q) {
    const DevClass& d = dclasses[q];
    if (d.n_items == 0) continue;
    TileBatchLaunch a;
    a.kind = d.kind;
    a.m = d.m;
    a.elastic = d.elastic;
    a.segs = d.segs.get();
    a.items = d.items.get();
    a.te = d.te;
    a.L = d.L;
    a.smem = d.L.total;
    a.grid = d.grid;
    a.stream = d.lane == 0 ? stream : lanes[d.lane - 1];
    tile_batch(d.ngll, a, true);
  }
  auto join = [&]() {
    for (int k = 1; k < used; ++k) {
      CUDA_CHECK(cudaEventRecord(join_ev[k - 1], lanes[k - 1]));
      CUDA_CHECK(cudaStreamWaitEvent(stream, join_ev[k - 1], 0));
    }
  };
  // solid halos first: the fluid's coupling term reads the solid's new
  // acceleration.  Timed runs (tiles_end) keep every tile ahead of the halos.
  if (tiles_end) {
    join();
    CUDA_CHECK(cudaEventRecord(tiles_end, stream));
  }
  if (n_halo_items[1] > 0) {
    halo_batch_kernel<2, true><<<n_halo_items[1], kHaloChunk, 0, stream>>>(dhalo_segs[1].get(), dhalo_items[1].get());
    CUDA_LAUNCH_CHECK();
  }
  if (n_halo_items[2] > 0) {
    cudaStream_t s3 = tiles_end || lane3() == 0 ? stream : lanes[lane3() - 1];
    halo_batch_kernel<3, true><<<n_halo_items[2], kHaloChunk, 0, s3>>>(dhalo_segs[2].get(), dhalo_items[2].get());
    CUDA_LAUNCH_CHECK();
  }
  if (!tiles_end) join();
  if (n_halo_items[0] > 0) {
    halo_batch_kernel<1, false><<<n_halo_items[0], kHaloChunk, 0, stream>>>(dhalo_segs[0].get(), dhalo_items[0].get());
    CUDA_LAUNCH_CHECK();
  }
  if (n_pv_items > 0) {
    particle_velocity_batch_kernel<<<n_pv_items, kRecChunk, 0, stream>>>(drec_segs.get(), dpv_items.get());
    CUDA_LAUNCH_CHECK();
  }
  if (n_rec_items > 0) {
    record_batch_kernel<<<n_rec_items, kRecChunk, 0, stream>>>(drec_segs.get(), drec_items.get());
    CUDA_LAUNCH_CHECK();
  }
  if (n_energy > 0) {
    energy_batch_kernel<<<n_energy, kReduceThreads, 0, stream>>>(denergy.get());
    CUDA_LAUNCH_CHECK();
  }
}

int32_t Batch::max_remaining() const {
  int32_t k = 0;
  for (const auto& m : members)
    if (m) k = std::max(k, m->s->remaining());
  return k;
}

// After k batched steps: each running solve did min(k, its remaining) steps
// and idled after its last one.
void Batch::credit(int32_t k) {
  std::vector<std::pair<std::size_t, Solver*>> done;
  for (std::size_t i = 0; i < members.size(); ++i) {
    if (!members[i] || !prepared[i] || members[i]->s->remaining() <= 0) continue;
    Solver& s = *members[i]->s;
    const int32_t d = std::min(k, s.remaining());
    s.batch_advanced(d);
    point_updates += member_points[i] * d;
    if (s.remaining() == 0) {
      dirty = true;
      done.push_back({i, &s});
    }
  }
  INSEM_REQUIRE(!*herr, INSEM_CUDA_ERR_TIMEOUT, "a tile's bulk copies did not arrive within the wait limit");
  if (!opts.check_finite) return;
  // every member that finished is checked; the error names all that failed
  // (each is marked: insem_cuda_solver_status), the others are complete
  std::string failed;
  for (const auto& [i, s] : done) {
    try {
      s->check_fields();
    } catch (const Error& e) {
      if (e.code != INSEM_CUDA_ERR_NONFINITE) throw;
      failed += (failed.empty() ? "" : ", ") + std::to_string(i);
    }
  }
  INSEM_REQUIRE(failed.empty(), INSEM_CUDA_ERR_NONFINITE,
                "batch members " + failed + ": the solution contains NaN or Inf (unstable time step?)");
}

void Batch::finish_steps() {
  batch_error_kernel<<<ceil_div(std::max(n_states, 1), 256), 256, 0, stream>>>(dstates.get(), n_states, derr.get());
  CUDA_LAUNCH_CHECK();
  CUDA_CHECK(cudaMemcpyAsync(herr, derr.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
  CUDA_CHECK(cudaStreamSynchronize(stream));
}

void Batch::advance(int32_t n) {
  DeviceGuard dg(opts.device);
  INSEM_REQUIRE(n >= 0, INSEM_CUDA_ERR_INVALID, "negative step count");
  point_updates = 0;
  last_ms = 0.0;
  const int32_t k = std::min(n, max_remaining());
  if (k == 0) return;
  if (dirty) rebuild();
  CUDA_CHECK(cudaMemsetAsync(derr.get(), 0, sizeof(int32_t), stream));
  CUDA_CHECK(cudaEventRecord(ev0, stream));
  for (int32_t j = 0; j < k; ++j) {
    if (graph) CUDA_CHECK(cudaGraphLaunch(graph, stream));
    else enqueue();
  }
  CUDA_CHECK(cudaEventRecord(ev1, stream));
  finish_steps();
  float ms = 0.0f;
  CUDA_CHECK(cudaEventElapsedTime(&ms, ev0, ev1));
  last_ms = ms;
  credit(k);
}

void Batch::stream_layout(int32_t* a, int32_t* r) {
  DeviceGuard dg(opts.device);
  const bool running = max_remaining() > 0;
  if (dirty && running) rebuild();
  if (a) *a = running ? amp_cols : 0;
  if (r) *r = running ? row_cols : 0;
}

int32_t Batch::advance_streamed(int32_t n, const float* amp_in, double* rows_out) {
  DeviceGuard dg(opts.device);
  INSEM_REQUIRE(n >= 0, INSEM_CUDA_ERR_INVALID, "negative step count");
  point_updates = 0;
  last_ms = 0.0;
  const int32_t k = std::min(n, max_remaining());
  if (k == 0) return 0;
  if (dirty) rebuild();
  CUDA_CHECK(cudaMemsetAsync(derr.get(), 0, sizeof(int32_t), stream));
  CUDA_CHECK(cudaEventRecord(ev0, stream));
  for (int32_t j = 0; j < k; ++j) {
    if (amp_cols > 0 && amp_in) {
      CUDA_CHECK(cudaMemcpyAsync(amp_stage.get(), amp_in + static_cast<std::size_t>(j) * amp_cols,
                                 amp_cols * sizeof(float), cudaMemcpyHostToDevice, stream));
      batch_amp_scatter_kernel<<<n_stream, 64, 0, stream>>>(dstream.get(), amp_stage.get());
      CUDA_LAUNCH_CHECK();
    }
    if (graph) CUDA_CHECK(cudaGraphLaunch(graph, stream));
    else enqueue();
    if (rows_out && row_cols > 0) {
      batch_row_gather_kernel<<<n_stream, 64, 0, stream>>>(dstream.get(), row_stage.get());
      CUDA_LAUNCH_CHECK();
      CUDA_CHECK(cudaMemcpyAsync(rows_out + static_cast<std::size_t>(j) * row_cols, row_stage.get(),
                                 row_cols * sizeof(double), cudaMemcpyDeviceToHost, stream));
    }
  }
  CUDA_CHECK(cudaEventRecord(ev1, stream));
  finish_steps();
  float ms = 0.0f;
  CUDA_CHECK(cudaEventElapsedTime(&ms, ev0, ev1));
  last_ms = ms;
  credit(k);
  return k;
}

void Batch::profile(int32_t n, double* tile_ms, double* step_ms) {
  DeviceGuard dg(opts.device);
  INSEM_REQUIRE(n >= 0, INSEM_CUDA_ERR_INVALID, "negative step count");
  point_updates = 0;
  const int32_t k = std::min(n, max_remaining());
  double tt = 0.0, ts = 0.0;
  if (k > 0) {
    if (dirty) rebuild();
    std::vector<cudaEvent_t> ev(4 * static_cast<std::size_t>(k));
    for (auto& e : ev) CUDA_CHECK(cudaEventCreate(&e));
    CUDA_CHECK(cudaMemsetAsync(derr.get(), 0, sizeof(int32_t), stream));
    for (int32_t j = 0; j < k; ++j) {
      CUDA_CHECK(cudaEventRecord(ev[4 * j], stream));
      enqueue(ev[4 * j + 1], ev[4 * j + 2]);
      CUDA_CHECK(cudaEventRecord(ev[4 * j + 3], stream));
    }
    finish_steps();
    for (int32_t j = 0; j < k; ++j) {
      float a = 0.0f, b = 0.0f;
      CUDA_CHECK(cudaEventElapsedTime(&a, ev[4 * j + 1], ev[4 * j + 2]));
      CUDA_CHECK(cudaEventElapsedTime(&b, ev[4 * j], ev[4 * j + 3]));
      tt += a;
      ts += b;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    credit(k);
  }
  if (tile_ms) *tile_ms = tt;
  if (step_ms) *step_ms = ts;
}

void Batch::run() { advance(max_remaining()); }

}  // namespace insem_b200

using namespace insem_b200;

struct insem_cuda_batch {
  std::unique_ptr<Batch> b;
};

extern "C" {

int insem_cuda_solver_prepare_for_batch(insem_cuda_solver* h) {
  return guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    h->s->batch_prepare();
  });
}

int insem_cuda_batch_create(const insem_cuda_options* options, insem_cuda_batch** out) {
  return guarded([&] {
    INSEM_REQUIRE(out, INSEM_CUDA_ERR_INVALID, "null argument");
    auto h = std::make_unique<insem_cuda_batch>();
    h->b = std::make_unique<Batch>(options);
    *out = h.release();
  });
}

void insem_cuda_batch_destroy(insem_cuda_batch* h) { delete h; }

int insem_cuda_batch_add(insem_cuda_batch* h, const insem_cuda_problem* problem, int32_t* index) {
  return guarded([&] {
    INSEM_REQUIRE(h && problem, INSEM_CUDA_ERR_INVALID, "null argument");
    const int32_t i = h->b->add(*problem);
    if (index) *index = i;
  });
}

int insem_cuda_batch_adopt(insem_cuda_batch* h, insem_cuda_solver* solver, int32_t* index) {
  return guarded([&] {
    INSEM_REQUIRE(h && solver, INSEM_CUDA_ERR_INVALID, "null argument");
    const int32_t i = h->b->adopt(solver);  // the batch owns the solve from here on
    if (index) *index = i;
  });
}

int insem_cuda_batch_advance(insem_cuda_batch* h, int32_t n) {
  return guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    h->b->advance(n);
  });
}

int insem_cuda_batch_run(insem_cuda_batch* h) {
  return guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    h->b->run();
  });
}

int insem_cuda_batch_remove(insem_cuda_batch* h, int32_t index) {
  return guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    h->b->remove(index);
  });
}

insem_cuda_solver* insem_cuda_batch_member(insem_cuda_batch* h, int32_t index) {
  insem_cuda_solver* out = nullptr;
  guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    out = h->b->member(index);
  });
  return out;
}

int insem_cuda_batch_advance_streamed(insem_cuda_batch* h, int32_t n, const float* amp_in, double* rows_out,
                                      int32_t* n_done) {
  return guarded([&] {
    INSEM_REQUIRE(h && n_done, INSEM_CUDA_ERR_INVALID, "null argument");
    *n_done = h->b->advance_streamed(n, amp_in, rows_out);
  });
}

int insem_cuda_batch_stream_layout(insem_cuda_batch* h, int32_t* amp_cols, int32_t* row_cols) {
  return guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    h->b->stream_layout(amp_cols, row_cols);
  });
}

int insem_cuda_batch_profile(insem_cuda_batch* h, int32_t n, double* tile_ms, double* step_ms) {
  return guarded([&] {
    INSEM_REQUIRE(h, INSEM_CUDA_ERR_INVALID, "null handle");
    h->b->profile(n, tile_ms, step_ms);
  });
}

int32_t insem_cuda_batch_size(const insem_cuda_batch* h) { return h ? h->b->size() : 0; }
int32_t insem_cuda_batch_active(const insem_cuda_batch* h) { return h ? h->b->active() : 0; }
int32_t insem_cuda_batch_steps_to_next_completion(const insem_cuda_batch* h) {
  return h ? h->b->steps_to_next_completion() : 0;
}
int32_t insem_cuda_batch_steps_to_completion(const insem_cuda_batch* h) { return h ? h->b->max_remaining() : 0; }
double insem_cuda_batch_last_advance_ms(const insem_cuda_batch* h) { return h ? h->b->last_ms : 0.0; }
int64_t insem_cuda_batch_point_updates(const insem_cuda_batch* h) { return h ? h->b->point_updates : 0; }
int32_t insem_cuda_batch_kernels_per_step(const insem_cuda_batch* h) { return h ? h->b->kernels_per_step : 0; }

}  // extern "C"
