// Device side of the C ABI: table upload, work planning, kernel launches,
// report compaction and results.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <functional>
#include <mutex>
#include <memory>
#include <tuple>
#include <vector>

#include "common.h"
#include "handles.h"
#include "match_kernel.cuh"
#include "sort_kernels.cuh"
#include "tables.h"

using namespace ngap;

namespace {

#define CUDA_TRY(expr)                                                                     \
  do {                                                                                     \
    cudaError_t _e = (expr);                                                               \
    if (_e != cudaSuccess) {                                                               \
      set_error("CUDA error %s at %s:%d: %s", cudaGetErrorName(_e), __FILE__, __LINE__,    \
                cudaGetErrorString(_e));                                                   \
      return NGAP_E_CUDA;                                                                  \
    }                                                                                      \
  } while (0)

// Device counters of an engine: [0] raw reports, [1] unique reports, [2..3]
// work, [5..6] the standalone sort's counts, [kRadixCount] keys left to the
// radix pipeline after the small-set sort.
constexpr int kNumCounters = 16;
constexpr int kDefaultQueue = 1 << 16;  // overflow-stack entries per warp
constexpr int kRadixCount = 8;

int bits_for(uint64_t x) {  // bits needed to hold values < x (x >= 1)
  int b = 0;
  while (b < 64 && (x - 1) >> b) b++;
  return b;
}

}  // namespace

// A report sort captured as a CUDA graph (see sort_reports).
struct SortGraph {
  std::vector<uint64_t> key;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  int chain = 0;  // kernels in the conditional radix pipeline
  void release() {
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    ge = nullptr;
    g = nullptr;
  }
};

// Plan caches key on these serial numbers, not on addresses: a new object
// may be allocated where a destroyed one was.
std::atomic<uint64_t> g_next_serial{1};

struct ngap_tables {
  uint64_t serial = g_next_serial.fetch_add(1);
  int device = 0;
  int num_groups = 0;
  std::vector<TileHost> tiles;
  std::vector<TileDev> dev_desc;
  TileDev* d_tiles = nullptr;
  std::vector<void*> allocs;
  int64_t bytes = 0;
  int32_t max_states = 0;
  int32_t image_region = 0;  // shared-memory bytes reserved for tile images
  std::vector<int32_t> plan_bytes;  // per tile: image size of the planning rule (TileHost)
  std::vector<char> tile_lean;      // per tile: plain, no sticky states (the lean kernel runs it)
  std::vector<int32_t> pair_nact;  // activation slots of each (activation, layered) tile pair
  int32_t max_nact = 0;            // largest pair

  ~ngap_tables() {
    for (void* p : allocs) cudaFree(p);
  }
  template <class T>
  int upload(const std::vector<T>& v, const T** out) {
    *out = nullptr;
    if (v.empty()) return NGAP_OK;
    void* p = nullptr;
    size_t b = v.size() * sizeof(T);
    CUDA_TRY(cudaMalloc(&p, b));
    allocs.push_back(p);
    bytes += (int64_t)b;
    CUDA_TRY(cudaMemcpy(p, v.data(), b, cudaMemcpyHostToDevice));
    *out = static_cast<const T*>(p);
    return NGAP_OK;
  }
};

struct UnitPlanKey {
  int64_t num_seg, seg_len;
  int is_dup, window, chunk;
  int64_t first_seg;
  bool operator<(const UnitPlanKey& o) const {
    return std::tie(num_seg, seg_len, is_dup, window, chunk, first_seg) <
           std::tie(o.num_seg, o.seg_len, o.is_dup, o.window, o.chunk, o.first_seg);
  }
};

struct ngap_engine {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  // input
  uint8_t* d_input = nullptr;
  size_t input_cap = 0;
  // units (cached plan for one tables object)
  uint64_t plan_tables = 0;  // serial of the tables the plain plan was made for
  UnitPlanKey plan_key{-1, -1, -1, -1, -1, -1};
  UnitDev* d_units = nullptr;
  size_t units_cap = 0;
  int32_t nunits = 0;
  TaskDev* d_tasks = nullptr;
  size_t tasks_cap = 0;
  int32_t ntasks = 0;
  int32_t ntasks1 = 0;       // tasks of activation tiles, launched first
  int32_t ntasks2 = 0;       // tasks of plain tiles without sticky states (the lean launch)
  int32_t free_range[6] = {0, 0, 0, 0, 0, 0};  // free units: [begin, count) of each launch
  int32_t free_tile[3] = {-1, -1, -1};  // the one tile of each launch's free units, or -1
  // worklist traces
  bool trace = false;
  unsigned long long* d_unit_work = nullptr;
  size_t unit_work_cap = 0;
  std::vector<UnitDev> h_units;  // the current plan's units (host copy)
  int64_t trace_seg_len = 0;     // plain matching: unit positions are made segment-relative
  int64_t act_entries = 0;   // activation slots the plan uses
  uint32_t* d_act = nullptr;
  uint32_t* d_act_list = nullptr;  // per row: slots with a first match (compacted)
  int64_t act_cap = 0;
  int32_t act_rows = 0;            // rows of the plan
  int64_t* d_row_off = nullptr;    // per row: first slot
  int32_t* d_row_n = nullptr;      // per row: slots
  uint32_t* d_act_cnt = nullptr;   // per row: matched slots
  int32_t rows_cap = 0;
  uint32_t* d_stk = nullptr; // per-slot sticky lists of layered units (beyond shared memory)
  int stk_cap = 0;
  // reports
  uint64_t rep_cap = 0;
  uint64_t* d_reports = nullptr;
  uint64_t* d_tmp = nullptr;
  uint64_t* d_unique = nullptr;
  uint32_t* d_hist = nullptr;
  size_t hist_cap = 0;
  // counters: [0] raw reports, [1] unique reports, [2] expanded, [3] injected
  unsigned long long* d_counters = nullptr;
  int* d_err = nullptr;
  unsigned int* d_unit_counter = nullptr;
  unsigned long long* h_counters = nullptr;  // pinned mirror: [0..3] counters, [4] err,
                                             // [kRadixCount] keys left to the radix pipeline
  // per-warp scratch
  uint32_t* d_carry = nullptr;
  uint32_t* d_marks = nullptr;
  uint32_t* d_ovf = nullptr;
  size_t slots = 0;
  int carry_cap = 0, mark_words = 0, ovf_cap = 0;
  int max_smem_set = -1;
  int bps_smem[3] = {-1, -1, -1}, bps_val[3] = {0, 0, 0};  // resident CTAs per SM, per PRIV
  // pinned staging of plan uploads (grow-only) and the event of the last one
  uint8_t* h_plan = nullptr;
  size_t h_plan_cap = 0;
  cudaEvent_t plan_ev = nullptr;
  bool plan_ev_pending = false;
  // timing
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  float match_ms = 0.f, sort_ms = 0.f;
  int launches = 0;
  int pending_status = NGAP_OK;
  bool ran = false;
  int grid = 0;
  // batched matching
  uint64_t batch_ts = 0;     // serial of the tableset the batched plan was made for
  std::vector<ngap_batch_stream> batch_streams;
  int batch_window = -1, batch_chunk = -1;
  uint32_t* d_stream_ids = nullptr;
  uint64_t stream_ids_cap = 0;
  cudaGraphExec_t graph = nullptr;
  std::vector<uint64_t> graph_key;
  bool graph_mode = false;
  int graph_launches = 0;
  cudaStream_t cap_stream = nullptr;  // capture/replay stream of the batched graph
  cudaEvent_t cap_ev[2] = {nullptr, nullptr};
  // report sorts as graphs with a conditional radix pipeline, per configuration
  std::vector<SortGraph> sort_graphs;
  cudaStream_t sort_cs = nullptr;     // capture stream of those graphs
  bool sort_graph_off = false;
  int sort_chain_pending = 0;         // pipeline kernels of the last graph sort, if it ran
  // test hook for the bounded device wait (ngap_engine_test_wait_timeout): armed for the
  // next ngap_match only
  int32_t test_skip_unit = -1;
  int32_t test_wait_rounds = 0;

  ~ngap_engine() {
    cudaFree(d_input);
    cudaFree(d_units);
    cudaFree(d_tasks);
    cudaFree(d_reports);
    cudaFree(d_tmp);
    cudaFree(d_unique);
    cudaFree(d_hist);
    cudaFree(d_counters);
    cudaFree(d_err);
    cudaFree(d_unit_counter);
    cudaFree(d_carry);
    cudaFree(d_marks);
    cudaFree(d_ovf);
    cudaFree(d_unit_work);
    cudaFree(d_act);
    cudaFree(d_act_list);
    cudaFree(d_row_off);
    cudaFree(d_row_n);
    cudaFree(d_act_cnt);
    cudaFree(d_stk);
    cudaFree(d_stream_ids);
    if (graph) cudaGraphExecDestroy(graph);
    for (auto& g : sort_graphs) g.release();
    if (sort_cs) cudaStreamDestroy(sort_cs);
    for (auto& c : cap_ev)
      if (c) cudaEventDestroy(c);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    if (h_counters) cudaFreeHost(h_counters);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (plan_ev) cudaEventSynchronize(plan_ev);
    if (plan_ev) cudaEventDestroy(plan_ev);
    if (h_plan) cudaFreeHost(h_plan);
  }
};

extern "C" {

int ngap_tables_build(const ngap_groups* g, const ngap_table_opts* opts, ngap_tables** out) {
  if (!g || !out) {
    set_error("ngap_tables_build: null argument");
    return NGAP_E_INVALID;
  }
  *out = nullptr;
  TableOpts to;
  int device = 0;
  int rc = table_opts_from(opts, "ngap_tables_build", to, &device);
  if (rc != NGAP_OK) return rc;
  std::unique_ptr<ngap_tables> t(new ngap_tables());
  t->device = device;
  CUDA_TRY(cudaSetDevice(device));
  rc = build_tiles(g->gs, to, t->tiles);
  if (rc != NGAP_OK) return rc;
  t->num_groups = (int)g->gs.groups.size();
  for (auto& th : t->tiles) {
    if (th.nstates >= kMaxTileStates - 1) {
      set_error("a connected component has %d states; at most %d are supported per tile",
                th.nstates, kMaxTileStates - 2);
      return NGAP_E_UNSUPPORTED;
    }
    t->max_states = std::max(t->max_states, th.nstates);
    t->tile_lean.push_back(th.nsticky == 0 && th.phase == 0 ? 1 : 0);
    TileDev d;
    d.group = th.group;
    d.nstates = th.nstates;
    d.naas = (int32_t)th.aas.size();
    d.nstart = (int32_t)th.start.size();
    d.depth = th.depth;
    d.max_path = th.max_path;
    d.ncls = th.ncls;
    d.cw = th.cw;
    d.nlive = th.nlive;
    d.narrow = th.narrow ? 1 : 0;
    d.fused = th.fused ? 1 : 0;
    d.image_bytes = (int32_t)th.image.size();
    d.off_cmask = th.off_cmask;
    d.off_rep = th.off_rep;
    d.off_cls = th.off_cls;
    d.inj_batch = th.inj_batch;
    d.inj_batch0 = th.inj_batch0;
    d.nsticky = th.nsticky;
    d.off_sticky = th.off_sticky;
    d.phase = th.phase;
    d.nact = th.nact;
    if (th.pair >= 0) {
      if ((int)t->pair_nact.size() <= th.pair) t->pair_nact.resize(th.pair + 1, 0);
      t->pair_nact[th.pair] = th.nact;
      t->max_nact = std::max(t->max_nact, th.nact);
    }
    if ((rc = t->upload(th.act_local, &d.act_local)) != NGAP_OK) return rc;
    if ((rc = t->upload(th.stk_union, &d.stk_union)) != NGAP_OK) return rc;
    if ((rc = t->upload(th.image, &d.image)) != NGAP_OK) return rc;
    if ((rc = t->upload(th.sid, &d.sid)) != NGAP_OK) return rc;
    if ((rc = t->upload(th.aas, &d.aas)) != NGAP_OK) return rc;
    if ((rc = t->upload(th.start, &d.start)) != NGAP_OK) return rc;
    for (int k = 0; k < kMaxDepth; k++) {
      const PrefixTableHost& ph = th.pt[k];
      PrefixTableDev& pd = d.pt[k];
      pd.dense = ph.dense ? 1 : 0;
      pd.inline1 = ph.inline1 ? 1 : 0;
      pd.hmask = ph.hmask;
      pd.cutoff = ph.cutoff;
      pd.has_reports = ph.rlist.empty() ? 0 : 1;
      if ((rc = t->upload(ph.voff, &pd.voff)) != NGAP_OK) return rc;
      if ((rc = t->upload(ph.roff, &pd.roff)) != NGAP_OK) return rc;
      const uint32_t* slots = nullptr;
      if ((rc = t->upload(ph.slots, &slots)) != NGAP_OK) return rc;
      pd.slots = reinterpret_cast<const uint4*>(slots);
      if ((rc = t->upload(ph.vlist, &pd.vlist)) != NGAP_OK) return rc;
      if ((rc = t->upload(ph.rlist, &pd.rlist)) != NGAP_OK) return rc;
    }
    t->dev_desc.push_back(d);
    t->plan_bytes.push_back((int32_t)th.plan_bytes);
    if (th.plan_bytes <= to.image_budget)
      t->image_region = std::max(t->image_region, (int32_t)th.plan_bytes);
  }
  t->image_region = (t->image_region + 127) & ~127;
  const TileDev* dt = nullptr;
  if ((rc = t->upload(t->dev_desc, &dt)) != NGAP_OK) return rc;
  t->d_tiles = const_cast<TileDev*>(dt);
  *out = t.release();
  return NGAP_OK;
}

void ngap_tables_destroy(ngap_tables* t) { delete t; }

int64_t ngap_tables_device_bytes(const ngap_tables* t) { return t ? t->bytes : 0; }

int ngap_engine_create(int device, ngap_engine** out) {
  if (!out) {
    set_error("ngap_engine_create: null argument");
    return NGAP_E_INVALID;
  }
  *out = nullptr;
  int ndev = 0;
  CUDA_TRY(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) {
    set_error("no CUDA device %d (%d present)", device, ndev);
    return NGAP_E_CUDA;
  }
  CUDA_TRY(cudaSetDevice(device));
  std::unique_ptr<ngap_engine> e(new ngap_engine());
  e->device = device;
  CUDA_TRY(cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, device));
  CUDA_TRY(cudaMalloc(&e->d_counters, kNumCounters * sizeof(unsigned long long)));
  CUDA_TRY(cudaFuncSetAttribute(small_sort_unique<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kSmallSortSmem));
  CUDA_TRY(cudaFuncSetAttribute(small_sort_unique<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kSmallSortSmem));
  CUDA_TRY(cudaMalloc(&e->d_err, sizeof(int)));
  CUDA_TRY(cudaMalloc(&e->d_unit_counter, 2 * sizeof(unsigned int)));  // tasks, free units
  CUDA_TRY(cudaMallocHost(&e->h_counters, kNumCounters * sizeof(unsigned long long)));
  for (auto& ev : e->ev) CUDA_TRY(cudaEventCreate(&ev));
  *out = e.release();
  return NGAP_OK;
}

void ngap_engine_destroy(ngap_engine* e) {
  if (e) {
    cudaSetDevice(e->device);
    delete e;
  }
}

}  // extern "C"

namespace {

// New capacity of a grow-only buffer that must hold `need` elements: at
// least twice the old one, so that a run of growing plans reallocates (a
// cudaMalloc, which waits for the device) only a few times.
template <class T>
T grown(T cap, T need) {
  return std::max(need, cap * 2);
}

// One host array to copy to a device buffer.
struct Upload {
  void* dst;
  const void* src;
  size_t bytes;
};

// Copies plan arrays to the device on stream st through the engine's pinned
// staging buffer, so that the host does not wait: a synchronous copy from
// pageable memory queues behind other streams' transfers on the copy
// engine (in a serving loop, the other slot's input copy). The staging
// buffer is written again only once the last upload has ended (an event).
// Inside a stream capture the copies stay synchronous, so that no captured
// node reads the reusable staging buffer.
int upload_plan(ngap_engine* e, cudaStream_t st, const std::vector<Upload>& parts) {
  size_t total = 0;
  for (const Upload& u : parts) total += (u.bytes + 15) & ~(size_t)15;
  if (total == 0) return NGAP_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CUDA_TRY(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) {
    for (const Upload& u : parts)
      if (u.bytes) CUDA_TRY(cudaMemcpy(u.dst, u.src, u.bytes, cudaMemcpyHostToDevice));
    return NGAP_OK;
  }
  if (e->plan_ev_pending) {
    CUDA_TRY(cudaEventSynchronize(e->plan_ev));
    e->plan_ev_pending = false;
  }
  if (total > e->h_plan_cap) {
    const size_t cap = grown(e->h_plan_cap, total);
    if (e->h_plan) cudaFreeHost(e->h_plan);
    e->h_plan = nullptr;
    e->h_plan_cap = 0;
    CUDA_TRY(cudaMallocHost(&e->h_plan, cap));
    e->h_plan_cap = cap;
  }
  if (!e->plan_ev) CUDA_TRY(cudaEventCreateWithFlags(&e->plan_ev, cudaEventDisableTiming));
  size_t off = 0;
  for (const Upload& u : parts) {
    if (u.bytes == 0) continue;
    std::memcpy(e->h_plan + off, u.src, u.bytes);
    CUDA_TRY(cudaMemcpyAsync(u.dst, e->h_plan + off, u.bytes, cudaMemcpyHostToDevice, st));
    off += (u.bytes + 15) & ~(size_t)15;
  }
  CUDA_TRY(cudaEventRecord(e->plan_ev, st));
  e->plan_ev_pending = true;
  return NGAP_OK;
}

int ensure_reports(ngap_engine* e, uint64_t cap) {
  if (cap <= e->rep_cap) return NGAP_OK;
  cudaFree(e->d_reports);
  cudaFree(e->d_tmp);
  cudaFree(e->d_unique);
  cudaFree(e->d_hist);
  e->d_reports = e->d_tmp = e->d_unique = nullptr;
  e->d_hist = nullptr;
  e->rep_cap = 0;
  CUDA_TRY(cudaMalloc(&e->d_reports, cap * sizeof(uint64_t)));
  CUDA_TRY(cudaMalloc(&e->d_tmp, cap * sizeof(uint64_t)));
  CUDA_TRY(cudaMalloc(&e->d_unique, cap * sizeof(uint64_t)));
  size_t ntiles = (cap + kSortTile - 1) / kSortTile;
  e->hist_cap = 16 * ntiles + 16;
  CUDA_TRY(cudaMalloc(&e->d_hist, e->hist_cap * sizeof(uint32_t)));
  e->rep_cap = cap;
  return NGAP_OK;
}

int ensure_slots(ngap_engine* e, size_t slots, int max_states, int max_nact, int ovf_cap) {
  int carry_cap = std::max(max_states, 32);
  int mark_words = (max_states + 31) / 32 + 1;
  // the overflow stacks only grow: a request for fewer entries than held
  // keeps them (more room changes no result, while reallocating would
  // cudaFree, which waits for every stream of the device)
  if (e->d_ovf && ovf_cap < e->ovf_cap) ovf_cap = e->ovf_cap;
  if (ovf_cap != e->ovf_cap && e->d_ovf) {  // queue capacity grew: reallocate everything
    e->slots = std::max(e->slots, slots);
    slots = e->slots;
    e->carry_cap = 0;
  }
  const int stk_cap = max_nact > kStickyCap ? max_nact : 0;
  if (slots <= e->slots && stk_cap > e->stk_cap) {  // only the sticky lists grow
    cudaFree(e->d_stk);
    e->d_stk = nullptr;
    e->stk_cap = 0;
    CUDA_TRY(cudaMalloc(&e->d_stk, e->slots * 2 * (size_t)stk_cap * sizeof(uint32_t)));
    e->stk_cap = stk_cap;
  }
  if (slots <= e->slots && carry_cap <= e->carry_cap && mark_words <= e->mark_words) return NGAP_OK;
  cudaFree(e->d_carry);
  cudaFree(e->d_marks);
  cudaFree(e->d_ovf);
  cudaFree(e->d_stk);
  e->d_carry = e->d_marks = e->d_ovf = e->d_stk = nullptr;
  e->stk_cap = 0;
  slots = std::max(slots, e->slots);
  e->slots = 0;
  if (stk_cap > 0) {
    CUDA_TRY(cudaMalloc(&e->d_stk, slots * 2 * (size_t)stk_cap * sizeof(uint32_t)));
    e->stk_cap = stk_cap;
  }
  CUDA_TRY(cudaMalloc(&e->d_carry, slots * (size_t)carry_cap * sizeof(uint32_t)));
  CUDA_TRY(cudaMalloc(&e->d_marks, slots * (size_t)mark_words * sizeof(uint32_t)));
  CUDA_TRY(cudaMemset(e->d_marks, 0, slots * (size_t)mark_words * sizeof(uint32_t)));
  CUDA_TRY(cudaMalloc(&e->d_ovf, slots * (size_t)ovf_cap * sizeof(uint32_t)));
  e->slots = slots;
  e->carry_cap = carry_cap;
  e->mark_words = mark_words;
  e->ovf_cap = ovf_cap;
  return NGAP_OK;
}

// Splits the work into units: unbounded tiles get one unit per segment;
// bounded tiles are cut into chunks of `chunk` emitted positions, each with
// max_path - 1 positions of warm-up (clamped at the segment start). Units of
// one tile are then cut into CTA tasks: the long per-segment units of
// unbounded tiles one per warp of a task and first, the chunks after them in
// tasks sized to give every CTA several tasks.
// One independent input range (a segment, or a whole stream in batched mode).
struct SegSpec {
  int64_t lo, hi;
  bool starts;      // start-of-data states active at lo
  uint64_t key_hi;  // stream index in the report key
  int64_t base;     // offsets in reports are relative to this
  int32_t index;    // segment or stream index
};

void add_units(const TileHost& th, int tile, const SegSpec& s, int window, int chunk_opt,
               std::pair<int64_t, int32_t> act, std::vector<UnitDev>& pass1,
               std::vector<UnitDev>& unbounded, std::vector<UnitDev>& bounded) {
  UnitDev u{};
  u.tile = tile;
  u.key_hi = s.key_hi;
  u.base = s.base;
  u.act_row = act.first;
  u.act_rowid = act.second;
  u.stream = s.index;
  std::vector<UnitDev>& chunks = th.phase == 1 ? pass1 : bounded;
  const bool starts = s.starts && !th.start.empty();
  if (th.max_path < 0) {
    u.flags = starts ? 1u : 0u;
    u.lo = s.lo;
    u.hi = s.hi;
    u.emit_lo = s.lo;
    unbounded.push_back(u);
    return;
  }
  const int64_t warm = th.max_path > 0 ? th.max_path - 1 : 0;
  // chunk length is independent of the window (the blocking algorithm runs
  // one-position windows); a chunk should span at least its warm-up
  const int64_t base = std::max<int64_t>(window, 2048);
  int64_t chunk = chunk_opt > 0 ? chunk_opt : std::max<int64_t>(base - warm, base / 2);
  chunk = std::max<int64_t>(chunk, 1);
  for (int64_t em = s.lo; em < s.hi; em += chunk) {
    u.lo = std::max(s.lo, em - warm);
    u.hi = std::min(em + chunk, s.hi);
    u.emit_lo = em;
    u.flags = (starts && u.lo == s.lo) ? 1u : 0u;
    chunks.push_back(u);
  }
}

// Activation rows: one per (tables index, pair, segment), nact slots each;
// the slots of pair q of tables n start at base[n][q], its rows at rbase[n][q].
struct ActRows {
  std::vector<std::vector<int64_t>> base;
  std::vector<std::vector<int32_t>> rbase;
  std::vector<int64_t> row_off;  // per row: first slot
  std::vector<int32_t> row_n;    // per row: slots
  int64_t total = 0;
  ActRows(const std::vector<const ngap_tables*>& ts, int64_t nseg) {
    for (const ngap_tables* t : ts) {
      base.emplace_back();
      rbase.emplace_back();
      for (int32_t nact : t->pair_nact) {
        base.back().push_back(total);
        rbase.back().push_back((int32_t)row_off.size());
        for (int64_t g = 0; g < nseg; g++) {
          row_off.push_back(total + g * nact);
          row_n.push_back(nact);
        }
        total += (int64_t)nact * nseg;
      }
    }
  }
  // (first slot, row id) of a unit of tile th over segment seg; (-1, -1) for plain tiles
  std::pair<int64_t, int32_t> row(int n, const TileHost& th, int64_t seg) const {
    if (th.pair < 0) return {-1, -1};
    return {base[n][th.pair] + seg * th.nact, rbase[n][th.pair] + (int32_t)seg};
  }
};

// Units (already grouped by tile) -> work of the launches. Units of tiles
// whose image is staged in shared memory become CTA tasks: the long units of
// cyclic tiles first, one per warp of a task; chunks after them in tasks sized
// to give every CTA several tasks. Units of tiles read in place (is_free)
// are taken one by one by warps (free units), after the tasks of their
// launch. Three launches: the activation tiles; the plain tiles without
// sticky states (is_lean: the lean kernel instance, with fewer registers
// spilled and a smaller code path); the rest. Layout of `units`, per launch
// in that order: [cyclic tasks][chunk tasks][cyclic free][chunk free];
// ntasks1 / ntasks2 count the tasks of the first two launches, free_range
// holds (begin, count) of each launch's free units.
void make_tasks(std::vector<UnitDev>& units, const std::vector<UnitDev>& pass1,
                const std::vector<UnitDev>& unbounded, const std::vector<UnitDev>& bounded,
                int grid, const std::function<bool(int)>& is_free,
                const std::function<bool(int)>& is_lean, std::vector<TaskDev>& tasks,
                int32_t* ntasks1, int32_t* ntasks2, int32_t free_range[6], int32_t free_tile[3]) {
  units.clear();
  tasks.clear();
  auto split = [&](const std::vector<UnitDev>& src, std::vector<UnitDev>& st,
                   std::vector<UnitDev>& fr) {
    for (const UnitDev& u : src) (is_free(u.tile) ? fr : st).push_back(u);
  };
  std::vector<UnitDev> p1s, p1f, ubs, ubf, bs, bf, lubs, lubf, lbs, lbf;
  split(pass1, p1s, p1f);
  std::vector<UnitDev> lean_ub, lean_b, rest_ub, rest_b;
  for (const UnitDev& u : unbounded) (is_lean(u.tile) ? lean_ub : rest_ub).push_back(u);
  for (const UnitDev& u : bounded) (is_lean(u.tile) ? lean_b : rest_b).push_back(u);
  split(lean_ub, lubs, lubf);
  split(lean_b, lbs, lbf);
  split(rest_ub, ubs, ubf);
  split(rest_b, bs, bf);
  // a launch whose free units all belong to one tile: its CTAs stage that
  // tile's descriptors in shared memory once
  auto one_tile = [](const std::vector<UnitDev>& a, const std::vector<UnitDev>& b) {
    int tile = -1;
    for (const auto* v : {&a, &b})
      for (const UnitDev& u : *v) {
        if (tile >= 0 && u.tile != tile) return -1;
        tile = u.tile;
      }
    return tile;
  };
  free_tile[0] = one_tile(p1f, {});
  free_tile[1] = one_tile(lubf, lbf);
  free_tile[2] = one_tile(ubf, bf);
  auto per = [&](size_t n) {
    return std::max<int64_t>(kWarpsPerCta,
                             std::min<int64_t>(512, (int64_t)n / std::max(1, 4 * grid)));
  };
  // a task holds at most `per` units and, past its first unit, about a
  // 16 * grid-th of the range's positions (at least 64 KiB), so that long
  // chunks do not make long tasks
  auto cut = [&](size_t b, size_t e, int64_t per) {
    int64_t total = 0;
    for (size_t k = b; k < e; k++) total += units[k].hi - units[k].lo;
    const int64_t cap = std::max<int64_t>(1 << 16, total / std::max(1, 16 * grid));
    size_t i = b;
    while (i < e) {
      size_t j = i;
      int64_t bytes = 0;
      while (j < e && units[j].tile == units[i].tile && (int64_t)(j - i) < per &&
             (j == i || bytes + (units[j].hi - units[j].lo) <= cap)) {
        bytes += units[j].hi - units[j].lo;
        j++;
      }
      TaskDev tk;
      tk.tile = units[i].tile;
      tk.ubegin = (int32_t)i;
      tk.uend = (int32_t)j;
      tk.pad = 0;
      tasks.push_back(tk);
      i = j;
    }
  };
  auto append = [&](const std::vector<UnitDev>& v) {
    const size_t b = units.size();
    units.insert(units.end(), v.begin(), v.end());
    return b;
  };
  size_t b = append(p1s);
  cut(b, units.size(), per(p1s.size()));
  *ntasks1 = (int32_t)tasks.size();
  free_range[0] = (int32_t)append(p1f);
  free_range[1] = (int32_t)p1f.size();
  auto launch = [&](const std::vector<UnitDev>& cs, const std::vector<UnitDev>& chs,
                    const std::vector<UnitDev>& cf, const std::vector<UnitDev>& chf,
                    int32_t* fr) {
    size_t bb = append(cs);
    cut(bb, units.size(), kWarpsPerCta);
    bb = append(chs);
    cut(bb, units.size(), per(chs.size()));
    fr[0] = (int32_t)append(cf);
    append(chf);
    fr[1] = (int32_t)(cf.size() + chf.size());
  };
  launch(lubs, lbs, lubf, lbf, free_range + 2);
  *ntasks2 = (int32_t)tasks.size() - *ntasks1;
  launch(ubs, bs, ubf, bf, free_range + 4);
}

ActRows plan_units(const ngap_tables* t, const UnitPlanKey& k, int grid,
                   std::vector<UnitDev>& units, std::vector<TaskDev>& tasks, int32_t* ntasks1,
                   int32_t* ntasks2, int32_t free_range[6], int32_t free_tile[3]) {
  std::vector<UnitDev> pass1, unbounded, bounded;
  ActRows rows({t}, k.num_seg);
  for (int ti = 0; ti < (int)t->tiles.size(); ti++) {
    for (int64_t s = 0; s < k.num_seg; s++) {
      SegSpec sp{s * k.seg_len, (s + 1) * k.seg_len, k.first_seg + s == 0 || k.is_dup != 0, 0ull,
                 0, (int32_t)s};
      add_units(t->tiles[ti], ti, sp, k.window, k.chunk, rows.row(0, t->tiles[ti], s), pass1,
                unbounded, bounded);
    }
  }
  const int32_t region = t->image_region;
  auto is_free = [&](int tile) { return t->plan_bytes[tile] > region; };
  auto is_lean = [&](int tile) { return t->tile_lean[tile] != 0; };
  make_tasks(units, pass1, unbounded, bounded, grid, is_free, is_lean, tasks, ntasks1, ntasks2,
             free_range, free_tile);
  return rows;
}

// Per-unit work counters when tracing (zeroed on st); null otherwise.
// d_unit_work holds two arrays of unit_work_cap words: work, then cycles
int trace_buffer(ngap_engine* e, cudaStream_t st, unsigned long long** work,
                 unsigned long long** cycles) {
  *work = *cycles = nullptr;
  if (!e->trace || e->nunits == 0) return NGAP_OK;
  if ((size_t)e->nunits > e->unit_work_cap) {
    const size_t cap = grown(e->unit_work_cap, (size_t)e->nunits);
    cudaFree(e->d_unit_work);
    e->d_unit_work = nullptr;
    e->unit_work_cap = 0;
    CUDA_TRY(cudaMalloc(&e->d_unit_work, 2 * cap * sizeof(unsigned long long)));
    e->unit_work_cap = cap;
  }
  CUDA_TRY(cudaMemsetAsync(e->d_unit_work, 0, (size_t)e->nunits * sizeof(unsigned long long), st));
  *work = e->d_unit_work;
  *cycles = e->d_unit_work + e->unit_work_cap;
  return NGAP_OK;
}

// Activation buffers of a plan (slots, compacted lists, row table).
int set_act_rows(ngap_engine* e, const ActRows& rows, std::vector<Upload>& ups) {
  e->act_entries = rows.total;
  e->act_rows = (int32_t)rows.row_off.size();
  if (e->act_entries > e->act_cap) {
    const int64_t cap = grown(e->act_cap, e->act_entries);
    cudaFree(e->d_act);
    cudaFree(e->d_act_list);
    e->d_act = e->d_act_list = nullptr;
    e->act_cap = 0;
    CUDA_TRY(cudaMalloc(&e->d_act, (size_t)cap * sizeof(uint32_t)));
    CUDA_TRY(cudaMalloc(&e->d_act_list, (size_t)cap * sizeof(uint32_t)));
    e->act_cap = cap;
  }
  if (e->act_rows > e->rows_cap) {
    const int32_t cap = grown(e->rows_cap, e->act_rows);
    cudaFree(e->d_row_off);
    cudaFree(e->d_row_n);
    cudaFree(e->d_act_cnt);
    e->d_row_off = nullptr;
    e->d_row_n = nullptr;
    e->d_act_cnt = nullptr;
    e->rows_cap = 0;
    CUDA_TRY(cudaMalloc(&e->d_row_off, (size_t)cap * sizeof(int64_t)));
    CUDA_TRY(cudaMalloc(&e->d_row_n, (size_t)cap * sizeof(int32_t)));
    CUDA_TRY(cudaMalloc(&e->d_act_cnt, (size_t)cap * sizeof(uint32_t)));
    e->rows_cap = cap;
  }
  if (e->act_rows > 0) {
    ups.push_back({e->d_row_off, rows.row_off.data(), rows.row_off.size() * sizeof(int64_t)});
    ups.push_back({e->d_row_n, rows.row_n.data(), rows.row_n.size() * sizeof(int32_t)});
  }
  return NGAP_OK;
}

// One warp per activation row: the slots with a first match, in slot order.
__global__ void act_compact(const int64_t* __restrict__ row_off, const int32_t* __restrict__ row_n,
                            int32_t nrows, const uint32_t* __restrict__ act,
                            uint32_t* __restrict__ list, uint32_t* __restrict__ cnt) {
  const int32_t row = (int32_t)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= nrows) return;  // whole warps
  const int64_t off = row_off[row];
  const int32_t n = row_n[row];
  uint32_t c = 0;
  for (int32_t i0 = 0; i0 < n; i0 += 32) {
    const int32_t i = i0 + lane;
    const bool ok = i < n && act[off + i] != 0xffffffffu;
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (ok) list[off + c + __popc(m & ((1u << lane) - 1u))] = (uint32_t)i;
    c += __popc(m);
  }
  if (lane == 0) cnt[row] = c;
}

// The matching launches of a plan: the activation tiles' tasks, then the rest
// (the layered tiles read what the first launch recorded).
// CTAs one launch needs: one per task, plus one per kWarpsPerCta free units,
// at most the grid.
int launch_grid(const ngap_engine* e, int ntasks, int nfree) {
  const int64_t want = (int64_t)ntasks + ((int64_t)nfree + kWarpsPerCta - 1) / kWarpsPerCta;
  return (int)std::max<int64_t>(1, std::min<int64_t>(e->grid, want));
}

int plan_grid(const ngap_engine* e, int full_grid) {
  const int64_t want = (int64_t)e->ntasks +
                       ((int64_t)e->free_range[1] + e->free_range[3] + e->free_range[5] +
                        kWarpsPerCta - 1) / kWarpsPerCta;
  return (int)std::max<int64_t>(1, std::min<int64_t>(full_grid, want));
}

// The matching launches of a plan: the activation tiles' work; the plain
// tiles without sticky states in the lean kernel instance; then the rest
// (the layered tiles read what the first launch recorded). Each launch takes
// its tasks first, then its free units.
template <int PRIV>
int launch_plan(ngap_engine* e, MatchParams mp, int smem, cudaStream_t st) {
  mp.free_cursor = e->d_unit_counter + 1;
  const TaskDev* const tasks0 = mp.tasks;
  if (e->act_entries > 0)
    CUDA_TRY(cudaMemsetAsync(e->d_act, 0xff, (size_t)e->act_entries * sizeof(uint32_t), st));
  auto run = [&](bool lean, int32_t tbegin, int32_t ntasks, int which) -> int {
    const int32_t nfree = e->free_range[2 * which + 1];
    if (ntasks == 0 && nfree == 0) return NGAP_OK;
    mp.tasks = tasks0 + tbegin;
    mp.ntasks = ntasks;
    mp.free_begin = e->free_range[2 * which];
    mp.nfree = nfree;
    mp.free_tile = e->free_tile[which];
    CUDA_TRY(cudaMemsetAsync(e->d_unit_counter, 0, 2 * sizeof(unsigned int), st));
    const int grid = launch_grid(e, ntasks, nfree);
    if (lean)
      match_kernel<PRIV, true><<<grid, kCtaThreads, smem, st>>>(mp);
    else
      match_kernel<PRIV, false><<<grid, kCtaThreads, smem, st>>>(mp);
    CUDA_TRY(cudaGetLastError());
    e->launches++;
    return NGAP_OK;
  };
  int rc = run(false, 0, e->ntasks1, 0);
  if (rc == NGAP_OK) rc = run(true, e->ntasks1, e->ntasks2, 1);
  if (rc != NGAP_OK) return rc;
  if (e->act_rows > 0) {
    act_compact<<<(e->act_rows + 7) / 8, 256, 0, st>>>(e->d_row_off, e->d_row_n, e->act_rows,
                                                       e->d_act, e->d_act_list, e->d_act_cnt);
    CUDA_TRY(cudaGetLastError());
    e->launches++;
  }
  return run(false, e->ntasks1 + e->ntasks2, e->ntasks - e->ntasks1 - e->ntasks2, 2);
}

int launch_any(ngap_engine* e, const MatchParams& mp, int smem, cudaStream_t st, int priv) {
  return priv == 0 ? launch_plan<0>(e, mp, smem, st)
                   : priv == 1 ? launch_plan<1>(e, mp, smem, st) : launch_plan<2>(e, mp, smem, st);
}

__global__ void swap_halves(uint64_t* a, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t x = a[i];
    a[i] = (x << 32) | (x >> 32);
  }
}

// The dynamic shared-memory limit is an attribute of the kernel function
// (per device, shared by every engine of the process), so it only ever grows.
std::mutex g_smem_mu;
int g_smem_set[64];

int set_smem(ngap_engine* e, int smem) {
  if (e->max_smem_set >= smem) return NGAP_OK;
  std::lock_guard<std::mutex> lock(g_smem_mu);
  const int dev = e->device & 63;
  if (g_smem_set[dev] >= smem) {
    e->max_smem_set = g_smem_set[dev];
    return NGAP_OK;
  }
  const void* kernels[6] = {(const void*)match_kernel<0, false>, (const void*)match_kernel<1, false>,
                            (const void*)match_kernel<2, false>, (const void*)match_kernel<0, true>,
                            (const void*)match_kernel<1, true>, (const void*)match_kernel<2, true>};
  cudaError_t ce = cudaSuccess;
  for (int k = 0; k < 6 && ce == cudaSuccess; k++)
    ce = cudaFuncSetAttribute(kernels[k], cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (ce != cudaSuccess) {
    set_error("shared memory request of %d bytes rejected: %s", smem, cudaGetErrorString(ce));
    return NGAP_E_CUDA;
  }
  g_smem_set[dev] = smem;
  e->max_smem_set = smem;
  return NGAP_OK;
}

template <int PRIV>
int blocks_per_sm(int smem, int* out) {
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, match_kernel<PRIV, false>, kCtaThreads,
                                                         smem));
  if (*out < 1) {
    set_error("the matching kernel does not fit on an SM with %d bytes of shared memory", smem);
    return NGAP_E_CUDA;
  }
  return NGAP_OK;
}

// blocks_per_sm of the engine's last shared-memory size per algorithm (the
// occupancy query costs a driver call on every match otherwise).
int cached_blocks_per_sm(ngap_engine* e, int priv, int smem, int* out) {
  if (e->bps_smem[priv] == smem) {
    *out = e->bps_val[priv];
    return NGAP_OK;
  }
  const int rc = priv == 0 ? blocks_per_sm<0>(smem, out)
                 : priv == 1 ? blocks_per_sm<1>(smem, out) : blocks_per_sm<2>(smem, out);
  if (rc == NGAP_OK) {
    e->bps_smem[priv] = smem;
    e->bps_val[priv] = *out;
  }
  return rc;
}

// One sort of report keys: d_in[0 .. *d_n) (clamped to cap) into unique
// reports at d_out (and stream indices at d_out_stream for MODE 1).
//   MODE 0: keys offset << 32 | id, written as id << 32 | offset;
//   MODE 1: keys stream << sshift | offset << oshift | id (batched matching).
// shifts: the 4-bit digits the radix pipeline sorts, least significant first.
struct SortJob {
  int mode;
  uint64_t* d_in;
  const unsigned long long* d_n;
  uint64_t cap;
  std::vector<int> shifts;
  int oshift, sshift;
  uint64_t* d_out;
  uint32_t* d_out_stream;
  unsigned long long* d_unique_n;
};

// The radix pipeline over *radix_n keys; kernels counts its launches.
int radix_chain(ngap_engine* e, const SortJob& j, const unsigned long long* radix_n,
                cudaStream_t st, int* kernels) {
  const uint32_t max_tiles = (uint32_t)((j.cap + kSortTile - 1) / kSortTile);
  const int grid = (int)std::max<uint32_t>(1, std::min<uint32_t>(max_tiles, e->num_sms * 8));
  // ping-pong between d_in (an engine-owned buffer) and d_tmp
  uint64_t* src = j.d_in;
  uint64_t* dst = e->d_tmp;
  int k = 0;
  for (int sh : j.shifts) {
    radix_hist<<<grid, kSortThreads, 0, st>>>(src, radix_n, j.cap, sh, e->d_hist);
    scan_exclusive_1block<<<1, kScanThreads, 0, st>>>(e->d_hist, radix_n, j.cap, 16, nullptr);
    radix_scatter<<<grid, kSortThreads, 0, st>>>(src, dst, radix_n, j.cap, sh, e->d_hist);
    k += 3;
    std::swap(src, dst);
  }
  unique_count<<<grid, kSortThreads, 0, st>>>(src, radix_n, j.cap, e->d_hist);
  scan_exclusive_1block<<<1, kScanThreads, 0, st>>>(e->d_hist, radix_n, j.cap, 1, j.d_unique_n);
  if (j.mode == 0)
    unique_write<<<grid, kSortThreads, 0, st>>>(src, radix_n, j.cap, e->d_hist, j.d_out);
  else
    unique_write_fields<<<grid, kSortThreads, 0, st>>>(src, radix_n, j.cap, e->d_hist, j.oshift,
                                                       j.sshift, j.d_out, j.d_out_stream);
  k += 3;
  *kernels = k;
  CUDA_TRY(cudaGetLastError());
  return NGAP_OK;
}

void* small_kernel(int mode) {
  return mode == 0 ? reinterpret_cast<void*>(small_sort_unique<0>)
                   : reinterpret_cast<void*>(small_sort_unique<1>);
}

// Builds the graph: the small-set kernel, then the radix pipeline in the body
// of a conditional (IF) node whose condition the small-set kernel sets when
// it leaves keys to the pipeline.
int build_sort_graph(ngap_engine* e, const SortJob& j, SortGraph& sg) {
  if (!e->sort_cs) CUDA_TRY(cudaStreamCreateWithFlags(&e->sort_cs, cudaStreamNonBlocking));
  CUDA_TRY(cudaGraphCreate(&sg.g, 0));
  cudaGraphConditionalHandle h = 0;
  CUDA_TRY(cudaGraphConditionalHandleCreate(&h, sg.g, 0, cudaGraphCondAssignDefault));
  unsigned long long* radix_n = e->d_counters + kRadixCount;
  uint64_t* d_in = j.d_in;
  const unsigned long long* d_n = j.d_n;
  uint64_t cap = j.cap;
  unsigned long long* d_unique_n = j.d_unique_n;
  int oshift = j.oshift, sshift = j.sshift;
  uint64_t* d_out = j.d_out;
  uint32_t* d_out_stream = j.d_out_stream;
  int set_cond = 1;
  void* args[] = {&d_in, &d_n, &cap, &radix_n, &d_unique_n, &oshift, &sshift, &d_out,
                  &d_out_stream, &h, &set_cond};
  cudaKernelNodeParams kp = {};
  kp.func = small_kernel(j.mode);
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(kSmallThreads);
  kp.sharedMemBytes = kSmallSortSmem;
  kp.kernelParams = args;
  cudaGraphNode_t kn = nullptr, cn = nullptr;
  CUDA_TRY(cudaGraphAddKernelNode(&kn, sg.g, nullptr, 0, &kp));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  CUDA_TRY(cudaGraphAddNode(&cn, sg.g, &kn, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  CUDA_TRY(cudaStreamBeginCaptureToGraph(e->sort_cs, body, nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal));
  int kernels = 0;
  const int rc = radix_chain(e, j, radix_n, e->sort_cs, &kernels);
  cudaGraph_t captured = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(e->sort_cs, &captured);
  if (rc != NGAP_OK) return rc;
  CUDA_TRY(ce);
  CUDA_TRY(cudaGraphInstantiate(&sg.ge, sg.g, 0));
  sg.chain = kernels;
  return NGAP_OK;
}

// Enqueues a sort on st. Outside stream capture it replays a cached graph
// (one launch; the radix pipeline runs only for more than kSmallSort keys);
// inside a capture, or where graphs are unavailable, it launches the small-set
// kernel and the pipeline, whose kernels find no keys after a small set.
int sort_reports(ngap_engine* e, const SortJob& j, cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CUDA_TRY(cudaStreamIsCapturing(st, &cs));
  if (cs == cudaStreamCaptureStatusNone && !e->sort_graph_off) {
    std::vector<uint64_t> key = {(uint64_t)j.mode,   (uint64_t)(uintptr_t)j.d_in,
                                 (uint64_t)(uintptr_t)j.d_n, j.cap,
                                 (uint64_t)j.oshift, (uint64_t)j.sshift,
                                 (uint64_t)(uintptr_t)j.d_out,
                                 (uint64_t)(uintptr_t)j.d_out_stream,
                                 (uint64_t)(uintptr_t)j.d_unique_n,
                                 (uint64_t)(uintptr_t)e->d_tmp, (uint64_t)(uintptr_t)e->d_hist};
    for (int sh : j.shifts) key.push_back((uint64_t)sh);
    SortGraph* sg = nullptr;
    for (auto& g : e->sort_graphs)
      if (g.key == key) sg = &g;
    if (!sg) {
      if (e->sort_graphs.size() >= 16) {  // keep a few configurations
        e->sort_graphs.front().release();
        e->sort_graphs.erase(e->sort_graphs.begin());
      }
      SortGraph ng;
      ng.key = key;
      if (build_sort_graph(e, j, ng) == NGAP_OK) {
        e->sort_graphs.push_back(ng);
        sg = &e->sort_graphs.back();
      } else {  // graphs unavailable here: launch the kernels directly from now on
        ng.release();
        cudaGetLastError();
        e->sort_graph_off = true;
      }
    }
    if (sg) {
      CUDA_TRY(cudaGraphLaunch(sg->ge, st));
      e->launches++;
      e->sort_chain_pending = sg->chain;
      return NGAP_OK;
    }
  }
  unsigned long long* radix_n = e->d_counters + kRadixCount;
  const cudaGraphConditionalHandle none = 0;
  const int set_cond = 0;
  if (j.mode == 0)
    small_sort_unique<0><<<1, kSmallThreads, kSmallSortSmem, st>>>(
        j.d_in, j.d_n, j.cap, radix_n, j.d_unique_n, j.oshift, j.sshift, j.d_out, j.d_out_stream,
        none, set_cond);
  else
    small_sort_unique<1><<<1, kSmallThreads, kSmallSortSmem, st>>>(
        j.d_in, j.d_n, j.cap, radix_n, j.d_unique_n, j.oshift, j.sshift, j.d_out, j.d_out_stream,
        none, set_cond);
  int kernels = 0;
  const int rc = radix_chain(e, j, radix_n, st, &kernels);
  e->launches += 1 + kernels;
  return rc;
}

// Sorts d_in[0 .. *d_n) (clamped to cap) into d_out as unique reference-encoded
// reports; *d_unique_n receives the count. off_bits / id_bits bound the key.
int sort_unique(ngap_engine* e, uint64_t* d_in, const unsigned long long* d_n, uint64_t cap,
                int off_bits, int id_bits, uint64_t* d_out, unsigned long long* d_unique_n,
                cudaStream_t st) {
  SortJob j{0, d_in, d_n, cap, {}, 32, 64, d_out, nullptr, d_unique_n};
  for (int b = 0; b < id_bits; b += 4) j.shifts.push_back(b);
  for (int b = 0; b < off_bits; b += 4) j.shifts.push_back(32 + b);
  return sort_reports(e, j, st);
}

// Batched keys stream << sshift | offset << oshift | id: radix passes over the
// three fields, then unique reports and their stream indices.
int sort_unique_fields(ngap_engine* e, const unsigned long long* d_n, uint64_t cap, int ibits,
                       int oshift, int obits, int sshift, int sbits,
                       unsigned long long* d_unique_n, cudaStream_t st) {
  SortJob j{1, e->d_reports, d_n, cap, {}, oshift, sshift, e->d_unique, e->d_stream_ids,
            d_unique_n};
  for (int b = 0; b < ibits; b += 4) j.shifts.push_back(b);
  for (int b = 0; b < obits; b += 4) j.shifts.push_back(oshift + b);
  for (int b = 0; b < sbits; b += 4) j.shifts.push_back(sshift + b);
  return sort_reports(e, j, st);
}

// --algorithm -> prefix depth, privatization and window.
int algo_config(int algo, int table_depth, int* depth, int* priv, int* window) {
  switch (algo) {
    case NGAP_ALGO_BLOCKING: *depth = 0; *window = 1; break;
    case NGAP_ALGO_NAP: *depth = 0; break;
    case NGAP_ALGO_NONBLOCKING: *depth = 1; break;
    case NGAP_ALGO_NONBLOCKING_R1: *depth = 1; *priv = 1; break;
    case NGAP_ALGO_NONBLOCKING_R2: *depth = 1; *priv = 2; break;
    case NGAP_ALGO_NONBLOCKING_PC: *depth = std::max(1, table_depth); break;
    case NGAP_ALGO_NONBLOCKING_ALL: *depth = std::max(1, table_depth); *priv = 1; break;
    default:
      set_error("not supported algoritm %d", algo);
      return NGAP_E_INVALID;
  }
  return NGAP_OK;
}

}  // namespace

extern "C" {

int ngap_match(ngap_engine* e, const ngap_tables* t, const uint8_t* input, int input_on_device,
               const ngap_match_params* p, void* stream) {
  if (!e || !t || !p) {
    set_error("ngap_match: null argument");
    return NGAP_E_INVALID;
  }
  if (p->num_seg <= 0 || p->seg_len <= 0) {
    set_error("ngap_match: num_seg and seg_len must be positive");
    return NGAP_E_INVALID;
  }
  if (!input) {
    set_error("ngap_match: null argument (input)");
    return NGAP_E_INVALID;
  }
  // each factor below 2^32 first, so that the product cannot wrap
  const uint64_t total = p->num_seg < (1ll << 32) && p->seg_len < (1ll << 32)
                             ? (uint64_t)p->num_seg * (uint64_t)p->seg_len
                             : ~0ull;
  if (total >= (1ull << 32)) {
    set_error("ngap_match: input of %llu bytes exceeds the 32-bit offsets of the report format",
              (unsigned long long)total);
    return NGAP_E_UNSUPPORTED;
  }
  if (t->num_groups > 1024) {
    set_error("ngap_match: at most 1024 groups fit the 32-bit report id");
    return NGAP_E_UNSUPPORTED;
  }
  CUDA_TRY(cudaSetDevice(e->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  e->stream = st;
  e->launches = 0;
  e->sort_chain_pending = 0;
  e->ran = false;
  int algo = p->algorithm;
  // automatic window: 2048 positions (against 1024: Hamming set 0.654 ->
  // 0.624 ms, high_frontier and the literal set 1-2 % faster; shortened
  // below when the shared memory of the warps and a staged image does not fit)
  int depth = 1, priv = 0, window = p->window > 0 ? p->window : 2048;
  int table_depth = 0;
  for (auto& th : t->tiles) table_depth = std::max(table_depth, th.depth);
  switch (algo) {
    case NGAP_ALGO_BLOCKING: depth = 0; window = 1; break;
    case NGAP_ALGO_NAP: depth = 0; break;
    case NGAP_ALGO_NONBLOCKING: depth = 1; break;
    case NGAP_ALGO_NONBLOCKING_R1: depth = 1; priv = 1; break;
    case NGAP_ALGO_NONBLOCKING_R2: depth = 1; priv = 2; break;
    case NGAP_ALGO_NONBLOCKING_PC: depth = std::max(1, table_depth); break;
    case NGAP_ALGO_NONBLOCKING_ALL: depth = std::max(1, table_depth); priv = 1; break;
    default:
      set_error("not supported algoritm %d", algo);
      return NGAP_E_INVALID;
  }
  window = std::min(window, kMaxWindow);
  // input: own 16-byte-aligned, padded copy
  size_t need = ((total + 15) & ~(uint64_t)15) + 64;
  if (need > e->input_cap) {
    cudaFree(e->d_input);
    e->d_input = nullptr;
    e->input_cap = 0;
    CUDA_TRY(cudaMalloc(&e->d_input, need));
    e->input_cap = need;
  }
  uint64_t cap = p->result_capacity > 0 ? p->result_capacity : 54619400ull;
  int rc = ensure_reports(e, cap);
  if (rc != NGAP_OK) return rc;
  // shared memory: the largest tile image that fits the budget, plus the warps
  // (a window too large for what is left is shortened)
  while (window > 64 && cta_smem_bytes(window, t->image_region) > 227 * 1024 - 1024) window /= 2;
  const int smem = cta_smem_bytes(window, t->image_region);
  if ((rc = set_smem(e, smem)) != NGAP_OK) return rc;
  int bps = 0;
  rc = cached_blocks_per_sm(e, priv, smem, &bps);
  if (rc != NGAP_OK) return rc;
  const int full_grid = e->num_sms * bps;
  // units and tasks
  UnitPlanKey key{p->num_seg, p->seg_len, p->is_dup ? 1 : 0, window, p->chunk, p->first_segment};
  if (e->plan_tables != t->serial || key < e->plan_key || e->plan_key < key) {
    std::vector<UnitDev> units;
    std::vector<TaskDev> tasks;
    int32_t ntasks1 = 0, ntasks2 = 0;
    const ActRows rows = plan_units(t, key, full_grid, units, tasks, &ntasks1, &ntasks2,
                                    e->free_range, e->free_tile);
    e->ntasks1 = ntasks1;
    e->ntasks2 = ntasks2;
    std::vector<Upload> ups;
    if ((rc = set_act_rows(e, rows, ups)) != NGAP_OK) return rc;
    if (units.size() > e->units_cap) {
      const size_t cap = grown(e->units_cap, units.size());
      cudaFree(e->d_units);
      e->d_units = nullptr;
      e->units_cap = 0;
      CUDA_TRY(cudaMalloc(&e->d_units, cap * sizeof(UnitDev)));
      e->units_cap = cap;
    }
    if (tasks.size() > e->tasks_cap) {
      const size_t cap = grown(e->tasks_cap, tasks.size());
      cudaFree(e->d_tasks);
      e->d_tasks = nullptr;
      e->tasks_cap = 0;
      CUDA_TRY(cudaMalloc(&e->d_tasks, cap * sizeof(TaskDev)));
      e->tasks_cap = cap;
    }
    if (!units.empty()) ups.push_back({e->d_units, units.data(), units.size() * sizeof(UnitDev)});
    if (!tasks.empty()) ups.push_back({e->d_tasks, tasks.data(), tasks.size() * sizeof(TaskDev)});
    if ((rc = upload_plan(e, st, ups)) != NGAP_OK) return rc;
    e->nunits = (int32_t)units.size();
    e->h_units = units;
    e->ntasks = (int32_t)tasks.size();
    e->plan_tables = t->serial;
    e->plan_key = key;
    e->batch_ts = 0;  // the batched plan cache no longer describes the buffers
  }
  const int grid = plan_grid(e, full_grid);
  e->grid = grid;
  // per-warp scratch for the full grid, whatever this plan uses: a later
  // larger plan then never reallocates (cudaMalloc waits for the device)
  rc = ensure_slots(e, (size_t)full_grid * kWarpsPerCta, t->max_states, t->max_nact, kDefaultQueue);
  if (rc != NGAP_OK) return rc;

  CUDA_TRY(cudaEventRecord(e->ev[0], st));
  if (input_on_device)
    CUDA_TRY(cudaMemcpyAsync(e->d_input, input, total, cudaMemcpyDeviceToDevice, st));
  else
    CUDA_TRY(cudaMemcpyAsync(e->d_input, input, total, cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemsetAsync(e->d_counters, 0, 8 * sizeof(unsigned long long), st));
  CUDA_TRY(cudaMemsetAsync(e->d_err, 0, sizeof(int), st));

  MatchParams mp;
  mp.tiles = t->d_tiles;
  mp.units = e->d_units;
  mp.tasks = e->d_tasks;
  mp.ntasks = e->ntasks;
  mp.image_region = t->image_region;
  mp.input = e->d_input;
  mp.window = window;
  mp.depth = depth;
  mp.active_threshold = p->active_threshold;
  mp.unique = p->unique;
  mp.report_off = p->report_off;
  mp.off_shift = 32;
  mp.rep_count = e->d_counters + 0;
  mp.reports = e->d_reports;
  mp.rep_cap = cap;
  mp.err = e->d_err;
  mp.task_counter = e->d_unit_counter;
  mp.carry = e->d_carry;
  mp.marks = e->d_marks;
  mp.ovf = e->d_ovf;
  mp.carry_cap = e->carry_cap;
  mp.mark_words = e->mark_words;
  mp.ovf_cap = e->ovf_cap;
  mp.work = e->d_counters + 2;
  mp.act = e->d_act;
  mp.act_list = e->d_act_list;
  mp.act_cnt = e->d_act_cnt;
  mp.stk_g = e->d_stk;
  mp.stk_g_cap = e->stk_cap;
  mp.wait_rounds = e->test_wait_rounds > 0 ? e->test_wait_rounds : kWaitRounds;
  mp.skip_copy_unit = e->test_skip_unit;
  e->test_wait_rounds = 0;  // the hook covers one match
  e->test_skip_unit = -1;
  if ((rc = trace_buffer(e, st, &mp.unit_work, &mp.unit_cycles)) != NGAP_OK) return rc;
  e->trace_seg_len = p->seg_len;
  CUDA_TRY(cudaEventRecord(e->ev[1], st));
  if (e->ntasks > 0 || e->free_range[1] > 0 || e->free_range[3] > 0 || e->free_range[5] > 0) {
    rc = launch_any(e, mp, smem, st, priv);
    if (rc != NGAP_OK) return rc;
  }
  CUDA_TRY(cudaEventRecord(e->ev[2], st));
  if (!p->report_off) {
    int off_bits = bits_for(total);
    int id_bits = 22 + bits_for((uint64_t)std::max(t->num_groups, 1));
    rc = sort_unique(e, e->d_reports, e->d_counters + 0, cap, off_bits, id_bits, e->d_unique,
                     e->d_counters + 1, st);
    if (rc != NGAP_OK) return rc;
  }
  CUDA_TRY(cudaEventRecord(e->ev[3], st));
  CUDA_TRY(cudaMemcpyAsync(e->h_counters, e->d_counters, 4 * sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaMemcpyAsync(e->h_counters + 4, e->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaMemcpyAsync(e->h_counters + kRadixCount, e->d_counters + kRadixCount,
                           sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  e->ran = true;
  return NGAP_OK;
}

int ngap_engine_sync(ngap_engine* e) {
  if (!e || !e->ran) {
    set_error("ngap_engine_sync: no match in flight");
    return NGAP_E_INVALID;
  }
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  CUDA_TRY(cudaEventElapsedTime(&e->match_ms, e->ev[1], e->ev[2]));
  CUDA_TRY(cudaEventElapsedTime(&e->sort_ms, e->ev[2], e->ev[3]));
  if (e->sort_chain_pending > 0 && e->h_counters[kRadixCount] > 0)  // the radix pipeline ran
    e->launches += e->sort_chain_pending;
  e->sort_chain_pending = 0;
  int err = (int)(e->h_counters[4] & 0xffffffffull);
  if (err & kErrTimeout) {
    set_error("a bounded device wait gave up; results are incomplete");
    return NGAP_E_TIMEOUT;
  }
  if (err & (kErrQueue | kErrCarry)) {
    set_error("a worklist overflowed its capacity; results are incomplete");
    return NGAP_E_OVERFLOW_QUEUE;
  }
  if (err & kErrResults) {
    set_error("%llu reports exceed the result capacity of %llu; results are truncated",
              (unsigned long long)e->h_counters[0], (unsigned long long)e->rep_cap);
    return NGAP_E_OVERFLOW_RESULTS;
  }
  return NGAP_OK;
}

int ngap_results_count(const ngap_engine* e, uint64_t* raw, uint64_t* unique) {
  if (!e) return NGAP_E_INVALID;
  if (raw) *raw = e->h_counters[0];
  if (unique) *unique = e->h_counters[1];
  return NGAP_OK;
}

const uint64_t* ngap_results_device(const ngap_engine* e) { return e ? e->d_unique : nullptr; }

int64_t ngap_results_copy(ngap_engine* e, uint64_t* host, uint64_t cap) {
  if (!e || !host) return -1;
  uint64_t n = std::min<uint64_t>(e->h_counters[1], cap);
  if (n == 0) return 0;
  if (cudaSetDevice(e->device) != cudaSuccess) return -1;
  cudaError_t ce = cudaMemcpy(host, e->d_unique, n * sizeof(uint64_t), cudaMemcpyDeviceToHost);
  if (ce != cudaSuccess) {
    set_error("cudaMemcpy: %s", cudaGetErrorString(ce));
    return -1;
  }
  return (int64_t)n;
}

int ngap_last_times_ms(const ngap_engine* e, float* match_ms, float* sort_ms) {
  if (!e) return NGAP_E_INVALID;
  if (match_ms) *match_ms = e->match_ms;
  if (sort_ms) *sort_ms = e->sort_ms;
  return NGAP_OK;
}

int ngap_last_launches(const ngap_engine* e) { return e ? e->launches : 0; }

int ngap_engine_work(const ngap_engine* e, uint64_t* expanded, uint64_t* injected) {
  if (!e) return NGAP_E_INVALID;
  if (expanded) *expanded = e->h_counters[2];
  if (injected) *injected = e->h_counters[3];
  return NGAP_OK;
}

int ngap_engine_memory(const ngap_engine* e, ngap_engine_mem* out) {
  if (!e || !out) {
    set_error("ngap_engine_memory: null argument");
    return NGAP_E_INVALID;
  }
  out->input = (int64_t)e->input_cap;
  out->reports = 3 * 8 * (int64_t)e->rep_cap + 4 * (int64_t)e->hist_cap + 4 * (int64_t)e->stream_ids_cap;
  out->scratch =
      (int64_t)e->slots * 4 * ((int64_t)e->carry_cap + e->mark_words + e->ovf_cap + 2 * e->stk_cap);
  out->plan = 8 * (int64_t)e->act_cap + 16 * (int64_t)e->rows_cap + 16 * (int64_t)e->unit_work_cap +
              (int64_t)sizeof(UnitDev) * (int64_t)e->units_cap +
              (int64_t)sizeof(TaskDev) * (int64_t)e->tasks_cap;
  return NGAP_OK;
}

int64_t ngap_engine_device_bytes(const ngap_engine* e) {
  ngap_engine_mem m;
  if (ngap_engine_memory(e, &m) != NGAP_OK) return 0;
  return m.input + m.reports + m.scratch + m.plan;
}

int ngap_engine_test_wait_timeout(ngap_engine* e, int32_t unit, int32_t wait_rounds) {
  if (!e || unit < 0 || wait_rounds < 1) {
    set_error("ngap_engine_test_wait_timeout: needs an engine, a unit >= 0 and wait_rounds >= 1");
    return NGAP_E_INVALID;
  }
  e->test_skip_unit = unit;
  e->test_wait_rounds = wait_rounds;
  return NGAP_OK;
}

int ngap_engine_set_trace(ngap_engine* e, int enable) {
  if (!e) {
    set_error("ngap_engine_set_trace: null engine");
    return NGAP_E_INVALID;
  }
  e->trace = enable != 0;
  return NGAP_OK;
}

int ngap_trace_copy(ngap_engine* e, ngap_unit_trace* out, int64_t cap, int64_t* n) {
  if (!e || !n) {
    set_error("ngap_trace_copy: bad argument");
    return NGAP_E_INVALID;
  }
  *n = 0;
  if (!e->trace || !e->ran || e->nunits == 0 || !e->d_unit_work) return NGAP_OK;
  if (!out) {  // count query
    *n = e->nunits;
    return NGAP_OK;
  }
  std::vector<unsigned long long> work(e->nunits), cycles(e->nunits);
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  CUDA_TRY(cudaMemcpy(work.data(), e->d_unit_work, work.size() * sizeof(unsigned long long),
                      cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(cycles.data(), e->d_unit_work + e->unit_work_cap,
                      cycles.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  const int64_t m = std::min<int64_t>(cap, e->nunits);
  for (int64_t i = 0; i < m; i++) {
    const UnitDev& u = e->h_units[i];
    const int64_t base = e->trace_seg_len > 0 ? (int64_t)u.stream * e->trace_seg_len : u.base;
    out[i].stream = u.stream;
    out[i].tile = u.tile;
    out[i].lo = u.emit_lo - base;
    out[i].hi = u.hi - base;
    out[i].work = work[i];
    out[i].cycles = cycles[i];
  }
  *n = m;
  return NGAP_OK;
}

int ngap_tables_stats_get(const ngap_tables* t, ngap_tables_stats* out) {
  if (!t || !out) {
    set_error("ngap_tables_stats_get: null argument");
    return NGAP_E_INVALID;
  }
  ngap_tables_stats st{};
  st.tiles = (int32_t)t->tiles.size();
  for (const TileHost& th : t->tiles) {
    if (th.phase == 1) continue;  // activation tiles repeat states of their layered pair
    st.states += th.nstates;
    for (uint32_t u : th.succ) st.edges += u != kNoSucc ? 1 : 0;
    st.aas += (int32_t)th.aas.size();
    st.depth = std::max(st.depth, th.depth);
    st.max_nlive = std::max(st.max_nlive, th.nlive);
    const PrefixTableHost& pt = th.pt[th.depth - 1];
    st.list_entries += pt.entries;
    st.cutoff += pt.cutoff;
    double space = 1.0;
    for (int d = 0; d < th.depth; d++) space *= (double)std::max(1, th.nlive);
    st.exp_list += (double)pt.entries / space;
    st.max_list = std::max<int32_t>(st.max_list, pt.max_len);
  }
  *out = st;
  return NGAP_OK;
}

int ngap_reports_sort_unique(ngap_engine* e, const uint64_t* d_in, uint64_t n, uint64_t* d_out,
                             uint64_t* n_out, void* stream) {
  if (!e || (!d_in && n) || !d_out || !n_out) {
    set_error("ngap_reports_sort_unique: null argument");
    return NGAP_E_INVALID;
  }
  CUDA_TRY(cudaSetDevice(e->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  *n_out = 0;
  if (n == 0) return NGAP_OK;
  int rc = ensure_reports(e, n);
  if (rc != NGAP_OK) return rc;
  // input arrives in the reference encoding (id << 32 | offset): swap halves
  // into sort keys in the engine's report buffer
  CUDA_TRY(cudaMemcpyAsync(e->d_reports, d_in, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
  unsigned long long hn = n;
  CUDA_TRY(cudaMemcpyAsync(e->d_counters + 5, &hn, sizeof(hn), cudaMemcpyHostToDevice, st));
  swap_halves<<<std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 4096)), 256, 0, st>>>(e->d_reports, n);
  CUDA_TRY(cudaGetLastError());
  rc = sort_unique(e, e->d_reports, e->d_counters + 5, n, 32, 32, d_out, e->d_counters + 6, st);
  if (rc != NGAP_OK) return rc;
  unsigned long long un = 0;
  CUDA_TRY(cudaMemcpyAsync(&un, e->d_counters + 6, sizeof(un), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  *n_out = un;
  return NGAP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched matching: many streams, several NFAs, one persistent launch.
// ---------------------------------------------------------------------------

struct ngap_tableset {
  uint64_t serial = g_next_serial.fetch_add(1);
  std::vector<const ngap_tables*> tables;
  std::vector<int> tile_base;  // first tile of each NFA in the combined descriptor array
  TileDev* d_tiles = nullptr;
  int ntiles = 0, image_region = 0, max_states = 0, max_groups = 1, max_depth = 1, device = 0;
  int max_nact = 0;
  std::vector<int32_t> plan_bytes;  // per tile of the combined array (planning size)
  std::vector<char> tile_lean;      // per tile of the combined array (ngap_tables::tile_lean)
  ~ngap_tableset() { cudaFree(d_tiles); }
};

extern "C" {

int ngap_tableset_create(const ngap_tables* const* tables, int n, ngap_tableset** out) {
  if (!tables || n <= 0 || !out) {
    set_error("ngap_tableset_create: bad argument");
    return NGAP_E_INVALID;
  }
  *out = nullptr;
  std::unique_ptr<ngap_tableset> ts(new ngap_tableset());
  std::vector<TileDev> all;
  for (int i = 0; i < n; i++) {
    const ngap_tables* t = tables[i];
    if (!t || (i > 0 && t->device != tables[0]->device)) {
      set_error("ngap_tableset_create: tables must exist and share one device");
      return NGAP_E_INVALID;
    }
    ts->tables.push_back(t);
    ts->tile_base.push_back((int)all.size());
    all.insert(all.end(), t->dev_desc.begin(), t->dev_desc.end());
    ts->plan_bytes.insert(ts->plan_bytes.end(), t->plan_bytes.begin(), t->plan_bytes.end());
    ts->tile_lean.insert(ts->tile_lean.end(), t->tile_lean.begin(), t->tile_lean.end());
    ts->image_region = std::max(ts->image_region, t->image_region);
    ts->max_states = std::max(ts->max_states, t->max_states);
    ts->max_groups = std::max(ts->max_groups, t->num_groups);
    ts->max_nact = std::max(ts->max_nact, t->max_nact);
    for (auto& th : t->tiles) ts->max_depth = std::max(ts->max_depth, th.depth);
  }
  ts->device = tables[0]->device;
  ts->ntiles = (int)all.size();
  CUDA_TRY(cudaSetDevice(ts->device));
  if (!all.empty()) {
    CUDA_TRY(cudaMalloc(&ts->d_tiles, all.size() * sizeof(TileDev)));
    CUDA_TRY(cudaMemcpy(ts->d_tiles, all.data(), all.size() * sizeof(TileDev),
                        cudaMemcpyHostToDevice));
  }
  *out = ts.release();
  return NGAP_OK;
}

void ngap_tableset_destroy(ngap_tableset* ts) { delete ts; }

int ngap_batch_match(ngap_engine* e, const ngap_tableset* ts, const uint8_t* input,
                     uint64_t input_bytes, int input_on_device, const ngap_batch_stream* streams,
                     int nstreams, const ngap_batch_params* p, void* stream) {
  if (!e || !ts || !p || !streams || nstreams <= 0 || (!input && input_bytes > 0)) {
    set_error("ngap_batch_match: bad argument");
    return NGAP_E_INVALID;
  }
  uint64_t max_len = 1;
  for (int i = 0; i < nstreams; i++) {
    const ngap_batch_stream& s = streams[i];
    if (s.nfa < 0 || s.nfa >= (int)ts->tables.size() || s.offset > input_bytes ||
        s.length > input_bytes - s.offset) {  // no wrap-around of offset + length
      set_error("ngap_batch_match: stream %d is out of range", i);
      return NGAP_E_INVALID;
    }
    max_len = std::max<uint64_t>(max_len, s.length + 1);
  }
  if (input_bytes >= (1ull << 32)) {
    set_error("ngap_batch_match: batches are limited to 4 GiB of input");
    return NGAP_E_UNSUPPORTED;
  }
  // report key: stream | offset in stream | id
  const int ibits = 22 + bits_for((uint64_t)std::max(ts->max_groups, 1));
  int obits = bits_for(max_len);
  int sbits = bits_for((uint64_t)nstreams);
  // field widths rounded up to the radix digit (4 bits) when the key still
  // fits: the same number of radix passes and far fewer distinct layouts, so
  // that the sort's CUDA graph (keyed by the layout) is reused across batches
  // of other lengths and stream counts instead of being captured again
  if (ibits + ((obits + 3) & ~3) + ((sbits + 3) & ~3) <= 64) {
    obits = (obits + 3) & ~3;
    sbits = (sbits + 3) & ~3;
  }
  const int oshift = ibits, sshift = ibits + obits;
  if (sshift + sbits > 64) {
    set_error("ngap_batch_match: stream count, stream length and group count exceed a 64-bit key");
    return NGAP_E_UNSUPPORTED;
  }
  CUDA_TRY(cudaSetDevice(e->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  e->stream = st;
  e->ran = false;
  // automatic window: 2048 positions (against 1024: Hamming set 0.654 ->
  // 0.624 ms, high_frontier and the literal set 1-2 % faster; shortened
  // below when the shared memory of the warps and a staged image does not fit)
  int depth = 1, priv = 0, window = p->window > 0 ? p->window : 2048;
  int rc = algo_config(p->algorithm, ts->max_depth, &depth, &priv, &window);
  if (rc != NGAP_OK) return rc;
  window = std::min(window, kMaxWindow);
  while (window > 64 && cta_smem_bytes(window, ts->image_region) > 227 * 1024 - 1024) window /= 2;
  const int smem = cta_smem_bytes(window, ts->image_region);
  if ((rc = set_smem(e, smem)) != NGAP_OK) return rc;
  int bps = 0;
  rc = cached_blocks_per_sm(e, priv, smem, &bps);
  if (rc != NGAP_OK) return rc;
  const int full_grid = e->num_sms * bps;
  // buffers (before any capture)
  size_t need = ((input_bytes + 15) & ~(uint64_t)15) + 64;
  if (need > e->input_cap) {
    cudaFree(e->d_input);
    e->d_input = nullptr;
    e->input_cap = 0;
    CUDA_TRY(cudaMalloc(&e->d_input, need));
    e->input_cap = need;
  }
  const uint64_t cap = p->result_capacity > 0 ? p->result_capacity : 54619400ull;
  if ((rc = ensure_reports(e, cap)) != NGAP_OK) return rc;
  if (cap > e->stream_ids_cap) {
    cudaFree(e->d_stream_ids);
    e->d_stream_ids = nullptr;
    e->stream_ids_cap = 0;
    CUDA_TRY(cudaMalloc(&e->d_stream_ids, cap * sizeof(uint32_t)));
    e->stream_ids_cap = cap;
  }
  // plan: tiles outer (tasks share a staged image), streams of the tile's NFA inner
  const std::vector<ngap_batch_stream> sv(streams, streams + nstreams);
  auto same_streams = [&]() {
    if (e->batch_streams.size() != sv.size()) return false;
    for (size_t i = 0; i < sv.size(); i++)
      if (sv[i].offset != e->batch_streams[i].offset || sv[i].length != e->batch_streams[i].length ||
          sv[i].nfa != e->batch_streams[i].nfa || sv[i].chunk != e->batch_streams[i].chunk)
        return false;
    return true;
  };
  bool replanned = false;
  if (e->batch_ts != ts->serial || e->batch_window != window || e->batch_chunk != p->chunk ||
      !same_streams() || e->plan_tables != 0) {
    std::vector<std::vector<int>> by_nfa(ts->tables.size());
    for (int i = 0; i < nstreams; i++) by_nfa[sv[i].nfa].push_back(i);
    std::vector<UnitDev> pass1, unbounded, bounded, units;
    std::vector<TaskDev> tasks;
    const ActRows rows(ts->tables, nstreams);
    for (size_t n = 0; n < ts->tables.size(); n++) {
      const ngap_tables* t = ts->tables[n];
      for (int ti = 0; ti < (int)t->tiles.size(); ti++)
        for (int si : by_nfa[n]) {
          const ngap_batch_stream& s = sv[si];
          if (s.length == 0) continue;
          SegSpec sp{(int64_t)s.offset, (int64_t)(s.offset + s.length), true,
                     (uint64_t)si << sshift, (int64_t)s.offset, si};
          add_units(t->tiles[ti], ts->tile_base[n] + ti, sp, window,
                    s.chunk > 0 ? s.chunk : p->chunk, rows.row((int)n, t->tiles[ti], si), pass1,
                    unbounded, bounded);
        }
    }
    const int32_t region = ts->image_region;
    auto is_free = [&](int tile) { return ts->plan_bytes[tile] > region; };
    auto is_lean = [&](int tile) { return ts->tile_lean[tile] != 0; };
    make_tasks(units, pass1, unbounded, bounded, full_grid, is_free, is_lean, tasks, &e->ntasks1,
               &e->ntasks2, e->free_range, e->free_tile);
    std::vector<Upload> ups;
    if ((rc = set_act_rows(e, rows, ups)) != NGAP_OK) return rc;
    if (units.size() > e->units_cap) {
      const size_t cap = grown(e->units_cap, units.size());
      cudaFree(e->d_units);
      e->d_units = nullptr;
      e->units_cap = 0;
      CUDA_TRY(cudaMalloc(&e->d_units, cap * sizeof(UnitDev)));
      e->units_cap = cap;
    }
    if (tasks.size() > e->tasks_cap) {
      const size_t cap = grown(e->tasks_cap, tasks.size());
      cudaFree(e->d_tasks);
      e->d_tasks = nullptr;
      e->tasks_cap = 0;
      CUDA_TRY(cudaMalloc(&e->d_tasks, cap * sizeof(TaskDev)));
      e->tasks_cap = cap;
    }
    if (!units.empty()) ups.push_back({e->d_units, units.data(), units.size() * sizeof(UnitDev)});
    if (!tasks.empty()) ups.push_back({e->d_tasks, tasks.data(), tasks.size() * sizeof(TaskDev)});
    if ((rc = upload_plan(e, st, ups)) != NGAP_OK) return rc;
    e->nunits = (int32_t)units.size();
    e->h_units = units;
    e->ntasks = (int32_t)tasks.size();
    e->plan_tables = 0;  // the plain plan cache no longer describes the buffers
    e->plan_key = UnitPlanKey{-1, -1, -1, -1, -1, -1};
    e->batch_ts = ts->serial;
    e->batch_streams = sv;
    e->batch_window = window;
    e->batch_chunk = p->chunk;
    replanned = true;
  }
  const int grid = plan_grid(e, full_grid);
  e->grid = grid;
  if ((rc = ensure_slots(e, (size_t)full_grid * kWarpsPerCta, ts->max_states, ts->max_nact,
                         p->queue_capacity > 0 ? std::max(p->queue_capacity, 1024) : kDefaultQueue)) != NGAP_OK)
    return rc;

  MatchParams mp;
  mp.tiles = ts->d_tiles;
  mp.units = e->d_units;
  mp.tasks = e->d_tasks;
  mp.ntasks = e->ntasks;
  mp.image_region = ts->image_region;
  mp.input = e->d_input;
  mp.window = window;
  mp.depth = depth;
  mp.active_threshold = p->active_threshold;
  mp.unique = p->unique;
  mp.report_off = p->report_off;
  mp.off_shift = oshift;
  mp.rep_count = e->d_counters + 0;
  mp.reports = e->d_reports;
  mp.rep_cap = cap;
  mp.err = e->d_err;
  mp.task_counter = e->d_unit_counter;
  mp.carry = e->d_carry;
  mp.marks = e->d_marks;
  mp.ovf = e->d_ovf;
  mp.carry_cap = e->carry_cap;
  mp.mark_words = e->mark_words;
  mp.ovf_cap = e->ovf_cap;
  mp.work = e->d_counters + 2;
  mp.act = e->d_act;
  mp.act_list = e->d_act_list;
  mp.act_cnt = e->d_act_cnt;
  mp.stk_g = e->d_stk;
  mp.stk_g_cap = e->stk_cap;
  mp.unit_work = mp.unit_cycles = nullptr;
  mp.wait_rounds = kWaitRounds;
  mp.skip_copy_unit = -1;
  e->trace_seg_len = 0;

  auto enqueue = [&](cudaStream_t qs) -> int {
    if (e->trace) {
      const int r = trace_buffer(e, qs, &mp.unit_work, &mp.unit_cycles);
      if (r != NGAP_OK) return r;
    }
    if (input_on_device)
      CUDA_TRY(cudaMemcpyAsync(e->d_input, input, input_bytes, cudaMemcpyDeviceToDevice, qs));
    else
      CUDA_TRY(cudaMemcpyAsync(e->d_input, input, input_bytes, cudaMemcpyHostToDevice, qs));
    CUDA_TRY(cudaMemsetAsync(e->d_counters, 0, 8 * sizeof(unsigned long long), qs));
    CUDA_TRY(cudaMemsetAsync(e->d_err, 0, sizeof(int), qs));
    int r = NGAP_OK;
    if (e->ntasks > 0 || e->free_range[1] > 0 || e->free_range[3] > 0 || e->free_range[5] > 0) {
      r = launch_any(e, mp, smem, qs, priv);
      if (r != NGAP_OK) return r;
    }
    if (!p->report_off) {
      r = sort_unique_fields(e, e->d_counters + 0, cap, ibits, oshift, obits, sshift, sbits,
                             e->d_counters + 1, qs);
      if (r != NGAP_OK) return r;
    }
    CUDA_TRY(cudaMemcpyAsync(e->h_counters, e->d_counters, 4 * sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, qs));
    CUDA_TRY(cudaMemcpyAsync(e->h_counters + 4, e->d_err, sizeof(int), cudaMemcpyDeviceToHost, qs));
    CUDA_TRY(cudaMemcpyAsync(e->h_counters + kRadixCount, e->d_counters + kRadixCount,
                             sizeof(unsigned long long), cudaMemcpyDeviceToHost, qs));
    return NGAP_OK;
  };

  e->launches = 0;
  e->sort_chain_pending = 0;
  if (!p->use_graph) {
    e->graph_mode = false;
    CUDA_TRY(cudaEventRecord(e->ev[0], st));
    CUDA_TRY(cudaEventRecord(e->ev[1], st));
    if ((rc = enqueue(st)) != NGAP_OK) return rc;
    CUDA_TRY(cudaEventRecord(e->ev[2], st));
    CUDA_TRY(cudaEventRecord(e->ev[3], st));
    e->ran = true;
    return NGAP_OK;
  }
  // CUDA graph: the same tableset, streams, parameters and input pointer replay
  // one captured pipeline (copy, match, sort, unique, counters). Capture and
  // replay use the engine's own stream (the legacy default stream cannot be
  // captured), ordered after and before the caller's stream by events.
  if (!e->cap_stream) {
    CUDA_TRY(cudaStreamCreateWithFlags(&e->cap_stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&e->cap_ev[0], cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&e->cap_ev[1], cudaEventDisableTiming));
  }
  cudaStream_t cs = e->cap_stream;
  std::vector<uint64_t> key = {ts->serial, (uint64_t)(uintptr_t)input, input_bytes,
                               (uint64_t)input_on_device, (uint64_t)p->algorithm,
                               (uint64_t)p->unique, (uint64_t)p->active_threshold,
                               (uint64_t)p->report_off, cap, (uint64_t)window, (uint64_t)p->chunk,
                               (uint64_t)e->trace, (uint64_t)e->ovf_cap};
  if (replanned || !e->graph || key != e->graph_key) {
    if (e->graph) {
      cudaGraphExecDestroy(e->graph);
      e->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    rc = enqueue(cs);
    cudaError_t ce = cudaStreamEndCapture(cs, &g);
    if (rc != NGAP_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ce != cudaSuccess) {
      set_error("CUDA graph capture failed: %s", cudaGetErrorString(ce));
      return NGAP_E_CUDA;
    }
    ce = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
      e->graph = nullptr;
      set_error("CUDA graph instantiation failed: %s", cudaGetErrorString(ce));
      return NGAP_E_CUDA;
    }
    e->graph_key = key;
    e->graph_launches = e->launches;
  }
  e->graph_mode = true;
  e->launches = e->graph_launches;
  CUDA_TRY(cudaEventRecord(e->cap_ev[0], st));  // after the caller's prior work
  CUDA_TRY(cudaStreamWaitEvent(cs, e->cap_ev[0], 0));
  CUDA_TRY(cudaEventRecord(e->ev[0], cs));
  CUDA_TRY(cudaEventRecord(e->ev[1], cs));
  CUDA_TRY(cudaGraphLaunch(e->graph, cs));
  CUDA_TRY(cudaEventRecord(e->ev[2], cs));
  CUDA_TRY(cudaEventRecord(e->ev[3], cs));
  CUDA_TRY(cudaEventRecord(e->cap_ev[1], cs));  // the caller's later work waits for the graph
  CUDA_TRY(cudaStreamWaitEvent(st, e->cap_ev[1], 0));
  e->stream = cs;
  e->ran = true;
  return NGAP_OK;
}

int ngap_batch_results(ngap_engine* e, uint64_t* reports, uint32_t* stream_ids, uint64_t cap,
                       uint64_t* n) {
  if (!e || !reports || !n) {
    set_error("ngap_batch_results: null argument");
    return NGAP_E_INVALID;
  }
  const uint64_t k = std::min<uint64_t>(e->h_counters[1], cap);
  *n = 0;
  if (k == 0) return NGAP_OK;
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaMemcpy(reports, e->d_unique, k * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  if (stream_ids)
    CUDA_TRY(cudaMemcpy(stream_ids, e->d_stream_ids, k * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  *n = k;
  return NGAP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Report sort + unique without any device allocation.
//
// Some callers cannot call cudaMalloc: a serving process whose device memory
// is owned by another allocator (a framework's caching allocator that has
// reserved the GPU), or a latency-critical loop where cudaMalloc's implicit
// device synchronisation is not acceptable. For them the scratch of the
// report sort lives in the file-scope array below, reserved on every GPU that
// loads this library until the process exits. It holds one ping-pong key
// buffer of kNoAllocMaxReports entries plus the digit histograms and
// counters (about 2 MiB). All calls share it and it keeps the last call's
// contents: calls whose work overlaps on the GPU (other streams, other host
// threads) race on it and must be serialised by the caller.
// ---------------------------------------------------------------------------
#include <mutex>

namespace {

constexpr uint64_t kNoAllocMaxReports = 1ull << 18;  // 262,144 reports
constexpr uint64_t kNoAllocTiles = (kNoAllocMaxReports + kSortTile - 1) / kSortTile;
constexpr size_t kNoAllocKeyBytes = kNoAllocMaxReports * sizeof(uint64_t);
constexpr size_t kNoAllocHistBytes = 16 * kNoAllocTiles * sizeof(uint32_t);
constexpr size_t kNoAllocBytes = kNoAllocKeyBytes + kNoAllocHistBytes + 4 * sizeof(unsigned long long);

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
constexpr int kNoAllocMaxDevices = 64;
uint8_t* g_noalloc_addr[kNoAllocMaxDevices] = {};
void* g_noalloc_ctx[kNoAllocMaxDevices] = {};  // context the address belongs to

// The calling thread's current CUDA context (driver cuCtxGetCurrent, reached
// through the runtime's entry-point lookup so that the library does not link
// the driver library), or nullptr when it cannot be read.
void* current_context() {
  using Fn = int (*)(void**);
  static Fn fn = []() -> Fn {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<Fn>(f);
  }();
  void* ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// Device address of the scratch array on the current device. In host code
// g_noalloc_scratch names a host-side stand-in, not device memory, so the
// address is looked up with that device current: once per device, and again
// whenever the device's current context is another one than at the lookup
// (after cudaDeviceReset, or a context the caller made current), whose
// address the old one is not.
int noalloc_scratch(int dev, uint8_t** out) {
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    set_error("device %d is beyond the %d devices the allocation-free path supports", dev,
              kNoAllocMaxDevices);
    return NGAP_E_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  void* ctx = current_context();
  if (!g_noalloc_addr[dev] || !ctx || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    cudaError_t ce = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (ce != cudaSuccess) {
      g_noalloc_addr[dev] = nullptr;
      set_error("cudaGetSymbolAddress of the sort scratch failed: %s", cudaGetErrorString(ce));
      return NGAP_E_CUDA;
    }
    g_noalloc_addr[dev] = static_cast<uint8_t*>(p);
    // the runtime may have made the primary context current just now
    g_noalloc_ctx[dev] = ctx ? ctx : current_context();
  }
  *out = g_noalloc_addr[dev];
  return NGAP_OK;
}

// Copies reference-encoded reports into sort keys (offset << 32 | id) and
// resets the counters: [0] = n, [1] = unique count.
__global__ void noalloc_prepare(const uint64_t* __restrict__ in, uint64_t n,
                                uint64_t* __restrict__ keys, unsigned long long* counters) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    counters[0] = n;
    counters[1] = 0;
    counters[2] = 0;
    counters[3] = 0;
  }
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t x = in[i];
    keys[i] = (x << 32) | (x >> 32);
  }
}

}  // namespace

extern "C" int ngap_reports_sort_unique_noalloc(const uint64_t* d_in, uint64_t n, uint64_t* d_out,
                                                uint64_t* n_out, void* stream) {
  if ((!d_in && n) || !d_out || !n_out) {
    set_error("ngap_reports_sort_unique_noalloc: null argument");
    return NGAP_E_INVALID;
  }
  if (n > kNoAllocMaxReports) {
    set_error("ngap_reports_sort_unique_noalloc: %llu reports exceed the allocation-free "
              "maximum of %llu", (unsigned long long)n, (unsigned long long)kNoAllocMaxReports);
    return NGAP_E_INVALID;
  }
  *n_out = 0;
  if (n == 0) return NGAP_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CUDA_TRY(cudaStreamIsCapturing(st, &cap));
  if (cap != cudaStreamCaptureStatusNone) {  // the call waits for the stream below
    set_error("ngap_reports_sort_unique_noalloc waits for its stream to return the unique "
              "count, so it cannot run while that stream is being captured");
    return NGAP_E_INVALID;
  }
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  uint8_t* base = nullptr;
  int rc = noalloc_scratch(dev, &base);
  if (rc != NGAP_OK) return rc;
  uint64_t* keys = reinterpret_cast<uint64_t*>(base);
  uint32_t* hist = reinterpret_cast<uint32_t*>(base + kNoAllocKeyBytes);
  unsigned long long* counters =
      reinterpret_cast<unsigned long long*>(base + kNoAllocKeyBytes + kNoAllocHistBytes);
  int sms = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const uint32_t tiles = (uint32_t)((n + kSortTile - 1) / kSortTile);
  const int grid = (int)std::max<uint32_t>(1, std::min<uint32_t>(tiles, (uint32_t)sms * 8));
  // 8 digit passes over the offset half and 8 over the id half; an even count
  // leaves the sorted keys back in the scratch buffer, d_out being the other
  // half of the ping-pong
  const int npass = 16;
  uint64_t* src = (npass % 2 == 0) ? keys : d_out;
  uint64_t* dst = (npass % 2 == 0) ? d_out : keys;
  noalloc_prepare<<<grid, 256, 0, st>>>(d_in, n, src, counters);
  for (int k = 0; k < npass; k++) {
    const int sh = k < 8 ? 4 * k : 32 + 4 * (k - 8);
    radix_hist<<<grid, kSortThreads, 0, st>>>(src, counters, n, sh, hist);
    scan_exclusive_1block<<<1, kScanThreads, 0, st>>>(hist, counters, n, 16, nullptr);
    radix_scatter<<<grid, kSortThreads, 0, st>>>(src, dst, counters, n, sh, hist);
    std::swap(src, dst);
  }
  unique_count<<<grid, kSortThreads, 0, st>>>(src, counters, n, hist);
  scan_exclusive_1block<<<1, kScanThreads, 0, st>>>(hist, counters, n, 1, counters + 1);
  unique_write<<<grid, kSortThreads, 0, st>>>(src, counters, n, hist, d_out);
  CUDA_TRY(cudaGetLastError());
  unsigned long long un = 0;
  CUDA_TRY(cudaMemcpyAsync(&un, counters + 1, sizeof(un), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  *n_out = un;
  return NGAP_OK;
}
