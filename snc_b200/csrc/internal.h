// Host-side structures shared by the C ABI implementation files.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/snc_b200.h"

namespace sncb {

void set_error(const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);  // records and maps to a status

// Failure injection on the host (api.cu): true when this device allocation is
// to fail (SNC_B200_FAIL_ALLOC / snc_b200_inject_alloc_failure).
bool alloc_fault();

// Wait bound and injected stall of a launch with grid barriers (api.cu):
// ns = 0 is the default bound; stall > 0 makes every grid wait of that launch
// run out.  consume: take one pending stall.
struct WaitCtl {
  unsigned long long ns;
  unsigned stall;
};
WaitCtl take_wait_ctl(bool consume);

#define SNCB_CUDA(call)                                  \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

template <typename T>
int dev_upload(T** d, const T* h, size_t n) {
  *d = nullptr;
  if (n == 0) n = 1;
  if (alloc_fault()) { set_error("device allocation failed (injected)"); return SNC_B200_ENOMEM; }
  SNCB_CUDA(cudaMalloc(reinterpret_cast<void**>(d), n * sizeof(T)));
  if (h) SNCB_CUDA(cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice));
  return SNC_B200_OK;
}

template <typename T>
int dev_alloc(T** d, size_t n) {
  *d = nullptr;
  if (n == 0) n = 1;
  if (alloc_fault()) { set_error("device allocation failed (injected)"); return SNC_B200_ENOMEM; }
  SNCB_CUDA(cudaMalloc(reinterpret_cast<void**>(d), n * sizeof(T)));
  return SNC_B200_OK;
}

inline void dev_free(void* p) {
  if (p) cudaFree(p);
}

// Device-resident graph.  Neurons with at least one incoming synapse own a
// ring column (col_of[j] >= 0, assigned in ascending id order); the delay
// ring of one sample is [ring_len][ncols] floats.  Edges are packed 8 bytes:
// x = ring column of the post | delay << 24, y = sign[pre] * weight.
struct OneShot;

struct Graph {
  int N = 0, S = 0, R = 0, ncols = 0, noc = 0, nic = 0, max_delay = 1;
  int sm_count = 0;
  // host copies used by the schedule builder and the adapters
  std::vector<int> row_ptr_h, chan_ptr_h, chan_ids_h, col_of_h;
  // device, CSR (insertion) order
  int* row_ptr = nullptr;   // [N+1]
  uint2* edges = nullptr;   // [S]
  int* post = nullptr;      // [S] post neuron ids (e-prop update)
  int* col_of = nullptr;    // [N]
  int* out_ch = nullptr;    // [N] output channel or -1
  uint8_t* role = nullptr;  // [N]
  int* channel = nullptr;   // [N]
  int* chan_ptr = nullptr;  // [nic+1] input channel -> input neurons (device copy)
  int* chan_ids = nullptr;
  int max_fan = 0;          // most input neurons of one channel
  // block partition for the multi-CTA (grid) kernels: block b owns neurons
  // [b*BS, min(N,(b+1)*BS)) and their ring columns [colbase[b], colbase[b+1]).
  int P = 0, BS = 0;
  int* colbase = nullptr;   // [P+1]
  // dest-grouped edges: each row's edges stably regrouped by destination
  // block; group g of row i is (block, first edge) for g in [gptr[i], gptr[i+1]).
  uint2* gedges = nullptr;  // [S]
  int* gptr = nullptr;      // [N+1]
  int2* groups = nullptr;   // [G]
  // inbox layout: destination block b receives at most (number of groups
  // targeting b) descriptors per step, stored from ibase[b].
  int G = 0;
  int* ibase = nullptr;     // [P+1]
  // leaky readout units (OUTPUT neurons with a channel, ascending id): rank of
  // each neuron among them or -1, and each rank's channel
  int n_ro = 0;
  int* ro_rank = nullptr;   // [N]
  int* ro_chan = nullptr;   // [n_ro]
  long long signature = 0;  // coarse shape class (log sizes, fan-in skew, ring length)
  unsigned long long hash = 0;  // content hash of the graph: the autotuner's cache key
  float fanin_cv = 0.f, density = 0.f;
  mutable OneShot* oneshot = nullptr;  // workspace of the one-call forwards
};

// Byte offsets of the arrays of a schedule image (identical on host and device).
struct SchedLayout {
  size_t steps = 0, order = 0, sptr_off = 0, stepbase = 0, raster_off = 0, sched_ptr = 0;
  size_t blk = 0;  // 0: no sched_blk
  size_t nid = 0, ext = 0, n_out = 0, total = 0;
};

// Host staging buffer: pageable (a vector) or pinned (cudaHostAlloc), grown
// on demand.
struct HostImage {
  bool pinned = false;
  unsigned char* p = nullptr;
  size_t cap = 0;
  std::vector<unsigned char> vec;
  explicit HostImage(bool pin = false) : pinned(pin) {}
  HostImage(const HostImage&) = delete;
  HostImage& operator=(const HostImage&) = delete;
  int reserve(size_t n);
  void release();
  ~HostImage() { release(); }
};

// A device allocation grown on demand (contents not kept when it grows).
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  int reserve(size_t n);
  void release();
  ~DevBuf() { release(); }
};

struct Inputs {
  const Graph* g = nullptr;
  int B = 0, Tmax = 0;
  long long total_steps = 0, raster_words = 0;
  std::vector<int> steps_h, order_h;
  std::vector<long long> sptr_off_h, raster_off_h, stepbase_h;
  int* steps = nullptr;         // [B]
  int* order = nullptr;         // [B] samples by descending step count
  long long* sptr_off = nullptr;  // [B] start of sample b's step pointers
  long long* stepbase = nullptr;  // [B] global index of sample b's first step
  int* sched_ptr = nullptr;     // concatenated [T_b + 1] absolute entry offsets
  int* sched_nid = nullptr;     // entries sorted by neuron within a step
  float* sched_ext = nullptr;   // drive summed in event order
  int* sched_blk = nullptr;     // [total_steps][P+1] first entry of each neuron
                                // block per step (null when too large)
  long long* raster_off = nullptr;  // [B] first raster word of sample b
  long long n_entries = 0;
  long long dev_bytes = 0;      // bytes copied to the device for this schedule
  SchedLayout layout;
  void* dblock = nullptr;       // the one device allocation holding every array
  bool owns_block = true;
  int* d_n_out = nullptr;       // device copy of n_entries
  int* d_err = nullptr;         // schedule builder's error word (work block)
};

struct Run {
  const Graph* g = nullptr;
  const Inputs* in = nullptr;
  int flags = 0;
  int W = 0;  // raster words per step
  // outputs
  int* counts = nullptr;                 // [B][noc]
  unsigned long long* spikes = nullptr;  // [B]
  unsigned long long* events = nullptr;  // [B]
  uint32_t* raster = nullptr;            // [raster_words]
  float* vfinal = nullptr;               // [B][N]
  // the small results (error words, counters, logits) come back through one
  // pinned block: asynchronous copies and a single synchronisation
  HostImage fetch_img{true};
  // control
  int* err = nullptr;
  unsigned* ctl = nullptr;  // [0] barrier counter, [1] work-queue counter
  // grid-path state (one wave of Bw samples in lockstep)
  int Bw = 0, Bw_cap = 0;
  float* v = nullptr;
  int* refr = nullptr;
  float* ring = nullptr;
  int* fired = nullptr;      // [Bw][2][N]
  int* fired_cnt = nullptr;  // [Bw][2][P]
  unsigned long long* inbox = nullptr;  // [Bw][2][G] (first edge << 32 | length)
  int* inbox_cnt = nullptr;             // [Bw][2][P]
  bool gplan_rsm = false;    // tier G keeps ring slices in shared memory
  size_t gplan_smem = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  int used_mode = -1, used_path = -1;
  // captured launch of the persistent path
  cudaGraphExec_t gexec = nullptr;
  int gexec_mode = -1;
  snc_lif gexec_lif{};
  cudaStream_t gexec_stream = nullptr;
  unsigned long long gexec_wait_ns = 0;  // wait bound baked into the graph
  int gexec_shape[4] = {-1, -1, -1, -1};  // launch shape baked into the graph
  // launch shape set by snc_b200_run_configure or an autotuned AUTO launch
  // (tier -1 / threads 0 / wave 0 / ring_smem -1: chosen automatically)
  int cfg_tier = -1, cfg_threads = 0, cfg_wave = 0, cfg_rsm = -1;
  bool cfg_explicit = false;  // set by the caller: AUTO launches keep it
  // leaky readout units (snc_b200_run_set_readout): decay, or < 0 when off;
  // final potential of every readout unit [B][n_ro] and the logits [B][noc]
  float ro_decay = -1.f, gexec_ro = -1.f;
  float* ro_v = nullptr;
  float* ro_logits = nullptr;
  cudaStream_t own_stream = nullptr;  // stands in for the legacy default stream
  bool graph_refused = false;         // stream capture failed once; launch directly
  bool used_graph = false;            // the last launch went through the graph
  // e-prop through the grid path (all null for a forward): the trainer's
  // weights in CSR and destination-grouped order, and what the deferred
  // eligibility reads -- psi per ring column and step, per-neuron fire counts
  const uint2* edges_w = nullptr;
  const uint2* gedges_w = nullptr;
  float* psi_hist = nullptr;  // [B][ncols][psi_T]
  int psi_T = 0;
  unsigned long long* fires = nullptr;
  float gamma = 0.f;
};

// One e-prop minibatch forward (tier S kernel with eligibility).
struct EpropLaunch {
  const Graph* g = nullptr;
  const Inputs* in = nullptr;
  const uint2* edges = nullptr;  // packed edges carrying the trainer's weights
  int* counts = nullptr;         // [B][max(1,noc)]
  unsigned long long* spikes = nullptr;
  unsigned long long* events = nullptr;
  float* elig = nullptr;         // [B][S] accumulated in the forward (null: none)
  unsigned long long* fires = nullptr;
  float* psi_hist = nullptr;     // [B][ncols][psi_T] surrogate per column and step
  int psi_T = 0;
  uint32_t* raster = nullptr;    // spike raster, at the inputs' raster offsets
  float gamma = 0.f, trace_decay = 0.f;
  snc_lif lif{};
  int mode = 2;
  int* err = nullptr;
  unsigned* ctl = nullptr;
};

// Per-graph workspace of snc_b200_forward / snc_b200_forward_batched.
struct OneShot {
  std::mutex mu;
  HostImage img{true};
  DevBuf keep, work;  // the schedule and the builder's work arrays
  Inputs in;
  Run run;
  int B_cap = 0;
  cudaStream_t stream = nullptr;
};

// schedule.cu: the per-step injection schedule of a batch (build_schedule,
// cpu_backend.cpp:43-65); ignore_sample maps every event to sample 0.
// Uploads the events of a batch and builds its schedule on the GPU in
// stream order on `st` (keep: the schedule, work: scratch; both grown).
// ev_device: the events already lie in device memory.
int stage_inputs(const Graph* g, const snc_input_event* ev, size_t n_ev, int B, const int32_t* steps,
                 bool ignore_sample, Inputs* in, HostImage* img, DevBuf* keep, DevBuf* work,
                 cudaStream_t st, bool ev_device);
// Exclusive prefix sums of int counts on the device (totals < 2^31): out[0..n]
// from in[0..n) in stream order; scratch holds scan_scratch_ints(n) ints.
size_t scan_scratch_ints(long long n);
int scan_exclusive(const int* in, int* out, long long n, int* scratch, cudaStream_t st);
// graphbuild.cu: packed and destination-grouped edges, groups and inbox
// bases of a validated graph, built on the device (g->N, S, BS, P, col_of_h set).
// api.cu: the per-neuron tables of a graph (O(N), host) and their upload;
// the content hash of a graph view; release of a graph's device arrays.
int setup_tables(Graph* g, int n, int m, int max_delay, const int32_t* row_ptr, const int* indeg,
                 const uint8_t* role, const int32_t* channel);
unsigned long long graph_hash_view(const snc_graph_view* v);
void free_graph(Graph* g);
int build_graph_device(const snc_graph_view* v, Graph* g);
// The same from columns already on the device (g->row_ptr, g->post and
// g->col_of set; weights, delays and per-neuron signs as device arrays).
int build_graph_device_cols(Graph* g, const float* w, const int* delays, const int8_t* sign);
// The schedule of a batch encoded on the device from its features.
int encode_inputs(const Graph* g, int enc, const float* features, int C, int B, const int32_t* steps,
                  float gain, float max_rate, float threshold, uint64_t seed, Inputs* in);
void place_schedule(Inputs* in, void* dev);
int upload_inputs(const Graph* g, const snc_input_event* ev, size_t n_ev, int B,
                  const int32_t* steps, bool ignore_sample, Inputs* in);
void free_inputs(Inputs* in);
int oneshot_forward(const Graph* g, const snc_input_event* ev, size_t n_ev, int B,
                    const int32_t* steps, bool ignore_sample, const snc_lif* lif, int mode,
                    int path, float* logits, int64_t* spikes, int64_t* events_out,
                    snc_run_stats* stats);
void free_oneshot(const Graph* g);

// api.cu
// Waits for the run and copies its results out.  d_sched_err, when given,
// is the schedule builder's overflow word, read in the same batch of copies
// into *sched_err.
int fetch_run(Run* r, float* logits, int64_t* spikes, int64_t* events, uint32_t* raster,
              float* v_final, snc_run_stats* stats, const int* d_sched_err = nullptr,
              int* sched_err = nullptr);
void free_run(Run* r);

// forward.cu
int launch_eprop_forward(const EpropLaunch& e, cudaStream_t stream);
int launch_run(Run* r, const snc_lif* lif, int mode, int path, cudaStream_t stream);
int tier_s_smem_bytes(const Graph* g, int mode, bool eprop);
// AUTO resolution: the autotuned choice cached for this graph and batch (mode,
// path and launch shape: shape[4] = tier, threads, wave, ring_smem), else a
// default rule (shape automatic).
int resolve_auto(const Graph* g, const Inputs* in, int* mode, int* path, int* shape);
// Checks a launch shape for this run's graph and inputs (tier G threads a
// multiple of 32 in [512, 768], wave within the batch and shared memory,
// ring slices that fit).  Returns SNC_B200_OK or SNC_B200_EUNSUPPORTED.
int check_shape(const Run* r, int mode, int tier, int threads, int wave, int rsm);

}  // namespace sncb

// The opaque handles of the C ABI.
struct snc_b200_graph : sncb::Graph {};
struct snc_b200_inputs : sncb::Inputs {};
struct snc_b200_run : sncb::Run {};
