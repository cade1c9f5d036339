// C ABI implementation: graph upload, input schedules, runs, one-call
// forwards and the delivery autotuner.  See include/snc_b200.h.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "internal.h"

namespace sncb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int cuda_fail(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();  // clear a non-sticky error
  if (e == cudaErrorMemoryAllocation) return SNC_B200_ENOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return SNC_B200_ENODEV;
  return SNC_B200_ECUDA;
}

// ---- failure injection and wait bounds ---------------------------------------
// Device allocations left before every further one fails: -1 = never fail;
// initialised from SNC_B200_FAIL_ALLOC (the number of allocations to allow).
static std::atomic<long long> g_alloc_left{[] {
  const char* e = std::getenv("SNC_B200_FAIL_ALLOC");
  return e && *e ? std::max(-1ll, std::atoll(e)) : -1ll;
}()};
static std::atomic<unsigned long long> g_wait_ns{0};
static std::atomic<int> g_stalls{0};

bool alloc_fault() {
  long long left = g_alloc_left.load();
  while (left >= 0) {
    if (left == 0) return true;
    if (g_alloc_left.compare_exchange_weak(left, left - 1)) return false;
  }
  return false;
}

WaitCtl take_wait_ctl(bool consume) {
  WaitCtl w{g_wait_ns.load(), 0};
  if (consume) {
    int n = g_stalls.load();
    while (n > 0 && !g_stalls.compare_exchange_weak(n, n - 1)) {
    }
    if (n > 0) w.stall = 1;
  }
  return w;
}

static int check_device() {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_error("no CUDA device");
    return SNC_B200_ENODEV;
  }
  int dev = 0, major = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (major != 10) {
    set_error("device is not compute capability 10.x (this library is built for sm_100a)");
    return SNC_B200_ENODEV;
  }
  return SNC_B200_OK;
}

// SNNGraph::validate (src/graph/snn_graph.cpp:30-56) plus this backend's limits.
static int validate_view(const snc_graph_view* v) {
  if (!v) { set_error("null graph"); return SNC_B200_EINVAL; }
  const int n = v->num_neurons, m = v->num_synapses;
  if (n < 0 || m < 0) { set_error("negative num_neurons / num_synapses"); return SNC_B200_EINVAL; }
  if (n > 0 && (!v->row_ptr || !v->role || !v->sign || !v->channel)) {
    set_error("null per-neuron array"); return SNC_B200_EINVAL;
  }
  if (m > 0 && (!v->post_ids || !v->weights || !v->delays)) {
    set_error("null CSR column array"); return SNC_B200_EINVAL;
  }
  if (n > 0 && v->row_ptr[0] != 0) { set_error("row_ptr[0] != 0"); return SNC_B200_EINVAL; }
  if (n > 0 && v->row_ptr[n] != m) { set_error("row_ptr.back() != num_synapses"); return SNC_B200_EINVAL; }
  for (int i = 0; i < n; ++i)
    if (v->row_ptr[i] > v->row_ptr[i + 1]) { set_error("row_ptr not monotone"); return SNC_B200_EINVAL; }
  for (int s = 0; s < m; ++s) {
    if (v->post_ids[s] < 0 || v->post_ids[s] >= n) { set_error("post id out of range"); return SNC_B200_EINVAL; }
    if (v->delays[s] < 1) { set_error("delay < 1"); return SNC_B200_EINVAL; }
    if (v->delays[s] > 255) { set_error("delay > 255 is outside this backend's limits"); return SNC_B200_EUNSUPPORTED; }
  }
  if (n >= (1 << 24)) { set_error("num_neurons >= 2^24 is outside this backend's limits"); return SNC_B200_EUNSUPPORTED; }
  return SNC_B200_OK;
}

void free_graph(Graph* g) {
  if (!g) return;
  free_oneshot(g);
  for (void* p : {(void*)g->row_ptr, (void*)g->edges, (void*)g->post, (void*)g->col_of,
                  (void*)g->out_ch, (void*)g->role, (void*)g->channel, (void*)g->colbase,
                  (void*)g->gedges, (void*)g->gptr, (void*)g->groups, (void*)g->ibase,
                  (void*)g->chan_ptr, (void*)g->chan_ids, (void*)g->ro_rank, (void*)g->ro_chan})
    dev_free(p);
}

// 64-bit content hash of a graph view (sizes and every array, weights by
// their bits): the autotuner's cache key.  Words are folded pairwise with a
// multiply-xorshift mix, one pass over the arrays.
unsigned long long graph_hash_view(const snc_graph_view* v) {
  unsigned long long h = 0x9E3779B97F4A7C15ull ^ ((unsigned long long)v->num_neurons << 32) ^
                         (unsigned)v->num_synapses;
  auto mix = [&h](unsigned long long x) {
    h ^= x + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 31;
  };
  auto words = [&mix](const void* p, size_t bytes) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    size_t i = 0;
    for (; i + 8 <= bytes; i += 8) {
      unsigned long long x;
      std::memcpy(&x, c + i, 8);
      mix(x);
    }
    unsigned long long tail = 0;
    std::memcpy(&tail, c + i, bytes - i);
    mix(tail ^ ((unsigned long long)bytes << 56));
  };
  const size_t n = (size_t)v->num_neurons, m = (size_t)v->num_synapses;
  words(v->row_ptr, 4 * (n + 1));
  words(v->post_ids, 4 * m);
  words(v->weights, 4 * m);
  words(v->delays, 4 * m);
  words(v->role, n);
  words(v->sign, n);
  words(v->channel, 4 * n);
  return h;
}

// The per-neuron tables of a graph on the host (O(N) work) from its sizes,
// largest delay, row pointers, in-degrees and per-neuron arrays, and their
// upload; the O(S) columns are packed on the device afterwards.
int setup_tables(Graph* g, int n, int m, int max_delay, const int32_t* row_ptr,
                        const int* indeg, const uint8_t* role_v, const int32_t* channel_v) {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&g->sm_count, cudaDevAttrMultiProcessorCount, dev);
  g->N = n;
  g->S = m;
  g->max_delay = max_delay;
  g->R = max_delay + 1;
  // rebuild_io_index (snn_graph.cpp:13-28)
  int max_in = -1, max_out = -1;
  for (int i = 0; i < n; ++i) {
    if (role_v[i] == 1) max_in = std::max(max_in, channel_v[i]);
    else if (role_v[i] == 2) max_out = std::max(max_out, channel_v[i]);
  }
  g->nic = max_in + 1;
  g->noc = max_out + 1;
  // channel -> INPUT neurons (ascending id), cpu_backend.cpp:50-55
  g->chan_ptr_h.assign(std::max(0, g->nic) + 1, 0);
  for (int i = 0; i < n; ++i)
    if (role_v[i] == 1 && channel_v[i] >= 0 && channel_v[i] < g->nic) g->chan_ptr_h[channel_v[i] + 1]++;
  for (int c = 0; c < g->nic; ++c) g->chan_ptr_h[c + 1] += g->chan_ptr_h[c];
  g->chan_ids_h.assign(g->chan_ptr_h[std::max(0, g->nic)], 0);
  {
    std::vector<int> fill(std::max(0, g->nic), 0);
    for (int i = 0; i < n; ++i)
      if (role_v[i] == 1 && channel_v[i] >= 0 && channel_v[i] < g->nic)
        g->chan_ids_h[g->chan_ptr_h[channel_v[i]] + fill[channel_v[i]]++] = i;
  }
  // ring columns for neurons with incoming synapses, ascending id
  g->col_of_h.assign(n, -1);
  int nc = 0;
  for (int i = 0; i < n; ++i)
    if (indeg[i] > 0) g->col_of_h[i] = nc++;
  g->ncols = nc;
  std::vector<int> out_ch(n, -1);
  for (int i = 0; i < n; ++i)
    if (role_v[i] == 2 && channel_v[i] >= 0) out_ch[i] = channel_v[i];
  g->row_ptr_h.assign(row_ptr, row_ptr + n + 1);
  // block partition for the grid kernels
  const int sm = std::max(1, g->sm_count);
  int BS = (n + sm - 1) / sm;
  BS = std::max(32, (BS + 31) / 32 * 32);
  const int P = std::max(1, (n + BS - 1) / BS);
  g->BS = BS;
  g->P = P;
  std::vector<int> colbase(P + 1, 0);
  {
    int c = 0;
    for (int b = 0; b < P; ++b) {
      colbase[b] = c;
      const int lo = b * BS, hi = std::min(n, lo + BS);
      for (int j = lo; j < hi; ++j)
        if (g->col_of_h[j] >= 0) ++c;
    }
    colbase[P] = c;
  }
  // fan-in skew and density for the autotuner signature
  {
    double mean = n ? (double)m / n : 0.0, var = 0.0;
    for (int i = 0; i < n; ++i) var += (indeg[i] - mean) * (indeg[i] - mean);
    var = n ? var / n : 0.0;
    g->fanin_cv = mean > 0 ? (float)(std::sqrt(var) / mean) : 0.f;
    g->density = n > 1 ? (float)((double)m / ((double)n * (n - 1))) : 0.f;
    const long long lg = (long long)std::log2(std::max(1, n)) * 64 + (long long)std::log2(std::max(1, m));
    g->signature = (lg << 16) ^ ((long long)(g->fanin_cv * 4) << 8) ^ (long long)g->R;
  }
  std::vector<uint8_t> role(role_v, role_v + n);
  std::vector<int> channel(channel_v, channel_v + n);
  // leaky readout units: the OUTPUT neurons with a channel, ascending id
  std::vector<int> ro_rank(n, -1), ro_chan;
  for (int i = 0; i < n; ++i)
    if (out_ch[i] >= 0) {
      ro_rank[i] = (int)ro_chan.size();
      ro_chan.push_back(out_ch[i]);
    }
  g->n_ro = (int)ro_chan.size();
  int rc;
  if ((rc = dev_upload(&g->col_of, g->col_of_h.data(), (size_t)n))) return rc;
  if ((rc = dev_upload(&g->out_ch, out_ch.data(), (size_t)n))) return rc;
  if ((rc = dev_upload(&g->role, role.data(), role.size()))) return rc;
  if ((rc = dev_upload(&g->channel, channel.data(), channel.size()))) return rc;
  if ((rc = dev_upload(&g->colbase, colbase.data(), colbase.size()))) return rc;
  if ((rc = dev_upload(&g->ro_rank, ro_rank.data(), ro_rank.size()))) return rc;
  if ((rc = dev_upload(&g->ro_chan, ro_chan.empty() ? nullptr : ro_chan.data(), ro_chan.size())))
    return rc;
  if ((rc = dev_upload(&g->chan_ptr, g->chan_ptr_h.data(), g->chan_ptr_h.size()))) return rc;
  if ((rc = dev_upload(&g->chan_ids, g->chan_ids_h.empty() ? nullptr : g->chan_ids_h.data(),
                       g->chan_ids_h.size())))
    return rc;
  g->max_fan = 0;
  for (int c = 0; c < g->nic; ++c) g->max_fan = std::max(g->max_fan, g->chan_ptr_h[c + 1] - g->chan_ptr_h[c]);
  return SNC_B200_OK;
}

static int upload_graph(const snc_graph_view* v, Graph* g) {
  int rc = validate_view(v);
  if (rc) return rc;
  g->hash = graph_hash_view(v);
  const int n = v->num_neurons, m = v->num_synapses;
  int max_delay = 1;
  for (int s = 0; s < m; ++s) max_delay = std::max(max_delay, v->delays[s]);
  std::vector<int> indeg(n, 0);
  for (int s = 0; s < m; ++s) indeg[v->post_ids[s]]++;
  if ((rc = setup_tables(g, n, m, max_delay, v->row_ptr, indeg.data(), v->role, v->channel))) return rc;
  // packed and destination-grouped edges, groups, inbox bases: on the device
  return build_graph_device(v, g);
}

// build_schedule (cpu_backend.cpp:43-65) for a batch: per (sample, step) the
// (neuron, drive) entries sorted by neuron, each drive summed from 0.0f in
// event order (cpu_backend.cpp:99).  ignore_sample maps every event to sample 0.
void free_run(Run* r) {
  if (!r) return;
  if (r->gexec) cudaGraphExecDestroy(r->gexec);
  for (void* p : {(void*)r->counts, (void*)r->spikes, (void*)r->events, (void*)r->raster,
                  (void*)r->vfinal, (void*)r->err, (void*)r->ctl, (void*)r->v, (void*)r->refr,
                  (void*)r->ring, (void*)r->fired, (void*)r->fired_cnt, (void*)r->inbox,
                  (void*)r->inbox_cnt, (void*)r->ro_v, (void*)r->ro_logits})
    dev_free(p);
  if (r->ev0) cudaEventDestroy(r->ev0);
  if (r->ev1) cudaEventDestroy(r->ev1);
  if (r->own_stream) cudaStreamDestroy(r->own_stream);
}

static int create_run(const Graph* g, const Inputs* in, int flags, Run* r) {
  r->g = g;
  r->in = in;
  r->flags = flags;
  r->W = (g->N + 31) / 32;
  const size_t B = (size_t)std::max(1, in->B);
  int rc;
  if ((rc = dev_alloc(&r->counts, B * std::max(1, g->noc)))) return rc;
  if ((rc = dev_alloc(&r->spikes, B))) return rc;
  if ((rc = dev_alloc(&r->events, B))) return rc;
  if (flags & SNC_B200_RUN_RASTER)
    if ((rc = dev_alloc(&r->raster, (size_t)std::max<long long>(1, in->raster_words)))) return rc;
  if (flags & SNC_B200_RUN_VFINAL)
    if ((rc = dev_alloc(&r->vfinal, B * std::max(1, g->N)))) return rc;
  if ((rc = dev_alloc(&r->err, 1))) return rc;
  if ((rc = dev_alloc(&r->ctl, 4))) return rc;
  SNCB_CUDA(cudaEventCreate(&r->ev0));
  SNCB_CUDA(cudaEventCreate(&r->ev1));
  return SNC_B200_OK;
}

int fetch_run(Run* r, float* logits, int64_t* spikes, int64_t* events, uint32_t* raster,
              float* v_final, snc_run_stats* stats, const int* d_sched_err, int* sched_err) {
  const Graph* g = r->g;
  const Inputs* in = r->in;
  SNCB_CUDA(cudaEventSynchronize(r->ev1));
  float ms = 0.f;
  SNCB_CUDA(cudaEventElapsedTime(&ms, r->ev0, r->ev1));
  r->last_ms = ms;
  const int B = in->B, noc = std::max(1, g->noc);
  const bool ro = logits && r->ro_decay >= 0.f && r->ro_logits && B > 0;
  // pinned block: err, schedule err | spikes [B] | events [B] | counts [B][noc] | readout [B][noc]
  const size_t Bn = (size_t)std::max(0, B);
  const size_t o_sp = 8, o_ev = o_sp + 8 * Bn, o_cnt = o_ev + 8 * Bn;
  const size_t o_lg = o_cnt + 4 * Bn * noc, total = o_lg + (ro ? 4 * Bn * noc : 0);
  int rc;
  if ((rc = r->fetch_img.reserve(total))) return rc;
  unsigned char* h = r->fetch_img.p;
  std::memset(h, 0, 8);
  const cudaStream_t s0 = cudaStreamPerThread;
  SNCB_CUDA(cudaMemcpyAsync(h, r->err, 4, cudaMemcpyDeviceToHost, s0));
  if (d_sched_err) SNCB_CUDA(cudaMemcpyAsync(h + 4, d_sched_err, 4, cudaMemcpyDeviceToHost, s0));
  if (B > 0) {
    SNCB_CUDA(cudaMemcpyAsync(h + o_sp, r->spikes, 8 * Bn, cudaMemcpyDeviceToHost, s0));
    SNCB_CUDA(cudaMemcpyAsync(h + o_ev, r->events, 8 * Bn, cudaMemcpyDeviceToHost, s0));
    SNCB_CUDA(cudaMemcpyAsync(h + o_cnt, r->counts, 4 * Bn * noc, cudaMemcpyDeviceToHost, s0));
    if (ro) SNCB_CUDA(cudaMemcpyAsync(h + o_lg, r->ro_logits, 4 * Bn * noc, cudaMemcpyDeviceToHost, s0));
  }
  SNCB_CUDA(cudaStreamSynchronize(s0));
  int err = 0;
  std::memcpy(&err, h, 4);
  if (sched_err) std::memcpy(sched_err, h + 4, 4);
  const int* counts = reinterpret_cast<const int*>(h + o_cnt);
  const unsigned long long* sp = reinterpret_cast<const unsigned long long*>(h + o_sp);
  const unsigned long long* evn = reinterpret_cast<const unsigned long long*>(h + o_ev);
  if (ro) {
    // leaky readout units: their potentials over the sample's steps
    const float* lg = reinterpret_cast<const float*>(h + o_lg);
    for (int b = 0; b < B; ++b)
      for (int c = 0; c < g->noc; ++c) logits[(size_t)b * g->noc + c] = lg[(size_t)b * noc + c];
  } else if (logits) {
    for (int b = 0; b < B; ++b)
      for (int c = 0; c < g->noc; ++c) logits[(size_t)b * g->noc + c] = (float)counts[(size_t)b * noc + c];
  }
  long long ts = 0, te = 0;
  for (int b = 0; b < B; ++b) {
    if (spikes) spikes[b] = (int64_t)sp[b];
    if (events) events[b] = (int64_t)evn[b];
    ts += (long long)sp[b];
    te += (long long)evn[b];
  }
  if (raster) {
    if (!(r->flags & SNC_B200_RUN_RASTER)) { set_error("run created without SNC_B200_RUN_RASTER"); return SNC_B200_EINVAL; }
    if (in->raster_words)
      SNCB_CUDA(cudaMemcpy(raster, r->raster, (size_t)in->raster_words * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  }
  if (v_final) {
    if (!(r->flags & SNC_B200_RUN_VFINAL)) { set_error("run created without SNC_B200_RUN_VFINAL"); return SNC_B200_EINVAL; }
    if (B > 0) SNCB_CUDA(cudaMemcpy(v_final, r->vfinal, (size_t)B * g->N * sizeof(float), cudaMemcpyDeviceToHost));
  }
  if (stats) {
    stats->spikes = ts;
    stats->synaptic_events = te;
    stats->overflow = err == SNC_B200_EOVERFLOW ? 1 : 0;
    stats->ms = ms;
  }
  if (err) {
    set_error(err == SNC_B200_ETIMEOUT ? "device barrier timed out" : "device error word set");
    return err < 0 ? err : SNC_B200_ECUDA;
  }
  return SNC_B200_OK;
}

// ---- autotuner --------------------------------------------------------------
// Tuned launches, keyed by the graph's content hash and the batch's shape
// (samples, total steps): a graph of similar size but other contents is tuned
// on its own.
struct TuneKey {
  unsigned long long hash;
  int B;
  long long steps;
  bool operator<(const TuneKey& o) const {
    if (hash != o.hash) return hash < o.hash;
    if (B != o.B) return B < o.B;
    return steps < o.steps;
  }
};
static std::mutex g_tune_mu;
static std::map<TuneKey, snc_launch_config> g_tune_cache;

static TuneKey tune_key(const Graph* g, const Inputs* in) {
  return TuneKey{g->hash, in->B, in->total_steps};
}

int resolve_auto(const Graph* g, const Inputs* in, int* mode, int* path, int* shape) {
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(tune_key(g, in));
    if (it != g_tune_cache.end()) {
      const snc_launch_config& c = it->second;
      if (*mode == SNC_B200_MODE_AUTO) *mode = c.mode;
      if (*path == SNC_B200_PATH_AUTO) *path = c.path;
      shape[0] = c.tier;
      shape[1] = c.block_threads;
      shape[2] = c.wave;
      shape[3] = c.ring_smem;
      return SNC_B200_OK;
    }
  }
  // untuned default: persistent path; bucketed delivery when the in-degree is
  // heavily skewed (many sources hammer few targets), atomic otherwise.
  if (*path == SNC_B200_PATH_AUTO) *path = SNC_B200_PATH_PERSISTENT;
  if (*mode == SNC_B200_MODE_AUTO) *mode = g->fanin_cv > 1.0f ? SNC_B200_MODE_BUCKET : SNC_B200_MODE_ATOMIC;
  shape[0] = -1;
  shape[1] = 0;
  shape[2] = 0;
  shape[3] = -1;
  return SNC_B200_OK;
}

}  // namespace sncb

using namespace sncb;

extern "C" {

int snc_b200_available(void) { return check_device() == SNC_B200_OK ? 1 : 0; }

int snc_b200_abi_version(void) { return SNC_B200_ABI_VERSION; }

int snc_b200_set_device(int device) {
  SNCB_CUDA(cudaSetDevice(device));
  return SNC_B200_OK;
}

const char* snc_b200_last_error(void) { return g_last_error.c_str(); }

int snc_b200_set_wait_limit(uint64_t ns) {
  g_wait_ns.store(ns);
  return SNC_B200_OK;
}

int snc_b200_inject_stall(int32_t n) {
  if (n < 0) { set_error("inject_stall: negative count"); return SNC_B200_EINVAL; }
  g_stalls.store(n);
  return SNC_B200_OK;
}

int snc_b200_inject_alloc_failure(int64_t after) {
  g_alloc_left.store(after < 0 ? -1 : after);
  return SNC_B200_OK;
}

int snc_b200_graph_upload(const snc_graph_view* v, snc_b200_graph** out) {
  if (!out) { set_error("null out"); return SNC_B200_EINVAL; }
  *out = nullptr;
  int rc = validate_view(v);
  if (rc) return rc;
  if ((rc = check_device())) return rc;
  auto* g = new snc_b200_graph();
  rc = upload_graph(v, g);
  if (rc) { free_graph(g); delete g; return rc; }
  *out = g;
  return SNC_B200_OK;
}

int snc_b200_graph_release(snc_b200_graph* g) {
  if (!g) return SNC_B200_OK;
  free_graph(g);
  delete g;
  return SNC_B200_OK;
}

int snc_b200_graph_info(const snc_b200_graph* g, int32_t* n, int32_t* s, int32_t* ring_len,
                        int32_t* n_out, int32_t* n_in) {
  if (!g) { set_error("null graph"); return SNC_B200_EINVAL; }
  if (n) *n = g->N;
  if (s) *s = g->S;
  if (ring_len) *ring_len = g->R;
  if (n_out) *n_out = g->noc;
  if (n_in) *n_in = g->nic;
  return SNC_B200_OK;
}

int snc_b200_graph_layout(const snc_b200_graph* g, uint32_t* edges, uint32_t* gedges, int32_t* gptr,
                          int32_t* groups, int32_t* col_of, int32_t* colbase, int32_t* ibase,
                          int32_t* block_size, int32_t* num_blocks, int32_t* num_groups) {
  if (!g) { set_error("null graph"); return SNC_B200_EINVAL; }
  const size_t S = (size_t)g->S, N = (size_t)g->N, P = (size_t)g->P, G = (size_t)g->G;
  if (edges && S) SNCB_CUDA(cudaMemcpy(edges, g->edges, S * 8, cudaMemcpyDeviceToHost));
  if (gedges && S) SNCB_CUDA(cudaMemcpy(gedges, g->gedges, S * 8, cudaMemcpyDeviceToHost));
  if (gptr) SNCB_CUDA(cudaMemcpy(gptr, g->gptr, (N + 1) * 4, cudaMemcpyDeviceToHost));
  if (groups && G) SNCB_CUDA(cudaMemcpy(groups, g->groups, G * 8, cudaMemcpyDeviceToHost));
  if (col_of && N) SNCB_CUDA(cudaMemcpy(col_of, g->col_of, N * 4, cudaMemcpyDeviceToHost));
  if (colbase) SNCB_CUDA(cudaMemcpy(colbase, g->colbase, (P + 1) * 4, cudaMemcpyDeviceToHost));
  if (ibase) SNCB_CUDA(cudaMemcpy(ibase, g->ibase, (P + 1) * 4, cudaMemcpyDeviceToHost));
  if (block_size) *block_size = g->BS;
  if (num_blocks) *num_blocks = g->P;
  if (num_groups) *num_groups = g->G;
  return SNC_B200_OK;
}

int snc_b200_inputs_upload(const snc_b200_graph* g, const snc_input_event* events, size_t n_events,
                           int32_t num_samples, const int32_t* steps, snc_b200_inputs** out) {
  if (!g || !out) { set_error("null argument"); return SNC_B200_EINVAL; }
  *out = nullptr;
  auto* in = new snc_b200_inputs();
  int rc = upload_inputs(g, events, n_events, num_samples, steps, false, in);
  if (rc) { free_inputs(in); delete in; return rc; }
  *out = in;
  return SNC_B200_OK;
}

int snc_b200_inputs_encode(const snc_b200_graph* g, int32_t encoder, const float* features,
                           int32_t n_channels, int32_t num_samples, const int32_t* steps,
                           float gain, float max_rate, float threshold, uint64_t seed,
                           snc_b200_inputs** out) {
  if (!g || !out) { set_error("null argument"); return SNC_B200_EINVAL; }
  *out = nullptr;
  auto* in = new snc_b200_inputs();
  int rc = encode_inputs(g, encoder, features, n_channels, num_samples, steps, gain, max_rate,
                         threshold, seed, in);
  if (rc) { free_inputs(in); delete in; return rc; }
  *out = in;
  return SNC_B200_OK;
}

int snc_b200_inputs_release(snc_b200_inputs* in) {
  if (!in) return SNC_B200_OK;
  free_inputs(in);
  delete in;
  return SNC_B200_OK;
}

int snc_b200_inputs_info(const snc_b200_inputs* in, int64_t* device_bytes, int64_t* entries) {
  if (!in) { set_error("null inputs"); return SNC_B200_EINVAL; }
  if (device_bytes) *device_bytes = in->dev_bytes;
  if (entries) *entries = in->n_entries;
  return SNC_B200_OK;
}

int snc_b200_inputs_read(const snc_b200_inputs* in, int32_t* sched_ptr, int32_t* neuron, float* drive) {
  if (!in) { set_error("null inputs"); return SNC_B200_EINVAL; }
  const size_t np = (size_t)(in->total_steps + in->B), ne = (size_t)in->n_entries;
  if (sched_ptr && np) SNCB_CUDA(cudaMemcpy(sched_ptr, in->sched_ptr, np * 4, cudaMemcpyDeviceToHost));
  if (neuron && ne) SNCB_CUDA(cudaMemcpy(neuron, in->sched_nid, ne * 4, cudaMemcpyDeviceToHost));
  if (drive && ne) SNCB_CUDA(cudaMemcpy(drive, in->sched_ext, ne * 4, cudaMemcpyDeviceToHost));
  return SNC_B200_OK;
}

int snc_b200_run_create(const snc_b200_graph* g, const snc_b200_inputs* in, int flags,
                        snc_b200_run** out) {
  if (!g || !in || !out || in->g != g) { set_error("bad run arguments"); return SNC_B200_EINVAL; }
  *out = nullptr;
  auto* r = new snc_b200_run();
  int rc = create_run(g, in, flags, r);
  if (rc) { free_run(r); delete r; return rc; }
  *out = r;
  return SNC_B200_OK;
}

int snc_b200_run_release(snc_b200_run* r) {
  if (!r) return SNC_B200_OK;
  free_run(r);
  delete r;
  return SNC_B200_OK;
}

int snc_b200_run_launch(snc_b200_run* r, const snc_lif* lif, int mode, int path, void* stream) {
  if (!r || !lif) { set_error("null argument"); return SNC_B200_EINVAL; }
  return launch_run(r, lif, mode, path, static_cast<cudaStream_t>(stream));
}

int snc_b200_run_fetch(snc_b200_run* r, float* logits, int64_t* spikes, int64_t* events,
                       uint32_t* raster, float* v_final, snc_run_stats* stats) {
  if (!r) { set_error("null run"); return SNC_B200_EINVAL; }
  return fetch_run(r, logits, spikes, events, raster, v_final, stats);
}

int snc_b200_run_used(const snc_b200_run* r, int* mode, int* path) {
  if (!r) { set_error("null run"); return SNC_B200_EINVAL; }
  if (mode) *mode = r->used_mode;
  if (path) *path = r->used_path;
  return SNC_B200_OK;
}

int snc_b200_run_used_graph(const snc_b200_run* r) {
  if (!r) { set_error("null run"); return SNC_B200_EINVAL; }
  return r->used_graph ? 1 : 0;
}

int snc_b200_forward(const snc_b200_graph* graph, const snc_graph_view* view,
                     const snc_input_event* events, size_t n_events, int32_t num_steps,
                     const snc_lif* lif, int mode, float* logits, snc_run_stats* stats) {
  if (!lif) { set_error("null lif"); return SNC_B200_EINVAL; }
  if (num_steps < 0) { set_error("negative num_steps"); return SNC_B200_EINVAL; }
  snc_b200_graph* owned = nullptr;
  int rc;
  if (!graph) {
    if ((rc = snc_b200_graph_upload(view, &owned))) return rc;
    graph = owned;
  }
  rc = oneshot_forward(graph, events, n_events, 1, &num_steps, true, lif, mode, SNC_B200_PATH_AUTO,
                       logits, nullptr, nullptr, stats);
  if (owned) snc_b200_graph_release(owned);
  return rc;
}

int snc_b200_forward_batched(const snc_b200_graph* graph, const snc_input_event* events,
                             size_t n_events, int32_t num_samples, const int32_t* steps,
                             const snc_lif* lif, int mode, float* logits, int64_t* spikes,
                             int64_t* events_out, snc_run_stats* stats) {
  if (!graph || !lif) { set_error("null argument"); return SNC_B200_EINVAL; }
  return oneshot_forward(graph, events, n_events, num_samples, steps, false, lif, mode,
                         SNC_B200_PATH_PERSISTENT, logits, spikes, events_out, stats);
}

int snc_b200_run_set_readout(snc_b200_run* r, float ro_decay) {
  if (!r) { set_error("null run"); return SNC_B200_EINVAL; }
  if (!(ro_decay >= 0.f)) {  // off (negative or NaN)
    r->ro_decay = -1.f;
    return SNC_B200_OK;
  }
  const Graph* g = r->g;
  const size_t B = (size_t)std::max(1, r->in->B);
  int rc;
  if (!r->ro_v && (rc = dev_alloc(&r->ro_v, B * std::max(1, g->n_ro)))) return rc;
  if (!r->ro_logits && (rc = dev_alloc(&r->ro_logits, B * std::max(1, g->noc)))) return rc;
  r->ro_decay = ro_decay;
  return SNC_B200_OK;
}

int snc_b200_run_configure(snc_b200_run* r, const snc_launch_config* cfg) {
  if (!r) { set_error("null run"); return SNC_B200_EINVAL; }
  if (!cfg) {  // back to automatic shapes
    r->cfg_tier = -1; r->cfg_threads = 0; r->cfg_wave = 0; r->cfg_rsm = -1;
    r->cfg_explicit = false;
    return SNC_B200_OK;
  }
  const int mode = cfg->mode >= 0 && cfg->mode <= SNC_B200_MODE_SORT ? cfg->mode : SNC_B200_MODE_SORT;
  int rc = check_shape(r, mode, cfg->tier, cfg->block_threads, cfg->wave, cfg->ring_smem);
  if (rc) return rc;
  r->cfg_tier = cfg->tier;
  r->cfg_threads = cfg->block_threads;
  r->cfg_wave = cfg->wave;
  r->cfg_rsm = cfg->ring_smem;
  r->cfg_explicit = true;
  return SNC_B200_OK;
}

int snc_b200_autotune_ex(const snc_b200_graph* g, const snc_b200_inputs* in, const snc_lif* lif,
                         snc_launch_config* cand, int32_t max_cand, int32_t* n_cand, int32_t* best) {
  if (!g || !in || !lif) { set_error("null argument"); return SNC_B200_EINVAL; }
  Run r;
  int rc = create_run(g, in, 0, &r);
  if (rc) { free_run(&r); return rc; }
  const int B = std::max(1, in->B);
  // the candidates: every delivery mode on the plain path (small batches
  // only: it runs the samples one after another), on the sample-per-CTA tier
  // (when a sample fits one CTA; it has no bucket variant) and on the all-SM
  // tier over its block sizes, wave sizes and ring placements
  std::vector<snc_launch_config> cs;
  auto add = [&](int m, int p, int tier, int thr, int wave, int rsm) {
    snc_launch_config c{m, p, tier, thr, wave, rsm, 0.f};
    if (p == SNC_B200_PATH_PERSISTENT && check_shape(&r, m, tier, thr, wave, rsm) != SNC_B200_OK) {
      set_error("");
      return;
    }
    cs.push_back(c);
  };
  if (B <= 8)
    for (int m = SNC_B200_MODE_ATOMIC; m <= SNC_B200_MODE_SORT; ++m)
      add(m, SNC_B200_PATH_PLAIN, -1, 0, 0, -1);
  for (int m : {SNC_B200_MODE_ATOMIC, SNC_B200_MODE_SORT})
    if (check_shape(&r, m, 0, 0, 0, -1) == SNC_B200_OK) add(m, SNC_B200_PATH_PERSISTENT, 0, 0, 0, -1);
  set_error("");
  const int thr0 = std::max(512, std::min(768, (g->BS + 31) / 32 * 32));
  std::vector<int> thrs = {thr0};
  for (int t : {512, 768})
    if (t != thr0) thrs.push_back(t);
  std::vector<int> waves = {0};  // 0: as many samples as fit
  if (B > 1 && B <= 64) waves.push_back(1);
  const bool big = B > 64;  // bound the tuning time: default shape only
  for (int m = SNC_B200_MODE_ATOMIC; m <= SNC_B200_MODE_SORT; ++m)
    for (int rsm : (m == SNC_B200_MODE_ATOMIC ? std::vector<int>{0} : std::vector<int>{1, 0}))
      for (int wave : waves)
        for (int thr : thrs) {
          if (big && (thr != thr0 || wave != 0)) continue;
          add(m, SNC_B200_PATH_PERSISTENT, 1, thr, wave, rsm);
        }
  int bi = -1;
  for (size_t i = 0; i < cs.size(); ++i) {
    snc_launch_config& c = cs[i];
    r.cfg_tier = c.tier; r.cfg_threads = c.block_threads; r.cfg_wave = c.wave; r.cfg_rsm = c.ring_smem;
    r.cfg_explicit = true;
    float t = 0.f;
    for (int rep = 0; rep < 2; ++rep) {  // the first launch warms up
      rc = launch_run(&r, lif, c.mode, c.path, nullptr);
      if (!rc) rc = fetch_run(&r, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
      if (rc) break;
      t = r.last_ms;
    }
    if (rc) { free_run(&r); return rc; }
    c.ms = t;
    if (bi < 0 || t < cs[bi].ms) bi = (int)i;
  }
  free_run(&r);
  if (bi < 0) { set_error("autotune: no candidate"); return SNC_B200_EUNSUPPORTED; }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[tune_key(g, in)] = cs[bi];
  }
  if (n_cand) *n_cand = (int32_t)cs.size();
  if (best) *best = bi;
  if (cand)
    for (int i = 0; i < (int)cs.size() && i < max_cand; ++i) cand[i] = cs[i];
  return SNC_B200_OK;
}

int snc_b200_autotune_lookup(const snc_b200_graph* g, const snc_b200_inputs* in, snc_launch_config* out) {
  if (!g || !in) { set_error("null argument"); return SNC_B200_EINVAL; }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune_cache.find(tune_key(g, in));
  if (it == g_tune_cache.end()) return 0;
  if (out) *out = it->second;
  return 1;
}

int snc_b200_autotune(const snc_b200_graph* g, const snc_b200_inputs* in, const snc_lif* lif,
                      int* mode, int* path, int* block_threads) {
  snc_launch_config best{};
  int n = 0, bi = 0;
  std::vector<snc_launch_config> cs(64);
  int rc = snc_b200_autotune_ex(g, in, lif, cs.data(), (int)cs.size(), &n, &bi);
  if (rc) return rc;
  best = cs[bi];
  if (mode) *mode = best.mode;
  if (path) *path = best.path;
  if (block_threads)
    *block_threads = best.path == SNC_B200_PATH_PLAIN ? 512
                     : best.tier == 0 ? 1024
                     : best.block_threads > 0 ? best.block_threads
                                              : std::max(512, std::min(768, (g->BS + 31) / 32 * 32));
  return SNC_B200_OK;
}

}  // extern "C"
