// ref_gpu_shim.cpp -- extern "C" entry points into the reference built WITH
// its CUDA backend: the unchanged src/runtime/cuda_backend.cu and
// src/training/cuda_trainer.cu compiled by nvcc for sm_100a, linked with the
// reference's unchanged CPU sources (snc_b200/adapter/Makefile,
// _build/libsncref_gpu.so).  It lets the benchmark time the reference's own
// GPU kernels on the same B200 and the same inputs as this backend:
//
//   snc::forward with Backend::CudaAtomic / CudaBucket / CudaSort
//       include/snc/runtime.hpp:57-58, src/runtime/cuda_backend.cu:186-361
//   snc::cudatrain::create / train_epoch / destroy
//       include/snc/cuda_trainer.hpp:26-57, src/training/cuda_trainer.cu
//
// Only marshalling lives here; no B200 code is linked into this library.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include "snc/cuda_trainer.hpp"
#include "snc/dataset.hpp"
#include "snc/encoders.hpp"
#include "snc/runtime.hpp"
#include "snc/snn_graph.hpp"

using namespace snc;

extern "C" {

void* refgpu_graph_create(int n, int s, const int32_t* row_ptr, const int32_t* post,
                          const float* w, const int32_t* delays, const uint8_t* role,
                          const int8_t* sign, const int32_t* channel) {
  auto* g = new SNNGraph();
  g->num_neurons = n;
  g->row_ptr.assign(row_ptr, row_ptr + n + 1);
  g->post_ids.assign(post, post + s);
  g->weights.assign(w, w + s);
  g->delays.assign(delays, delays + s);
  g->branch_ids.assign(s, 0);
  g->role.resize(n);
  g->sign.resize(n);
  g->channel.assign(channel, channel + n);
  for (int i = 0; i < n; ++i) {
    g->role[i] = static_cast<GraphRole>(role[i]);
    g->sign[i] = sign[i];
  }
  g->rebuild_io_index();
  return g;
}

void refgpu_graph_destroy(void* g) { delete static_cast<SNNGraph*>(g); }

int refgpu_available(void) { return cuda::available() ? 1 : 0; }

// snc::forward on one sample with backend 2 cuda-atomic, 3 cuda-bucket,
// 4 cuda-sort (the reference's enum values).  Writes the logits, spike and
// event counts, the backend actually used (a failed GPU run falls back to
// the CPU) and the wall time of the whole call (graph upload, schedule
// flattening, loop, read-back, frees); returns RunStats.ms (the loop alone).
double refgpu_forward(void* gp, const InputEvent* ev, int64_t n_ev, int num_steps, float threshold,
                      float decay, float reset, int refractory, int backend, float* logits,
                      int64_t* spikes, int64_t* events, int* used_backend, double* wall_ms) {
  const SNNGraph& g = *static_cast<SNNGraph*>(gp);
  std::vector<InputEvent> events_v(ev, ev + n_ev);
  LIFParams lif;
  lif.threshold = threshold;
  lif.decay = decay;
  lif.reset = reset;
  lif.refractory = refractory;
  const auto t0 = std::chrono::steady_clock::now();
  ForwardResult r = forward(g, events_v, num_steps, lif, static_cast<Backend>(backend));
  const auto t1 = std::chrono::steady_clock::now();
  for (size_t c = 0; c < r.logits.size(); ++c) logits[c] = r.logits[c];
  *spikes = r.stats.spikes;
  *events = r.stats.synaptic_events;
  *used_backend = static_cast<int>(r.used_backend);
  *wall_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  return r.stats.ms;
}

// cudatrain on a dataset of n samples x dim features (x in [0, 1]) with
// labels y: creates a session (batch `batch`), trains `epochs` epochs and
// returns the wall time of the train_epoch calls in ms (session creation
// excluded), or -1 when the GPU trainer is unavailable.  Poisson encoding
// with max_rate, num_steps steps per sample, the reference's own defaults
// otherwise.  spikes / events: totals of the last epoch.
double refgpu_train(void* gp, int num_steps, float threshold, float decay, float reset,
                    int refractory, float max_rate, float lr, float surrogate_scale, int n,
                    int dim, int classes, const float* x, const int32_t* y, int batch, int epochs,
                    int64_t* spikes, int64_t* events) {
  const SNNGraph& g = *static_cast<SNNGraph*>(gp);
  TrainConfig cfg;
  cfg.num_steps = num_steps;
  cfg.lif.threshold = threshold;
  cfg.lif.decay = decay;
  cfg.lif.reset = reset;
  cfg.lif.refractory = refractory;
  cfg.encoder = Encoder::Poisson;
  cfg.enc.max_rate = max_rate;
  cfg.lr = lr;
  cfg.surrogate_scale = surrogate_scale;
  if (!cudatrain::available(cfg)) return -1.0;
  Dataset d, empty;
  d.dim = empty.dim = dim;
  d.classes = empty.classes = classes;
  for (int i = 0; i < n; ++i) {
    d.x.emplace_back(x + (size_t)i * dim, x + (size_t)(i + 1) * dim);
    d.y.push_back(y[i]);
  }
  CudaTrainSession* s = cudatrain::create(g, cfg, batch);
  if (!s) return -1.0;
  const auto t0 = std::chrono::steady_clock::now();
  EpochStats st;
  for (int e = 0; e < epochs; ++e) st = cudatrain::train_epoch(s, d, empty, e);
  const auto t1 = std::chrono::steady_clock::now();
  cudatrain::destroy(s);
  *spikes = st.spikes;
  *events = st.synaptic_events;
  return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

}  // extern "C"
