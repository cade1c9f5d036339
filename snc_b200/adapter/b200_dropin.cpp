// Reference-side drop-in: the reference's own CUDA hooks implemented over the
// C ABI of libsnc_b200.so.
//
// Two builds of this file (snc_b200/adapter/Makefile):
//   default          the link-time swap described below: snc::cuda and
//                    snc::cudatrain ARE the B200 backend;
//   SNC_B200_BESIDE  against the reference's backend table extended by
//                    beside.py: this file defines only snc::b200 (the
//                    b200-atomic / b200-bucket / b200-sort backends), and the
//                    reference's own cuda_backend.cu and cuda_trainer.cu are
//                    linked unchanged beside it.
//
//   snc::cuda::available / snc::cuda::forward   include/snc/runtime.hpp:61-69
//   snc::cudatrain::*                           include/snc/cuda_trainer.hpp:26-57
//
// Linked in place of src/runtime/cuda_backend.cu and
// src/training/cuda_trainer.cu -- the same link-time swap the reference makes
// with its stubs (CMakeLists.txt:60-65) -- every caller of snc::forward with a
// cuda-* Backend (snc_bench, --compare-backends) and of cudatrain (snc_train
// --device cuda, snc_cotrain) runs on the B200 kernels without a source
// change.  cuda-atomic / cuda-bucket / cuda-sort select this backend's ATOMIC /
// BUCKET / SORT delivery; cuda-sort is bit-identical to the cpu backend.
//
// Behaviour kept from the reference: a forward that cannot run returns false
// (snc::forward then falls back to the CPU and reports used_backend = Cpu,
// src/runtime/cpu_backend.cpp:197-205); cudatrain::create returns nullptr when
// no device is usable.  Changed on purpose: the graph is uploaded once and
// cached (the reference re-uploads per call, cuda_backend.cu:247-285);
// minibatch inputs are host-encoded with snc::encode (same per-sample seeds
// as the CPU Trainer, src/training/trainer.cpp:225-226,257) instead of
// cuRAND draws, so every GPU run is reproducible.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <numeric>
#include <random>
#include <vector>

#include "snc/cuda_trainer.hpp"
#include "snc/dataset.hpp"
#include "snc/encoders.hpp"
#include "snc/runtime.hpp"
#include "snc/snn_graph.hpp"
#include "snc_b200.h"

static_assert(sizeof(snc::InputEvent) == sizeof(snc_input_event), "InputEvent layout");

namespace snc {

#ifndef SNC_B200_BESIDE
struct CudaTrainSession {
  const SNNGraph* g = nullptr;
  TrainConfig cfg;
  int batch = 1;
  snc_b200_graph* gh = nullptr;
  snc_b200_eprop* s = nullptr;
};
#endif

namespace {

snc_graph_view view_of(const SNNGraph& g) {
  snc_graph_view v;
  v.num_neurons = g.num_neurons;
  v.num_synapses = g.num_synapses();
  v.row_ptr = g.row_ptr.data();
  v.post_ids = g.post_ids.data();
  v.weights = g.weights.data();
  v.delays = g.delays.data();
  v.role = reinterpret_cast<const uint8_t*>(g.role.data());
  v.sign = g.sign.data();
  v.channel = g.channel.data();
  return v;
}

// Cheap fingerprint of a graph's contents (sizes, storage addresses and a
// strided sample of every array): a graph edited in place is re-uploaded.
uint64_t fingerprint(const SNNGraph& g) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](uint64_t x) { h = (h ^ x) * 1099511628211ull; };
  mix((uint64_t)g.num_neurons);
  mix((uint64_t)g.num_synapses());
  mix((uint64_t)(uintptr_t)g.post_ids.data());
  mix((uint64_t)(uintptr_t)g.weights.data());
  const size_t S = g.post_ids.size(), N = g.row_ptr.size();
  const size_t stride = std::max<size_t>(1, S / 4096);
  for (size_t i = 0; i < S; i += stride) {
    uint32_t wb;
    std::memcpy(&wb, &g.weights[i], 4);
    mix(((uint64_t)(uint32_t)g.post_ids[i] << 32) ^ wb ^ ((uint64_t)g.delays[i] << 20));
  }
  for (size_t i = 0; i < N; i += std::max<size_t>(1, N / 1024)) mix((uint64_t)g.row_ptr[i]);
  return h;
}

struct CacheEntry {
  const SNNGraph* g;
  uint64_t fp;
  snc_b200_graph* h;
};
std::mutex g_mu;
std::vector<CacheEntry> g_cache;  // small, most recent last

snc_b200_graph* cached_graph(const SNNGraph& g) {
  const uint64_t fp = fingerprint(g);
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto& e : g_cache)
    if (e.g == &g && e.fp == fp) return e.h;
  snc_graph_view v = view_of(g);
  snc_b200_graph* h = nullptr;
  if (snc_b200_graph_upload(&v, &h) != SNC_B200_OK) return nullptr;
  for (auto it = g_cache.begin(); it != g_cache.end();)
    if (it->g == &g) { snc_b200_graph_release(it->h); it = g_cache.erase(it); } else ++it;
  if (g_cache.size() >= 4) {
    snc_b200_graph_release(g_cache.front().h);
    g_cache.erase(g_cache.begin());
  }
  g_cache.push_back({&g, fp, h});
  return h;
}

int mode_of(Backend b) {
#ifdef SNC_B200_BESIDE
  if (b == Backend::B200Atomic) return SNC_B200_MODE_ATOMIC;
  if (b == Backend::B200Bucket) return SNC_B200_MODE_BUCKET;
#else
  if (b == Backend::CudaAtomic) return SNC_B200_MODE_ATOMIC;
  if (b == Backend::CudaBucket) return SNC_B200_MODE_BUCKET;
#endif
  return SNC_B200_MODE_SORT;
}

}  // namespace

#ifdef SNC_B200_BESIDE
namespace b200 {
#else
namespace cuda {
#endif

bool available() { return snc_b200_available() == 1; }

bool forward(const SNNGraph& g, const std::vector<InputEvent>& events, int num_steps,
             const LIFParams& lif, Backend variant, ForwardResult& out) {
  if (g.num_neurons == 0 || num_steps <= 0) return false;  // cuda_backend.cu:192
  snc_b200_graph* h = cached_graph(g);
  if (!h) return false;
  const snc_lif l{lif.threshold, lif.decay, lif.reset, lif.refractory, 0};
  std::vector<float> logits(std::max(0, g.num_output_channels));
  snc_run_stats st{};
  const int rc = snc_b200_forward(h, nullptr, reinterpret_cast<const snc_input_event*>(events.data()),
                                  events.size(), num_steps, &l, mode_of(variant), logits.data(), &st);
  if (rc != SNC_B200_OK) return false;
  out.logits = std::move(logits);
  out.stats.spikes = st.spikes;
  out.stats.synaptic_events = st.synaptic_events;
  out.stats.overflow = st.overflow;
  out.stats.ms = st.ms;
  out.used_backend = variant;
  return true;
}

#ifdef SNC_B200_BESIDE
}  // namespace b200
#else
}  // namespace cuda

namespace cudatrain {

// Encoding happens on the host, so every encoder works on the GPU path.
bool available(const TrainConfig&) { return snc_b200_available() == 1; }

CudaTrainSession* create(const SNNGraph& g, const TrainConfig& cfg, int batch) {
  if (!available(cfg)) return nullptr;
  auto* s = new CudaTrainSession();
  s->g = &g;
  s->cfg = cfg;
  s->batch = std::max(1, batch);
  // initial feedback matrix and weights drawn as cuda_trainer.cu:284-290
  const int oc = std::max(1, g.num_output_channels);
  int n_internal = 0;
  for (int i = 0; i < g.num_neurons; ++i)
    if (g.role[i] == GraphRole::INTERNAL) ++n_internal;
  std::mt19937_64 rng(cfg.seed);
  std::normal_distribution<float> bn(0.0f, cfg.feedback_scale);
  std::vector<float> bmat((size_t)std::max(1, n_internal) * oc, 0.0f);
  for (size_t k = 0; k < (size_t)n_internal * oc; ++k) bmat[k] = bn(rng);
  std::uniform_real_distribution<float> wu(0.0f, cfg.w_init);
  std::vector<float> w(g.num_synapses());
  for (float& x : w) x = wu(rng);
  snc_graph_view v = view_of(g);
  snc_eprop_cfg ec{cfg.lr, cfg.w_max, cfg.surrogate_scale, cfg.lif.decay,
                   cfg.train_hidden ? 1 : 0, SNC_B200_MODE_SORT};
  const snc_lif l{cfg.lif.threshold, cfg.lif.decay, cfg.lif.reset, cfg.lif.refractory, 0};
  if (snc_b200_graph_upload(&v, &s->gh) != SNC_B200_OK ||
      snc_b200_eprop_create(s->gh, &l, &ec, s->batch, w.data(), bmat.data(), &s->s) != SNC_B200_OK) {
    destroy(s);
    return nullptr;
  }
  return s;
}

void destroy(CudaTrainSession* s) {
  if (!s) return;
  snc_b200_eprop_release(s->s);
  snc_b200_graph_release(s->gh);
  delete s;
}

void set_weights(CudaTrainSession* s, const std::vector<float>& w) {
  if (s && static_cast<int>(w.size()) == s->g->num_synapses()) snc_b200_eprop_set_weights(s->s, w.data());
}

std::vector<float> get_weights(const CudaTrainSession* s) {
  std::vector<float> w(s ? s->g->num_synapses() : 0);
  if (s) snc_b200_eprop_get_weights(s->s, w.data());
  return w;
}

namespace {

// Encode samples order[off .. off+bs) with the CPU Trainer's seeds and run
// them as one minibatch.  Returns the counts [bs][oc].
bool run(CudaTrainSession* s, const Dataset& d, const std::vector<int>& order, int off, int bs,
         bool train, int epoch, std::vector<float>& counts, snc_run_stats& st) {
  const TrainConfig& cfg = s->cfg;
  const SNNGraph& g = *s->g;
  std::vector<InputEvent> ev;
  std::vector<int32_t> steps(bs, cfg.num_steps), labels(bs);
  for (int b = 0; b < bs; ++b) {
    const int idx = order[off + b];
    const uint64_t seed = train ? cfg.seed ^ (0xD1B54A32D192ED03ULL * (uint64_t)(idx + 1)) ^
                                      (static_cast<uint64_t>(epoch) << 32)
                                : cfg.seed ^ (0xD1B54A32D192ED03ULL * (uint64_t)(idx + 1));
    auto e = encode(cfg.encoder, d.x[idx].data(), g.num_input_channels, cfg.num_steps, cfg.enc,
                    seed, b);
    ev.insert(ev.end(), e.begin(), e.end());
    labels[b] = d.y[idx];
  }
  const int oc = std::max(1, g.num_output_channels);
  counts.assign((size_t)bs * oc, 0.0f);
  std::vector<float> c((size_t)bs * std::max(1, g.num_output_channels));
  const int rc = snc_b200_eprop_batch(s->s, reinterpret_cast<const snc_input_event*>(ev.data()),
                                      ev.size(), bs, steps.data(), labels.data(), train ? 1 : 0,
                                      c.data(), &st);
  if (rc != SNC_B200_OK) return false;
  for (int b = 0; b < bs; ++b)
    for (int k = 0; k < g.num_output_channels; ++k)
      counts[(size_t)b * oc + k] = c[(size_t)b * g.num_output_channels + k];
  return true;
}

int argmax(const float* c, int oc) {
  int best = 0;
  for (int k = 1; k < oc; ++k)
    if (c[k] > c[best]) best = k;
  return best;
}

}  // namespace

double evaluate(CudaTrainSession* s, const Dataset& d) {
  if (!s || d.size() == 0) return 0.0;
  std::vector<int> order(d.size());
  std::iota(order.begin(), order.end(), 0);
  const int oc = std::max(1, s->g->num_output_channels);
  int correct = 0;
  std::vector<float> counts;
  snc_run_stats st{};
  for (int off = 0; off < d.size(); off += s->batch) {
    const int bs = std::min(s->batch, d.size() - off);
    if (!run(s, d, order, off, bs, false, 0, counts, st)) return 0.0;
    for (int b = 0; b < bs; ++b)
      if (argmax(&counts[(size_t)b * oc], oc) == d.y[order[off + b]]) ++correct;
  }
  return static_cast<double>(correct) / d.size();
}

EpochStats train_epoch(CudaTrainSession* s, const Dataset& train, const Dataset& test, int epoch) {
  EpochStats out;
  if (!s || train.size() == 0) return out;
  std::vector<int> order(train.size());
  std::iota(order.begin(), order.end(), 0);
  std::mt19937_64 rng(0x9e3779b97f4a7c15ULL * (epoch + 1));  // cuda_trainer.cu:456-457
  std::shuffle(order.begin(), order.end(), rng);
  const int oc = std::max(1, s->g->num_output_channels);
  double loss_sum = 0.0;
  int correct = 0;
  std::vector<float> counts;
  for (int off = 0; off < train.size(); off += s->batch) {
    const int bs = std::min(s->batch, train.size() - off);
    snc_run_stats st{};
    if (!run(s, train, order, off, bs, true, epoch, counts, st)) return out;
    out.spikes += st.spikes;
    out.synaptic_events += st.synaptic_events;
    for (int b = 0; b < bs; ++b) {
      const float* c = &counts[(size_t)b * oc];
      const int y = train.y[order[off + b]];
      float mx = c[0];
      for (int k = 1; k < oc; ++k) mx = std::max(mx, c[k]);
      double sum = 0.0;
      for (int k = 0; k < oc; ++k) sum += std::exp(c[k] - mx);
      loss_sum += -(c[y] - mx) + std::log(sum);
      if (argmax(c, oc) == y) ++correct;
    }
  }
  out.loss = loss_sum / train.size();
  out.train_acc = static_cast<double>(correct) / train.size();
  out.test_acc = evaluate(s, test);
  out.energy = 1.0 * out.spikes + 0.2 * out.synaptic_events;
  return out;
}

void reset_stats(CudaTrainSession* s) {
  if (s) snc_b200_eprop_reset_stats(s->s);
}

void collect_stats(const CudaTrainSession* s, std::vector<long long>& syn, std::vector<long long>& neur) {
  syn.assign(s ? s->g->num_synapses() : 0, 0);
  neur.assign(s ? s->g->num_neurons : 0, 0);
  if (!s) return;
  std::vector<int64_t> a(syn.size()), b(neur.size());
  snc_b200_eprop_collect_stats(s->s, a.data(), b.data());
  for (size_t i = 0; i < a.size(); ++i) syn[i] = a[i];
  for (size_t i = 0; i < b.size(); ++i) neur[i] = b[i];
}

}  // namespace cudatrain
#endif  // SNC_B200_BESIDE
}  // namespace snc
