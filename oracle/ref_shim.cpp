// ref_shim.cpp -- extern "C" entry points into the UNCHANGED reference code.
//
// TEST INFRASTRUCTURE ONLY.  Compiled together with the reference's own
// sources (src/runtime/cpu_backend.cpp, src/training/{encoders,trainer,
// datasets}.cpp, src/graph/snn_graph.cpp, ...) into oracle/_ref/ by
// oracle/Makefile.  tests/ use it to pin the C restatement in snc_oracle.c,
// tests/golden/make_golden.py uses it to write golden vectors, and bench.py's
// reference arm times the reference CPU backend through it.
//
// Every function here only marshals plain arrays into the reference's types
// and calls the reference API:
//   snc::forward               include/snc/runtime.hpp:57-58
//   snc::encode                include/snc/encoders.hpp:42-45
//   snc::make_static_snc etc.  include/snc/snn_graph.hpp:118-132
//   snc::make_synthetic        include/snc/dataset.hpp:27
//   snc::Trainer               include/snc/trainer.hpp:59-107
//   snc::Connectome            include/snc/connectome.hpp:58-101
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "snc/connectome.hpp"
#include "snc/dataset.hpp"
#include "snc/encoders.hpp"
#include "snc/runtime.hpp"
#include "snc/snn_graph.hpp"
#include "snc/trainer.hpp"

using namespace snc;

namespace {

SNNGraph* from_arrays(int n, int s, const int32_t* row_ptr, const int32_t* post,
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

SNNGraph* g_last_generated = nullptr;

}  // namespace

extern "C" {

void* ref_graph_create(int n, int s, const int32_t* row_ptr, const int32_t* post,
                       const float* w, const int32_t* delays, const uint8_t* role,
                       const int8_t* sign, const int32_t* channel) {
  return from_arrays(n, s, row_ptr, post, w, delays, role, sign, channel);
}

void ref_graph_destroy(void* g) { delete static_cast<SNNGraph*>(g); }

int ref_graph_validate(void* g, char* err, int err_len) {
  std::string e;
  bool ok = static_cast<SNNGraph*>(g)->validate(e);
  if (err && err_len > 0) {
    std::strncpy(err, e.c_str(), static_cast<size_t>(err_len - 1));
    err[err_len - 1] = 0;
  }
  return ok ? 1 : 0;
}

// snc::forward on one sample.  backend: 0 cpu, 1 openmp.
// Returns RunStats.ms (the reference's own loop timing).
double ref_forward(void* gp, const InputEvent* ev, int64_t n_ev, int num_steps,
                   float threshold, float decay, float reset, int refractory,
                   int backend, float* logits, int64_t* spikes, int64_t* events) {
  const SNNGraph& g = *static_cast<SNNGraph*>(gp);
  std::vector<InputEvent> events_v(ev, ev + n_ev);
  LIFParams lif;
  lif.threshold = threshold;
  lif.decay = decay;
  lif.reset = reset;
  lif.refractory = refractory;
  ForwardResult r = forward(g, events_v, num_steps, lif,
                            backend == 1 ? Backend::OpenMP : Backend::Cpu);
  for (size_t c = 0; c < r.logits.size(); ++c) logits[c] = r.logits[c];
  *spikes = r.stats.spikes;
  *events = r.stats.synaptic_events;
  return r.stats.ms;
}

// snc::encode.  Returns the number of events written (capacity-limited).
int64_t ref_encode(int enc, const float* features, int n_channels, int num_steps,
                   float gain, float max_rate, float threshold, uint64_t seed,
                   int sample_id, InputEvent* out, int64_t capacity) {
  EncoderParams p;
  p.gain = gain;
  p.max_rate = max_rate;
  p.threshold = threshold;
  std::vector<InputEvent> ev =
      encode(static_cast<Encoder>(enc), features, n_channels, num_steps, p, seed, sample_id);
  int64_t n = static_cast<int64_t>(ev.size());
  if (out) std::memcpy(out, ev.data(), sizeof(InputEvent) * static_cast<size_t>(n < capacity ? n : capacity));
  return n;
}

// Generators (structure: 0 dense, 1 random-sparse, 2 static-snc), as
// snc_bench's build_graph (src/bench/snc_bench.cpp:123-134).  The graph is
// kept until the next call; sizes come back first, arrays via ref_last_graph.
void ref_generate(int structure, const int32_t* layers, int n_layers, int synapse_budget,
                  float weight, int delay, float inhib, uint64_t seed, int* n_out, int* s_out) {
  std::vector<int> L(layers, layers + n_layers);
  delete g_last_generated;
  g_last_generated = new SNNGraph(
      structure == 0   ? make_dense(L, weight, delay)
      : structure == 1 ? make_random_sparse(L, synapse_budget, weight, delay, inhib, seed)
                       : make_static_snc(L, synapse_budget, weight, delay, inhib, seed));
  *n_out = g_last_generated->num_neurons;
  *s_out = g_last_generated->num_synapses();
}

void ref_last_graph(int32_t* row_ptr, int32_t* post, float* w, int32_t* delays,
                    uint8_t* role, int8_t* sign, int32_t* channel) {
  const SNNGraph& g = *g_last_generated;
  std::memcpy(row_ptr, g.row_ptr.data(), sizeof(int32_t) * g.row_ptr.size());
  std::memcpy(post, g.post_ids.data(), sizeof(int32_t) * g.post_ids.size());
  std::memcpy(w, g.weights.data(), sizeof(float) * g.weights.size());
  std::memcpy(delays, g.delays.data(), sizeof(int32_t) * g.delays.size());
  for (int i = 0; i < g.num_neurons; ++i) {
    role[i] = static_cast<uint8_t>(g.role[i]);
    sign[i] = g.sign[i];
    channel[i] = g.channel[i];
  }
}

// snc::make_synthetic -> features [n][dim], labels [n].
void ref_make_synthetic(int n, int dim, int classes, float noise, uint64_t seed,
                        float* x, int32_t* y) {
  Dataset d = make_synthetic(n, dim, classes, noise, seed);
  for (int i = 0; i < n; ++i) {
    std::memcpy(x + static_cast<size_t>(i) * dim, d.x[i].data(), sizeof(float) * dim);
    y[i] = d.y[i];
  }
}

// One epoch of the reference per-sample e-prop Trainer on a one-sample
// dataset (train and test both = that sample), so the caller can replay the
// exact update.  Writes the trainer's weights before and after the epoch, the
// events the trainer encoded for that sample (same encode() call and seed as
// Trainer::train_epoch, src/training/trainer.cpp:223-236), and the random
// feedback matrix drawn the way the Trainer's constructor draws it
// (src/training/trainer.cpp:14-40), using the same library generators.
int64_t ref_trainer_one_sample(void* gp, int num_steps, float threshold, float decay,
                               float reset, int refractory, int encoder, float gain,
                               float max_rate, float lr, float w_init, float w_max,
                               float surrogate_scale, float feedback_scale,
                               int train_hidden, uint64_t seed, const float* x, int label,
                               int epoch, float* w_before, float* w_after, float* bmat,
                               InputEvent* ev_out, int64_t ev_capacity) {
  const SNNGraph& g = *static_cast<SNNGraph*>(gp);
  TrainConfig cfg;
  cfg.num_steps = num_steps;
  cfg.lif.threshold = threshold;
  cfg.lif.decay = decay;
  cfg.lif.reset = reset;
  cfg.lif.refractory = refractory;
  cfg.encoder = static_cast<Encoder>(encoder);
  cfg.enc.gain = gain;
  cfg.enc.max_rate = max_rate;
  cfg.lr = lr;
  cfg.w_init = w_init;
  cfg.w_max = w_max;
  cfg.surrogate_scale = surrogate_scale;
  cfg.feedback_scale = feedback_scale;
  cfg.train_hidden = train_hidden != 0;
  cfg.seed = seed;
  Trainer tr(g, cfg);
  std::memcpy(w_before, tr.weights().data(), sizeof(float) * tr.weights().size());

  // Replicate the constructor's draws to expose B (it has no getter).
  {
    std::mt19937_64 rng(cfg.seed);
    std::uniform_real_distribution<float> wu(0.0f, cfg.w_init);
    for (int s = 0; s < g.num_synapses(); ++s) (void)wu(rng);
    int n_internal = 0;
    for (int i = 0; i < g.num_neurons; ++i)
      if (g.role[i] == GraphRole::INTERNAL) ++n_internal;
    const int classes = std::max(1, g.num_output_channels);
    std::normal_distribution<float> bn(0.0f, cfg.feedback_scale);
    for (int k = 0; k < n_internal * classes; ++k) bmat[k] = bn(rng);
  }

  Dataset d;
  d.dim = g.num_input_channels;
  d.classes = std::max(1, g.num_output_channels);
  d.x.push_back(std::vector<float>(x, x + d.dim));
  d.y.push_back(label);
  const uint64_t sseed =
      cfg.seed ^ (0xD1B54A32D192ED03ULL * 1ULL) ^ (static_cast<uint64_t>(epoch) << 32);
  std::vector<InputEvent> ev = encode(cfg.encoder, x, g.num_input_channels, num_steps, cfg.enc, sseed);
  const int64_t n = static_cast<int64_t>(ev.size());
  if (ev_out)
    std::memcpy(ev_out, ev.data(), sizeof(InputEvent) * static_cast<size_t>(n < ev_capacity ? n : ev_capacity));
  tr.train_epoch(d, d, epoch);
  std::memcpy(w_after, tr.weights().data(), sizeof(float) * tr.weights().size());
  return n;
}

// ---- Connectome (the co-training loop's structural state) -------------------

void* ref_con_layered_local(const int32_t* layers, int n_layers, int budget, int delay, float w_init,
                            uint64_t seed) {
  std::vector<int> l(layers, layers + n_layers);
  return new Connectome(Connectome::layered_local(l, budget, delay, w_init, seed));
}

void ref_con_destroy(void* h) { delete static_cast<Connectome*>(h); }

int ref_con_num_synapses(void* h) { return static_cast<Connectome*>(h)->num_synapses(); }

// to_graph() CSR (row_ptr [n+1], post, delay) and edge_weights() (signed).
int ref_con_read(void* h, int32_t* row_ptr, int32_t* post, int32_t* delay, float* w_signed) {
  auto* c = static_cast<Connectome*>(h);
  const SNNGraph g = c->to_graph();
  const std::vector<float> w = c->edge_weights();
  std::memcpy(row_ptr, g.row_ptr.data(), sizeof(int32_t) * g.row_ptr.size());
  std::memcpy(post, g.post_ids.data(), sizeof(int32_t) * g.post_ids.size());
  std::memcpy(delay, g.delays.data(), sizeof(int32_t) * g.delays.size());
  std::memcpy(w_signed, w.data(), sizeof(float) * w.size());
  return g.num_neurons;
}

void ref_con_set_weights(void* h, const float* w, int n) {
  static_cast<Connectome*>(h)->set_edge_weights(std::vector<float>(w, w + n));
}

// structural_update with the given activity and configuration; out[3] =
// pruned, grown, synapses.
void ref_con_update(void* h, const int64_t* fires, int n_fires, int grow_per_epoch, int delay,
                    float w_grow_init, float locality_window, int protect_rounds,
                    int max_attempts_mult, int reward_modulated, float reward_chance,
                    float reward_floor, float reward, int32_t* out) {
  ActivityStats st;
  st.neuron_fires.assign(fires, fires + n_fires);
  StructConfig cfg;
  cfg.grow_per_epoch = grow_per_epoch;
  cfg.delay = delay;
  cfg.w_grow_init = w_grow_init;
  cfg.locality_window = locality_window;
  cfg.protect_rounds = protect_rounds;
  cfg.max_attempts_mult = max_attempts_mult;
  cfg.reward_modulated = reward_modulated != 0;
  cfg.reward_chance = reward_chance;
  cfg.reward_floor = reward_floor;
  const StructReport r = static_cast<Connectome*>(h)->structural_update(st, cfg, reward);
  out[0] = r.pruned;
  out[1] = r.grown;
  out[2] = r.synapses;
}

}  // extern "C"
