/*
 * snc_oracle.c -- CPU restatement of the SNC spiking substrate's hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA backend in
 * snc_b200/ is compared against; it is loaded only by tests/, by
 * __graft_entry__.smoke() and by bench.py's cpu_baseline leg.  The product
 * path never links or calls it.
 *
 * Each function restates one piece of the reference (blazer502/snc) in plain
 * C, citing the file:line it follows.  Floating-point expressions are written
 * so that every IEEE operation of the reference appears here in the same order
 * (build with -ffp-contract=off so no fused multiply-add is formed): the spike
 * rasters are then bit-identical to the reference's serial CPU backend built
 * with the same flag.
 *
 * Two extensions beyond the reference are restated here too, and are checked
 * against the unchanged reference wherever both apply:
 *   - reset_mode = 1 (subtractive reset: v -= threshold on a spike); the
 *     reference only resets to a constant (include/snc/runtime.hpp:37);
 *   - per-sample step counts in the batched forward (the reference runs one
 *     sample per forward() call, include/snc/runtime.hpp:57-58).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int32_t num_neurons;
  int32_t num_synapses;
  const int32_t* row_ptr;  /* [N+1] */
  const int32_t* post_ids; /* [S] */
  const float* weights;    /* [S] */
  const int32_t* delays;   /* [S] */
  const uint8_t* role;     /* [N] 0 internal, 1 input, 2 output */
  const int8_t* sign;      /* [N] +1 / -1 */
  const int32_t* channel;  /* [N] */
} orc_graph;

typedef struct {
  int32_t sample_id;
  int32_t channel_id;
  int32_t time;
  float amplitude;
} orc_event;

typedef struct {
  float threshold;
  float decay;
  float reset;
  int32_t refractory;
  int32_t reset_mode; /* 0: v = reset (reference), 1: v -= threshold */
} orc_lif;

enum { ORC_OK = 0, ORC_EINVAL = -1, ORC_ENOMEM = -3 };

/* ---- graph-derived views --------------------------------------------------
 * SNNGraph::rebuild_io_index (src/graph/snn_graph.cpp:13-28): input/output
 * neuron lists in ascending id order; channel counts are 1 + max channel. */
static void io_counts(const orc_graph* g, int* nic, int* noc) {
  int max_in = -1, max_out = -1;
  for (int i = 0; i < g->num_neurons; ++i) {
    if (g->role[i] == 1 && g->channel[i] > max_in) max_in = g->channel[i];
    if (g->role[i] == 2 && g->channel[i] > max_out) max_out = g->channel[i];
  }
  *nic = max_in + 1;
  *noc = max_out + 1;
}

int orc_num_output_channels(const orc_graph* g) {
  int nic, noc;
  io_counts(g, &nic, &noc);
  return noc;
}

int orc_ring_len(const orc_graph* g) {
  /* cpu_backend.cpp:77-80: ring one past the largest delay (min max_delay 1). */
  int max_delay = 1;
  for (int s = 0; s < g->num_synapses; ++s)
    if (g->delays[s] > max_delay) max_delay = g->delays[s];
  return max_delay + 1;
}

/* build_schedule (src/runtime/cpu_backend.cpp:43-65): resolve every event's
 * channel to the INPUT neurons of that channel (ascending id), keep events
 * with time in [0,T) and a valid channel, grouped per step in event order.
 * Output is CSR by step: step_ptr[T+1], nid[], amp[]. */
typedef struct {
  int* step_ptr;
  int* nid;
  float* amp;
} schedule;

static void free_schedule(schedule* s) {
  free(s->step_ptr);
  free(s->nid);
  free(s->amp);
}

static int build_schedule(const orc_graph* g, const orc_event* ev, size_t n_ev,
                          int sample, int T, schedule* out) {
  int nic, noc;
  io_counts(g, &nic, &noc);
  /* channel -> input neurons, CSR */
  int* cptr = (int*)calloc((size_t)(nic > 0 ? nic : 0) + 1, sizeof(int));
  int* cids = NULL;
  int n_in = 0;
  for (int i = 0; i < g->num_neurons; ++i)
    if (g->role[i] == 1) {
      int c = g->channel[i];
      if (c >= 0 && c < nic) { cptr[c + 1]++; ++n_in; }
    }
  for (int c = 0; c < nic; ++c) cptr[c + 1] += cptr[c];
  cids = (int*)malloc(sizeof(int) * (size_t)(n_in > 0 ? n_in : 1));
  int* cfill = (int*)calloc((size_t)(nic > 0 ? nic : 1), sizeof(int));
  for (int i = 0; i < g->num_neurons; ++i)
    if (g->role[i] == 1) {
      int c = g->channel[i];
      if (c >= 0 && c < nic) cids[cptr[c] + cfill[c]++] = i;
    }
  free(cfill);

  out->step_ptr = (int*)calloc((size_t)T + 1, sizeof(int));
  size_t total = 0;
  for (size_t k = 0; k < n_ev; ++k) {
    const orc_event* e = &ev[k];
    if (sample >= 0 && e->sample_id != sample) continue;
    if (e->time < 0 || e->time >= T) continue;
    if (e->channel_id < 0 || e->channel_id >= nic) continue;
    int fan = cptr[e->channel_id + 1] - cptr[e->channel_id];
    out->step_ptr[e->time + 1] += fan;
    total += (size_t)fan;
  }
  for (int t = 0; t < T; ++t) out->step_ptr[t + 1] += out->step_ptr[t];
  out->nid = (int*)malloc(sizeof(int) * (total ? total : 1));
  out->amp = (float*)malloc(sizeof(float) * (total ? total : 1));
  int* fill = (int*)calloc((size_t)T + 1, sizeof(int));
  for (size_t k = 0; k < n_ev; ++k) {
    const orc_event* e = &ev[k];
    if (sample >= 0 && e->sample_id != sample) continue;
    if (e->time < 0 || e->time >= T) continue;
    if (e->channel_id < 0 || e->channel_id >= nic) continue;
    for (int q = cptr[e->channel_id]; q < cptr[e->channel_id + 1]; ++q) {
      int pos = out->step_ptr[e->time] + fill[e->time]++;
      out->nid[pos] = cids[q];
      out->amp[pos] = e->amplitude;
    }
  }
  free(fill);
  free(cptr);
  free(cids);
  return ORC_OK;
}

/* The drive run_cpu injects at each step (cpu_backend.cpp:85-95 adds every
 * scheduled amplitude into a zeroed per-step buffer in schedule order):
 * per step, the driven neurons in ascending id with their summed drive.
 * step_ptr [T+1]; nid / ext hold at most cap entries.  Returns the number of
 * entries, or -1 when cap is too small. */
long long orc_schedule_merged(const orc_graph* g, const orc_event* ev, size_t n_ev, int sample,
                              int T, int* step_ptr, int* nid, float* ext, long long cap) {
  schedule sch;
  build_schedule(g, ev, n_ev, sample, T, &sch);
  const int N = g->num_neurons;
  float* acc = (float*)calloc((size_t)(N > 0 ? N : 1), sizeof(float));
  unsigned char* hit = (unsigned char*)calloc((size_t)(N > 0 ? N : 1), 1);
  long long n = 0;
  int fail = 0;
  step_ptr[0] = 0;
  for (int t = 0; t < T && !fail; ++t) {
    for (int k = sch.step_ptr[t]; k < sch.step_ptr[t + 1]; ++k) {
      acc[sch.nid[k]] += sch.amp[k];
      hit[sch.nid[k]] = 1;
    }
    for (int i = 0; i < N; ++i)
      if (hit[i]) {
        if (n >= cap) { fail = 1; break; }
        nid[n] = i;
        ext[n] = acc[i];
        ++n;
        acc[i] = 0.0f;
        hit[i] = 0;
      }
    step_ptr[t + 1] = (int)n;
  }
  free(acc);
  free(hit);
  free_schedule(&sch);
  return fail ? -1 : n;
}

/* run_cpu, serial branch (src/runtime/cpu_backend.cpp:67-191).
 *  logits   [noc]           summed output spike counts per channel
 *  raster   [T][ceil(N/32)] bit j of word (t, i/32) set when neuron i fired at t
 *  v_out    [N]             membrane potential after the last step
 * raster / v_out may be NULL. */
/* ro_decay >= 0: OUTPUT neurons with a channel are leaky readout units
 * (python/snc/shd_model.py:139-140,147 on the substrate): v = v * ro_decay +
 * ext + slot, never firing; logits[channel] = sum, ascending id, of v / T. */
static int forward_ro(const orc_graph* g, const orc_event* ev, size_t n_ev, int sample, int T,
                      const orc_lif* lif, float ro_decay, float* logits, int64_t* spikes_out,
                      int64_t* events_out, uint32_t* raster, float* v_out);

int orc_forward(const orc_graph* g, const orc_event* ev, size_t n_ev, int sample,
                int T, const orc_lif* lif, float* logits, int64_t* spikes_out,
                int64_t* events_out, uint32_t* raster, float* v_out) {
  return forward_ro(g, ev, n_ev, sample, T, lif, -1.0f, logits, spikes_out, events_out, raster, v_out);
}

static int forward_ro(const orc_graph* g, const orc_event* ev, size_t n_ev, int sample, int T,
                      const orc_lif* lif, float ro_decay, float* logits, int64_t* spikes_out,
                      int64_t* events_out, uint32_t* raster, float* v_out) {
  const int n = g->num_neurons;
  int nic, noc;
  io_counts(g, &nic, &noc);
  if (logits)
    for (int c = 0; c < noc; ++c) logits[c] = 0.0f;
  if (spikes_out) *spikes_out = 0;
  if (events_out) *events_out = 0;
  if (n <= 0 || T <= 0) return ORC_OK;
  const int W = (n + 31) / 32;
  if (raster) memset(raster, 0, sizeof(uint32_t) * (size_t)W * (size_t)T);

  const int ring_len = orc_ring_len(g);
  float* v = (float*)calloc((size_t)n, sizeof(float));
  float* ext = (float*)calloc((size_t)n, sizeof(float));
  int* refr = (int*)calloc((size_t)n, sizeof(int));
  float* ring = (float*)calloc((size_t)ring_len * (size_t)n, sizeof(float));
  int* fired = (int*)malloc(sizeof(int) * (size_t)n);
  if (!v || !ext || !refr || !ring || !fired) {
    free(v); free(ext); free(refr); free(ring); free(fired);
    return ORC_ENOMEM;
  }
  schedule sch;
  build_schedule(g, ev, n_ev, sample, T, &sch);

  int64_t spikes = 0, syn_events = 0;
  for (int t = 0; t < T; ++t) {
    float* slot = &ring[(size_t)(t % ring_len) * (size_t)n];
    /* cpu_backend.cpp:99 -- external drive, event order */
    for (int k = sch.step_ptr[t]; k < sch.step_ptr[t + 1]; ++k)
      ext[sch.nid[k]] += sch.amp[k];
    /* cpu_backend.cpp:129-143 -- integrate / fire / reset / refractory */
    int nf = 0;
    for (int i = 0; i < n; ++i) {
      if (ro_decay >= 0.0f && g->role[i] == 2 && g->channel[i] >= 0) {
        v[i] = v[i] * ro_decay + ext[i] + slot[i];
      } else if (refr[i] > 0) {
        --refr[i];
        v[i] = lif->reset;
      } else {
        v[i] = v[i] * lif->decay + ext[i] + slot[i];
        if (v[i] >= lif->threshold) {
          v[i] = lif->reset_mode == 1 ? v[i] - lif->threshold : lif->reset;
          refr[i] = lif->refractory;
          fired[nf++] = i;
        }
      }
      ext[i] = 0.0f;
      slot[i] = 0.0f;
    }
    spikes += nf;
    /* cpu_backend.cpp:149-151 -- decode output spikes into logits */
    for (int k = 0; k < nf; ++k) {
      int i = fired[k];
      if (g->role[i] == 2 && g->channel[i] >= 0 && logits) logits[g->channel[i]] += 1.0f;
      if (raster) raster[(size_t)t * W + (size_t)(i >> 5)] |= 1u << (i & 31);
    }
    /* cpu_backend.cpp:172-181 -- expand fired rows into the delay ring */
    for (int k = 0; k < nf; ++k) {
      int i = fired[k];
      const float s = (float)g->sign[i];
      for (int e = g->row_ptr[i]; e < g->row_ptr[i + 1]; ++e) {
        const int dt = (t + g->delays[e]) % ring_len;
        ring[(size_t)dt * (size_t)n + (size_t)g->post_ids[e]] += s * g->weights[e];
        ++syn_events;
      }
    }
  }
  if (ro_decay >= 0.0f && logits)
    for (int i = 0; i < n; ++i)
      if (g->role[i] == 2 && g->channel[i] >= 0) logits[g->channel[i]] += v[i] / (float)T;
  if (v_out) memcpy(v_out, v, sizeof(float) * (size_t)n);
  if (spikes_out) *spikes_out = spikes;
  if (events_out) *events_out = syn_events;
  free_schedule(&sch);
  free(v); free(ext); free(refr); free(ring); free(fired);
  return ORC_OK;
}

/* Batched forward: one orc_forward per sample with its own step count
 * (events carry sample_id, include/snc/encoders.hpp:22).  Outputs are
 * concatenated per sample: logits [B][noc], spikes/events [B], raster
 * [sum_b T_b][W] (sample-major), v_out [B][N]. */
int orc_forward_batched_ro(const orc_graph* g, const orc_event* ev, size_t n_ev,
                           int num_samples, const int32_t* steps, const orc_lif* lif,
                           float ro_decay, float* logits, int64_t* spikes, int64_t* events,
                           uint32_t* raster, float* v_out);

int orc_forward_batched(const orc_graph* g, const orc_event* ev, size_t n_ev,
                        int num_samples, const int32_t* steps, const orc_lif* lif,
                        float* logits, int64_t* spikes, int64_t* events,
                        uint32_t* raster, float* v_out) {
  return orc_forward_batched_ro(g, ev, n_ev, num_samples, steps, lif, -1.0f, logits, spikes, events,
                                raster, v_out);
}

/* orc_forward_batched with leaky readout units (ro_decay >= 0). */
int orc_forward_batched_ro(const orc_graph* g, const orc_event* ev, size_t n_ev,
                           int num_samples, const int32_t* steps, const orc_lif* lif,
                           float ro_decay, float* logits, int64_t* spikes, int64_t* events,
                           uint32_t* raster, float* v_out) {
  int nic, noc;
  io_counts(g, &nic, &noc);
  const int W = (g->num_neurons + 31) / 32;
  size_t roff = 0;
  for (int b = 0; b < num_samples; ++b) {
    int rc = forward_ro(g, ev, n_ev, b, steps[b], lif, ro_decay,
                         logits ? logits + (size_t)b * noc : NULL,
                         spikes ? spikes + b : NULL, events ? events + b : NULL,
                         raster ? raster + roff : NULL,
                         v_out ? v_out + (size_t)b * g->num_neurons : NULL);
    if (rc) return rc;
    roff += (size_t)steps[b] * (size_t)W;
  }
  return ORC_OK;
}

/* ---- minibatch e-prop -----------------------------------------------------
 * Restates the GPU minibatch trainer's rule (src/training/cuda_trainer.cu):
 *  k_integrate_fire  :67-103  LIF + triangular surrogate psi + pre trace tr
 *  k_eligibility     :105-112 E[b,s] += psi[b,post] * tr[b,pre]  (fp32)
 *  k_deliver         :114-129 signed trainer weights, g.sign ignored
 *  k_softmax_delta   :131-142 softmax(counts) - onehot(label)
 *  k_learning_signal :144-161 L = delta (output) or B.delta (internal)
 *  k_apply           :163-172 w -= lr/T * (sum_b L*E) / bs, clamped
 * with two documented differences: inputs are host-encoded InputEvents routed
 * through the graph's channel->INPUT map (as the CPU Trainer does,
 * src/training/trainer.cpp:187-196) instead of cuRAND draws into neuron id ==
 * channel, and each sample may have its own step count T_b, in which case the
 * update uses lr / T_b per sample (lr / T when all are equal, as the
 * reference).  trace_decay is a separate parameter; the reference uses
 * lif.decay for it.
 *
 *  w          [S]      signed weights, updated in place when train != 0
 *  bmat       [n_internal][noc]  random feedback matrix (row per INTERNAL
 *                     neuron in ascending id order)
 *  labels     [B]
 *  counts     [B][noc] output spike counts (out)
 *  elig       [B][S]   eligibility after the window (out, may be NULL)
 *  fires      [N]      per-neuron firing counts, accumulated (may be NULL)
 *  grad_out   [S]      when not NULL (and train != 0): sum_b L*E / T_b is
 *                     written here and w is left unchanged (the gradient of
 *                     one data-parallel shard)
 */
int orc_eprop_batch(const orc_graph* g, float* w, const orc_event* ev, size_t n_ev,
                    int B, const int32_t* steps, const orc_lif* lif, float trace_decay,
                    float gamma, float lr, float w_max, int train_hidden,
                    const float* bmat, const int32_t* labels, int train,
                    float* counts, float* elig, int64_t* spikes_out,
                    int64_t* events_out, int64_t* fires, float* grad_out) {
  const int n = g->num_neurons, S = g->num_synapses;
  int nic, noc;
  io_counts(g, &nic, &noc);
  const int oc = noc > 1 ? noc : 1;
  const int ring_len = orc_ring_len(g);
  const float thr = lif->threshold;
  float* E = (float*)calloc((size_t)B * (size_t)(S > 0 ? S : 1), sizeof(float));
  float* L = (float*)calloc((size_t)B * (size_t)n, sizeof(float));
  int* src = (int*)malloc(sizeof(int) * (size_t)(S > 0 ? S : 1));
  int* internal_row = (int*)malloc(sizeof(int) * (size_t)n);
  float* v = (float*)malloc(sizeof(float) * (size_t)n);
  float* ext = (float*)malloc(sizeof(float) * (size_t)n);
  float* tr = (float*)malloc(sizeof(float) * (size_t)n);
  float* psi = (float*)malloc(sizeof(float) * (size_t)n);
  int* refr = (int*)malloc(sizeof(int) * (size_t)n);
  unsigned char* fired = (unsigned char*)malloc((size_t)n);
  float* ring = (float*)malloc(sizeof(float) * (size_t)ring_len * (size_t)n);
  if (!E || !L || !src || !internal_row || !v || !ext || !tr || !psi || !refr || !fired || !ring)
    return ORC_ENOMEM;
  for (int i = 0; i < n; ++i)
    for (int e = g->row_ptr[i]; e < g->row_ptr[i + 1]; ++e) src[e] = i;
  int n_internal = 0;
  for (int i = 0; i < n; ++i) internal_row[i] = g->role[i] == 0 ? n_internal++ : -1;
  int64_t spikes = 0, syn = 0;

  for (int b = 0; b < B; ++b) {
    const int T = steps[b];
    memset(v, 0, sizeof(float) * (size_t)n);
    memset(ext, 0, sizeof(float) * (size_t)n);
    memset(tr, 0, sizeof(float) * (size_t)n);
    memset(refr, 0, sizeof(int) * (size_t)n);
    memset(ring, 0, sizeof(float) * (size_t)ring_len * (size_t)n);
    float* cnt = counts + (size_t)b * oc;
    for (int c = 0; c < oc; ++c) cnt[c] = 0.0f;
    float* Eb = E + (size_t)b * S;
    schedule sch;
    build_schedule(g, ev, n_ev, b, T, &sch);
    for (int t = 0; t < T; ++t) {
      float* slot = &ring[(size_t)(t % ring_len) * (size_t)n];
      for (int k = sch.step_ptr[t]; k < sch.step_ptr[t + 1]; ++k) ext[sch.nid[k]] += sch.amp[k];
      for (int j = 0; j < n; ++j) {
        float vpre;
        int f = 0;
        if (refr[j] > 0) {
          --refr[j];
          v[j] = lif->reset;
          vpre = lif->reset;
        } else {
          float nv = v[j] * lif->decay + ext[j] + slot[j];
          vpre = nv;
          if (nv >= thr) {
            v[j] = lif->reset_mode == 1 ? nv - thr : lif->reset;
            refr[j] = lif->refractory;
            f = 1;
          } else {
            v[j] = nv;
          }
        }
        ext[j] = 0.0f;
        slot[j] = 0.0f;
        const float d = fabsf(vpre - thr) / (thr > 0.0f ? thr : 1.0f);
        psi[j] = d < 1.0f ? gamma * (1.0f - d) : 0.0f;
        tr[j] = trace_decay * tr[j] + (1.0f - trace_decay) * (f ? 1.0f : 0.0f);
        fired[j] = (unsigned char)f;
        if (f) {
          ++spikes;
          if (fires) ++fires[j];
          if (g->role[j] == 2 && g->channel[j] >= 0 && g->channel[j] < oc) cnt[g->channel[j]] += 1.0f;
        }
      }
      if (train || elig)
        for (int s = 0; s < S; ++s) Eb[s] += psi[g->post_ids[s]] * tr[src[s]];
      for (int i = 0; i < n; ++i) {
        if (!fired[i]) continue;
        for (int e = g->row_ptr[i]; e < g->row_ptr[i + 1]; ++e) {
          const int dt = (t + g->delays[e]) % ring_len;
          ring[(size_t)dt * (size_t)n + (size_t)g->post_ids[e]] += w[e];
          ++syn;
        }
      }
    }
    free_schedule(&sch);
  }

  if (train) {
    float* delta = (float*)malloc(sizeof(float) * (size_t)B * oc);
    for (int b = 0; b < B; ++b) {
      const float* c = counts + (size_t)b * oc;
      float mx = c[0];
      for (int k = 1; k < oc; ++k) mx = fmaxf(mx, c[k]);
      float sum = 0.0f;
      for (int k = 0; k < oc; ++k) sum += expf(c[k] - mx);
      for (int k = 0; k < oc; ++k)
        delta[b * oc + k] = expf(c[k] - mx) / sum - (k == labels[b] ? 1.0f : 0.0f);
    }
    for (int b = 0; b < B; ++b)
      for (int j = 0; j < n; ++j) {
        float lv = 0.0f;
        if (g->role[j] == 2 && g->channel[j] >= 0 && g->channel[j] < oc) {
          lv = delta[b * oc + g->channel[j]];
        } else if (train_hidden && internal_row[j] >= 0) {
          const float* br = &bmat[(size_t)internal_row[j] * oc];
          float s = 0.0f;
          for (int k = 0; k < oc; ++k) s += br[k] * delta[b * oc + k];
          lv = s;
        }
        L[(size_t)b * n + j] = lv;
      }
    int uniform = 1;
    for (int b = 1; b < B; ++b) if (steps[b] != steps[0]) uniform = 0;
    for (int s = 0; s < S; ++s) {
      float acc = 0.0f;
      if (grad_out) {
        /* data-parallel form: the shard's gradient, weights untouched */
        for (int b = 0; b < B; ++b)
          acc += L[(size_t)b * n + g->post_ids[s]] * E[(size_t)b * S + s] /
                 (float)(steps[b] > 1 ? steps[b] : 1);
        grad_out[s] = acc;
      } else if (uniform) {
        for (int b = 0; b < B; ++b) acc += L[(size_t)b * n + g->post_ids[s]] * E[(size_t)b * S + s];
        const float lr_over_T = lr / (float)(steps[0] > 1 ? steps[0] : 1);
        float nw = w[s] - lr_over_T * acc / (float)B;
        w[s] = fminf(fmaxf(nw, -w_max), w_max);
      } else {
        for (int b = 0; b < B; ++b)
          acc += L[(size_t)b * n + g->post_ids[s]] * E[(size_t)b * S + s] /
                 (float)(steps[b] > 1 ? steps[b] : 1);
        float nw = w[s] - lr * acc / (float)B;
        w[s] = fminf(fmaxf(nw, -w_max), w_max);
      }
    }
    free(delta);
  }
  if (elig) memcpy(elig, E, sizeof(float) * (size_t)B * (size_t)S);
  if (spikes_out) *spikes_out = spikes;
  if (events_out) *events_out = syn;
  free(E); free(L); free(src); free(internal_row); free(v); free(ext);
  free(tr); free(psi); free(refr); free(fired); free(ring);
  return ORC_OK;
}
