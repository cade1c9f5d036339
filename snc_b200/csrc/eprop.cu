// Minibatch e-prop (the cudatrain:: session of the reference, re-designed):
// the forward with surrogate / trace / eligibility runs in the
// sample-per-CTA persistent kernel (forward.cu, k_tier_s<.., true>), the
// update in three small kernels below.
//
// Reference: src/training/cuda_trainer.cu
//   k_softmax_delta   :131-142   softmax(counts) - onehot(label)
//   k_learning_signal :144-161   L = delta (OUTPUT) / B . delta (INTERNAL)
//   k_apply           :163-172   w -= lr/T * (sum_b L*E) / bs, clamp
// Every floating-point operation is written out (__fmul_rn / __fadd_rn) in
// the order of the CPU restatement, so results match it up to the expf of the
// softmax.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "internal.h"

struct snc_b200_eprop {
  const sncb::Graph* g = nullptr;
  snc_lif lif{};
  snc_eprop_cfg cfg{};
  int max_batch = 0, n_internal = 0, oc = 1;
  uint2* edges = nullptr;                // trainer weights, CSR order
  float* bmat = nullptr;                 // [n_internal][oc]
  int* internal_row = nullptr;           // [N]
  float* elig = nullptr;                 // [max_batch][S]
  int* counts = nullptr;                 // [max_batch][oc]
  float* delta = nullptr;                // [max_batch][oc]
  float* L = nullptr;                    // [max_batch][N]
  int* labels = nullptr;                 // [max_batch]
  int* steps = nullptr;                  // [max_batch]
  unsigned long long* spikes = nullptr;  // [max_batch]
  unsigned long long* events = nullptr;  // [max_batch]
  unsigned long long* fires = nullptr;   // [N]
  int* err = nullptr;
  unsigned* ctl = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int last_B = 0;
  bool have_elig = false;
  // deferred eligibility: the forward records psi per ring column and step
  // and the spike raster; k_raster_t and k_elig_col then build E from them
  sncb::DevBuf psi_hist, raster, raster_t;
  // incoming synapses of every ring column: (edge, pre) pairs grouped by
  // column (cin[cptr[c] .. cptr[c+1])), and the prefix of their 32-synapse
  // groups (gptr) -- the deferred eligibility's work items
  int* cptr = nullptr;            // [ncols + 1]
  int2* cin = nullptr;            // [S]
  int* gptr = nullptr;            // [ncols + 1]
  int n_groups = 0;
  // grid mode: one sample's state does not fit one CTA's shared memory, so
  // the forward runs on the all-SM kernel, which reads destination-grouped
  // edges: a grouped copy of the trainer's weights, kept in step with them
  bool grid = false;
  int* gperm = nullptr;           // [S] CSR edge -> its grouped position
  uint2* gedges = nullptr;        // [S+2]
  sncb::Run* run = nullptr;
};

namespace sncb {

__global__ void k_softmax_delta(int B, int oc, const int* counts, const int* labels, float* delta) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const int* c = counts + (size_t)b * oc;
  float mx = (float)c[0];
  for (int k = 1; k < oc; ++k) mx = fmaxf(mx, (float)c[k]);
  float sum = 0.f;
  for (int k = 0; k < oc; ++k) sum = __fadd_rn(sum, expf(__fsub_rn((float)c[k], mx)));
  for (int k = 0; k < oc; ++k)
    delta[(size_t)b * oc + k] = __fsub_rn(__fdiv_rn(expf(__fsub_rn((float)c[k], mx)), sum),
                                          k == labels[b] ? 1.f : 0.f);
}

__global__ void k_learning_signal(int B, int N, int oc, int train_hidden, const uint8_t* role,
                                  const int* channel, const int* internal_row, const float* bmat,
                                  const float* delta, float* L) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (long long)B * N) return;
  const int b = (int)(tid / N), j = (int)(tid % N);
  float lv = 0.f;
  if (role[j] == 2 && channel[j] >= 0 && channel[j] < oc) {
    lv = delta[(size_t)b * oc + channel[j]];
  } else if (train_hidden && internal_row[j] >= 0) {
    const float* br = bmat + (size_t)internal_row[j] * oc;
    float s = 0.f;
    for (int k = 0; k < oc; ++k) s = __fadd_rn(s, __fmul_rn(br[k], delta[(size_t)b * oc + k]));
    lv = s;
  }
  L[tid] = lv;
}

__global__ void k_apply(int S, int N, int B, int uniform, float lr, float lr_over_T, float w_max,
                        const int* post, const int* steps, const float* L, const float* E,
                        uint2* edges) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const int p = post[s];
  float acc = 0.f;
  float nw;
  const float w = __uint_as_float(edges[s].y);
  if (uniform) {
    for (int b = 0; b < B; ++b)
      acc = __fadd_rn(acc, __fmul_rn(L[(size_t)b * N + p], E[(size_t)b * S + s]));
    nw = __fsub_rn(w, __fdiv_rn(__fmul_rn(lr_over_T, acc), (float)B));
  } else {
    for (int b = 0; b < B; ++b)
      acc = __fadd_rn(acc, __fdiv_rn(__fmul_rn(L[(size_t)b * N + p], E[(size_t)b * S + s]),
                                     (float)max(1, steps[b])));
    nw = __fsub_rn(w, __fdiv_rn(__fmul_rn(lr, acc), (float)B));
  }
  nw = fminf(fmaxf(nw, -w_max), w_max);
  edges[s].y = __float_as_uint(nw);
}

__global__ void k_set_weights(int S, const float* w, uint2* edges) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < S) edges[s].y = __float_as_uint(w[s]);
}

__global__ void k_get_weights(int S, const uint2* edges, float* w) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < S) w[s] = __uint_as_float(edges[s].y);
}

static inline int grid_of(long long n, int b = 256) { return (int)std::max(1ll, (n + b - 1) / b); }

// The grouped copy of the trainer's weights follows the CSR edges.
__global__ void k_sync_gedges(int S, const uint2* edges, const int* gperm, uint2* gedges) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < S) gedges[gperm[e]].y = edges[e].y;
}

static int sync_gedges(snc_b200_eprop* s, cudaStream_t st) {
  if (!s->grid || s->g->S == 0) return SNC_B200_OK;
  k_sync_gedges<<<grid_of(s->g->S), 256, 0, st>>>(s->g->S, s->edges, s->gperm, s->gedges);
  SNCB_CUDA(cudaGetLastError());
  return SNC_B200_OK;
}

// Most bytes the psi history of one minibatch may take; beyond it the
// eligibility is accumulated inside the forward instead.
constexpr size_t kPsiHistMax = size_t(2) << 30;

// The spike raster ([t][word] bits, raster_off per sample) transposed to
// one run of time bits per neuron: rt[b][i][w] bit u = fired_i(32 w + u)
// (zero from step T_b on).  A warp per (sample, 32 steps, 32 neurons): each
// lane reads one step's word and 32 ballots turn the 32 x 32 bit tile.
__global__ void k_raster_t(int B, int N, int W, int TW, const int* steps, const long long* raster_off,
                           const uint32_t* raster, uint32_t* rt) {
  const int lane = threadIdx.x & 31;
  const long long tiles = (long long)B * TW * W;
  for (long long wi = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); wi < tiles;
       wi += (long long)gridDim.x * (blockDim.x >> 5)) {
    const int b = (int)(wi / ((long long)TW * W));
    const int r = (int)(wi - (long long)b * TW * W);
    const int wt = r / W, wn = r - wt * W;
    const int t = 32 * wt + lane;
    const uint32_t word = t < steps[b] ? raster[raster_off[b] + (size_t)t * W + wn] : 0u;
    uint32_t mine = 0;
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      const uint32_t m = __ballot_sync(0xffffffffu, (word >> k) & 1u);
      if (lane == k) mine = m;
    }
    const int i = 32 * wn + lane;
    if (i < N) rt[((size_t)b * N + i) * TW + wt] = mine;
  }
}

// Eligibility of every synapse after the forward of a minibatch
// (cuda_trainer.cu:105-112 restated per synapse): for sample b and synapse e
// (pre i, post column c), E[b][e] = sum over t = 0..T_b-1, in step order, of
// psi[b][t][c] * tr_i(t), with the pre trace rebuilt from the spikes,
// tr_i(t) = decay * tr_i(t-1) + (1 - decay) * fired_i(t), and every product
// and sum rounded as the per-step update rounds it; steps whose trace is
// exactly zero add nothing (trainer.cpp:243-244).  One warp per (sample, 32
// incoming synapses of one column): the column's psi history is read once
// per 32 steps (one gather of 32 steps, then broadcast by shuffles; the
// history is step-major so that the forward writes each step's values for
// all columns contiguously) and each
// lane's pre spikes come 32 steps to a word from the transposed raster.
__global__ void k_elig_col(int B, int N, int S, int nc, int G, const int* cptr, const int2* cin,
                           const int* gptr, const int* steps, const uint32_t* rt, int TW,
                           const float* psi, int psi_T, float decay, float* elig) {
  const int lane = threadIdx.x & 31;
  const float c1 = __fsub_rn(1.f, decay);
  for (long long wi = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
       wi < (long long)B * G; wi += (long long)gridDim.x * (blockDim.x >> 5)) {
    const int b = (int)(wi / G), gi = (int)(wi - (long long)b * G);
    const int c = upper_index(gptr, nc, gi);
    const int idx = cptr[c] + 32 * (gi - gptr[c]) + lane;
    const bool valid = idx < cptr[c + 1];
    const int2 ep = valid ? cin[idx] : make_int2(0, 0);
    const int T = steps[b];
    const float* pc = psi + (size_t)b * psi_T * nc + c;  // step-major: stride nc
    const uint32_t* rw = rt + ((size_t)b * N + ep.y) * TW;
    float acc = 0.f, tr = 0.f;
    for (int t0 = 0; t0 < T; t0 += 32) {
      const float pv = t0 + lane < T ? pc[(size_t)(t0 + lane) * nc] : 0.f;
      const uint32_t word = valid ? rw[t0 >> 5] : 0u;
      // one step: decay * tr + (1 - decay) * fired, rounded as the per-step
      // update rounds it (with no spike the second product is +0 and the sum
      // is decay * tr itself)
      auto step = [&](int u) {
        const float p = __shfl_sync(0xffffffffu, pv, u);
        const float dt = __fmul_rn(decay, tr);
        tr = (word >> u) & 1u ? __fadd_rn(dt, c1) : dt;
        if (tr != 0.f) acc = __fadd_rn(acc, __fmul_rn(p, tr));
      };
      if (T - t0 >= 32) {
#pragma unroll
        for (int u = 0; u < 32; ++u) step(u);
      } else {
        for (int u = 0; u < T - t0; ++u) step(u);
      }
    }
    if (valid) elig[(size_t)b * S + ep.x] = acc;
  }
}

static void free_session(snc_b200_eprop* s) {
  for (void* p : {(void*)s->edges, (void*)s->bmat, (void*)s->internal_row, (void*)s->elig,
                  (void*)s->counts, (void*)s->delta, (void*)s->L, (void*)s->labels,
                  (void*)s->steps, (void*)s->spikes, (void*)s->events, (void*)s->fires,
                  (void*)s->err, (void*)s->ctl})
    dev_free(p);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  s->psi_hist.release();
  s->raster.release();
  s->raster_t.release();
  dev_free(s->cptr);
  dev_free(s->cin);
  dev_free(s->gptr);
  if (s->run) {
    // the run borrows the session's outputs and control words
    s->run->counts = nullptr;
    s->run->spikes = nullptr;
    s->run->events = nullptr;
    s->run->err = nullptr;
    s->run->ctl = nullptr;
    s->run->raster = nullptr;
    free_run(s->run);
    delete s->run;
    s->run = nullptr;
  }
  dev_free(s->gperm);
  dev_free(s->gedges);
}

static int create_session(snc_b200_eprop* s, const Graph* g, const snc_lif* lif,
                          const snc_eprop_cfg* cfg, int max_batch, const float* w,
                          const float* feedback) {
  s->g = g;
  s->lif = *lif;
  s->cfg = *cfg;
  s->max_batch = max_batch;
  s->oc = std::max(1, g->noc);
  const int N = g->N, S = g->S;
  std::vector<uint8_t> role(N);
  SNCB_CUDA(cudaMemcpy(role.data(), g->role, N, cudaMemcpyDeviceToHost));
  std::vector<int> irow(N, -1);
  for (int i = 0; i < N; ++i)
    if (role[i] == 0) irow[i] = s->n_internal++;
  // trainer edges: the graph's packed edges with the trainer's weights
  std::vector<uint2> edges((size_t)S + 2);
  SNCB_CUDA(cudaMemcpy(edges.data(), g->edges, ((size_t)S + 2) * sizeof(uint2), cudaMemcpyDeviceToHost));
  for (int e = 0; e < S; ++e) std::memcpy(&edges[e].y, &w[e], 4);
  int rc;
  if ((rc = dev_upload(&s->edges, edges.data(), edges.size()))) return rc;
  {
    // incoming synapses per ring column, for the deferred eligibility
    const int nc = std::max(1, g->ncols);
    std::vector<int> cptr(nc + 1, 0), gptr(nc + 1, 0);
    for (int e = 0; e < S; ++e) cptr[(edges[e].x & 0xFFFFFFu) + 1]++;
    for (int c = 0; c < nc; ++c) {
      gptr[c + 1] = gptr[c] + (cptr[c + 1] + 31) / 32;
      cptr[c + 1] += cptr[c];
    }
    std::vector<int2> cin((size_t)std::max(1, S));
    std::vector<int> fill(cptr.begin(), cptr.end() - 1);
    for (int i = 0; i < N; ++i)
      for (int e = g->row_ptr_h[i]; e < g->row_ptr_h[i + 1]; ++e)
        cin[fill[edges[e].x & 0xFFFFFFu]++] = make_int2(e, i);
    s->n_groups = gptr[nc];
    if ((rc = dev_upload(&s->cptr, cptr.data(), cptr.size()))) return rc;
    if ((rc = dev_upload(&s->gptr, gptr.data(), gptr.size()))) return rc;
    if ((rc = dev_upload(&s->cin, cin.data(), cin.size()))) return rc;
  }
  if ((rc = dev_upload(&s->bmat, feedback, (size_t)std::max(1, s->n_internal) * s->oc))) return rc;
  if ((rc = dev_upload(&s->internal_row, irow.data(), (size_t)N))) return rc;
  const size_t B = (size_t)max_batch;
  if ((rc = dev_alloc(&s->elig, B * std::max(1, S)))) return rc;
  if ((rc = dev_alloc(&s->counts, B * s->oc))) return rc;
  if ((rc = dev_alloc(&s->delta, B * s->oc))) return rc;
  if ((rc = dev_alloc(&s->L, B * std::max(1, N)))) return rc;
  if ((rc = dev_alloc(&s->labels, B))) return rc;
  if ((rc = dev_alloc(&s->steps, B))) return rc;
  if ((rc = dev_alloc(&s->spikes, B))) return rc;
  if ((rc = dev_alloc(&s->events, B))) return rc;
  if ((rc = dev_alloc(&s->fires, (size_t)std::max(1, N)))) return rc;
  if ((rc = dev_alloc(&s->err, 1))) return rc;
  if ((rc = dev_alloc(&s->ctl, 4))) return rc;
  SNCB_CUDA(cudaMemset(s->fires, 0, (size_t)std::max(1, N) * sizeof(unsigned long long)));
  SNCB_CUDA(cudaEventCreate(&s->ev0));
  SNCB_CUDA(cudaEventCreate(&s->ev1));
  // grid mode when a sample's state and eligibility inputs do not fit one CTA
  {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const int mode = cfg->mode == SNC_B200_MODE_SORT ? SNC_B200_MODE_SORT : SNC_B200_MODE_ATOMIC;
    s->grid = tier_s_smem_bytes(g, mode, true) > optin;
  }
  if (s->grid) {
    // the stable regroup of every row by destination block, as the graph's
    // grouped edges were built
    std::vector<int> post((size_t)std::max(1, S));
    if (S) SNCB_CUDA(cudaMemcpy(post.data(), g->post, (size_t)S * 4, cudaMemcpyDeviceToHost));
    std::vector<int> perm((size_t)std::max(1, S)), idx;
    std::vector<uint2> ge((size_t)S + 2, make_uint2(0, 0));
    for (int i = 0; i < N; ++i) {
      const int rs = g->row_ptr_h[i], re = g->row_ptr_h[i + 1];
      idx.resize(re - rs);
      for (int q = 0; q < re - rs; ++q) idx[q] = rs + q;
      std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return post[x] / g->BS < post[y] / g->BS; });
      for (int q = 0; q < re - rs; ++q) {
        perm[idx[q]] = rs + q;
        ge[rs + q] = edges[idx[q]];
      }
    }
    if ((rc = dev_upload(&s->gperm, perm.data(), perm.size()))) return rc;
    if ((rc = dev_upload(&s->gedges, ge.data(), ge.size()))) return rc;
    s->run = new Run();
    Run& r = *s->run;
    r.g = g;
    r.W = (N + 31) / 32;
    r.counts = s->counts;
    r.spikes = s->spikes;
    r.events = s->events;
    r.err = s->err;
    r.ctl = s->ctl;
    SNCB_CUDA(cudaEventCreate(&r.ev0));
    SNCB_CUDA(cudaEventCreate(&r.ev1));
  }
  return SNC_B200_OK;
}

// grad[s] = sum_b L[b, post(s)] * E[b, s] / T_b (data-parallel e-prop).
__global__ void k_gradient(int S, int N, int B, const int* post, const int* steps, const float* L,
                           const float* E, float* grad) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const int p = post[s];
  float acc = 0.f;
  for (int b = 0; b < B; ++b)
    acc = __fadd_rn(acc, __fdiv_rn(__fmul_rn(L[(size_t)b * N + p], E[(size_t)b * S + s]),
                                   (float)max(1, steps[b])));
  grad[s] = acc;
}

__global__ void k_apply_grad(int S, float lr, float w_max, int total_batch, const float* grad,
                             uint2* edges) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const float w = __uint_as_float(edges[s].y);
  float nw = __fsub_rn(w, __fdiv_rn(__fmul_rn(lr, grad[s]), (float)total_batch));
  nw = fminf(fmaxf(nw, -w_max), w_max);
  edges[s].y = __float_as_uint(nw);
}

// train: 0 forward only, 1 update the weights, 2 write the gradient to grad.
static int run_batch(snc_b200_eprop* s, const snc_input_event* ev, size_t n_ev, int B,
                     const int32_t* steps, const int32_t* labels, int train, float* counts_out,
                     snc_run_stats* stats, float* grad = nullptr) {
  const Graph* g = s->g;
  if (B < 1 || B > s->max_batch || !steps || (train && !labels)) {
    set_error("e-prop batch: bad sample count, steps or labels");
    return SNC_B200_EINVAL;
  }
  Inputs in;
  int rc = upload_inputs(g, ev, n_ev, B, steps, false, &in);
  if (rc) { free_inputs(&in); return rc; }
  cudaStream_t st = nullptr;
  const int oc = s->oc, N = g->N, S = g->S;
  bool ok = true;
  auto chk = [&](cudaError_t e, const char* what) {
    if (ok && e != cudaSuccess) { rc = cuda_fail(e, what); ok = false; }
  };
  chk(cudaMemsetAsync(s->counts, 0, (size_t)B * oc * sizeof(int), st), "memset counts");
  chk(cudaMemsetAsync(s->spikes, 0, (size_t)B * 8, st), "memset spikes");
  chk(cudaMemsetAsync(s->events, 0, (size_t)B * 8, st), "memset events");
  chk(cudaMemsetAsync(s->ctl, 0, 16, st), "memset ctl");
  chk(cudaMemsetAsync(s->err, 0, 4, st), "memset err");
  // deferred eligibility when the psi history of this minibatch fits its budget
  const int W = (N + 31) / 32;
  const size_t psi_bytes = (size_t)B * std::max(1, g->ncols) * std::max(1, in.Tmax) * sizeof(float);
  const bool deferred = train && psi_bytes <= kPsiHistMax;
  if (train && s->grid && !deferred) {
    free_inputs(&in);
    set_error("e-prop: the minibatch's psi history exceeds its budget on the grid path; use fewer samples or steps");
    return SNC_B200_EUNSUPPORTED;
  }
  if (deferred) {
    if ((rc = s->psi_hist.reserve(psi_bytes))) { free_inputs(&in); return rc; }
    if ((rc = s->raster.reserve((size_t)std::max(1ll, in.raster_words) * sizeof(uint32_t)))) {
      free_inputs(&in);
      return rc;
    }
    const size_t tw = ((size_t)std::max(1, in.Tmax) + 31) / 32;
    if ((rc = s->raster_t.reserve((size_t)B * std::max(1, N) * tw * sizeof(uint32_t)))) {
      free_inputs(&in);
      return rc;
    }
  }
  if (train && !deferred) chk(cudaMemsetAsync(s->elig, 0, (size_t)B * S * sizeof(float), st), "memset elig");
  if (train) {
    chk(cudaMemcpyAsync(s->labels, labels, (size_t)B * 4, cudaMemcpyHostToDevice, st), "labels");
    chk(cudaMemcpyAsync(s->steps, steps, (size_t)B * 4, cudaMemcpyHostToDevice, st), "steps");
  }
  chk(cudaEventRecord(s->ev0, st), "event");
  if (ok && s->grid) {
    // the all-SM kernel with the trainer's weights, recording psi and the
    // raster for the deferred eligibility
    Run& r = *s->run;
    r.in = &in;
    r.flags = SNC_B200_RUN_FORCE_GRID | (deferred ? SNC_B200_RUN_RASTER : 0);
    r.raster = deferred ? static_cast<uint32_t*>(s->raster.p) : nullptr;
    r.edges_w = s->edges;
    r.gedges_w = s->gedges;
    r.fires = train ? s->fires : nullptr;
    r.psi_hist = deferred ? static_cast<float*>(s->psi_hist.p) : nullptr;
    r.psi_T = std::max(1, in.Tmax);
    r.gamma = s->cfg.surrogate_scale;
    const int mode = s->cfg.mode == SNC_B200_MODE_SORT ? SNC_B200_MODE_SORT : SNC_B200_MODE_ATOMIC;
    rc = launch_run(&r, &s->lif, mode, SNC_B200_PATH_PERSISTENT, nullptr);
    ok = rc == SNC_B200_OK;
  } else if (ok) {
    EpropLaunch e;
    e.g = g;
    e.in = &in;
    e.edges = s->edges;
    e.counts = s->counts;
    e.spikes = s->spikes;
    e.events = s->events;
    e.elig = train && !deferred ? s->elig : nullptr;
    e.fires = train ? s->fires : nullptr;
    if (deferred) {
      e.psi_hist = static_cast<float*>(s->psi_hist.p);
      e.psi_T = std::max(1, in.Tmax);
      e.raster = static_cast<uint32_t*>(s->raster.p);
    }
    e.gamma = s->cfg.surrogate_scale;
    e.trace_decay = s->cfg.trace_decay;
    e.lif = s->lif;
    e.mode = s->cfg.mode == SNC_B200_MODE_SORT ? SNC_B200_MODE_SORT : SNC_B200_MODE_ATOMIC;
    e.err = s->err;
    e.ctl = s->ctl;
    rc = launch_eprop_forward(e, st);
    ok = rc == SNC_B200_OK;
  }
  if (ok) {
    if (deferred) {
      int dev = 0, sms = 148;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      const int TW = (std::max(1, in.Tmax) + 31) / 32;
      uint32_t* rt = static_cast<uint32_t*>(s->raster_t.p);
      const long long tiles = (long long)B * TW * W;
      k_raster_t<<<(int)std::max(1ll, std::min((tiles + 7) / 8, (long long)sms * 8)), 256, 0, st>>>(
          B, N, W, TW, in.steps, in.raster_off, static_cast<const uint32_t*>(s->raster.p), rt);
      const long long warps = (long long)B * s->n_groups;
      if (warps > 0)
        k_elig_col<<<(int)std::max(1ll, std::min((warps + 7) / 8, (long long)sms * 16)), 256, 0, st>>>(
            B, N, S, std::max(1, g->ncols), s->n_groups, s->cptr, s->cin, s->gptr, in.steps, rt, TW,
            static_cast<const float*>(s->psi_hist.p), std::max(1, in.Tmax), s->cfg.trace_decay, s->elig);
      chk(cudaGetLastError(), "deferred eligibility");
    }
  }
  if (ok && train) {
    bool uniform = true;
    for (int b = 1; b < B; ++b) uniform = uniform && steps[b] == steps[0];
    const float lr_over_T = s->cfg.lr / (float)std::max(1, steps[0]);
    k_softmax_delta<<<grid_of(B), 256, 0, st>>>(B, oc, s->counts, s->labels, s->delta);
    k_learning_signal<<<grid_of((long long)B * N), 256, 0, st>>>(
        B, N, oc, s->cfg.train_hidden, g->role, g->channel, s->internal_row, s->bmat, s->delta, s->L);
    if (train == 2)
      k_gradient<<<grid_of(S), 256, 0, st>>>(S, N, B, g->post, s->steps, s->L, s->elig, grad);
    else
      k_apply<<<grid_of(S), 256, 0, st>>>(S, N, B, uniform ? 1 : 0, s->cfg.lr, lr_over_T,
                                          s->cfg.w_max, g->post, s->steps, s->L, s->elig, s->edges);
    chk(cudaGetLastError(), "e-prop update kernels");
    if (train == 1 && ok) {
      const int r2 = sync_gedges(s, st);
      if (r2) { rc = r2; ok = false; }
    }
  }
  chk(cudaEventRecord(s->ev1, st), "event");
  chk(cudaEventSynchronize(s->ev1), "synchronize");
  if (ok) {
    std::vector<int> cnt((size_t)B * oc);
    std::vector<unsigned long long> sp(B), en(B);
    chk(cudaMemcpy(cnt.data(), s->counts, cnt.size() * 4, cudaMemcpyDeviceToHost), "counts");
    chk(cudaMemcpy(sp.data(), s->spikes, (size_t)B * 8, cudaMemcpyDeviceToHost), "spikes");
    chk(cudaMemcpy(en.data(), s->events, (size_t)B * 8, cudaMemcpyDeviceToHost), "events");
    int err = 0;
    chk(cudaMemcpy(&err, s->err, 4, cudaMemcpyDeviceToHost), "err");
    if (ok && counts_out)
      for (int b = 0; b < B; ++b)
        for (int c = 0; c < g->noc; ++c) counts_out[(size_t)b * g->noc + c] = (float)cnt[(size_t)b * oc + c];
    if (ok && stats) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, s->ev0, s->ev1);
      stats->spikes = stats->synaptic_events = 0;
      for (int b = 0; b < B; ++b) {
        stats->spikes += (long long)sp[b];
        stats->synaptic_events += (long long)en[b];
      }
      stats->overflow = err == SNC_B200_EOVERFLOW ? 1 : 0;
      stats->ms = ms;
    }
    if (ok && err) {
      set_error("device error word set");
      rc = err;
      ok = false;
    }
  }
  s->last_B = B;
  s->have_elig = ok && train;
  free_inputs(&in);
  return rc;
}

}  // namespace sncb

using namespace sncb;

extern "C" {

int snc_b200_eprop_create(const snc_b200_graph* g, const snc_lif* lif, const snc_eprop_cfg* cfg,
                          int32_t max_batch, const float* weights, const float* feedback,
                          snc_b200_eprop** out) {
  if (!g || !lif || !cfg || !weights || !out || max_batch < 1) {
    set_error("e-prop create: bad argument");
    return SNC_B200_EINVAL;
  }
  *out = nullptr;
  auto* s = new snc_b200_eprop();
  int rc = create_session(s, static_cast<const Graph*>(g), lif, cfg, max_batch, weights, feedback);
  if (rc) { free_session(s); delete s; return rc; }
  *out = s;
  return SNC_B200_OK;
}

int snc_b200_eprop_path(const snc_b200_eprop* s) {
  if (!s) { set_error("null session"); return SNC_B200_EINVAL; }
  return s->grid ? SNC_B200_PATH_PERSISTENT : SNC_B200_PATH_PLAIN;
}

int snc_b200_eprop_release(snc_b200_eprop* s) {
  if (!s) return SNC_B200_OK;
  free_session(s);
  delete s;
  return SNC_B200_OK;
}

int snc_b200_eprop_set_weights(snc_b200_eprop* s, const float* w) {
  if (!s || !w) { set_error("null argument"); return SNC_B200_EINVAL; }
  float* d = nullptr;
  int rc = dev_upload(&d, w, (size_t)std::max(1, s->g->S));
  if (rc) return rc;
  k_set_weights<<<grid_of(s->g->S), 256>>>(s->g->S, d, s->edges);
  rc = sync_gedges(s, nullptr);
  if (rc) { dev_free(d); return rc; }
  cudaError_t e = cudaDeviceSynchronize();
  dev_free(d);
  if (e != cudaSuccess) return cuda_fail(e, "set_weights");
  return SNC_B200_OK;
}

int snc_b200_eprop_get_weights(snc_b200_eprop* s, float* w) {
  if (!s || !w) { set_error("null argument"); return SNC_B200_EINVAL; }
  float* d = nullptr;
  int rc = dev_alloc(&d, (size_t)std::max(1, s->g->S));
  if (rc) return rc;
  k_get_weights<<<grid_of(s->g->S), 256>>>(s->g->S, s->edges, d);
  cudaError_t e = cudaMemcpy(w, d, (size_t)s->g->S * sizeof(float), cudaMemcpyDeviceToHost);
  dev_free(d);
  if (e != cudaSuccess) return cuda_fail(e, "get_weights");
  return SNC_B200_OK;
}

int snc_b200_eprop_batch(snc_b200_eprop* s, const snc_input_event* events, size_t n_events,
                         int32_t num_samples, const int32_t* steps, const int32_t* labels,
                         int train, float* counts, snc_run_stats* stats) {
  if (!s) { set_error("null session"); return SNC_B200_EINVAL; }
  return run_batch(s, events, n_events, num_samples, steps, labels, train, counts, stats);
}

int snc_b200_eprop_gradient(snc_b200_eprop* s, const snc_input_event* events, size_t n_events,
                            int32_t num_samples, const int32_t* steps, const int32_t* labels,
                            float* grad, float* counts, snc_run_stats* stats) {
  if (!s || !grad) { set_error("null argument"); return SNC_B200_EINVAL; }
  return run_batch(s, events, n_events, num_samples, steps, labels, 2, counts, stats, grad);
}

int snc_b200_eprop_apply(snc_b200_eprop* s, const float* grad, int32_t total_batch) {
  if (!s || !grad || total_batch < 1) { set_error("bad argument"); return SNC_B200_EINVAL; }
  k_apply_grad<<<grid_of(s->g->S), 256>>>(s->g->S, s->cfg.lr, s->cfg.w_max, total_batch, grad,
                                          s->edges);
  SNCB_CUDA(cudaGetLastError());
  int rc = sync_gedges(s, nullptr);
  if (rc) return rc;
  SNCB_CUDA(cudaDeviceSynchronize());
  return SNC_B200_OK;
}

int snc_b200_eprop_get_eligibility(snc_b200_eprop* s, float* elig) {
  if (!s || !elig) { set_error("null argument"); return SNC_B200_EINVAL; }
  if (!s->have_elig) { set_error("no training minibatch has run"); return SNC_B200_EINVAL; }
  SNCB_CUDA(cudaMemcpy(elig, s->elig, (size_t)s->last_B * s->g->S * sizeof(float), cudaMemcpyDeviceToHost));
  return SNC_B200_OK;
}

int snc_b200_eprop_reset_stats(snc_b200_eprop* s) {
  if (!s) { set_error("null session"); return SNC_B200_EINVAL; }
  SNCB_CUDA(cudaMemset(s->fires, 0, (size_t)std::max(1, s->g->N) * sizeof(unsigned long long)));
  return SNC_B200_OK;
}

// Every spike of neuron i delivers each of its outgoing synapses once
// (cuda_trainer.cu:182-185), so a synapse's delivery count is its pre
// neuron's firing count.
int snc_b200_eprop_collect_stats(snc_b200_eprop* s, int64_t* syn_deliveries, int64_t* neuron_fires) {
  if (!s) { set_error("null session"); return SNC_B200_EINVAL; }
  const Graph* g = s->g;
  std::vector<unsigned long long> f((size_t)std::max(1, g->N));
  SNCB_CUDA(cudaMemcpy(f.data(), s->fires, (size_t)g->N * 8, cudaMemcpyDeviceToHost));
  if (neuron_fires)
    for (int i = 0; i < g->N; ++i) neuron_fires[i] = (int64_t)f[i];
  if (syn_deliveries)
    for (int i = 0; i < g->N; ++i)
      for (int e = g->row_ptr_h[i]; e < g->row_ptr_h[i + 1]; ++e) syn_deliveries[e] = (int64_t)f[i];
  return SNC_B200_OK;
}

}  // extern "C"
