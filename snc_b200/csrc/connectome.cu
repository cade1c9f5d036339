// The co-training loop's structural state on the device: a layered edge list
// with per-edge ages (the reference's snc::Connectome,
// src/structure/connectome.cpp) kept as a CSR whose rows are the reference's
// adjacency lists in their order, its prune / regrow step
// (structural_update, connectome.cpp:121-219) as device passes, and its
// compilation to a device graph (to_graph, :84-101).
//
// structural_update on the device:
//   1. the K weakest eligible synapses (age >= protect_rounds) by a radix
//      select over 64-bit keys (|w| bits << 32 | CSR position): eight 8-bit
//      histogram passes find the K-th key, every eligible key at or below it
//      is pruned -- the K smallest by (|w|, position);
//   2. the freed posts in CSR order (an exclusive scan of the prune flags);
//   3. one local regrowth per freed post (connectome.cpp:195-201): a block
//      per distinct freed post takes, for its m-th occurrence, the m-th best
//      pre of its window by (fire count desc, index asc) among those not
//      wired to it after the prune -- exactly the reference's sequential
//      loop, whose growth for one post never changes another post's choice;
//   4. fallback growth (:203-217), sequential by nature: one block steps the
//      attempts with draws made on the host by the reference's distribution,
//      the host's generator then replays exactly the draws consumed;
//   5. the new CSR: kept edges in their order, grown edges appended to their
//      pre's row in growth order, every age advanced (:212-215).
// Host round trips: the radix passes' 256-bin histograms and O(K) lists of
// freed posts and grown edges; the O(S) arrays never leave the device.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <random>
#include <vector>

#include "device_common.cuh"
#include "internal.h"

namespace sncb {

namespace {

constexpr int kAgeCap = 1 << 20;

__device__ __forceinline__ unsigned long long prune_key(const float* w, int e) {
  return ((unsigned long long)__float_as_uint(fabsf(w[e])) << 32) | (unsigned)e;
}

// Histogram of key byte `shift` over the eligible keys matching `prefix`
// under `mask`.
__global__ void k_con_hist(int S, const float* w, const int* age, int protect,
                           unsigned long long prefix, unsigned long long mask, int shift,
                           unsigned* hist) {
  __shared__ unsigned h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < S; e += gridDim.x * blockDim.x) {
    if (age[e] < protect) continue;
    const unsigned long long k = prune_key(w, e);
    if ((k & mask) == prefix) atomicAdd(&h[(k >> shift) & 255u], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], h[i]);
}

__global__ void k_con_mark(int S, const float* w, const int* age, int protect, int any,
                           unsigned long long last, int* rm) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < S; e += gridDim.x * blockDim.x)
    rm[e] = any && age[e] >= protect && prune_key(w, e) <= last ? 1 : 0;
}

__global__ void k_con_freed(int S, const int* rm, const int* rmscan, const int* post, int* freed) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < S; e += gridDim.x * blockDim.x)
    if (rm[e]) freed[rmscan[e]] = post[e];
}

struct Window {
  int b0, bn, klo, khi;  // klo > khi: empty
};

// The locality window of post p (grow_local, connectome.cpp:181-186), with
// the reference's float roundings.
__device__ __forceinline__ Window window_of(int p, const int* layer, const float* pos,
                                            const int* lbeg, const int* lcnt, float w) {
  Window win{0, 0, 1, 0};
  const int pl = layer[p] - 1;
  if (pl < 0) return win;
  win.b0 = lbeg[pl];
  win.bn = lcnt[pl];
  if (win.bn <= 0) return win;  // an empty pre layer: no candidates
  const float span = (float)(win.bn - 1);
  const int lo = (int)ceilf(__fmul_rn(__fsub_rn(pos[p], w), span));
  const int hi = (int)floorf(__fmul_rn(__fadd_rn(pos[p], w), span));
  win.klo = min(max(lo, 0), win.bn - 1);
  win.khi = min(max(hi, 0), win.bn - 1);
  return win;
}

__device__ __forceinline__ long long fire_of(const long long* fires, int n_fires, int i) {
  return i < n_fires ? fires[i] : 0ll;
}

// Whether pre q has a kept edge to post p.
__device__ __forceinline__ bool wired(const int* row_ptr, const int* post, const int* rm, int q, int p) {
  for (int e = row_ptr[q]; e < row_ptr[q + 1]; ++e)
    if (post[e] == p && !rm[e]) return true;
  return false;
}

// Candidate order of grow_local: higher fire count first, then lower index
// (the reference keeps the first strict maximum of an ascending scan).
__device__ __forceinline__ bool better(long long fa, int ka, long long fb, int kb) {
  return fa > fb || (fa == fb && ka < kb);
}

// Block-wide best of (fire, kk) pairs; kk = INT_MAX for none.
__device__ void block_best(long long& f, int& k, long long* sf, int* sk) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const long long f2 = __shfl_down_sync(0xffffffffu, f, o);
    const int k2 = __shfl_down_sync(0xffffffffu, k, o);
    if (better(f2, k2, f, k)) { f = f2; k = k2; }
  }
  if (lane == 0) { sf[warp] = f; sk[warp] = k; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < nw; ++i)
      if (better(sf[i], sk[i], sf[0], sk[0])) { sf[0] = sf[i]; sk[0] = sk[i]; }
  }
  __syncthreads();
  f = sf[0];
  k = sk[0];
  __syncthreads();
}

struct GrowArgs {
  const int* row_ptr;
  const int* post;
  const int* rm;
  const int* layer;
  const float* pos;
  const int* lbeg;
  const int* lcnt;
  const long long* fires;
  int n_fires;
  float window;
};

// One block per distinct freed post: its m picks, successive maxima in the
// candidate order among the window's pres not wired to it.
__global__ void k_con_grow_local(GrowArgs a, const int* gpost, const int* gcnt, const int* gfirst,
                                 int* picks) {
  __shared__ long long sf[32];
  __shared__ int sk[32];
  const int p = gpost[blockIdx.x], m = gcnt[blockIdx.x];
  int* out = picks + gfirst[blockIdx.x];
  const Window win = window_of(p, a.layer, a.pos, a.lbeg, a.lcnt, a.window);
  long long pf = LLONG_MAX;  // previous pick: candidates strictly after it in the order
  int pk = -1;
  for (int r = 0; r < m; ++r) {
    long long bf = LLONG_MIN;
    int bk = INT_MAX;
    for (int kk = win.klo + (int)threadIdx.x; kk <= win.khi; kk += blockDim.x) {
      const int q = win.b0 + kk;
      const long long f = fire_of(a.fires, a.n_fires, q);
      if (!better(pf, pk, f, kk)) continue;  // at or before the previous pick
      if (!better(f, kk, bf, bk)) continue;
      if (wired(a.row_ptr, a.post, a.rm, q, p)) continue;
      bf = f;
      bk = kk;
    }
    block_best(bf, bk, sf, sk);
    if (threadIdx.x == 0) out[r] = bk == INT_MAX ? -1 : win.b0 + bk;
    if (bk == INT_MAX) {
      for (int r2 = r + 1 + (int)threadIdx.x; r2 < m; r2 += blockDim.x) out[r2] = -1;
      break;
    }
    pf = bf;
    pk = bk;
  }
}

// Fallback growth (connectome.cpp:203-217), one block: attempts in order,
// each with four posts drawn on the host, the least active non-input post
// grown from its window's best unwired pre.  `grown` (q, p) holds the local
// pass's edges on entry; the fallback appends.  out[0] attempts, out[1] grown.
__global__ void k_con_fallback(GrowArgs a, int pruned, int grown0, int max_attempts, const int* draws,
                               int2* grown, int* out) {
  __shared__ long long sf[32];
  __shared__ int sk[32];
  __shared__ int s_p;
  constexpr int kLocal = 1024;
  __shared__ int s_pre[kLocal];  // pres already grown onto this attempt's post
  __shared__ int s_nl;
  int n_grown = grown0, attempts = 0;
  while (n_grown < pruned && attempts < max_attempts) {
    const int* d = draws + 4 * attempts;
    ++attempts;
    if (threadIdx.x == 0) {
      int p = -1;
      for (int t = 0; t < 4; ++t) {
        const int q = d[t];
        if (a.layer[q] == 0) continue;
        if (p < 0 || fire_of(a.fires, a.n_fires, q) < fire_of(a.fires, a.n_fires, p)) p = q;
      }
      s_p = p;
      s_nl = 0;
    }
    __syncthreads();
    const int p = s_p;
    if (p < 0) {
      __syncthreads();
      continue;
    }
    for (int i = threadIdx.x; i < n_grown; i += blockDim.x)
      if (grown[i].y == p) {
        const int slot = atomicAdd(&s_nl, 1);
        if (slot < kLocal) s_pre[slot] = grown[i].x;
      }
    __syncthreads();
    const int nl = s_nl;
    const Window win = window_of(p, a.layer, a.pos, a.lbeg, a.lcnt, a.window);
    long long bf = LLONG_MIN;
    int bk = INT_MAX;
    for (int kk = win.klo + (int)threadIdx.x; kk <= win.khi; kk += blockDim.x) {
      const int q = win.b0 + kk;
      const long long f = fire_of(a.fires, a.n_fires, q);
      if (!better(f, kk, bf, bk)) continue;
      if (wired(a.row_ptr, a.post, a.rm, q, p)) continue;
      bool dup = false;
      if (nl <= kLocal) {
        for (int i = 0; i < nl && !dup; ++i) dup = s_pre[i] == q;
      } else {
        for (int i = 0; i < n_grown && !dup; ++i) dup = grown[i].x == q && grown[i].y == p;
      }
      if (dup) continue;
      bf = f;
      bk = kk;
    }
    block_best(bf, bk, sf, sk);
    if (bk != INT_MAX) {
      if (threadIdx.x == 0) grown[n_grown] = make_int2(win.b0 + bk, p);
      ++n_grown;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = attempts;
    out[1] = n_grown;
  }
}

// New row lengths: kept + grown.
__global__ void k_con_newlen(int n, const int* row_ptr, const int* rmscan, const int* gcount, int* len) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int b = row_ptr[q], e = row_ptr[q + 1];
    len[q] = (e - b) - (rmscan[e] - rmscan[b]) + gcount[q];
  }
}

__global__ void k_con_count_grown(int G, const int2* grown, int* gcount) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G; i += gridDim.x * blockDim.x)
    atomicAdd(&gcount[grown[i].x], 1);
}

__device__ __forceinline__ int aged(int a) { return a < kAgeCap ? a + 1 : a; }

// Kept edges to their new places (a warp per row keeps their order).
__global__ void k_con_scatter_kept(int n, const int* row_ptr, const int* rmscan, const int* nrow,
                                   const int* post, const int* delay, const float* w, const int* age,
                                   int* post2, int* delay2, float* w2, int* age2) {
  const int lane = threadIdx.x & 31;
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarp = (gridDim.x * blockDim.x) >> 5;
  for (int q = wid; q < n; q += nwarp) {
    const int b = row_ptr[q], e1 = row_ptr[q + 1];
    for (int e = b + lane; e < e1; e += 32) {
      if (rmscan[e + 1] != rmscan[e]) continue;  // pruned
      const int d = nrow[q] + (e - b) - (rmscan[e] - rmscan[b]);
      post2[d] = post[e];
      delay2[d] = delay[e];
      w2[d] = w[e];
      age2[d] = aged(age[e]);
    }
  }
}

// Grown edges after their pre's kept edges, in growth order (rank).
__global__ void k_con_place_grown(int G, const int* gq, const int* gp, const int* grank,
                                  const int* row_ptr, const int* rmscan, const int* nrow, int delay,
                                  float w0, int* post2, int* delay2, float* w2, int* age2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G; i += gridDim.x * blockDim.x) {
    const int q = gq[i];
    const int b = row_ptr[q], e = row_ptr[q + 1];
    const int d = nrow[q] + (e - b) - (rmscan[e] - rmscan[b]) + grank[i];
    post2[d] = gp[i];
    delay2[d] = delay;
    w2[d] = w0;
    age2[d] = aged(0);
  }
}

__global__ void k_con_abs(int S, const float* w, float* out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < S; e += gridDim.x * blockDim.x)
    out[e] = fabsf(w[e]);
}

__global__ void k_con_indeg(int S, const int* post, int* indeg) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < S; e += gridDim.x * blockDim.x)
    atomicAdd(&indeg[post[e]], 1);
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x ^= x >> 33;
  x *= 0xFF51AFD7ED558CCDull;
  x ^= x >> 33;
  x *= 0xC4CEB9FE1A85EC53ull;
  x ^= x >> 33;
  return x;
}

// Order-sensitive content hash of the graph arrays (the autotuner's key):
// the XOR over elements of mix(array tag, index, value).
__global__ void k_con_hash(int n, int S, const int* row_ptr, const int* post, const int* delay,
                           const float* w, unsigned long long* h) {
  unsigned long long acc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S || i <= n; i += gridDim.x * blockDim.x) {
    if (i <= n) acc ^= mix64((1ull << 62) ^ ((unsigned long long)i << 32) ^ (unsigned)row_ptr[i]);
    if (i < S) {
      acc ^= mix64((2ull << 62) ^ ((unsigned long long)i << 32) ^ (unsigned)post[i]);
      acc ^= mix64((3ull << 62) ^ ((unsigned long long)i << 32) ^ (unsigned)delay[i]);
      acc ^= mix64((0ull << 62) ^ ((unsigned long long)i << 32) ^ __float_as_uint(fabsf(w[i])));
    }
  }
  if (acc) atomicXor(h, acc);
}

__global__ void k_fill_i8(int8_t* p, int n, int8_t v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

inline unsigned grid_for(long long n, int threads, int sms) {
  return (unsigned)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, (long long)sms * 8));
}

float layer_pos(int k, int cnt) { return cnt > 1 ? static_cast<float>(k) / (cnt - 1) : 0.5f; }

}  // namespace

}  // namespace sncb

using namespace sncb;

struct snc_b200_connectome {
  int n = 0, S = 0, max_delay = 1, sms = 148;
  size_t cap = 0;
  std::vector<int> layer_begin, layer_count;
  std::vector<uint8_t> role;
  std::vector<int32_t> channel;
  std::mt19937_64 rng;
  int* layer = nullptr;
  float* pos = nullptr;
  int* lbeg = nullptr;
  int* lcnt = nullptr;
  int* row_ptr = nullptr;  // [n + 1]
  int* post = nullptr;     // [cap]
  int* delay = nullptr;
  float* w = nullptr;      // signed
  int* age = nullptr;
};

namespace {

void con_free(snc_b200_connectome* c) {
  for (void* p : {(void*)c->layer, (void*)c->pos, (void*)c->lbeg, (void*)c->lcnt, (void*)c->row_ptr,
                  (void*)c->post, (void*)c->delay, (void*)c->w, (void*)c->age})
    dev_free(p);
}

int con_edges_alloc(int** post, int** delay, float** w, int** age, size_t n) {
  int rc;
  if ((rc = dev_alloc(post, n))) return rc;
  if ((rc = dev_alloc(delay, n))) return rc;
  if ((rc = dev_alloc(w, n))) return rc;
  return dev_alloc(age, n);
}

}  // namespace

extern "C" int snc_b200_connectome_layered_local(const int32_t* layers, int32_t num_layers,
                                                 int32_t synapse_budget, int32_t delay, float w_init,
                                                 uint64_t seed, snc_b200_connectome** out) {
  if (!out || (num_layers > 0 && !layers) || num_layers < 0 || delay < 1) {
    set_error("connectome_layered_local: layers, num_layers >= 0, delay >= 1, output pointer");
    return SNC_B200_EINVAL;
  }
  *out = nullptr;
  long long n_ll = 0;
  for (int l = 0; l < num_layers; ++l) {
    if (layers[l] < 0) { set_error("connectome_layered_local: negative layer size"); return SNC_B200_EINVAL; }
    n_ll += layers[l];
  }
  if (n_ll >= (1ll << 30)) { set_error("connectome_layered_local: too many neurons"); return SNC_B200_EINVAL; }
  if (delay > 255) { set_error("delay > 255 is outside this backend's limits"); return SNC_B200_EUNSUPPORTED; }
  // Connectome::layered_local (connectome.cpp:14-62), on the host: the
  // initial wiring consumes the generator in the reference's order.
  auto* c = new snc_b200_connectome();
  const int n = (int)n_ll, L = num_layers;
  c->n = n;
  c->max_delay = delay;
  c->rng.seed(seed);
  std::vector<int> layer(n);
  std::vector<float> pos(n);
  c->role.assign(n, 0);
  c->channel.assign(n, -1);
  c->layer_begin.resize(L);
  c->layer_count.resize(L);
  int idx = 0;
  for (int l = 0; l < L; ++l) {
    c->layer_begin[l] = idx;
    c->layer_count[l] = layers[l];
    for (int k = 0; k < layers[l]; ++k, ++idx) {
      layer[idx] = l;
      pos[idx] = layer_pos(k, layers[l]);
      if (l == 0) { c->role[idx] = 1; c->channel[idx] = k; }
      else if (l == L - 1) { c->role[idx] = 2; c->channel[idx] = k; }
    }
  }
  long long forward_pre = 0;
  for (int l = 0; l + 1 < L; ++l) forward_pre += layers[l];
  const int fanout = forward_pre > 0 ? std::max(1, (int)(synapse_budget / forward_pre)) : 0;
  std::vector<int> row_ptr(n + 1, 0), post;
  std::uniform_real_distribution<float> jitter(-0.5f, 0.5f);
  for (int l = 0; l + 1 < L; ++l) {
    const int from0 = c->layer_begin[l], from_n = c->layer_count[l];
    const int to0 = c->layer_begin[l + 1], to_n = c->layer_count[l + 1];
    const int k = std::min(fanout, to_n);
    for (int a = 0; a < from_n; ++a) {
      const float pa = layer_pos(a, from_n) + jitter(c->rng) / std::max(1, to_n);
      int centre = (int)std::lround(pa * (to_n - 1));
      centre = std::clamp(centre, 0, std::max(0, to_n - 1));
      const int lo = std::clamp(centre - k / 2, 0, std::max(0, to_n - k));
      for (int j = 0; j < k; ++j) post.push_back(to0 + lo + j);
      row_ptr[from0 + a + 1] = k;
    }
  }
  for (int i = 0; i < n; ++i) row_ptr[i + 1] += row_ptr[i];
  const int S = (int)post.size();
  c->S = S;
  c->cap = (size_t)std::max(1, S);
  std::vector<int> dl(S, delay), ag(S, kAgeCap);  // initial edges are prune-eligible at once
  std::vector<float> wv(S, w_init);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, dev);
  int rc;
  auto fail = [&](int code) {
    con_free(c);
    delete c;
    return code;
  };
  if ((rc = dev_upload(&c->layer, layer.data(), (size_t)n))) return fail(rc);
  if ((rc = dev_upload(&c->pos, pos.data(), (size_t)n))) return fail(rc);
  if ((rc = dev_upload(&c->lbeg, c->layer_begin.data(), (size_t)L))) return fail(rc);
  if ((rc = dev_upload(&c->lcnt, c->layer_count.data(), (size_t)L))) return fail(rc);
  if ((rc = dev_upload(&c->row_ptr, row_ptr.data(), (size_t)n + 1))) return fail(rc);
  if ((rc = con_edges_alloc(&c->post, &c->delay, &c->w, &c->age, c->cap))) return fail(rc);
  cudaError_t ce = cudaSuccess;
  if (S && ((ce = cudaMemcpy(c->post, post.data(), 4 * (size_t)S, cudaMemcpyHostToDevice)) != cudaSuccess ||
            (ce = cudaMemcpy(c->delay, dl.data(), 4 * (size_t)S, cudaMemcpyHostToDevice)) != cudaSuccess ||
            (ce = cudaMemcpy(c->w, wv.data(), 4 * (size_t)S, cudaMemcpyHostToDevice)) != cudaSuccess ||
            (ce = cudaMemcpy(c->age, ag.data(), 4 * (size_t)S, cudaMemcpyHostToDevice)) != cudaSuccess))
    return fail(cuda_fail(ce, "connectome_layered_local: upload"));
  *out = c;
  return SNC_B200_OK;
}

extern "C" int snc_b200_connectome_release(snc_b200_connectome* c) {
  if (!c) return SNC_B200_OK;
  con_free(c);
  delete c;
  return SNC_B200_OK;
}

extern "C" int snc_b200_connectome_info(const snc_b200_connectome* c, int32_t* num_neurons,
                                        int32_t* num_synapses) {
  if (!c) { set_error("null connectome"); return SNC_B200_EINVAL; }
  if (num_neurons) *num_neurons = c->n;
  if (num_synapses) *num_synapses = c->S;
  return SNC_B200_OK;
}

extern "C" int snc_b200_connectome_read(const snc_b200_connectome* c, int32_t* row_ptr, int32_t* post,
                                        int32_t* delay, float* weight, int32_t* age) {
  if (!c) { set_error("null connectome"); return SNC_B200_EINVAL; }
  const size_t S = (size_t)c->S;
  if (row_ptr) SNCB_CUDA(cudaMemcpy(row_ptr, c->row_ptr, 4 * ((size_t)c->n + 1), cudaMemcpyDeviceToHost));
  if (S && post) SNCB_CUDA(cudaMemcpy(post, c->post, 4 * S, cudaMemcpyDeviceToHost));
  if (S && delay) SNCB_CUDA(cudaMemcpy(delay, c->delay, 4 * S, cudaMemcpyDeviceToHost));
  if (S && weight) SNCB_CUDA(cudaMemcpy(weight, c->w, 4 * S, cudaMemcpyDeviceToHost));
  if (S && age) SNCB_CUDA(cudaMemcpy(age, c->age, 4 * S, cudaMemcpyDeviceToHost));
  return SNC_B200_OK;
}

extern "C" int snc_b200_connectome_set_weights(snc_b200_connectome* c, const float* w, int64_t n) {
  if (!c || (n > 0 && !w) || n < 0) { set_error("connectome_set_weights: connectome, weights, n >= 0"); return SNC_B200_EINVAL; }
  const size_t k = (size_t)std::min<int64_t>(n, c->S);
  if (k) SNCB_CUDA(cudaMemcpy(c->w, w, 4 * k, cudaMemcpyHostToDevice));
  return SNC_B200_OK;
}

extern "C" int snc_b200_connectome_update(snc_b200_connectome* c, const int64_t* neuron_fires,
                                          int64_t n_fires, const snc_struct_config* cfg, float reward,
                                          snc_struct_report* out) {
  if (!c || !cfg || !out || (n_fires > 0 && !neuron_fires) || n_fires < 0 || cfg->delay < 1 ||
      cfg->grow_per_epoch < 0 || cfg->max_attempts_mult < 0) {
    set_error("connectome_update: connectome, config (delay >= 1, grow_per_epoch >= 0), fires, output");
    return SNC_B200_EINVAL;
  }
  if (cfg->delay > 255) { set_error("delay > 255 is outside this backend's limits"); return SNC_B200_EUNSUPPORTED; }
  const int n = c->n, S = c->S, sms = c->sms;
  // rewire count (connectome.cpp:126-133)
  int grow_target = cfg->grow_per_epoch;
  if (cfg->reward_modulated) {
    const float denom = std::max(1e-3f, 1.0f - cfg->reward_chance);
    const float comp = std::clamp((reward - cfg->reward_chance) / denom, 0.0f, 1.0f);
    const float frac = std::clamp(1.0f - comp, cfg->reward_floor, 1.0f);
    grow_target = std::max(0, (int)std::lround(cfg->grow_per_epoch * frac));
  }
  // work: rm [S] | rmscan [S + 1] | freed [S] | scan scratch | hist [256] | fires [n_fires] | misc
  DevBuf work;
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t Sx = (size_t)std::max(1, S);
  const size_t o_rm = 0, o_rs = al(o_rm + 4 * Sx), o_fr = al(o_rs + 4 * (Sx + 1));
  const size_t o_sc = al(o_fr + 4 * Sx);
  const size_t o_h = al(o_sc + 4 * scan_scratch_ints(std::max(S, n + 1)));
  const size_t o_f = al(o_h + 4 * 256), o_m = al(o_f + 8 * (size_t)std::max<int64_t>(1, n_fires));
  const size_t total = al(o_m + 64);
  int rc;
  if ((rc = work.reserve(total))) return rc;
  unsigned char* Wb = static_cast<unsigned char*>(work.p);
  int* rm = reinterpret_cast<int*>(Wb + o_rm);
  int* rmscan = reinterpret_cast<int*>(Wb + o_rs);
  int* freed = reinterpret_cast<int*>(Wb + o_fr);
  int* scratch = reinterpret_cast<int*>(Wb + o_sc);
  unsigned* hist = reinterpret_cast<unsigned*>(Wb + o_h);
  long long* fires = reinterpret_cast<long long*>(Wb + o_f);
  int* misc = reinterpret_cast<int*>(Wb + o_m);
  if (n_fires) SNCB_CUDA(cudaMemcpy(fires, neuron_fires, 8 * (size_t)n_fires, cudaMemcpyHostToDevice));
  const unsigned gS = grid_for(S, 256, sms);
  // 1. the K weakest eligible synapses: radix select of the K-th key
  unsigned long long prefix = 0, mask = 0;
  int K = 0;
  if (grow_target > 0 && S > 0) {
    long long rank = grow_target;  // 1-based rank of the last pruned key
    for (int shift = 56; shift >= 0; shift -= 8) {
      SNCB_CUDA(cudaMemset(hist, 0, 4 * 256));
      k_con_hist<<<gS, 256>>>(S, c->w, c->age, cfg->protect_rounds, prefix, mask, shift, hist);
      SNCB_CUDA(cudaGetLastError());
      unsigned h[256];
      SNCB_CUDA(cudaMemcpy(h, hist, sizeof(h), cudaMemcpyDeviceToHost));
      long long tot = 0;
      for (int i = 0; i < 256; ++i) tot += h[i];
      if (shift == 56) {
        K = (int)std::min<long long>(grow_target, tot);  // min(grow_target, candidates)
        rank = K;
        if (K == 0) break;
      }
      long long below = 0;
      int bin = 0;
      for (; bin < 256; ++bin) {
        if (below + h[bin] >= rank) break;
        below += h[bin];
      }
      rank -= below;
      prefix |= (unsigned long long)bin << shift;
      mask |= 255ull << shift;
    }
  }
  k_con_mark<<<gS, 256>>>(S, c->w, c->age, cfg->protect_rounds, K > 0 ? 1 : 0, prefix, rm);
  SNCB_CUDA(cudaGetLastError());
  if ((rc = scan_exclusive(rm, rmscan, S, scratch, nullptr))) return rc;
  k_con_freed<<<gS, 256>>>(S, rm, rmscan, c->post, freed);
  SNCB_CUDA(cudaGetLastError());
  int pruned = 0;
  SNCB_CUDA(cudaMemcpy(&pruned, rmscan + S, 4, cudaMemcpyDeviceToHost));
  std::vector<int> freed_h(pruned);
  if (pruned) SNCB_CUDA(cudaMemcpy(freed_h.data(), freed, 4 * (size_t)pruned, cudaMemcpyDeviceToHost));
  // 2-3. one local regrowth per freed post, grouped by post
  std::map<int, std::vector<int>> by_post;  // post -> freed indices, ascending
  for (int f = 0; f < pruned; ++f) by_post[freed_h[f]].push_back(f);
  const int ng = (int)by_post.size();
  std::vector<int> gpost, gcnt, gfirst, slot_of(pruned);
  for (auto& kv : by_post) {
    gpost.push_back(kv.first);
    gcnt.push_back((int)kv.second.size());
    gfirst.push_back(gfirst.empty() ? 0 : gfirst.back() + gcnt[gcnt.size() - 2]);
    for (size_t j = 0; j < kv.second.size(); ++j) slot_of[kv.second[j]] = gfirst.back() + (int)j;
  }
  GrowArgs ga;
  ga.row_ptr = c->row_ptr;
  ga.post = c->post;
  ga.rm = rm;
  ga.layer = c->layer;
  ga.pos = c->pos;
  ga.lbeg = c->lbeg;
  ga.lcnt = c->lcnt;
  ga.fires = fires;
  ga.n_fires = (int)std::min<int64_t>(n_fires, (int64_t)1 << 30);
  ga.window = cfg->locality_window;
  std::vector<int2> grown;  // (pre, post) in growth order
  const int max_attempts = cfg->max_attempts_mult * std::max(1, pruned);
  DevBuf gw;
  // groups: gpost | gcnt | gfirst | picks [pruned]; grown list [pruned]; draws [4 max_attempts]
  const size_t ngx = (size_t)std::max(1, ng), px = (size_t)std::max(1, pruned);
  const size_t q_gp = 0, q_gc = al(4 * ngx), q_gf = al(q_gc + 4 * ngx), q_pk = al(q_gf + 4 * ngx);
  const size_t q_gr = al(q_pk + 4 * px), q_dr = al(q_gr + 8 * px);
  if ((rc = gw.reserve(al(q_dr + 16 * (size_t)std::max(1, max_attempts))))) return rc;
  unsigned char* G = static_cast<unsigned char*>(gw.p);
  int* d_picks = reinterpret_cast<int*>(G + q_pk);
  int2* d_grown = reinterpret_cast<int2*>(G + q_gr);
  if (ng) {
    SNCB_CUDA(cudaMemcpy(G + q_gp, gpost.data(), 4 * (size_t)ng, cudaMemcpyHostToDevice));
    SNCB_CUDA(cudaMemcpy(G + q_gc, gcnt.data(), 4 * (size_t)ng, cudaMemcpyHostToDevice));
    SNCB_CUDA(cudaMemcpy(G + q_gf, gfirst.data(), 4 * (size_t)ng, cudaMemcpyHostToDevice));
    k_con_grow_local<<<ng, 256>>>(ga, reinterpret_cast<int*>(G + q_gp), reinterpret_cast<int*>(G + q_gc),
                                  reinterpret_cast<int*>(G + q_gf), d_picks);
    SNCB_CUDA(cudaGetLastError());
    std::vector<int> picks(pruned);
    SNCB_CUDA(cudaMemcpy(picks.data(), d_picks, 4 * (size_t)pruned, cudaMemcpyDeviceToHost));
    for (int f = 0; f < pruned; ++f)
      if (picks[slot_of[f]] >= 0) grown.push_back(make_int2(picks[slot_of[f]], freed_h[f]));
  }
  // 4. fallback growth onto under-driven posts (random draws)
  int attempts = 0;
  std::mt19937_64 rng_next = c->rng;
  if ((int)grown.size() < pruned && max_attempts > 0) {
    const int lo = c->layer_begin.size() > 1 ? c->layer_begin[1] : 0, hi = std::max(0, n - 1);
    std::vector<int> draws(4 * (size_t)max_attempts);
    {
      std::mt19937_64 ahead = c->rng;  // the draws the attempts may consume
      std::uniform_int_distribution<int> any_post(lo, hi);
      for (auto& d : draws) d = any_post(ahead);
    }
    if (!grown.empty())
      SNCB_CUDA(cudaMemcpy(d_grown, grown.data(), 8 * grown.size(), cudaMemcpyHostToDevice));
    SNCB_CUDA(cudaMemcpy(G + q_dr, draws.data(), 4 * draws.size(), cudaMemcpyHostToDevice));
    k_con_fallback<<<1, 256>>>(ga, pruned, (int)grown.size(), max_attempts,
                               reinterpret_cast<int*>(G + q_dr), d_grown, misc);
    SNCB_CUDA(cudaGetLastError());
    int res[2];
    SNCB_CUDA(cudaMemcpy(res, misc, sizeof(res), cudaMemcpyDeviceToHost));
    attempts = res[0];
    grown.resize(res[1]);
    if (res[1]) SNCB_CUDA(cudaMemcpy(grown.data(), d_grown, 8 * (size_t)res[1], cudaMemcpyDeviceToHost));
    // the reference's generator advances by exactly the draws consumed (kept
    // aside until the new CSR is in place)
    std::uniform_int_distribution<int> any_post(lo, hi);
    for (long long i = 0; i < 4ll * attempts; ++i) (void)any_post(rng_next);
  }
  // 5. the new CSR
  const int Gn = (int)grown.size();
  std::vector<int> gq(Gn), gp(Gn), grank(Gn);
  {
    std::map<int, int> seen;
    for (int i = 0; i < Gn; ++i) {
      gq[i] = grown[i].x;
      gp[i] = grown[i].y;
      grank[i] = seen[gq[i]]++;
    }
  }
  DevBuf nb;
  const size_t nx = (size_t)n + 1, gx = (size_t)std::max(1, Gn);
  const size_t r_gc = 0, r_len = al(4 * nx), r_row = al(r_len + 4 * nx), r_gq = al(r_row + 4 * nx);
  const size_t r_gp = al(r_gq + 4 * gx), r_rk = al(r_gp + 4 * gx), r_g2 = al(r_rk + 4 * gx);
  if ((rc = nb.reserve(al(r_g2 + 8 * gx)))) return rc;
  unsigned char* NB = static_cast<unsigned char*>(nb.p);
  int* gcount = reinterpret_cast<int*>(NB + r_gc);
  int* nlen = reinterpret_cast<int*>(NB + r_len);
  int* nrow = reinterpret_cast<int*>(NB + r_row);
  SNCB_CUDA(cudaMemset(gcount, 0, 4 * nx));
  if (Gn) {
    SNCB_CUDA(cudaMemcpy(NB + r_gq, gq.data(), 4 * (size_t)Gn, cudaMemcpyHostToDevice));
    SNCB_CUDA(cudaMemcpy(NB + r_gp, gp.data(), 4 * (size_t)Gn, cudaMemcpyHostToDevice));
    SNCB_CUDA(cudaMemcpy(NB + r_rk, grank.data(), 4 * (size_t)Gn, cudaMemcpyHostToDevice));
    SNCB_CUDA(cudaMemcpy(NB + r_g2, grown.data(), 8 * (size_t)Gn, cudaMemcpyHostToDevice));
    k_con_count_grown<<<grid_for(Gn, 256, sms), 256>>>(Gn, reinterpret_cast<int2*>(NB + r_g2), gcount);
  }
  k_con_newlen<<<grid_for(n, 256, sms), 256>>>(n, c->row_ptr, rmscan, gcount, nlen);
  SNCB_CUDA(cudaGetLastError());
  if ((rc = scan_exclusive(nlen, nrow, n, scratch, nullptr))) return rc;
  int S2 = 0;
  SNCB_CUDA(cudaMemcpy(&S2, nrow + n, 4, cudaMemcpyDeviceToHost));
  int *post2 = nullptr, *delay2 = nullptr, *age2 = nullptr;
  float* w2 = nullptr;
  const size_t cap2 = std::max<size_t>((size_t)std::max(1, S2), c->cap);
  if ((rc = con_edges_alloc(&post2, &delay2, &w2, &age2, cap2))) {
    for (void* p : {(void*)post2, (void*)delay2, (void*)w2, (void*)age2}) dev_free(p);
    return rc;
  }
  k_con_scatter_kept<<<grid_for((long long)n * 32, 256, sms), 256>>>(
      n, c->row_ptr, rmscan, nrow, c->post, c->delay, c->w, c->age, post2, delay2, w2, age2);
  if (Gn)
    k_con_place_grown<<<grid_for(Gn, 256, sms), 256>>>(
        Gn, reinterpret_cast<int*>(NB + r_gq), reinterpret_cast<int*>(NB + r_gp),
        reinterpret_cast<int*>(NB + r_rk), c->row_ptr, rmscan, nrow, cfg->delay, cfg->w_grow_init, post2,
        delay2, w2, age2);
  cudaError_t ce = cudaGetLastError();
  if (ce == cudaSuccess) ce = cudaMemcpy(c->row_ptr, nrow, 4 * nx, cudaMemcpyDeviceToDevice);
  if (ce == cudaSuccess) ce = cudaDeviceSynchronize();
  if (ce != cudaSuccess) {
    for (void* p : {(void*)post2, (void*)delay2, (void*)w2, (void*)age2}) dev_free(p);
    return cuda_fail(ce, "connectome_update: new CSR");
  }
  for (void* p : {(void*)c->post, (void*)c->delay, (void*)c->w, (void*)c->age}) dev_free(p);
  c->post = post2;
  c->delay = delay2;
  c->w = w2;
  c->age = age2;
  c->cap = cap2;
  c->S = S2;
  c->rng = rng_next;
  if (Gn) c->max_delay = std::max(c->max_delay, cfg->delay);
  out->pruned = pruned;
  out->grown = Gn;
  out->synapses = S2;
  return SNC_B200_OK;
}

extern "C" int snc_b200_connectome_graph(const snc_b200_connectome* c, snc_b200_graph** out) {
  if (!c || !out) { set_error("connectome_graph: connectome, output pointer"); return SNC_B200_EINVAL; }
  *out = nullptr;
  {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      cudaGetLastError();
      set_error("no CUDA device");
      return SNC_B200_ENODEV;
    }
  }
  const int n = c->n, S = c->S, sms = c->sms;
  auto* g = new snc_b200_graph();
  auto fail = [&](int code) {
    free_graph(g);
    delete g;
    return code;
  };
  DevBuf work;
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t o_w = 0, o_in = al(4 * (size_t)std::max(1, S)), o_sg = al(o_in + 4 * ((size_t)n + 1));
  const size_t o_h = al(o_sg + (size_t)std::max(1, n));
  int rc;
  if ((rc = work.reserve(al(o_h + 8)))) return fail(rc);
  unsigned char* Wb = static_cast<unsigned char*>(work.p);
  float* wabs = reinterpret_cast<float*>(Wb + o_w);
  int* indeg = reinterpret_cast<int*>(Wb + o_in);
  int8_t* sign = reinterpret_cast<int8_t*>(Wb + o_sg);
  unsigned long long* hh = reinterpret_cast<unsigned long long*>(Wb + o_h);
  if ((rc = dev_alloc(&g->row_ptr, (size_t)n + 1))) return fail(rc);
  if ((rc = dev_alloc(&g->post, (size_t)std::max(1, S)))) return fail(rc);
  cudaError_t ce;
  if ((ce = cudaMemcpy(g->row_ptr, c->row_ptr, 4 * ((size_t)n + 1), cudaMemcpyDeviceToDevice)) != cudaSuccess ||
      (S && (ce = cudaMemcpy(g->post, c->post, 4 * (size_t)S, cudaMemcpyDeviceToDevice)) != cudaSuccess) ||
      (ce = cudaMemset(indeg, 0, 4 * ((size_t)n + 1))) != cudaSuccess ||
      (ce = cudaMemset(hh, 0, 8)) != cudaSuccess)
    return fail(cuda_fail(ce, "connectome_graph: staging"));
  if (S) {
    k_con_abs<<<grid_for(S, 256, sms), 256>>>(S, c->w, wabs);
    k_con_indeg<<<grid_for(S, 256, sms), 256>>>(S, c->post, indeg);
  }
  if (n) k_fill_i8<<<grid_for(n, 256, sms), 256>>>(sign, n, 1);
  k_con_hash<<<grid_for(std::max(S, n + 1), 256, sms), 256>>>(n, S, c->row_ptr, c->post, c->delay, c->w, hh);
  if ((ce = cudaGetLastError()) != cudaSuccess) return fail(cuda_fail(ce, "connectome_graph kernels"));
  std::vector<int> row_ptr(n + 1), indeg_h(n + 1);
  unsigned long long h = 0;
  if ((ce = cudaMemcpy(row_ptr.data(), c->row_ptr, 4 * ((size_t)n + 1), cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (ce = cudaMemcpy(indeg_h.data(), indeg, 4 * ((size_t)n + 1), cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (ce = cudaMemcpy(&h, hh, 8, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail(cuda_fail(ce, "connectome_graph: tables"));
  for (int i = 0; i < n; ++i) h = (h ^ ((unsigned long long)c->role[i] << 32 ^ (unsigned)c->channel[i])) * 0x100000001B3ull;
  g->hash = h ^ 0xBB67AE8584CAA73Bull;
  if ((rc = setup_tables(g, n, S, c->max_delay, row_ptr.data(), indeg_h.data(), c->role.data(),
                         c->channel.data())))
    return fail(rc);
  if ((rc = build_graph_device_cols(g, wabs, c->delay, sign))) return fail(rc);
  *out = g;
  return SNC_B200_OK;
}
