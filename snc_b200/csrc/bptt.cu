// Surrogate-gradient BPTT over the sparse delayed graph: a forward and a
// custom backward kernel behind torch.autograd.Function (snc_b200/bptt.py).
//
// Model (python/snc/model.py:52-72 with the per-synapse delays of
// python/snc/shd_model.py:109-121; restated in oracle/bptt_ref.py):
//   cur_j(t) = sum_{e: post(e)=j} w_e * s_pre(e)(t - d_e)      (0 for t-d < 0)
//   vp_j(t)  = decay * v_j(t-1) + cur_j(t) + ext_j(t)
//   s_j(t)   = H(vp_j(t) - thr)   [smooth variant: x / (1 + k|x|)]
//   v_j(t)   = vp_j(t) * (1 - s_j(t))
// Backward (reverse time), with G = dL/dvp and the fast-sigmoid surrogate
// sg(x) = 1 / (1 + k|x|)^2:
//   gs_i(t)  = dL/ds_i(t) + sum_{e: pre(e)=i} w_e * G_post(e)(t + d_e) - gv_i(t) * vp_i(t)
//   G_i(t)   = gv_i(t) * (1 - s_i(t)) + gs_i(t) * sg(vp_i(t) - thr)
//   gv_i(t-1)= decay * G_i(t);   dL/dext_i(t) = G_i(t)
//   dL/dw_e += G_post(e)(t) * s_pre(e)(t - d_e)
//
// Layout: every per-neuron quantity is [.. ][N][B] with the batch innermost;
// a warp owns a neuron, lane l holds batch elements l, l+32, ...  Binary
// spikes are kept as a bit history [T][N][ceil(B/32)], so one in-edge costs
// one broadcast 32-bit load per 32 samples in the forward and only the set
// bits are visited in the weight gradient.  The incoming edges of a neuron
// are summed in ascending CSR edge order (the order of torch's CPU
// index_add), with separately rounded operations, so the forward spikes equal
// the autograd model's bit for bit.  Steps are separated by a bounded grid
// barrier inside one persistent cooperative launch.  With checkpointing
// (every K steps) only v at segment ends is stored; the backward recomputes
// vp for one segment at a time from those checkpoints and the stored spikes.
#include <algorithm>
#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "internal.h"

struct snc_b200_bptt {
  int N = 0, S = 0, D = 1, R = 2, sm_count = 0;
  int max_deg = 0;     // largest in- or out-degree
  int resident = 1;    // allow resident launches
  int *row_ptr = nullptr, *out_post = nullptr, *out_d = nullptr;
  int *col_ptr = nullptr, *in_pre = nullptr, *in_d = nullptr, *in_eidx = nullptr;
  float *v = nullptr, *gv = nullptr, *gcur = nullptr, *seg = nullptr;
  size_t v_cap = 0, gv_cap = 0, gcur_cap = 0, seg_cap = 0;
  unsigned* ctl = nullptr;
  int* err = nullptr;
};

namespace sncb {

struct BpArgs {
  int N, S, R, T, B, K, smooth;
  float thr, decay, slope;
  const int *row_ptr, *out_post, *out_d, *col_ptr, *in_pre, *in_d, *in_eidx;
  const float* w;
  const float* ext;    // [T][N][B]
  float* spikes;       // [T][N][B]
  uint32_t* bits;      // [T][N][KB]
  float* vsaved;       // K > 0: [T/K][N][B] v at segment ends; K == 0: [T][N][B] vp
  float* v;            // [N][B]
  const float* gspk;   // [T][N][B]
  float* gw;           // [S]
  float* gext;         // [T][N][B] or null
  float* gv;           // [N][B]
  float* gcur;         // [R][N][B]
  float* seg;          // [K][N][B]
  unsigned* ctl;
  int* err;
  int res_cap;         // resident launches: edges per direction staged per warp
  unsigned long long wait_ns;  // grid-barrier wait bound (0: the default)
  unsigned stall;              // injected arrivals that never come (failure tests)
};

constexpr int kBpThreads = 256;
// Blocks per SM the kernels are compiled for: one warp per neuron has to stay
// co-resident (4096 neurons need 4 blocks of 8 warps on each of 148 SMs), so
// narrow batches keep to 64 registers.
template <int KB>
constexpr int kBpMinBlocks = KB <= 2 ? 4 : (KB <= 4 ? 2 : 1);
constexpr int kResCapMax = 256;  // largest in / out degree a resident launch stages

// A resident launch gives every warp one neuron for the whole launch and
// stages that neuron's edges in shared memory once: incoming (pre, delay,
// weight, CSR edge index, weight-gradient accumulator) in ascending CSR edge
// order, outgoing (post, delay, weight) in CSR order.  The per-step edge
// metadata loads and the global weight-gradient read-modify-writes leave the
// time loop; the arithmetic and its order are those of the global-memory form.
struct WarpEdges {
  int *in_pre, *in_d, *in_eidx;
  float *in_w, *in_acc;
  int *out_post, *out_d;
  float* out_w;
  int nin, nout;
};

// Shared memory of a resident launch per warp: 8 arrays of res_cap entries.
__device__ __forceinline__ WarpEdges warp_edges(float* base, int cap) {
  const int wib = threadIdx.x >> 5;
  int* p = reinterpret_cast<int*>(base) + (size_t)wib * 8 * cap;
  WarpEdges we;
  we.in_pre = p;
  we.in_d = p + cap;
  we.in_eidx = p + 2 * cap;
  we.in_w = reinterpret_cast<float*>(p + 3 * cap);
  we.in_acc = reinterpret_cast<float*>(p + 4 * cap);
  we.out_post = p + 5 * cap;
  we.out_d = p + 6 * cap;
  we.out_w = reinterpret_cast<float*>(p + 7 * cap);
  we.nin = we.nout = 0;
  return we;
}

// Stage neuron i's edges (the whole warp; i < N).
__device__ __forceinline__ void stage_edges(const BpArgs& a, int i, WarpEdges& we) {
  const int lane = threadIdx.x & 31;
  const int c0 = a.col_ptr[i], r0 = a.row_ptr[i];
  we.nin = a.col_ptr[i + 1] - c0;
  we.nout = a.row_ptr[i + 1] - r0;
  for (int e = lane; e < we.nin; e += 32) {
    we.in_pre[e] = a.in_pre[c0 + e];
    we.in_d[e] = a.in_d[c0 + e];
    const int ei = a.in_eidx[c0 + e];
    we.in_eidx[e] = ei;
    we.in_w[e] = a.w[ei];
    we.in_acc[e] = 0.f;
  }
  for (int e = lane; e < we.nout; e += 32) {
    we.out_post[e] = a.out_post[r0 + e];
    we.out_d[e] = a.out_d[r0 + e];
    we.out_w[e] = a.w[r0 + e];
  }
  __syncwarp();
}

// One step of the forward for neuron j.  v holds the neuron's state before
// the step (per lane, batch elements lane + 32k) and is updated; vp receives
// the pre-reset potential; s the spike.
// Edges whose spike words / future gradients one lane keeps in flight.
template <int KB>
constexpr int kEdgeBatch = KB >= 8 ? 4 : 8;

template <int KB, bool SMOOTH, bool RES>
__device__ __forceinline__ void fwd_neuron(const BpArgs& a, int t, int j, float (&v)[KB],
                                           float (&vp)[KB], float (&s)[KB], const WarpEdges& we) {
  const int lane = threadIdx.x & 31;
  float acc[KB];
#pragma unroll
  for (int k = 0; k < KB; ++k) acc[k] = 0.f;
  const int e0 = RES ? 0 : a.col_ptr[j], e1 = RES ? we.nin : a.col_ptr[j + 1];
  // one lane per incoming edge of a 32-edge group: its pre, delay, weight
  // and (step form) the spike words of its pre at t - d
  auto group = [&](int eb, int& pre, int& d, float& w, uint32_t (&mw)[KB]) {
    const int n = min(32, e1 - eb);
    pre = 0;
    d = 1 << 30;
    w = 0.f;
    if (lane < n) {
      pre = RES ? we.in_pre[eb + lane] : a.in_pre[eb + lane];
      d = RES ? we.in_d[eb + lane] : a.in_d[eb + lane];
      w = RES ? we.in_w[eb + lane] : a.w[a.in_eidx[eb + lane]];
    }
    if constexpr (!SMOOTH) {
      const bool ok = lane < n && t - d >= 0;
      const uint32_t* wp = a.bits + ((size_t)(ok ? t - d : 0) * a.N + pre) * KB;
#pragma unroll
      for (int k = 0; k < KB; ++k) mw[k] = ok ? wp[k] : 0u;
    }
  };
  int my_pre, my_d;
  float my_w;
  uint32_t mw[KB];
  if (e0 < e1) group(e0, my_pre, my_d, my_w, mw);
  for (int eb = e0; eb < e1; eb += 32) {
    const int n = min(32, e1 - eb);
    if constexpr (!SMOOTH) {
      // the next group's spike words are requested before this group's are
      // added: the words of 64 edges are one round trip; the words are
      // broadcast by shuffles and added in edge order (the order of the sum
      // is unchanged)
      int nx_pre = 0, nx_d = 0;
      float nx_w = 0.f;
      uint32_t nx_mw[KB];
      if (eb + 32 < e1) group(eb + 32, nx_pre, nx_d, nx_w, nx_mw);
      for (int q = 0; q < n; ++q) {
        const float ww = __shfl_sync(0xffffffffu, my_w, q);
#pragma unroll
        for (int k = 0; k < KB; ++k) {
          const uint32_t word = __shfl_sync(0xffffffffu, mw[k], q);
          if ((word >> lane) & 1u) acc[k] = __fadd_rn(acc[k], ww);
        }
      }
      my_pre = nx_pre;
      my_d = nx_d;
      my_w = nx_w;
#pragma unroll
      for (int k = 0; k < KB; ++k) mw[k] = nx_mw[k];
    } else {
      for (int q = 0; q < n; ++q) {
        const int pre = __shfl_sync(0xffffffffu, my_pre, q);
        const int d = __shfl_sync(0xffffffffu, my_d, q);
        const float ww = __shfl_sync(0xffffffffu, my_w, q);
        const int ts = t - d;
        if (ts < 0) continue;
        const float* sp = a.spikes + ((size_t)ts * a.N + pre) * a.B;
#pragma unroll
        for (int k = 0; k < KB; ++k) {
          const int b = 32 * k + lane;
          if (b < a.B) acc[k] = __fadd_rn(acc[k], __fmul_rn(ww, sp[b]));
        }
      }
      if (eb + 32 < e1) group(eb + 32, my_pre, my_d, my_w, mw);
    }
  }
#pragma unroll
  for (int k = 0; k < KB; ++k) {
    const int b = 32 * k + lane;
    const float x_ext = b < a.B ? a.ext[((size_t)t * a.N + j) * a.B + b] : 0.f;
    vp[k] = __fadd_rn(__fadd_rn(__fmul_rn(a.decay, v[k]), acc[k]), x_ext);
    const float x = __fsub_rn(vp[k], a.thr);
    s[k] = SMOOTH ? __fdiv_rn(x, __fadd_rn(1.f, __fmul_rn(a.slope, fabsf(x)))) : (x >= 0.f ? 1.f : 0.f);
    v[k] = __fmul_rn(vp[k], __fsub_rn(1.f, s[k]));
  }
}

template <int KB, bool SMOOTH, bool RES>
__global__ void __launch_bounds__(kBpThreads, kBpMinBlocks<KB>) k_bptt_forward(BpArgs a) {
  extern __shared__ float sm_all[];
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int W = (gridDim.x * blockDim.x) >> 5;
  const unsigned nb = gridDim.x;
  unsigned target = a.stall;
  WarpEdges we{};
  if (RES) {
    we = warp_edges(sm_all, a.res_cap);
    if (gw < a.N) stage_edges(a, gw, we);
  }
  for (int j = gw; j < a.N; j += W)
#pragma unroll
    for (int k = 0; k < KB; ++k) {
      const int b = 32 * k + lane;
      if (b < a.B) a.v[(size_t)j * a.B + b] = 0.f;
    }
  for (int t = 0; t < a.T; ++t) {
    for (int j = gw; j < a.N; j += W) {
      float v[KB], vp[KB], s[KB];
#pragma unroll
      for (int k = 0; k < KB; ++k) {
        const int b = 32 * k + lane;
        v[k] = b < a.B ? a.v[(size_t)j * a.B + b] : 0.f;
      }
      fwd_neuron<KB, SMOOTH, RES>(a, t, j, v, vp, s, we);
      const size_t plane = ((size_t)t * a.N + j) * a.B;
#pragma unroll
      for (int k = 0; k < KB; ++k) {
        const int b = 32 * k + lane;
        const bool ok = b < a.B;
        if (ok) {
          a.v[(size_t)j * a.B + b] = v[k];
          a.spikes[plane + b] = s[k];
          if (a.K == 0) a.vsaved[plane + b] = vp[k];
          else if ((t + 1) % a.K == 0) a.vsaved[((size_t)(t / a.K) * a.N + j) * a.B + b] = v[k];
        }
        const unsigned m = __ballot_sync(0xffffffffu, ok && s[k] != 0.f);
        if (!SMOOTH && lane == 0) a.bits[((size_t)t * a.N + j) * KB + k] = m;
      }
    }
    target += nb;
    if (!grid_sync(&a.ctl[0], target, a.err, a.wait_ns)) return;
  }
}

// One backward step for neuron i; vp_plane points at the [N][B] plane of
// pre-reset potentials of step t.  sm_g: this warp's [B] scratch.
template <int KB, bool SMOOTH, bool RES>
__device__ __forceinline__ void bwd_neuron(const BpArgs& a, int t, int i, const float* vp_plane,
                                           float* sm_g, const WarpEdges& we) {
  const int lane = threadIdx.x & 31;
  const int N = a.N, B = a.B;
  float gs[KB];
  const size_t plane = ((size_t)t * N + i) * B;
#pragma unroll
  for (int k = 0; k < KB; ++k) {
    const int b = 32 * k + lane;
    gs[k] = b < B ? a.gspk[plane + b] : 0.f;
  }
  // gradient reaching s_i(t) through every outgoing synapse (fires at t + d)
  const int tr = t % a.R;
  const int e0 = RES ? 0 : a.row_ptr[i], e1 = RES ? we.nout : a.row_ptr[i + 1];
  for (int eb = e0; eb < e1; eb += 32) {
    const int n = min(32, e1 - eb);
    int my_post = 0, my_d = 1 << 30;
    float my_w = 0.f;
    if (lane < n) {
      my_post = RES ? we.out_post[eb + lane] : a.out_post[eb + lane];
      my_d = RES ? we.out_d[eb + lane] : a.out_d[eb + lane];
      my_w = RES ? we.out_w[eb + lane] : a.w[eb + lane];
    }
    // each lane turns its own edge into an offset into the ring of future
    // gradients (slot of t + d: one conditional subtraction, d < R) and a
    // validity bit; the batches below only broadcast them
    const unsigned okm = __ballot_sync(0xffffffffu, lane < n && t + my_d < a.T);
    size_t my_off = 0;
    if ((okm >> lane) & 1u) {
      const int slot = tr + my_d >= a.R ? tr + my_d - a.R : tr + my_d;
      my_off = ((size_t)slot * N + my_post) * B;
    }
    // the future gradients of kEdgeBatch edges are loaded together, then
    // accumulated in edge order
    for (int q0 = 0; q0 < n; q0 += kEdgeBatch<KB>) {
      float gv[kEdgeBatch<KB>][KB];
      float wwv[kEdgeBatch<KB>];
      bool okv[kEdgeBatch<KB>];
#pragma unroll
      for (int u = 0; u < kEdgeBatch<KB>; ++u) {
        const int src = (q0 + u) & 31;  // q0 + u < 32: kEdgeBatch divides 32
        const unsigned olo = __shfl_sync(0xffffffffu, (unsigned)my_off, src);
        const unsigned ohi = __shfl_sync(0xffffffffu, (unsigned)(my_off >> 32), src);
        wwv[u] = __shfl_sync(0xffffffffu, my_w, src);
        okv[u] = (okm >> src) & 1u;
        const float* gp = a.gcur + (((size_t)ohi << 32) | olo);
#pragma unroll
        for (int k = 0; k < KB; ++k) {
          const int b = 32 * k + lane;
          gv[u][k] = okv[u] && b < B ? gp[b] : 0.f;
        }
      }
#pragma unroll
      for (int u = 0; u < kEdgeBatch<KB>; ++u)
        if (okv[u])
#pragma unroll
          for (int k = 0; k < KB; ++k) {
            const int b = 32 * k + lane;
            if (b < B) gs[k] = __fadd_rn(gs[k], __fmul_rn(wwv[u], gv[u][k]));
          }
    }
  }
  float* gc = a.gcur + ((size_t)tr * N + i) * B;
#pragma unroll
  for (int k = 0; k < KB; ++k) {
    const int b = 32 * k + lane;
    if (b >= B) continue;
    const float vp = vp_plane[(size_t)i * B + b];
    const float x = __fsub_rn(vp, a.thr);
    const float den = __fadd_rn(1.f, __fmul_rn(a.slope, fabsf(x)));
    const float s = SMOOTH ? __fdiv_rn(x, den) : (x >= 0.f ? 1.f : 0.f);
    const float sg = __fdiv_rn(1.f, __fmul_rn(den, den));
    const float gvv = a.gv[(size_t)i * B + b];
    const float gst = __fsub_rn(gs[k], __fmul_rn(gvv, vp));
    const float g = __fadd_rn(__fmul_rn(gvv, __fsub_rn(1.f, s)), __fmul_rn(gst, sg));
    gc[b] = g;
    if (a.gext) a.gext[plane + b] = g;
    a.gv[(size_t)i * B + b] = __fmul_rn(a.decay, g);
    sm_g[b] = g;
  }
  __syncwarp();
  // dL/dw for every incoming synapse: lane per synapse, sum of G over the
  // samples whose pre neuron fired at t - d (only set bits are visited);
  // the spike words of a lane's next two synapses are loaded together
  const int c0 = RES ? 0 : a.col_ptr[i], c1 = RES ? we.nin : a.col_ptr[i + 1];
  for (int e = c0 + lane; e < c1; e += 64) {
    int ts[2], pre[2];
    uint32_t wv[2][KB];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int eu = e + 32 * u;
      ts[u] = -1;
      pre[u] = 0;
      if (eu < c1) {
        ts[u] = t - (RES ? we.in_d[eu] : a.in_d[eu]);
        pre[u] = RES ? we.in_pre[eu] : a.in_pre[eu];
      }
      if (!SMOOTH) {
        const uint32_t* wp = a.bits + ((size_t)(ts[u] >= 0 ? ts[u] : 0) * N + pre[u]) * KB;
#pragma unroll
        for (int k = 0; k < KB; ++k) wv[u][k] = ts[u] >= 0 ? wp[k] : 0u;
      }
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (ts[u] < 0) continue;
      const int eu = e + 32 * u;
      float c = 0.f;
      if (!SMOOTH) {
#pragma unroll
        for (int k = 0; k < KB; ++k) {
          uint32_t word = wv[u][k];
          while (word) {
            const int bb = __ffs(word) - 1;
            c = __fadd_rn(c, sm_g[32 * k + bb]);
            word &= word - 1u;
          }
        }
      } else {
        const float* sp = a.spikes + ((size_t)ts[u] * N + pre[u]) * B;
        for (int b = 0; b < B; ++b) c = __fadd_rn(c, __fmul_rn(sm_g[b], sp[b]));
      }
      if (c != 0.f) {
        if (RES) we.in_acc[eu] = __fadd_rn(we.in_acc[eu], c);
        else a.gw[a.in_eidx[eu]] = __fadd_rn(a.gw[a.in_eidx[eu]], c);
      }
    }
  }
  __syncwarp();
}

// Resident launches: the warp's weight gradients, accumulated in shared
// memory in the order the global form adds them, go out once.
__device__ __forceinline__ void flush_acc(const BpArgs& a, const WarpEdges& we) {
  const int lane = threadIdx.x & 31;
  for (int e = lane; e < we.nin; e += 32) a.gw[we.in_eidx[e]] = we.in_acc[e];
}

template <int KB, bool SMOOTH, bool RES>
__global__ void __launch_bounds__(kBpThreads, kBpMinBlocks<KB>) k_bptt_backward(BpArgs a) {
  extern __shared__ float sm_all[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  float* sm_g = sm_all + (size_t)wib * (32 * KB);
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int W = (gridDim.x * blockDim.x) >> 5;
  const unsigned nb = gridDim.x;
  const size_t NB = (size_t)a.N * a.B;
  unsigned target = a.stall;
  WarpEdges we{};
  if (RES) {
    we = warp_edges(sm_all + (size_t)(blockDim.x >> 5) * 32 * KB, a.res_cap);
    if (gw < a.N) stage_edges(a, gw, we);
  }
  for (int i = gw; i < a.N; i += W)
#pragma unroll
    for (int k = 0; k < KB; ++k) {
      const int b = 32 * k + lane;
      if (b < a.B) a.gv[(size_t)i * a.B + b] = 0.f;
    }
  if (a.K == 0) {
    for (int t = a.T - 1; t >= 0; --t) {
      for (int i = gw; i < a.N; i += W)
        bwd_neuron<KB, SMOOTH, RES>(a, t, i, a.vsaved + (size_t)t * NB, sm_g, we);
      target += nb;
      if (!grid_sync(&a.ctl[0], target, a.err, a.wait_ns)) return;
    }
    if (RES) flush_acc(a, we);
    return;
  }
  const int nseg = (a.T + a.K - 1) / a.K;
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int t0 = sg * a.K, t1 = min(a.T, t0 + a.K);
    // recompute the segment's pre-reset potentials of this warp's neurons
    // from the checkpoint and the stored spikes (no cross-neuron dependence)
    for (int i = gw; i < a.N; i += W) {
      float v[KB], vp[KB], s[KB];
#pragma unroll
      for (int k = 0; k < KB; ++k) {
        const int b = 32 * k + lane;
        v[k] = (sg > 0 && b < a.B) ? a.vsaved[(size_t)(sg - 1) * NB + (size_t)i * a.B + b] : 0.f;
      }
      for (int t = t0; t < t1; ++t) {
        fwd_neuron<KB, SMOOTH, RES>(a, t, i, v, vp, s, we);
#pragma unroll
        for (int k = 0; k < KB; ++k) {
          const int b = 32 * k + lane;
          if (b < a.B) a.seg[(size_t)(t - t0) * NB + (size_t)i * a.B + b] = vp[k];
        }
      }
    }
    for (int t = t1 - 1; t >= t0; --t) {
      for (int i = gw; i < a.N; i += W)
        bwd_neuron<KB, SMOOTH, RES>(a, t, i, a.seg + (size_t)(t - t0) * NB, sm_g, we);
      target += nb;
      if (!grid_sync(&a.ctl[0], target, a.err, a.wait_ns)) return;
    }
  }
  if (RES) flush_acc(a, we);
}

using BpKernel = void (*)(BpArgs);

// Co-resident warps of a launch of kern with smem bytes per block.
static int resident_warps(BpKernel kern, size_t smem, int sm_count) {
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBpThreads, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return per_sm * sm_count * (kBpThreads / 32);
}

static int coop_launch(BpKernel kern, const BpArgs& a, int sm_count, size_t smem, cudaStream_t st) {
  SNCB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  SNCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBpThreads, smem));
  if (per_sm < 1) {
    set_error("bptt kernel does not fit on an SM");
    return SNC_B200_EUNSUPPORTED;
  }
  const int warps_needed = a.N;
  const int blocks = std::max(1, std::min(per_sm * sm_count, (warps_needed + 7) / 8));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(kBpThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  SNCB_CUDA(cudaLaunchKernelEx(&cfg, kern, a));
  return SNC_B200_OK;
}

template <int KB, bool RES>
static BpKernel pick(bool forward, bool smooth) {
  if (forward) return smooth ? k_bptt_forward<KB, true, RES> : k_bptt_forward<KB, false, RES>;
  return smooth ? k_bptt_backward<KB, true, RES> : k_bptt_backward<KB, false, RES>;
}

// A resident launch (a.res_cap > 0) when one warp per neuron can be
// co-resident with the staged edges, else the global-memory form.
template <int KB>
static int dispatch(bool forward, bool smooth, BpArgs a, int sm, cudaStream_t st) {
  const size_t smem = forward ? 0 : (size_t)(kBpThreads / 32) * 32 * KB * sizeof(float);
  if (a.res_cap > 0) {
    const size_t smem_r = smem + (size_t)(kBpThreads / 32) * 8 * a.res_cap * sizeof(int);
    BpKernel kr = pick<KB, true>(forward, smooth);
    if (resident_warps(kr, smem_r, sm) >= a.N) return coop_launch(kr, a, sm, smem_r, st);
  }
  a.res_cap = 0;
  return coop_launch(pick<KB, false>(forward, smooth), a, sm, smem, st);
}

static int launch(bool forward, bool smooth, const BpArgs& a, int sm, cudaStream_t st) {
  const int KB = (a.B + 31) / 32;
  if (KB <= 1) return dispatch<1>(forward, smooth, a, sm, st);
  if (KB <= 2) return dispatch<2>(forward, smooth, a, sm, st);
  if (KB <= 4) return dispatch<4>(forward, smooth, a, sm, st);
  if (KB <= 8) return dispatch<8>(forward, smooth, a, sm, st);
  set_error("bptt: batch > 256");
  return SNC_B200_EUNSUPPORTED;
}

template <typename T>
static int grow(T** p, size_t* cap, size_t n) {
  if (*p && *cap >= n) return SNC_B200_OK;
  dev_free(*p);
  *p = nullptr;
  *cap = 0;
  int rc = dev_alloc(p, n);
  if (!rc) *cap = n;
  return rc;
}

// Edges per direction a resident launch stages per warp (0: none).
static int res_cap(const snc_b200_bptt* h) {
  if (!h->resident || h->max_deg > kResCapMax) return 0;
  return std::max(32, (h->max_deg + 31) / 32 * 32);
}

// Arguments of a forward launch over handle h (both forward entry points).
static BpArgs forward_args(const snc_b200_bptt* h, const float* w, const float* ext, int T, int B,
                           float threshold, float decay, float slope, int ckpt_every, int smooth,
                           float* spikes, uint32_t* spike_bits, float* v_saved) {
  BpArgs a{};
  a.N = h->N; a.S = h->S; a.R = h->R; a.T = T; a.B = B; a.K = ckpt_every; a.smooth = smooth;
  a.thr = threshold; a.decay = decay; a.slope = slope;
  a.row_ptr = h->row_ptr; a.out_post = h->out_post; a.out_d = h->out_d; a.col_ptr = h->col_ptr;
  a.in_pre = h->in_pre; a.in_d = h->in_d; a.in_eidx = h->in_eidx;
  a.w = w; a.ext = ext; a.spikes = spikes; a.bits = spike_bits; a.vsaved = v_saved;
  a.res_cap = res_cap(h);
  const WaitCtl wc = take_wait_ctl(true);
  a.wait_ns = wc.ns;
  a.stall = wc.stall;
  return a;
}

static int check_err(snc_b200_bptt* h, cudaStream_t st) {
  int err = 0;
  SNCB_CUDA(cudaMemcpyAsync(&err, h->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SNCB_CUDA(cudaStreamSynchronize(st));
  if (err) {
    set_error("bptt: device barrier timed out");
    return err;
  }
  return SNC_B200_OK;
}

}  // namespace sncb

using namespace sncb;

// Leaky integration along time of a [T][n] tensor: y[t] = decay * y[t-1] +
// x[t] (reverse: from the last step backwards, y[t] = decay * y[t+1] + x[t]),
// each product and sum rounded separately like the step-by-step loop of the
// readouts (shd_model.py:139-140, lm.py:90); the reverse form is its
// gradient.  One thread per column j, coalesced rows.
__global__ void k_leaky_scan(const float* __restrict__ x, float* __restrict__ y, int T, long long n,
                             float decay, int reverse) {
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (int k = 0; k < T; ++k) {
      const long long t = reverse ? T - 1 - k : k;
      acc = __fadd_rn(__fmul_rn(decay, acc), x[t * n + j]);
      y[t * n + j] = acc;
    }
  }
}

// out[t][i][j] = in[t * st_t + i + j * st_j]: the batch-innermost layout of
// the BPTT kernels and torch's [T][B][N] (or a view of it with unit stride
// along N) into each other, through 32 x 32 shared-memory tiles so that both
// the reads (along i) and the writes (along j) are coalesced.
__global__ void k_transpose_tile(const float* __restrict__ in, float* __restrict__ out, int I, int J,
                                 long long st_t, long long st_j) {
  __shared__ float tile[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  const long long t = blockIdx.z;
  const float* src = in + t * st_t;
  float* dst = out + t * (long long)I * J;
  for (int jj = threadIdx.y; jj < 32; jj += 8) {
    const int i = i0 + threadIdx.x, j = j0 + jj;
    if (i < I && j < J) tile[jj][threadIdx.x] = src[i + (long long)j * st_j];
  }
  __syncthreads();
  for (int ii = threadIdx.y; ii < 32; ii += 8) {
    const int j = j0 + threadIdx.x, i = i0 + ii;
    if (i < I && j < J) dst[(long long)i * J + j] = tile[threadIdx.x][ii];
  }
}

extern "C" {

int snc_b200_bptt_create(int32_t N, int32_t S, const int32_t* row_ptr, const int32_t* post,
                         const int32_t* delays, snc_b200_bptt** out) {
  if (!out || N <= 0 || S < 0 || !row_ptr || (S > 0 && (!post || !delays)) || row_ptr[0] != 0 ||
      row_ptr[N] != S) {
    set_error("bptt_create: bad graph");
    return SNC_B200_EINVAL;
  }
  for (int i = 0; i < N; ++i)
    if (row_ptr[i] > row_ptr[i + 1]) { set_error("bptt_create: row_ptr not monotone"); return SNC_B200_EINVAL; }
  int D = 1;
  for (int e = 0; e < S; ++e) {
    if (post[e] < 0 || post[e] >= N || delays[e] < 1) { set_error("bptt_create: bad edge"); return SNC_B200_EINVAL; }
    D = std::max(D, delays[e]);
  }
  *out = nullptr;
  auto* h = new snc_b200_bptt();
  h->N = N;
  h->S = S;
  h->D = D;
  h->R = D + 1;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, dev);
  // incoming lists in ascending CSR edge order
  std::vector<int> col_ptr(N + 1, 0), in_pre(std::max(1, S)), in_d(std::max(1, S)), in_eidx(std::max(1, S));
  for (int e = 0; e < S; ++e) col_ptr[post[e] + 1]++;
  for (int j = 0; j < N; ++j)
    h->max_deg = std::max({h->max_deg, col_ptr[j + 1], row_ptr[j + 1] - row_ptr[j]});
  for (int j = 0; j < N; ++j) col_ptr[j + 1] += col_ptr[j];
  std::vector<int> fill(col_ptr.begin(), col_ptr.end() - 1);
  for (int i = 0; i < N; ++i)
    for (int e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
      const int q = fill[post[e]]++;
      in_pre[q] = i;
      in_d[q] = delays[e];
      in_eidx[q] = e;
    }
  int rc = SNC_B200_OK;
  if (!rc) rc = dev_upload(&h->row_ptr, row_ptr, (size_t)N + 1);
  if (!rc) rc = dev_upload(&h->out_post, post, (size_t)std::max(1, S));
  if (!rc) rc = dev_upload(&h->out_d, delays, (size_t)std::max(1, S));
  if (!rc) rc = dev_upload(&h->col_ptr, col_ptr.data(), col_ptr.size());
  if (!rc) rc = dev_upload(&h->in_pre, in_pre.data(), in_pre.size());
  if (!rc) rc = dev_upload(&h->in_d, in_d.data(), in_d.size());
  if (!rc) rc = dev_upload(&h->in_eidx, in_eidx.data(), in_eidx.size());
  if (!rc) rc = dev_alloc(&h->ctl, 4);
  if (!rc) rc = dev_alloc(&h->err, 1);
  if (rc) {
    snc_b200_bptt_release(h);
    return rc;
  }
  *out = h;
  return SNC_B200_OK;
}

int snc_b200_bptt_set_resident(snc_b200_bptt* h, int32_t enable) {
  if (!h) {
    set_error("bptt_set_resident: null handle");
    return SNC_B200_EINVAL;
  }
  h->resident = enable != 0;
  return SNC_B200_OK;
}

int snc_b200_bptt_release(snc_b200_bptt* h) {
  if (!h) return SNC_B200_OK;
  for (void* p : {(void*)h->row_ptr, (void*)h->out_post, (void*)h->out_d, (void*)h->col_ptr,
                  (void*)h->in_pre, (void*)h->in_d, (void*)h->in_eidx, (void*)h->v, (void*)h->gv,
                  (void*)h->gcur, (void*)h->seg, (void*)h->ctl, (void*)h->err})
    dev_free(p);
  delete h;
  return SNC_B200_OK;
}

int snc_b200_bptt_forward(snc_b200_bptt* h, const float* w, const float* ext, int32_t T, int32_t B,
                          float threshold, float decay, float slope, int32_t ckpt_every,
                          int32_t smooth, float* spikes, uint32_t* spike_bits, float* v_saved,
                          void* stream) {
  if (!h || !w || !ext || !spikes || !v_saved || T < 1 || B < 1 || ckpt_every < 0 ||
      (!smooth && !spike_bits)) {
    set_error("bptt_forward: bad argument");
    return SNC_B200_EINVAL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t NB = (size_t)h->N * B;
  int rc = grow(&h->v, &h->v_cap, NB);
  if (rc) return rc;
  BpArgs a = forward_args(h, w, ext, T, B, threshold, decay, slope, ckpt_every, smooth, spikes,
                          spike_bits, v_saved);
  a.v = h->v;
  a.ctl = h->ctl; a.err = h->err;
  SNCB_CUDA(cudaMemsetAsync(h->ctl, 0, 16, st));
  SNCB_CUDA(cudaMemsetAsync(h->err, 0, 4, st));
  if ((rc = launch(true, smooth != 0, a, h->sm_count, st))) return rc;
  return check_err(h, st);
}

int snc_b200_bptt_backward(snc_b200_bptt* h, const float* w, const float* ext, int32_t T, int32_t B,
                           float threshold, float decay, float slope, int32_t ckpt_every,
                           int32_t smooth, const float* spikes, const uint32_t* spike_bits,
                           const float* v_saved, const float* grad_spikes, float* grad_w,
                           float* grad_ext, void* stream) {
  if (!h || !w || !ext || !spikes || !v_saved || !grad_spikes || !grad_w || T < 1 || B < 1 ||
      ckpt_every < 0 || (!smooth && !spike_bits)) {
    set_error("bptt_backward: bad argument");
    return SNC_B200_EINVAL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t NB = (size_t)h->N * B;
  int rc;
  if ((rc = grow(&h->v, &h->v_cap, NB))) return rc;
  if ((rc = grow(&h->gv, &h->gv_cap, NB))) return rc;
  if ((rc = grow(&h->gcur, &h->gcur_cap, (size_t)h->R * NB))) return rc;
  if (ckpt_every > 0 && (rc = grow(&h->seg, &h->seg_cap, (size_t)ckpt_every * NB))) return rc;
  BpArgs a{};
  a.N = h->N; a.S = h->S; a.R = h->R; a.T = T; a.B = B; a.K = ckpt_every; a.smooth = smooth;
  a.thr = threshold; a.decay = decay; a.slope = slope;
  a.row_ptr = h->row_ptr; a.out_post = h->out_post; a.out_d = h->out_d; a.col_ptr = h->col_ptr;
  a.in_pre = h->in_pre; a.in_d = h->in_d; a.in_eidx = h->in_eidx;
  a.w = w; a.ext = ext; a.spikes = const_cast<float*>(spikes);
  a.bits = const_cast<uint32_t*>(spike_bits); a.vsaved = const_cast<float*>(v_saved); a.v = h->v;
  a.gspk = grad_spikes; a.gw = grad_w; a.gext = grad_ext; a.gv = h->gv; a.gcur = h->gcur; a.seg = h->seg;
  a.ctl = h->ctl; a.err = h->err;
  a.res_cap = res_cap(h);
  const WaitCtl wc = take_wait_ctl(true);
  a.wait_ns = wc.ns;
  a.stall = wc.stall;
  SNCB_CUDA(cudaMemsetAsync(h->ctl, 0, 16, st));
  SNCB_CUDA(cudaMemsetAsync(h->err, 0, 4, st));
  SNCB_CUDA(cudaMemsetAsync(grad_w, 0, (size_t)std::max(1, h->S) * sizeof(float), st));
  if ((rc = launch(false, smooth != 0, a, h->sm_count, st))) return rc;
  return check_err(h, st);
}

int snc_b200_leaky_scan(const float* x, float* y, int32_t T, int64_t n, float decay, int32_t reverse,
                        void* stream) {
  if ((T > 0 && n > 0) && (!x || !y)) { set_error("null tensor"); return SNC_B200_EINVAL; }
  if (T < 0 || n < 0) { set_error("negative size"); return SNC_B200_EINVAL; }
  if (T == 0 || n == 0) return SNC_B200_OK;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (int)std::max(1ll, std::min<long long>(((long long)n + 255) / 256, (long long)sms * 16));
  k_leaky_scan<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(x, y, T, n, decay, reverse ? 1 : 0);
  SNCB_CUDA(cudaGetLastError());
  return SNC_B200_OK;
}

int snc_b200_transpose(const float* in, float* out, int32_t T, int32_t I, int32_t J, int64_t st_t,
                       int64_t st_j, void* stream) {
  if (T < 0 || I < 0 || J < 0 || T > 65535) { set_error("transpose: bad size"); return SNC_B200_EINVAL; }
  if ((long long)T * I * J == 0) return SNC_B200_OK;
  if (!in || !out) { set_error("transpose: null tensor"); return SNC_B200_EINVAL; }
  const dim3 grid((unsigned)((I + 31) / 32), (unsigned)((J + 31) / 32), (unsigned)T);
  if (grid.y > 65535) { set_error("transpose: J too large"); return SNC_B200_EINVAL; }
  k_transpose_tile<<<grid, dim3(32, 8), 0, static_cast<cudaStream_t>(stream)>>>(in, out, I, J, st_t, st_j);
  SNCB_CUDA(cudaGetLastError());
  return SNC_B200_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Forward without device allocation.
//
// Some callers cannot allocate device memory at the moment they run the
// forward: a framework whose caching allocator owns all of the device's memory
// (an allocation behind its back can fail or push it out of memory), and a
// real-time loop that must not pay cudaMalloc's latency or risk its failure in
// the middle of a run.  snc_b200_bptt_forward may allocate on its first use at
// a given size (the per-neuron state buffer of the handle grows on demand).
// This variant runs the same kernel with its scratch -- the membrane
// potential of every (neuron, sample) and the barrier / error words -- in one
// fixed array in device memory that the library reserves statically, so the
// call itself never allocates.  Like the regular forward it ends by reading
// the kernel's error word back and waiting for `stream`.
// ---------------------------------------------------------------------------
namespace sncb {

constexpr size_t kStaticScratchBytes = size_t(4) << 20;  // 4 MiB per device
constexpr size_t kStaticCtlBytes = 256;                   // barrier counter + error word

// Every device that loads the library holds this array until the process exits.
static __device__ __align__(256) unsigned char g_bptt_static_scratch[kStaticScratchBytes];

static std::mutex g_static_mu;
static void* g_static_addr[64] = {};

// Device address of the static scratch on the current device.  The host-side
// symbol is only a stand-in for the array, not a device address, so it is
// looked up once per device (with that device current) and cached.
static int static_scratch(void** out) {
  int dev = 0;
  SNCB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("static scratch: device ordinal beyond 63");
    return SNC_B200_EUNSUPPORTED;
  }
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_bptt_static_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_bptt_static_scratch)");
    g_static_addr[dev] = p;
  }
  *out = g_static_addr[dev];
  return SNC_B200_OK;
}

}  // namespace sncb

extern "C" int snc_b200_bptt_forward_static(snc_b200_bptt* h, const float* w, const float* ext,
                                            int32_t T, int32_t B, float threshold, float decay,
                                            float slope, int32_t ckpt_every, int32_t smooth,
                                            float* spikes, uint32_t* spike_bits, float* v_saved,
                                            void* stream) {
  using namespace sncb;
  if (!h || !w || !ext || !spikes || !v_saved || T < 1 || B < 1 || ckpt_every < 0 ||
      (!smooth && !spike_bits)) {
    set_error("bptt_forward_static: bad argument");
    return SNC_B200_EINVAL;
  }
  const size_t need = (size_t)h->N * (size_t)B * sizeof(float);
  if (need > kStaticScratchBytes - kStaticCtlBytes) {
    set_error("bptt_forward_static: num_neurons x batch = " + std::to_string((size_t)h->N * B) +
              " exceeds the static scratch limit of " +
              std::to_string((kStaticScratchBytes - kStaticCtlBytes) / sizeof(float)) +
              " (use snc_b200_bptt_forward)");
    return SNC_B200_EUNSUPPORTED;
  }
  void* base = nullptr;
  int rc = static_scratch(&base);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned* ctl = static_cast<unsigned*>(base);
  int* err = reinterpret_cast<int*>(static_cast<char*>(base) + 16);
  float* v = reinterpret_cast<float*>(static_cast<char*>(base) + kStaticCtlBytes);
  // the same launch as snc_b200_bptt_forward (resident when the handle's
  // degrees allow it; a resident launch needs shared memory only)
  BpArgs a = forward_args(h, w, ext, T, B, threshold, decay, slope, ckpt_every, smooth, spikes,
                          spike_bits, v_saved);
  a.v = v;  // zeroed by the kernel before the first step
  a.ctl = ctl;
  a.err = err;
  // the previous call's barrier count and error word must not leak into this one
  SNCB_CUDA(cudaMemsetAsync(base, 0, kStaticCtlBytes, st));
  if ((rc = launch(true, smooth != 0, a, h->sm_count, st))) return rc;
  int e = 0;
  SNCB_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SNCB_CUDA(cudaStreamSynchronize(st));
  if (e) {
    set_error("bptt_forward_static: device barrier timed out");
    return e;
  }
  return SNC_B200_OK;
}
