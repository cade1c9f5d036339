// Forward kernels of the spiking substrate: LIF integration over the CSR
// graph with integer delays in a delay ring and event-driven delivery.
//
// Reference semantics: run_cpu, src/runtime/cpu_backend.cpp:67-191 (serial
// branch).  Per step t of one sample:
//   ext[i]   = drive of step t summed in event order        (:99)
//   if refr: refr--, v = reset                              (:130-132)
//   else     v = v*decay + ext + ring[t%R][i]; fire if v >= thr  (:134-139)
//   ring[t%R][i] = 0                                         (:142)
//   logits[channel] += 1 for fired OUTPUT neurons           (:149-151)
//   for fired i in ascending id, for e in row(i) in order:
//            ring[(t+d_e)%R][post_e] += sign_i * w_e         (:173-181)
//
// Three kernel families share the per-step phases below:
//   tier S  (k_tier_s)  one CTA simulates one sample with its whole state
//           and delay ring in shared memory; CTAs pull samples from a work
//           queue (longest first), so uneven step counts balance across SMs.
//   tier G  (k_tier_g)  every SM cooperates on a wave of samples in lockstep;
//           CTA b owns neuron block b (its v, refr, ring columns) and a
//           bounded software grid barrier separates the phases.
//   plain   (k_plain_a / k_plain_b) the tier-G phases as one kernel launch
//           each per step, one sample after another: the per-sample path.
//
// Delivery modes (include/snc_b200.h): ATOMIC red.add, BUCKET post-block
// owner accumulates with atomics, SORT post-block owner applies each ring
// cell's contributions in (pre, edge) order -- bit-identical to the CPU.
#include <algorithm>
#include <climits>
#include <cstring>
#include <initializer_list>

#include "device_common.cuh"
#include "internal.h"

namespace sncb {

enum { MODE_ATOMIC = 0, MODE_BUCKET = 1, MODE_SORT = 2 };

struct FwdArgs {
  // graph
  int N, S, R, ncols, noc, P, BS;
  const int* row_ptr;
  const uint2* edges;
  const uint2* gedges;
  const int* gptr;
  const int2* groups;
  const int* col_of;
  const int* out_ch;
  const int* colbase;
  // inputs
  int B;
  const int* order;
  const int* steps;
  const long long* sptr_off;
  const int* sched_ptr;
  const int* sched_nid;
  const float* sched_ext;
  const long long* raster_off;
  // outputs
  int* counts;
  unsigned long long* spikes;
  unsigned long long* events;
  uint32_t* raster;
  float* vfinal;
  int W;
  // grid state
  int Bw;
  float* v;
  int* refr;
  float* ring;
  int* fired;
  int* fired_cnt;
  // control
  int* err;
  unsigned* ctl;
  LifP lif;
};

// Shared-memory bytes of the tier-S kernel for this graph (0 when the SORT
// staging chunk is not needed).
static size_t tier_s_bytes(int N, int ncols, int R, int noc, int mode, bool eprop, int nthr) {
  size_t words = (size_t)R * ncols + 4 * (size_t)N + (size_t)noc;
  if (mode == MODE_SORT) words += (size_t)N + 1 + ncols + 3 * (size_t)nthr;
  if (eprop) words += (size_t)N + ncols;
  return words * 4 + 16;
}

int tier_s_smem_bytes(const Graph* g, int mode, bool eprop) {
  return (int)tier_s_bytes(g->N, g->ncols, g->R, std::max(1, g->noc), mode, eprop, 1024);
}

// ---------------------------------------------------------------------------
// one LIF neuron (cpu_backend.cpp:129-143, plus reset_mode 1 = subtractive)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int lif_step(const LifP& p, float& v, int& refr, float ext, float rin) {
  if (refr > 0) {
    --refr;
    v = p.reset;
    return 0;
  }
  const float nv = lif_integrate(v, p.decay, ext, rin);
  if (nv >= p.thr) {
    v = p.reset_mode ? __fsub_rn(nv, p.thr) : p.reset;
    refr = p.refractory;
    return 1;
  }
  v = nv;
  return 0;
}

// Ring slot of a delivery made at step slot `s0` with delay d (1 <= d < R).
__device__ __forceinline__ int ring_slot(int s0, int d, int R) {
  const int s = s0 + d;
  return s >= R ? s - R : s;
}

// Ordered apply of one chunk of staged events.  For every ring column with a
// non-empty list, the contributions are added to their cells in increasing
// staging index, i.e. in (pre, edge) order.  Lists are built with atomicExch
// (arbitrary order) and replayed by repeated minimum selection.
template <bool GLOBAL_RING>
__device__ __forceinline__ void apply_ordered(int* head, int ncols_local, const int* st_slot,
                                              const float* st_w, const int* st_next,
                                              float* ring, int ring_stride, int col0) {
  for (int c = threadIdx.x; c < ncols_local; c += blockDim.x) {
    const int h = head[c];
    if (h < 0) continue;
    head[c] = -1;
    int last = -1;
    for (;;) {
      int best = INT_MAX;
      for (int p = h; p >= 0; p = st_next[p])
        if (p > last && p < best) best = p;
      if (best == INT_MAX) break;
      float* cell = ring + (size_t)st_slot[best] * ring_stride + col0 + c;
      if (GLOBAL_RING) {
        __stcg(cell, __fadd_rn(__ldcg(cell), st_w[best]));
      } else {
        *cell = __fadd_rn(*cell, st_w[best]);
      }
      last = best;
    }
  }
}

// ---------------------------------------------------------------------------
// tier S: one CTA per sample, state in shared memory
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(1024, 1) k_tier_s(FwdArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int scratch[40];
  __shared__ long long lscratch[40];
  __shared__ int s_q;
  const int N = a.N, R = a.R, nc = a.ncols, noc = a.noc;
  const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = nthr >> 5;
  const int CH = nthr;
  float* ring = reinterpret_cast<float*>(smem_raw);
  float* v = ring + (size_t)R * nc;
  int* refr = reinterpret_cast<int*>(v + N);
  float* ext = reinterpret_cast<float*>(refr + N);
  int* fired = reinterpret_cast<int*>(ext + N);
  int* counts = fired + N;
  int* pref = counts + noc;
  int* head = pref + (N + 1);
  int* st_slot = head + nc;
  float* st_w = reinterpret_cast<float*>(st_slot + CH);
  int* st_next = reinterpret_cast<int*>(st_w + CH);

  for (;;) {
    if (tid == 0) s_q = (int)atomicAdd(&a.ctl[1], 1u);
    __syncthreads();
    const int q = s_q;
    if (q >= a.B) break;
    const int b = a.order[q];
    const int T = a.steps[b];
    for (int i = tid; i < R * nc; i += nthr) ring[i] = 0.f;
    for (int i = tid; i < N; i += nthr) {
      v[i] = 0.f;
      refr[i] = 0;
      ext[i] = 0.f;
    }
    for (int i = tid; i < noc; i += nthr) counts[i] = 0;
    if (MODE == MODE_SORT)
      for (int i = tid; i < nc; i += nthr) head[i] = -1;
    __syncthreads();
    const int* sp = a.sched_ptr + a.sptr_off[b];
    uint32_t* rast = a.raster ? a.raster + a.raster_off[b] : nullptr;
    long long my_spikes = 0, my_events = 0;
    int s0 = 0;
    for (int t = 0; t < T; ++t) {
      float* slot = ring + (size_t)s0 * nc;
      for (int k = sp[t] + tid; k < sp[t + 1]; k += nthr) ext[a.sched_nid[k]] = a.sched_ext[k];
      __syncthreads();
      // integrate / fire, ascending fired list via ballot compaction
      int nf = 0;
      for (int base = 0; base < N; base += nthr) {
        const int j = base + tid;
        int f = 0;
        if (j < N) {
          float vv = v[j];
          int rr = refr[j];
          const float e = ext[j];
          ext[j] = 0.f;
          const int c = a.col_of[j];
          float rin = 0.f;
          if (c >= 0) {
            rin = slot[c];
            slot[c] = 0.f;
          }
          f = lif_step(a.lif, vv, rr, e, rin);
          v[j] = vv;
          refr[j] = rr;
          if (f) {
            ++my_spikes;
            my_events += a.row_ptr[j + 1] - a.row_ptr[j];
            const int oc = a.out_ch[j];
            if (oc >= 0) atomicAdd(&counts[oc], 1);
          }
        }
        int tot;
        unsigned m;
        const int pos = ballot_compact(f, scratch, &tot, &m);
        if (rast && lane == 0 && base + warp * 32 < N)
          rast[(size_t)t * a.W + ((base + warp * 32) >> 5)] = m;
        if (f) fired[nf + pos] = j;
        nf += tot;
      }
      __syncthreads();
      if (MODE != MODE_SORT) {
        // warp per fired row; two edges per lane per 128-bit load
        for (int k = warp; k < nf; k += nwarps) {
          const int j = fired[k];
          const int rs = a.row_ptr[j], re = a.row_ptr[j + 1];
          for (int e = (rs & ~1) + 2 * lane; e < re; e += 64) {
            const uint4 pr = *reinterpret_cast<const uint4*>(a.edges + e);
            if (e >= rs) {
              const uint2 ed = make_uint2(pr.x, pr.y);
              atomicAdd(&ring[(size_t)ring_slot(s0, edge_delay(ed), R) * nc + edge_col(ed)], edge_w(ed));
            }
            if (e + 1 < re) {
              const uint2 ed = make_uint2(pr.z, pr.w);
              atomicAdd(&ring[(size_t)ring_slot(s0, edge_delay(ed), R) * nc + edge_col(ed)], edge_w(ed));
            }
          }
        }
      } else {
        int base = 0;
        for (int k0 = 0; k0 < nf; k0 += nthr) {
          const int k = k0 + tid;
          const int len = k < nf ? a.row_ptr[fired[k] + 1] - a.row_ptr[fired[k]] : 0;
          int tot;
          const int ex = block_exclusive_scan(len, scratch, &tot);
          if (k < nf) pref[k] = base + ex;
          base += tot;
        }
        __syncthreads();
        const int E = base;
        for (int e0 = 0; e0 < E; e0 += CH) {
          const int ce = min(CH, E - e0);
          for (int qq = tid; qq < ce; qq += nthr) {
            const int e = e0 + qq;
            const int k = upper_index(pref, nf, e);
            const uint2 ed = a.edges[a.row_ptr[fired[k]] + (e - pref[k])];
            st_slot[qq] = ring_slot(s0, edge_delay(ed), R);
            st_w[qq] = edge_w(ed);
            st_next[qq] = atomicExch(&head[edge_col(ed)], qq);
          }
          __syncthreads();
          apply_ordered<false>(head, nc, st_slot, st_w, st_next, ring, nc, 0);
          __syncthreads();
        }
      }
      __syncthreads();
      s0 = (s0 + 1 == R) ? 0 : s0 + 1;
    }
    for (int i = tid; i < noc; i += nthr) a.counts[(size_t)b * noc + i] = counts[i];
    if (a.vfinal)
      for (int i = tid; i < N; i += nthr) a.vfinal[(size_t)b * N + i] = v[i];
    const long long ts = block_sum_ll(my_spikes, lscratch);
    const long long te = block_sum_ll(my_events, lscratch);
    if (tid == 0) {
      a.spikes[b] = (unsigned long long)ts;
      a.events[b] = (unsigned long long)te;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// tier G / plain: phases of one step for neuron block b of wave slot k
// ---------------------------------------------------------------------------
struct GSmem {
  float* ext;    // [BS]
  int* fired;    // [BS]
  int* pa;       // [P+1]
  int* seg_s;    // [nthr]
  int* seg_l;    // [nthr]
  int* seg_p;    // [nthr]
  int* head;     // [BS]
  int* st_slot;  // [CH]
  float* st_w;   // [CH]
  int* st_next;  // [CH]
};

__device__ __forceinline__ GSmem carve_g(unsigned char* raw, int BS, int P, int nthr, int CH) {
  GSmem s;
  s.ext = reinterpret_cast<float*>(raw);
  s.fired = reinterpret_cast<int*>(s.ext + BS);
  s.pa = s.fired + BS;
  s.seg_s = s.pa + (P + 1);
  s.seg_l = s.seg_s + nthr;
  s.seg_p = s.seg_l + nthr;
  s.head = s.seg_p + nthr;
  s.st_slot = s.head + BS;
  s.st_w = reinterpret_cast<float*>(s.st_slot + CH);
  s.st_next = reinterpret_cast<int*>(s.st_w + CH);
  return s;
}

static size_t tier_g_bytes(int BS, int P, int nthr) {
  const int CH = nthr * 2;
  return 4 * ((size_t)BS * 3 + (P + 1) + 3 * (size_t)nthr + 3 * (size_t)CH) + 16;
}

// Phase A: drive, integrate / fire own neurons, publish the ascending fired
// list; in ATOMIC mode also deliver own fired rows into the (global) ring.
template <int MODE>
__device__ void phase_a(const FwdArgs& a, const GSmem& sm, int* scratch, long long* lsc, int k,
                        int sample, int t, int b) {
  __shared__ int s_rng[2];
  const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = nthr >> 5;
  const int lo = b * a.BS, hi = min(a.N, lo + a.BS);
  const int R = a.R, nc = a.ncols, N = a.N;
  const int par = t & 1;
  const int s0 = t % R;
  float* ringk = a.ring + (size_t)k * R * nc;
  float* vk = a.v + (size_t)k * N;
  int* rk = a.refr + (size_t)k * N;
  const int* sp = a.sched_ptr + a.sptr_off[sample];
  for (int i = tid; i < hi - lo; i += nthr) sm.ext[i] = 0.f;
  if (tid == 0) {
    const int k0 = sp[t], k1 = sp[t + 1];
    s_rng[0] = lower_bound_i(a.sched_nid, k0, k1, lo);
    s_rng[1] = lower_bound_i(a.sched_nid, k0, k1, hi);
  }
  __syncthreads();
  for (int q = s_rng[0] + tid; q < s_rng[1]; q += nthr) sm.ext[a.sched_nid[q] - lo] = a.sched_ext[q];
  __syncthreads();
  uint32_t* rast = a.raster ? a.raster + a.raster_off[sample] + (size_t)t * a.W : nullptr;
  int nf = 0;
  long long my_events = 0;
  for (int base = lo; base < hi; base += nthr) {
    const int j = base + tid;
    int f = 0;
    if (j < hi) {
      float vv = vk[j];
      int rr = rk[j];
      const int c = a.col_of[j];
      float rin = 0.f;
      if (c >= 0) {
        float* cell = ringk + (size_t)s0 * nc + c;
        rin = __ldcg(cell);
        __stcg(cell, 0.f);
      }
      f = lif_step(a.lif, vv, rr, sm.ext[j - lo], rin);
      vk[j] = vv;
      rk[j] = rr;
      if (f) {
        my_events += a.row_ptr[j + 1] - a.row_ptr[j];
        const int oc = a.out_ch[j];
        if (oc >= 0) atomicAdd(&a.counts[(size_t)sample * a.noc + oc], 1);
      }
    }
    int tot;
    unsigned m;
    const int pos = ballot_compact(f, scratch, &tot, &m);
    if (rast && lane == 0 && base + warp * 32 < hi) rast[(base + warp * 32) >> 5] = m;
    if (f) sm.fired[nf + pos] = j;
    nf += tot;
  }
  __syncthreads();
  int* fo = a.fired + ((size_t)k * 2 + par) * N + lo;
  for (int i = tid; i < nf; i += nthr) __stcg(&fo[i], sm.fired[i]);
  const long long ev = block_sum_ll(my_events, lsc);
  if (tid == 0) {
    __stcg(&a.fired_cnt[((size_t)k * 2 + par) * a.P + b], nf);
    if (nf) {
      atomicAdd(&a.spikes[sample], (unsigned long long)nf);
      atomicAdd(&a.events[sample], (unsigned long long)ev);
    }
  }
  if (MODE == MODE_ATOMIC) {
    for (int q = warp; q < nf; q += nwarps) {
      const int j = sm.fired[q];
      const int rs = a.row_ptr[j], re = a.row_ptr[j + 1];
      for (int e = (rs & ~1) + 2 * lane; e < re; e += 64) {
        const uint4 pr = *reinterpret_cast<const uint4*>(a.gedges + e);
        if (e >= rs) {
          const uint2 ed = make_uint2(pr.x, pr.y);
          atomicAdd(&ringk[(size_t)ring_slot(s0, edge_delay(ed), R) * nc + edge_col(ed)], edge_w(ed));
        }
        if (e + 1 < re) {
          const uint2 ed = make_uint2(pr.z, pr.w);
          atomicAdd(&ringk[(size_t)ring_slot(s0, edge_delay(ed), R) * nc + edge_col(ed)], edge_w(ed));
        }
      }
    }
  }
  __syncthreads();
}

// Phase B (BUCKET / SORT): as owner of the ring columns of block b, gather the
// row segments of every fired neuron that target this block, in ascending pre
// order, and apply them.
template <int MODE>
__device__ void phase_b(const FwdArgs& a, const GSmem& sm, int* scratch, int k, int t, int b) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int CH = nthr * 2;
  const int R = a.R, nc = a.ncols, P = a.P;
  const int par = t & 1;
  const int s0 = t % R;
  const int cb0 = a.colbase[b], cb1 = a.colbase[b + 1];
  float* ringk = a.ring + (size_t)k * R * nc;
  const int* cntk = a.fired_cnt + ((size_t)k * 2 + par) * P;
  const int* fk = a.fired + ((size_t)k * 2 + par) * a.N;
  int F;
  {
    const int cnt = tid < P ? __ldcg(&cntk[tid]) : 0;
    const int ex = block_exclusive_scan(cnt, scratch, &F);
    if (tid < P) sm.pa[tid] = ex;
    __syncthreads();
  }
  if (cb1 == cb0 || F == 0) return;
  for (int f0 = 0; f0 < F; f0 += nthr) {
    const int f = f0 + tid;
    int gs = 0, gl = 0;
    if (f < F) {
      const int blk = upper_index(sm.pa, P, f);
      const int i = __ldcg(&fk[(size_t)blk * a.BS + (f - sm.pa[blk])]);
      const int g0 = a.gptr[i], g1 = a.gptr[i + 1];
      for (int g = g0; g < g1; ++g) {
        const int2 gr = a.groups[g];
        if (gr.x == b) {
          const int ge = (g + 1 < g1) ? a.groups[g + 1].y : a.row_ptr[i + 1];
          gs = gr.y;
          gl = ge - gr.y;
          break;
        }
        if (gr.x > b) break;
      }
    }
    int nseg;
    unsigned m;
    const int pos = ballot_compact(gl > 0, scratch, &nseg, &m);
    if (gl > 0) {
      sm.seg_s[pos] = gs;
      sm.seg_l[pos] = gl;
    }
    __syncthreads();
    int E;
    {
      const int len = tid < nseg ? sm.seg_l[tid] : 0;
      const int ex = block_exclusive_scan(len, scratch, &E);
      if (tid < nseg) sm.seg_p[tid] = ex;
      __syncthreads();
    }
    for (int e0 = 0; e0 < E; e0 += CH) {
      const int ce = min(CH, E - e0);
      for (int qq = tid; qq < ce; qq += nthr) {
        const int e = e0 + qq;
        const int s = upper_index(sm.seg_p, nseg, e);
        const uint2 ed = a.gedges[sm.seg_s[s] + (e - sm.seg_p[s])];
        const int slot = ring_slot(s0, edge_delay(ed), R);
        if (MODE == MODE_BUCKET) {
          atomicAdd(&ringk[(size_t)slot * nc + edge_col(ed)], edge_w(ed));
        } else {
          sm.st_slot[qq] = slot;
          sm.st_w[qq] = edge_w(ed);
          sm.st_next[qq] = atomicExch(&sm.head[edge_col(ed) - cb0], qq);
        }
      }
      __syncthreads();
      if (MODE == MODE_SORT) {
        apply_ordered<true>(sm.head, cb1 - cb0, sm.st_slot, sm.st_w, sm.st_next, ringk, nc, cb0);
        __syncthreads();
      }
    }
  }
}

// Zero the state a CTA owns for wave slot k: v / refr of its neurons and its
// ring columns in every slot.
__device__ void init_block_state(const FwdArgs& a, int k, int b) {
  const int lo = b * a.BS, hi = min(a.N, lo + a.BS);
  const int cb0 = a.colbase[b], cb1 = a.colbase[b + 1];
  float* vk = a.v + (size_t)k * a.N;
  int* rk = a.refr + (size_t)k * a.N;
  for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
    vk[j] = 0.f;
    rk[j] = 0;
  }
  float* ringk = a.ring + (size_t)k * a.R * a.ncols;
  const int w = cb1 - cb0;
  for (int i = threadIdx.x; i < a.R * w; i += blockDim.x)
    __stcg(&ringk[(size_t)(i / w) * a.ncols + cb0 + (i % w)], 0.f);
}

template <int MODE>
__global__ void __launch_bounds__(512, 1) k_tier_g(FwdArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int scratch[40];
  __shared__ long long lscratch[40];
  const GSmem sm = carve_g(smem_raw, a.BS, a.P, blockDim.x, blockDim.x * 2);
  const int b = blockIdx.x;
  const unsigned nb = gridDim.x;
  unsigned target = 0;
  const int nwaves = (a.B + a.Bw - 1) / a.Bw;
  if (MODE == MODE_SORT)
    for (int i = threadIdx.x; i < a.BS; i += blockDim.x) sm.head[i] = -1;
  for (int w = 0; w < nwaves; ++w) {
    const int q0 = w * a.Bw;
    const int nk = min(a.Bw, a.B - q0);
    for (int k = 0; k < nk; ++k) init_block_state(a, k, b);
    const int Tw = a.steps[a.order[q0]];
    target += nb;
    if (!grid_sync(&a.ctl[0], target, a.err)) return;
    for (int t = 0; t < Tw; ++t) {
      for (int k = 0; k < nk; ++k) {
        const int smp = a.order[q0 + k];
        if (t < a.steps[smp]) phase_a<MODE>(a, sm, scratch, lscratch, k, smp, t, b);
      }
      target += nb;
      if (!grid_sync(&a.ctl[0], target, a.err)) return;
      if (MODE != MODE_ATOMIC) {
        for (int k = 0; k < nk; ++k) {
          const int smp = a.order[q0 + k];
          if (t < a.steps[smp]) phase_b<MODE>(a, sm, scratch, k, t, b);
        }
      }
    }
    if (a.vfinal) {
      const int lo = b * a.BS, hi = min(a.N, lo + a.BS);
      for (int k = 0; k < nk; ++k) {
        const int smp = a.order[q0 + k];
        for (int j = lo + threadIdx.x; j < hi; j += blockDim.x)
          a.vfinal[(size_t)smp * a.N + j] = a.v[(size_t)k * a.N + j];
      }
    }
    target += nb;
    if (!grid_sync(&a.ctl[0], target, a.err)) return;
  }
}

template <int MODE>
__global__ void __launch_bounds__(512) k_plain_a(FwdArgs a, int sample, int t) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int scratch[40];
  __shared__ long long lscratch[40];
  const GSmem sm = carve_g(smem_raw, a.BS, a.P, blockDim.x, blockDim.x * 2);
  phase_a<MODE>(a, sm, scratch, lscratch, 0, sample, t, blockIdx.x);
}

template <int MODE>
__global__ void __launch_bounds__(512) k_plain_b(FwdArgs a, int t) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int scratch[40];
  const GSmem sm = carve_g(smem_raw, a.BS, a.P, blockDim.x, blockDim.x * 2);
  if (MODE == MODE_SORT)
    for (int i = threadIdx.x; i < a.BS; i += blockDim.x) sm.head[i] = -1;
  __syncthreads();
  phase_b<MODE>(a, sm, scratch, 0, t, blockIdx.x);
}

__global__ void k_plain_init(FwdArgs a) {
  init_block_state(a, 0, blockIdx.x);
}

__global__ void k_copy_v(FwdArgs a, int sample) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < a.N; j += gridDim.x * blockDim.x)
    a.vfinal[(size_t)sample * a.N + j] = a.v[j];
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static FwdArgs make_args(Run* r, const snc_lif* lif) {
  const Graph* g = r->g;
  const Inputs* in = r->in;
  FwdArgs a{};
  a.N = g->N; a.S = g->S; a.R = g->R; a.ncols = g->ncols; a.noc = std::max(1, g->noc);
  a.P = g->P; a.BS = g->BS;
  a.row_ptr = g->row_ptr; a.edges = g->edges; a.gedges = g->gedges; a.gptr = g->gptr;
  a.groups = g->groups; a.col_of = g->col_of; a.out_ch = g->out_ch; a.colbase = g->colbase;
  a.B = in->B; a.order = in->order; a.steps = in->steps; a.sptr_off = in->sptr_off;
  a.sched_ptr = in->sched_ptr; a.sched_nid = in->sched_nid; a.sched_ext = in->sched_ext;
  a.raster_off = in->raster_off;
  a.counts = r->counts; a.spikes = r->spikes; a.events = r->events;
  a.raster = (r->flags & SNC_B200_RUN_RASTER) ? r->raster : nullptr;
  a.vfinal = (r->flags & SNC_B200_RUN_VFINAL) ? r->vfinal : nullptr;
  a.W = r->W;
  a.Bw = r->Bw; a.v = r->v; a.refr = r->refr; a.ring = r->ring; a.fired = r->fired;
  a.fired_cnt = r->fired_cnt;
  a.err = r->err; a.ctl = r->ctl;
  a.lif = LifP{lif->threshold, lif->decay, lif->reset, lif->refractory, lif->reset_mode};
  return a;
}

static int ensure_grid_state(Run* r, int Bw) {
  if (r->v && r->Bw >= Bw) return SNC_B200_OK;
  const Graph* g = r->g;
  dev_free(r->v); dev_free(r->refr); dev_free(r->ring); dev_free(r->fired); dev_free(r->fired_cnt);
  r->v = nullptr; r->refr = nullptr; r->ring = nullptr; r->fired = nullptr; r->fired_cnt = nullptr;
  int rc;
  if ((rc = dev_alloc(&r->v, (size_t)Bw * g->N))) return rc;
  if ((rc = dev_alloc(&r->refr, (size_t)Bw * g->N))) return rc;
  if ((rc = dev_alloc(&r->ring, (size_t)Bw * g->R * std::max(1, g->ncols)))) return rc;
  if ((rc = dev_alloc(&r->fired, (size_t)Bw * 2 * g->N))) return rc;
  if ((rc = dev_alloc(&r->fired_cnt, (size_t)Bw * 2 * g->P))) return rc;
  r->Bw = Bw;
  return SNC_B200_OK;
}

template <int MODE>
static int launch_tier_s(Run* r, const FwdArgs& a, cudaStream_t st) {
  const Graph* g = r->g;
  const int nthr = 1024;
  const size_t smem = tier_s_bytes(g->N, g->ncols, g->R, a.noc, MODE, false, nthr);
  SNCB_CUDA(cudaFuncSetAttribute(k_tier_s<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  SNCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tier_s<MODE>, nthr, smem));
  if (per_sm < 1) {
    set_error("tier S does not fit on an SM");
    return SNC_B200_EUNSUPPORTED;
  }
  const int grid = std::max(1, std::min(r->in->B, per_sm * g->sm_count));
  k_tier_s<MODE><<<grid, nthr, smem, st>>>(a);
  SNCB_CUDA(cudaGetLastError());
  return SNC_B200_OK;
}

template <int MODE>
static int launch_tier_g(Run* r, const FwdArgs& a, cudaStream_t st) {
  const Graph* g = r->g;
  const int nthr = 512;
  const size_t smem = tier_g_bytes(g->BS, g->P, nthr);
  SNCB_CUDA(cudaFuncSetAttribute(k_tier_g<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  SNCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tier_g<MODE>, nthr, smem));
  if (per_sm * g->sm_count < g->P) {
    set_error("grid tier: blocks cannot be co-resident");
    return SNC_B200_EUNSUPPORTED;
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(g->P);
  cfg.blockDim = dim3(nthr);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  SNCB_CUDA(cudaLaunchKernelEx(&cfg, k_tier_g<MODE>, a));
  return SNC_B200_OK;
}

template <int MODE>
static int launch_plain(Run* r, FwdArgs a, cudaStream_t st) {
  const Graph* g = r->g;
  const Inputs* in = r->in;
  const int nthr = 512;
  const size_t smem = tier_g_bytes(g->BS, g->P, nthr);
  SNCB_CUDA(cudaFuncSetAttribute(k_plain_a<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  SNCB_CUDA(cudaFuncSetAttribute(k_plain_b<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (int q = 0; q < in->B; ++q) {
    const int smp = in->order_h[q];
    const int T = in->steps_h[smp];
    k_plain_init<<<g->P, nthr, 0, st>>>(a);
    for (int t = 0; t < T; ++t) {
      k_plain_a<MODE><<<g->P, nthr, smem, st>>>(a, smp, t);
      if (MODE != MODE_ATOMIC) k_plain_b<MODE><<<g->P, nthr, smem, st>>>(a, t);
    }
    if (a.vfinal) k_copy_v<<<std::max(1, std::min(1024, (g->N + 255) / 256)), 256, 0, st>>>(a, smp);
  }
  SNCB_CUDA(cudaGetLastError());
  return SNC_B200_OK;
}

static bool tier_s_fits(const Graph* g, int mode) {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return tier_s_bytes(g->N, g->ncols, g->R, std::max(1, g->noc), mode, false, 1024) <= (size_t)optin;
}

// Launch body without timing / graph handling.
static int launch_body(Run* r, const FwdArgs& a, int mode, int path, cudaStream_t st) {
  const Graph* g = r->g;
  if (path == SNC_B200_PATH_PERSISTENT && tier_s_fits(g, mode) &&
      !(r->flags & SNC_B200_RUN_FORCE_GRID)) {
    if (mode == MODE_SORT) return launch_tier_s<MODE_SORT>(r, a, st);
    return launch_tier_s<MODE_ATOMIC>(r, a, st);
  }
  if (path == SNC_B200_PATH_PERSISTENT) {
    if (mode == MODE_SORT) return launch_tier_g<MODE_SORT>(r, a, st);
    if (mode == MODE_BUCKET) return launch_tier_g<MODE_BUCKET>(r, a, st);
    return launch_tier_g<MODE_ATOMIC>(r, a, st);
  }
  if (mode == MODE_SORT) return launch_plain<MODE_SORT>(r, a, st);
  if (mode == MODE_BUCKET) return launch_plain<MODE_BUCKET>(r, a, st);
  return launch_plain<MODE_ATOMIC>(r, a, st);
}

int launch_run(Run* r, const snc_lif* lif, int mode, int path, cudaStream_t st) {
  const Graph* g = r->g;
  const Inputs* in = r->in;
  if (mode == SNC_B200_MODE_AUTO || path == SNC_B200_PATH_AUTO) {
    int m = mode, p = path;
    int rc = resolve_auto(g, in, &m, &p);
    if (rc) return rc;
    if (mode == SNC_B200_MODE_AUTO) mode = m;
    if (path == SNC_B200_PATH_AUTO) path = p;
  }
  if (mode < 0 || mode > MODE_SORT || path < 0 || path > SNC_B200_PATH_PERSISTENT) {
    set_error("bad mode or path");
    return SNC_B200_EINVAL;
  }
  const bool tier_s = path == SNC_B200_PATH_PERSISTENT && tier_s_fits(g, mode) &&
                      !(r->flags & SNC_B200_RUN_FORCE_GRID);
  int rc;
  if (!tier_s) {
    int Bw = 1;
    if (path == SNC_B200_PATH_PERSISTENT) {
      // lockstep wave size: bounded by a 4 GiB state budget and 64 samples
      const size_t per = (size_t)4 * ((size_t)g->R * std::max(1, g->ncols) + 4 * (size_t)g->N);
      Bw = (int)std::max<size_t>(1, std::min<size_t>({(size_t)in->B, (size_t)64, ((size_t)4 << 30) / per}));
    }
    if ((rc = ensure_grid_state(r, Bw))) return rc;
  }
  const FwdArgs a = make_args(r, lif);
  const size_t B = (size_t)std::max(1, in->B);
  SNCB_CUDA(cudaMemsetAsync(r->counts, 0, B * std::max(1, g->noc) * sizeof(int), st));
  SNCB_CUDA(cudaMemsetAsync(r->spikes, 0, B * sizeof(unsigned long long), st));
  SNCB_CUDA(cudaMemsetAsync(r->events, 0, B * sizeof(unsigned long long), st));
  SNCB_CUDA(cudaMemsetAsync(r->ctl, 0, 4 * sizeof(unsigned), st));
  SNCB_CUDA(cudaMemsetAsync(r->err, 0, sizeof(int), st));
  if ((r->flags & SNC_B200_RUN_RASTER) && in->raster_words)
    SNCB_CUDA(cudaMemsetAsync(r->raster, 0, (size_t)in->raster_words * sizeof(uint32_t), st));
  SNCB_CUDA(cudaEventRecord(r->ev0, st));
  if (in->B > 0) {
    const bool use_graph = (r->flags & SNC_B200_RUN_GRAPH) && path == SNC_B200_PATH_PERSISTENT;
    if (use_graph) {
      const bool same = r->gexec && r->gexec_mode == mode && r->gexec_stream == st &&
                        std::memcmp(&r->gexec_lif, lif, sizeof(snc_lif)) == 0;
      if (!same) {
        if (r->gexec) cudaGraphExecDestroy(r->gexec);
        r->gexec = nullptr;
        cudaGraph_t cg = nullptr;
        SNCB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        rc = launch_body(r, a, mode, path, st);
        cudaError_t ce = cudaStreamEndCapture(st, &cg);
        if (rc) { if (cg) cudaGraphDestroy(cg); return rc; }
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
        ce = cudaGraphInstantiate(&r->gexec, cg, 0);
        cudaGraphDestroy(cg);
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
        r->gexec_mode = mode;
        r->gexec_lif = *lif;
        r->gexec_stream = st;
      }
      SNCB_CUDA(cudaGraphLaunch(r->gexec, st));
    } else {
      if ((rc = launch_body(r, a, mode, path, st))) return rc;
    }
  }
  SNCB_CUDA(cudaEventRecord(r->ev1, st));
  r->used_mode = mode;
  r->used_path = path;
  return SNC_B200_OK;
}

}  // namespace sncb
