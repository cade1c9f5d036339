// Input schedules -- the reference's build_schedule (src/runtime/cpu_backend.cpp:43-65)
// batched over samples -- built on the GPU, and the per-graph workspace of the
// one-call forwards.
//
// The schedule of a batch lists, for every global step gs (sample b's step t
// is gs = stepbase[b] + t), the input neurons driven at that step in
// ascending id with their drive: the amplitudes of every event reaching the
// neuron at that step summed in event order, exactly as the CPU backend sums
// them.  The host uploads the events as they are plus five per-sample arrays;
// the device then
//   1. counts each step's (event, input neuron) entries      k_sched_count
//   2. scans the counts into per-step ranges                  scan_exclusive
//   3. scatters the entries into their step's range           k_sched_scatter
//      under the key (neuron << 32 | event index)
//   4. sorts each step's range by that key (shared-memory     k_sched_bucket
//      bitonic tiles, merged in global memory when a step
//      holds more than one tile) and sums every neuron's run
//      of amplitudes in key order, i.e. in event order
//   5. scans the merged counts and lays out the final arrays  k_sched_finish
// The key orders equal neurons by event index, which is the order the CPU
// backend adds them in, so the result is bit-identical to a serial build
// whatever order the atomics in step 3 produce.
//
// Device layout of a schedule (one allocation, each array 256-B aligned):
//   steps[B] i32 | order[B] i32 | sptr_off[B] i64 | stepbase[B] i64 |
//   raster_off[B] i64 | sched_ptr[TS + B] i32 | sched_blk[TS][P+1] i32 |
//   sched_nid[E] i32 | sched_ext[E] f32 | n_entries i32
#include <algorithm>
#include <cstring>
#include <numeric>

#include "device_common.cuh"
#include "internal.h"

namespace sncb {

namespace {

constexpr size_t kAlign = 256;
constexpr long long kMaxBlkEntries = 64ll << 20;  // sched_blk is skipped above this
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanBlock = kScanThreads * kScanItems;
constexpr int kSbThreads = 256;
constexpr int kSbTile = 2048;  // keys sorted in shared memory at once

inline size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

typedef unsigned long long u64;

// ---- exclusive scan of int counts (totals < 2^31) -----------------------------

// out[i] = sum of in[0..i) within this block's kScanBlock items; bsum[block] =
// the block's total.  A single-block launch also writes out[n] = total.
// in and out may alias (each item is read and written by one thread).
__global__ void __launch_bounds__(kScanThreads) k_scan_local(const int* in, int* out, long long n, int* bsum) {
  __shared__ int scratch[33];
  const long long base = (long long)blockIdx.x * kScanBlock + (long long)threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    v[j] = base + j < n ? in[base + j] : 0;
    s += v[j];
  }
  int tot;
  int ex = block_exclusive_scan(s, scratch, &tot);
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    if (base + j < n) out[base + j] = ex;
    ex += v[j];
  }
  if (threadIdx.x == 0) {
    bsum[blockIdx.x] = tot;
    if (gridDim.x == 1) out[n] = tot;
  }
}

// Adds the scanned block totals bex[0..nb] to every block; out[n] = bex[nb].
__global__ void __launch_bounds__(kScanThreads) k_scan_add(int* out, long long n, const int* bex) {
  const long long base = (long long)blockIdx.x * kScanBlock + (long long)threadIdx.x * kScanItems;
  const int add = bex[blockIdx.x];
#pragma unroll
  for (int j = 0; j < kScanItems; ++j)
    if (base + j < n) out[base + j] += add;
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = bex[gridDim.x];
}

}  // namespace

// Ints of scratch scan_exclusive needs for n items.
size_t scan_scratch_ints(long long n) {
  size_t s = 0;
  long long nb = std::max<long long>(1, (n + kScanBlock - 1) / kScanBlock);
  while (true) {
    s += (size_t)nb + 1;
    if (nb == 1) break;
    nb = (nb + kScanBlock - 1) / kScanBlock;
  }
  return s + 64;
}

// out[0..n] = exclusive prefix sums of in[0..n) and the total.
int scan_exclusive(const int* in, int* out, long long n, int* scratch, cudaStream_t st) {
  const long long nb = std::max<long long>(1, (n + kScanBlock - 1) / kScanBlock);
  k_scan_local<<<(unsigned)nb, kScanThreads, 0, st>>>(in, out, n, scratch);
  SNCB_CUDA(cudaGetLastError());
  if (nb == 1) return SNC_B200_OK;
  int rc = scan_exclusive(scratch, scratch, nb, scratch + nb + 1, st);
  if (rc) return rc;
  k_scan_add<<<(unsigned)nb, kScanThreads, 0, st>>>(out, n, scratch);
  SNCB_CUDA(cudaGetLastError());
  return SNC_B200_OK;
}

namespace {

// ---- schedule kernels ----------------------------------------------------------

struct SchedArgs {
  const snc_input_event* ev;
  long long n_ev;
  int B, TS, ignore_sample, nic, N, P, BS;
  const int* steps;
  const long long* stepbase;
  const int* cptr;   // [nic+1] channel -> input neurons
  const int* cids;
  int* gstep;        // [n_ev] global step or -1
  int* cnt;          // [TS]   entries per step
  int* boff;         // [TS+1] first entry of each step (raw)
  int* cursor;       // [TS]
  u64* keys;         // [cap] neuron << 32 | event index
  float* amps;       // [cap]
  u64* keys2;        // [cap] merge buffer
  float* amps2;
  int* tnid;         // [cap] merged, at the step's raw offset
  float* text;
  int* mcnt;         // [TS]   merged entries per step
  int* moff;         // [TS+1]
  long long cap;     // raw entry capacity
  // final schedule
  int* sptr;
  int* blk;          // null when skipped
  int* nid;
  float* ext;
  int* n_out;
  int* err;
};

__global__ void k_sched_count(SchedArgs a) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < a.n_ev;
       k += (long long)gridDim.x * blockDim.x) {
    const snc_input_event e = a.ev[k];
    const int b = a.ignore_sample ? 0 : e.sample_id;
    int gs = -1;
    if (b >= 0 && b < a.B && e.time >= 0 && e.time < a.steps[b] && e.channel_id >= 0 &&
        e.channel_id < a.nic) {
      gs = (int)(a.stepbase[b] + e.time);
      const int f = a.cptr[e.channel_id + 1] - a.cptr[e.channel_id];
      if (f) atomicAdd(&a.cnt[gs], f);
    }
    a.gstep[k] = gs;
  }
}

__global__ void k_sched_scatter(SchedArgs a) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < a.n_ev;
       k += (long long)gridDim.x * blockDim.x) {
    const int gs = a.gstep[k];
    if (gs < 0) continue;
    const snc_input_event e = a.ev[k];
    const int c0 = a.cptr[e.channel_id], f = a.cptr[e.channel_id + 1] - c0;
    if (!f) continue;
    const long long base = (long long)a.boff[gs] + atomicAdd(&a.cursor[gs], f);
    if (base + f > a.cap) {  // cannot happen when cap bounds the entries; never write past it
      atomicCAS(a.err, 0, -7);
      continue;
    }
    for (int q = 0; q < f; ++q) {
      a.keys[base + q] = ((u64)(unsigned)a.cids[c0 + q] << 32) | (u64)k;
      a.amps[base + q] = e.amplitude;
    }
  }
}

// In-place ascending bitonic sort of m (a power of two, <= kSbTile) keys in
// shared memory, carrying one float each.  Ends with __syncthreads.
__device__ void bitonic_sort(u64* k, float* v, int m) {
  for (int size = 2; size <= m; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < (m >> 1); i += blockDim.x) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const u64 x = k[lo], y = k[hi];
        if ((x > y) == up) {
          k[lo] = y;
          k[hi] = x;
          const float t = v[lo];
          v[lo] = v[hi];
          v[hi] = t;
        }
      }
      __syncthreads();
    }
}

// Merges every neuron's run in the n sorted keys: the drive is summed in key
// (= event) order starting from 0.0f, as cpu_backend.cpp sums it.  Writes the
// merged entries to onid/oext and returns their number (in every thread).
__device__ int merge_runs(const u64* keys, const float* amps, int n, int* onid, float* oext, int* scratch) {
  int total = 0;
  for (int t0 = 0; t0 < n; t0 += blockDim.x) {
    const int i = t0 + threadIdx.x;
    const int head = i < n && (i == 0 || (keys[i] >> 32) != (keys[i - 1] >> 32));
    int tot;
    const int r = block_exclusive_scan(head, scratch, &tot);
    if (head) {
      const u64 id = keys[i] >> 32;
      float acc = 0.0f;
      int j = i;
      do {
        acc = __fadd_rn(acc, amps[j]);
        ++j;
      } while (j < n && (keys[j] >> 32) == id);
      onid[total + r] = (int)id;
      oext[total + r] = acc;
    }
    total += tot;
  }
  return total;
}

// First index in [lo, hi) of a sorted key array whose key is >= x.
__device__ __forceinline__ long long lower_bound_u64(const u64* a, long long lo, long long hi, u64 x) {
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kSbThreads) k_sched_bucket(SchedArgs a) {
  __shared__ u64 sk[kSbTile];
  __shared__ float sv[kSbTile];
  __shared__ int scratch[33];
  for (int gs = blockIdx.x; gs < a.TS; gs += gridDim.x) {
    const long long lo = a.boff[gs];
    const int n = a.boff[gs + 1] - a.boff[gs];
    int merged = 0;
    if (n > 0 && n <= kSbTile) {
      int m = 1;
      while (m < n) m <<= 1;
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        sk[i] = i < n ? a.keys[lo + i] : ~0ull;
        sv[i] = i < n ? a.amps[lo + i] : 0.f;
      }
      __syncthreads();
      bitonic_sort(sk, sv, m);
      merged = merge_runs(sk, sv, n, a.tnid + lo, a.text + lo, scratch);
    } else if (n > kSbTile) {
      // sorted tiles, then pairwise merges of runs in global memory: an
      // element's place is its index in its run plus the number of keys of
      // the other run below it (keys are unique)
      u64* src = a.keys + lo;
      float* srcv = a.amps + lo;
      u64* dst = a.keys2 + lo;
      float* dstv = a.amps2 + lo;
      for (int t0 = 0; t0 < n; t0 += kSbTile) {
        const int len = min(kSbTile, n - t0);
        int m = 1;
        while (m < len) m <<= 1;
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
          sk[i] = i < len ? src[t0 + i] : ~0ull;
          sv[i] = i < len ? srcv[t0 + i] : 0.f;
        }
        __syncthreads();
        bitonic_sort(sk, sv, m);
        for (int i = threadIdx.x; i < len; i += blockDim.x) {
          src[t0 + i] = sk[i];
          srcv[t0 + i] = sv[i];
        }
        __syncthreads();
      }
      for (long long w = kSbTile; w < n; w *= 2) {
        for (long long i = threadIdx.x; i < n; i += blockDim.x) {
          const long long r0 = (i / (2 * w)) * (2 * w);
          const long long mid = min(r0 + w, (long long)n), end = min(r0 + 2 * w, (long long)n);
          const u64 key = src[i];
          const long long pos = i < mid ? (i - r0) + (lower_bound_u64(src, mid, end, key) - mid)
                                        : (i - mid) + (lower_bound_u64(src, r0, mid, key) - r0);
          dst[r0 + pos] = key;
          dstv[r0 + pos] = srcv[i];
        }
        __syncthreads();
        u64* tk = src; src = dst; dst = tk;
        float* tv = srcv; srcv = dstv; dstv = tv;
      }
      merged = merge_runs(src, srcv, n, a.tnid + lo, a.text + lo, scratch);
    }
    if (threadIdx.x == 0) a.mcnt[gs] = merged;
    __syncthreads();
  }
}

// Largest b with stepbase[b] <= gs (the sample whose steps contain gs).
__device__ __forceinline__ int sample_of(const long long* stepbase, int B, long long gs) {
  int lo = 0, hi = B;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (stepbase[mid] <= gs) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kSbThreads) k_sched_finish(SchedArgs a) {
  for (int gs = blockIdx.x; gs < a.TS; gs += gridDim.x) {
    const int src = a.boff[gs], dst = a.moff[gs], m = a.moff[gs + 1] - dst;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      a.nid[dst + i] = a.tnid[src + i];
      a.ext[dst + i] = a.text[src + i];
    }
    if (a.blk) {
      int* row = a.blk + (size_t)gs * (a.P + 1);
      for (int p = threadIdx.x; p <= a.P; p += blockDim.x)
        row[p] = p == a.P ? dst + m : dst + lower_bound_i(a.tnid + src, 0, m, min(a.N, p * a.BS));
    }
    if (threadIdx.x == 0) a.sptr[gs + sample_of(a.stepbase, a.B, gs)] = dst;
  }
  // the closing pointer of every sample
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < a.B; b += gridDim.x * blockDim.x)
    a.sptr[a.stepbase[b] + b + a.steps[b]] = a.moff[a.stepbase[b] + a.steps[b]];
  if (blockIdx.x == 0 && threadIdx.x == 0) *a.n_out = a.moff[a.TS];
}

}  // namespace

int HostImage::reserve(size_t n) {
  if (n <= cap) return SNC_B200_OK;
  const size_t want = std::max(n, cap + cap / 2);
  if (pinned) {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    void* q = nullptr;
    SNCB_CUDA(cudaHostAlloc(&q, want, cudaHostAllocDefault));
    p = static_cast<unsigned char*>(q);
  } else {
    vec.resize(want);
    p = vec.data();
  }
  cap = want;
  return SNC_B200_OK;
}

void HostImage::release() {
  if (pinned && p) cudaFreeHost(p);
  vec.clear();
  vec.shrink_to_fit();
  p = nullptr;
  cap = 0;
}

int DevBuf::reserve(size_t n) {
  if (n <= cap) return SNC_B200_OK;
  const size_t want = std::max(n, cap + cap / 2);
  release();
  if (alloc_fault()) { set_error("device allocation failed (injected)"); return SNC_B200_ENOMEM; }
  SNCB_CUDA(cudaMalloc(&p, want));
  cap = want;
  return SNC_B200_OK;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
}

int stage_inputs(const Graph* g, const snc_input_event* ev, size_t n_ev, int B, const int32_t* steps,
                 bool ignore_sample, Inputs* in, HostImage* img, DevBuf* keep, DevBuf* work,
                 cudaStream_t st, bool ev_device) {
  if (B < 0 || (B > 0 && !steps) || (n_ev > 0 && !ev)) {
    set_error("bad inputs arguments");
    return SNC_B200_EINVAL;
  }
  for (int b = 0; b < B; ++b)
    if (steps[b] < 0) { set_error("negative step count"); return SNC_B200_EINVAL; }
  if (n_ev > 0xFFFFFFFFull) { set_error("more than 2^32 events in one schedule"); return SNC_B200_EUNSUPPORTED; }
  // per-sample arrays (host)
  in->g = g;
  in->B = B;
  in->steps_h.assign(steps, steps + B);
  in->stepbase_h.assign(B, 0);
  in->sptr_off_h.assign(B, 0);
  long long TS = 0;
  for (int b = 0; b < B; ++b) {
    in->stepbase_h[b] = TS;
    in->sptr_off_h[b] = TS + b;
    TS += steps[b];
  }
  if (TS > (long long)INT32_MAX - B) { set_error("too many steps in one schedule"); return SNC_B200_EUNSUPPORTED; }
  in->total_steps = TS;
  in->Tmax = B ? *std::max_element(steps, steps + B) : 0;
  const int W = (g->N + 31) / 32;
  in->raster_off_h.assign(B, 0);
  for (int b = 0; b < B; ++b) in->raster_off_h[b] = in->stepbase_h[b] * W;
  in->raster_words = TS * W;
  // samples by descending step count (longest first balances uneven lengths)
  in->order_h.resize(B);
  std::iota(in->order_h.begin(), in->order_h.end(), 0);
  std::stable_sort(in->order_h.begin(), in->order_h.end(), [&](int x, int y) { return steps[x] > steps[y]; });
  // a bound on the (event, input neuron) entries: the events themselves when
  // every channel drives at most one neuron, else counted here (device
  // events: every event at the largest fan-out)
  long long cap = (long long)n_ev;
  if (g->max_fan > 1 && ev_device) {
    cap = (long long)n_ev * g->max_fan;
  } else if (g->max_fan > 1) {
    cap = 0;
    const int* cp = g->chan_ptr_h.data();
    for (size_t k = 0; k < n_ev; ++k) {
      const int c = ev[k].channel_id;
      if (c >= 0 && c < g->nic) cap += cp[c + 1] - cp[c];
    }
  }
  if (cap > (long long)INT32_MAX) { set_error("schedule too large"); return SNC_B200_EUNSUPPORTED; }
  const long long capn = std::max<long long>(1, cap);
  // layout of the kept block
  const long long nblk = TS * (long long)(g->P + 1);
  const bool with_blk = nblk > 0 && nblk <= kMaxBlkEntries;
  SchedLayout& L = in->layout;
  size_t off = 0;
  L.steps = off;      off = align_up(off + (size_t)B * 4);
  L.order = off;      off = align_up(off + (size_t)B * 4);
  L.sptr_off = off;   off = align_up(off + (size_t)B * 8);
  L.stepbase = off;   off = align_up(off + (size_t)B * 8);
  L.raster_off = off; off = align_up(off + (size_t)B * 8);
  const size_t head_bytes = off;
  L.sched_ptr = off;  off = align_up(off + (size_t)(TS + B) * 4);
  L.blk = with_blk ? off : 0;
  if (with_blk) off = align_up(off + (size_t)nblk * 4);
  L.nid = off;        off = align_up(off + (size_t)capn * 4);
  L.ext = off;        off = align_up(off + (size_t)capn * 4);
  L.n_out = off;      off = align_up(off + 4);
  L.total = off;
  // layout of the work block
  const size_t ts1 = (size_t)TS + 1;
  size_t w = 0;
  const size_t w_ev = w;     w = align_up(w + std::max<size_t>(1, n_ev) * sizeof(snc_input_event));
  const size_t w_gstep = w;  w = align_up(w + std::max<size_t>(1, n_ev) * 4);
  const size_t w_cnt = w;    w = align_up(w + ts1 * 4);      // cnt and cursor are zeroed together
  const size_t w_cursor = w; w = align_up(w + ts1 * 4);
  const size_t w_zero_end = w;
  const size_t w_boff = w;   w = align_up(w + ts1 * 4);
  const size_t w_keys = w;   w = align_up(w + (size_t)capn * 8);
  const size_t w_amps = w;   w = align_up(w + (size_t)capn * 4);
  const size_t w_keys2 = w;  w = align_up(w + (size_t)capn * 8);
  const size_t w_amps2 = w;  w = align_up(w + (size_t)capn * 4);
  const size_t w_tnid = w;   w = align_up(w + (size_t)capn * 4);
  const size_t w_text = w;   w = align_up(w + (size_t)capn * 4);
  const size_t w_mcnt = w;   w = align_up(w + ts1 * 4);
  const size_t w_moff = w;   w = align_up(w + ts1 * 4);
  const size_t w_err = w;    w = align_up(w + 4);
  const size_t w_scan = w;   w = align_up(w + scan_scratch_ints((long long)TS) * 4);
  int rc;
  if ((rc = keep->reserve(L.total))) return rc;
  if ((rc = work->reserve(w))) return rc;
  if ((rc = img->reserve(head_bytes))) return rc;
  unsigned char* h = img->p;
  if (B) {
    std::memcpy(h + L.steps, in->steps_h.data(), (size_t)B * 4);
    std::memcpy(h + L.order, in->order_h.data(), (size_t)B * 4);
    std::memcpy(h + L.sptr_off, in->sptr_off_h.data(), (size_t)B * 8);
    std::memcpy(h + L.stepbase, in->stepbase_h.data(), (size_t)B * 8);
    std::memcpy(h + L.raster_off, in->raster_off_h.data(), (size_t)B * 8);
  }
  unsigned char* K = static_cast<unsigned char*>(keep->p);
  unsigned char* Wk = static_cast<unsigned char*>(work->p);
  place_schedule(in, K);
  SNCB_CUDA(cudaMemcpyAsync(K, h, head_bytes, cudaMemcpyHostToDevice, st));
  if (n_ev && !ev_device)
    SNCB_CUDA(cudaMemcpyAsync(Wk + w_ev, ev, n_ev * sizeof(snc_input_event), cudaMemcpyHostToDevice, st));
  SNCB_CUDA(cudaMemsetAsync(Wk + w_cnt, 0, w_zero_end - w_cnt, st));
  SNCB_CUDA(cudaMemsetAsync(Wk + w_err, 0, 4, st));
  in->dev_bytes = (long long)(head_bytes + (ev_device ? 0 : n_ev * sizeof(snc_input_event)));

  SchedArgs a;
  a.ev = ev_device ? ev : reinterpret_cast<const snc_input_event*>(Wk + w_ev);
  a.n_ev = (long long)n_ev;
  a.B = B;
  a.TS = (int)TS;
  a.ignore_sample = ignore_sample ? 1 : 0;
  a.nic = g->nic;
  a.N = g->N;
  a.P = g->P;
  a.BS = g->BS;
  a.steps = in->steps;
  a.stepbase = in->stepbase;
  a.cptr = g->chan_ptr;
  a.cids = g->chan_ids;
  a.gstep = reinterpret_cast<int*>(Wk + w_gstep);
  a.cnt = reinterpret_cast<int*>(Wk + w_cnt);
  a.cursor = reinterpret_cast<int*>(Wk + w_cursor);
  a.boff = reinterpret_cast<int*>(Wk + w_boff);
  a.keys = reinterpret_cast<u64*>(Wk + w_keys);
  a.amps = reinterpret_cast<float*>(Wk + w_amps);
  a.keys2 = reinterpret_cast<u64*>(Wk + w_keys2);
  a.amps2 = reinterpret_cast<float*>(Wk + w_amps2);
  a.tnid = reinterpret_cast<int*>(Wk + w_tnid);
  a.text = reinterpret_cast<float*>(Wk + w_text);
  a.mcnt = reinterpret_cast<int*>(Wk + w_mcnt);
  a.moff = reinterpret_cast<int*>(Wk + w_moff);
  a.cap = cap;
  a.sptr = in->sched_ptr;
  a.blk = in->sched_blk;
  a.nid = in->sched_nid;
  a.ext = in->sched_ext;
  a.n_out = reinterpret_cast<int*>(K + L.n_out);
  a.err = reinterpret_cast<int*>(Wk + w_err);
  int* scan = reinterpret_cast<int*>(Wk + w_scan);
  const int sms = std::max(1, g->sm_count);
  if (n_ev) {
    const unsigned eg = (unsigned)std::min<long long>(((long long)n_ev + 255) / 256, (long long)sms * 16);
    k_sched_count<<<eg, 256, 0, st>>>(a);
    SNCB_CUDA(cudaGetLastError());
    if ((rc = scan_exclusive(a.cnt, a.boff, TS, scan, st))) return rc;
    k_sched_scatter<<<eg, 256, 0, st>>>(a);
    SNCB_CUDA(cudaGetLastError());
  } else {
    if ((rc = scan_exclusive(a.cnt, a.boff, TS, scan, st))) return rc;
  }
  const unsigned sg = (unsigned)std::max<long long>(1, std::min<long long>(TS, (long long)sms * 8));
  if (TS > 0) {
    k_sched_bucket<<<sg, kSbThreads, 0, st>>>(a);
    SNCB_CUDA(cudaGetLastError());
  }
  if ((rc = scan_exclusive(a.mcnt, a.moff, TS, scan, st))) return rc;
  k_sched_finish<<<sg, kSbThreads, 0, st>>>(a);
  SNCB_CUDA(cudaGetLastError());
  in->d_err = a.err;
  return SNC_B200_OK;
}

void place_schedule(Inputs* in, void* dev) {
  unsigned char* d = static_cast<unsigned char*>(dev);
  const SchedLayout& L = in->layout;
  in->steps = reinterpret_cast<int*>(d + L.steps);
  in->order = reinterpret_cast<int*>(d + L.order);
  in->sptr_off = reinterpret_cast<long long*>(d + L.sptr_off);
  in->stepbase = reinterpret_cast<long long*>(d + L.stepbase);
  in->raster_off = reinterpret_cast<long long*>(d + L.raster_off);
  in->sched_ptr = reinterpret_cast<int*>(d + L.sched_ptr);
  in->sched_blk = L.blk ? reinterpret_cast<int*>(d + L.blk) : nullptr;
  in->sched_nid = reinterpret_cast<int*>(d + L.nid);
  in->sched_ext = reinterpret_cast<float*>(d + L.ext);
  in->d_n_out = reinterpret_cast<int*>(d + L.n_out);
}

// A schedule of its own (snc_b200_inputs_upload, e-prop batches): built on
// the legacy stream and waited for, the work block freed afterwards.
int upload_inputs(const Graph* g, const snc_input_event* ev, size_t n_ev, int B,
                  const int32_t* steps, bool ignore_sample, Inputs* in) {
  HostImage img;
  DevBuf keep, work;
  int rc = stage_inputs(g, ev, n_ev, B, steps, ignore_sample, in, &img, &keep, &work, nullptr, false);
  in->dblock = keep.p;
  in->owns_block = true;
  keep.p = nullptr;  // owned by `in` from here on
  keep.cap = 0;
  if (rc) return rc;
  int host[2] = {0, 0};
  SNCB_CUDA(cudaMemcpy(&host[0], in->d_err, 4, cudaMemcpyDeviceToHost));
  SNCB_CUDA(cudaMemcpy(&host[1], in->d_n_out, 4, cudaMemcpyDeviceToHost));
  in->d_err = nullptr;
  if (host[0]) { set_error("schedule entries exceeded their bound"); return SNC_B200_EOVERFLOW; }
  in->n_entries = host[1];
  return SNC_B200_OK;
}

void free_inputs(Inputs* in) {
  if (!in) return;
  if (in->owns_block) dev_free(in->dblock);
  in->dblock = nullptr;
}

// ---- input encoders on the device --------------------------------------------
// snc::encode (src/training/encoders.cpp:25-71) for a whole batch: events are
// generated on the device from the features and fed to the schedule builder,
// so only the features cross the bus.  Direct and latency equal the
// reference's events exactly; Poisson draws its uniforms from Philox-4x32-10
// (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as easy as 1, 2,
// 3", SC 2011) instead of the reference's mt19937_64 stream -- the same
// Bernoulli rule u < min(1, v * max_rate), different draws.  Counter
// (t / 4, channel, sample, 0), key (seed low, seed high); word t % 4 of the
// output gives u = (word >> 8) * 2^-24.

namespace {

struct EncArgs {
  const float* feat;  // [B][C]
  const int* steps;   // [B]
  int B, C, enc;
  float gain, max_rate, thr;
  uint2 key;
  int* cnt;                // [B * C] events per (sample, channel)
  const int* off;          // [B * C + 1] their first slot
  snc_input_event* ev;     // [off[B * C]]
};


// Events of one (sample, channel); writes them to out when it is non-null.
__device__ int encode_one(const EncArgs& a, int b, int c, snc_input_event* out) {
  const int T = a.steps[b];
  const float v = a.feat[(size_t)b * a.C + c];
  if (!(v > a.thr) || T <= 0) return 0;
  if (a.enc == SNC_B200_ENCODER_DIRECT) {
    if (out) {
      const float amp = __fmul_rn(v, a.gain);
      for (int t = 0; t < T; ++t) out[t] = snc_input_event{b, c, t, amp};
    }
    return T;
  }
  if (a.enc == SNC_B200_ENCODER_LATENCY) {
    const float vc = fminf(1.f, v);
    const float x = __fmul_rn((float)(T - 1), __fsub_rn(1.f, vc));
    int t = (int)floor((double)x + 0.5);  // lround of a non-negative float
    t = min(max(t, 0), T - 1);
    if (out) out[0] = snc_input_event{b, c, t, a.gain};
    return 1;
  }
  const float prob = fminf(1.f, __fmul_rn(v, a.max_rate));
  int n = 0;
  for (int q = 0; 4 * q < T; ++q) {
    const uint4 w = philox4x32_10(make_uint4((unsigned)q, (unsigned)c, (unsigned)b, 0u), a.key);
    const unsigned ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int t = 4 * q + j;
      if (t < T && (float)(ws[j] >> 8) * (1.f / 16777216.f) < prob) {
        if (out) out[n] = snc_input_event{b, c, t, a.gain};
        ++n;
      }
    }
  }
  return n;
}

__global__ void k_enc_count(EncArgs a) {
  const long long n = (long long)a.B * a.C;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    a.cnt[i] = encode_one(a, (int)(i / a.C), (int)(i % a.C), nullptr);
}

__global__ void k_enc_write(EncArgs a) {
  const long long n = (long long)a.B * a.C;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    encode_one(a, (int)(i / a.C), (int)(i % a.C), a.ev + a.off[i]);
}

}  // namespace

int encode_inputs(const Graph* g, int enc, const float* features, int C, int B, const int32_t* steps,
                  float gain, float max_rate, float threshold, uint64_t seed, Inputs* in) {
  if (enc < SNC_B200_ENCODER_DIRECT || enc > SNC_B200_ENCODER_LATENCY || C < 0 || B < 0 ||
      (B > 0 && !steps) || ((long long)B * C > 0 && !features)) {
    set_error("encode: bad arguments");
    return SNC_B200_EINVAL;
  }
  long long bound = 0;  // events at most: every step of every (sample, channel)
  for (int b = 0; b < B; ++b) {
    if (steps[b] < 0) { set_error("negative step count"); return SNC_B200_EINVAL; }
    bound += (long long)C * steps[b];
  }
  if (bound > (long long)INT32_MAX) { set_error("encode: more than 2^31 possible events"); return SNC_B200_EUNSUPPORTED; }
  const long long nbc = (long long)B * C;
  DevBuf encw;
  size_t w = 0;
  const size_t w_feat = w;  w = align_up(w + (size_t)std::max(1ll, nbc) * 4);
  const size_t w_steps = w; w = align_up(w + (size_t)std::max(1, B) * 4);
  const size_t w_cnt = w;   w = align_up(w + (size_t)std::max(1ll, nbc) * 4);
  const size_t w_off = w;   w = align_up(w + (size_t)(nbc + 1) * 4);
  const size_t w_scan = w;  w = align_up(w + scan_scratch_ints(nbc) * 4);
  int rc;
  if ((rc = encw.reserve(w))) return rc;
  unsigned char* E = static_cast<unsigned char*>(encw.p);
  if (nbc) SNCB_CUDA(cudaMemcpy(E + w_feat, features, (size_t)nbc * 4, cudaMemcpyHostToDevice));
  if (B) SNCB_CUDA(cudaMemcpy(E + w_steps, steps, (size_t)B * 4, cudaMemcpyHostToDevice));
  EncArgs a;
  a.feat = reinterpret_cast<const float*>(E + w_feat);
  a.steps = reinterpret_cast<const int*>(E + w_steps);
  a.B = B;
  a.C = C;
  a.enc = enc;
  a.gain = gain;
  a.max_rate = max_rate;
  a.thr = threshold;
  a.key = make_uint2((unsigned)(seed & 0xFFFFFFFFull), (unsigned)(seed >> 32));
  a.cnt = reinterpret_cast<int*>(E + w_cnt);
  a.off = reinterpret_cast<const int*>(E + w_off);
  a.ev = nullptr;
  const int sms = std::max(1, g->sm_count);
  const unsigned grid = (unsigned)std::max(1ll, std::min((nbc + 255) / 256, (long long)sms * 8));
  if (nbc) {
    k_enc_count<<<grid, 256>>>(a);
    SNCB_CUDA(cudaGetLastError());
  }
  if ((rc = scan_exclusive(a.cnt, reinterpret_cast<int*>(E + w_off), nbc, reinterpret_cast<int*>(E + w_scan), nullptr)))
    return rc;
  int n_ev = 0;
  SNCB_CUDA(cudaMemcpy(&n_ev, E + w_off + (size_t)nbc * 4, 4, cudaMemcpyDeviceToHost));
  DevBuf evbuf;
  if ((rc = evbuf.reserve((size_t)std::max(1, n_ev) * sizeof(snc_input_event)))) return rc;
  a.ev = static_cast<snc_input_event*>(evbuf.p);
  if (n_ev) {
    k_enc_write<<<grid, 256>>>(a);
    SNCB_CUDA(cudaGetLastError());
  }
  HostImage img;
  DevBuf keep, work;
  rc = stage_inputs(g, a.ev, (size_t)n_ev, B, steps, false, in, &img, &keep, &work, nullptr, true);
  in->dblock = keep.p;
  in->owns_block = true;
  keep.p = nullptr;
  keep.cap = 0;
  if (rc) return rc;
  int host[2] = {0, 0};
  SNCB_CUDA(cudaMemcpy(&host[0], in->d_err, 4, cudaMemcpyDeviceToHost));
  SNCB_CUDA(cudaMemcpy(&host[1], in->d_n_out, 4, cudaMemcpyDeviceToHost));
  in->d_err = nullptr;
  if (host[0]) { set_error("schedule entries exceeded their bound"); return SNC_B200_EOVERFLOW; }
  in->n_entries = host[1];
  in->dev_bytes += (long long)nbc * 4 + (long long)B * 4;  // plus the features and step counts
  return SNC_B200_OK;
}

// ---- one-call forward workspace ---------------------------------------------
// snc_b200_forward and snc_b200_forward_batched are called once per sample or
// batch by the reference's runtime; allocating and freeing device memory on
// every call would cost more than the simulation.  The workspace keeps the
// schedule's blocks, a pinned staging buffer, the run's outputs and grid
// state and a stream per graph, grown on demand; calls on one graph are
// serialised by its mutex.

static std::mutex g_oneshot_mu;  // creation of Graph::oneshot

int oneshot_forward(const Graph* g, const snc_input_event* ev, size_t n_ev, int B,
                    const int32_t* steps, bool ignore_sample, const snc_lif* lif, int mode,
                    int path, float* logits, int64_t* spikes, int64_t* events_out,
                    snc_run_stats* stats) {
  OneShot* ws;
  {
    std::lock_guard<std::mutex> lk(g_oneshot_mu);
    if (!g->oneshot) g->oneshot = new OneShot();
    ws = g->oneshot;
  }
  std::lock_guard<std::mutex> lk(ws->mu);
  int rc;
  if (!ws->stream) SNCB_CUDA(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking));
  Inputs& in = ws->in;
  in.owns_block = false;
  if ((rc = stage_inputs(g, ev, n_ev, B, steps, ignore_sample, &in, &ws->img, &ws->keep, &ws->work,
                         ws->stream, false)))
    return rc;
  in.dblock = ws->keep.p;
  Run& r = ws->run;
  if (!r.g) {
    r.g = g;
    r.in = &in;
    r.flags = 0;
    r.W = (g->N + 31) / 32;
    SNCB_CUDA(cudaEventCreate(&r.ev0));
    SNCB_CUDA(cudaEventCreate(&r.ev1));
    if ((rc = dev_alloc(&r.err, 1))) return rc;
    if ((rc = dev_alloc(&r.ctl, 4))) return rc;
  }
  const int Bc = std::max(1, B);
  if (Bc > ws->B_cap) {
    for (void* p : {(void*)r.counts, (void*)r.spikes, (void*)r.events}) dev_free(p);
    r.counts = nullptr;
    r.spikes = nullptr;
    r.events = nullptr;
    ws->B_cap = 0;
    if ((rc = dev_alloc(&r.counts, (size_t)Bc * std::max(1, g->noc)))) return rc;
    if ((rc = dev_alloc(&r.spikes, (size_t)Bc))) return rc;
    if ((rc = dev_alloc(&r.events, (size_t)Bc))) return rc;
    ws->B_cap = Bc;
  }
  if ((rc = launch_run(&r, lif, mode, path, ws->stream))) return rc;
  int err = 0;
  rc = fetch_run(&r, logits, spikes, events_out, nullptr, nullptr, stats, in.d_err, &err);
  if (err && !rc) {
    set_error("schedule entries exceeded their bound");
    rc = SNC_B200_EOVERFLOW;
    if (stats) stats->overflow = 1;
  }
  return rc;
}

void free_oneshot(const Graph* g) {
  OneShot* ws = g->oneshot;
  if (!ws) return;
  free_run(&ws->run);
  ws->keep.release();
  ws->work.release();
  ws->img.release();
  if (ws->stream) cudaStreamDestroy(ws->stream);
  delete ws;
  g->oneshot = nullptr;
}

}  // namespace sncb
