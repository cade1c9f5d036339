// Device helpers shared by the forward, e-prop and BPTT kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sncb {

// Default wall-clock bound of every spin-wait in this library: a wait that
// has not finished after this many nanoseconds sets the error word and
// returns.  Launches carry their own bound (snc_b200_set_wait_limit); 0
// selects this default.
constexpr unsigned long long kSpinTimeoutNs = 2000000000ull;  // 2 s
constexpr int kErrTimeout = -5;                               // SNC_B200_ETIMEOUT

struct LifP {
  float thr, decay, reset;
  int refractory, reset_mode;
};

// cpu_backend.cpp:134 -- v * decay + ext + slot as three separately rounded
// IEEE operations in the CPU's order (no fused multiply-add), so the GPU and
// the serial CPU backend produce identical bits from identical inputs.
__device__ __forceinline__ float lif_integrate(float v, float decay, float ext, float ring) {
  return __fadd_rn(__fadd_rn(__fmul_rn(v, decay), ext), ring);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_volatile_i32(const int* p) {
  return *reinterpret_cast<const volatile int*>(p);
}

__device__ __forceinline__ void red_release_add_u32(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Block-wide exclusive scan of one int per thread (blockDim a multiple of 32,
// at most 1024).  scratch: >= 33 ints of shared memory.  Returns this
// thread's exclusive prefix and writes the block total to *total.
__device__ __forceinline__ int block_exclusive_scan(int x, int* scratch, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  int incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) scratch[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int s = lane < nw ? scratch[lane] : 0;
    int si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += y;
    }
    if (lane < nw) scratch[lane] = si - s;
    if (lane == 31) scratch[32] = si;
  }
  __syncthreads();
  const int res = scratch[warp] + incl - x;
  *total = scratch[32];
  __syncthreads();
  return res;
}

// Block-wide sum of one 64-bit value per thread; result valid in all threads.
__device__ __forceinline__ long long block_sum_ll(long long x, long long* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  if (lane == 0) scratch[warp] = x;
  __syncthreads();
  if (warp == 0) {
    long long s = lane < nw ? scratch[lane] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) scratch[32] = s;
  }
  __syncthreads();
  const long long r = scratch[32];
  __syncthreads();
  return r;
}

// Arrival count `c` has not reached `target` yet.  Counter and targets grow
// modulo 2^32; compared by signed distance, a long launch whose count wraps
// (about 30 M barriers of a 143-CTA grid) still waits correctly, since every
// arrival lies within a few grids of the target being waited on.
__device__ __forceinline__ bool before(unsigned c, unsigned target) {
  return static_cast<int>(c - target) < 0;
}

// Software grid barrier for a cooperatively launched (co-resident) grid.
// `ctr` counts arrivals and is never reset inside a launch; the n-th barrier
// of the launch waits for ctr >= n * gridDim.x (modulo 2^32, see before()).
// The wait is bounded: after limit_ns (kSpinTimeoutNs when 0) it records
// kErrTimeout in *err and every CTA returns false, so callers leave their
// loops and the context stays usable.
__device__ __forceinline__ bool grid_sync(unsigned* ctr, unsigned target, int* err,
                                          unsigned long long limit_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    // release: the CTA's writes (ordered before this thread by bar.sync)
    // become visible before the arrival is counted
    red_release_add_u32(ctr, 1u);
    int ok = 1;
    unsigned long long t0 = 0;
    unsigned spins = 0;
    while (before(ld_acquire_u32(ctr), target)) {
      if ((++spins & 255u) == 0) {
        if (ld_volatile_i32(err) != 0) { ok = 0; break; }
        const unsigned long long now = global_ns();
        if (t0 == 0) t0 = now;
        else if (now - t0 > (limit_ns ? limit_ns : kSpinTimeoutNs)) {
          atomicCAS(err, 0, kErrTimeout);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;  // the acquire load orders later reads after the other CTAs' writes
  }
  __syncthreads();
  return s_ok != 0;
}

// grid_sync split in two: arrive publishes this CTA's writes and counts it
// in; wait blocks until `target` arrivals (bounded as in grid_sync).  Work
// between the two must not touch data other CTAs write before the barrier.
__device__ __forceinline__ void grid_arrive(unsigned* ctr) {
  __syncthreads();
  if (threadIdx.x == 0) red_release_add_u32(ctr, 1u);
}

__device__ __forceinline__ bool grid_wait(unsigned* ctr, unsigned target, int* err,
                                          unsigned long long limit_ns) {
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned long long t0 = 0;
    unsigned spins = 0;
    while (before(ld_acquire_u32(ctr), target)) {
      if ((++spins & 255u) == 0) {
        if (ld_volatile_i32(err) != 0) { ok = 0; break; }
        const unsigned long long now = global_ns();
        if (t0 == 0) t0 = now;
        else if (now - t0 > (limit_ns ? limit_ns : kSpinTimeoutNs)) {
          atomicCAS(err, 0, kErrTimeout);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;  // the acquire load orders later reads after the other CTAs' writes
  }
  __syncthreads();
  return s_ok != 0;
}

// Largest k in [0, n) with a[k] <= x, for a non-decreasing a with a[0] <= x.
__device__ __forceinline__ int upper_index(const int* a, int n, int x) {
  int lo = 0, hi = n;  // invariant: a[lo] <= x, answer in [lo, hi)
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (a[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

// First k in [lo, hi) with a[k] >= x (hi when none).
__device__ __forceinline__ int lower_bound_i(const int* a, int lo, int hi, int x) {
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Philox-4x32 with 10 rounds (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC 2011): counter c, key k.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const unsigned hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const unsigned hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// Edge packing: x = ring column (24 bits) | delay << 24, y = signed weight bits.
__device__ __forceinline__ int edge_col(uint2 e) { return static_cast<int>(e.x & 0xFFFFFFu); }
__device__ __forceinline__ int edge_delay(uint2 e) { return static_cast<int>(e.x >> 24); }
__device__ __forceinline__ float edge_w(uint2 e) { return __uint_as_float(e.y); }

}  // namespace sncb

namespace sncb {

// Ordered compaction of one flag per thread with warp ballot / popc: returns
// the number of flagged threads before this one in thread order, writes the
// block total to *total and this warp's ballot to *mask.  scratch >= 33 ints.
__device__ __forceinline__ int ballot_compact(int flag, int* scratch, int* total, unsigned* mask) {
  const unsigned m = __ballot_sync(0xffffffffu, flag);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  if (lane == 0) scratch[warp] = __popc(m);
  __syncthreads();
  if (warp == 0) {
    const int c = lane < nw ? scratch[lane] : 0;
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane < nw) scratch[lane] = incl - c;
    if (lane == 31) scratch[32] = incl;
  }
  __syncthreads();
  const int pos = scratch[warp] + __popc(m & ((1u << lane) - 1u));
  *total = scratch[32];
  *mask = m;
  __syncthreads();
  return pos;
}

// ballot_compact with one CTA barrier instead of three: every warp scans the
// per-warp counts itself, and the caller alternates between two 32-int
// buffers (a buffer is written again only two calls later, after every
// thread has passed the barrier of the call in between).  blockDim <= 1024.
__device__ __forceinline__ int ballot_compact_1(int flag, int* buf, int* total, unsigned* mask) {
  const unsigned m = __ballot_sync(0xffffffffu, flag);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  if (lane == 0) buf[warp] = __popc(m);
  __syncthreads();
  const int c = lane < nw ? buf[lane] : 0;
  int incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const int before = __shfl_sync(0xffffffffu, incl - c, warp);
  *total = __shfl_sync(0xffffffffu, incl, 31);
  *mask = m;
  return before + __popc(m & ((1u << lane) - 1u));
}

}  // namespace sncb
