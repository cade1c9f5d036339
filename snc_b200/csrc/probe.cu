// The atomic half of the delivery roofline: the rate at which this GPU's L2
// completes float reductions (red.global.add.f32, the ATOMIC delivery's
// primitive) at scattered addresses of a buffer the size of a delay ring.
// Every thread of an all-SM grid issues a stream of reductions at addresses
// from its own linear congruential sequence (Numerical Recipes' constants),
// so a warp's 32 lanes hit 32 unrelated words -- the access pattern of events
// landing on random ring columns.
#include <algorithm>

#include "internal.h"

namespace sncb {

namespace {

__global__ void k_red_probe(float* buf, unsigned n, long long per_thread, unsigned seed) {
  unsigned x = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u ^ seed;
  for (long long i = 0; i < per_thread; ++i) {
    x = x * 1664525u + 1013904223u;
    atomicAdd(buf + __umulhi(x, n), 1.0f);  // result unused: compiled as a reduction
  }
}

}  // namespace

}  // namespace sncb

using namespace sncb;

extern "C" int snc_b200_probe_red_rate(int64_t n_slots, int64_t n_ops, double* reds_per_s) {
  if (!reds_per_s || n_slots < 1 || n_slots > (1ll << 31) || n_ops < 1) {
    set_error("probe_red_rate: 1 <= n_slots <= 2^31, n_ops >= 1, output pointer");
    return SNC_B200_EINVAL;
  }
  *reds_per_s = 0.0;
  int dev = 0, sms = 148;
  SNCB_CUDA(cudaGetDevice(&dev));
  SNCB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int threads = 256, blocks = sms * 8;
  const long long nthr = (long long)threads * blocks;
  const long long per = std::max(1ll, (long long)(n_ops / nthr));
  float* buf = nullptr;
  int rc;
  if ((rc = dev_alloc(&buf, (size_t)n_slots))) return rc;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  if (ce == cudaSuccess) ce = cudaMemset(buf, 0, (size_t)n_slots * 4);
  float ms = 0.f;
  for (int rep = 0; rep < 2 && ce == cudaSuccess; ++rep) {  // the first launch warms the L2
    cudaEventRecord(e0);
    k_red_probe<<<blocks, threads>>>(buf, (unsigned)n_slots, per, 0x9E3779B9u + rep);
    cudaEventRecord(e1);
    ce = cudaEventSynchronize(e1);
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  dev_free(buf);
  if (ce != cudaSuccess) return cuda_fail(ce, "probe_red_rate");
  *reds_per_s = (double)nthr * (double)per / ((double)ms * 1e-3);
  return SNC_B200_OK;
}
