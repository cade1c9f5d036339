// SNCG graph files parsed and packed on the device.
//
// The wire format is snc_export's (src/bench/snc_export.cpp:107-123, read by
// python/snc/graph.py:11-24): little-endian int32 words
//   'SNCG', N, S, n_in, n_out, pre[S], post[S], delays[S], role[N], channel[N]
// with pre[] in CSR order (non-decreasing), optionally followed by this
// backend's weights section 'SNCW', S, weights[S] (fp32), sign[N] (int32)
// that older readers ignore; without it every weight is 1 and every sign +1
// (snc_b200.graph.graph_from_sncg does the same on the host).
//
// The host checks the header and sizes and copies the file image to the
// device once.  The O(S) work runs there: range and order checks of every
// edge, the largest delay, in-degrees (k_sncg_edges), the CSR row pointers
// from the sorted pre[] (k_sncg_rows), and then the packing of the delivery
// layout (build_graph_device_cols).  Only O(N) arrays come back to the host
// for the per-neuron tables.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "device_common.cuh"
#include "internal.h"

namespace sncb {

namespace {

constexpr int32_t kSncgMagic = 0x534E4347;  // 'SNCG'
constexpr int32_t kSncwMagic = 0x534E4357;  // 'SNCW'

enum : unsigned {
  kBadPre = 1,      // pre out of range or not in CSR order
  kBadPost = 2,     // post out of range
  kBadDelay = 4,    // delay < 1
  kBigDelay = 8,    // delay > 255 (this backend's limit)
};

// Per edge: range and order checks, the largest delay, in-degrees.
__global__ void k_sncg_edges(const int* __restrict__ pre, const int* __restrict__ post,
                             const int* __restrict__ delays, int S, int N, int* indeg,
                             unsigned* flags, int* max_delay) {
  unsigned bad = 0;
  int dmax = 1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < S; e += gridDim.x * blockDim.x) {
    const int p = pre[e], q = post[e], d = delays[e];
    if (p < 0 || p >= N || (e > 0 && pre[e - 1] > p)) bad |= kBadPre;
    if (q < 0 || q >= N) bad |= kBadPost;
    else atomicAdd(&indeg[q], 1);
    if (d < 1) bad |= kBadDelay;
    if (d > 255) bad |= kBigDelay;
    dmax = max(dmax, d);
  }
  if (bad) atomicOr(flags, bad);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dmax = max(dmax, __shfl_down_sync(0xffffffffu, dmax, o));
  if ((threadIdx.x & 31) == 0) atomicMax(max_delay, dmax);
}

// row_ptr[i] = first edge whose pre is >= i (pre[] sorted), i in [0, N].
__global__ void k_sncg_rows(const int* __restrict__ pre, int S, int N, int* row_ptr) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= N; i += gridDim.x * blockDim.x)
    row_ptr[i] = lower_bound_i(pre, 0, S, i);
}

__global__ void k_fill_f32(float* p, size_t n, float v) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    p[i] = v;
}

}  // namespace

}  // namespace sncb

using namespace sncb;

extern "C" int snc_b200_graph_upload_sncg(const void* data, size_t bytes, snc_b200_graph** out) {
  if (!out || !data) { set_error("null argument"); return SNC_B200_EINVAL; }
  *out = nullptr;
  const unsigned char* img = static_cast<const unsigned char*>(data);
  if (bytes < 20) { set_error("SNCG: shorter than its header"); return SNC_B200_EINVAL; }
  int32_t hdr[5];
  std::memcpy(hdr, img, sizeof(hdr));
  if (hdr[0] != kSncgMagic) { set_error("SNCG: bad magic"); return SNC_B200_EINVAL; }
  const int N = hdr[1], S = hdr[2];
  if (N < 0 || S < 0) { set_error("SNCG: negative N or S"); return SNC_B200_EINVAL; }
  if (N >= (1 << 24)) { set_error("num_neurons >= 2^24 is outside this backend's limits"); return SNC_B200_EUNSUPPORTED; }
  const size_t base = 20 + 12 * (size_t)S + 8 * (size_t)N;  // end of the reference's arrays
  if (bytes < base) { set_error("SNCG: truncated file"); return SNC_B200_EINVAL; }
  bool has_w = false;
  if (bytes >= base + 8) {
    int32_t w2[2];
    std::memcpy(w2, img + base, 8);
    has_w = w2[0] == kSncwMagic && w2[1] == S && bytes >= base + 8 + 4 * (size_t)S + 4 * (size_t)N;
  }
  int rc = SNC_B200_OK;
  // host views of the per-neuron arrays (O(N)) and of the columns for the hash
  const int32_t* h_pre = reinterpret_cast<const int32_t*>(img + 20);
  const int32_t* h_post = h_pre + S;
  const int32_t* h_del = h_post + S;
  const int32_t* h_role = h_del + S;
  const int32_t* h_chan = h_role + N;
  std::vector<uint8_t> role8(N);
  std::vector<int8_t> sign8(N, 1);
  for (int i = 0; i < N; ++i) {
    int32_t r;
    std::memcpy(&r, h_role + i, 4);
    if (r < 0 || r > 2) { set_error("SNCG: role outside 0..2"); return SNC_B200_EINVAL; }
    role8[i] = (uint8_t)r;
  }
  std::vector<int32_t> chan(N);
  if (N) std::memcpy(chan.data(), h_chan, 4 * (size_t)N);
  std::vector<float> ones;
  const float* h_w = nullptr;
  if (has_w) {
    h_w = reinterpret_cast<const float*>(img + base + 8);
    const int32_t* h_sign = reinterpret_cast<const int32_t*>(h_w + S);
    for (int i = 0; i < N; ++i) {
      int32_t sg;
      std::memcpy(&sg, h_sign + i, 4);
      if (sg != 1 && sg != -1) { set_error("SNCG: sign not +1 / -1"); return SNC_B200_EINVAL; }
      sign8[i] = (int8_t)sg;
    }
  } else {
    ones.assign(S, 1.0f);
    h_w = ones.data();
  }
  {  // the edge checks need the device
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      cudaGetLastError();
      set_error("no CUDA device");
      return SNC_B200_ENODEV;
    }
  }
  auto* g = new snc_b200_graph();
  DevBuf dimg, work;
  auto fail = [&](int code) {
    free_graph(g);
    delete g;
    return code;
  };

  // the file image on the device: pre, post, delays (and weights) in place
  const size_t img_bytes = has_w ? base + 8 + 4 * (size_t)S : base;
  if ((rc = dimg.reserve(std::max<size_t>(img_bytes, 4)))) return fail(rc);
  auto dcp = [&](void* dst, const void* src, size_t n, cudaMemcpyKind k) {
    return n ? cudaMemcpy(dst, src, n, k) : cudaSuccess;
  };
  cudaError_t ce = dcp(dimg.p, img, img_bytes, cudaMemcpyHostToDevice);
  if (ce != cudaSuccess) return fail(cuda_fail(ce, "cudaMemcpy(SNCG image)"));
  const int* d_pre = reinterpret_cast<const int*>(static_cast<unsigned char*>(dimg.p) + 20);
  const int* d_post = d_pre + S;
  const int* d_del = d_post + S;
  // work: indeg [N] | flags, max delay | sign8 [N] | ones [S] when no weights
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t o_indeg = 0, o_ctl = al(4 * (size_t)std::max(1, N)), o_sign = al(o_ctl + 8);
  const size_t o_ones = al(o_sign + (size_t)std::max(1, N));
  const size_t wbytes = o_ones + (has_w ? 0 : 4 * (size_t)std::max(1, S));
  if ((rc = work.reserve(wbytes))) return fail(rc);
  unsigned char* W = static_cast<unsigned char*>(work.p);
  int* d_indeg = reinterpret_cast<int*>(W + o_indeg);
  unsigned* d_flags = reinterpret_cast<unsigned*>(W + o_ctl);
  int* d_maxd = reinterpret_cast<int*>(W + o_ctl + 4);
  int8_t* d_sign = reinterpret_cast<int8_t*>(W + o_sign);
  const float* d_w = has_w ? reinterpret_cast<const float*>(static_cast<unsigned char*>(dimg.p) + base + 8)
                           : reinterpret_cast<const float*>(W + o_ones);
  const int one = 1;
  if ((ce = cudaMemset(W, 0, o_sign)) != cudaSuccess) return fail(cuda_fail(ce, "cudaMemset"));
  if ((ce = cudaMemcpy(d_maxd, &one, 4, cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(cuda_fail(ce, "cudaMemcpy"));
  if ((ce = dcp(d_sign, sign8.data(), (size_t)N, cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(cuda_fail(ce, "cudaMemcpy(sign)"));
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (!has_w && S) {
    k_fill_f32<<<sms * 4, 256>>>(reinterpret_cast<float*>(W + o_ones), (size_t)S, 1.0f);
  }
  if (S) k_sncg_edges<<<sms * 8, 256>>>(d_pre, d_post, d_del, S, N, d_indeg, d_flags, d_maxd);
  if ((rc = dev_alloc(&g->row_ptr, (size_t)N + 1))) return fail(rc);
  k_sncg_rows<<<std::max(1, std::min(sms * 8, (N + 256) / 256)), 256>>>(d_pre, S, N, g->row_ptr);
  if ((ce = cudaGetLastError()) != cudaSuccess) return fail(cuda_fail(ce, "SNCG kernels"));
  unsigned flags = 0;
  int max_delay = 1;
  std::vector<int> indeg(N), row_ptr(N + 1);
  if ((ce = cudaMemcpy(&flags, d_flags, 4, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (ce = cudaMemcpy(&max_delay, d_maxd, 4, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (ce = dcp(indeg.data(), d_indeg, 4 * (size_t)N, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (ce = cudaMemcpy(row_ptr.data(), g->row_ptr, 4 * ((size_t)N + 1), cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail(cuda_fail(ce, "cudaMemcpy(SNCG results)"));
  if (flags & kBadPre) { set_error("SNCG: pre id out of range or pre[] not in CSR order"); return fail(SNC_B200_EINVAL); }
  if (flags & kBadPost) { set_error("post id out of range"); return fail(SNC_B200_EINVAL); }
  if (flags & kBadDelay) { set_error("delay < 1"); return fail(SNC_B200_EINVAL); }
  if (flags & kBigDelay) { set_error("delay > 255 is outside this backend's limits"); return fail(SNC_B200_EUNSUPPORTED); }
  // the content hash of the same arrays a view upload would hash
  snc_graph_view v{N, S, row_ptr.data(), h_post, h_w, h_del, role8.data(), sign8.data(), chan.data()};
  g->hash = graph_hash_view(&v);
  if ((rc = setup_tables(g, N, S, max_delay, row_ptr.data(), indeg.data(), role8.data(), chan.data())))
    return fail(rc);
  if ((rc = dev_alloc(&g->post, (size_t)S))) return fail(rc);
  if ((ce = dcp(g->post, d_post, 4 * (size_t)S, cudaMemcpyDeviceToDevice)) != cudaSuccess)
    return fail(cuda_fail(ce, "cudaMemcpy(post)"));
  if ((rc = build_graph_device_cols(g, d_w, d_del, d_sign))) return fail(rc);
  *out = g;
  return SNC_B200_OK;
}
