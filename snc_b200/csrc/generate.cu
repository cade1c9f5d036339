// Grid graphs generated on the device: the large recurrent substrate of the
// benchmark's C2 configuration (neurons on a 2-D torus, most targets local,
// a few long-range, heavy-tailed in-degree) built where it is used, from a
// counter-based generator, instead of on the host and copied over.
//
// Every random number is one Philox-4x32-10 word (Salmon et al., SC 2011)
// keyed by the seed and counted by (neuron, draw, stream); every derived
// quantity is integer arithmetic or one correctly rounded float operation,
// so a host restatement reproduces the graph bit for bit:
//   local target d of neuron i = (x, y): r = Philox(i, d, 0, 0),
//     dx = rint(c_disp * float(sum of the four 16-bit halves of r.x, r.y
//          - 2^17)), dy likewise from r.z, r.w (an Irwin-Hall(4) variate:
//          mean 0, standard deviation sigma, |dx| <= 2 sqrt(3) sigma),
//     candidate j = ((y + dy) mod H) * W + (x + dx) mod W, kept when
//     Philox(i, d, 1, 0).x < accept[j] (accept[j] / 2^32 is j's acceptance
//     probability: the in-degree skew), or unconditionally from draw
//     max_draws on; draws continue until out_degree - long_range targets;
//   long-range target q: mulhi(Philox(i, q, 2, 0).x, N);
//   synapse s of row i: r = Philox(i, s, 3, 0), weight = c_w * float(sum of
//     the halves of r.x, r.y - 2^17), delay = 1 + mulhi(r.z, max_delay);
// rows are neuron-major in draw order (the CSR order).  c_disp = sigma *
// sqrt(3) / 2^16 and c_w = w_std * sqrt(3) / 2^16 are rounded to float once.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "internal.h"

namespace sncb {

namespace {

struct GenArgs {
  int W, H, N, k, k_loc, max_delay, max_draws;
  float c_disp, c_w;
  uint2 key;
  const unsigned* accept;  // [N]
  int* post;               // [N * k]
  float* w;                // [N * k]
  int* delay;              // [N * k]
  int* indeg;              // [N]
  int* dmax;               // the largest delay drawn
};

__device__ __forceinline__ int halves_sum(unsigned a, unsigned b) {
  return (int)(a >> 16) + (int)(a & 0xFFFFu) + (int)(b >> 16) + (int)(b & 0xFFFFu) - 131072;
}

// One thread per neuron: its row in draw order.
__global__ void k_gen_grid(GenArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.N; i += gridDim.x * blockDim.x) {
    const int x = i % a.W, y = i / a.W;
    const size_t row = (size_t)i * a.k;
    int got = 0;
    for (int d = 0; got < a.k_loc; ++d) {
      const uint4 r = philox4x32_10(make_uint4((unsigned)i, (unsigned)d, 0u, 0u), a.key);
      const int dx = __float2int_rn(__fmul_rn((float)halves_sum(r.x, r.y), a.c_disp));
      const int dy = __float2int_rn(__fmul_rn((float)halves_sum(r.z, r.w), a.c_disp));
      const int cx = ((x + dx) % a.W + a.W) % a.W, cy = ((y + dy) % a.H + a.H) % a.H;
      const int j = cy * a.W + cx;
      const unsigned u = philox4x32_10(make_uint4((unsigned)i, (unsigned)d, 1u, 0u), a.key).x;
      if (u < a.accept[j] || d >= a.max_draws) a.post[row + got++] = j;
    }
    for (int q = 0; q < a.k - a.k_loc; ++q) {
      const unsigned u = philox4x32_10(make_uint4((unsigned)i, (unsigned)q, 2u, 0u), a.key).x;
      a.post[row + a.k_loc + q] = (int)__umulhi(u, (unsigned)a.N);
    }
    int dm = 1;
    for (int s = 0; s < a.k; ++s) {
      const uint4 r = philox4x32_10(make_uint4((unsigned)i, (unsigned)s, 3u, 0u), a.key);
      a.w[row + s] = __fmul_rn((float)halves_sum(r.x, r.y), a.c_w);
      const int d = 1 + (int)__umulhi(r.z, (unsigned)a.max_delay);
      a.delay[row + s] = d;
      dm = max(dm, d);
      atomicAdd(&a.indeg[a.post[row + s]], 1);
    }
    atomicMax(a.dmax, dm);
  }
}

__global__ void k_row_ptr_regular(int* row_ptr, int N, int k) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= N; i += gridDim.x * blockDim.x)
    row_ptr[i] = i * k;
}

}  // namespace

}  // namespace sncb

using namespace sncb;

extern "C" int snc_b200_graph_generate_grid(const snc_grid_graph* p, const uint32_t* accept,
                                            const uint8_t* role, const int8_t* sign,
                                            const int32_t* channel, snc_b200_graph** out) {
  if (!out || !p || !accept || !role || !sign || !channel) { set_error("null argument"); return SNC_B200_EINVAL; }
  *out = nullptr;
  const long long n_ll = (long long)p->width * p->height;
  if (p->width < 1 || p->height < 1 || n_ll >= (1 << 24) || p->out_degree < 0 || p->long_range < 0 ||
      p->long_range > p->out_degree || !(p->sigma >= 0.f) || p->max_delay < 1 || p->max_draws < 0 ||
      n_ll * p->out_degree >= (1ll << 31)) {
    set_error("generate_grid: width, height >= 1, N < 2^24, 0 <= long_range <= out_degree, "
              "sigma >= 0, max_delay >= 1, max_draws >= 0, N * out_degree < 2^31");
    return SNC_B200_EINVAL;
  }
  if (p->max_delay > 255) { set_error("delay > 255 is outside this backend's limits"); return SNC_B200_EUNSUPPORTED; }
  const int N = (int)n_ll, k = p->out_degree, S = N * k;
  for (int i = 0; i < N; ++i)
    if (role[i] > 2 || (sign[i] != 1 && sign[i] != -1)) {
      set_error("generate_grid: role outside 0..2 or sign not +1 / -1");
      return SNC_B200_EINVAL;
    }
  {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      cudaGetLastError();
      set_error("no CUDA device");
      return SNC_B200_ENODEV;
    }
  }
  auto* g = new snc_b200_graph();
  auto fail = [&](int code) {
    free_graph(g);
    delete g;
    return code;
  };
  // work: accept [N] | weights [S] | delays [S] | in-degrees [N], max delay | signs [N]
  DevBuf work;
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t o_acc = 0, o_w = al(4 * (size_t)std::max(1, N));
  const size_t o_d = al(o_w + 4 * (size_t)std::max(1, S));
  const size_t o_in = al(o_d + 4 * (size_t)std::max(1, S));
  const size_t o_sg = al(o_in + 4 * ((size_t)N + 1));
  int rc;
  if ((rc = work.reserve(al(o_sg + (size_t)std::max(1, N))))) return fail(rc);
  unsigned char* Wb = static_cast<unsigned char*>(work.p);
  if ((rc = dev_alloc(&g->row_ptr, (size_t)N + 1))) return fail(rc);
  if ((rc = dev_alloc(&g->post, (size_t)S))) return fail(rc);
  cudaError_t ce;
  if ((N && (ce = cudaMemcpy(Wb + o_acc, accept, 4 * (size_t)N, cudaMemcpyHostToDevice)) != cudaSuccess) ||
      (N && (ce = cudaMemcpy(Wb + o_sg, sign, (size_t)N, cudaMemcpyHostToDevice)) != cudaSuccess) ||
      (ce = cudaMemset(Wb + o_in, 0, 4 * ((size_t)N + 1))) != cudaSuccess)
    return fail(cuda_fail(ce, "generate_grid: staging"));
  GenArgs a;
  a.W = p->width;
  a.H = p->height;
  a.N = N;
  a.k = k;
  a.k_loc = k - p->long_range;
  a.max_delay = p->max_delay;
  a.max_draws = p->max_draws > 0 ? p->max_draws : 1000 * std::max(1, k);
  a.c_disp = (float)((double)p->sigma * std::sqrt(3.0) / 65536.0);
  a.c_w = (float)((double)p->w_std * std::sqrt(3.0) / 65536.0);
  a.key = make_uint2((unsigned)(p->seed & 0xFFFFFFFFull), (unsigned)(p->seed >> 32));
  a.accept = reinterpret_cast<const unsigned*>(Wb + o_acc);
  a.post = g->post;
  a.w = reinterpret_cast<float*>(Wb + o_w);
  a.delay = reinterpret_cast<int*>(Wb + o_d);
  a.indeg = reinterpret_cast<int*>(Wb + o_in);
  a.dmax = a.indeg + N;  // stays 0 for an empty graph: max_delay 1 below
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (N) k_gen_grid<<<std::max(1, std::min(sms * 8, (N + 127) / 128)), 128>>>(a);
  k_row_ptr_regular<<<std::max(1, std::min(sms * 8, (N + 256) / 256)), 256>>>(g->row_ptr, N, k);
  if ((ce = cudaGetLastError()) != cudaSuccess) return fail(cuda_fail(ce, "generate_grid kernels"));
  std::vector<int> indeg(N + 1), row_ptr(N + 1);
  for (int i = 0; i <= N; ++i) row_ptr[i] = i * k;
  if ((ce = cudaMemcpy(indeg.data(), a.indeg, 4 * ((size_t)N + 1), cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail(cuda_fail(ce, "generate_grid: in-degrees"));
  const int max_delay = std::max(1, indeg[N]);
  // the autotuner's key of a generated graph: everything that determines it
  {
    const int32_t none = 0;
    snc_graph_view v{N, 0, row_ptr.data(), &none, reinterpret_cast<const float*>(&none), &none, role,
                     sign, channel};
    unsigned long long h = graph_hash_view(&v) ^ 0x6A09E667F3BCC908ull;
    uint32_t f[2];
    std::memcpy(&f[0], &p->sigma, 4);
    std::memcpy(&f[1], &p->w_std, 4);
    const uint32_t words[] = {(uint32_t)p->width, (uint32_t)p->height, (uint32_t)k,
                              (uint32_t)p->long_range, (uint32_t)p->max_delay, (uint32_t)a.max_draws,
                              (uint32_t)(p->seed & 0xFFFFFFFFull), (uint32_t)(p->seed >> 32), f[0], f[1]};
    for (uint32_t wv : words) h = (h ^ wv) * 0x100000001B3ull;
    for (int i = 0; i < N; ++i) h = (h ^ accept[i]) * 0x100000001B3ull;
    g->hash = h;
  }
  if ((rc = setup_tables(g, N, S, max_delay, row_ptr.data(), indeg.data(), role, channel))) return fail(rc);
  if ((rc = build_graph_device_cols(g, a.w, a.delay, reinterpret_cast<const int8_t*>(Wb + o_sg))))
    return fail(rc);
  *out = g;
  return SNC_B200_OK;
}
