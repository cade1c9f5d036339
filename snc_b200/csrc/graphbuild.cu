// Device-side build of an uploaded graph's delivery layout.  The host
// validates the graph (SNNGraph::validate rules, src/graph/snn_graph.cpp:30-56),
// computes the per-neuron tables and copies the raw CSR columns; the kernels
// here build what the forward kernels read:
//   edges   [S+2]  packed (ring column | delay << 24, sign[pre] * w), CSR order
//   gedges  [S+2]  the same edges, each row stably regrouped by destination
//                  neuron block (post / BS): within a block the CSR order stays
//   gptr    [N+1], groups [G]  (destination block, first gedge) per row segment
//   ibase   [P+1]  inbox base of every destination block (groups targeting it)
// One warp per row: a counting sort over the P <= kMaxBlocks destination
// blocks in shared memory, made stable by placing the row's edges 32 at a
// time in order with match.any ranks.
#include <algorithm>
#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "internal.h"

namespace sncb {

namespace {

constexpr int kMaxBlocks = 256;       // destination blocks a row can name
constexpr int kRowWarps = 8;          // warps (rows in flight) per CTA

struct BuildArgs {
  int N, BS, P;
  const int* row_ptr;
  const int* post;
  const float* w;
  const int* delays;
  const int8_t* sign;
  const int* col_of;
  int* gcount;     // [N] groups per row
  const int* gptr; // [N+1]
  uint2* edges;
  uint2* gedges;
  int2* groups;
  int* icount;     // [P] groups per destination block
};

// Groups (distinct destination blocks) of every row.
__global__ void __launch_bounds__(32 * kRowWarps) k_group_count(BuildArgs a) {
  __shared__ unsigned char seen[kRowWarps][kMaxBlocks];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  unsigned char* sn = seen[wl];
  for (int i = blockIdx.x * kRowWarps + wl; i < a.N; i += gridDim.x * kRowWarps) {
    for (int b = lane; b < a.P; b += 32) sn[b] = 0;
    __syncwarp();
    const int rs = a.row_ptr[i], re = a.row_ptr[i + 1];
    for (int e = rs + lane; e < re; e += 32) sn[a.post[e] / a.BS] = 1;
    __syncwarp();
    int n = 0;
    for (int b = lane; b < a.P; b += 32) n += sn[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
    if (lane == 0) a.gcount[i] = n;
    __syncwarp();
  }
}

// Packed edges, their stable regroup by destination block, the groups, and
// the groups per destination block.
__global__ void __launch_bounds__(32 * kRowWarps) k_regroup(BuildArgs a) {
  __shared__ int cnt[kRowWarps][kMaxBlocks];  // edges per block, then next free slot
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const unsigned below = (1u << lane) - 1u;
  int* cn = cnt[wl];
  constexpr int kPer = kMaxBlocks / 32;  // blocks per lane in the scans
  for (int i = blockIdx.x * kRowWarps + wl; i < a.N; i += gridDim.x * kRowWarps) {
    const int rs = a.row_ptr[i], re = a.row_ptr[i + 1];
    if (rs == re) continue;  // warp-uniform
    for (int b = lane; b < kMaxBlocks; b += 32) cn[b] = 0;
    __syncwarp();
    const float sg = (float)a.sign[i];
    for (int e = rs + lane; e < re; e += 32) {
      const int p = a.post[e];
      atomicAdd(&cn[p / a.BS], 1);
      const float wv = __fmul_rn(sg, a.w[e]);
      a.edges[e] = make_uint2((uint32_t)a.col_of[p] | ((uint32_t)a.delays[e] << 24), __float_as_uint(wv));
    }
    __syncwarp();
    // exclusive scans over the blocks in ascending order: first slot of each
    // block's segment and the group index of each non-empty block
    int c[kPer], sum = 0, nz = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      c[k] = cn[lane * kPer + k];
      sum += c[k];
      nz += c[k] > 0;
    }
    int xs = sum, xz = nz;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int ys = __shfl_up_sync(0xffffffffu, xs, o), yz = __shfl_up_sync(0xffffffffu, xz, o);
      if (lane >= o) {
        xs += ys;
        xz += yz;
      }
    }
    int off = xs - sum, g = xz - nz;
    const int g0 = a.gptr[i];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int b = lane * kPer + k;
      cn[b] = off;
      if (c[k] > 0) {
        a.groups[g0 + g] = make_int2(b, rs + off);
        atomicAdd(&a.icount[b], 1);
        ++g;
      }
      off += c[k];
    }
    __syncwarp();
    // stable placement, 32 edges at a time in CSR order
    for (int e0 = rs; e0 < re; e0 += 32) {
      const int e = e0 + lane;
      const bool valid = e < re;
      const int b = valid ? a.post[e] / a.BS : -1 - lane;
      const unsigned peers = __match_any_sync(0xffffffffu, b);
      int slot = 0;
      if (valid) slot = cn[b] + __popc(peers & below);
      __syncwarp();
      if (valid) {
        const int p = a.post[e];
        a.gedges[rs + slot] = make_uint2((uint32_t)a.col_of[p] | ((uint32_t)a.delays[e] << 24),
                                         __float_as_uint(__fmul_rn(sg, a.w[e])));
        if ((peers & ~(below | (1u << lane))) == 0) cn[b] = slot + 1;  // the last of its block
      }
      __syncwarp();
    }
  }
}

}  // namespace

// The build proper: g->row_ptr, g->post and g->col_of are on the device;
// w, delays and sign are device columns.
static int build_core(Graph* g, const float* w, const int* delays, const int8_t* sign) {
  const int n = g->N, m = g->S, P = g->P;
  if (P > kMaxBlocks) {
    set_error("more neuron blocks than the device graph build handles");
    return SNC_B200_EUNSUPPORTED;
  }
  DevBuf raw;
  size_t off = 0;
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t o_gc = off;    off = al(off + (size_t)std::max(1, n) * 4);
  const size_t o_ic = off;    off = al(off + (size_t)P * 4);
  const size_t o_scan = off;  off = al(off + scan_scratch_ints(std::max(n, P)) * 4);
  int rc;
  if ((rc = raw.reserve(off))) return rc;
  unsigned char* R = static_cast<unsigned char*>(raw.p);
  if ((rc = dev_alloc(&g->edges, (size_t)m + 2))) return rc;
  if ((rc = dev_alloc(&g->gedges, (size_t)m + 2))) return rc;
  if ((rc = dev_alloc(&g->gptr, (size_t)n + 1))) return rc;
  if ((rc = dev_alloc(&g->ibase, (size_t)P + 1))) return rc;
  SNCB_CUDA(cudaMemset(g->edges + m, 0, 2 * sizeof(uint2)));
  SNCB_CUDA(cudaMemset(g->gedges + m, 0, 2 * sizeof(uint2)));
  SNCB_CUDA(cudaMemset(R + o_ic, 0, (size_t)P * 4));
  BuildArgs a;
  a.N = n;
  a.BS = g->BS;
  a.P = P;
  a.row_ptr = g->row_ptr;
  a.post = g->post;
  a.w = w;
  a.delays = delays;
  a.sign = sign;
  a.col_of = g->col_of;
  a.gcount = reinterpret_cast<int*>(R + o_gc);
  a.gptr = g->gptr;
  a.edges = g->edges;
  a.gedges = g->gedges;
  a.groups = nullptr;
  a.icount = reinterpret_cast<int*>(R + o_ic);
  int* scan = reinterpret_cast<int*>(R + o_scan);
  const unsigned grid = (unsigned)std::max(1, std::min((n + kRowWarps - 1) / kRowWarps, g->sm_count * 16));
  if (n) {
    k_group_count<<<grid, 32 * kRowWarps>>>(a);
    SNCB_CUDA(cudaGetLastError());
  }
  if ((rc = scan_exclusive(a.gcount, g->gptr, n, scan, nullptr))) return rc;
  int G = 0;
  SNCB_CUDA(cudaMemcpy(&G, g->gptr + n, 4, cudaMemcpyDeviceToHost));
  g->G = G;
  if ((rc = dev_alloc(&g->groups, (size_t)std::max(1, G)))) return rc;
  a.groups = g->groups;
  if (n) {
    k_regroup<<<grid, 32 * kRowWarps>>>(a);
    SNCB_CUDA(cudaGetLastError());
  }
  if ((rc = scan_exclusive(a.icount, g->ibase, P, scan, nullptr))) return rc;
  SNCB_CUDA(cudaDeviceSynchronize());
  return SNC_B200_OK;
}

int build_graph_device(const snc_graph_view* v, Graph* g) {
  const int n = g->N, m = g->S;
  DevBuf cols;
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t o_w = 0;
  const size_t o_d = al(o_w + (size_t)std::max(1, m) * 4);
  const size_t o_sign = al(o_d + (size_t)std::max(1, m) * 4);
  int rc;
  if ((rc = cols.reserve(al(o_sign + (size_t)std::max(1, n))))) return rc;
  unsigned char* C = static_cast<unsigned char*>(cols.p);
  if ((rc = dev_upload(&g->row_ptr, v->row_ptr, (size_t)n + 1))) return rc;
  if ((rc = dev_upload(&g->post, v->post_ids, (size_t)m))) return rc;
  if (m) {
    SNCB_CUDA(cudaMemcpy(C + o_w, v->weights, (size_t)m * 4, cudaMemcpyHostToDevice));
    SNCB_CUDA(cudaMemcpy(C + o_d, v->delays, (size_t)m * 4, cudaMemcpyHostToDevice));
  }
  if (n) SNCB_CUDA(cudaMemcpy(C + o_sign, v->sign, (size_t)n, cudaMemcpyHostToDevice));
  return build_core(g, reinterpret_cast<const float*>(C + o_w), reinterpret_cast<const int*>(C + o_d),
                    reinterpret_cast<const int8_t*>(C + o_sign));
}

int build_graph_device_cols(Graph* g, const float* w, const int* delays, const int8_t* sign) {
  return build_core(g, w, delays, sign);
}

}  // namespace sncb
