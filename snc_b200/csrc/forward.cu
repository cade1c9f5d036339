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
//           CTA b owns neuron block b: its v / refr and (SORT, BUCKET) its
//           ring columns live in shared memory for the whole launch, and a
//           bounded software grid barrier separates the two phases of a step.
//   plain   (k_plain_a / k_plain_b) the same phases as one kernel launch
//           each per step with state in global memory, one sample after
//           another: the per-sample path.
//
// Delivery modes (include/snc_b200.h):
//   ATOMIC  the owner of a fired neuron adds its row into the global ring
//           with red.add (one barrier per step).
//   BUCKET  the owner of a fired neuron posts one (first edge, length)
//           descriptor per destination block to that block's inbox; after the
//           barrier each block expands its inbox and accumulates into its
//           shared-memory ring slice with shared atomics.
//   SORT    as BUCKET, but every ring cell receives its contributions in
//           (pre, edge) order -- per-cell lists in a shared hash table, each
//           ordered by gedges index or staging order: the result is
//           bit-identical to the serial CPU backend.
#include <algorithm>
#include <climits>
#include <cstring>
#include <initializer_list>

#include "device_common.cuh"
#include "internal.h"

namespace sncb {

enum { MODE_ATOMIC = 0, MODE_BUCKET = 1, MODE_SORT = 2 };

constexpr int kGThreads = 512;      // plain-path block size; tier G minimum
constexpr int kGThreadsMax = 768;   // tier G block size bound (one CTA per SM)
constexpr int kGChunk = 1024;       // staged events per ordered-apply chunk
constexpr int kGDesc = 1024;        // inbox descriptors handled per chunk
constexpr int kMaxWave = 64;        // samples per lockstep wave

struct FwdArgs {
  // graph
  int N, S, R, ncols, noc, P, BS, G;
  const int* row_ptr;
  const uint2* edges;
  const uint2* gedges;
  const int* gptr;
  const int2* groups;
  const int* col_of;
  const int* out_ch;
  const int* colbase;
  const int* ibase;
  // inputs
  int B;
  const int* order;
  const int* steps;
  const long long* sptr_off;
  const long long* stepbase;
  const int* sched_ptr;
  const int* sched_nid;
  const float* sched_ext;
  const int* sched_blk;  // [total_steps][P+1] or null
  const long long* raster_off;
  // outputs
  int* counts;
  unsigned long long* spikes;
  unsigned long long* events;
  uint32_t* raster;
  float* vfinal;
  int W;
  // grid / plain state
  int Bw;
  float* v;
  int* refr;
  float* ring;
  int* fired;
  int* fired_cnt;
  unsigned long long* inbox;  // [Bw][2][G]
  int* inbox_cnt;             // [Bw][2][P]
  // control
  int* err;
  unsigned* ctl;
  LifP lif;
  // e-prop (tier S only): eligibility [B][S], per-neuron fire counts
  float* elig;
  unsigned long long* fires;
  float gamma, trace_decay;
  int s_table;  // tier S SORT: 1 the whole-chunk cell table, 2 also the cell bitmaps
  int s_lean;   // tier S SORT with the table: the column-list arrays left out
  // deferred eligibility: psi of every ring column and step, [B][ncols][psi_T]
  // (null: eligibility accumulated in the forward into elig)
  float* psi_hist;
  int psi_T;
  // bound of the grid barrier's waits (0: the default) and arrivals that no
  // block makes (a stall injected for failure tests: every wait runs out)
  unsigned long long wait_ns;
  unsigned stall;
  // leaky readout units (ro_on): OUTPUT neurons integrate v = ro_decay * v +
  // drive + ring and never fire; each sample's final potentials go to
  // ro_v [B][n_ro] at their rank, k_readout_logits turns them into logits
  int ro_on;
  float ro_decay;
  const int* ro_rank;
  const int* ro_chan;
  int n_ro;
  float* ro_v;
  float* ro_logits;
  // post-neuron partitions (plain kernels only): first neuron block of the
  // grid, no inbox descriptors posted, delivery by scanning every block's
  // fired list (SORT)
  int blk0;
  int no_post;
  int scan_only;
};

// Shared-memory bytes of the tier-S kernel for this graph.
// Tier S SORT may add a per-cell table for whole chunks: kSTable keys, as
// many list heads and one link per staged event.
constexpr int kSTable = 2048;

// With table == 2 four bitmaps of the ring's cells follow (two alternating
// pairs: seen, hit more than once).
static size_t cell_bitmap_words(int ncols, int R) { return ((size_t)R * ncols + 31) / 32; }

static size_t tier_s_bytes(int N, int ncols, int R, int noc, int mode, bool eprop, int nthr,
                           int table = 0, bool lean = false) {
  size_t words = (size_t)R * ncols + 4 * (size_t)N + (size_t)noc;
  // SORT: row prefix, then the column-list arrays (head, tail, staged column,
  // slot, weight, link) or, lean, the staged weights alone
  if (mode == MODE_SORT)
    words += (size_t)N + 1 + (table && lean ? (size_t)nthr : 2 * (size_t)ncols + 4 * (size_t)nthr);
  if (eprop) words += (size_t)N + ncols;
  if (mode == MODE_SORT && table) words += 2 * (size_t)kSTable + nthr;
  if (mode == MODE_SORT && table == 2) words += 4 * cell_bitmap_words(ncols, R);
  return words * 4 + 16;
}

int tier_s_smem_bytes(const Graph* g, int mode, bool eprop) {
  return (int)tier_s_bytes(g->N, g->ncols, g->R, std::max(1, g->noc), mode, eprop, 1024);
}

// ---------------------------------------------------------------------------
// one LIF neuron (cpu_backend.cpp:129-143, plus reset_mode 1 = subtractive)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int lif_step(const LifP& p, float& v, int& refr, float ext, float rin,
                                        float* vpre = nullptr) {
  if (refr > 0) {
    --refr;
    v = p.reset;
    if (vpre) *vpre = p.reset;
    return 0;
  }
  const float nv = lif_integrate(v, p.decay, ext, rin);
  if (vpre) *vpre = nv;
  if (nv >= p.thr) {
    v = p.reset_mode ? __fsub_rn(nv, p.thr) : p.reset;
    refr = p.refractory;
    return 1;
  }
  v = nv;
  return 0;
}

// A leaky readout unit (shd_model.py:139-140 with the substrate's delivered
// current as its input): v = ro_decay * v + ext + ring, rounded like the LIF
// integration; it never fires or resets.
__device__ __forceinline__ int readout_step(float ro_decay, float& v, float ext, float rin,
                                            float* vpre = nullptr) {
  v = lif_integrate(v, ro_decay, ext, rin);
  if (vpre) *vpre = v;
  return 0;
}

// logits[b][c] = sum over the readout units of channel c, ascending id, of
// their final potential / T_b (shd_model.py:147 averages the readout over
// the steps).  One block per sample, a thread per channel.
__global__ void k_readout_logits(const float* __restrict__ ro_v, const int* __restrict__ ro_chan,
                                 int n_ro, const int* __restrict__ steps, int noc,
                                 float* __restrict__ logits) {
  const int b = blockIdx.x;
  const float T = (float)max(1, steps[b]);
  for (int c = threadIdx.x; c < noc; c += blockDim.x) {
    float acc = 0.f;
    for (int r = 0; r < n_ro; ++r)
      if (ro_chan[r] == c) acc = __fadd_rn(acc, __fdiv_rn(ro_v[(size_t)b * n_ro + r], T));
    logits[(size_t)b * noc + c] = acc;
  }
}

// Ring slot of a delivery made at step slot `s0` with delay d (1 <= d < R).
__device__ __forceinline__ int ring_slot(int s0, int d, int R) {
  const int s = s0 + d;
  return s >= R ? s - R : s;
}

template <bool GLOBAL_RING>
__device__ __forceinline__ void apply_one(float* ring, int ring_stride, int col0, int c, int slot,
                                          float w) {
  float* cell = ring + (size_t)slot * ring_stride + col0 + c;
  if (GLOBAL_RING) {
    __stcg(cell, __fadd_rn(__ldcg(cell), w));
  } else {
    *cell = __fadd_rn(*cell, w);
  }
}

// Chunks up to kCountMax events take the per-cell apply; above it tier S
// uses unordered lists that every column sorts on its own, while tier G links
// in order (its post blocks own hub columns whose per-step event count can be
// large).
constexpr int kCountMax = 256;
constexpr int kRegSort = 16;
constexpr int kFirstFlag = 1 << 30;  // marks a group's first event of its column in st_col

// Ordered apply of a small chunk (ce <= kCountMax <= blockDim.x, so thread q
// owns staged event q) through its ring cells.  A hash table of kCellTable
// keys (column, slot) -- zeroed by the caller before staging -- holds one
// unordered list per cell (atomicExch heads, one link per event).  The first
// arrival at a cell owns it: alone there, it applies its event; otherwise it
// collects the cell's list (kCellSort entries in registers, sorted; longer
// lists by repeated minimum selection) and applies it in order.  A step's
// events spread over many more cells than columns -- a column's events carry
// different delays -- so lists are short and no thread walks a hub column's
// whole chain.
constexpr int kCellTable = 2 * kCountMax;  // keys, then list heads (q + 1, 0 = empty)
constexpr int kCellSort = 8;
static_assert(2 * kCellTable <= kGChunk, "the table lives in st_next");
static_assert(kCellTable + kCountMax <= kGChunk, "the links live in st_col beyond the chunk");

// Table sizes (keys; as many list heads follow) and their hash bits.
template <int TS>
constexpr int kTabBits = TS == 2048 ? 11 : (TS == 1024 ? 10 : 9);

// Enters staged event q of cell (c, sl) into a table of TS keys (at most TS / 2
// distinct cells); returns its entry.
template <int TS>
__device__ __forceinline__ unsigned cell_insert(int* tab, int* link, int q, int c, int sl, bool* first) {
  static_assert(TS == 512 || TS == 1024 || TS == 2048, "table size");
  unsigned* key = reinterpret_cast<unsigned*>(tab);
  const unsigned k = (unsigned)c * 256u + (unsigned)sl + 1u;  // slot < 256, 0 = empty
  unsigned h = (k * 2654435761u) >> (32 - kTabBits<TS>);
  // at most TS / 2 keys: a free or equal entry is always found
  for (int probe = 0; probe < TS; ++probe) {
    const unsigned old = atomicCAS(&key[h], 0u, k);
    if (old == 0u || old == k) break;
    h = (h + 1u) & (TS - 1);
  }
  const int prev = atomicExch(&tab[TS + h], q + 1);
  link[q] = prev;
  *first = prev == 0;
  return h;
}

// The owner's part (after a barrier that follows every cell_insert): apply
// the cell's events in increasing order -- their staging index, or with
// KEYED their order key okey[x] (unique per event) -- then x.
template <bool GLOBAL_RING, bool KEYED>
__device__ __forceinline__ void cell_apply_list(int top, const int* link, const int* okey,
                                                const float* st_w, int q, int c, int sl, float* ring,
                                                int ring_stride, int col0) {
  if (top == q + 1) {
    apply_one<GLOBAL_RING>(ring, ring_stride, col0, c, sl, st_w[q]);
    return;
  }
  auto ord = [&](int x) -> long long {
    return KEYED ? ((long long)okey[x] << 10) | x : (long long)x;  // x < kGChunk = 1024
  };
  long long r[kCellSort];
#pragma unroll
  for (int i = 0; i < kCellSort; ++i) r[i] = LLONG_MAX;
  int p = top;
#pragma unroll
  for (int i = 0; i < kCellSort; ++i) {
    if (p != 0) {
      // insert into the sorted r (its largest entry is free)
      r[kCellSort - 1] = ord(p - 1);
#pragma unroll
      for (int m = kCellSort - 1; m > 0; --m) {
        const long long lo = min(r[m - 1], r[m]), hi = max(r[m - 1], r[m]);
        r[m - 1] = lo;
        r[m] = hi;
      }
      p = link[p - 1];
    }
  }
  if (p == 0) {
#pragma unroll
    for (int i = 0; i < kCellSort; ++i)
      if (r[i] != LLONG_MAX) apply_one<GLOBAL_RING>(ring, ring_stride, col0, c, sl, st_w[(int)(r[i] & 1023)]);
    return;
  }
  long long last = -1;
  for (;;) {
    long long best = LLONG_MAX;
    for (int x = top; x != 0; x = link[x - 1]) {
      const long long o = ord(x - 1);
      if (o > last && o < best) best = o;
    }
    if (best == LLONG_MAX) break;
    apply_one<GLOBAL_RING>(ring, ring_stride, col0, c, sl, st_w[(int)(best & 1023)]);
    last = best;
  }
}

template <bool GLOBAL_RING, bool KEYED, int TS>
__device__ __forceinline__ void cell_apply(const int* tab, const int* link, const int* okey,
                                           const float* st_w, unsigned h, int q, int c, int sl,
                                           float* ring, int ring_stride, int col0) {
  cell_apply_list<GLOBAL_RING, KEYED>(tab[TS + h], link, okey, st_w, q, c, sl, ring, ring_stride, col0);
}

template <bool GLOBAL_RING>
__device__ void apply_cells(int ce, int* tab, int* st_col, const int* st_slot, const float* st_w,
                            float* ring, int ring_stride, int col0) {
  int* link = st_col + kCellTable;
  const int q = threadIdx.x;
  int c = 0, sl = 0;
  unsigned h = 0;
  bool first = false;
  if (q < ce) {
    c = st_col[q];
    sl = st_slot[q];
    h = cell_insert<kCellTable>(tab, link, q, c, sl, &first);
  }
  __syncthreads();
  if (first)
    cell_apply<GLOBAL_RING, false, kCellTable>(tab, link, nullptr, st_w, h, q, c, sl, ring, ring_stride,
                                               col0);
  __syncthreads();
}

// Ordered apply of one chunk of staged events.  Staging index q is the
// (pre, edge) order of the CPU backend.  The events were staged with their
// block-local column st_col[q] (head / tail of every local column = -1).
// Every ring cell must receive its contributions in increasing q.
//  - chunks up to kCountMax events: apply_cells (above);
//  - chunks up to serial_max: every warp links the events of its 32-event groups
//    (match.any: successor within the group, first event of each column
//    flagged), then one warp joins the groups in staging order through the
//    column tails -- one shared-memory round trip per group; one thread per
//    column then replays its list: O(events), no sorting, and hub columns
//    with many events in one step stay linear.
//  - large chunks: lists are built in parallel with atomicExch (arbitrary
//    order); each column thread loads up to kRegSort list entries into
//    registers, sorts them there and replays them; longer lists fall back to
//    repeated minimum selection.
template <bool GLOBAL_RING>
__device__ void apply_ordered(int ce, int* head, int* tail, int ncols_local, int* st_col,
                              const int* st_slot, const float* st_w, int* st_next, float* ring,
                              int ring_stride, int col0, int serial_max) {
  __syncthreads();
  if (ce <= kCountMax && ce <= (int)blockDim.x) {
    apply_cells<GLOBAL_RING>(ce, st_next, st_col, st_slot, st_w, ring, ring_stride, col0);
    return;
  }
  if (ce > serial_max) {
    for (int q = threadIdx.x; q < ce; q += blockDim.x) st_next[q] = atomicExch(&head[st_col[q]], q);
    __syncthreads();
    for (int c = threadIdx.x; c < ncols_local; c += blockDim.x) {
      const int h = head[c];
      if (h < 0) continue;
      head[c] = -1;
      int r[kRegSort];
#pragma unroll
      for (int i = 0; i < kRegSort; ++i) r[i] = INT_MAX;
      int p = h;
#pragma unroll
      for (int i = 0; i < kRegSort; ++i) {
        if (p >= 0) {
          // insert p into the sorted r[0..kRegSort) (largest slot is free)
          r[kRegSort - 1] = p;
#pragma unroll
          for (int k = kRegSort - 1; k > 0; --k) {
            const int lo = min(r[k - 1], r[k]), hi = max(r[k - 1], r[k]);
            r[k - 1] = lo;
            r[k] = hi;
          }
          p = st_next[p];
        }
      }
      if (p < 0) {
#pragma unroll
        for (int i = 0; i < kRegSort; ++i)
          if (r[i] != INT_MAX) apply_one<GLOBAL_RING>(ring, ring_stride, col0, c, st_slot[r[i]], st_w[r[i]]);
      } else {
        int last = -1;
        for (;;) {
          int best = INT_MAX;
          for (int x = h; x >= 0; x = st_next[x])
            if (x > last && x < best) best = x;
          if (best == INT_MAX) break;
          apply_one<GLOBAL_RING>(ring, ring_stride, col0, c, st_slot[best], st_w[best]);
          last = best;
        }
      }
    }
    __syncthreads();
    return;
  }
  {
    // 1. every warp links its own 32-event groups (match.any): successor
    //    within the group or -1, first event of each column flagged
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    for (int g0 = warp * 32; g0 < ce; g0 += nwarps * 32) {
      const int q = g0 + lane;
      const bool valid = q < ce;
      const int c = valid ? st_col[q] : -1 - lane;
      const unsigned peers = __match_any_sync(0xffffffffu, c);
      const unsigned higher = peers & ~below & ~(1u << lane);
      if (valid) {
        st_next[q] = higher ? g0 + __ffs(higher) - 1 : -1;
        if (!(peers & below)) st_col[q] = c | kFirstFlag;
      }
    }
  }
  __syncthreads();
  // 2. one warp joins the groups in order through the column tails
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    for (int g0 = 0; g0 < ce; g0 += 32) {
      const int q = g0 + lane;
      int c = 0, t = -1;
      bool first = false, last = false;
      if (q < ce) {
        const int cf = st_col[q];
        first = (cf & kFirstFlag) != 0;
        c = cf & ~kFirstFlag;
        last = st_next[q] < 0;
        if (first) t = tail[c];
      }
      __syncwarp();
      if (first) {
        if (t >= 0) st_next[t] = q;
        else head[c] = q;
      }
      if (last) tail[c] = q;
      __syncwarp();
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < ncols_local; c += blockDim.x) {
    int p = head[c];
    if (p < 0) continue;
    head[c] = -1;
    tail[c] = -1;
    for (; p >= 0; p = st_next[p]) apply_one<GLOBAL_RING>(ring, ring_stride, col0, c, st_slot[p], st_w[p]);
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// tier S: one CTA per sample, state in shared memory
// ---------------------------------------------------------------------------
template <int MODE, bool EP>
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
  // the column-list apply's arrays (SORT without the cell table); the lean
  // table layout of the e-prop kernel keeps only the staged weights of them
  // (the forward keeps the fixed layout, measured faster)
  const bool lists = MODE == MODE_SORT && !(EP && a.s_lean);
  int* head = pref + (N + 1);
  int* tail = head + (lists ? nc : 0);
  int* st_col = tail + (lists ? nc : 0);
  int* st_slot = st_col + (lists ? CH : 0);
  float* st_w = reinterpret_cast<float*>(st_slot + (lists ? CH : 0));
  int* st_next = reinterpret_cast<int*>(st_w + CH);
  // e-prop: pre-synaptic trace per neuron, surrogate psi per ring column
  float* tr = MODE == MODE_SORT ? reinterpret_cast<float*>(st_next + (lists ? CH : 0))
                                : reinterpret_cast<float*>(counts + noc);
  float* psi = tr + N;
  // SORT with a.s_table: the per-cell table for whole chunks (kSTable keys,
  // kSTable list heads, CH links)
  int* ctab = reinterpret_cast<int*>(EP ? psi + nc : tr);
  // s_table 2: bitmaps of the ring's cells after the table's links, two
  // pairs (seen, more than once) used by alternate chunks
  const int nbw = (int)(((size_t)R * nc + 31) / 32);
  unsigned* cbits = reinterpret_cast<unsigned*>(ctab + 2 * kSTable + CH);
  if (MODE == MODE_SORT && a.s_table) {
    for (int i = tid; i < 2 * kSTable; i += nthr) ctab[i] = 0;  // ordered by the loop's first barrier
    if (a.s_table == 2)
      for (int i = tid; i < 4 * nbw; i += nthr) cbits[i] = 0u;
  }

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
      if (EP) tr[i] = 0.f;
    }
    for (int i = tid; i < noc; i += nthr) counts[i] = 0;
    if (lists)
      for (int i = tid; i < nc; i += nthr) {
        head[i] = -1;
        tail[i] = -1;
      }
    __syncthreads();
    const int* sp = a.sched_ptr + a.sptr_off[b];
    uint32_t* rast = a.raster ? a.raster + a.raster_off[b] : nullptr;
    long long my_spikes = 0, my_events = 0;
    int s0 = 0;
    __shared__ int s_bc[2][32];  // ballot_compact_1 buffers, alternated
    int bcp = 0;
    // the drive of step t: thread i holds entry i of the step's schedule in
    // registers, loaded a step ahead (entries beyond blockDim.x are read in
    // the step itself); a step's entries name distinct neurons
    int pf_lo = T > 0 ? sp[0] : 0, pf_hi = T > 0 ? sp[1] : 0, pf_nid = -1;
    float pf_ext = 0.f;
    if (pf_lo + tid < pf_hi) {
      pf_nid = a.sched_nid[pf_lo + tid];
      pf_ext = a.sched_ext[pf_lo + tid];
    }
    for (int t = 0; t < T; ++t) {
      float* slot = ring + (size_t)s0 * nc;
      if (pf_nid >= 0) ext[pf_nid] = pf_ext;
      for (int k = pf_lo + nthr + tid; k < pf_hi; k += nthr) ext[a.sched_nid[k]] = a.sched_ext[k];
      __syncthreads();
      pf_nid = -1;
      if (t + 1 < T) {
        pf_lo = sp[t + 1];
        pf_hi = sp[t + 2];
        if (pf_lo + tid < pf_hi) {
          pf_nid = a.sched_nid[pf_lo + tid];
          pf_ext = a.sched_ext[pf_lo + tid];
        }
      }
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
          float vpre;
          const int oc = a.out_ch[j];
          f = a.ro_on && oc >= 0 ? readout_step(a.ro_decay, vv, e, rin, &vpre)
                                 : lif_step(a.lif, vv, rr, e, rin, &vpre);
          v[j] = vv;
          refr[j] = rr;
          if (EP) {
            // cuda_trainer.cu:93-95: triangular surrogate and pre trace
            const float thr = a.lif.thr;
            const float dd = __fdiv_rn(fabsf(__fsub_rn(vpre, thr)), thr > 0.f ? thr : 1.f);
            if (c >= 0) {
              const float ps = dd < 1.f ? __fmul_rn(a.gamma, __fsub_rn(1.f, dd)) : 0.f;
              psi[c] = ps;
              if (a.psi_hist) a.psi_hist[((size_t)b * a.psi_T + t) * nc + c] = ps;
            }
            tr[j] = __fadd_rn(__fmul_rn(a.trace_decay, tr[j]),
                              __fmul_rn(__fsub_rn(1.f, a.trace_decay), f ? 1.f : 0.f));
            if (f && a.fires) atomicAdd(&a.fires[j], 1ull);
          }
          if (f) {
            ++my_spikes;
            my_events += a.row_ptr[j + 1] - a.row_ptr[j];
            if (oc >= 0) atomicAdd(&counts[oc], 1);
          }
        }
        int tot;
        unsigned m;
        const int pos = ballot_compact_1(f, s_bc[bcp], &tot, &m);
        bcp ^= 1;
        if (rast && lane == 0 && base + warp * 32 < N)
          rast[(size_t)t * a.W + ((base + warp * 32) >> 5)] = m;
        if (f) fired[nf + pos] = j;
        nf += tot;
      }
      __syncthreads();
      if (EP && a.elig) {
        // cuda_trainer.cu:105-112: E[b,s] += psi[post] * tr[pre]; rows whose
        // trace is exactly zero add +0 and are skipped (trainer.cpp:243-244)
        float* Eb = a.elig + (size_t)b * a.S;
        for (int i = warp; i < N; i += nwarps) {
          const float tri = tr[i];
          if (tri == 0.f) continue;
          const int rs = a.row_ptr[i], re = a.row_ptr[i + 1];
          for (int e = rs + lane; e < re; e += 32) {
            const uint2 ed = a.edges[e];
            Eb[e] = __fadd_rn(Eb[e], __fmul_rn(psi[edge_col(ed)], tri));
          }
        }
      }
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
          int len = 0;
          if (k < nf) {
            const int rs = a.row_ptr[fired[k]];
            len = a.row_ptr[fired[k] + 1] - rs;
            fired[k] = rs;  // row start from here on (the list is not used again this step)
          }
          int tot;
          const int ex = block_exclusive_scan(len, scratch, &tot);
          if (k < nf) pref[k] = base + ex;
          base += tot;
        }
        __syncthreads();
        const int E = base;
        if (a.s_table) {
          // per-cell apply of whole chunks (CH = blockDim.x: thread q stages
          // event q of the chunk and enters it in its cell's list; staging
          // order is the (pre, edge) order)
          // the table is all zero between chunks: every cell's owner clears
          // its entry once it has applied the cell (nobody else reads it)
          // thread q's edge of the next chunk is requested before this
          // chunk's cells are applied, so the load overlaps the apply
          const int q = tid;
          auto edge_of = [&](int e) {
            const int k = upper_index(pref, nf, e);
            return a.edges[fired[k] + (e - pref[k])];
          };
          uint2 ed_next = q < E ? edge_of(q) : make_uint2(0u, 0u);
          if (a.s_table == 2) {
            // Only cells hit more than once in a chunk need the table: every
            // event marks its cell in the chunk's bitmap pair (a second mark
            // sets the "more than once" bit); after one barrier a cell hit
            // once takes its event directly and the others go through the
            // table, applied after a second barrier.  Each event clears its
            // cell's seen word once it has read it (the events of shared cells
            // also their "more" word); the pairs alternate, so a
            // chunk's marks never meet the previous chunk's clears.  (A
            // shared-memory atomic add for the single events and bulk clears
            // of the idle pair both measured slower.)
            int pair = 0;
            for (int e0 = 0; e0 < E; e0 += CH, pair ^= 1) {
              const int ce = min(CH, E - e0);
              const uint2 ed = ed_next;
              unsigned* seen = cbits + (size_t)pair * 2 * nbw;
              unsigned* more = seen + nbw;
              int c = 0, sl = 0, bw = 0;
              unsigned bm = 0, h = 0;
              float w = 0.f;
              if (q < ce) {
                sl = ring_slot(s0, edge_delay(ed), R);
                c = edge_col(ed);
                w = edge_w(ed);
                const int bit = sl * nc + c;
                bw = bit >> 5;
                bm = 1u << (bit & 31);
                if (atomicOr(&seen[bw], bm) & bm) atomicOr(&more[bw], bm);
              }
              // the next chunk's edge: its row search overlaps the marks and
              // the barrier, its load the apply
              if (e0 + CH + q < E) ed_next = edge_of(e0 + CH + q);
              __syncthreads();
              bool first = false, shared_cell = false;
              if (q < ce) {
                shared_cell = (more[bw] & bm) != 0u;
                if (!shared_cell) {
                  apply_one<false>(ring, nc, 0, c, sl, w);
                } else {
                  st_w[q] = w;
                  h = cell_insert<kSTable>(ctab, ctab + 2 * kSTable, q, c, sl, &first);
                }
              }
              __syncthreads();
              if (q < ce) {
                seen[bw] = 0u;
                if (shared_cell) more[bw] = 0u;  // other words of `more` stayed zero
              }
              if (first) {
                cell_apply<false, false, kSTable>(ctab, ctab + 2 * kSTable, nullptr, st_w, h, q, c, sl, ring,
                                                  nc, 0);
                ctab[h] = 0;
                ctab[kSTable + h] = 0;
              }
            }
            // the step's closing barrier orders the last chunk's apply
          } else
          for (int e0 = 0; e0 < E; e0 += CH) {
            const int ce = min(CH, E - e0);
            const uint2 ed = ed_next;
            int c = 0, sl = 0;
            unsigned h = 0;
            bool first = false;
            if (q < ce) {
              sl = ring_slot(s0, edge_delay(ed), R);
              c = edge_col(ed);
              st_w[q] = edge_w(ed);
              h = cell_insert<kSTable>(ctab, ctab + 2 * kSTable, q, c, sl, &first);
            }
            __syncthreads();
            if (e0 + CH + q < E) ed_next = edge_of(e0 + CH + q);
            if (first) {
              cell_apply<false, false, kSTable>(ctab, ctab + 2 * kSTable, nullptr, st_w, h, q, c, sl, ring,
                                                nc, 0);
              ctab[h] = 0;
              ctab[kSTable + h] = 0;
            }
            __syncthreads();
          }
        } else
        for (int e0 = 0; e0 < E; e0 += CH) {
          const int ce = min(CH, E - e0);
          for (int qq = tid; qq < ce; qq += nthr) {
            const int e = e0 + qq;
            const int k = upper_index(pref, nf, e);
            const uint2 ed = a.edges[fired[k] + (e - pref[k])];
            st_slot[qq] = ring_slot(s0, edge_delay(ed), R);
            st_w[qq] = edge_w(ed);
            st_col[qq] = edge_col(ed);
          }
          if (ce <= kCountMax)  // apply_cells' table (st_next has CH = 1024 entries)
            for (int i = tid; i < 2 * kCellTable; i += nthr) st_next[i] = 0;
          __syncthreads();
          apply_ordered<false>(ce, head, tail, nc, st_col, st_slot, st_w, st_next, ring, nc, 0,
                               kCountMax);
          __syncthreads();
        }
      }
      __syncthreads();
      s0 = (s0 + 1 == R) ? 0 : s0 + 1;
    }
    for (int i = tid; i < noc; i += nthr) a.counts[(size_t)b * noc + i] = counts[i];
    if (a.vfinal)
      for (int i = tid; i < N; i += nthr) a.vfinal[(size_t)b * N + i] = v[i];
    if (a.ro_on)
      for (int i = tid; i < N; i += nthr)
        if (a.ro_rank[i] >= 0) a.ro_v[(size_t)b * a.n_ro + a.ro_rank[i]] = v[i];
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
// Shared memory of a tier-G / plain CTA.  PERSIST (tier G) keeps v / refr
// of its wave slots and cached row / group pointers of its neurons; RSM keeps
// the ring columns of its block ([Bw][R][BS]) for SORT / BUCKET.
struct GSmem {
  float* v;                  // PERSIST [Bw][BS]
  int* refr;                 // PERSIST [Bw][BS]
  int* col;                  // PERSIST [BS]   ring column (global index) or -1
  int* rp;                   // PERSIST [BS+1] row_ptr of the block's neurons
  int* gp;                   // PERSIST [BS+1] gptr of the block's neurons
  int* och;                  // PERSIST [BS]   output channel or -1
  float* ring;               // RSM [Bw][R][BS]
  float* ext;                // [Bw][BS] (one drive buffer per wave slot)
  int* fired;                // [BS]
  int* pa;                   // [P+1]
  int* ib;                   // [P+1] inbox base of every destination block
  int* head;                 // [BS]
  int* tail;                 // [BS]
  unsigned long long* desc;  // [kGDesc]
  unsigned long long* dsort; // [kGDesc]
  int* seg_p;                // [kGDesc]
  int* st_col;               // [kGChunk]
  int* st_slot;              // [kGChunk]
  float* st_w;               // [kGChunk]
  int* st_next;              // [kGChunk]
};

static size_t g_smem_bytes(int BS, int P, int R, int Bw, bool persist, bool rsm) {
  size_t b = 0;
  b += 8 * (size_t)kGDesc * 2;                         // desc, dsort
  b += 4 * ((size_t)BS * 3 + (size_t)Bw * BS + 2 * (P + 1) + kGDesc + 4 * (size_t)kGChunk);
  if (persist) b += 4 * ((size_t)Bw * BS * 2 + 2 * (size_t)BS + 2 * ((size_t)BS + 1));
  if (rsm) b += 4 * (size_t)Bw * R * BS;
  return b + 64;
}

__device__ __forceinline__ GSmem carve_g(unsigned char* raw, int BS, int P, int R, int Bw,
                                         bool persist, bool rsm) {
  GSmem s{};
  s.desc = reinterpret_cast<unsigned long long*>(raw);
  s.dsort = s.desc + kGDesc;
  float* f = reinterpret_cast<float*>(s.dsort + kGDesc);
  s.ext = f;
  s.fired = reinterpret_cast<int*>(s.ext + (size_t)Bw * BS);
  s.head = s.fired + BS;
  s.tail = s.head + BS;
  s.pa = s.tail + BS;
  s.ib = s.pa + (P + 1);
  s.seg_p = s.ib + (P + 1);
  s.st_col = s.seg_p + kGDesc;
  s.st_slot = s.st_col + kGChunk;
  s.st_w = reinterpret_cast<float*>(s.st_slot + kGChunk);
  s.st_next = reinterpret_cast<int*>(s.st_w + kGChunk);
  int* p = s.st_next + kGChunk;
  if (persist) {
    s.v = reinterpret_cast<float*>(p);
    s.refr = reinterpret_cast<int*>(s.v + (size_t)Bw * BS);
    s.col = s.refr + (size_t)Bw * BS;
    s.rp = s.col + BS;
    s.gp = s.rp + (BS + 1);
    s.och = s.gp + (BS + 1);
    p = s.och + BS;
  }
  if (rsm) s.ring = reinterpret_cast<float*>(p);
  return s;
}

// Scatter block b's share of step t's injection schedule into ext (dense
// over the block's neurons, zero elsewhere; integration re-zeroes what it
// reads).  Only reads the read-only inputs, so it may run between the arrival
// at and the wait on a grid barrier.
__device__ void load_ext(const FwdArgs& a, float* ext, int sample, long long gstep, int t, int b) {
  __shared__ int s_rng[2];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int lo = b * a.BS, hi = min(a.N, lo + a.BS);
  int k0, k1;
  if (a.sched_blk) {
    const int* sb = a.sched_blk + gstep * (a.P + 1) + b;
    k0 = sb[0];
    k1 = sb[1];
  } else {
    if (tid == 0) {
      const int* sp = a.sched_ptr + a.sptr_off[sample];
      const int q0 = sp[t], q1 = sp[t + 1];
      s_rng[0] = lower_bound_i(a.sched_nid, q0, q1, lo);
      s_rng[1] = lower_bound_i(a.sched_nid, q0, q1, hi);
    }
    __syncthreads();
    k0 = s_rng[0];
    k1 = s_rng[1];
    __syncthreads();
  }
  for (int q = k0 + tid; q < k1; q += nthr) ext[a.sched_nid[q] - lo] = a.sched_ext[q];
}

// Phase A: drive, integrate / fire the block's neurons, publish the ascending
// fired list, then deliver (ATOMIC) or post inbox descriptors (BUCKET, SORT).
// ext_ready: the drive of this step is already in the slot's ext buffer.
// acc: per-slot spike / event totals in shared memory ([0, kMaxWave) spikes,
// [kMaxWave, 2 kMaxWave) events) that the caller adds to the sample's totals
// once per wave; null: added to the global totals every step.
// EPR: record e-prop's psi and fire counts (the all-SM e-prop forward only).
template <int MODE, bool PERSIST, bool RSM, bool EPR = false>
__device__ void phase_a(const FwdArgs& a, const GSmem& sm, int* scratch, unsigned long long* acc,
                        int k, int sample, long long gstep, int t, int b, int cb0, bool ext_ready) {
  const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = nthr >> 5;
  const int lo = b * a.BS, hi = min(a.N, lo + a.BS);
  const int R = a.R, nc = a.ncols, N = a.N, BS = a.BS, P = a.P;
  const int par = t & 1;
  const int s0 = t % R;
  float* ext = sm.ext + (PERSIST ? (size_t)k * BS : 0);
  if (!ext_ready) load_ext(a, ext, sample, gstep, t, b);
  __syncthreads();
  uint32_t* rast = a.raster ? a.raster + a.raster_off[sample] + (size_t)t * a.W : nullptr;
  int nf = 0;
  long long my_events = 0;
  __shared__ int s_bc[2][32];  // ballot_compact_1 buffers, alternated
  int bcp = 0;
  for (int base = lo; base < hi; base += nthr) {
    const int j = base + tid, jj = j - lo;
    int f = 0;
    if (j < hi) {
      float vv = PERSIST ? sm.v[k * BS + jj] : a.v[(size_t)k * N + j];
      int rr = PERSIST ? sm.refr[k * BS + jj] : a.refr[(size_t)k * N + j];
      const int c = PERSIST ? sm.col[jj] : a.col_of[j];
      float rin = 0.f;
      if (c >= 0) {
        if (RSM) {
          float* cell = sm.ring + ((size_t)k * R + s0) * BS + (c - cb0);
          rin = *cell;
          *cell = 0.f;
        } else {
          float* cell = a.ring + ((size_t)k * R + s0) * nc + c;
          rin = __ldcg(cell);
          __stcg(cell, 0.f);
        }
      }
      const float e = ext[jj];
      ext[jj] = 0.f;
      float vpre;
      const int oc = PERSIST ? sm.och[jj] : a.out_ch[j];
      f = a.ro_on && oc >= 0 ? readout_step(a.ro_decay, vv, e, rin, EPR ? &vpre : nullptr)
                             : lif_step(a.lif, vv, rr, e, rin, EPR ? &vpre : nullptr);
      if (EPR && c >= 0) {
        // e-prop (cuda_trainer.cu:93-94): the triangular surrogate of this
        // column and step, for the deferred eligibility
        const float thr = a.lif.thr;
        const float dd = __fdiv_rn(fabsf(__fsub_rn(vpre, thr)), thr > 0.f ? thr : 1.f);
        a.psi_hist[((size_t)sample * a.psi_T + t) * nc + c] =
            dd < 1.f ? __fmul_rn(a.gamma, __fsub_rn(1.f, dd)) : 0.f;
      }
      if (PERSIST) {
        sm.v[k * BS + jj] = vv;
        sm.refr[k * BS + jj] = rr;
      } else {
        a.v[(size_t)k * N + j] = vv;
        a.refr[(size_t)k * N + j] = rr;
      }
      if (f) {
        my_events += PERSIST ? sm.rp[jj + 1] - sm.rp[jj] : a.row_ptr[j + 1] - a.row_ptr[j];
        if (MODE != MODE_ATOMIC && PERSIST) {
          // the row's groups are read again when this step's descriptors are
          // posted: start bringing them into L1 while the fired list is built
          const int2* gr = a.groups + sm.gp[jj];
          asm volatile("prefetch.global.L1 [%0];" ::"l"(gr));
          asm volatile("prefetch.global.L1 [%0];" ::"l"(a.groups + max(sm.gp[jj], sm.gp[jj + 1] - 1)));
        }
        if (oc >= 0) atomicAdd(&a.counts[(size_t)sample * a.noc + oc], 1);
        if (EPR && a.fires) atomicAdd(&a.fires[j], 1ull);
      }
    }
    int tot;
    unsigned m;
    const int pos = ballot_compact_1(f, s_bc[bcp], &tot, &m);
    bcp ^= 1;
    if (rast && lane == 0 && base + warp * 32 < hi) rast[(base + warp * 32) >> 5] = m;
    if (f) sm.fired[nf + pos] = j;
    nf += tot;
  }
  __syncthreads();
  if (MODE == MODE_SORT) {
    // the ascending fired list, for phase_b_scan (SORT steps whose inbox
    // overflows); the other modes never read it
    int* fo = a.fired + ((size_t)k * 2 + par) * N + lo;
    for (int i = tid; i < nf; i += nthr) __stcg(&fo[i], sm.fired[i]);
  }
  {
    unsigned long long wev = (unsigned long long)my_events;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wev += __shfl_down_sync(0xffffffffu, wev, o);
    if (lane == 0 && wev) atomicAdd(acc ? &acc[kMaxWave + k] : &a.events[sample], wev);
  }
  if (tid == 0) {
    if (MODE == MODE_SORT) __stcg(&a.fired_cnt[((size_t)k * 2 + par) * P + b], nf);
    if (nf) atomicAdd(acc ? &acc[k] : &a.spikes[sample], (unsigned long long)nf);
  }
  if (MODE == MODE_ATOMIC) {
    float* ringk = a.ring + (size_t)k * R * nc;
    for (int q = warp; q < nf; q += nwarps) {
      const int j = sm.fired[q];
      const int rs = PERSIST ? sm.rp[j - lo] : a.row_ptr[j];
      const int re = PERSIST ? sm.rp[j - lo + 1] : a.row_ptr[j + 1];
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
  } else if (!a.no_post) {
    // one descriptor (first edge, length) per destination block of each
    // fired row; a warp posts the groups of one row in parallel
    int* cnt = a.inbox_cnt + ((size_t)k * 2 + par) * P;
    unsigned long long* box = a.inbox + ((size_t)k * 2 + par) * a.G;
    for (int q = warp; q < nf; q += nwarps) {
      const int j = sm.fired[q];
      const int g0 = PERSIST ? sm.gp[j - lo] : a.gptr[j];
      const int g1 = PERSIST ? sm.gp[j - lo + 1] : a.gptr[j + 1];
      const int re = PERSIST ? sm.rp[j - lo + 1] : a.row_ptr[j + 1];
      for (int g = g0 + lane; g < g1; g += 32) {
        const int2 gr = a.groups[g];
        const int ge = (g + 1 < g1) ? a.groups[g + 1].y : re;
        const int pos = atomicAdd(&cnt[gr.x], 1);
        __stcg(&box[sm.ib[gr.x] + pos],
               ((unsigned long long)(unsigned)gr.y << 32) | (unsigned)(ge - gr.y));
      }
    }
  }
  // no closing barrier: every caller's next step starts with one (the next
  // slot's phase A, grid_arrive, or the end of the launch)
}

// Ring view of one wave slot for the post-owner phase: shared-memory slice
// (local columns, stride BS) or the global ring (global columns, stride ncols).
template <bool RSM>
__device__ __forceinline__ float* ring_base(const FwdArgs& a, const GSmem& sm, int k) {
  return RSM ? sm.ring + (size_t)k * a.R * a.BS : a.ring + (size_t)k * a.R * a.ncols;
}

// SORT fallback when a block's inbox exceeds kGDesc descriptors: walk every
// block's ascending fired list (ascending pre order overall) and stage the
// segments that target this block in that order.
template <bool RSM>
__device__ void phase_b_scan(const FwdArgs& a, const GSmem& sm, int* scratch, int k, int t, int b,
                             int cb0, int cb1) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int R = a.R, P = a.P;
  const int par = t & 1;
  const int s0 = t % R;
  const int* cntk = a.fired_cnt + ((size_t)k * 2 + par) * P;
  const int* fk = a.fired + ((size_t)k * 2 + par) * a.N;
  float* rb = ring_base<RSM>(a, sm, k);
  const int stride = RSM ? a.BS : a.ncols;
  const int col0 = RSM ? 0 : cb0;
  int F;
  {
    const int cnt = tid < P ? __ldcg(&cntk[tid]) : 0;
    const int ex = block_exclusive_scan(cnt, scratch, &F);
    if (tid < P) sm.pa[tid] = ex;
    __syncthreads();
  }
  int* seg_s = reinterpret_cast<int*>(sm.desc);
  int* seg_l = reinterpret_cast<int*>(sm.dsort);
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
      seg_s[pos] = gs;
      seg_l[pos] = gl;
    }
    __syncthreads();
    int E;
    {
      const int len = tid < nseg ? seg_l[tid] : 0;
      const int ex = block_exclusive_scan(len, scratch, &E);
      if (tid < nseg) sm.seg_p[tid] = ex;
      __syncthreads();
    }
    for (int e0 = 0; e0 < E; e0 += kGChunk) {
      const int ce = min(kGChunk, E - e0);
      for (int qq = tid; qq < ce; qq += nthr) {
        const int e = e0 + qq;
        const int s = upper_index(sm.seg_p, nseg, e);
        const uint2 ed = a.gedges[seg_s[s] + (e - sm.seg_p[s])];
        sm.st_slot[qq] = ring_slot(s0, edge_delay(ed), R);
        sm.st_w[qq] = edge_w(ed);
        sm.st_col[qq] = edge_col(ed) - cb0;
      }
      if (ce <= kCountMax)  // apply_cells' table
        for (int i = tid; i < 2 * kCellTable; i += nthr) sm.st_next[i] = 0;
      apply_ordered<!RSM>(ce, sm.head, sm.tail, cb1 - cb0, sm.st_col, sm.st_slot, sm.st_w,
                          sm.st_next, rb, stride, col0, kGChunk);
    }
  }
}

// Phase B for at most 64 inbox descriptors (SORT; 32 for BUCKET) -- the
// common step: warp 0 holds them from the speculative read (lane l:
// descriptors l and l + 32) and scans
// their lengths with shuffles (no rank pass).  BUCKET accumulates straight
// away; SORT stages each event with its gedges index as order key -- within
// one destination block the gedges order is the (pre, edge) order of the CPU
// backend, since gedges keeps the CSR row order and regroups each row stably
// by destination block -- and applies it per ring cell (cell_insert /
// cell_apply with a 1024-key table in the descriptor buffer) with no
// descriptor sort.  Returns false, with nothing applied, for a SORT step of
// more than kFastMax events: the general path takes it.
constexpr int kFastDesc = 64;
constexpr int kFastMax = 512;
static_assert(2 * 2 * kFastMax * sizeof(int) <= kGDesc * sizeof(unsigned long long),
              "the fast path's table lives in the descriptor buffer");

template <int MODE, bool RSM>
__device__ bool phase_b_fast(const FwdArgs& a, const GSmem& sm, int k, int t, int cb0, int cnt,
                             unsigned long long spec, unsigned long long spec2, bool tail_sync) {
  __shared__ int s_E;
  const int tid = threadIdx.x, nthr = blockDim.x;
  int* tab = reinterpret_cast<int*>(sm.desc);
  if (tid < 32) {
    const unsigned long long d0 = tid < cnt ? spec : 0ull;
    const unsigned long long d1 = MODE == MODE_SORT && tid + 32 < cnt ? spec2 : 0ull;
    const int l0 = (int)(d0 & 0xffffffffu), l1 = (int)(d1 & 0xffffffffu);
    int i0 = l0, i1 = l1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y0 = __shfl_up_sync(0xffffffffu, i0, o), y1 = __shfl_up_sync(0xffffffffu, i1, o);
      if (tid >= o) {
        i0 += y0;
        i1 += y1;
      }
    }
    const int t0 = __shfl_sync(0xffffffffu, i0, 31);
    if (tid < cnt) {
      sm.dsort[tid] = d0;
      sm.seg_p[tid] = i0 - l0;
    }
    if (tid + 32 < cnt) {
      sm.dsort[tid + 32] = d1;
      sm.seg_p[tid + 32] = t0 + i1 - l1;
    }
    if (tid == 31) s_E = t0 + i1;
  }
  if (MODE == MODE_SORT)
    for (int i = tid; i < 2 * 2 * kFastMax; i += nthr) tab[i] = 0;
  __syncthreads();
  const int E = s_E;
  if (MODE == MODE_SORT && (E > kFastMax || E > nthr)) return false;
  const int R = a.R, s0 = t % R;
  float* rb = ring_base<RSM>(a, sm, k);
  const int stride = RSM ? a.BS : a.ncols;
  const int col0 = RSM ? 0 : cb0;
  if (MODE == MODE_BUCKET) {
    for (int qq = tid; qq < E; qq += nthr) {
      const int d = upper_index(sm.seg_p, cnt, qq);
      const uint2 ed = a.gedges[(int)(sm.dsort[d] >> 32) + (qq - sm.seg_p[d])];
      const int cidx = RSM ? edge_col(ed) - cb0 : edge_col(ed);
      atomicAdd(&rb[(size_t)ring_slot(s0, edge_delay(ed), R) * stride + cidx], edge_w(ed));
    }
    if (tail_sync) __syncthreads();
    return true;
  }
  const int q = tid;  // E <= blockDim.x
  int c = 0, sl = 0;
  unsigned h = 0;
  bool first = false;
  if (q < E) {
    const int d = upper_index(sm.seg_p, cnt, q);
    const int edge = (int)(sm.dsort[d] >> 32) + (q - sm.seg_p[d]);
    const uint2 ed = a.gedges[edge];
    sl = ring_slot(s0, edge_delay(ed), R);
    c = edge_col(ed) - cb0;
    sm.st_w[q] = edge_w(ed);
    sm.st_slot[q] = edge;  // order key
    h = cell_insert<2 * kFastMax>(tab, sm.st_col, q, c, sl, &first);
  }
  __syncthreads();
  if (first)
    cell_apply<!RSM, true, 2 * kFastMax>(tab, sm.st_col, sm.st_slot, sm.st_w, h, q, c, sl, rb, stride,
                                         col0);
  if (tail_sync) __syncthreads();
  return true;
}

// Phase B (BUCKET / SORT): as owner of the ring columns of block b, expand
// this step's inbox descriptors and accumulate them into the block's ring
// slice -- unordered (BUCKET) or per ring cell in (pre, edge) order (SORT).
// tail_sync: close with a barrier (another phase B of this step follows;
// otherwise the caller's next step -- phase A, the end of the wave or of the
// launch -- starts with one).
template <int MODE, bool RSM>
__device__ void phase_b(const FwdArgs& a, const GSmem& sm, int* scratch, int k, int t, int b,
                        int cb0, int cb1, bool tail_sync) {
  __shared__ int s_cnt;
  if (MODE == MODE_SORT && a.scan_only) {  // partitions: no inbox, every fired list
    phase_b_scan<RSM>(a, sm, scratch, k, t, b, cb0, cb1);
    return;
  }
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int R = a.R;
  const int par = t & 1;
  const int s0 = t % R;
  int* cntp = a.inbox_cnt + ((size_t)k * 2 + par) * a.P + b;
  const unsigned long long* box = a.inbox + ((size_t)k * 2 + par) * a.G + sm.ib[b];
  // read the first descriptor slots in the same round trip as the count
  // (slots beyond the count hold stale descriptors and are ignored)
  const int cap = sm.ib[b + 1] - sm.ib[b];
  unsigned long long spec = 0, spec2 = 0;
  if (tid < kGDesc && tid < cap) spec = __ldcg(&box[tid]);
  if (MODE == MODE_SORT && tid < 32 && tid + 32 < cap) spec2 = __ldcg(&box[tid + 32]);
  if (tid == 0) {
    s_cnt = __ldcg(cntp);
    // reset for step t + 2 (written again only after the next grid barrier)
    if (s_cnt) __stcg(cntp, 0);
  }
  __syncthreads();
  const int cnt = s_cnt;
  if (cnt == 0) return;
  if (cnt <= (MODE == MODE_SORT ? kFastDesc : 32) &&
      phase_b_fast<MODE, RSM>(a, sm, k, t, cb0, cnt, spec, spec2, tail_sync))
    return;
  if (MODE == MODE_SORT && cnt > kGDesc) {
    phase_b_scan<RSM>(a, sm, scratch, k, t, b, cb0, cb1);
    return;
  }
  float* rb = ring_base<RSM>(a, sm, k);
  const int stride = RSM ? a.BS : a.ncols;
  const int col0 = RSM ? 0 : cb0;
  for (int d0 = 0; d0 < cnt; d0 += kGDesc) {
    const int dn = min(kGDesc, cnt - d0);
    for (int i = tid; i < dn; i += nthr) sm.desc[i] = (d0 == 0 && i == tid) ? spec : __ldcg(&box[d0 + i]);
    __syncthreads();
    const unsigned long long* src = sm.desc;
    int E;
    if (dn <= 64) {
      // few descriptors: each finds its rank (by first edge for SORT, by
      // position for BUCKET) and its segment offset in one pass, no scan
      __shared__ int s_E;
      if (tid < dn) {
        const unsigned long long key = sm.desc[tid];
        const unsigned kf = (unsigned)(key >> 32);
        int r = 0, off = 0;
        for (int q = 0; q < dn; ++q) {
          const unsigned long long o = sm.desc[q];
          const bool lt = MODE == MODE_SORT ? (unsigned)(o >> 32) < kf : q < tid;
          r += lt;
          off += lt ? (int)(o & 0xffffffffu) : 0;
        }
        sm.dsort[r] = key;
        sm.seg_p[r] = off;
        if (r == dn - 1) s_E = off + (int)(key & 0xffffffffu);
      }
      __syncthreads();
      src = sm.dsort;
      E = s_E;
    } else {
      if (MODE == MODE_SORT) {
        // rank sort by first edge (first edges of distinct rows are distinct)
        for (int i = tid; i < dn; i += nthr) {
          const unsigned long long key = sm.desc[i];
          int r = 0;
          for (int q = 0; q < dn; ++q) r += (sm.desc[q] >> 32) < (key >> 32);
          sm.dsort[r] = key;
        }
        __syncthreads();
        src = sm.dsort;
      }
      // prefix of segment lengths, two descriptors per thread
      const int i0 = 2 * tid, i1 = 2 * tid + 1;
      const int l0 = i0 < dn ? (int)(src[i0] & 0xffffffffu) : 0;
      const int l1 = i1 < dn ? (int)(src[i1] & 0xffffffffu) : 0;
      const int ex = block_exclusive_scan(l0 + l1, scratch, &E);
      if (i0 < dn) sm.seg_p[i0] = ex;
      if (i1 < dn) sm.seg_p[i1] = ex + l0;
      __syncthreads();
    }
    for (int e0 = 0; e0 < E; e0 += kGChunk) {
      const int ce = min(kGChunk, E - e0);
      for (int qq = tid; qq < ce; qq += nthr) {
        const int e = e0 + qq;
        const int d = upper_index(sm.seg_p, dn, e);
        const int edge = (int)(src[d] >> 32) + (e - sm.seg_p[d]);
        const uint2 ed = a.gedges[edge];
        const int slot = ring_slot(s0, edge_delay(ed), R);
        if (MODE == MODE_BUCKET) {
          // shared slice: block-local column; global ring: global column
          const int cidx = RSM ? edge_col(ed) - cb0 : edge_col(ed);
          atomicAdd(&rb[(size_t)slot * stride + cidx], edge_w(ed));
        } else {
          sm.st_slot[qq] = slot;
          sm.st_w[qq] = edge_w(ed);
          sm.st_col[qq] = edge_col(ed) - cb0;
        }
      }
      if (MODE == MODE_SORT) {
        if (ce <= kCountMax)  // apply_cells' table
          for (int i = tid; i < 2 * kCellTable; i += nthr) sm.st_next[i] = 0;
        apply_ordered<!RSM>(ce, sm.head, sm.tail, cb1 - cb0, sm.st_col, sm.st_slot, sm.st_w,
                            sm.st_next, rb, stride, col0, kGChunk);
      } else {
        __syncthreads();
      }
    }
  }
}

template <int MODE, bool RSM, bool EPR>
__global__ void __launch_bounds__(kGThreadsMax, 1) k_tier_g(FwdArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int scratch[40];
  __shared__ unsigned long long s_acc[2 * kMaxWave];
  __shared__ int s_samp[kMaxWave], s_T[kMaxWave];
  __shared__ long long s_gb[kMaxWave];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const GSmem sm = carve_g(smem_raw, a.BS, a.P, a.R, a.Bw, true, RSM);
  const int b = blockIdx.x;
  const int BS = a.BS, R = a.R;
  const int lo = b * BS, hi = min(a.N, lo + BS);
  const int cb0 = a.colbase[b], cb1 = a.colbase[b + 1];
  const unsigned nb = gridDim.x;
  unsigned target = a.stall;
  for (int jj = tid; jj < BS; jj += nthr) {
    sm.col[jj] = lo + jj < hi ? a.col_of[lo + jj] : -1;
    sm.och[jj] = lo + jj < hi ? a.out_ch[lo + jj] : -1;
    sm.head[jj] = -1;
    sm.tail[jj] = -1;
  }
  for (int i = tid; i < a.Bw * BS; i += nthr) sm.ext[i] = 0.f;
  for (int jj = tid; jj <= BS; jj += nthr) {
    const int j = min(lo + jj, hi);
    sm.rp[jj] = a.row_ptr[j];
    sm.gp[jj] = a.gptr[j];
  }
  for (int i = tid; i <= a.P; i += nthr) sm.ib[i] = a.ibase[i];
  const int nwaves = (a.B + a.Bw - 1) / a.Bw;
  for (int w = 0; w < nwaves; ++w) {
    const int q0 = w * a.Bw;
    const int nk = min(a.Bw, a.B - q0);
    if (tid < nk) {
      const int smp = a.order[q0 + tid];
      s_samp[tid] = smp;
      s_T[tid] = a.steps[smp];
      s_gb[tid] = a.stepbase[smp];
      s_acc[tid] = 0;
      s_acc[kMaxWave + tid] = 0;
    }
    for (int i = tid; i < nk * BS; i += nthr) {
      sm.v[i] = 0.f;
      sm.refr[i] = 0;
    }
    if (RSM) {
      for (int i = tid; i < nk * R * BS; i += nthr) sm.ring[i] = 0.f;
    } else {
      const int wcol = cb1 - cb0;
      for (int k = 0; k < nk; ++k) {
        float* ringk = a.ring + (size_t)k * R * a.ncols;
        for (int i = tid; i < R * wcol; i += nthr)
          __stcg(&ringk[(size_t)(i / wcol) * a.ncols + cb0 + (i % wcol)], 0.f);
      }
    }
    target += nb;
    if (!grid_sync(&a.ctl[0], target, a.err, a.wait_ns)) return;
    const int Tw = s_T[0];
    for (int t = 0; t < Tw; ++t) {
      for (int k = 0; k < nk; ++k)
        if (t < s_T[k])
          phase_a<MODE, true, RSM, EPR>(a, sm, scratch, s_acc, k, s_samp[k], s_gb[k] + t, t, b, cb0,
                                   t > 0);
      // arrive, fetch the next step's drive while the other blocks catch up,
      // then wait
      target += nb;
      grid_arrive(&a.ctl[0]);
      for (int k = 0; k < nk; ++k)
        if (t + 1 < s_T[k])
          load_ext(a, sm.ext + (size_t)k * BS, s_samp[k], s_gb[k] + t + 1, t + 1, b);
      if (!grid_wait(&a.ctl[0], target, a.err, a.wait_ns)) return;
      if (MODE != MODE_ATOMIC)
        for (int k = 0; k < nk; ++k)
          if (t < s_T[k]) {
            bool more = false;
            for (int k2 = k + 1; k2 < nk; ++k2) more |= t < s_T[k2];
            phase_b<MODE, RSM>(a, sm, scratch, k, t, b, cb0, cb1, more);
          }
    }
    __syncthreads();
    if (tid < nk) {
      if (s_acc[tid]) atomicAdd(&a.spikes[s_samp[tid]], s_acc[tid]);
      if (s_acc[kMaxWave + tid]) atomicAdd(&a.events[s_samp[tid]], s_acc[kMaxWave + tid]);
    }
    if (a.vfinal)
      for (int k = 0; k < nk; ++k)
        for (int j = lo + tid; j < hi; j += nthr)
          a.vfinal[(size_t)s_samp[k] * a.N + j] = sm.v[k * BS + (j - lo)];
    if (a.ro_on)
      for (int k = 0; k < nk; ++k)
        for (int j = lo + tid; j < hi; j += nthr)
          if (sm.och[j - lo] >= 0)
            a.ro_v[(size_t)s_samp[k] * a.n_ro + a.ro_rank[j]] = sm.v[k * BS + (j - lo)];
    target += nb;
    if (!grid_sync(&a.ctl[0], target, a.err, a.wait_ns)) return;
  }
}

template <int MODE>
__global__ void __launch_bounds__(kGThreads) k_plain_a(FwdArgs a, int sample, long long gstep, int t) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int scratch[40];
  const GSmem sm = carve_g(smem_raw, a.BS, a.P, a.R, 1, false, false);
  for (int jj = threadIdx.x; jj < a.BS; jj += blockDim.x) sm.ext[jj] = 0.f;
  for (int i = threadIdx.x; i <= a.P; i += blockDim.x) sm.ib[i] = a.ibase[i];
  __syncthreads();
  const int b = a.blk0 + blockIdx.x;
  phase_a<MODE, false, false>(a, sm, scratch, nullptr, 0, sample, gstep, t, b, a.colbase[b], false);
}

template <int MODE>
__global__ void __launch_bounds__(kGThreads) k_plain_b(FwdArgs a, int t) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int scratch[40];
  const GSmem sm = carve_g(smem_raw, a.BS, a.P, a.R, 1, false, false);
  for (int jj = threadIdx.x; jj < a.BS; jj += blockDim.x) {
    sm.head[jj] = -1;
    sm.tail[jj] = -1;
  }
  for (int i = threadIdx.x; i <= a.P; i += blockDim.x) sm.ib[i] = a.ibase[i];
  __syncthreads();
  const int b = a.blk0 + blockIdx.x;
  phase_b<MODE, false>(a, sm, scratch, 0, t, b, a.colbase[b], a.colbase[b + 1], false);
}

// Zero wave slot 0's global state of block b (plain path, once per sample).
__global__ void k_plain_init(FwdArgs a) {
  const int b = a.blk0 + blockIdx.x;
  const int lo = b * a.BS, hi = min(a.N, lo + a.BS);
  const int cb0 = a.colbase[b], cb1 = a.colbase[b + 1];
  for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
    a.v[j] = 0.f;
    a.refr[j] = 0;
  }
  const int w = cb1 - cb0;
  for (int i = threadIdx.x; i < a.R * w; i += blockDim.x)
    a.ring[(size_t)(i / w) * a.ncols + cb0 + (i % w)] = 0.f;
}

__global__ void k_copy_v(FwdArgs a, int sample) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < a.N; j += gridDim.x * blockDim.x) {
    if (a.vfinal) a.vfinal[(size_t)sample * a.N + j] = a.v[j];
    if (a.ro_on && a.ro_rank[j] >= 0) a.ro_v[(size_t)sample * a.n_ro + a.ro_rank[j]] = a.v[j];
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static FwdArgs make_args(Run* r, const snc_lif* lif) {
  const Graph* g = r->g;
  const Inputs* in = r->in;
  FwdArgs a{};
  a.N = g->N; a.S = g->S; a.R = g->R; a.ncols = g->ncols; a.noc = std::max(1, g->noc);
  a.P = g->P; a.BS = g->BS; a.G = g->G;
  a.row_ptr = g->row_ptr; a.edges = g->edges; a.gedges = g->gedges; a.gptr = g->gptr;
  a.groups = g->groups; a.col_of = g->col_of; a.out_ch = g->out_ch; a.colbase = g->colbase;
  a.ibase = g->ibase;
  a.B = in->B; a.order = in->order; a.steps = in->steps; a.sptr_off = in->sptr_off;
  a.stepbase = in->stepbase;
  a.sched_ptr = in->sched_ptr; a.sched_nid = in->sched_nid; a.sched_ext = in->sched_ext;
  a.sched_blk = in->sched_blk;
  a.raster_off = in->raster_off;
  a.counts = r->counts; a.spikes = r->spikes; a.events = r->events;
  a.raster = (r->flags & SNC_B200_RUN_RASTER) ? r->raster : nullptr;
  a.vfinal = (r->flags & SNC_B200_RUN_VFINAL) ? r->vfinal : nullptr;
  a.W = r->W;
  a.Bw = r->Bw; a.v = r->v; a.refr = r->refr; a.ring = r->ring; a.fired = r->fired;
  a.fired_cnt = r->fired_cnt; a.inbox = r->inbox; a.inbox_cnt = r->inbox_cnt;
  a.err = r->err; a.ctl = r->ctl;
  a.lif = LifP{lif->threshold, lif->decay, lif->reset, lif->refractory, lif->reset_mode};
  if (r->edges_w) a.edges = r->edges_w;
  if (r->gedges_w) a.gedges = r->gedges_w;
  a.psi_hist = r->psi_hist;
  a.psi_T = r->psi_T;
  a.fires = r->fires;
  a.gamma = r->gamma;
  a.ro_on = r->ro_decay >= 0.f && r->ro_v && r->ro_logits ? 1 : 0;
  a.ro_decay = a.ro_on ? r->ro_decay : 0.f;
  a.ro_rank = g->ro_rank;
  a.ro_chan = g->ro_chan;
  a.n_ro = g->n_ro;
  a.ro_v = r->ro_v;
  a.ro_logits = r->ro_logits;
  return a;
}

static int ensure_grid_state(Run* r, int Bw) {
  if (r->v && r->Bw_cap >= Bw) {
    r->Bw = Bw;
    return SNC_B200_OK;
  }
  const Graph* g = r->g;
  for (void* p : {(void*)r->v, (void*)r->refr, (void*)r->ring, (void*)r->fired,
                  (void*)r->fired_cnt, (void*)r->inbox, (void*)r->inbox_cnt})
    dev_free(p);
  r->v = nullptr; r->refr = nullptr; r->ring = nullptr; r->fired = nullptr;
  r->fired_cnt = nullptr; r->inbox = nullptr; r->inbox_cnt = nullptr;
  int rc;
  if ((rc = dev_alloc(&r->v, (size_t)Bw * g->N))) return rc;
  if ((rc = dev_alloc(&r->refr, (size_t)Bw * g->N))) return rc;
  if ((rc = dev_alloc(&r->ring, (size_t)Bw * g->R * std::max(1, g->ncols)))) return rc;
  if ((rc = dev_alloc(&r->fired, (size_t)Bw * 2 * g->N))) return rc;
  if ((rc = dev_alloc(&r->fired_cnt, (size_t)Bw * 2 * g->P))) return rc;
  if ((rc = dev_alloc(&r->inbox, (size_t)Bw * 2 * std::max(1, g->G)))) return rc;
  if ((rc = dev_alloc(&r->inbox_cnt, (size_t)Bw * 2 * g->P))) return rc;
  r->Bw = Bw;
  r->Bw_cap = Bw;
  return SNC_B200_OK;
}

static int optin_smem() {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return optin;
}

template <int MODE, bool EP>
static int launch_tier_s_kernel(const Graph* g, int B, const FwdArgs& a_in, cudaStream_t st) {
  const int nthr = 1024;
  FwdArgs a = a_in;
  size_t smem = tier_s_bytes(g->N, g->ncols, g->R, a.noc, MODE, EP, nthr);
  SNCB_CUDA(cudaFuncSetAttribute(k_tier_s<MODE, EP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  SNCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tier_s<MODE, EP>, nthr, smem));
  a.s_table = 0;
  a.s_lean = 0;
  if (MODE == MODE_SORT) {
    // the per-cell table (and the cell bitmaps with it) when it fits without
    // costing a CTA per SM; the richest layout that fits, the full one before
    // the lean one (e-prop only)
    for (int v = 0; v < 4 && !a.s_table; ++v) {
      const int tab = 2 - v / 2;
      const bool lean = (v & 1) != 0;
      if (lean && !EP) continue;
      const size_t smem_t = tier_s_bytes(g->N, g->ncols, g->R, a.noc, MODE, EP, nthr, tab, lean);
      int per_sm_t = 0;
      if ((int)smem_t <= optin_smem() &&
          cudaFuncSetAttribute(k_tier_s<MODE, EP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_t) ==
              cudaSuccess &&
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_t, k_tier_s<MODE, EP>, nthr, smem_t) ==
              cudaSuccess &&
          per_sm_t >= per_sm && per_sm_t >= 1) {
        smem = smem_t;
        a.s_table = tab;
        a.s_lean = lean ? 1 : 0;
      } else {
        cudaGetLastError();
      }
    }
    if (!a.s_table)
      SNCB_CUDA(cudaFuncSetAttribute(k_tier_s<MODE, EP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  if (per_sm < 1) {
    set_error("tier S does not fit on an SM");
    return SNC_B200_EUNSUPPORTED;
  }
  const int grid = std::max(1, std::min(B, per_sm * g->sm_count));
  k_tier_s<MODE, EP><<<grid, nthr, smem, st>>>(a);
  SNCB_CUDA(cudaGetLastError());
  return SNC_B200_OK;
}

template <int MODE>
static int launch_tier_s(Run* r, const FwdArgs& a, cudaStream_t st) {
  return launch_tier_s_kernel<MODE, false>(r->g, r->in->B, a, st);
}

// e-prop forward of one minibatch (tier S with eligibility), see eprop.cu.
int launch_eprop_forward(const EpropLaunch& e, cudaStream_t st) {
  const Graph* g = e.g;
  const Inputs* in = e.in;
  if (tier_s_bytes(g->N, g->ncols, g->R, std::max(1, g->noc), e.mode, true, 1024) >
      (size_t)optin_smem()) {
    set_error("e-prop: one sample's state does not fit in one CTA's shared memory");
    return SNC_B200_EUNSUPPORTED;
  }
  FwdArgs a{};
  a.N = g->N; a.S = g->S; a.R = g->R; a.ncols = g->ncols; a.noc = std::max(1, g->noc);
  a.P = g->P; a.BS = g->BS; a.G = g->G;
  a.row_ptr = g->row_ptr; a.edges = e.edges; a.gedges = g->gedges; a.col_of = g->col_of;
  a.out_ch = g->out_ch;
  a.B = in->B; a.order = in->order; a.steps = in->steps; a.sptr_off = in->sptr_off;
  a.stepbase = in->stepbase; a.sched_ptr = in->sched_ptr; a.sched_nid = in->sched_nid;
  a.sched_ext = in->sched_ext; a.raster_off = in->raster_off;
  a.counts = e.counts; a.spikes = e.spikes; a.events = e.events;
  a.W = (g->N + 31) / 32;
  a.err = e.err; a.ctl = e.ctl;
  a.lif = LifP{e.lif.threshold, e.lif.decay, e.lif.reset, e.lif.refractory, e.lif.reset_mode};
  a.elig = e.elig; a.fires = e.fires; a.gamma = e.gamma; a.trace_decay = e.trace_decay;
  a.psi_hist = e.psi_hist; a.psi_T = e.psi_T;
  a.raster = e.raster;
  if (e.mode == MODE_SORT) return launch_tier_s_kernel<MODE_SORT, true>(g, in->B, a, st);
  return launch_tier_s_kernel<MODE_ATOMIC, true>(g, in->B, a, st);
}

// Wave size and ring placement of the tier-G kernel for this run.
struct GPlan {
  bool rsm;
  int Bw;
  size_t smem;
};

// want_rsm: -1 automatic (shared-memory ring slices when one sample fits),
// 0 global ring, 1 shared-memory slices (rsm false in the result when they do
// not fit); want_wave: 0 automatic (as many samples as fit), else at most that.
// Static shared memory of the tier-G kernels (the largest instance): the
// dynamic allocation may use what the opt-in limit leaves beside it.
static size_t tier_g_static_smem() {
  static size_t cached = 0;
  static bool done = false;
  if (!done) {
    const void* fns[] = {(const void*)k_tier_g<MODE_ATOMIC, false, false>,
                         (const void*)k_tier_g<MODE_BUCKET, true, false>,
                         (const void*)k_tier_g<MODE_BUCKET, false, false>,
                         (const void*)k_tier_g<MODE_SORT, true, false>,
                         (const void*)k_tier_g<MODE_SORT, false, false>,
                         (const void*)k_tier_g<MODE_ATOMIC, false, true>,
                         (const void*)k_tier_g<MODE_SORT, true, true>,
                         (const void*)k_tier_g<MODE_SORT, false, true>};
    size_t m = 0;
    for (const void* f : fns) {
      cudaFuncAttributes fa{};
      if (cudaFuncGetAttributes(&fa, f) == cudaSuccess) m = std::max(m, fa.sharedSizeBytes);
      else cudaGetLastError();
    }
    cached = m;
    done = true;
  }
  return cached;
}

static GPlan plan_tier_g(const Graph* g, int B, int mode, int want_rsm = -1, int want_wave = 0) {
  const size_t optin = (size_t)optin_smem() - std::min((size_t)optin_smem(), tier_g_static_smem());
  GPlan p{false, 1, 0};
  int cap = std::max(1, std::min(B, kMaxWave));
  if (want_wave > 0) cap = std::min(cap, want_wave);
  if (mode != MODE_ATOMIC && want_rsm != 0) {
    int bw = 0;
    while (bw < cap && g_smem_bytes(g->BS, g->P, g->R, bw + 1, true, true) <= optin) ++bw;
    if (bw >= 1) {
      p.rsm = true;
      p.Bw = bw;
    }
  }
  if (!p.rsm) {
    int bw = 0;
    while (bw < cap && g_smem_bytes(g->BS, g->P, g->R, bw + 1, true, false) <= optin) ++bw;
    p.Bw = std::max(1, bw);
  }
  p.smem = g_smem_bytes(g->BS, g->P, g->R, p.Bw, true, p.rsm);
  return p;
}

// Tier-G block size: one thread per neuron of the block when it fits, so the
// integration of a step is a single pass (at least kGThreads, which the
// descriptor prefix scan relies on).
static int tier_g_threads(const Graph* g) {
  return std::max(kGThreads, std::min(kGThreadsMax, (g->BS + 31) / 32 * 32));
}

template <int MODE, bool RSM, bool EPR>
static int launch_tier_g(Run* r, const FwdArgs& a, size_t smem, cudaStream_t st) {
  const Graph* g = r->g;
  const int nthr = r->cfg_threads > 0 ? r->cfg_threads : tier_g_threads(g);
  SNCB_CUDA(cudaFuncSetAttribute(k_tier_g<MODE, RSM, EPR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  SNCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tier_g<MODE, RSM, EPR>, nthr, smem));
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
  SNCB_CUDA(cudaLaunchKernelEx(&cfg, k_tier_g<MODE, RSM, EPR>, a));
  return SNC_B200_OK;
}

template <int MODE>
static int launch_plain(Run* r, FwdArgs a, cudaStream_t st) {
  const Graph* g = r->g;
  const Inputs* in = r->in;
  const int nthr = kGThreads;
  const size_t smem = g_smem_bytes(g->BS, g->P, g->R, 1, false, false);
  SNCB_CUDA(cudaFuncSetAttribute(k_plain_a<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  SNCB_CUDA(cudaFuncSetAttribute(k_plain_b<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (int q = 0; q < in->B; ++q) {
    const int smp = in->order_h[q];
    const int T = in->steps_h[smp];
    const long long gb = in->stepbase_h[smp];
    k_plain_init<<<g->P, nthr, 0, st>>>(a);
    for (int t = 0; t < T; ++t) {
      k_plain_a<MODE><<<g->P, nthr, smem, st>>>(a, smp, gb + t, t);
      if (MODE != MODE_ATOMIC) k_plain_b<MODE><<<g->P, nthr, smem, st>>>(a, t);
    }
    if (a.vfinal || a.ro_on)
      k_copy_v<<<std::max(1, std::min(1024, (g->N + 255) / 256)), 256, 0, st>>>(a, smp);
  }
  SNCB_CUDA(cudaGetLastError());
  return SNC_B200_OK;
}

static bool tier_s_fits(const Graph* g, int mode) {
  return tier_s_bytes(g->N, g->ncols, g->R, std::max(1, g->noc), mode, false, 1024) <=
         (size_t)optin_smem();
}

static bool use_tier_s(const Run* r, int mode, int path) {
  return path == SNC_B200_PATH_PERSISTENT && tier_s_fits(r->g, mode) &&
         !(r->flags & SNC_B200_RUN_FORCE_GRID) && r->cfg_tier != 1;
}

int check_shape(const Run* r, int mode, int tier, int threads, int wave, int rsm) {
  const Graph* g = r->g;
  if (tier == 0 && !tier_s_fits(g, mode)) {
    set_error("launch shape: one sample's state does not fit one CTA (tier 0)");
    return SNC_B200_EUNSUPPORTED;
  }
  if (tier < -1 || tier > 1 || wave < 0 || rsm < -1 || rsm > 1 ||
      (threads != 0 && (threads % 32 != 0 || threads < kGThreads || threads > kGThreadsMax))) {
    set_error("launch shape: tier -1..1, threads 0 or a multiple of 32 in [512, 768], wave >= 0, "
              "ring_smem -1..1");
    return SNC_B200_EUNSUPPORTED;
  }
  if (rsm == 1 && mode != MODE_ATOMIC) {
    const GPlan p = plan_tier_g(g, std::max(1, r->in->B), mode, 1, wave);
    if (!p.rsm) {
      set_error("launch shape: ring slices do not fit in shared memory");
      return SNC_B200_EUNSUPPORTED;
    }
  }
  return SNC_B200_OK;
}

static int launch_kernels(Run* r, const FwdArgs& a, int mode, int path, cudaStream_t st);

// Launch body without timing / graph handling: the forward, then the logits
// of the leaky readout units when they are on.
static int launch_body(Run* r, const FwdArgs& a, int mode, int path, cudaStream_t st) {
  int rc = launch_kernels(r, a, mode, path, st);
  if (rc || !a.ro_on) return rc;
  if (r->in->B > 0) {
    k_readout_logits<<<r->in->B, 32, 0, st>>>(a.ro_v, a.ro_chan, a.n_ro, r->in->steps, a.noc,
                                              a.ro_logits);
    SNCB_CUDA(cudaGetLastError());
  }
  return SNC_B200_OK;
}

static int launch_kernels(Run* r, const FwdArgs& a, int mode, int path, cudaStream_t st) {
  if (use_tier_s(r, mode, path)) {
    if (mode == MODE_SORT) return launch_tier_s<MODE_SORT>(r, a, st);
    return launch_tier_s<MODE_ATOMIC>(r, a, st);
  }
  if (path == SNC_B200_PATH_PERSISTENT) {
    const size_t smem = r->gplan_smem;
    if (r->psi_hist || r->fires) {  // e-prop: ATOMIC or SORT delivery
      if (mode == MODE_ATOMIC) return launch_tier_g<MODE_ATOMIC, false, true>(r, a, smem, st);
      if (r->gplan_rsm) return launch_tier_g<MODE_SORT, true, true>(r, a, smem, st);
      return launch_tier_g<MODE_SORT, false, true>(r, a, smem, st);
    }
    if (mode == MODE_ATOMIC) return launch_tier_g<MODE_ATOMIC, false, false>(r, a, smem, st);
    if (r->gplan_rsm) {
      if (mode == MODE_SORT) return launch_tier_g<MODE_SORT, true, false>(r, a, smem, st);
      return launch_tier_g<MODE_BUCKET, true, false>(r, a, smem, st);
    }
    if (mode == MODE_SORT) return launch_tier_g<MODE_SORT, false, false>(r, a, smem, st);
    return launch_tier_g<MODE_BUCKET, false, false>(r, a, smem, st);
  }
  if (mode == MODE_SORT) return launch_plain<MODE_SORT>(r, a, st);
  if (mode == MODE_BUCKET) return launch_plain<MODE_BUCKET>(r, a, st);
  return launch_plain<MODE_ATOMIC>(r, a, st);
}

int launch_run(Run* r, const snc_lif* lif, int mode, int path, cudaStream_t st) {
  const Graph* g = r->g;
  const Inputs* in = r->in;
  if (mode == SNC_B200_MODE_AUTO || path == SNC_B200_PATH_AUTO) {
    int m = mode, p = path, shape[4] = {-1, 0, 0, -1};
    int rc = resolve_auto(g, in, &m, &p, shape);
    if (rc) return rc;
    if (mode == SNC_B200_MODE_AUTO) mode = m;
    if (path == SNC_B200_PATH_AUTO) path = p;
    if (!r->cfg_explicit) {  // the tuned shape, unless the caller set one
      r->cfg_tier = shape[0];
      r->cfg_threads = shape[1];
      r->cfg_wave = shape[2];
      r->cfg_rsm = shape[3];
    }
  }
  if (mode < 0 || mode > MODE_SORT || path < 0 || path > SNC_B200_PATH_PERSISTENT) {
    set_error("bad mode or path");
    return SNC_B200_EINVAL;
  }
  int rc;
  if (!use_tier_s(r, mode, path)) {
    int Bw = 1;
    if (path == SNC_B200_PATH_PERSISTENT) {
      const GPlan p = plan_tier_g(g, in->B, mode, r->cfg_rsm, r->cfg_wave);
      Bw = p.Bw;
      r->gplan_rsm = p.rsm;
      r->gplan_smem = p.smem;
    }
    if ((rc = ensure_grid_state(r, Bw))) return rc;
  }
  FwdArgs a = make_args(r, lif);
  const bool grid = path == SNC_B200_PATH_PERSISTENT && !use_tier_s(r, mode, path);
  const WaitCtl wc = take_wait_ctl(grid && in->B > 0);  // only grid launches wait
  a.wait_ns = wc.ns;
  a.stall = wc.stall;
  const size_t B = (size_t)std::max(1, in->B);
  // The legacy default stream cannot be captured; a run owns a blocking
  // stream (ordered with the legacy stream) that stands in for it.
  if (!st) {
    if (!r->own_stream) SNCB_CUDA(cudaStreamCreate(&r->own_stream));
    st = r->own_stream;
  }
  SNCB_CUDA(cudaMemsetAsync(r->counts, 0, B * std::max(1, g->noc) * sizeof(int), st));
  SNCB_CUDA(cudaMemsetAsync(r->spikes, 0, B * sizeof(unsigned long long), st));
  SNCB_CUDA(cudaMemsetAsync(r->events, 0, B * sizeof(unsigned long long), st));
  SNCB_CUDA(cudaMemsetAsync(r->ctl, 0, 4 * sizeof(unsigned), st));
  SNCB_CUDA(cudaMemsetAsync(r->err, 0, sizeof(int), st));
  if (r->inbox_cnt)
    SNCB_CUDA(cudaMemsetAsync(r->inbox_cnt, 0, (size_t)r->Bw_cap * 2 * g->P * sizeof(int), st));
  if ((r->flags & SNC_B200_RUN_RASTER) && in->raster_words)
    SNCB_CUDA(cudaMemsetAsync(r->raster, 0, (size_t)in->raster_words * sizeof(uint32_t), st));
  SNCB_CUDA(cudaEventRecord(r->ev0, st));
  r->used_graph = false;
  if (in->B > 0) {
    // an injected stall is never captured: the graph keeps the normal launch
    bool use_graph = (r->flags & SNC_B200_RUN_GRAPH) && path == SNC_B200_PATH_PERSISTENT &&
                     !r->graph_refused && a.stall == 0;
    if (use_graph) {
      const int shape[4] = {r->cfg_tier, r->cfg_threads, r->cfg_wave, r->cfg_rsm};
      const bool same = r->gexec && r->gexec_mode == mode && r->gexec_stream == st &&
                        r->gexec_wait_ns == a.wait_ns && r->gexec_ro == (a.ro_on ? a.ro_decay : -1.f) &&
                        std::memcmp(r->gexec_shape, shape, sizeof(shape)) == 0 &&
                        std::memcmp(&r->gexec_lif, lif, sizeof(snc_lif)) == 0;
      if (!same) {
        if (r->gexec) cudaGraphExecDestroy(r->gexec);
        r->gexec = nullptr;
        cudaGraph_t cg = nullptr;
        cudaError_t ce = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (ce == cudaSuccess) {
          rc = launch_body(r, a, mode, path, st);
          ce = cudaStreamEndCapture(st, &cg);
          if (rc) {
            if (cg) cudaGraphDestroy(cg);
            return rc;
          }
          if (ce == cudaSuccess) ce = cudaGraphInstantiate(&r->gexec, cg, 0);
          if (cg) cudaGraphDestroy(cg);
        }
        if (ce != cudaSuccess) {
          // capture refused: remember it and launch directly from now on
          cudaGetLastError();
          r->gexec = nullptr;
          r->graph_refused = true;
          use_graph = false;
        } else {
          r->gexec_mode = mode;
          r->gexec_lif = *lif;
          r->gexec_stream = st;
          r->gexec_wait_ns = a.wait_ns;
          std::memcpy(r->gexec_shape, shape, sizeof(shape));
          r->gexec_ro = a.ro_on ? a.ro_decay : -1.f;
        }
      }
    }
    if (use_graph) {
      SNCB_CUDA(cudaGraphLaunch(r->gexec, st));
      r->used_graph = true;
    } else {
      if ((rc = launch_body(r, a, mode, path, st))) return rc;
    }
  }
  SNCB_CUDA(cudaEventRecord(r->ev1, st));
  r->used_mode = mode;
  r->used_path = path;
  return SNC_B200_OK;
}

// ---------------------------------------------------------------------------
// post-neuron partitions (one sample; the neuron-partitioned C2 mode)
// ---------------------------------------------------------------------------
// Rank r of a partitioned run owns neuron blocks [blk_lo, blk_hi) -- their
// state and ring columns -- and keeps the whole graph.  Per step: integrate
// the own blocks (k_plain_a without inbox posting; spike bits go to the
// raster row of the step), exchange the raster row's words (the caller:
// an all-gather), rebuild every block's ascending fired list from the full
// row (k_mask_fired), then deliver into the own columns by scanning those
// lists in (pre, edge) order (k_plain_b with scan_only): the contributions
// of every ring cell arrive in the serial CPU backend's order, so the union
// of the ranks' results equals a single-device run bit for bit.

// Fired lists and counts of every block from one step's spike bits.
__global__ void k_mask_fired(const uint32_t* __restrict__ mask, int N, int BS, int* fired,
                             int* fired_cnt, int P) {
  __shared__ int scratch[40];
  const int b = blockIdx.x;
  const int lo = b * BS, hi = min(N, lo + BS);
  const int w0 = lo >> 5, w1 = (hi + 31) >> 5;  // BS is a multiple of 32
  int base = 0;
  for (int c0 = w0; c0 < w1; c0 += blockDim.x) {
    const int w = c0 + threadIdx.x;
    uint32_t m = w < w1 ? mask[w] : 0u;
    if (w == w1 - 1 && (hi & 31)) m &= (1u << (hi & 31)) - 1u;  // bits beyond N
    int tot;
    const int ex = block_exclusive_scan(__popc(m), scratch, &tot);
    int pos = base + ex;
    while (m) {
      const int bit = __ffs(m) - 1;
      m &= m - 1u;
      fired[lo + pos++] = (w << 5) + bit;
    }
    base += tot;
  }
  if (threadIdx.x == 0) fired_cnt[b] = base;
}

struct Part {
  Run run;
  int blk_lo = 0, blk_hi = 0;
  snc_lif lif{};
  FwdArgs a{};
  size_t smem = 0;
};

static int part_create(const Graph* g, const Inputs* in, int blk_lo, int blk_hi, const snc_lif* lif,
                       Part* p) {
  if (in->B != 1) { set_error("partition: one sample per run"); return SNC_B200_EINVAL; }
  if (blk_lo < 0 || blk_hi > g->P || blk_lo >= blk_hi) {
    set_error("partition: blocks must satisfy 0 <= block_lo < block_hi <= num_blocks");
    return SNC_B200_EINVAL;
  }
  Run* r = &p->run;
  r->g = g;
  r->in = in;
  r->flags = SNC_B200_RUN_RASTER | SNC_B200_RUN_VFINAL;
  r->W = (g->N + 31) / 32;
  int rc;
  if ((rc = dev_alloc(&r->counts, (size_t)std::max(1, g->noc)))) return rc;
  if ((rc = dev_alloc(&r->spikes, 1))) return rc;
  if ((rc = dev_alloc(&r->events, 1))) return rc;
  if ((rc = dev_alloc(&r->raster, (size_t)std::max<long long>(1, in->raster_words)))) return rc;
  if ((rc = dev_alloc(&r->vfinal, (size_t)std::max(1, g->N)))) return rc;
  if ((rc = dev_alloc(&r->err, 1))) return rc;
  if ((rc = dev_alloc(&r->ctl, 4))) return rc;
  if ((rc = ensure_grid_state(r, 1))) return rc;
  p->blk_lo = blk_lo;
  p->blk_hi = blk_hi;
  p->lif = *lif;
  p->a = make_args(r, lif);
  p->a.blk0 = blk_lo;
  p->a.no_post = 1;
  p->a.scan_only = 1;
  p->smem = g_smem_bytes(g->BS, g->P, g->R, 1, false, false);
  SNCB_CUDA(cudaFuncSetAttribute(k_plain_a<MODE_SORT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem));
  SNCB_CUDA(cudaFuncSetAttribute(k_plain_b<MODE_SORT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem));
  return SNC_B200_OK;
}

static int part_integrate(Part* p, int t, uint32_t* mask, cudaStream_t st) {
  Run* r = &p->run;
  const Graph* g = r->g;
  const int T = r->in->steps_h[0];
  if (t < 0 || t >= T) { set_error("partition: step outside the sample"); return SNC_B200_EINVAL; }
  const int nb = p->blk_hi - p->blk_lo;
  if (t == 0) {
    SNCB_CUDA(cudaMemsetAsync(r->err, 0, sizeof(int), st));
    SNCB_CUDA(cudaMemsetAsync(r->ctl, 0, 4 * sizeof(unsigned), st));
    SNCB_CUDA(cudaMemsetAsync(r->counts, 0, (size_t)std::max(1, g->noc) * sizeof(int), st));
    SNCB_CUDA(cudaMemsetAsync(r->spikes, 0, sizeof(unsigned long long), st));
    SNCB_CUDA(cudaMemsetAsync(r->events, 0, sizeof(unsigned long long), st));
    SNCB_CUDA(cudaMemsetAsync(r->raster, 0, (size_t)std::max<long long>(1, r->in->raster_words) * 4, st));
    k_plain_init<<<nb, kGThreads, 0, st>>>(p->a);
  }
  const long long gb = r->in->stepbase_h[0];
  k_plain_a<MODE_SORT><<<nb, kGThreads, p->smem, st>>>(p->a, 0, gb + t, t);
  SNCB_CUDA(cudaGetLastError());
  if (mask) {  // this partition's words of the step's spike bits
    const size_t w0 = (size_t)p->blk_lo * g->BS / 32;
    const size_t w1 = std::min<size_t>((size_t)r->W, (size_t)p->blk_hi * g->BS / 32);
    if (w1 > w0)
      SNCB_CUDA(cudaMemcpyAsync(mask + w0, r->raster + (size_t)t * r->W + w0, (w1 - w0) * 4,
                                cudaMemcpyDeviceToDevice, st));
  }
  return SNC_B200_OK;
}

static int part_deliver(Part* p, int t, const uint32_t* mask, cudaStream_t st) {
  Run* r = &p->run;
  const Graph* g = r->g;
  const int par = t & 1;
  k_mask_fired<<<g->P, 256, 0, st>>>(mask, g->N, g->BS, r->fired + (size_t)par * g->N,
                                     r->fired_cnt + (size_t)par * g->P, g->P);
  k_plain_b<MODE_SORT><<<p->blk_hi - p->blk_lo, kGThreads, p->smem, st>>>(p->a, t);
  SNCB_CUDA(cudaGetLastError());
  if (t == r->in->steps_h[0] - 1)
    k_copy_v<<<std::max(1, std::min(1024, (g->N + 255) / 256)), 256, 0, st>>>(p->a, 0);
  return SNC_B200_OK;
}

}  // namespace sncb

struct snc_b200_part : sncb::Part {};

using namespace sncb;

extern "C" {

int snc_b200_part_create(const snc_b200_graph* g, const snc_b200_inputs* in, int32_t block_lo,
                         int32_t block_hi, const snc_lif* lif, snc_b200_part** out) {
  if (!g || !in || !lif || !out) { set_error("null argument"); return SNC_B200_EINVAL; }
  *out = nullptr;
  auto* p = new snc_b200_part();
  const int rc = part_create(g, in, block_lo, block_hi, lif, p);
  if (rc) {
    free_run(&p->run);
    delete p;
    return rc;
  }
  *out = p;
  return SNC_B200_OK;
}

int snc_b200_part_release(snc_b200_part* p) {
  if (!p) return SNC_B200_OK;
  free_run(&p->run);
  delete p;
  return SNC_B200_OK;
}

int snc_b200_part_integrate(snc_b200_part* p, int32_t t, uint32_t* mask, void* stream) {
  if (!p) { set_error("null partition"); return SNC_B200_EINVAL; }
  return part_integrate(p, t, mask, static_cast<cudaStream_t>(stream));
}

int snc_b200_part_deliver(snc_b200_part* p, int32_t t, const uint32_t* mask, void* stream) {
  if (!p || !mask) { set_error("null argument"); return SNC_B200_EINVAL; }
  const int T = p->run.in->steps_h[0];
  if (t < 0 || t >= T) { set_error("partition: step outside the sample"); return SNC_B200_EINVAL; }
  return part_deliver(p, t, mask, static_cast<cudaStream_t>(stream));
}

int snc_b200_part_fetch(snc_b200_part* p, float* logits, int64_t* spikes, int64_t* events,
                        uint32_t* raster, float* v_final) {
  if (!p) { set_error("null partition"); return SNC_B200_EINVAL; }
  SNCB_CUDA(cudaDeviceSynchronize());
  int err = 0;
  SNCB_CUDA(cudaMemcpy(&err, p->run.err, 4, cudaMemcpyDeviceToHost));
  if (err) { set_error("device error word set"); return err < 0 ? err : SNC_B200_ECUDA; }
  const Graph* g = p->run.g;
  if (logits && g->noc) {
    std::vector<int> c(g->noc);
    SNCB_CUDA(cudaMemcpy(c.data(), p->run.counts, (size_t)g->noc * 4, cudaMemcpyDeviceToHost));
    for (int k = 0; k < g->noc; ++k) logits[k] = (float)c[k];
  }
  unsigned long long sp = 0, ev = 0;
  SNCB_CUDA(cudaMemcpy(&sp, p->run.spikes, 8, cudaMemcpyDeviceToHost));
  SNCB_CUDA(cudaMemcpy(&ev, p->run.events, 8, cudaMemcpyDeviceToHost));
  if (spikes) *spikes = (int64_t)sp;
  if (events) *events = (int64_t)ev;
  if (raster && p->run.in->raster_words)
    SNCB_CUDA(cudaMemcpy(raster, p->run.raster, (size_t)p->run.in->raster_words * 4, cudaMemcpyDeviceToHost));
  if (v_final) SNCB_CUDA(cudaMemcpy(v_final, p->run.vfinal, (size_t)g->N * 4, cudaMemcpyDeviceToHost));
  return SNC_B200_OK;
}

}  // extern "C"
