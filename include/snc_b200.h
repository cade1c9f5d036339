/*
 * snc_b200.h -- C ABI of the B200 (sm_100a) execution and training core for
 * the SNC spiking substrate.
 *
 * Plain pointers and sizes only.  Every entry point returns SNC_B200_OK (0) or
 * a negative snc_b200_status; no C++ exception crosses this boundary.  Unless
 * a function says "device pointers", every pointer is HOST memory and every
 * call is synchronous, like the reference's cuda::forward
 * (src/runtime/cuda_backend.cu:186-361 ends in cudaDeviceSynchronize).
 *
 * Reference interfaces this ABI replaces (paths inside blazer502/snc):
 *   snc::cuda::available / snc::cuda::forward   include/snc/runtime.hpp:61-69
 *   snc::forward + Backend names                include/snc/runtime.hpp:21-31,57-58
 *   snc::cudatrain::*                           include/snc/cuda_trainer.hpp:26-57
 *   python/snc SNN / SurrogateSpike (BPTT)      python/snc/model.py:17-72
 */
#ifndef SNC_B200_H_
#define SNC_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SNC_B200_ABI_VERSION 1

typedef enum {
  SNC_B200_OK = 0,
  SNC_B200_EINVAL = -1,       /* bad argument or invalid graph */
  SNC_B200_ENODEV = -2,       /* no usable sm_100 device */
  SNC_B200_ENOMEM = -3,       /* device allocation failed */
  SNC_B200_ECUDA = -4,        /* CUDA runtime error (see snc_b200_last_error) */
  SNC_B200_ETIMEOUT = -5,     /* a bounded device wait gave up */
  SNC_B200_EUNSUPPORTED = -6, /* graph or config outside this backend's limits */
  SNC_B200_EOVERFLOW = -7     /* a device work buffer overflowed */
} snc_b200_status;

/* Read-only view of a reference SNNGraph (include/snc/snn_graph.hpp:43-77):
 * CSR over OUTGOING synapses, edges in insertion order within each row.
 * branch_ids is informational in the reference and not needed here. */
typedef struct {
  int32_t num_neurons;
  int32_t num_synapses;
  const int32_t* row_ptr;  /* [N+1] */
  const int32_t* post_ids; /* [S] */
  const float* weights;    /* [S] non-negative efficacy (sign on the pre) */
  const int32_t* delays;   /* [S] >= 1 */
  const uint8_t* role;     /* [N] 0 INTERNAL, 1 INPUT, 2 OUTPUT */
  const int8_t* sign;      /* [N] +1 / -1 */
  const int32_t* channel;  /* [N] input feature / output class, -1 otherwise */
} snc_graph_view;

/* InputEvent (include/snc/encoders.hpp:21-26), same 16-byte layout. */
typedef struct {
  int32_t sample_id;
  int32_t channel_id;
  int32_t time;
  float amplitude;
} snc_input_event;

/* LIFParams (include/snc/runtime.hpp:34-39) plus reset_mode:
 * 0 = v := reset after a spike (the reference), 1 = v := v - threshold. */
typedef struct {
  float threshold;
  float decay;
  float reset;
  int32_t refractory;
  int32_t reset_mode;
} snc_lif;

/* RunStats (include/snc/runtime.hpp:41-46).  overflow is set on an
 * SNC_B200_EOVERFLOW return (the reference declares it but never sets it). */
typedef struct {
  int64_t spikes;
  int64_t synaptic_events;
  int32_t overflow;
  double ms; /* device time of the step loop (CUDA events) */
} snc_run_stats;

/* Delivery strategies, the reference's cuda-atomic / cuda-bucket / cuda-sort
 * (src/runtime/cuda_backend.cu:1-14), re-designed:
 *   ATOMIC  warp-per-fired-row, coalesced CSR reads, red.add into the ring
 *   BUCKET  events binned by owning post block, accumulated by that block
 *   SORT    events applied per ring cell in (step, pre, edge) order: spike
 *           rasters and membrane potentials bit-identical to the serial CPU
 *           backend (cpu_backend.cpp:172-181)
 *   AUTO    chosen per graph by the built-in autotuner (cached per graph) */
enum {
  SNC_B200_MODE_ATOMIC = 0,
  SNC_B200_MODE_BUCKET = 1,
  SNC_B200_MODE_SORT = 2,
  SNC_B200_MODE_AUTO = 3
};

/* Execution paths for a batch of samples. */
enum {
  SNC_B200_PATH_PLAIN = 0,      /* per sample, one kernel launch per phase per step */
  SNC_B200_PATH_PERSISTENT = 1, /* all steps of all samples in one persistent launch */
  SNC_B200_PATH_AUTO = 2
};

typedef struct snc_b200_graph snc_b200_graph;   /* device-resident graph */
typedef struct snc_b200_inputs snc_b200_inputs; /* device-resident input schedule */
typedef struct snc_b200_run snc_b200_run;       /* device-resident results of one run */

/* ---- device and errors ----------------------------------------------------*/

/* 1 when a usable device of compute capability 10.x is present (replaces
 * snc::cuda::available, src/runtime/cuda_backend.cu:181-184). */
int snc_b200_available(void);
int snc_b200_abi_version(void);
/* Make `device` current for this host thread (the library links its own
 * CUDA runtime, so a framework's current-device setting does not reach it). */
int snc_b200_set_device(int device);
/* Text of the last error on this host thread ("" if none). */
const char* snc_b200_last_error(void);

/* ---- failure detection ---------------------------------------------------
 * No reference counterpart: the reference's GPU path has no device-side
 * waits and reports failure only by cuda::forward returning false
 * (src/runtime/cpu_backend.cpp:197-205).
 *
 * Wall-clock bound of every device-side spin wait (the grid barriers of the
 * all-SM forward and of the BPTT kernels) for launches made from now on, in
 * nanoseconds; 0 restores the default of 2 s.  A wait that runs out makes
 * every block of the launch return, and the call reports SNC_B200_ETIMEOUT;
 * the context stays usable.  Process-wide. */
int snc_b200_set_wait_limit(uint64_t ns);
/* Test hook: the next `n` launches that contain grid barriers (all-SM
 * forward, BPTT forward / backward) wait at their barriers for one arrival
 * that no block makes, so every such wait runs out after the wait limit and
 * the launch reports SNC_B200_ETIMEOUT.  Nothing faults; the next launch
 * without a pending stall runs normally.  Process-wide. */
int snc_b200_inject_stall(int32_t n);
/* Test hook: allow `after` more device allocations of this library, then
 * fail every further one with SNC_B200_ENOMEM (after < 0: never fail).  The
 * environment variable SNC_B200_FAIL_ALLOC sets the initial value, so a
 * process that cannot call this (the reference's CLIs linked with the
 * adapter) can still be made to take its CPU fallback.  Process-wide. */
int snc_b200_inject_alloc_failure(int64_t after);
/* Measurement: the rate (reductions per second) at which this GPU completes
 * float reductions to scattered addresses of a buffer of `n_slots` floats --
 * `n_ops` reductions from an all-SM grid, each warp's lanes on unrelated
 * words, the second of two launches timed.  The denominator of the ATOMIC
 * delivery mode's roofline (one reduction per synaptic event into the delay
 * ring, the reference's k_step delivery, src/runtime/cuda_backend.cu:71-75);
 * no reference counterpart of its own. */
int snc_b200_probe_red_rate(int64_t n_slots, int64_t n_ops, double* reds_per_s);

/* ---- graph ----------------------------------------------------------------*/

/* Validate (as SNNGraph::validate, src/graph/snn_graph.cpp:30-56) and upload a
 * graph once; the reference re-uploads per call (cuda_backend.cu:247-285).
 * Limits: N < 2^24, max delay <= 255. */
int snc_b200_graph_upload(const snc_graph_view* g, snc_b200_graph** out);
int snc_b200_graph_release(snc_b200_graph* g);
/* Upload a graph from the bytes of an SNCG file (the format snc_export
 * writes, src/bench/snc_export.cpp:107-123, read by python/snc/graph.py:
 * 11-24; pre[] in CSR order), optionally followed by the weights section
 * 'SNCW', S, weights[S] fp32, sign[N] int32 that the reference's readers
 * ignore (without it every weight is 1 and every sign +1).  The image is
 * copied to the device once and its edges are checked, counted and packed
 * there; the same validation and limits as snc_b200_graph_upload apply. */
int snc_b200_graph_upload_sncg(const void* data, size_t bytes, snc_b200_graph** out);

/* Generate a grid graph on the device (no reference counterpart: the
 * reference builds every graph on the host; this is the benchmark's large
 * recurrent substrate built where it runs).  N = width x height neurons on a
 * torus (id = y * width + x), out_degree synapses per neuron: out_degree -
 * long_range local targets at a displacement of standard deviation sigma
 * per axis (an Irwin-Hall(4) variate), candidate j kept with probability
 * accept[j] / 2^32 (the in-degree skew; from draw max_draws on every
 * candidate is kept, 0 = 1000 x out_degree), then long_range targets uniform
 * over all neurons; weights w_std x an Irwin-Hall(4) variate, delays uniform
 * in 1..max_delay.  Every draw is a Philox-4x32-10 word keyed by seed and
 * counted by (neuron, draw, stream) and every derived value is integer
 * arithmetic or one correctly rounded float operation, so the graph is the
 * same on any host (snc_b200.workloads.grid_graph_host builds it with
 * numpy).  role, sign, channel [N] as in snc_graph_view. */
typedef struct {
  int32_t width, height;
  int32_t out_degree, long_range;
  float sigma, w_std;
  int32_t max_delay; /* <= 255 */
  int32_t max_draws;
  uint64_t seed;
} snc_grid_graph;
int snc_b200_graph_generate_grid(const snc_grid_graph* p, const uint32_t* accept, const uint8_t* role,
                                 const int8_t* sign, const int32_t* channel, snc_b200_graph** out);
/* Basic shape: N, S, ring length, output channels, input channels. */
int snc_b200_graph_info(const snc_b200_graph* g, int32_t* n, int32_t* s, int32_t* ring_len,
                        int32_t* n_out, int32_t* n_in);
/* Copies the device layout of an uploaded graph back (no counterpart in the
 * reference; for checking it): edges and gedges [S] as (ring column | delay
 * << 24, float bits of sign * weight) pairs, gptr [N+1], groups [G] as
 * (destination block, first gedge) pairs, col_of [N], colbase and ibase
 * [P+1]; block_size and num_blocks receive BS and P, num_groups G.  Any
 * pointer may be NULL. */
int snc_b200_graph_layout(const snc_b200_graph* g, uint32_t* edges, uint32_t* gedges, int32_t* gptr,
                          int32_t* groups, int32_t* col_of, int32_t* colbase, int32_t* ibase,
                          int32_t* block_size, int32_t* num_blocks, int32_t* num_groups);

/* ---- inputs ----------------------------------------------------------------
 * Build the per-step injection schedule of a batch of samples on the host
 * (channel -> INPUT neurons, cpu_backend.cpp:43-65; the drive of one neuron at
 * one step is summed in event order) and upload it.  events[k].sample_id picks
 * the sample in [0, num_samples); steps[b] is sample b's step count. */
int snc_b200_inputs_upload(const snc_b200_graph* g, const snc_input_event* events,
                           size_t n_events, int32_t num_samples, const int32_t* steps,
                           snc_b200_inputs** out);
int snc_b200_inputs_release(snc_b200_inputs* in);

/* Input encoders (include/snc/encoders.hpp:21-45, src/training/encoders.cpp:25-71)
 * run on the device: the schedule of a batch built straight from its
 * features [num_samples][n_channels] (host, row-major), sample b spanning
 * steps[b] steps; only the features and step counts are copied.  Encoders as
 * the reference's enum: direct (every step, amplitude v * gain) and latency
 * (one spike at lround((T-1) * (1 - min(1, v)))) give exactly the schedule of
 * the reference's encode() events; poisson keeps the rule u < min(1, v *
 * max_rate) with amplitude gain but draws u from Philox-4x32-10 (Salmon et al.,
 * SC 2011) keyed by seed and counted by (step / 4, channel, sample): the same
 * statistics as encode(), not the same draws.  Channels with v <= threshold
 * emit nothing. */
#define SNC_B200_ENCODER_DIRECT 0
#define SNC_B200_ENCODER_POISSON 1
#define SNC_B200_ENCODER_LATENCY 2
int snc_b200_inputs_encode(const snc_b200_graph* g, int32_t encoder, const float* features,
                           int32_t n_channels, int32_t num_samples, const int32_t* steps,
                           float gain, float max_rate, float threshold, uint64_t seed,
                           snc_b200_inputs** out);
/* Bytes the schedule occupies on the device (= bytes copied host to device). */
int snc_b200_inputs_info(const snc_b200_inputs* in, int64_t* device_bytes, int64_t* entries);
/* Copies the schedule back (no counterpart in the reference; for checking
 * it): sched_ptr [total steps + num_samples] (sample b's step t starts at
 * sched_ptr[stepbase_b + b + t], its closing entry follows its last step),
 * neuron and drive [entries]: per step the driven input neurons in ascending
 * id and their amplitudes summed in event order.  Any pointer may be NULL. */
int snc_b200_inputs_read(const snc_b200_inputs* in, int32_t* sched_ptr, int32_t* neuron, float* drive);

/* ---- run --------------------------------------------------------------------
 * Run a batch on the device without host synchronisation.  stream is a
 * cudaStream_t (NULL = the legacy default stream).  flags: */
enum {
  SNC_B200_RUN_RASTER = 1, /* keep spike rasters (bit per neuron per step) */
  SNC_B200_RUN_VFINAL = 2, /* keep final membrane potentials */
  SNC_B200_RUN_GRAPH = 4,  /* persistent path: launch through a captured CUDA graph */
  SNC_B200_RUN_FORCE_GRID = 8 /* persistent path: use the all-SM tier even when one
                                 sample fits in one CTA (tuning and tests) */
};
int snc_b200_run_create(const snc_b200_graph* g, const snc_b200_inputs* in, int flags,
                        snc_b200_run** out);
int snc_b200_run_release(snc_b200_run* r);
/* Execute (or re-execute) the run: state is reset, results overwritten. */
int snc_b200_run_launch(snc_b200_run* r, const snc_lif* lif, int mode, int path, void* stream);
/* Wait for the run and copy results to host arrays (any may be NULL):
 *   logits [B][n_out], spikes [B], events [B], raster [sum_b steps[b]][ceil(N/32)]
 *   (sample-major), v_final [B][N], stats (totals; ms = device time of the
 *   last launch). */
int snc_b200_run_fetch(snc_b200_run* r, float* logits, int64_t* spikes, int64_t* events,
                       uint32_t* raster, float* v_final, snc_run_stats* stats);
/* Leaky readout units (the readout of python/snc/shd_model.py:139-140,147
 * on the substrate): with ro_decay >= 0 every OUTPUT neuron that has a
 * channel stops spiking and integrates v = ro_decay * v + drive + delivered
 * input (each product and sum rounded separately), and run_fetch's logits
 * become, per channel, the sum over its readout units in ascending id of
 * their potential after the sample's last step divided by its step count.
 * ro_decay < 0 turns them off (spike-count logits, the default).  Applies to
 * this run's following launches on every path. */
int snc_b200_run_set_readout(snc_b200_run* r, float ro_decay);
/* The mode and path the last launch actually used (after AUTO resolution). */
int snc_b200_run_used(const snc_b200_run* r, int* mode, int* path);
/* 1 when the last launch went through the captured CUDA graph, 0 when it was
 * launched directly (no SNC_B200_RUN_GRAPH, plain path, or capture refused). */
int snc_b200_run_used_graph(const snc_b200_run* r);

/* ---- one-call forward (the reference's cuda::forward, runtime.hpp:66-68) ---
 * One sample: events are that sample's InputEvents (sample_id ignored);
 * logits [n_out].  Uses the plain path, like the reference backend.  The
 * graph is uploaded and released inside the call when `graph` is NULL and
 * `view` is given; pass an uploaded handle to avoid that. */
int snc_b200_forward(const snc_b200_graph* graph, const snc_graph_view* view,
                     const snc_input_event* events, size_t n_events, int32_t num_steps,
                     const snc_lif* lif, int mode, float* logits, snc_run_stats* stats);

/* Batched forward through the persistent path: many samples with uneven step
 * counts in one launch.  logits [B][n_out]; spikes / events [B] may be NULL. */
int snc_b200_forward_batched(const snc_b200_graph* graph, const snc_input_event* events,
                             size_t n_events, int32_t num_samples, const int32_t* steps,
                             const snc_lif* lif, int mode, float* logits, int64_t* spikes,
                             int64_t* events_out, snc_run_stats* stats);

/* ---- post-neuron partitions ----------------------------------------------------
 * One sample's forward split by post neuron across devices (the optional
 * partitioned mode of a graph too large for one device; the reference runs
 * one sample on one device, src/runtime/cuda_backend.cu:186-361).  A
 * partition owns neuron blocks [block_lo, block_hi) of the graph's block
 * partition (snc_b200_graph_layout's block_size / num_blocks): their state
 * and delay-ring columns; every rank keeps the whole graph.  Per step t:
 *   snc_b200_part_integrate  integrates the partition's neurons and writes
 *       their spike bits into words [block_lo * BS / 32, block_hi * BS / 32)
 *       of mask (DEVICE, ceil(N / 32) words; may be NULL);
 *   the caller makes every partition's words available in every rank's
 *       mask (an all-gather of the step's spike bits: 12.5 KB for 100k
 *       neurons);
 *   snc_b200_part_deliver  delivers every fired neuron's synapses into the
 *       partition's columns in the serial CPU backend's (pre, edge) order.
 * The ranks' results together equal one device's SORT run bit for bit.
 * in holds one sample; lif as in snc_b200_run_launch.  fetch: logits (the
 * partition's output spikes), spikes and events of the partition's neurons,
 * the raster [T][ceil(N/32)] with the partition's bits, v_final [N] (valid
 * for the partition's neurons).  Calls are ordered on `stream`. */
typedef struct snc_b200_part snc_b200_part;
int snc_b200_part_create(const snc_b200_graph* g, const snc_b200_inputs* in, int32_t block_lo,
                         int32_t block_hi, const snc_lif* lif, snc_b200_part** out);
int snc_b200_part_release(snc_b200_part* p);
int snc_b200_part_integrate(snc_b200_part* p, int32_t t, uint32_t* mask, void* stream);
int snc_b200_part_deliver(snc_b200_part* p, int32_t t, const uint32_t* mask, void* stream);
int snc_b200_part_fetch(snc_b200_part* p, float* logits, int64_t* spikes, int64_t* events,
                        uint32_t* raster, float* v_final);

/* ---- launch shapes and the delivery autotuner ---------------------------------
 * No reference counterpart: the reference picks its backend by a flag
 * (src/bench/snc_bench.cpp:301-317).
 *
 * A launch's shape on the persistent path: tier 0 runs one sample per CTA
 * with the sample's whole state in shared memory (when it fits), tier 1 runs
 * every SM on a wave of samples in lockstep; on tier 1, block_threads threads
 * per block (a multiple of 32 in [512, 768]), wave samples per wave and the
 * delay-ring slices in shared (ring_smem 1) or global (0) memory.  -1 / 0 in
 * a field: chosen automatically.  ms is filled by the autotuner. */
typedef struct {
  int32_t mode;          /* SNC_B200_MODE_ATOMIC / _BUCKET / _SORT */
  int32_t path;          /* SNC_B200_PATH_PLAIN / _PERSISTENT */
  int32_t tier;          /* persistent path: 0 sample per CTA, 1 all SMs; -1 automatic */
  int32_t block_threads; /* tier 1: threads per block; 0 automatic */
  int32_t wave;          /* tier 1: samples in lockstep; 0 as many as fit */
  int32_t ring_smem;     /* tier 1 (bucket, sort): 1 shared, 0 global; -1 automatic */
  float ms;              /* autotuner: device time of the candidate's timed launch */
} snc_launch_config;

/* Fix the shape of this run's launches (mode and path of cfg are only used to
 * check it; they stay arguments of snc_b200_run_launch).  NULL: back to
 * automatic.  SNC_B200_EUNSUPPORTED for a shape the graph or device cannot
 * take (tier 0 when a sample does not fit one CTA, ring slices that do not
 * fit). */
int snc_b200_run_configure(snc_b200_run* r, const snc_launch_config* cfg);

/* Time every candidate on this graph and these inputs: each delivery mode on
 * the plain path (batches of at most 8 samples), on tier 0 (atomic and sort,
 * when a sample fits one CTA) and on tier 1 over block_threads {the block's
 * neuron count rounded to 32, 512, 768}, wave {as many as fit, 1 (batches of
 * 2-64)} and ring placement {shared, global} (bucket, sort); batches above 64
 * samples time tier 1 in its default shape only.  Each candidate is launched
 * twice and its second device time kept.  The fastest is cached under the
 * graph's content hash and the batch's sample and step counts, and AUTO
 * launches with that key use its mode, path and shape.  cand[0 .. max_cand)
 * receives the candidates, *n_cand their number, *best the winner's index
 * (any may be NULL). */
int snc_b200_autotune_ex(const snc_b200_graph* g, const snc_b200_inputs* in, const snc_lif* lif,
                         snc_launch_config* cand, int32_t max_cand, int32_t* n_cand, int32_t* best);
/* snc_b200_autotune_ex returning the winner's mode, path and threads per
 * block (1024 for tier 0, 512 for the plain path). */
int snc_b200_autotune(const snc_b200_graph* g, const snc_b200_inputs* in, const snc_lif* lif,
                      int* mode, int* path, int* block_threads);
/* 1 and the cached winner in *out when this graph and batch shape were tuned,
 * 0 otherwise. */
int snc_b200_autotune_lookup(const snc_b200_graph* g, const snc_b200_inputs* in, snc_launch_config* out);

/* ---- minibatch e-prop (replaces snc::cudatrain, cuda_trainer.hpp:26-57) ----
 * The learning rule of src/training/cuda_trainer.cu: LIF + triangular
 * surrogate psi = gamma * max(0, 1 - |v - thr| / thr), pre trace
 * tr = d * tr + (1 - d) * spike, eligibility E[b,s] += psi[post] * tr[pre]
 * every step, then softmax(spike counts) - onehot(label), learning signal L
 * (delta for OUTPUT neurons, feedback matrix . delta for INTERNAL ones) and
 * w -= lr * mean_b(L[b,post] * E[b,s] / T_b), clamped to +-w_max.  Inputs are
 * InputEvents (the caller encodes, as the CPU Trainer does) instead of cuRAND
 * draws; samples of one minibatch may have different step counts. */
typedef struct {
  float lr;              /* TrainConfig::lr */
  float w_max;           /* TrainConfig::w_max */
  float surrogate_scale; /* TrainConfig::surrogate_scale (gamma) */
  float trace_decay;     /* pre-trace decay; the reference uses lif.decay */
  int32_t train_hidden;  /* TrainConfig::train_hidden */
  int32_t mode;          /* delivery: SNC_B200_MODE_SORT (bit-exact) or _ATOMIC */
} snc_eprop_cfg;

typedef struct snc_b200_eprop snc_b200_eprop; /* cudatrain::CudaTrainSession */

/* cudatrain::create: weights [S] (signed, CSR order) and the feedback matrix
 * [n_internal][max(1, n_out)] (one row per INTERNAL neuron, ascending id) are
 * supplied by the caller; max_batch bounds the samples of one minibatch. */
int snc_b200_eprop_create(const snc_b200_graph* g, const snc_lif* lif, const snc_eprop_cfg* cfg,
                          int32_t max_batch, const float* weights, const float* feedback,
                          snc_b200_eprop** out);
/* Which forward a session runs: SNC_B200_PATH_PLAIN when one sample's state
 * fits one CTA (the sample-per-CTA kernel), SNC_B200_PATH_PERSISTENT when it
 * does not (the all-SM kernel on a destination-grouped copy of the weights). */
int snc_b200_eprop_path(const snc_b200_eprop* s);
int snc_b200_eprop_release(snc_b200_eprop* s);                    /* cudatrain::destroy */
int snc_b200_eprop_set_weights(snc_b200_eprop* s, const float* w); /* [S] */
int snc_b200_eprop_get_weights(snc_b200_eprop* s, float* w);       /* [S] */
/* One minibatch (cuda_trainer.cu run_batch, :304-350): events with sample_id
 * in [0, B), steps [B], labels [B].  train = 0 runs the forward only (no
 * eligibility, no update, no statistics).  counts [B][n_out] may be NULL. */
int snc_b200_eprop_batch(snc_b200_eprop* s, const snc_input_event* events, size_t n_events,
                         int32_t num_samples, const int32_t* steps, const int32_t* labels,
                         int train, float* counts, snc_run_stats* stats);
/* Data-parallel e-prop.  snc_b200_eprop_gradient runs a training minibatch
 * but, instead of updating the weights, writes grad[s] = sum_b L[b,post(s)] *
 * E[b,s] / T_b over this call's samples into `grad` (DEVICE pointer, [S]
 * fp32).  snc_b200_eprop_apply then sets w = clamp(w - lr * grad /
 * total_batch, +-w_max).  Summing the gradients of disjoint sample shards
 * (one all-reduce) and applying once equals one minibatch over their union up
 * to the order of the float sum. */
int snc_b200_eprop_gradient(snc_b200_eprop* s, const snc_input_event* events, size_t n_events,
                            int32_t num_samples, const int32_t* steps, const int32_t* labels,
                            float* grad, float* counts, snc_run_stats* stats);
int snc_b200_eprop_apply(snc_b200_eprop* s, const float* grad, int32_t total_batch);
/* Eligibility [B][S] of the last training minibatch. */
int snc_b200_eprop_get_eligibility(snc_b200_eprop* s, float* elig);
/* cudatrain::reset_stats / collect_stats: per-synapse deliveries [S] and
 * per-neuron firings [N] accumulated over training minibatches. */
int snc_b200_eprop_reset_stats(snc_b200_eprop* s);
int snc_b200_eprop_collect_stats(snc_b200_eprop* s, int64_t* syn_deliveries, int64_t* neuron_fires);

/* ---- connectome: the co-training loop's structural state (replaces
 * snc::Connectome, include/snc/connectome.hpp:58-101, for the loop of
 * src/training/cotrain_main.cpp:271-283) -------------------------------------
 * A layered edge list with per-edge ages kept on the device as a CSR (rows in
 * the reference's adjacency order), pruned and regrown there by
 * snc_b200_connectome_update and turned into a device graph without a host
 * round trip.  Random draws (initial jitter, fallback growth) come from the
 * host's std::mt19937_64 through the same library distributions as the
 * reference, so a connectome made here from the same seed evolves as the
 * reference's does; one documented difference: among eligible synapses of
 * equal |weight| at the K-th place the lowest CSR positions are pruned
 * (std::nth_element leaves that choice to the library). */
typedef struct snc_b200_connectome snc_b200_connectome;

typedef struct {                /* StructConfig, connectome.hpp:33-48 */
  int32_t grow_per_epoch;
  int32_t delay;
  float w_grow_init;
  float locality_window;
  int32_t protect_rounds;
  int32_t max_attempts_mult;
  int32_t reward_modulated;
  float reward_chance;
  float reward_floor;
} snc_struct_config;

typedef struct {                /* StructReport, connectome.hpp:50-54 */
  int32_t pruned;
  int32_t grown;
  int32_t synapses;
} snc_struct_report;

/* Connectome::layered_local (connectome.cpp:14-62). */
int snc_b200_connectome_layered_local(const int32_t* layers, int32_t num_layers,
                                      int32_t synapse_budget, int32_t delay, float w_init,
                                      uint64_t seed, snc_b200_connectome** out);
int snc_b200_connectome_release(snc_b200_connectome* c);
int snc_b200_connectome_info(const snc_b200_connectome* c, int32_t* num_neurons,
                             int32_t* num_synapses);
/* to_graph()'s CSR (row_ptr [N+1], post, delay), edge_weights() (signed,
 * the same order) and the structural ages; NULL arrays are skipped. */
int snc_b200_connectome_read(const snc_b200_connectome* c, int32_t* row_ptr, int32_t* post,
                             int32_t* delay, float* weight, int32_t* age);
/* set_edge_weights (connectome.cpp:112-119): the first n weights in CSR
 * order, the rest unchanged. */
int snc_b200_connectome_set_weights(snc_b200_connectome* c, const float* w, int64_t n);
/* structural_update (connectome.cpp:121-219): prune the K weakest eligible
 * synapses (K from grow_per_epoch, reward-modulated if asked), regrow one
 * local synapse per freed post from the most active unconnected pre in its
 * window, then fallback growth onto under-driven random posts, then age every
 * synapse.  neuron_fires [n_fires] are the inner loop's firing counts
 * (snc_b200_eprop_collect_stats). */
int snc_b200_connectome_update(snc_b200_connectome* c, const int64_t* neuron_fires, int64_t n_fires,
                               const snc_struct_config* cfg, float reward, snc_struct_report* out);
/* to_graph (connectome.cpp:84-101) on the device: |weight|, sign +1, the
 * layers' roles and channels. */
int snc_b200_connectome_graph(const snc_b200_connectome* c, snc_b200_graph** out);

/* ---- surrogate-gradient BPTT (replaces the autograd unrolling of the bridge,
 * python/snc/model.py:52-72, with the per-synapse delays of
 * python/snc/shd_model.py:109-121) -------------------------------------------
 * Graph: CSR over outgoing synapses (row_ptr [N+1], post [S], delays [S]).
 * All tensors are DEVICE pointers, batch innermost: ext / spikes / grads are
 * [T][N][B] fp32, weights [S] in CSR order.  Calls are ordered on `stream`
 * (a cudaStream_t) and return after it has drained; one handle must not be
 * used from two streams at once (it owns the workspaces).
 *   forward:  v = decay*v + sum_e w_e s_pre(t - d_e) + ext; s = H(v - thr)
 *             (smooth != 0: s = x / (1 + slope |x|)); v = v * (1 - s).
 *             Saves spike_bits [T][N][ceil(B/32)] and v_saved: with
 *             ckpt_every = K > 0, v after every K-th step ([ceil(T/K)][N][B]),
 *             with K = 0 the pre-reset potential of every step ([T][N][B]).
 *   backward: fast-sigmoid surrogate 1 / (1 + slope |x|)^2; grad_w [S] is
 *             overwritten, grad_ext may be NULL.  Recomputes each K-step
 *             segment from the checkpoints when K > 0. */
typedef struct snc_b200_bptt snc_b200_bptt;
int snc_b200_bptt_create(int32_t num_neurons, int32_t num_synapses, const int32_t* row_ptr,
                         const int32_t* post, const int32_t* delays, snc_b200_bptt** out);
int snc_b200_bptt_release(snc_b200_bptt* h);
int snc_b200_bptt_forward(snc_b200_bptt* h, const float* w, const float* ext, int32_t T, int32_t B,
                          float threshold, float decay, float slope, int32_t ckpt_every,
                          int32_t smooth, float* spikes, uint32_t* spike_bits, float* v_saved,
                          void* stream);
int snc_b200_bptt_backward(snc_b200_bptt* h, const float* w, const float* ext, int32_t T, int32_t B,
                           float threshold, float decay, float slope, int32_t ckpt_every,
                           int32_t smooth, const float* spikes, const uint32_t* spike_bits,
                           const float* v_saved, const float* grad_spikes, float* grad_w,
                           float* grad_ext, void* stream);
/* Resident launches (default on): when one warp per neuron fits on the device
 * and no neuron has more than 256 incoming or outgoing synapses, forward and
 * backward stage every neuron's edges in shared memory for the whole launch
 * and accumulate the weight gradients there; results are bit-identical to the
 * global-memory form, which enable = 0 selects.  No reference counterpart
 * (a tuning switch of this backend). */
int snc_b200_bptt_set_resident(snc_b200_bptt* h, int32_t enable);
/* Leaky integration along time (the leaky readouts of python/snc/shd_model.py:
 * 139-140 and python/snc/lm.py:90 as one kernel): x, y [T][n] fp32 device
 * tensors, y[t] = decay * y[t-1] + x[t] with y[-1] = 0, or with reverse != 0
 * y[t] = decay * y[t+1] + x[t] from the last step (the gradient); the product
 * and the sum are rounded separately, as the step loop does.  x and y must not
 * overlap.  Asynchronous on stream. */
int snc_b200_leaky_scan(const float* x, float* y, int32_t T, int64_t n, float decay, int32_t reverse,
                        void* stream);
/* Layout change between torch's [T][B][N] and the batch-innermost [T][N][B]
 * of the BPTT kernels: out[t][i][j] = in[t * st_t + i + j * st_j] (element
 * strides; unit stride along i), out contiguous [T][I][J]; T <= 65535.
 * Data movement only.  Asynchronous on stream.  No reference counterpart (the
 * reference bridge keeps torch's layout). */
int snc_b200_transpose(const float* in, float* out, int32_t T, int32_t I, int32_t J, int64_t st_t,
                       int64_t st_j, void* stream);

/* The BPTT forward for callers that cannot allocate device memory when they
 * call it (no counterpart in the reference, which allocates inside every GPU
 * call): a framework whose caching allocator owns all of the device's memory,
 * so that an allocation behind its back can fail or starve it, and a
 * real-time loop that must not pay cudaMalloc's latency or risk its failure
 * mid-run.  Same arguments, launch and results as snc_b200_bptt_forward; the
 * caller still provides every input and output buffer, and the call makes no
 * cudaMalloc / cudaFree.  Like snc_b200_bptt_forward it returns after reading
 * the kernel's error word back and waiting for `stream`.
 * Its scratch -- the membrane state of num_neurons x B samples and the
 * barrier / error words -- is one static 4 MiB array per device that every
 * device loading the library keeps until exit, so num_neurons * B must not
 * exceed 1,048,512 (SNC_B200_EUNSUPPORTED otherwise).  All calls share that
 * array: calls whose work overlaps on the GPU (different streams, threads or
 * handles without ordering) race and must not be issued.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) and
 * caches it; make that first call before any stream capture. */
int snc_b200_bptt_forward_static(snc_b200_bptt* h, const float* w, const float* ext, int32_t T,
                                 int32_t B, float threshold, float decay, float slope,
                                 int32_t ckpt_every, int32_t smooth, float* spikes,
                                 uint32_t* spike_bits, float* v_saved, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SNC_B200_H_ */
