/*
 * lpa_capi.h -- C ABI of the B200 label-propagation library (liblpa_b200.so).
 *
 * One synchronous label-propagation iteration over a CGR-compressed graph,
 * run by hand-written sm_100a kernels.  Plain pointers and sizes only; every
 * call returns an lpa_status and no exception crosses the boundary.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   - the propagator classes NovaPlusPropagator / NovaPropagator /
 *     CGLPPropagator: run(), iterate(), get_labels(), preprocess(),
 *     transfer_data() (baselines/novaplus/novaplus_propogator.cuh:100-199,
 *     :340-373; baselines/cglp/cglp_propagator.cuh:205-335;
 *     include/label_propagator.h:26-33);
 *   - the kernels they launch (baselines/novaplus/kernel.cuh:14-191,
 *     include/decoder.cuh:50-1025) -- reached only through these entry points;
 *   - the GPU decompress test harness (include/decompressor.cuh:116-144,
 *     test/decompress_test.cu:42-79) -> lpa_decode_csr;
 *   - the CPU format layer (src/compressor.cpp, src/file.cpp) -> lpa_hg_*.
 *
 * Ownership: host buffers passed in are copied; the caller keeps them.
 * Device memory belongs to the handle.  Threading: a handle is not
 * thread-safe; separate handles may be used from separate threads.
 */
#ifndef LPA_CAPI_H
#define LPA_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lpa_handle lpa_handle; /* one device-resident graph (propagator) */
typedef struct lpa_batch lpa_batch;   /* many graphs propagated together */

typedef enum lpa_status {
  LPA_OK = 0,
  LPA_ERR_CUDA = 1,        /* a CUDA runtime call failed */
  LPA_ERR_OOM = 2,         /* a device allocation failed */
  LPA_ERR_BAD_STREAM = 3,  /* the decoder left a vertex's bit range, or an id >= n */
  LPA_ERR_TIMEOUT = 4,     /* a bounded device wait gave up */
  LPA_ERR_INVALID_ARG = 5, /* bad pointer, size or option */
  LPA_ERR_IO = 6,          /* a file is missing or malformed */
  LPA_ERR_NO_DEVICE = 7,   /* no usable CUDA device */
  LPA_ERR_CAPACITY = 8     /* a work item exceeded a planned capacity (internal) */
} lpa_status;

/* Kernel variants.  All of them produce identical labels. */
typedef enum lpa_variant {
  LPA_VARIANT_WARP = 0,     /* V1: warp per vertex (degree <= 256)              */
  LPA_VARIANT_PACKED = 1,   /* V2: several vertices per warp (degree <= 32)     */
  LPA_VARIANT_BLOCK = 2,    /* V3: block per vertex                             */
  LPA_VARIANT_TWO_PASS = 3  /* V4: decode to a CSR scratch, then propagate      */
} lpa_variant;

typedef enum lpa_dispatch {
  LPA_DISPATCH_FIXED = 0,   /* degree buckets: <16 packed, <128 warp, >=128 block */
  LPA_DISPATCH_LEARNED = 1, /* MLP cost model over segment features, judged by FIXED */
  LPA_DISPATCH_FORCE = 2    /* force_variant wherever it is capable, FIXED elsewhere */
} lpa_dispatch;

/* The compressed mixed graph: the content of the reference's .graph, .offset,
 * .vertices.bin, .graph.small.bin and .offset.small.bin files (File::
 * load_graph, src/file.cpp:24-74), with 64-bit bit offsets. */
typedef struct lpa_graph_desc {
  uint64_t num_vertices;        /* n = number of positions in vertices[] */
  uint64_t num_compressed;      /* n_c: positions [0, n_c) are in the bitstream */
  const uint32_t *words;        /* bitstream as big-endian 32-bit words (File::graph) */
  uint64_t num_words;
  const uint64_t *offsets;      /* n_c + 1 bit offsets, offsets[0] = 0 */
  const uint32_t *vertices;     /* position -> vertex id, n entries */
  const uint32_t *small_graph;  /* neighbours of positions >= n_c (CSR) */
  uint64_t num_small_arcs;
  const uint32_t *small_offset; /* n - n_c + 1 entries; NULL when n == n_c */
} lpa_graph_desc;

typedef struct lpa_opts {
  int device;              /* CUDA device ordinal */
  uint32_t cms_threshold;  /* degree >= this uses the count-min sketch; 0: never */
  uint64_t cms_seed;       /* seeds the sketch's row hashes */
  int dispatch;            /* lpa_dispatch */
  int force_variant;       /* lpa_variant, with LPA_DISPATCH_FORCE */
  void *stream;            /* cudaStream_t to run on; NULL: the handle makes one */
  int record_timings;      /* 1: per-launch events; 2: also per-segment device cycles */
  int verbose;             /* per-iteration log lines on stdout */
  int batch_mode;          /* lpa_batch_mode, for lpa_batch_create */
  /* LPA_BATCH_QUEUE: how many times (about 200 ns each) a block of the
   * persistent kernel looks at an empty queue slot, while graphs are still
   * running, before it gives up and the run returns LPA_ERR_TIMEOUT.
   * 0: the default, 2^25 (about 7 s). */
  uint64_t queue_wait_limit;
  /* Out-of-core streaming (include/outofcore.cuh:10-96 streams CSR batches
   * the same way).  0: the whole compressed graph resides on the device.
   * Otherwise the bitstream stays in pinned host memory and every iteration
   * processes the compressed positions in ranges, each range's stream words
   * copied from host memory on a second stream while the previous range is
   * processed.  The ranges are cut so that two stream buffers (a quarter of
   * the budget each) and the two-pass label scratch (half) fit in this many
   * bytes; per-vertex arrays, labels and the small CSR stay resident.
   * LPA_ERR_CAPACITY when one vertex alone does not fit.  Single graphs only:
   * lpa_batch_create rejects it. */
  uint64_t stream_budget;
} lpa_opts;

typedef enum lpa_batch_mode {
  LPA_BATCH_LOCKSTEP = 0, /* the batch concatenated into one graph, run by one handle */
  LPA_BATCH_QUEUE = 1     /* one persistent launch fed by a device work queue */
} lpa_batch_mode;

typedef struct lpa_info {
  uint64_t num_vertices, num_compressed, num_arcs, num_small_arcs;
  uint64_t stream_bits;
  uint64_t num_segments;
  uint64_t max_degree;
  uint64_t bytes_algorithmic; /* one iteration's compulsory bytes (see lpa_info docs) */
  uint64_t device_bytes;      /* device memory held by the handle */
} lpa_info;

typedef struct lpa_stats {
  uint64_t iterations;              /* iterations run since lpa_init_labels */
  uint64_t last_changed;            /* changed count of the last iteration */
  double last_iter_ms;              /* device time of the last iteration */
  double variant_ms[4];             /* device time per variant, last iteration */
  uint64_t variant_segments[4];     /* segments assigned per variant */
  uint64_t variant_arcs[4];         /* arcs assigned per variant */
  double mlp_loss;                  /* last training loss of the cost model */
  uint64_t mlp_updates;             /* SGD steps taken */
  uint64_t dispatch_reverts;        /* times the learned plan was judged slower */
  int learned_active;               /* 1 when the learned plan is in use */
  uint64_t launches;                /* kernel launches enqueued by this handle */
  double decode_ms;                 /* two-pass decode kernel, last iteration */
  double iterate_ms;                /* persistent iteration kernel, last iteration */
  double count_ms;                  /* two-pass count kernel, last iteration */
  double packed_ms;                 /* lane-per-vertex kernel of the tiny bucket, last iteration */
  uint64_t stream_ranges;           /* out-of-core streaming: ranges per iteration (0: resident) */
  uint64_t stream_bytes;            /* out-of-core streaming: stream bytes copied to the device so far */
} lpa_stats;

/* ---------------------------------------------------------------- basics -- */
const char *lpa_status_str(lpa_status s);
const char *lpa_version(void);
void lpa_opts_default(lpa_opts *o);

/* --------------------------------------------------- propagator handle ---- */
/* Copies the graph to the device, derives every compressed vertex's degree by
 * decoding it once, and builds the dispatch plan.  Replaces
 * NovaPlusPropagator::preprocess / transfer_data
 * (baselines/novaplus/novaplus_propogator.cuh:201-204,340-373). */
lpa_status lpa_create(const lpa_graph_desc *g, const lpa_opts *o, struct lpa_handle **out);
lpa_status lpa_destroy(struct lpa_handle *h);
lpa_status lpa_get_info(struct lpa_handle *h, lpa_info *info);
const char *lpa_last_error(struct lpa_handle *h);

/* L[v] = v (initialize_labels, baselines/novaplus/kernel.cuh:57-64). */
lpa_status lpa_init_labels(struct lpa_handle *h);
/* Sets the current labels from host memory (n entries). */
lpa_status lpa_set_labels(struct lpa_handle *h, const uint32_t *host, size_t n);
/* One synchronous iteration; *changed_out (may be NULL) receives the number
 * of vertices whose label changed.  Replaces NovaPlusPropagator::iterate
 * (baselines/novaplus/novaplus_propogator.cuh:131-199). */
lpa_status lpa_iterate(struct lpa_handle *h, uint64_t *changed_out);
/* Runs up to max_iter iterations; with early_exit it stops after an iteration
 * that changed nothing (device-side test inside a CUDA graph).  Replaces
 * NovaPlusPropagator::run (baselines/novaplus/novaplus_propogator.cuh:100-129). */
lpa_status lpa_run(struct lpa_handle *h, int max_iter, int early_exit, int *iters_done);
/* Per-iteration changed counts of the last lpa_run (count entries). */
lpa_status lpa_get_changed_history(struct lpa_handle *h, uint64_t *out, size_t count);
/* Copies the current labels to host memory (n entries).  Replaces
 * LabelPropagator::get_labels (include/label_propagator.h:30-35). */
lpa_status lpa_get_labels(struct lpa_handle *h, uint32_t *host_out, size_t n);
lpa_status lpa_get_stats(struct lpa_handle *h, lpa_stats *st);

/* Decodes the whole graph on the device into a CSR indexed by vertex id:
 * row_out has n + 1 entries, clm_out num_arcs entries; each list holds the
 * interval neighbours then the residual neighbours, each part ascending (sort
 * a list to compare with the reference's .clm).  Parity hook replacing the
 * decompress test harness (include/decompressor.cuh:116-144). */
lpa_status lpa_decode_csr(struct lpa_handle *h, uint64_t *row_out, uint32_t *clm_out);

/* Degree of every position as decoded on the device (n entries). */
lpa_status lpa_get_degrees(struct lpa_handle *h, uint32_t *deg_out, size_t n);

/* Dispatch control.  Assign a variant to one segment (-1: all segments whose
 * degrees it supports), rebuilding the launch lists. */
lpa_status lpa_set_dispatch(struct lpa_handle *h, int dispatch, int force_variant);
/* An explicit plan: variant[s] for every segment s (count = lpa_info.num_segments),
 * e.g. a plan found by a tuner.  A variant a segment cannot run is rejected
 * (LPA_ERR_INVALID_ARG) and the plan is left as it was.  The handle switches to
 * LPA_DISPATCH_FORCE semantics (no learning) until the next lpa_set_dispatch.
 * No counterpart in the reference, which hard-codes its degree buckets
 * (baselines/novaplus/novaplus_propogator.cuh:219-220). */
lpa_status lpa_set_plan(struct lpa_handle *h, const uint8_t *variant, size_t count);

/* Work shapes and cache policies of the two-pass kernels: the autotuner's knobs.  No
 * counterpart in the reference, whose shapes are compile-time constants. */
typedef struct lpa_tune {
  uint32_t group_positions;  /* positions (degree <= 32) per several-vertices warp item, 1..32; default 32 */
  uint32_t warp_positions;   /* vertices per one-vertex-at-a-time warp item, 1..32; default 4 */
  uint32_t warp_max_degree;  /* largest degree one warp counts (32..511); a block counts larger; default 511 */
  uint32_t warp_claim;       /* warp items a warp claims from the queue at once, 1..8; default 2 */
  uint32_t bulk_stage;       /* 1: several-vertices warp items stage their labels with one bulk copy
                                (cp.async.bulk into shared memory) instead of per-lane loads; default 0 */
  uint32_t gather_cache;     /* cache path of the two-pass pre-pass's label reads: 0 (default) the labels
                                of the lowest 8192 ids through L1, the rest through L2 only; 1 all through
                                L2 only, leaving L1 to the bitstream; 2 all through L1 (hot labels) */
  uint32_t stage_stream;     /* how the pre-pass moves each decode group's stream span ahead of its decode:
                                0 (default) not at all (per-lane loads); 1 a bulk prefetch of the next
                                group's span into L2; 2 a bulk copy of the next group's span into one of
                                the warp's two shared-memory buffers (mbarrier-completed), overlapping the
                                current group's decode */
} lpa_tune;
lpa_status lpa_get_tune(struct lpa_handle *h, lpa_tune *out);
/* Installs the knobs (out of range: LPA_ERR_INVALID_ARG) and rebuilds the work lists. */
lpa_status lpa_set_tune(struct lpa_handle *h, const lpa_tune *t);
/* Autotuner: searches the knobs one at a time (coordinate descent, two
 * sweeps) for the current plan.  Every candidate runs `repeats` iterations
 * (default 2 when <= 0), each from the same label state, and is judged by the
 * iteration's kernel busy time on the GPU clock; the labels and the iteration
 * count are as before the call.  With cache_path, a result found there for
 * this GPU, graph, sketch threshold and plan is installed without a search,
 * and a new result is appended.  The best knobs are installed and returned in
 * out (may be NULL). */
lpa_status lpa_autotune(struct lpa_handle *h, const char *cache_path, int repeats, lpa_tune *out);
/* Per segment, a bit mask of the variants able to run it (bit v: lpa_variant
 * v), the plans lpa_set_plan accepts. */
lpa_status lpa_get_capable(struct lpa_handle *h, uint8_t *mask, size_t count);
/* Per-segment view of the plan: begin/end positions, bucket, variant. */
lpa_status lpa_get_segments(struct lpa_handle *h, uint32_t *begin, uint32_t *end, uint8_t *bucket,
                            uint8_t *variant, size_t count);

/* ------------------------------------------------ dispatch cost model ---- */
/* The 6 -> 32 -> 32 -> 4 fp32 MLP behind LPA_DISPATCH_LEARNED (no reference
 * counterpart; the reference dispatches by fixed degree buckets only).
 * Parameters are 1412 floats: W1[32][6] b1[32] W2[32][32] b2[32] W3[4][32] b3[4]. */
#define LPA_MLP_PARAMS 1412
/* Gradient (1412 floats) of sum_k 0.5 (y_k[variant_k] - target_k)^2 over n
 * samples x (n x 6), computed by the library's own backward kernel. */
lpa_status lpa_mlp_gradient(int device, const float *params, const float *x, const uint8_t *variant,
                            const float *target, size_t n, float *grad_out, float *loss_out);
/* Forward pass on the device: out receives n x 4 predicted log-costs. */
lpa_status lpa_mlp_predict(int device, const float *params, const float *x, size_t n, float *out);
/* The handle's current parameters (the initial ones before any training). */
lpa_status lpa_get_mlp(struct lpa_handle *h, float *params, size_t n);
/* The last learned plan (variant per segment) and its predictions (4 per segment). */
lpa_status lpa_get_learned_plan(struct lpa_handle *h, uint8_t *plan, float *pred, size_t count);
/* The cost model's own plan: per segment, the capable variant with the least
 * predicted cost, as the model gave it after exploring -- before the learner's
 * trials compare it with the merged candidate (every capable segment on the
 * two-pass kernels) and with the fixed plan.  LPA_ERR_INVALID_ARG until the
 * learner has explored. */
lpa_status lpa_get_mlp_plan(struct lpa_handle *h, uint8_t *plan, size_t count);
/* Device cycles per segment of the last iteration that recorded them. */
lpa_status lpa_get_segment_cycles(struct lpa_handle *h, uint64_t *cycles, size_t count);

/* ------------------------------------------------ no-allocation path ----- */
/* One synchronous iteration (the two-pass path: decode to a CSR, then count)
 * that allocates nothing, for callers that cannot call cudaMalloc -- a fixed
 * device-memory budget already spent, buffers owned by the caller's own pool,
 * or a context where allocation is not allowed.  No counterpart in the
 * reference.
 *   g          : every pointer in it is DEVICE memory owned by the caller; the
 *                stream words need at least 4 zero words after the last bit.
 *                g->vertices must be a permutation of 0..n-1 (as every
 *                compressor output is).
 *   labels_in / labels_out : device, n entries each, distinct buffers; with
 *                vertices a permutation, every vertex's output is written.
 *   stream     : cudaStream_t (NULL: the legacy default stream).
 *   changed_out: host, may be NULL.
 * Working memory is one static 16 MiB device array inside the library, held
 * by every GPU that loads it.  Limits: degrees (n), offsets (n_c + 1) and the
 * decoded ids of the compressed positions must fit in it, and every degree
 * must be <= 1023 and below cms_threshold (when non-zero); otherwise the call
 * returns LPA_ERR_CAPACITY without launching the decode.  The first call on a
 * device looks up the array's address, which also makes the device load the
 * library's kernels and claim the array (lazy module loading): make it before
 * the caller spends its memory budget and before any stream capture.  It
 * returns LPA_ERR_OOM when the device cannot hold the array.  The address is
 * kept for the process's life: resetting the device (cudaDeviceReset) after
 * it is not supported.  One array serves every call on a device: calls whose
 * work overlaps on the GPU (other streams, other host threads) race on it. */
lpa_status lpa_iterate_noalloc(const lpa_graph_desc *g, const uint32_t *labels_in, uint32_t *labels_out,
                               uint32_t cms_threshold, void *stream, uint64_t *changed_out);

/* ------------------------------------------ host format layer (lpa_hg_*) --- */
/* A host graph owns a CSR (by vertex id) and/or its compressed form, produced
 * by the fast bit-identical encoder that replaces CgrCompressor
 * (src/compressor.cpp:70-515) and File (src/file.cpp:24-262). */
typedef struct lpa_host_graph lpa_host_graph;

lpa_status lpa_hg_generate_road(uint32_t width, uint32_t height, double keep_p, double extra_p,
                                int max_dist, uint64_t seed, lpa_host_graph **out);
lpa_status lpa_hg_generate_rmat(int scale, double edge_factor, double a, double b, double c,
                                uint64_t seed, int bfs_relabel, uint64_t n_limit, lpa_host_graph **out);
lpa_status lpa_hg_generate_copy(uint64_t n, uint32_t out_degree, double copy_p, int copy_offset,
                                double zipf_s, uint64_t seed, lpa_host_graph **out);
/* Takes a CSR (lists sorted, no duplicates). */
lpa_status lpa_hg_from_csr(uint64_t n, const uint64_t *row, const uint32_t *clm, lpa_host_graph **out);
/* Reference edge-list ingest (File::read_from_edge_list, src/file.cpp:115-195). */
lpa_status lpa_hg_read_edge_list(const char *path, int one_way, lpa_host_graph **out);
/* Reference edge list written back out (both arcs, or each edge once). */
lpa_status lpa_hg_write_edge_list(lpa_host_graph *g, const char *path, int both_arcs);
/* CgrCompressor(3, 4, 256, 256) + write_cgr(path, small_thresh, large_thresh). */
lpa_status lpa_hg_compress(lpa_host_graph *g, int small_thresh, int large_thresh, int threads);
/* The same compression on a GPU, byte-identical to lpa_hg_compress: bit
 * sizing and writing run one thread per compressed vertex on `device`.  Only
 * the reference parameters.  LPA_ERR_CUDA when the device fails or is absent. */
lpa_status lpa_hg_compress_gpu(lpa_host_graph *g, int small_thresh, int large_thresh, int device);
/* Loads the reference's compressed files (64-bit offsets). */
lpa_status lpa_hg_load_cgr(const char *base, int small_thresh, lpa_host_graph **out);
lpa_status lpa_hg_write_cgr(lpa_host_graph *g, const char *base);
/* Reference .row/.clm. */
lpa_status lpa_hg_write_csr(lpa_host_graph *g, const char *base);
lpa_status lpa_hg_csr(lpa_host_graph *g, uint64_t *n, const uint64_t **row, const uint32_t **clm);
/* Fills desc with pointers into g (valid while g lives). */
lpa_status lpa_hg_desc(lpa_host_graph *g, lpa_graph_desc *desc);
/* The graphs as one: positions [0, n_c) hold every graph's compressed
 * positions in graph order, then every graph's small positions; graph k's ids
 * are shifted by the vertex counts of graphs 0..k-1; the bitstreams are
 * concatenated bit for bit, so every offset is exact.  A vertex decodes to its
 * own graph's arcs, shifted, because CGR codes ids relative to the vertex
 * itself and to each other.  LPA_ERR_CAPACITY when the ids or small arcs
 * leave 32 bits.  No counterpart in the reference. */
lpa_status lpa_hg_concat(const lpa_graph_desc *graphs, size_t num_graphs, lpa_host_graph **out);
lpa_status lpa_hg_free(lpa_host_graph *g);

/* ------------------------------------------------- batched graphs ---------- */
/* Many independent graphs propagated together, each with its own convergence
 * test and labels (ids local to the graph), bit-exact against running each
 * graph alone.  opts->batch_mode picks how: LPA_BATCH_LOCKSTEP concatenates
 * the batch into one graph with shifted ids and runs it through one handle
 * (any dispatch, the autotuner and the CUDA-graph loop apply), iterating until
 * every graph has stopped; LPA_BATCH_QUEUE runs one persistent kernel fed
 * from a device work queue, where a graph leaves as soon as it converges.
 * Lockstep falls back to the queue when the batch has 2^32 - 1 vertices or
 * small arcs or more.  The reference runs one graph per process
 * (src/main.cpp). */
lpa_status lpa_batch_create(const lpa_graph_desc *graphs, size_t num_graphs, const lpa_opts *o,
                            struct lpa_batch **out);
lpa_status lpa_batch_run(struct lpa_batch *b, int max_iter, int early_exit, uint32_t *iters_per_graph);
lpa_status lpa_batch_get_labels(struct lpa_batch *b, size_t graph, uint32_t *host_out, size_t n);
lpa_status lpa_batch_destroy(struct lpa_batch *b);
/* The lockstep batch's handle (the concatenated graph), for lpa_autotune,
 * lpa_set_dispatch, lpa_get_stats and lpa_get_info; NULL in queue mode.  Owned
 * by the batch.  Its labels are shifted ids: read them with
 * lpa_batch_get_labels. */
struct lpa_handle *lpa_batch_handle(struct lpa_batch *b);

#ifdef __cplusplus
}
#endif
#endif /* LPA_CAPI_H */
