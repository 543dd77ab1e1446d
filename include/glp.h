/*
 * glp.h -- C ABI of the B200 label-propagation engine (libglp_b200.so).
 *
 * The reference (Gibyeng/GLP) has no C ABI: its surface is header-only C++
 * templates.  Each entry point below names the reference interface it
 * replaces, so a binding for any FFI (ctypes, cgo, JNI, N-API) can be written
 * against plain pointers and sizes.
 *
 * Conventions
 *   - Every call returns 0 on success or a negative GLP_E* code; no exception
 *     crosses the ABI.  glp_last_error() gives the message of the calling
 *     thread's last failure.
 *   - Vertex ids and labels are int32; the CSR has n+1 int32 offsets and m
 *     int32 column indices (m < 2^31), exactly the reference's
 *     CSRGraph<int32_t,int32_t> layout (header/graph.h:61-198).
 *   - A handle is thread-compatible, not thread-safe: one thread at a time.
 *   - Streams are passed as void* (a cudaStream_t); NULL means the engine's
 *     own stream for that handle.
 *   - There is no CPU fallback: without a usable CUDA device every compute
 *     call fails with GLP_ENODEV.
 */
#ifndef GLP_B200_GLP_H
#define GLP_B200_GLP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define GLP_OK 0
#define GLP_EINVAL (-1)   /* bad argument or malformed CSR */
#define GLP_ENOMEM (-2)   /* device or host allocation failed, or over budget */
#define GLP_ECUDA (-3)    /* a CUDA call failed */
#define GLP_ENOTSUP (-4)  /* method / option not supported */
#define GLP_ENODEV (-5)   /* no usable CUDA device */
#define GLP_ETIMEOUT (-6) /* a bounded wait ran out */
#define GLP_ECANCELED (-7)/* request cancelled */
#define GLP_EKERNEL (-8)  /* a kernel reported an internal error flag */
#define GLP_EAGAIN (-9)   /* nothing ready yet (server poll) */

/* ---- methods (main.cu:63-101 switch) ----------------------------------- */
#define GLP_METHOD_CLASSIC 1 /* prop/classicLprop.cuh */
#define GLP_METHOD_LAYERED 2 /* prop/MultiLprop.cuh + tutorial/CPUlp.cuh:169-262 */
#define GLP_METHOD_SLPA 3    /* prop/SLPAprop.cuh, semantics tutorial/Base5prop.cuh */
#define GLP_METHOD_USER 4    /* prop/UserdefinedLprop.cuh + README.md:72-101 hooks */
#define GLP_METHOD_SEEDED 5  /* prop/seedLprop.cuh: seeds fixed, glp_graph_set_seeds */

/* ---- counting back-ends (method/hashtable.cuh, countmin.cuh, frequent.cuh)
 * Every back-end gives the same labels, bit for bit.  CM and FA change how
 * the big tier (degrees mid_max+1 .. big_max) counts: a summary decides the
 * vertices whose mode it can prove, and the exact kernel counts the rest, as
 * the reference's sketch kernel re-scans (header/kernel.cuh:1420-1566).  The
 * other tiers always count exactly. */
#define GLP_BACKEND_EXACT 0 /* shared/global hash tables (GlobalHT) */
#define GLP_BACKEND_CM 1    /* one-probe table + 3-row count-min sketch screen, exact fallback */
#define GLP_BACKEND_FA 2    /* Misra-Gries frequent-items screen (one warp per vertex), exact fallback */

/* ---- built-in hook sets for method 4 ----------------------------------- */
#define GLP_HOOKS_CLASSIC 0 /* README.md:83-101 example: (L[sid], 1), score = freq */
#define GLP_HOOKS_LAYERED 1 /* score = dstar*freq - vol[l], UpdateVertex counts vol */
#define GLP_HOOKS_WEIGHTED_DEGREE 2 /* freq = w / deg(sid) in FP64 (non-monotone score demo) */

#define GLP_MAX_LAYERS 32

typedef struct glp_graph glp_graph;

/* Parameters.  glp_params_default() fills every field; callers then change
 * what they need.  Replaces the constants hard-coded in the reference's
 * perform_lp (prop/classicLprop.cuh:176-198, :381; prop/MultiLprop.cuh:148;
 * prop/SLPAprop.cuh:31). */
typedef struct glp_params {
  int32_t struct_size;            /* = sizeof(glp_params) */
  int32_t backend;                /* GLP_BACKEND_* */
  /* layered LP: layer s uses the integer score dstar[s]*k - vol[l], which
   * orders labels exactly as k - gamma*(vol-k) with gamma = 1/(dstar-1). */
  int32_t nlayers;
  int32_t dstar[GLP_MAX_LAYERS];
  /* SLPA */
  int32_t slpa_T;                 /* memory slots per vertex (1..64) */
  double slpa_r;                  /* post-processing threshold */
  uint64_t seed;                  /* speaker hash seed */
  /* method 4 */
  int32_t hooks;                  /* GLP_HOOKS_* */
  /* degree tiers (0 = engine default / autotuned) */
  int32_t tiny_max;               /* thread per vertex up to this degree (<= 8) */
  int32_t mid_max;                /* warp per vertex up to this degree (32..256) */
  int32_t big_max;                /* block per vertex up to this degree (mid_max..24576 unweighted,
                                     mid_max..12288 weighted); above: hubs.  0 = the largest the
                                     graph allows (24576 unweighted, 12288 weighted) */
  int32_t hub_chunk;              /* edges per hub streaming block (256..65536) */
  int32_t use_graph;              /* capture the iteration loop in a CUDA graph */
  int32_t async;                  /* 1: enqueue on the stream and return without
                                     synchronising (device outputs only, no
                                     callback); kernel error flags are then
                                     reported by glp_graph_check(); the
                                     stream must stay valid until the next
                                     call on the handle */
  int32_t batch_threads;          /* glp_batch_run: threads per block, 512 or 1024 (0 = tuned / default) */
  int32_t barrier_limit_us;       /* glp_batch_run: how long a grid barrier of the persistent kernel
                                     waits before the run gives up with GLP_ETIMEOUT (0 = 5 s) */
  int32_t fault_skip_cta;         /* glp_batch_run, for tests of the failure path: 1 + the index of a
                                     block that never arrives at the first grid barrier, so that the
                                     other blocks' bounded waits run out (0 = off) */
  int32_t majority_permille;      /* classic / SLPA steps after the first: below this many changes per
                                     1000 vertices in the previous step, a step first decides the vertices
                                     whose own label holds a strict majority (0 = 500); every mode is exact */
  int32_t frontier_permille;      /* below this many changes per 1000 vertices, only neighbours of changed
                                     vertices are recomputed (one-graph runs: symmetric graphs; batched
                                     runs: vertices with a changed neighbour, any CSR; 0 = 50 one-graph,
                                     10 batched; -1 = never) */
  int32_t l2_window;              /* 1: keep the label array being gathered in L2 through a persisting
                                     access-policy window on the run's streams (off by default) */
  int32_t cycle_stop;             /* classic runs on symmetric graphs: 0 (default) stops running steps
                                     once a step ends in a two-step cycle (L_{t+1} = L_{t-1} for every
                                     vertex), after which every labeling is known: the results and the
                                     per-iteration outputs are those of all niter steps; -1 runs every
                                     step */
  int32_t serial_step;            /* 1: every kernel of a step runs on the run's own
                                     stream instead of three forked streams, so that
                                     the per-tier event times of glp_outputs are each
                                     tier's own duration (profiling; slower) */
  int32_t mid_prefetch;           /* mid tier of unweighted classic steps: 0 (default) loads the next
                                     vertex's first 128 neighbour labels while the current vertex is
                                     counted; -1 loads them in turn */
  int32_t batch_blocks;           /* batched runs: at most this many CTAs in the cooperative
                                     grid (0: as many as fit every SM); a small grid can start
                                     while other kernels hold part of the GPU */
  int32_t big_staged;             /* unweighted full-count steps, big-tier degrees up to 1024: 1 stages
                                     each row's columns in shared memory with a bulk copy issued one
                                     vertex ahead (cp.async.bulk); 0 (default) loads them thread by thread
                                     (measured 2.5 % faster on R-MAT scale 24) */
  int32_t reserved[5];            /* zero */
} glp_params;

/* Per-iteration observer (parity checks).  labels is a HOST copy of the
 * labels after iteration `iter` (0-based; layered: layer*niter + iter).
 * Return non-zero to stop the run early (status GLP_ECANCELED). */
typedef int (*glp_iter_cb)(int32_t iter, const int32_t* labels, int32_t n, void* user);

/* Outputs of glp_run.  labels is required; the others are optional. */
typedef struct glp_outputs {
  int32_t* labels;      /* [n] final labels */
  int32_t* slpa_comm;   /* [n][slpa_T] communities kept by post-processing, ascending, -1 padded */
  int32_t* slpa_ncomm;  /* [n] number of communities kept */
  int32_t* slpa_mem;    /* [slpa_T][n] speaker memory, -1 = empty */
  int32_t* vol;         /* [n] layered: label volumes after the last iteration */
  int64_t* changed;     /* [iterations] labels changed per iteration (host) */
  float* tier_ms;       /* [8] host: summed device ms per kernel group (tiny, group16,
                           group32, mid, big, hub, aux, majority pre-pass), timed
                           with CUDA events on the run's stream; NULL = none */
  int64_t* launches;    /* [1] host: kernels this run launched */
  float* iter_ms;       /* [iterations] host: device ms of each iteration's step
                           kernels (timed like tier_ms; needs tier_ms) */
  float* step_tier_ms;  /* [iterations][8] host: per-iteration tier_ms (needs tier_ms) */
  int32_t on_device;    /* 1: labels/slpa/vol pointers are device pointers */
} glp_outputs;

const char* glp_last_error(void);
const char* glp_version(void);
int glp_params_default(glp_params* p);

/* Graph handle.  Replaces CSRGraph + the propagator's preprocess()
 * (header/graph.h:61-198, prop/classicLprop.cuh:65-78): the CSR is copied
 * to (or adopted on) the device once and stays resident across runs.
 * weights may be NULL; non-NULL weights must be >= 0 (integer edge weights,
 * summed exactly).  on_device = 1: the pointers are device pointers
 * (copied device-to-device).  The CSR is validated (monotone offsets, columns
 * in [0,n)); a malformed CSR returns GLP_EINVAL. */
int glp_graph_create(const int32_t* offsets, const int32_t* cols, const int32_t* weights, int32_t n,
                     int64_t m, int32_t on_device, glp_graph** out);
/* As glp_graph_create, with flags: GLP_GRAPH_SYMMETRIC asserts that every
 * edge is stored in both directions (what CSRGraph builds for undirected
 * input, header/graph.h:97-115), which lets converged classic steps
 * recompute only the neighbours of changed vertices.  Without the flag the
 * engine checks symmetry on the device the first time it could use it
 * (rows must be strictly ascending to qualify). */
#define GLP_GRAPH_SYMMETRIC 1u
int glp_graph_create_ex(const int32_t* offsets, const int32_t* cols, const int32_t* weights, int32_t n,
                        int64_t m, int32_t on_device, uint32_t flags, glp_graph** out);
void glp_graph_destroy(glp_graph* g);
int glp_graph_info(const glp_graph* g, int32_t* n, int64_t* m, int32_t* max_degree);
/* Degree-tier plan for these params.  out[0..6]: vertices per tier
 * [isolated, tiny, group16, group32, mid, big, hub]; out[7]: hub hash
 * buckets; out[8..14]: CSR entries (edges) per tier in the same order;
 * out[15]: hub streaming chunks.  Mirrors the bin report of
 * prop/classicLprop.cuh:213-227. */
int glp_graph_plan(glp_graph* g, const glp_params* p, int64_t out[16]);
/* The same plan computed from host offsets alone (no device needed),
 * planned as for an unweighted graph. */
int glp_plan_offsets(const int32_t* offsets, int32_t n, const glp_params* p, int64_t out[16]);
/* Reports (and clears) kernel error flags raised by asynchronous runs. */
int glp_graph_check(glp_graph* g);

/* Graph construction on the device from an edge list (count pairs
 * src[i] -> dst[i], ids in [0, n); host or device arrays).  Replaces the
 * reference's offline normaliser and loader (tools/normalize.cpp:262-348,
 * header/graph.h:226-258): self loops dropped; unless GLP_EDGES_DIRECTED,
 * every edge stored in both directions; duplicate entries dropped; unless
 * GLP_EDGES_KEEP_IDS, vertices renumbered by degree descending, ties by the
 * smaller original id; rows ascending.  old_id (nullable, n entries, host or
 * device as the edges) receives the original id of each vertex.  count <
 * 2^30. */
#define GLP_EDGES_DIRECTED 1u
#define GLP_EDGES_KEEP_IDS 2u
int glp_graph_from_edges(const int32_t* src, const int32_t* dst, int64_t count, int32_t n, int32_t on_device,
                         uint32_t flags, int32_t* old_id, glp_graph** out);
/* Copies a handle's CSR out: offsets [n+1], cols [m], weights [m] (nullable;
 * ignored for an unweighted graph), device pointers when on_device. */
int glp_graph_export(const glp_graph* g, int32_t* offsets, int32_t* cols, int32_t* weights, int32_t on_device);

/* Device view of a handle for method-4 hook sets compiled outside the
 * library (include/glp_hooks.cuh).  Replaces the reference's route for user
 * hooks -- editing the __device__ stubs of header/kernel.cuh:6071-6085 and
 * rebuilding (README.md:72-101) -- with a resident graph that user code
 * reads in place. */
typedef struct glp_device_view {
  int32_t n;
  int32_t max_degree;
  int64_t m;
  int32_t device;               /* CUDA device of the handle */
  int32_t sms;                  /* its streaming multiprocessors */
  const int32_t* off;           /* [n+1] device CSR offsets */
  const int32_t* cols;          /* [m] device CSR columns */
  const int32_t* w;             /* [m] device weights, NULL when unweighted */
  int32_t* labels[2];           /* [n] each: both set to the vertex ids */
  unsigned long long* changed;  /* [niter] per-iteration change counters, zeroed */
  uint32_t* err;                /* one error word, zeroed */
  uint32_t* hook_keys;          /* [2m] spill table keys for degrees above 256 (else NULL) */
  double* hook_vals;            /* [2m] spill table values (else NULL) */
  void* stream;                 /* the handle's stream */
} glp_device_view;
/* Prepares the handle's buffers for a run of niter iterations written outside
 * the library and fills *out: label buffers (set to the vertex ids), niter
 * change counters and the error word (zeroed), and the spill tables when a
 * degree exceeds 256.  The pointers stay valid until the next call on the
 * handle or glp_graph_destroy.  Synchronous. */
int glp_graph_device_view(glp_graph* g, int32_t niter, glp_device_view* out);

/* ---- counting summaries on the device (parity inspection) --------------
 * The count-min sketch SharedCM<W,3> of method/countmin.cuh:9-262 built over
 * the whole neighbourhood of each listed vertex under `labels` (n entries,
 * host or device): every neighbour u adds its edge weight (1 when the graph
 * is unweighted) to cell cm_hash_r(L[u]+1) % width of row r, with the row
 * hashes of countmin.cuh:97-125.  ref_compat = 1 adds the third row's
 * increment into the second row, as countmin.cuh:190 does.  rows: host,
 * [nv][3][width] uint32; width in [1, 4096]. */
int glp_graph_cm_sketch(glp_graph* g, const int32_t* labels, int32_t labels_on_device, const int32_t* vertices,
                        int32_t nv, int32_t width, int32_t ref_compat, uint32_t* rows);
/* The frequent-items table SharedFA<C> of method/frequent.cuh:10-106 fed the
 * neighbour labels of each listed vertex one at a time in CSR order (edge
 * weights are not used): key = label+1, linear probing from
 * fmix32(key) % capacity, and when every slot holds another key a decrement
 * round (clean: counts drop by one; ref_compat = 1: frequent.cuh:96-100 as
 * written, every count becomes 0) after which the key is dropped; keys
 * whose count was 1 are freed.  keys/vals: host [nv][capacity] (key 0 =
 * empty slot); rounds: host [nv] decrement rounds.  capacity in [1, 65536]. */
int glp_graph_fa_summary(glp_graph* g, const int32_t* labels, int32_t labels_on_device, const int32_t* vertices,
                         int32_t nv, int32_t capacity, int32_t ref_compat, uint32_t* keys, uint32_t* vals,
                         int32_t* rounds);

/* Seeds of method 5 (seeded LP; prop/seedLprop.cuh, whose seed list is read
 * from a file, :161-181).  seeds[v] != 0 marks vertex v as a seed (n bytes,
 * host or device); NULL clears them.  A method-5 run labels every seed with
 * its own id and every other vertex -1 (unlabelled, as
 * initialize_labels_by_seeds, header/kernel.cuh:453-466); then, every
 * iteration, a seed keeps its label and any other vertex takes the label of
 * largest count (weight sum) among its LABELLED neighbours, ties -> the
 * largest label, keeping its own when none is labelled. */
int glp_graph_set_seeds(glp_graph* g, const uint8_t* seeds, int32_t on_device);

/* Cancellation of runs on this handle: while flag (host memory, NULL = none)
 * is non-zero, glp_run stops at the next iteration boundary with
 * GLP_ECANCELED, after the work it already enqueued has finished (the
 * handle then has nothing in flight).  Another thread may set the flag at
 * any time.  No counterpart in the reference (its runs cannot be stopped). */
int glp_graph_set_cancel_flag(glp_graph* g, const volatile int32_t* flag);

/* Run `method` for niter iterations (layered: nlayers*niter).  Replaces
 * XProp<V,E>::run(niter) of prop/classicLprop.cuh:454-462,
 * prop/MultiLprop.cuh:384-392, prop/SLPAprop.cuh and
 * prop/UserdefinedLprop.cuh, selected as main.cu:63-101 does.  Labels start
 * at the vertex id (kernel.cuh:444-451).  Unlike the reference, labels are
 * returned.  The call is synchronous with respect to the host. */
int glp_run(glp_graph* g, int32_t method, const glp_params* p, int32_t niter, glp_outputs* out,
            glp_iter_cb cb, void* cb_user, void* stream);

/* ---- synthetic graph samplers (input synthesis for tests and benchmarks) --
 * Deterministic counter-based sampling: sample i depends only on (seed, i),
 * so host and device produce identical edge lists.  on_device selects where
 * src/dst live.  R-MAT quadrant probabilities a,b,c (d = 1-a-b-c). */
int glp_sample_rmat(int32_t scale, double a, double b, double c, uint64_t seed, int64_t first, int64_t count,
                    int32_t* src, int32_t* dst, int32_t on_device);
/* Planted partition: n vertices in k equal communities (community of v =
 * v / ceil(n/k)); samples [0, n_intra) are intra-community, the rest are
 * inter-community. */
int glp_sample_planted(int32_t n, int32_t k, int64_t n_intra, uint64_t seed, int64_t first, int64_t count,
                       int32_t* src, int32_t* dst, int32_t on_device);
/* Overlapping planted partition (SLPA workload): every vertex is in its home
 * community v / ceil(n/k); a fraction `overlap` of vertices (chosen by hash)
 * also belongs to a second community.  An edge picks u, one of u's
 * communities, and a uniform member of it. */
int glp_sample_overlap(int32_t n, int32_t k, double overlap, uint64_t seed, int64_t first, int64_t count,
                       int32_t* src, int32_t* dst, int32_t on_device);
/* Edge weight w = 1 + (H(seed, min(u,v), max(u,v)) mod wmax): symmetric. */
int glp_edge_weights(const int32_t* off, const int32_t* cols, int32_t n, int64_t m, int32_t wmax, uint64_t seed,
                     int32_t* w, int32_t on_device);

/* ---- reference-format graph I/O (tools/ + header/graph.h) ---------------
 * Load a binary int32 (u,v) pair file with the semantics of
 * load_edgelist_bin + CSRGraph (header/graph.h:69-147, :226-258): self
 * loops dropped, symmetrised unless direct, duplicates kept, neighbour order
 * = file order, n = max id + 1.  Returns host buffers owned by the library
 * (free with glp_free_host). */
int glp_load_edgelist_bin(const char* path, int32_t direct, int32_t** offsets, int32_t** cols, int32_t* n,
                          int64_t* m);
void glp_free_host(void* p);

/* ----------------------------------------------------------------------
 * Batched classic LP.  The reference runs one graph per propagator (its
 * two-graph precursor, tutorial/MultiGprop.cuh:585-800, launches each graph
 * separately); a batch packs many independent graphs into one
 * device-resident multi-CSR and propagates all of them in ONE persistent
 * cooperative kernel launch per run.
 *
 * glp_batch_create: graph g is offsets[g] (n[g]+1 int32) and cols[g] (m[g]
 * int32, ids local to the graph), host or device arrays (on_device),
 * unweighted.  The packed labels of a run hold graph g's labels at
 * [vbase_g, vbase_g + n[g]), vbase_g = n[0] + ... + n[g-1]; they equal what
 * glp_run(method 1) gives that graph alone, bit for bit.  Every degree must
 * be <= 4096 (GLP_ENOTSUP otherwise: run such a graph with glp_run). */
typedef struct glp_batch glp_batch;
int glp_batch_create(int32_t ngraphs, const int32_t* const* offsets, const int32_t* const* cols, const int32_t* n,
                     const int64_t* m, int32_t on_device, glp_batch** out);
/* As glp_batch_create, with a per-graph iteration count niter[g] (>= 0,
 * non-decreasing over g, at most 8 distinct values) that glp_batch_run uses
 * when given GLP_BATCH_OWN_ITERATIONS: graphs of smaller counts stop
 * updating after their count; their labels are what a solo run of that
 * count gives. */
#define GLP_BATCH_OWN_ITERATIONS (-1)
int glp_batch_create_ex(int32_t ngraphs, const int32_t* const* offsets, const int32_t* const* cols, const int32_t* n,
                        const int64_t* m, int32_t on_device, const int32_t* niter, glp_batch** out);
/* Packs a new set of graphs into an existing batch, reusing its device
 * buffers (they only grow): a round-by-round caller allocates nothing once
 * the batch has seen its largest round.  Arguments as glp_batch_create_ex. */
int glp_batch_repack(glp_batch* b, int32_t ngraphs, const int32_t* const* offsets, const int32_t* const* cols,
                     const int32_t* n, const int64_t* m, int32_t on_device, const int32_t* niter);
void glp_batch_destroy(glp_batch* b);
int glp_batch_info(const glp_batch* b, int64_t* n, int64_t* m, int32_t* max_degree, int32_t* ngraphs);
/* niter synchronous classic iterations of every graph (or, with
 * GLP_BATCH_OWN_ITERATIONS, each graph's own count).  labels: the packed
 * labels (host, or device when on_device); changed: optional host array of
 * the largest iteration count, labels changed per iteration over the batch.  params (nullable; other
 * values = the tuned or default choice): tiny_max in {8,16,32} = largest
 * degree counted by one thread per vertex (above it, up to 32, lane groups);
 * mid_max 64 = degrees 33..64 by 16-lane groups, 32 = by whole warps;
 * batch_threads in {512,1024} = threads per block; use_graph = 1 captures the
 * run (counter resets, the persistent launch, a device-side label copy) in a
 * CUDA graph once and replays it while niter, the configuration, the stream
 * and the device label pointer stay the same.  Synchronous with respect to
 * the host. */
int glp_batch_run(glp_batch* b, const glp_params* p, int32_t niter, int32_t* labels, int32_t on_device,
                  int64_t* changed, void* stream);
/* Autotuner: times every kernel configuration (threads per block x thread
 * tier bound x counting of degrees 33..64) on this batch for probe_iters iterations and
 * keeps the fastest for later runs.  best (nullable) receives the choice in
 * the glp_batch_run parameter fields; times_ms (nullable, >= 12 entries)
 * the time of each candidate (-1: does not fit); ncand the candidate count. */
int glp_batch_tune(glp_batch* b, int32_t probe_iters, glp_params* best, float* times_ms, int32_t* ncand);

/* ----------------------------------------------------------------------
 * Served LP.  No counterpart in the reference (it runs one graph per
 * process).  A server keeps graphs and label state in HBM while requests of
 * mixed size and method arrive: admission is FIFO against an HBM budget;
 * small classic requests (unweighted, every degree <= 4096, at most
 * batch_max_vertices vertices) are packed into rounds of the persistent
 * batched kernel, each round taking every such request admitted so far
 * (continuous batching at round granularity); the rest run as one-graph
 * solves on plain_workers threads whose device work overlaps the rounds,
 * shortest expected job first (aged by waiting time); short one-graph
 * solves (short_job_us) have a worker of their own.  The rounds and the
 * short solves run on streams of the device's highest priority.
 * Every result equals glp_run of that request alone. */
typedef struct glp_server glp_server;
typedef struct glp_server_config {
  int32_t struct_size;         /* = sizeof(glp_server_config) */
  int32_t device;              /* -1: the caller's current device */
  int64_t hbm_budget_bytes;    /* admission budget (default 150e9) */
  int32_t max_batch_graphs;    /* requests per batched round (default 4096) */
  int32_t plain_workers;       /* concurrent one-graph solves (default 1) */
  int32_t batch_max_vertices;  /* larger graphs take the one-graph path (default 2^22) */
  int32_t short_job_us;        /* one-graph requests expected to take less than this
                                  (default 0: 20000 us; -1: none) run on a worker of
                                  their own at the device's highest stream priority,
                                  next to the batched rounds, instead of queueing
                                  behind long solves */
  int32_t lone_one_graph;      /* 1: a round of one request runs as a one-graph solve
                                  (default 0: in the batched kernel like any round, on
                                  a grid sized to it) */
  int32_t reserved[6];
} glp_server_config;
typedef struct glp_request_stats {
  double submit_s, admit_s, start_s, done_s; /* seconds since the server started */
  int32_t path;                /* 0: one-graph engine, 1: batched round */
  int32_t batch_graphs;        /* requests in its round (path 1) */
  int32_t status;              /* GLP_OK or the failure code */
  int32_t reserved[5];
} glp_request_stats;
int glp_server_config_default(glp_server_config* c);
int glp_server_start(const glp_server_config* c, glp_server** out);
/* Submits one solve of `method` for niter iterations on a HOST CSR; the
 * labels land in labels_out (host, n entries).  offsets/cols/weights and
 * labels_out must stay valid until the request is done.  *id names it. */
int glp_server_submit(glp_server* s, const int32_t* offsets, const int32_t* cols, const int32_t* weights, int32_t n,
                      int64_t m, int32_t method, const glp_params* p, int32_t niter, int32_t* labels_out,
                      int64_t* id);
/* Resident graphs: glp_server_add_graph copies a CSR (host, or device when
 * on_device) into HBM once, counted against the budget; requests on it are
 * submitted with glp_server_submit_graph and reuse it (and the plans built
 * for it) with no upload; glp_server_remove_graph frees it once no request
 * uses it. */
int glp_server_add_graph(glp_server* s, const int32_t* offsets, const int32_t* cols, const int32_t* weights, int32_t n,
                         int64_t m, int32_t on_device, int64_t* graph_id);
int glp_server_submit_graph(glp_server* s, int64_t graph_id, int32_t method, const glp_params* p, int32_t niter,
                            int32_t* labels_out, int64_t* id);
/* A resident graph built on the device from an edge list, with the
 * semantics and arguments of glp_graph_from_edges; requests on it go through
 * glp_server_submit_graph. */
int glp_server_add_edges(glp_server* s, const int32_t* src, const int32_t* dst, int64_t count, int32_t n,
                         int32_t on_device, uint32_t flags, int32_t* old_id, int64_t* graph_id);
int glp_server_remove_graph(glp_server* s, int64_t graph_id);
/* GLP_EAGAIN while the request waits or runs; its status once done. */
int glp_server_poll(glp_server* s, int64_t id, glp_request_stats* stats);
/* Waits up to timeout_ms (< 0: no limit); GLP_ETIMEOUT when it runs out. */
int glp_server_wait(glp_server* s, int64_t id, int32_t timeout_ms, glp_request_stats* stats);
/* Forgets a finished request. */
int glp_server_release(glp_server* s, int64_t id);
/* Cancels a request: one still waiting for admission, or admitted and not
 * started, ends at once with GLP_ECANCELED and gives back its budget; a
 * one-graph solve in progress stops at its next iteration boundary; a request
 * already inside a batched round finishes that round and its result is
 * discarded.  Either way the request then reports GLP_ECANCELED, unless it
 * had already finished (its result stands).  GLP_EINVAL for an unknown id. */
int glp_server_cancel(glp_server* s, int64_t id);
int glp_server_info(glp_server* s, int64_t* pending, int64_t* in_flight, int64_t* used_bytes, int64_t* rounds);
/* Finishes every submitted request, then stops the threads and frees. */
int glp_server_stop(glp_server* s);

/* ----------------------------------------------------------------------
 * Allocation-free classic LP.  No counterpart in the reference.
 *
 * Method 1 (classic, unweighted; the rule of glp_run) for niter iterations
 * over a CSR the caller already holds on the current device, with labels
 * starting at the vertex ids and written to d_labels (device, n entries).
 * The call allocates no device or pinned host memory: its second label
 * buffer, per-iteration change counters and flag words live in a fixed
 * static device array (about 4.2 MB per device).  Limits: n <= 1048576
 * vertices, niter <= 4096, every degree <= 4096; larger inputs, like a
 * malformed CSR, return GLP_EINVAL with the limit in glp_last_error().
 * `changed` (host, nullable) receives niter change counts.  Work runs on
 * `stream` (NULL: the legacy default stream) and the call is synchronous: it
 * returns after that work has finished.  Every call looks up the current
 * device's copy of the scratch (cudaGetSymbolAddress, which allocates
 * nothing), so the address stays right after a context reset.  The scratch
 * is shared: calls on one device that overlap (from several host threads)
 * race and must be serialised by the caller. */
int glp_run_classic_noalloc(const int32_t* d_offsets, const int32_t* d_cols, int32_t n, int64_t m, int32_t niter,
                            int32_t* d_labels, int64_t* changed, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GLP_B200_GLP_H */
