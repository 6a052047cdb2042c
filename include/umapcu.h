/*
 * umapcu.h -- C ABI of the B200 (sm_100a) UMAP hot path.
 *
 * Drop-in boundary for manifolds-rs's UMAP fuzzy-graph construction and
 * layout optimiser. Every entry point names the reference interface it
 * replaces (paths relative to the manifolds-rs crate root). Plain pointers
 * and sizes only; all "host" pointers are ordinary CPU memory owned by the
 * caller, "device" pointers are CUDA global memory owned by the caller.
 * The library owns the device buffers it allocates internally and frees
 * them before returning (or in the matching *_destroy call).
 *
 * Threading: every call is synchronous with respect to its own inputs and
 * outputs and runs on a stream the library creates per call (or per state
 * handle). Distinct state handles may be used from distinct threads.
 */
#ifndef UMAPCU_H
#define UMAPCU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; each maps 1:1 onto a ManifoldsError variant
 * (src/errors.rs:7-118). */
typedef enum umapcu_status {
    UMAPCU_OK = 0,
    UMAPCU_NO_DATA = 1,                /* ManifoldsError::NoData (errors.rs:78) */
    UMAPCU_NO_GRAPH_EDGES = 2,         /* ManifoldsError::NoGraphEdges (errors.rs:82) */
    UMAPCU_DEGENERATE_LOCAL_RADII = 3, /* ManifoldsError::DegenerateLocalRadii (errors.rs:101) */
    UMAPCU_CUDA_ALLOC = 4,             /* ManifoldsError::CubeclUtilsError (errors.rs:54): allocation */
    UMAPCU_CUDA_LAUNCH = 5,            /* ManifoldsError::CubeclUtilsError: launch / runtime error */
    UMAPCU_TIMEOUT = 6,                /* a bounded device wait gave up */
    UMAPCU_BAD_ARG = 7,                /* invalid argument (null pointer, n_dim out of range, ...) */
    UMAPCU_NO_DEVICE = 8,              /* no CUDA device usable */
    UMAPCU_CAPACITY = 9,               /* output capacity / device budget / scratch too small */
    UMAPCU_CANCELLED = 10              /* a served job was cancelled or the server shut down */
} umapcu_status;

/* Optimiser selection: the string keys of parse_umap_optimiser_gpu
 * (src/training/umap_optimiser_gpu.rs:44-52). "adam_gpu" -> ADAM. SGD is the
 * per-node-gather SGD (clipped attractive term, y += lr_e * grad). */
enum { UMAPCU_OPT_ADAM = 0, UMAPCU_OPT_SGD = 1 };

/* Negative sampler. REF_HASH reproduces gpu_hash_neg
 * (umap_optimiser_gpu.rs:611-624) bit for bit; PHILOX is Philox4x32-10
 * keyed on (seed), counter (CSR entry, epoch, negative/4). */
enum { UMAPCU_NEG_REF_HASH = 0, UMAPCU_NEG_PHILOX = 1 };

/* UmapOptimParams<f32> (src/training/umap_optimisers.rs:24-45). */
typedef struct umapcu_optim_params {
    float a, b, lr, gamma;
    uint32_t n_epochs, neg_sample_rate;
    float min_dist, beta1, beta2, eps;
} umapcu_optim_params;

/* UmapGraphParams<f32> (src/data/graph.rs:30-41). */
typedef struct umapcu_graph_params {
    float bandwidth, local_connectivity, mix_weight;
} umapcu_graph_params;

/* DensState<f32> (src/utils/density.rs:140-160) with its DensParams
 * (density.rs:69-79). r and mu_sum are host arrays of length n. */
typedef struct umapcu_dens {
    float lambda, frac, var_shift;
    const float *r;
    const float *mu_sum;
    float mu_tot;
} umapcu_dens;

/* Human-readable name of a status code. */
const char *umapcu_status_string(umapcu_status s);

/* Library version string ("umapcu <major>.<minor>.<patch> sm_100a"). */
const char *umapcu_version(void);

/* ---------------------------------------------------------------------
 * Parameters (host)
 * ------------------------------------------------------------------- */

/* Replaces UmapOptimParams::fit_params
 * (src/training/umap_optimisers.rs:139-209), f32 instantiation; fits the
 * a, b of 1/(1 + a x^2b) to min_dist/spread on the host. */
umapcu_status umapcu_fit_ab(float min_dist, float spread, float *a, float *b);

/* ---------------------------------------------------------------------
 * Fuzzy simplicial set (graph construction), host buffers
 * ------------------------------------------------------------------- */

/* Replaces smooth_knn_dist (src/data/graph.rs:499-565). knn_dist is
 * [n * k] row-major (self excluded, ascending per row). Writes sigma[n],
 * rho[n]. */
umapcu_status umapcu_smooth_knn_dist(const float *knn_dist, uint32_t n, uint32_t k,
                                     float local_connectivity, float bandwidth, uint32_t n_iter,
                                     float *sigma, float *rho);

/* Replaces the graph stage of construct_umap_graph / construct_umap_graph_gpu
 * (src/lib.rs:296-306, :3421-3431): smooth_knn_dist -> knn_to_coo
 * (graph.rs:585-662) -> symmetrise_graph (graph.rs:684-694, via
 * symmetrise_csr :387-468) -> filter_weak_edges (graph.rs:776-853).
 * Output COO (row, col, val), grouped by row, columns ascending, nnz
 * entries; capacity must be >= 2 * n * k (returns UMAPCU_CAPACITY
 * otherwise). sigma/rho may be NULL. */
umapcu_status umapcu_construct_umap_graph(const int32_t *knn_idx, const float *knn_dist, uint32_t n,
                                          uint32_t k, const umapcu_graph_params *params,
                                          uint32_t n_epochs, uint64_t capacity, uint32_t *row,
                                          uint32_t *col, float *val, uint64_t *nnz, float *sigma,
                                          float *rho);

/* Replaces DensState::new (src/utils/density.rs:181-201): the constant
 * densMAP state from the symmetrised COO and the kNN lists. Writes
 * r[n], mu_sum[n], *mu_tot. Returns UMAPCU_DEGENERATE_LOCAL_RADII like the
 * reference. */
umapcu_status umapcu_dens_state_new(uint32_t n, uint64_t nnz, const uint32_t *row,
                                    const uint32_t *col, const float *val, const int32_t *knn_idx,
                                    const float *knn_dist, uint32_t k, int distances_squared,
                                    float *r, float *mu_sum, float *mu_tot);

/* ---------------------------------------------------------------------
 * Layout optimiser, host buffers (the "adam_gpu" slot)
 * ------------------------------------------------------------------- */

/* Replaces optimise_embedding_adam_gpu
 * (src/training/umap_optimiser_gpu.rs:1302-1369). embd is [n * n_dim]
 * row-major, optimised in place. The graph is the adjacency list
 * graph[i] = [(adj_col[p], adj_w[p]) for p in adj_ptr[i]..adj_ptr[i+1]]
 * (the reference's Vec<Vec<(usize, T)>>); only i < j entries are used.
 * dens may be NULL (plain UMAP). n_dim in 1..8. */
umapcu_status umapcu_optimise_embedding(float *embd, uint32_t n, uint32_t n_dim,
                                        const uint64_t *adj_ptr, const uint32_t *adj_col,
                                        const float *adj_w, const umapcu_optim_params *params,
                                        const umapcu_dens *dens, uint64_t seed, uint32_t optimiser,
                                        uint32_t sampler, int verbose);

/* ---------------------------------------------------------------------
 * Device-resident optimiser state (UmapGpuState, umap_optimiser_gpu.rs:
 * 278-453): upload once, run epochs, read back. Used for parity tests of
 * single epochs and by callers that keep the state on the GPU.
 * ------------------------------------------------------------------- */

typedef struct umapcu_state umapcu_state;

/* Replaces UmapCsrGraph::from_graph + UmapGpuState::upload
 * (umap_optimiser_gpu.rs:132-209, :374-452). Builds the CSR on the device.
 * Returns NO_DATA / NO_GRAPH_EDGES like the reference. */
umapcu_status umapcu_state_create(const float *embd, uint32_t n, uint32_t n_dim,
                                  const uint64_t *adj_ptr, const uint32_t *adj_col,
                                  const float *adj_w, const umapcu_optim_params *params,
                                  const umapcu_dens *dens, uint64_t seed, uint32_t sampler,
                                  umapcu_state **out);

void umapcu_state_destroy(umapcu_state *st);

/* Number of nodes / unique undirected edges / CSR entries of the state. */
umapcu_status umapcu_state_sizes(const umapcu_state *st, uint64_t *n, uint64_t *n_edges);

/* Reads back the device CSR (offsets[n+1], edge_idx[2E], other[2E],
 * eps[E], mu[E]); any pointer may be NULL. Same layout as UmapCsrGraph. */
umapcu_status umapcu_state_read_csr(const umapcu_state *st, uint32_t *offsets, uint32_t *edge_idx,
                                    uint32_t *other, float *eps, float *mu);

/* Runs epochs [first, first + count) of the loop at
 * umap_optimiser_gpu.rs:1336-1360 (densMAP update when active -> gradient
 * -> Adam/SGD step -> schedule advance). */
umapcu_status umapcu_state_run(umapcu_state *st, uint32_t first_epoch, uint32_t count,
                               uint32_t optimiser);

/* umapcu_state_run without the final synchronisation: the epochs are only
 * enqueued on the state's stream (see umapcu_state_set_stream), for callers
 * that order their own work, or time it with events, on that stream. */
umapcu_status umapcu_state_enqueue(umapcu_state *st, uint32_t first_epoch, uint32_t count,
                                   uint32_t optimiser);

/* One epoch with inspection hooks, for parity tests (mirrors
 * launch_grad_accum + launch_adam_update + launch_edge_schedule_update,
 * umap_optimiser_gpu.rs:1016-1227). injected: NULL or host [2E * neg_rate]
 * negative node per (CSR entry, negative). grad/has_update: NULL or host
 * [n * n_dim] / [n] outputs of the gradient pass. */
umapcu_status umapcu_state_epoch_debug(umapcu_state *st, uint32_t epoch, uint32_t optimiser,
                                       const uint32_t *injected, float *grad, uint32_t *has_update);

/* Reads the embedding / Adam moments [n * n_dim] and the per-edge
 * schedule cursors [E]; any pointer may be NULL. */
umapcu_status umapcu_state_read(const umapcu_state *st, float *embd, float *m, float *v,
                                float *cursor);

/* Restarts the run: embedding := embd (host [n * n_dim], NULL keeps the
 * current one), Adam moments := 0, schedule cursors := periods
 * (UmapGpuState::upload initial state, umap_optimiser_gpu.rs:410-441). */
umapcu_status umapcu_state_reset(umapcu_state *st, const float *embd);

/* x^b in the layout kernels: 0 (default) = 2^(b log2 x) on the MUFU units
 * (about 1e-6 relative error), 1 = CUDA's powf. */
umapcu_status umapcu_state_set_precise_pow(umapcu_state *st, int precise);

/* Launches the state's kernels on the caller's CUDA stream (a cudaStream_t
 * passed as void*); NULL restores the state's own stream. The caller must
 * order its own work on that stream. */
umapcu_status umapcu_state_set_stream(umapcu_state *st, void *cuda_stream);

/* umapcu_state_run with CUDA events around every launch: *epoch_ms is the
 * summed duration of the fused epoch kernels, *dens_ms of the densMAP
 * updates (either may be NULL). */
umapcu_status umapcu_state_run_profiled(umapcu_state *st, uint32_t first_epoch, uint32_t count,
                                        uint32_t optimiser, float *epoch_ms, float *dens_ms);

/* Overwrites embedding / moments ([n * n_dim], any may be NULL). */
umapcu_status umapcu_state_write(umapcu_state *st, const float *embd, const float *m,
                                 const float *v);

/* densMAP per-epoch state after the last density update (umap_dens_radii +
 * umap_dens_weights, umap_optimiser_gpu.rs:487-586, :1089-1143): re[n],
 * phi_sum[n], weight[n], *coeff, and the f32 statistics (mean, std, cov).
 * Forces a density update from the current embedding first. */
umapcu_status umapcu_state_dens_update(umapcu_state *st, float *re, float *phi_sum, float *weight,
                                       float *coeff, float *stats3);

/* ---------------------------------------------------------------------
 * Batched form: many independent layouts of uneven size advanced together
 * (no counterpart in the reference, which optimises one embedding per call
 * of optimise_embedding_adam_gpu, umap_optimiser_gpu.rs:1302-1369). Each
 * problem gives the arguments of one umapcu_optimise_embedding call; all
 * share n_dim (2..4) and n_epochs. Results equal the single-problem path's
 * for the same (embedding, graph, params, seed).
 * ------------------------------------------------------------------- */

typedef struct umapcu_batch umapcu_batch;

/* Uploads every problem and builds its CSR on the device. Arrays of
 * n_problems pointers / values; params and seeds per problem. With the
 * hash sampler and neg_sample_rate 5 everywhere it also precomputes each
 * problem's edge schedule as per-epoch bitmasks (1 bit per CSR entry and
 * epoch, held until umapcu_batch_destroy; not when they would take more
 * than half the free device memory, nor with UMAPCU_NO_SCHEDULE_LISTS set),
 * which the runs scan in place of the cursors with identical results. */
umapcu_status umapcu_batch_create(uint32_t n_problems, const uint32_t *n, uint32_t n_dim,
                                  const float *const *embd, const uint64_t *const *adj_ptr,
                                  const uint32_t *const *adj_col, const float *const *adj_w,
                                  const umapcu_optim_params *params, const uint64_t *seeds,
                                  uint32_t sampler, umapcu_batch **out);

void umapcu_batch_destroy(umapcu_batch *b);

/* Times the candidate launch configurations (persistent kernel with 4/6/8
 * CTAs per SM or one launch per epoch; scan super-chunk of 4 or 8 x 32
 * entries) on this batch for a few epochs and keeps the fastest. */
umapcu_status umapcu_batch_autotune(umapcu_batch *b, uint32_t *mode, uint32_t *ctas_per_sm, uint32_t *ku);

/* Runs all epochs of every problem from its initial state (one CUDA graph:
 * reset + the persistent launch, mode 1, or one launch per epoch, mode 2;
 * mode 0 = the autotuned configuration). *ms = device time of the run.
 * Returns UMAPCU_TIMEOUT if a bounded device wait gave up. */
umapcu_status umapcu_batch_run(umapcu_batch *b, uint32_t mode, float *ms);

/* Final embedding [n * n_dim] of one problem after umapcu_batch_run. */
umapcu_status umapcu_batch_read(const umapcu_batch *b, uint32_t problem, float *embd);

/* Failure-detection check of the persistent kernel's bounded waits: runs
 * the batch with the epoch barrier of one problem made unsatisfiable and a
 * wait limit of wait_limit polls; returns the status the kernel reported
 * (UMAPCU_TIMEOUT when the bound works). The batch must be rerun after. */
umapcu_status umapcu_batch_wait_check(umapcu_batch *b, uint32_t poisoned_problem, uint32_t wait_limit);

/* ---------------------------------------------------------------------
 * Served form: continuous batching of layout jobs (no counterpart in the
 * reference). A server thread owns the device: it admits submitted jobs in
 * arrival order within a device-memory budget and a job-count limit, and
 * every tick advances all admitted jobs by tick_epochs epochs -- each from
 * its own current epoch -- in one persistent launch. Each job's result equals
 * the single-problem path's for the same arguments, alone or in any mix.
 * All calls are thread-safe.
 * ------------------------------------------------------------------- */

typedef struct umapcu_server umapcu_server;

/* Starts a server on the current device. device_budget_bytes bounds the
 * summed peak-memory estimate of admitted jobs; all jobs share n_dim (2..4). */
umapcu_status umapcu_server_create(uint64_t device_budget_bytes, uint32_t max_jobs, uint32_t tick_epochs,
                                   uint32_t n_dim, umapcu_server **out);

/* The device-memory estimate the server's admission charges a job against
 * its budget (the CSR build's temporaries dominate): for placement front
 * ends that spread jobs over several servers. */
umapcu_status umapcu_server_job_bytes(uint32_t n, uint32_t n_dim, uint64_t nnz, uint32_t n_epochs,
                                      uint64_t *bytes);

/* Queues one job (the arguments of umapcu_optimise_embedding, copied) and
 * returns at once with its ticket. UMAPCU_CAPACITY if the job alone exceeds
 * the budget. */
umapcu_status umapcu_server_submit(umapcu_server *sv, uint32_t n, uint32_t n_dim, const float *embd,
                                   const uint64_t *adj_ptr, const uint32_t *adj_col, const float *adj_w,
                                   const umapcu_optim_params *params, uint64_t seed, uint32_t sampler,
                                   uint64_t *ticket);

/* Checkpoint of a job (no counterpart in the reference, which keeps a
 * layout's state only for the duration of one call,
 * umap_optimiser_gpu.rs:278-348): copies the job's current embedding (and,
 * when m / v are not NULL, its Adam moments) [n * n_dim] and the number of
 * epochs it has run. A running job is read between two ticks (the call waits
 * for the next tick boundary; the job keeps running); a job not admitted yet
 * returns the state it was submitted with. UMAPCU_BAD_ARG for a finished,
 * failed or unknown job, or one with a snapshot already in progress. */
umapcu_status umapcu_server_snapshot(umapcu_server *sv, uint64_t ticket, float *embd, float *m, float *v,
                                     uint32_t *epochs_done);

/* Queues a job that resumes from a snapshot: the arguments of the job's
 * umapcu_server_submit (same graph, parameters, seed and sampler) plus its
 * snapshot's embedding, moments and epoch count (< params->n_epochs). The
 * job runs epochs [epochs_done, n_epochs), its schedule cursors re-derived
 * from the edge periods, and its result equals the uninterrupted job's. */
umapcu_status umapcu_server_submit_resume(umapcu_server *sv, uint32_t n, uint32_t n_dim, const float *embd,
                                          const uint64_t *adj_ptr, const uint32_t *adj_col, const float *adj_w,
                                          const umapcu_optim_params *params, uint64_t seed, uint32_t sampler,
                                          const float *m, const float *v, uint32_t epochs_done, uint64_t *ticket);

/* *state: 0 pending, 1 running, 2 done, 3 failed or cancelled. */
umapcu_status umapcu_server_poll(umapcu_server *sv, uint64_t ticket, int *state);

/* Cancels a job that has not been admitted yet (its wait returns
 * UMAPCU_CANCELLED). */
umapcu_status umapcu_server_cancel(umapcu_server *sv, uint64_t ticket);

/* Blocks until the job finishes, copies its embedding [n * n_dim] (if
 * embd_out is not NULL) and forgets the ticket. *latency_s = submit to
 * completion, *queue_s = submit to admission. Returns the job's status. */
umapcu_status umapcu_server_wait(umapcu_server *sv, uint64_t ticket, float *embd_out, double *latency_s,
                                 double *queue_s);

umapcu_status umapcu_server_stats(umapcu_server *sv, uint64_t *completed, uint64_t *ticks,
                                  uint64_t *peak_bytes, uint32_t *peak_jobs);

/* Stops the server after the current tick; unfinished jobs fail with
 * UMAPCU_CANCELLED. */
void umapcu_server_destroy(umapcu_server *sv);

/* Layout optimisation that allocates no device memory. No counterpart in
 * the reference: for callers that cannot allocate device memory when they
 * need a layout (a host framework that has reserved the device for its own
 * allocator, or a deployment whose device-memory budget is fixed at
 * start-up). It is an ordinary host call (it makes CUDA runtime calls): never
 * call it from a stream callback or a host function node, where CUDA forbids
 * runtime calls. Runs all params->n_epochs Adam epochs (plain UMAP, no
 * densMAP) of the same fused epoch kernel as umapcu_optimise_embedding on
 * the caller's stream (a cudaStream_t passed as void*, NULL = legacy default
 * stream); returns once the work is enqueued. Inputs and outputs are device
 * memory owned by the caller: d_embd [n * n_dim] (in/out; 8-byte aligned for
 * n_dim = 2, 16-byte aligned for n_dim = 4, 4-byte aligned otherwise), the
 * optimiser CSR d_offsets [n + 1], d_other and d_period [n_entries] (4-byte
 * aligned; per CSR entry: other endpoint and edge sampling period, as
 * umapcu_state_read_csr returns them, periods expanded per entry through
 * edge_idx). A misaligned pointer returns UMAPCU_BAD_ARG before anything is
 * launched. All scratch (Adam moments, the second embedding buffer,
 * schedule cursors) lives in one 16 MiB device array that every GPU loading
 * the library holds until exit: a call needs 8 * n_entries + 12 * n * n_dim
 * bytes (each part rounded up to 256) of its first 16 MiB - 256 bytes, and
 * larger problems return UMAPCU_CAPACITY. The array is shared by every call
 * on a device and keeps the last call's contents (each call re-initialises
 * what it reads); calls that overlap on the GPU race on it. The library
 * built with UMAPCU_CHECKED (libumapcu_checked.so) also bounds-checks the
 * caller's CSR on the device (offsets in order and within n_entries, other
 * endpoints below n), skips any access outside it, returns UMAPCU_BAD_ARG,
 * and for that waits for the epochs before returning. The first call on a
 * device looks the
 * array's device address up (cudaGetSymbolAddress) and, under CUDA's default
 * lazy module loading, is also when the library's device code and this
 * array are loaded onto that device, which takes device memory: make one
 * call per device at start-up, before the caller reserves the device's
 * memory and before any stream capture (or run with
 * CUDA_MODULE_LOADING=EAGER). */
umapcu_status umapcu_optimise_csr_noalloc(float *d_embd, uint32_t n, uint32_t n_dim,
                                          const uint32_t *d_offsets, const uint32_t *d_other,
                                          const float *d_period, uint64_t n_entries,
                                          const umapcu_optim_params *params, uint64_t seed,
                                          uint32_t sampler, void *cuda_stream);

/* ---------------------------------------------------------------------
 * Kernel-level test hooks (host buffers), each the reference launcher it
 * names, run through the same device functions as the fused epoch kernel.
 * ------------------------------------------------------------------- */

/* umap_adam_update + launch_adam_update (umap_optimiser_gpu.rs:887-923,
 * :1155-1196): in place on m, v, embd ([n * n_dim]). */
umapcu_status umapcu_adam_update(const float *grad, const uint32_t *has_update, float *m, float *v,
                                 float *embd, uint32_t n, uint32_t n_dim,
                                 const umapcu_optim_params *params, uint32_t epoch);

/* umap_edge_schedule_update (umap_optimiser_gpu.rs:940-955): in place on
 * cursor[n_edges]. */
umapcu_status umapcu_edge_schedule_update(const float *eps, float *cursor, uint64_t n_edges,
                                          uint32_t epoch);

/* x^b as the layout kernels evaluate it (F::powf in umap_grad_accum and
 * umap_dens_radii, umap_optimiser_gpu.rs:528, :754, :832), for x > 0:
 * out[i] = x[i]^b; precise selects CUDA's powf. */
umapcu_status umapcu_eval_pow(const float *x, uint32_t n, float b, int precise, float *out);

/* gpu_hash_neg (umap_optimiser_gpu.rs:611-624) and the Philox sampler,
 * evaluated on the device for count consecutive neg indices. */
umapcu_status umapcu_sample_negatives(uint32_t sampler, uint64_t seed, uint32_t node,
                                      uint32_t entry, uint32_t epoch, uint32_t edge_local,
                                      uint32_t count, uint32_t n, uint32_t *out);

/* Schedule lists of a state (no reference counterpart): a state made by
 * umapcu_state_create precomputes, for every epoch of params.n_epochs, the
 * CSR entries the edge schedule (umap_optimiser_gpu.rs:940-955) activates
 * (the same f32 cursor arithmetic), so its epochs read those records instead
 * of scanning every entry's cursor. Results are bit-identical to the scan;
 * runs that skip or repeat epochs fall back to the scan until
 * umapcu_state_reset. The one-shot umapcu_optimise_embedding (and a state
 * whose lists do not fit in half the free device memory) precomputes the
 * same schedule as per-epoch bitmasks instead (1 bit per CSR entry and
 * epoch; its epochs scan the bits in place of the cursors), again
 * bit-identical. Set UMAPCU_NO_SCHEDULE_LISTS to disable both forms.
 * lists_active: 1 when lists are built; n_records: records held (8 bytes
 * each); build_ms: list build time. */
umapcu_status umapcu_state_schedule_info(const umapcu_state *st, int *lists_active, uint64_t *n_records,
                                         float *build_ms);

/* Precomputed forms of the edge schedule a state can hold (see
 * umapcu_state_schedule_info): none (every epoch scans and advances the
 * cursors), per-epoch bitmasks, or per-epoch record lists. */
enum { UMAPCU_SCHED_SCAN = 0, UMAPCU_SCHED_BITS = 1, UMAPCU_SCHED_LISTS = 2 };

/* Replaces the state's precomputed schedule by `form`, built now from the
 * edge periods on the state's stream (bitmasks: asynchronously, without a
 * host synchronisation when nothing was held before; lists: synchronously).
 * Results are bit-identical in every form. UMAPCU_CAPACITY when the form
 * does not fit (half the free device memory); the state then scans. */
umapcu_status umapcu_state_set_schedule(umapcu_state *st, uint32_t form);

/* The form the state holds now (UMAPCU_SCHED_*). */
umapcu_status umapcu_state_schedule_form(const umapcu_state *st, uint32_t *form);

/* ---------------------------------------------------- memory hygiene
 * (no counterpart in the reference, whose UmapGpuState holds device memory
 * for one call only, umap_optimiser_gpu.rs:278-348). The library keeps two
 * things between calls: the one-shot call's schedule-bitmask block (one per
 * device, up to 1 bit per CSR entry and epoch) and, in each device's default
 * stream-ordered memory pool (a process-wide object), the blocks its calls
 * freed -- it raises that pool's release threshold, which otherwise returns
 * freed memory to the driver at every synchronisation. */

/* keep = 0: put back every pool release threshold the library raised (and
 * trim those pools), and leave the pools alone from now on; keep = 1 (the
 * default): raise them again on the next call. */
umapcu_status umapcu_set_pool_retention(int keep);

/* Frees the current device's cached bitmask block and trims its default
 * pool to the memory in use. */
umapcu_status umapcu_release_cached(void);

/* Devices (no counterpart in the reference, which takes one device per
 * call). Every entry point works on the calling thread's current CUDA
 * device; a multi-device front end selects it per call. */
umapcu_status umapcu_device_count(int *count);
umapcu_status umapcu_set_device(int device);

/* Measurement hook: the rate of random 8-byte gathers from an L2-resident
 * table of table_bytes (4 KiB .. 64 MiB), in GB/s of gathered bytes -- the
 * load form of the epoch kernel's coordinate gathers (float2 rows,
 * evict_last L2 policy), so the denominator of its L2 roofline. */
umapcu_status umapcu_probe_l2_gather(uint64_t table_bytes, float *gbs);

/* ------------------------------------------------ kNN, metrics, kNN cache */

/* Distance metrics of the neighbour search (NearestNeighbourParams::
 * dist_metric, src/data/nearest_neighbours.rs:44, "euclidean" | "cosine").
 * Euclidean distances are returned SQUARED, as the reference's ANN backends
 * return them (src/lib.rs:435); cosine distance is 1 - <x/|x|, y/|y|>. */
enum { UMAPCU_METRIC_EUCLIDEAN_SQ = 0, UMAPCU_METRIC_COSINE = 1 };

/* Exact k nearest neighbours of every row of x [n * dim] (host), self
 * excluded: replaces run_ann_search with AnnSearch::Exhaustive
 * (src/data/nearest_neighbours.rs:225-364, which queries k + 1 and drops the
 * first) as the source of the precomputed kNN (PreComputedKnn, src/lib.rs:79).
 * knn_idx / knn_dist [n * k] (host), ascending by distance, ties by index.
 * Each distance is the sequential f32 FMA chain over the dimensions in order
 * (d = fma(x_i - y_i, x_i - y_i, d)). Needs 0 < k <= 32 and n > k. */
umapcu_status umapcu_knn_exact(const float *x, uint32_t n, uint32_t dim, uint32_t k, uint32_t metric,
                               int32_t *knn_idx, float *knn_dist);

/* The same on device buffers, for the rows d_queries [n_queries] of d_x
 * (nullptr: every row, n_queries = n), on `stream` (cudaStream_t; nullptr =
 * legacy default stream). d_idx / d_dist [n_queries * k]. */
umapcu_status umapcu_knn_exact_dev(const float *d_x, uint32_t n, uint32_t dim, const uint32_t *d_queries,
                                   uint32_t n_queries, uint32_t k, uint32_t metric, uint32_t *d_idx,
                                   float *d_dist, void *stream);

/* Embedding quality (no reference counterpart; the reference has no
 * metrics). trust: trustworthiness@k with sklearn.manifold.trustworthiness's
 * definition over the query rows (all rows when queries is nullptr, then
 * equal to sklearn's value up to f32 distance rounding); knn_preservation:
 * mean |kNN_X(i)[:k] & kNN_Y(i)| / k with kNN_X from knn_idx [n * knn_k].
 * Either output may be nullptr. Needs 2k < n. */
umapcu_status umapcu_embedding_quality(const float *x, uint32_t n, uint32_t dim, const float *y, uint32_t n_dim,
                                       const int32_t *knn_idx, uint32_t knn_k, uint32_t k,
                                       const uint32_t *queries, uint32_t n_queries, uint32_t metric,
                                       double *trust, double *knn_preservation);

/* Fuzzy cross-entropy of an embedding against its graph (COO, host):
 * sum over entries of w log(w/q) + (1-w) log((1-w)/(1-q)),
 * q = 1 / (1 + a |y_i - y_j|^(2b)), q and w clamped to [1e-12, 1 - 1e-12],
 * in f64. */
umapcu_status umapcu_fuzzy_cross_entropy(const uint32_t *row, const uint32_t *col, const float *w, uint64_t nnz,
                                         const float *y, uint32_t n, uint32_t n_dim, float a, float b,
                                         double *out);

/* kNN cache file (no reference counterpart: the reference keeps
 * PreComputedKnn in memory, src/lib.rs:79). Little-endian: a 48-byte header
 * {"UMAPKNN\0", u32 version = 1, u32 metric, u64 n, u32 k, u32 flags
 * (bit 0: self excluded), u64 payload checksum (FNV-1a 64 over the payload),
 * u64 reserved = 0}, then idx i32 [n * k], then dist f32 [n * k]. Loading
 * checks magic, version, sizes and checksum (UMAPCU_BAD_ARG on mismatch). */
umapcu_status umapcu_knn_save(const char *path, uint32_t n, uint32_t k, uint32_t metric, const int32_t *knn_idx,
                              const float *knn_dist);
umapcu_status umapcu_knn_load_header(const char *path, uint32_t *n, uint32_t *k, uint32_t *metric);
umapcu_status umapcu_knn_load(const char *path, uint32_t n, uint32_t k, int32_t *knn_idx, float *knn_dist);

/* ------------------------------------------------------- spectral init */

/* Smallest eigenpairs of a symmetric sparse matrix (CSR host arrays, f64
 * values): replaces compute_smallest_eigenpairs_lanczos
 * (src/utils/math.rs:617-628). min(4 k + 30, n) Lanczos steps on the device
 * with full reorthogonalisation, early stop on breakdown. evals [k]
 * ascending, evecs [n * k] (row i = point i); *n_found <= n_components
 * (fewer after an early breakdown, as in the reference). */
umapcu_status umapcu_smallest_eigenpairs(uint32_t n, const uint64_t *ptr, const uint32_t *col, const double *val,
                                         uint32_t n_components, uint64_t seed, float *evals, float *evecs,
                                         uint32_t *n_found);

/* Spectral initialisation of a symmetric graph (COO host arrays): replaces
 * spectral_layout without a data matrix (src/data/init.rs:986-1004).
 * Connected: eigenvectors 1..n_comp of -D^-1/2 A D^-1/2, centred, scaled so
 * the largest |coordinate| is `range` (<= 0: 10), plus N(0, 1e-4) noise.
 * Several components: centroids on the simplex, each component's spectral
 * layout (random when it has fewer than 2 n_comp points) around its
 * centroid, then centred and scaled. embd [n * n_comp]. The Lanczos start
 * vector, the random fallbacks and the noise come from this library's own
 * seeded streams, not the reference's StdRng. */
umapcu_status umapcu_spectral_layout(const uint32_t *row, const uint32_t *col, const float *val, uint64_t nnz,
                                     uint32_t n, uint32_t n_comp, uint64_t seed, float range, float *embd);

#ifdef __cplusplus
}
#endif

#endif /* UMAPCU_H */
