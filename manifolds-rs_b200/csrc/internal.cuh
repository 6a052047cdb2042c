// Shared internals of the umapcu CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "umapcu.h"

namespace umapcu {

// A named NVTX range for the scope (stages of the entry points: graph, CSR
// build, schedule, epochs, admission, ticks, ...). Header-only NVTX: without
// a profiler attached a range costs a function call and nothing else.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// Internal error carrier: thrown inside the library, caught at the C ABI.
struct Error {
    umapcu_status status;
    const char *what;
};

[[noreturn]] inline void fail(umapcu_status s, const char *what) { throw Error{s, what}; }

inline void check_cuda(cudaError_t e, const char *what, umapcu_status kind = UMAPCU_CUDA_LAUNCH)
{
    if (e != cudaSuccess) {
        if (e == cudaErrorMemoryAllocation) kind = UMAPCU_CUDA_ALLOC;
        if (getenv("UMAPCU_DEBUG"))
            fprintf(stderr, "umapcu: %s failed: %s\n", what, cudaGetErrorString(e));
        cudaGetLastError();
        fail(kind, what);
    }
}

#define UMAPCU_CK(x) ::umapcu::check_cuda((x), #x)

// Stream-ordered device buffer (cudaMallocAsync / cudaFreeAsync).
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    DevBuf() = default;
    DevBuf(size_t count, cudaStream_t stream) { alloc(count, stream); }
    void alloc(size_t count, cudaStream_t stream)
    {
        release();
        s = stream;
        n = count;
        if (count) check_cuda(cudaMallocAsync((void **)&p, count * sizeof(T), stream), "cudaMallocAsync",
                              UMAPCU_CUDA_ALLOC);
    }
    void release()
    {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept
    {
        if (this != &o) { release(); p = o.p; n = o.n; s = o.s; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    size_t bytes() const { return n * sizeof(T); }
};

// RAII stream owned by one API call / state.
struct Stream {
    cudaStream_t s = nullptr;
    Stream() { check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate"); }
    // highest = true: the device's greatest stream priority (its CTAs are
    // dispatched ahead of default-priority work as SMs free up)
    explicit Stream(bool highest)
    {
        int lo = 0, hi = 0;
        check_cuda(cudaDeviceGetStreamPriorityRange(&lo, &hi), "cudaDeviceGetStreamPriorityRange");
        check_cuda(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, highest ? hi : lo), "cudaStreamCreate");
    }
    ~Stream()
    {
        if (s) { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
    }
    Stream(const Stream &) = delete;
    Stream &operator=(const Stream &) = delete;
};

// RAII event without timing: ordering between streams.
struct Event {
    cudaEvent_t e = nullptr;
    Event() { check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate"); }
    ~Event()
    {
        if (e) cudaEventDestroy(e);
    }
    Event(const Event &) = delete;
    Event &operator=(const Event &) = delete;
    void record(cudaStream_t s) { check_cuda(cudaEventRecord(e, s), "cudaEventRecord"); }
};

template <typename T>
inline void h2d(T *dst, const T *src, size_t count, cudaStream_t s)
{
    if (count) check_cuda(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, s), "h2d");
}
template <typename T>
inline void d2h(T *dst, const T *src, size_t count, cudaStream_t s)
{
    if (count) check_cuda(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, s), "d2h");
}
inline void sync(cudaStream_t s) { check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize"); }
inline void check_launch(const char *what) { check_cuda(cudaGetLastError(), what); }

inline unsigned ceil_div(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

int device_sm_count();
// Keeps freed stream-ordered allocations cached in the current device's
// default pool (release threshold raised from 0); set once per device, and
// not at all after umapcu_set_pool_retention(0).
void keep_pool_memory();

// launch_adam_update host scalars (umap_optimiser_gpu.rs:1164-1175), f32:
// fused = lr * (1 - e/N) * ad_scale, epsc = sqrt(1 - beta2^t) * eps, and the
// plain learning-rate schedule lr * (1 - e/N).
inline void epoch_scalars(const umapcu_optim_params &p, uint32_t epoch, float *fused, float *epsc, float *lr_e)
{
    const float one = 1.0f;
    float lr_alpha = p.lr * (one - (float)epoch / (float)p.n_epochs);
    float t = (float)(epoch + 1);
    float beta1t = powf(p.beta1, t);
    float beta2t = powf(p.beta2, t);
    float sqrt_b2t1 = sqrtf(one - beta2t);
    float ad_scale = sqrt_b2t1 / (one - beta1t);
    *epsc = sqrt_b2t1 * p.eps;
    *fused = lr_alpha * ad_scale;
    *lr_e = lr_alpha;
}

// ------------------------------------------------------------------ graph

struct DeviceCoo {
    DevBuf<uint32_t> row, col;
    DevBuf<float> val;
    uint64_t nnz = 0;
};

// smooth_knn_dist on device buffers (graph.rs:499-565).
void smooth_knn_dist_dev(const float *d_dist, uint32_t n, uint32_t k, float local_connectivity,
                         float bandwidth, uint32_t n_iter, float *d_sigma, float *d_rho, cudaStream_t s);

// The full graph stage (lib.rs:296-306) on device buffers; the kNN arrays
// stay owned by the caller.
void construct_graph_dev(const int32_t *d_idx, const float *d_dist, uint32_t n, uint32_t k,
                         const umapcu_graph_params &gp, uint32_t n_epochs, DeviceCoo &out,
                         float *d_sigma, float *d_rho, cudaStream_t s);

// densMAP constant state (density.rs:181-201) on device buffers.
umapcu_status dens_state_dev(uint32_t n, uint64_t nnz, const uint32_t *d_row, const uint32_t *d_col,
                             const float *d_val, const int32_t *d_idx, const float *d_dist, uint32_t k,
                             int distances_squared, float *d_r, float *d_mu_sum, float *h_mu_tot,
                             cudaStream_t s);

// Optimiser CSR (UmapCsrGraph::from_graph, umap_optimiser_gpu.rs:132-209),
// stored per CSR entry: other node, edge id, (cursor, period) schedule,
// edge weight.
struct DeviceCsr {
    uint32_t n = 0;
    uint64_t n_edges = 0;
    DevBuf<uint32_t> offsets;   // [n + 1]
    DevBuf<uint32_t> other;     // [2E + 8] (8 padding entries)
    DevBuf<uint32_t> edge_id;   // [2E]
    DevBuf<float2> sched;       // [2E + 8] (cursor, period); 8 padding entries for 16-byte copies
    DevBuf<float> mu_entry;     // [2E] edge weight per entry (densMAP)
    DevBuf<float> eps;          // [E] period per edge
    DevBuf<float> mu;           // [E] weight per edge
};

// Builds the optimiser CSR from a device adjacency (adj_ptr [n+1], u64).
// Returns NO_DATA / NO_GRAPH_EDGES / OK.
umapcu_status build_csr_dev(uint32_t n, const uint64_t *d_adj_ptr, const uint32_t *d_adj_col,
                            const float *d_adj_w, uint64_t nnz, DeviceCsr &csr, cudaStream_t s);

// The same build in two phases: the structure needs only the row pointers
// and columns (everything but the weights, periods and schedule), so it can
// run while the weights are still being copied; the weights phase then
// completes the CSR. `tmp` carries the edges' adjacency positions between
// the two.
struct CsrBuild {
    DevBuf<uint32_t> epos;  // [E] adjacency position of each edge's upper entry
};
umapcu_status build_csr_structure(uint32_t n, const uint64_t *d_adj_ptr, const uint32_t *d_adj_col, uint64_t nnz,
                                  DeviceCsr &csr, CsrBuild &tmp, cudaStream_t s);
void build_csr_weights(const float *d_adj_w, DeviceCsr &csr, CsrBuild &tmp, cudaStream_t s);

// Several graphs built as one (the served form's admission). The graphs'
// adjacencies are concatenated: lptr holds each graph's own row pointers
// (graph t's n_t + 1 entries start at lptr + node_base[t] + t, counting from
// 0), adj_col / adj_w its entries from job_entry_base[t], columns local to
// the graph; node_base [n_jobs + 1] and job_entry_base [n_jobs + 1] are the
// graphs' first global node and first entry. The CSR spans all nodes; each
// node's row equals the single-graph build's (same entries in the same order,
// `other` local to the graph, periods normalised by the graph's own maximum
// weight), so graph t's slice (offsets + node_base[t], the shared other /
// sched arrays) is a drop-in for its own build. h_job_edges [n_jobs] receives
// edges per graph. A column outside its graph returns BAD_ARG.
umapcu_status build_csr_multi(uint32_t n_total, uint32_t n_jobs, const uint32_t *d_node_base,
                              const uint64_t *d_job_entry_base, const uint64_t *d_lptr, const uint32_t *d_adj_col,
                              const float *d_adj_w, uint64_t nnz, DeviceCsr &csr, uint64_t *h_job_edges,
                              cudaStream_t s);

// Exact kNN of the rows d_qidx [nq] of d_x (nullptr: rows 0..nq-1), self
// excluded, ascending (distance, index); knn.cu.
void knn_dev(const float *d_x, uint32_t n, uint32_t dim, const uint32_t *d_qidx, uint32_t nq, uint32_t k,
             uint32_t metric, uint32_t *d_idx, float *d_dist, cudaStream_t s);
// d_counts [nq][k]: points strictly before each given neighbour in the
// query's (distance, index) order, self excluded; knn.cu.
void knn_rank_dev(const float *d_x, uint32_t n, uint32_t dim, const uint32_t *d_qidx, uint32_t nq,
                  const uint32_t *d_nbr, uint32_t k, uint32_t metric, uint32_t *d_counts, cudaStream_t s);

// Per-epoch lists of active CSR entries (schedule.cu): rec [n_records]
// (entry, other endpoint), the entry packed as (node index within its
// 32-node segment << kRecNodeShift) | offset within the node's row;
// ptr [n_epochs * n_units + 1] record offsets per (epoch, work unit);
// unit_base [nseg + 1] each segment's first work unit. Lists are not built
// for a graph with a node of kRecOffsetMask + 1 or more entries.
constexpr uint32_t kRecNodeShift = 27;
constexpr uint32_t kRecOffsetMask = (1u << kRecNodeShift) - 1u;
struct ScheduleLists {
    DevBuf<uint2> rec;
    DevBuf<uint64_t> ptr;
    DevBuf<uint32_t> unit_base;
    uint64_t n_records = 0;
    uint32_t n_epochs = 0, nseg = 0, n_units = 0;
};
// Builds the lists for epochs [0, n_epochs) from the reset schedule (cursor
// = period); false when they would not fit (half the free device memory) or
// n_epochs is out of range, `out` then empty.
bool build_schedule_lists(const DeviceCsr &csr, uint32_t n_epochs, ScheduleLists &out, cudaStream_t s);
// Per-epoch bitmasks of active CSR entries (schedule.cu): bits
// [n_epochs][words], bit p & 31 of word p >> 5 of epoch e set when entry p
// is active in epoch e (words = ceil(2E / 32)). 1 bit per entry and epoch
// against the lists' 8 bytes per active entry, and built in well under a
// millisecond at 1M points: the precomputed schedule of a one-shot run.
// The buffer comes from a per-device cache (one block, grown to the largest
// request, kept between calls): a one-shot call then allocates no more
// stream-ordered pool memory than it would without the bitmasks.
struct ScheduleBits {
    uint32_t *bits = nullptr;
    size_t cap = 0;  // words of the held block
    int dev = -1;
    cudaStream_t built_on = nullptr;  // synchronised before the block goes back to the cache
    uint64_t words = 0;
    uint32_t n_epochs = 0;
    // Epochs [first, n_epochs) are written on `side` and complete with
    // `rest` (first = 0: all on built_on); users wait for `rest` before
    // epoch `first`.
    uint32_t first = 0;
    cudaStream_t side = nullptr;
    cudaEvent_t rest = nullptr;
    cudaStream_t waited = nullptr;  // the stream that last waited for `rest`
    ScheduleBits() = default;
    ScheduleBits(const ScheduleBits &) = delete;
    ScheduleBits &operator=(const ScheduleBits &) = delete;
    ~ScheduleBits() { release(); }
    // Gives the block back (to the device's cache when it is empty, else to
    // the driver) once the stream that built it is idle; `bits` then null.
    void release();
};
// Frees the current device's cached bitmask block (none cached: no-op).
void release_cached_bits();
// Builds the bitmasks for epochs [0, n_epochs) from the reset schedule;
// false when they would not fit (half the free device memory), `out` then
// empty.
bool build_schedule_bits(const DeviceCsr &csr, uint32_t n_epochs, ScheduleBits &out, cudaStream_t s);
// Epochs whose bit words build_schedule_bits writes before the rest, for
// bitmasks of at least kBitsSplitWords words (64 MB; smaller ones are built
// in one launch).
constexpr uint32_t kBitsFirst = 8;
constexpr size_t kBitsSplitWords = (size_t)16 << 20;
// The bitmask kernel alone: bits [n_epochs][ceil(n_entries / 32)] of the
// entries' reset schedule (sched[p].y = period), into caller memory; only
// the words of epochs [e_begin, n_epochs) are written.
void launch_schedule_bits(const float2 *sched, uint64_t n_entries, uint32_t n_epochs, uint32_t *bits,
                          cudaStream_t s, uint32_t e_begin = 0);

// Writes into csr.sched the cursors after `epochs` epochs from the reset
// schedule (the state the per-epoch scan would have left).
void materialise_schedule(DeviceCsr &csr, uint32_t epochs, cudaStream_t s);
// The same for the `count` entries from offsets[node_lo] on (one job's rows
// of a multi-graph CSR).
void materialise_schedule_range(DeviceCsr &csr, uint32_t node_lo, uint64_t count, uint32_t epochs, cudaStream_t s);

// Resets every entry's schedule cursor to its period (upload state,
// umap_optimiser_gpu.rs:425-430).
void reset_schedule_dev(DeviceCsr &csr, cudaStream_t s);

}  // namespace umapcu
