// C ABI of umapcu: host runtime around the graph and layout kernels.
//
// The host side mirrors optimise_embedding_adam_gpu
// (src/training/umap_optimiser_gpu.rs:1302-1369): upload once, run the
// epoch loop on one stream, read the embedding back once. Per-epoch scalars
// (learning-rate schedule, Adam bias correction) are evaluated on the host
// in f32 exactly as launch_adam_update does (:1164-1175). densMAP statistics
// stay on the device (no per-epoch readback).
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <atomic>
#include <chrono>
#include <memory>
#include <mutex>

#include "internal.cuh"
#include "layout.cuh"

using namespace umapcu;

// ------------------------------------------------------------------ state

struct umapcu_state {
    Stream own;
    struct {
        cudaStream_t s = nullptr;
    } stream;
    uint32_t n = 0, n_dim = 0;
    umapcu_optim_params p{};
    uint64_t seed = 0;
    uint32_t sampler = UMAPCU_NEG_REF_HASH;
    bool precise_pow = false;
    DeviceCsr csr;
    DevBuf<float> y[2];
    int cur = 0;
    DevBuf<float> m, v;
    bool dens = false;
    float lambda = 0, frac = 0, var_shift = 0, mu_tot = 0;
    DevBuf<float> r;
    DevBuf<float4> dens_node;
    DevBuf<double> part;
    DevBuf<uint32_t> ticket;
    DevBuf<float> stats;
    // schedule lists (schedule.cu): usable while the epochs run so far are
    // 0, 1, ..., sched_epoch - 1 from the reset schedule; the cursors in
    // csr.sched then lag (sched_lazy) until something needs them
    ScheduleLists lists;
    ScheduleBits bits;  // the bitmask form, used when there are no lists
    DevBuf<uint32_t> err;  // checked builds: a kernel's report of a bad index
    bool lists_ok = false, bits_ok = false, sched_continuous = true, sched_lazy = false;
    uint32_t sched_epoch = 0;
    float lists_build_ms = 0.0f;
};

namespace {

template <typename F>
umapcu_status guard(F &&f)
{
    try {
        return f();
    } catch (const Error &e) {
        return e.status;
    } catch (const std::bad_alloc &) {
        return UMAPCU_CUDA_ALLOC;
    } catch (...) {
        return UMAPCU_CUDA_LAUNCH;
    }
}

// DensState::is_active (density.rs:244-250), T = f32
bool dens_active(float lambda, float frac, uint32_t epoch, uint32_t n_epochs)
{
    if (lambda <= 0.0f || n_epochs == 0) return false;
    float progress = (float)(epoch + 1) / (float)n_epochs;
    return progress > 1.0f - frac;
}

void validate_params(const umapcu_optim_params *p, uint32_t n_dim)
{
    if (!p) fail(UMAPCU_BAD_ARG, "params is null");
    if (n_dim < 1 || n_dim > 8) fail(UMAPCU_BAD_ARG, "n_dim must be in 1..8");
    if (p->n_epochs == 0) fail(UMAPCU_BAD_ARG, "n_epochs must be positive");
}

void dens_update(umapcu_state *st)
{
    DensArgs D{};
    D.n = st->n;
    D.offsets = st->csr.offsets.p;
    D.other = st->csr.other.p;
    D.y = st->y[st->cur].p;
    D.a = st->p.a;
    D.b = st->p.b;
    D.r = st->r.p;
    D.dens_node = st->dens_node.p;
    D.part = st->part.p;
    D.ticket = st->ticket.p;
    D.stats = st->stats.p;
    D.var_shift = st->var_shift;
    D.lambda = st->lambda;
    D.mu_tot = st->mu_tot;
    D.precise_pow = st->precise_pow;
    D.n_entries = 2 * st->csr.n_edges;
    D.err = st->err.p;
    launch_dens_update(D, st->n_dim, st->stream.s);
}

// Cursors in csr.sched brought up to date (after list-mode epochs).
void sync_cursors(umapcu_state *st)
{
    if (!st->sched_lazy) return;
    materialise_schedule(st->csr, st->sched_epoch, st->stream.s);
    st->sched_lazy = false;
}

// Checked builds: the status a kernel reported since the last look (the
// word is cleared); other builds: UMAPCU_OK without touching the device.
umapcu_status take_error(umapcu_state *st)
{
#ifdef UMAPCU_CHECKED
    uint32_t h = 0;
    d2h(&h, st->err.p, 1, st->stream.s);
    check_cuda(cudaMemsetAsync(st->err.p, 0, sizeof(uint32_t), st->stream.s), "memset err");
    sync(st->stream.s);
    return (umapcu_status)h;
#else
    (void)st;
    return UMAPCU_OK;
#endif
}

void run_epoch(umapcu_state *st, uint32_t epoch, uint32_t optimiser, const uint32_t *d_inj, float *d_grad,
               uint32_t *d_act, bool skip_dens = false)
{
    const bool dens_on = st->dens && dens_active(st->lambda, st->frac, epoch, st->p.n_epochs);
    if (dens_on && !skip_dens) dens_update(st);
    const bool in_order = st->sched_continuous && epoch == st->sched_epoch;
    const bool use_lists = st->lists_ok && in_order && epoch < st->lists.n_epochs;
    const bool use_bits = !use_lists && st->bits_ok && in_order && epoch < st->bits.n_epochs;
    if (!use_lists && !use_bits) sync_cursors(st);  // the scan reads and advances the cursors
    if (!in_order) st->sched_continuous = false;
    EpochArgs A{};
    if (use_lists) {
        A.rec = st->lists.rec.p;
        A.seg_ptr = st->lists.ptr.p + (size_t)epoch * st->lists.n_units;
        A.seg_unit = st->lists.unit_base.p;
        st->sched_lazy = true;
    } else if (use_bits) {
        A.bits = st->bits.bits + (size_t)epoch * st->bits.words;
        st->sched_lazy = true;
        if (st->bits.rest && epoch >= st->bits.first && st->bits.waited != st->stream.s) {
            // the later epochs' words (build_schedule_bits): once per stream
            check_cuda(cudaStreamWaitEvent(st->stream.s, st->bits.rest, 0), "cudaStreamWaitEvent");
            st->bits.waited = st->stream.s;
        }
    }
    if (in_order) st->sched_epoch = epoch + 1;
    A.n = st->n;
    A.offsets = st->csr.offsets.p;
    A.other = st->csr.other.p;
    A.sched = st->csr.sched.p;
    A.mu_entry = st->csr.mu_entry.p;
    A.y_cur = st->y[st->cur].p;
    A.y_next = st->y[st->cur ^ 1].p;
    A.m = st->m.p;
    A.v = st->v.p;
    A.dens_node = st->dens_node.p;
    A.dens_stats = st->stats.p;
    A.injected = d_inj;
    A.dbg_grad = d_grad;
    A.dbg_active = d_act;
    A.epoch = epoch;
    A.epoch_f = (float)epoch;
    epoch_scalars(st->p, epoch, &A.fused, &A.epsc, &A.lr_sgd);
    A.a = st->p.a;
    A.b = st->p.b;
    A.two_a_b = 2.0f * st->p.a * st->p.b;
    A.two_gamma_b = 2.0f * st->p.gamma * st->p.b;
    A.omb1 = 1.0f - st->p.beta1;
    A.omb2 = 1.0f - st->p.beta2;
    A.neg_rate = st->p.neg_sample_rate;
    A.sampler = st->sampler;
    A.seed32 = (uint32_t)st->seed;
    A.seed_lo = (uint32_t)st->seed;
    A.seed_hi = (uint32_t)(st->seed >> 32);
    A.fastmod_M = fastmod_magic(st->n);
    A.optimiser = optimiser;
    A.precise_pow = st->precise_pow;
    A.n_entries = 2 * st->csr.n_edges;
    A.err = st->err.p;
    launch_epoch(A, st->n_dim, dens_on, st->stream.s);
    st->cur ^= 1;
}

// Optional phase timing of the host-buffer entry points (UMAPCU_TIMING=1):
// synchronises at each mark and prints the elapsed wall time to stderr.
struct PhaseTimer {
    bool on = getenv("UMAPCU_TIMING") != nullptr;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    void mark(const char *what, cudaStream_t s)
    {
        if (!on) return;
        sync(s);
        auto t1 = std::chrono::steady_clock::now();
        fprintf(stderr, "umapcu timing: %-18s %9.3f ms\n", what,
                std::chrono::duration<double, std::milli>(t1 - t0).count());
        t0 = t1;
    }
};


umapcu_status create_state(const float *embd, uint32_t n, uint32_t n_dim, const uint64_t *adj_ptr,
                           const uint32_t *adj_col, const float *adj_w, const umapcu_optim_params *params,
                           const umapcu_dens *dens, uint64_t seed, uint32_t sampler,
                           std::unique_ptr<umapcu_state> &out, bool lists)
{
    if (n == 0) return UMAPCU_NO_DATA;
    if (!embd || !adj_ptr) return UMAPCU_BAD_ARG;
    validate_params(params, n_dim);
    if (sampler > UMAPCU_NEG_PHILOX) return UMAPCU_BAD_ARG;
    const uint64_t nnz = adj_ptr[n];
    if (nnz && (!adj_col || !adj_w)) return UMAPCU_BAD_ARG;
    if (dens && (!dens->r)) return UMAPCU_BAD_ARG;
    keep_pool_memory();
    auto st = std::make_unique<umapcu_state>();
    st->stream.s = st->own.s;
    cudaStream_t s = st->stream.s;
    PhaseTimer T;
    st->n = n;
    st->n_dim = n_dim;
    st->p = *params;
    st->seed = seed;
    st->sampler = sampler;
    const uint64_t nt = (uint64_t)n * n_dim;
    st->y[0].alloc(nt, s);
    st->y[1].alloc(nt, s);
    st->m.alloc(nt, s);
    st->v.alloc(nt, s);
    {
        // The row pointers and columns go first; the weights (then the
        // embedding) follow on a second stream while the CSR's structure is
        // built from the former (build_csr_structure), and the weights phase
        // waits for them.
        NvtxRange r("umapcu graph upload + CSR build");
        DevBuf<uint64_t> dptr(n + 1, s);
        DevBuf<uint32_t> dcol(nnz, s);
        DevBuf<float> dw(nnz, s);
        Event col_in, w_in;
        Stream side;  // declared after dw: on unwinding it is synchronised before dw is freed
        h2d(dptr.p, adj_ptr, n + 1, s);
        h2d(dcol.p, adj_col, nnz, s);
        col_in.record(s);
        check_cuda(cudaStreamWaitEvent(side.s, col_in.e, 0), "cudaStreamWaitEvent");
        h2d(dw.p, adj_w, nnz, side.s);
        h2d(st->y[0].p, embd, nt, side.s);
        w_in.record(side.s);
        CsrBuild tmp;
        const umapcu_status rc = build_csr_structure(n, dptr.p, dcol.p, nnz, st->csr, tmp, s);
        check_cuda(cudaStreamWaitEvent(s, w_in.e, 0), "cudaStreamWaitEvent");  // dw is freed on s
        if (rc != UMAPCU_OK) return rc;
        build_csr_weights(dw.p, st->csr, tmp, s);
        T.mark("graph H2D + CSR build", s);
    }
    // The schedule precomputed for epochs 0 .. n_epochs - 1 (schedule.cu):
    // record lists pay for their build (~10 ms at 1M points) over repeated or
    // resumed runs of a resident state; a one-shot call (or a state whose
    // lists do not fit) takes the bitmasks, built in well under a millisecond.
    // UMAPCU_NO_SCHEDULE_LISTS set: neither, every epoch scans the cursors.
    const bool precompute = !getenv("UMAPCU_NO_SCHEDULE_LISTS");
    NvtxRange r_sched("umapcu schedule precompute");
    if (lists && precompute) {
        sync(s);
        const auto t0 = std::chrono::steady_clock::now();
        st->lists_ok = build_schedule_lists(st->csr, params->n_epochs, st->lists, s);
        sync(s);
        st->lists_build_ms =
            (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        T.mark("schedule lists", s);
    }
    if (!st->lists_ok && precompute) {
        st->bits_ok = build_schedule_bits(st->csr, params->n_epochs, st->bits, s);
        T.mark("schedule bitmasks", s);
    }
    st->err.alloc(1, s);
    check_cuda(cudaMemsetAsync(st->err.p, 0, sizeof(uint32_t), s), "memset err");
    check_cuda(cudaMemsetAsync(st->m.p, 0, nt * sizeof(float), s), "memset m");
    check_cuda(cudaMemsetAsync(st->v.p, 0, nt * sizeof(float), s), "memset v");
    if (dens) {
        st->dens = true;
        st->lambda = dens->lambda;
        st->frac = dens->frac;
        st->var_shift = dens->var_shift;
        st->mu_tot = dens->mu_tot;
        st->r.alloc(n, s);
        h2d(st->r.p, dens->r, n, s);
        st->dens_node.alloc(n, s);
        check_cuda(cudaMemsetAsync(st->dens_node.p, 0, n * sizeof(float4), s), "memset dens");
        const uint32_t np = dens_partials(n);
        st->part.alloc(4ull * np, s);
        st->ticket.alloc(1, s);
        check_cuda(cudaMemsetAsync(st->ticket.p, 0, sizeof(uint32_t), s), "memset ticket");
        st->stats.alloc(8, s);
        check_cuda(cudaMemsetAsync(st->stats.p, 0, 8 * sizeof(float), s), "memset stats");
    }
    sync(s);
    T.mark("state upload", s);
    out = std::move(st);
    return UMAPCU_OK;
}

__global__ void k_edge_cursor(uint32_t n, const uint32_t *__restrict__ offsets, const uint32_t *__restrict__ other,
                              const uint32_t *__restrict__ edge_id, const float2 *__restrict__ sched,
                              float *__restrict__ cursor)
{
    uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= n) return;
    for (uint32_t p = offsets[node]; p < offsets[node + 1]; p++)
        if (node < other[p]) cursor[edge_id[p]] = sched[p].x;
}

__global__ void k_dens_weight_out(uint32_t n, const float4 *__restrict__ dn, const float *__restrict__ st,
                                  float *__restrict__ re, float *__restrict__ phi, float *__restrict__ w)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 x = dn[i];
    re[i] = x.w;
    phi[i] = x.x;
    w[i] = x.z - st[2] * (x.w - st[0]) * st[3];
}

}  // namespace

// Keep freed stream-ordered allocations cached in the device's default pool
// across calls (the default release threshold of 0 returns them to the
// driver at every synchronisation). The pool is process-wide, so the
// threshold the library found is remembered and put back by
// umapcu_set_pool_retention(0), after which the library leaves it alone.
namespace {
std::atomic<bool> g_pool_retention{true};
std::mutex g_pool_mu;
struct PoolRecord {
    bool raised = false;
    uint64_t prev = 0;
};
PoolRecord g_pool[64];

void restore_pool_locked(int dev)
{
    if (!g_pool[dev].raised) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t prev = g_pool[dev].prev;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &prev);
        cudaMemPoolTrimTo(pool, 0);
    }
    g_pool[dev].raised = false;
}
}  // namespace

void umapcu::keep_pool_memory()
{
    if (!g_pool_retention.load()) return;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (g_pool[dev].raised || !g_pool_retention.load()) return;
    cudaMemPool_t pool;
    uint64_t prev = 0, thr = UINT64_MAX;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess ||
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &prev) != cudaSuccess)
        return;
    if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr) == cudaSuccess) {
        g_pool[dev].raised = true;
        g_pool[dev].prev = prev;
    }
}

// ------------------------------------------------------------------ ABI

extern "C" {

const char *umapcu_status_string(umapcu_status s)
{
    switch (s) {
        case UMAPCU_OK: return "ok";
        case UMAPCU_NO_DATA: return "no data";
        case UMAPCU_NO_GRAPH_EDGES: return "no graph edges";
        case UMAPCU_DEGENERATE_LOCAL_RADII: return "degenerate local radii";
        case UMAPCU_CUDA_ALLOC: return "CUDA allocation failed";
        case UMAPCU_CUDA_LAUNCH: return "CUDA launch or runtime error";
        case UMAPCU_TIMEOUT: return "bounded device wait timed out";
        case UMAPCU_BAD_ARG: return "bad argument";
        case UMAPCU_NO_DEVICE: return "no CUDA device";
        case UMAPCU_CAPACITY: return "capacity exceeded (output buffer, device budget or scratch)";
        case UMAPCU_CANCELLED: return "cancelled";
    }
    return "unknown status";
}

#ifdef UMAPCU_CHECKED
const char *umapcu_version(void) { return "umapcu 0.2.0 sm_100a checked"; }
#else
const char *umapcu_version(void) { return "umapcu 0.2.0 sm_100a"; }
#endif

// fit_params (src/training/umap_optimisers.rs:139-209), T = f32
umapcu_status umapcu_fit_ab(float min_dist, float spread, float *a_out, float *b_out)
{
    if (!a_out || !b_out || !(spread > 0.0f)) return UMAPCU_BAD_ARG;
    const int n_points = 300;
    const uint32_t n_iter = 300;
    float xv[300], yv[300];
    const float three = 3.0f, two = 2.0f, one = 1.0f;
    float max_x = spread * three;
    float step = max_x / (float)(n_points - 1);
    for (int i = 0; i < n_points; i++) {
        float x = step * (float)i;
        xv[i] = x;
        yv[i] = x < min_dist ? one : expf(-(x - min_dist) / spread);
    }
    float a = one, b = one;
    for (uint32_t it = 0; it < n_iter; it++) {
        float grad_a = 0.0f, grad_b = 0.0f;
        const float n_points_t = (float)n_points;
        for (int i = 0; i < n_points; i++) {
            float x = xv[i];
            if (x <= 0.0f) continue;
            float x_2b = powf(x, two * b);
            float denom = one + a * x_2b;
            float pred = one / denom;
            float err = pred - yv[i];
            grad_a += err * (-x_2b / (denom * denom));
            float log_x = logf(x);
            grad_b += err * (-two * a * x_2b * log_x / (denom * denom));
        }
        grad_a /= n_points_t;
        grad_b /= n_points_t;
        a -= 1.0f * grad_a;
        b -= 1.0f * grad_b;
        a = fminf(fmaxf(a, 0.001f), 10.0f);
        b = fminf(fmaxf(b, 0.1f), 2.0f);
    }
    *a_out = a;
    *b_out = b;
    return UMAPCU_OK;
}

umapcu_status umapcu_smooth_knn_dist(const float *knn_dist, uint32_t n, uint32_t k, float local_connectivity,
                                     float bandwidth, uint32_t n_iter, float *sigma, float *rho)
{
    return guard([&]() -> umapcu_status {
        if (n == 0) return UMAPCU_NO_DATA;
        if (!knn_dist || !sigma || !rho || k == 0) return UMAPCU_BAD_ARG;
        Stream S;
        const uint64_t nk = (uint64_t)n * k;
        DevBuf<float> d(nk, S.s), sg(n, S.s), rh(n, S.s);
        h2d(d.p, knn_dist, nk, S.s);
        smooth_knn_dist_dev(d.p, n, k, local_connectivity, bandwidth, n_iter, sg.p, rh.p, S.s);
        d2h(sigma, sg.p, n, S.s);
        d2h(rho, rh.p, n, S.s);
        sync(S.s);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_construct_umap_graph(const int32_t *knn_idx, const float *knn_dist, uint32_t n, uint32_t k,
                                          const umapcu_graph_params *params, uint32_t n_epochs,
                                          uint64_t capacity, uint32_t *row, uint32_t *col, float *val,
                                          uint64_t *nnz, float *sigma, float *rho)
{
    return guard([&]() -> umapcu_status {
        if (n == 0) return UMAPCU_NO_DATA;
        if (!knn_idx || !knn_dist || !params || !nnz || k == 0 || n_epochs == 0) return UMAPCU_BAD_ARG;
        const uint64_t nk = (uint64_t)n * k;
        if (capacity < 2 * nk) return UMAPCU_CAPACITY;
        if (!row || !col || !val) return UMAPCU_BAD_ARG;
        for (uint64_t i = 0; i < nk; i++)
            if (knn_idx[i] < 0 || (uint32_t)knn_idx[i] >= n) return UMAPCU_BAD_ARG;
        NvtxRange r("umapcu construct_umap_graph");
        Stream S;
        DevBuf<int32_t> di(nk, S.s);
        DevBuf<float> dd(nk, S.s), sg(n, S.s), rh(n, S.s);
        h2d(di.p, knn_idx, nk, S.s);
        h2d(dd.p, knn_dist, nk, S.s);
        DeviceCoo coo;
        construct_graph_dev(di.p, dd.p, n, k, *params, n_epochs, coo, sg.p, rh.p, S.s);
        *nnz = coo.nnz;
        d2h(row, coo.row.p, coo.nnz, S.s);
        d2h(col, coo.col.p, coo.nnz, S.s);
        d2h(val, coo.val.p, coo.nnz, S.s);
        if (sigma) d2h(sigma, sg.p, n, S.s);
        if (rho) d2h(rho, rh.p, n, S.s);
        sync(S.s);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_dens_state_new(uint32_t n, uint64_t nnz, const uint32_t *row, const uint32_t *col,
                                    const float *val, const int32_t *knn_idx, const float *knn_dist, uint32_t k,
                                    int distances_squared, float *r, float *mu_sum, float *mu_tot)
{
    return guard([&]() -> umapcu_status {
        if (n == 0) return UMAPCU_NO_DATA;
        if (!r || !mu_sum || !mu_tot || !knn_idx || !knn_dist || k == 0) return UMAPCU_BAD_ARG;
        if (nnz && (!row || !col || !val)) return UMAPCU_BAD_ARG;
        for (uint64_t e = 0; e < nnz; e++)
            if (row[e] >= n || col[e] >= n || (e && row[e] < row[e - 1])) return UMAPCU_BAD_ARG;
        const uint64_t nk = (uint64_t)n * k;
        for (uint64_t i = 0; i < nk; i++)
            if (knn_idx[i] < 0 || (uint32_t)knn_idx[i] >= n) return UMAPCU_BAD_ARG;
        Stream S;
        DevBuf<uint32_t> dr(nnz, S.s), dc(nnz, S.s);
        DevBuf<float> dv(nnz, S.s), dd(nk, S.s), outr(n, S.s), outm(n, S.s);
        DevBuf<int32_t> di(nk, S.s);
        h2d(dr.p, row, nnz, S.s);
        h2d(dc.p, col, nnz, S.s);
        h2d(dv.p, val, nnz, S.s);
        h2d(di.p, knn_idx, nk, S.s);
        h2d(dd.p, knn_dist, nk, S.s);
        umapcu_status rc =
            dens_state_dev(n, nnz, dr.p, dc.p, dv.p, di.p, dd.p, k, distances_squared, outr.p, outm.p, mu_tot, S.s);
        if (rc != UMAPCU_OK) return rc;
        d2h(r, outr.p, n, S.s);
        d2h(mu_sum, outm.p, n, S.s);
        sync(S.s);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_state_create(const float *embd, uint32_t n, uint32_t n_dim, const uint64_t *adj_ptr,
                                  const uint32_t *adj_col, const float *adj_w, const umapcu_optim_params *params,
                                  const umapcu_dens *dens, uint64_t seed, uint32_t sampler, umapcu_state **out)
{
    return guard([&]() -> umapcu_status {
        if (!out) return UMAPCU_BAD_ARG;
        *out = nullptr;
        std::unique_ptr<umapcu_state> st;
        umapcu_status rc = create_state(embd, n, n_dim, adj_ptr, adj_col, adj_w, params, dens, seed, sampler, st, true);
        if (rc == UMAPCU_OK) *out = st.release();
        return rc;
    });
}

void umapcu_state_destroy(umapcu_state *st) { delete st; }

umapcu_status umapcu_state_sizes(const umapcu_state *st, uint64_t *n, uint64_t *n_edges)
{
    if (!st) return UMAPCU_BAD_ARG;
    if (n) *n = st->n;
    if (n_edges) *n_edges = st->csr.n_edges;
    return UMAPCU_OK;
}

umapcu_status umapcu_state_schedule_info(const umapcu_state *st, int *lists_active, uint64_t *n_records,
                                         float *build_ms)
{
    if (!st) return UMAPCU_BAD_ARG;
    if (lists_active) *lists_active = st->lists_ok ? 1 : 0;
    if (n_records) *n_records = st->lists.n_records;
    if (build_ms) *build_ms = st->lists_build_ms;
    return UMAPCU_OK;
}

umapcu_status umapcu_state_read_csr(const umapcu_state *st, uint32_t *offsets, uint32_t *edge_idx, uint32_t *other,
                                    float *eps, float *mu)
{
    return guard([&]() -> umapcu_status {
        if (!st) return UMAPCU_BAD_ARG;
        cudaStream_t s = st->stream.s;
        const uint64_t E = st->csr.n_edges;
        if (offsets) d2h(offsets, st->csr.offsets.p, st->n + 1, s);
        if (edge_idx) d2h(edge_idx, st->csr.edge_id.p, 2 * E, s);
        if (other) d2h(other, st->csr.other.p, 2 * E, s);
        if (eps) d2h(eps, st->csr.eps.p, E, s);
        if (mu) d2h(mu, st->csr.mu.p, E, s);
        sync(s);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_state_run(umapcu_state *st, uint32_t first_epoch, uint32_t count, uint32_t optimiser)
{
    return guard([&]() -> umapcu_status {
        if (!st || optimiser > UMAPCU_OPT_SGD) return UMAPCU_BAD_ARG;
        NvtxRange r("umapcu state run");
        for (uint32_t e = first_epoch; e < first_epoch + count; e++) run_epoch(st, e, optimiser, nullptr, nullptr, nullptr);
        sync(st->stream.s);
        return take_error(st);
    });
}

umapcu_status umapcu_state_enqueue(umapcu_state *st, uint32_t first_epoch, uint32_t count, uint32_t optimiser)
{
    return guard([&]() -> umapcu_status {
        if (!st || optimiser > UMAPCU_OPT_SGD) return UMAPCU_BAD_ARG;
        for (uint32_t e = first_epoch; e < first_epoch + count; e++) run_epoch(st, e, optimiser, nullptr, nullptr, nullptr);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_state_epoch_debug(umapcu_state *st, uint32_t epoch, uint32_t optimiser,
                                       const uint32_t *injected, float *grad, uint32_t *has_update)
{
    return guard([&]() -> umapcu_status {
        if (!st || optimiser > UMAPCU_OPT_SGD) return UMAPCU_BAD_ARG;
        cudaStream_t s = st->stream.s;
        DevBuf<uint32_t> inj, act;
        DevBuf<float> g;
        if (injected) {
            const uint64_t cnt = 2 * st->csr.n_edges * st->p.neg_sample_rate;
            for (uint64_t i = 0; i < cnt; i++)
                if (injected[i] >= st->n) return UMAPCU_BAD_ARG;
            inj.alloc(cnt, s);
            h2d(inj.p, injected, cnt, s);
        }
        if (grad) g.alloc((uint64_t)st->n * st->n_dim, s);
        if (has_update) act.alloc(st->n, s);
        run_epoch(st, epoch, optimiser, inj.p, g.p, act.p);
        if (grad) d2h(grad, g.p, (uint64_t)st->n * st->n_dim, s);
        if (has_update) d2h(has_update, act.p, st->n, s);
        sync(s);
        return take_error(st);
    });
}

umapcu_status umapcu_state_read(const umapcu_state *st, float *embd, float *m, float *v, float *cursor)
{
    return guard([&]() -> umapcu_status {
        if (!st) return UMAPCU_BAD_ARG;
        cudaStream_t s = st->stream.s;
        const uint64_t nt = (uint64_t)st->n * st->n_dim;
        if (embd) d2h(embd, st->y[st->cur].p, nt, s);
        if (m) d2h(m, st->m.p, nt, s);
        if (v) d2h(v, st->v.p, nt, s);
        if (cursor) {
            sync_cursors(const_cast<umapcu_state *>(st));
            DevBuf<float> c(st->csr.n_edges, s);
            k_edge_cursor<<<ceil_div(st->n, 256), 256, 0, s>>>(st->n, st->csr.offsets.p, st->csr.other.p,
                                                               st->csr.edge_id.p, st->csr.sched.p, c.p);
            check_launch("k_edge_cursor");
            d2h(cursor, c.p, st->csr.n_edges, s);
            sync(s);
        }
        sync(s);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_state_write(umapcu_state *st, const float *embd, const float *m, const float *v)
{
    return guard([&]() -> umapcu_status {
        if (!st) return UMAPCU_BAD_ARG;
        cudaStream_t s = st->stream.s;
        const uint64_t nt = (uint64_t)st->n * st->n_dim;
        if (embd) h2d(st->y[st->cur].p, embd, nt, s);
        if (m) h2d(st->m.p, m, nt, s);
        if (v) h2d(st->v.p, v, nt, s);
        sync(s);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_state_reset(umapcu_state *st, const float *embd)
{
    return guard([&]() -> umapcu_status {
        if (!st) return UMAPCU_BAD_ARG;
        cudaStream_t s = st->stream.s;
        const uint64_t nt = (uint64_t)st->n * st->n_dim;
        if (embd) h2d(st->y[st->cur].p, embd, nt, s);
        check_cuda(cudaMemsetAsync(st->m.p, 0, nt * sizeof(float), s), "memset m");
        check_cuda(cudaMemsetAsync(st->v.p, 0, nt * sizeof(float), s), "memset v");
        reset_schedule_dev(st->csr, s);
        st->sched_epoch = 0;
        st->sched_continuous = true;
        st->sched_lazy = false;
        sync(s);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_state_set_precise_pow(umapcu_state *st, int precise)
{
    if (!st) return UMAPCU_BAD_ARG;
    st->precise_pow = precise != 0;
    return UMAPCU_OK;
}

umapcu_status umapcu_eval_pow(const float *x, uint32_t n, float b, int precise, float *out)
{
    return guard([&]() -> umapcu_status {
        if (!x || !out) return UMAPCU_BAD_ARG;
        Stream S;
        DevBuf<float> dx(n, S.s), dy(n, S.s);
        h2d(dx.p, x, n, S.s);
        launch_eval_pow(dx.p, n, b, precise != 0, dy.p, S.s);
        d2h(out, dy.p, n, S.s);
        sync(S.s);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_state_set_stream(umapcu_state *st, void *cuda_stream)
{
    return guard([&]() -> umapcu_status {
        if (!st) return UMAPCU_BAD_ARG;
        sync(st->stream.s);
        st->stream.s = cuda_stream ? (cudaStream_t)cuda_stream : st->own.s;
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_state_run_profiled(umapcu_state *st, uint32_t first_epoch, uint32_t count, uint32_t optimiser,
                                        float *epoch_ms, float *dens_ms)
{
    return guard([&]() -> umapcu_status {
        if (!st || optimiser > UMAPCU_OPT_SGD) return UMAPCU_BAD_ARG;
        cudaStream_t s = st->stream.s;
        std::vector<cudaEvent_t> ev(4 * (size_t)count + 4);
        for (auto &e : ev) check_cuda(cudaEventCreate(&e), "cudaEventCreate");
        std::vector<int> dens_on(count);
        for (uint32_t i = 0; i < count; i++) {
            const uint32_t e = first_epoch + i;
            dens_on[i] = st->dens && dens_active(st->lambda, st->frac, e, st->p.n_epochs);
            check_cuda(cudaEventRecord(ev[4 * i], s), "record");
            if (dens_on[i]) dens_update(st);
            check_cuda(cudaEventRecord(ev[4 * i + 1], s), "record");
            run_epoch(st, e, optimiser, nullptr, nullptr, nullptr, /*skip_dens=*/true);
            check_cuda(cudaEventRecord(ev[4 * i + 2], s), "record");
        }
        sync(s);
        double tot_e = 0, tot_d = 0;
        for (uint32_t i = 0; i < count; i++) {
            float a = 0, b = 0;
            check_cuda(cudaEventElapsedTime(&a, ev[4 * i], ev[4 * i + 1]), "elapsed");
            check_cuda(cudaEventElapsedTime(&b, ev[4 * i + 1], ev[4 * i + 2]), "elapsed");
            tot_d += dens_on[i] ? a : 0.0;
            tot_e += b;
        }
        for (auto &e : ev) cudaEventDestroy(e);
        if (epoch_ms) *epoch_ms = (float)tot_e;
        if (dens_ms) *dens_ms = (float)tot_d;
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_state_dens_update(umapcu_state *st, float *re, float *phi_sum, float *weight, float *coeff,
                                       float *stats3)
{
    return guard([&]() -> umapcu_status {
        if (!st || !st->dens) return UMAPCU_BAD_ARG;
        cudaStream_t s = st->stream.s;
        dens_update(st);
        DevBuf<float> dre(st->n, s), dphi(st->n, s), dw(st->n, s);
        k_dens_weight_out<<<ceil_div(st->n, 256), 256, 0, s>>>(st->n, st->dens_node.p, st->stats.p, dre.p, dphi.p,
                                                               dw.p);
        check_launch("k_dens_weight_out");
        float h[5];
        d2h(h, st->stats.p, 5, s);
        if (re) d2h(re, dre.p, st->n, s);
        if (phi_sum) d2h(phi_sum, dphi.p, st->n, s);
        if (weight) d2h(weight, dw.p, st->n, s);
        sync(s);
        if (coeff) *coeff = h[4];
        if (stats3) { stats3[0] = h[0]; stats3[1] = h[1]; stats3[2] = h[2]; }
        return take_error(st);
    });
}

umapcu_status umapcu_optimise_embedding(float *embd, uint32_t n, uint32_t n_dim, const uint64_t *adj_ptr,
                                        const uint32_t *adj_col, const float *adj_w,
                                        const umapcu_optim_params *params, const umapcu_dens *dens, uint64_t seed,
                                        uint32_t optimiser, uint32_t sampler, int verbose)
{
    return guard([&]() -> umapcu_status {
        if (optimiser > UMAPCU_OPT_SGD) return UMAPCU_BAD_ARG;
        std::unique_ptr<umapcu_state> st;
        umapcu_status rc = create_state(embd, n, n_dim, adj_ptr, adj_col, adj_w, params, dens, seed, sampler, st, false);
        if (rc != UMAPCU_OK) return rc;
        if (verbose)
            printf("Running %u epochs with GPU-accelerated %s optimisation.\n", params->n_epochs,
                   optimiser == UMAPCU_OPT_SGD ? "SGD" : "Adam");
        const uint64_t nt = (uint64_t)n * n_dim;
        PhaseTimer T;
        NvtxRange r("umapcu epochs");
        for (uint32_t e = 0; e < params->n_epochs; e++) {
            const bool log_now = verbose && ((e + 1) % 100 == 0 || e + 1 == params->n_epochs);
            if (!log_now) {
                run_epoch(st.get(), e, optimiser, nullptr, nullptr, nullptr);
                continue;
            }
            DevBuf<float> g(nt, st->stream.s);
            run_epoch(st.get(), e, optimiser, nullptr, g.p, nullptr);
            std::vector<float> hg(nt);
            d2h(hg.data(), g.p, nt, st->stream.s);
            sync(st->stream.s);
            double ss = 0.0;
            for (float x : hg) ss += (double)x * x;
            printf(" Epoch %u / %u: grad norm %.2f\n", e + 1, params->n_epochs, sqrt(ss));
        }
        T.mark("epochs", st->stream.s);
        d2h(embd, st->y[st->cur].p, nt, st->stream.s);
        sync(st->stream.s);
        T.mark("embedding D2H", st->stream.s);
        return take_error(st.get());
    });
}

umapcu_status umapcu_adam_update(const float *grad, const uint32_t *has_update, float *m, float *v, float *embd,
                                 uint32_t n, uint32_t n_dim, const umapcu_optim_params *params, uint32_t epoch)
{
    return guard([&]() -> umapcu_status {
        if (!grad || !has_update || !m || !v || !embd || !params || n_dim == 0) return UMAPCU_BAD_ARG;
        if (n == 0) return UMAPCU_NO_DATA;
        Stream S;
        const uint64_t nt = (uint64_t)n * n_dim;
        DevBuf<float> dg(nt, S.s), dm(nt, S.s), dv(nt, S.s), dy(nt, S.s);
        DevBuf<uint32_t> dh(n, S.s);
        h2d(dg.p, grad, nt, S.s);
        h2d(dm.p, m, nt, S.s);
        h2d(dv.p, v, nt, S.s);
        h2d(dy.p, embd, nt, S.s);
        h2d(dh.p, has_update, n, S.s);
        float fused, epsc, lr_e;
        epoch_scalars(*params, epoch, &fused, &epsc, &lr_e);
        launch_adam_apply(dg.p, dh.p, dm.p, dv.p, dy.p, nt, n_dim, fused, epsc, 1.0f - params->beta1,
                          1.0f - params->beta2, S.s);
        d2h(m, dm.p, nt, S.s);
        d2h(v, dv.p, nt, S.s);
        d2h(embd, dy.p, nt, S.s);
        sync(S.s);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_edge_schedule_update(const float *eps, float *cursor, uint64_t n_edges, uint32_t epoch)
{
    return guard([&]() -> umapcu_status {
        if (!eps || !cursor) return UMAPCU_BAD_ARG;
        Stream S;
        DevBuf<float> de(n_edges, S.s), dc(n_edges, S.s);
        h2d(de.p, eps, n_edges, S.s);
        h2d(dc.p, cursor, n_edges, S.s);
        launch_schedule(de.p, dc.p, n_edges, epoch, S.s);
        d2h(cursor, dc.p, n_edges, S.s);
        sync(S.s);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_sample_negatives(uint32_t sampler, uint64_t seed, uint32_t node, uint32_t entry,
                                      uint32_t epoch, uint32_t edge_local, uint32_t count, uint32_t n,
                                      uint32_t *out)
{
    return guard([&]() -> umapcu_status {
        if (!out || n == 0 || sampler > UMAPCU_NEG_PHILOX) return UMAPCU_BAD_ARG;
        Stream S;
        DevBuf<uint32_t> d(count, S.s);
        launch_sample(sampler, seed, node, entry, epoch, edge_local, count, n, d.p, S.s);
        d2h(out, d.p, count, S.s);
        sync(S.s);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_state_set_schedule(umapcu_state *st, uint32_t form)
{
    return guard([&]() -> umapcu_status {
        if (!st || form > UMAPCU_SCHED_LISTS) return UMAPCU_BAD_ARG;
        cudaStream_t s = st->stream.s;
        if (st->lists_ok || st->bits_ok) {
            // cursors brought up to date, and every launch that reads the
            // old form finished, before it is freed
            sync_cursors(st);
            sync(s);
            st->lists = ScheduleLists();
            st->bits.release();
            st->lists_ok = st->bits_ok = false;
        }
        if (form == UMAPCU_SCHED_SCAN) return UMAPCU_OK;
        if (form == UMAPCU_SCHED_LISTS) {
            sync(s);
            const auto t0 = std::chrono::steady_clock::now();
            st->lists_ok = build_schedule_lists(st->csr, st->p.n_epochs, st->lists, s);
            sync(s);
            st->lists_build_ms =
                (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            return st->lists_ok ? UMAPCU_OK : UMAPCU_CAPACITY;
        }
        st->bits_ok = build_schedule_bits(st->csr, st->p.n_epochs, st->bits, s);
        return st->bits_ok ? UMAPCU_OK : UMAPCU_CAPACITY;
    });
}

umapcu_status umapcu_state_schedule_form(const umapcu_state *st, uint32_t *form)
{
    if (!st || !form) return UMAPCU_BAD_ARG;
    *form = st->lists_ok ? UMAPCU_SCHED_LISTS : st->bits_ok ? UMAPCU_SCHED_BITS : UMAPCU_SCHED_SCAN;
    return UMAPCU_OK;
}

umapcu_status umapcu_set_pool_retention(int keep)
{
    g_pool_retention.store(keep != 0);
    if (keep) return UMAPCU_OK;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    for (int dev = 0; dev < 64; dev++) restore_pool_locked(dev);
    return UMAPCU_OK;
}

umapcu_status umapcu_release_cached(void)
{
    return guard([&]() -> umapcu_status {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return UMAPCU_NO_DEVICE;
        release_cached_bits();
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_device_count(int *count)
{
    if (!count) return UMAPCU_BAD_ARG;
    *count = 0;
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) {
        cudaGetLastError();
        return UMAPCU_NO_DEVICE;
    }
    *count = c;
    return UMAPCU_OK;
}

umapcu_status umapcu_set_device(int device)
{
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) {
        cudaGetLastError();
        return UMAPCU_NO_DEVICE;
    }
    if (device < 0 || device >= c) return UMAPCU_BAD_ARG;
    return cudaSetDevice(device) == cudaSuccess ? UMAPCU_OK : UMAPCU_NO_DEVICE;
}

umapcu_status umapcu_probe_l2_gather(uint64_t table_bytes, float *gbs)
{
    return guard([&]() -> umapcu_status {
        if (!gbs || table_bytes < 4096 || table_bytes > (64ull << 20)) return UMAPCU_BAD_ARG;
        Stream S;
        *gbs = probe_l2_gather(table_bytes, S.s);
        return UMAPCU_OK;
    });
}

}  // extern "C"
