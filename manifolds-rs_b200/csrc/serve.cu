// Served form: a request loop that runs many layout jobs concurrently on one
// GPU with continuous batching.
//
// Clients submit jobs (one optimise_embedding_adam_gpu call's arguments each,
// copied on submit) from any thread. The server's threads own the device:
//   * admission (two threads, one high-priority stream each): a thread takes
//     the pending jobs that fit, in arrival order, as one group (job count
//     under max_jobs, the device-memory estimate of admitted work -- CSR
//     build peak + state -- within the budget), stages the group's graphs,
//     initial layouts and epoch scalars into page-locked memory, moves them
//     in one DMA and builds all the group's CSRs in one multi-graph build
//     (build_csr_multi: each job's rows equal its own build); the group's
//     state lives in shared buffers, one slice per job;
//   * tick: one persistent launch of the multi-problem kernel advances every
//     active job by tick_epochs epochs, each from its own current epoch
//     (jobs admitted at different times are at different epochs in the same
//     launch), with the per-problem bounded barriers of the batched form;
//   * completion: a completion thread reads finished jobs back and wakes
//     their waiters while the next tick runs; a group's buffers and budget
//     are released when its last job finishes. Admitted groups join at the
//     next tick boundary.
// The tick kernel is launched with 6 of the 8 resident CTAs per SM its
// registers allow (UMAPCU_SERVE_CTAS_PER_SM overrides), so the admission
// kernels find room on the SMs while a tick runs.
// A job's arithmetic does not depend on the jobs it shares a launch or a
// group with (per-job seed, node indices and buffer slices), so its result is
// the same alone and in any mix. Failures are reported per job (allocation,
// a graph without edges, device error, bounded-wait timeout); cancellation
// works on pending jobs.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "batch_device.cuh"

using namespace umapcu;

namespace {

enum JobState { kPending = 0, kActive = 1, kDone = 2, kFailed = 3 };

// Jobs admitted together share one graph build and one set of buffers; the
// buffers are released when the group's last job finishes.
struct AdmitGroup {
    DeviceCsr csr;                // all the group's nodes; each job uses its slice
    DevBuf<float> y0, y1, m, v;   // per-job slices, 256-byte aligned
    DevBuf<float4> scal;          // per-job epoch scalars
    // the edge schedule of every CSR entry of the group, per epoch, as
    // bitmasks [max n_epochs][bits_words] (bit p of an epoch: entry p active):
    // the ticks scan these in place of the cursors
    DevBuf<uint32_t> bits;
    uint64_t bits_words = 0;
    uint64_t bytes = 0;           // admission estimate held against the budget
    uint32_t remaining = 0;       // jobs still running
};

struct ServeJob {
    uint64_t id = 0;
    uint32_t n = 0, n_dim = 0;
    umapcu_optim_params params{};
    uint64_t seed = 0;
    uint32_t sampler = 0;
    uint64_t nnz = 0;
    // the job's inputs, copied on submit into one block (page-locked arena,
    // or the heap when the arena is full): ptr | col | w | embd | scalars
    char *blk = nullptr;
    int chunk = -1;                // arena chunk, -1: heap
    std::vector<char> heap;
    size_t o_col = 0, o_w = 0, o_y = 0, o_sc = 0, blk_bytes = 0;
    uint64_t bytes = 0;
    std::shared_ptr<AdmitGroup> grp;
    uint32_t node_base = 0;       // first node of the job in the group's CSR
    uint64_t y_off = 0, sc_off = 0, n_edges = 0;
    uint32_t epochs_done = 0;
    // a resumed job: epochs run before it was submitted, and its Adam moments
    // in the submit block (o_m = 0: the moments start at zero)
    uint32_t start_epoch = 0;
    size_t o_m = 0, o_v = 0;
    // a snapshot request, answered by the tick thread between two ticks
    struct Snapshot {
        float *y = nullptr, *m = nullptr, *v = nullptr;
        uint32_t epochs = 0;
        umapcu_status rc = UMAPCU_OK;
        bool done = false;
    };
    Snapshot *snap = nullptr;
    std::vector<float> result;
    int state = kPending;
    umapcu_status rc = UMAPCU_OK;
    double t_submit = 0, t_admit = 0, t_done = 0;
};

// Peak device bytes of admitting and running a job: the CSR build's
// temporaries dominate (about 64 B per adjacency entry), plus the state and
// the schedule bitmasks (one bit per CSR entry -- at most nnz -- and epoch).
uint64_t job_bytes(uint32_t n, uint32_t n_dim, uint64_t nnz, uint32_t n_epochs)
{
    return 72ull * nnz + 24ull * n * n_dim + 16ull * n_epochs + (nnz + 32) / 8 * n_epochs + (1ull << 20);
}

}  // namespace

constexpr int kAdmitThreads = 2;
constexpr int kTickCtasPerSm = 6;
constexpr uint32_t kGroupMaxJobs = 512;
constexpr uint64_t kGroupMaxEntries = 1ull << 30;  // adjacency entries per group build

// Page-locked host staging of one admission thread (grows, never shrinks):
// a group's graphs, initial layouts and epoch scalars go to the device in one
// DMA.
struct PinnedStage {
    char *p = nullptr;
    size_t cap = 0;
    char *ensure(size_t bytes)
    {
        if (bytes > cap) {
            if (p) cudaFreeHost(p);
            p = nullptr;
            cap = std::max(bytes, 2 * cap);
            check_cuda(cudaHostAlloc((void **)&p, cap, cudaHostAllocDefault), "cudaHostAlloc", UMAPCU_CUDA_ALLOC);
        }
        return p;
    }
    ~PinnedStage()
    {
        if (p) cudaFreeHost(p);
    }
};

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Page-locked arena for submitted inputs: chunks of kChunk bytes, each a bump
// allocator that resets when its last block is released. Submit copies a
// job's inputs straight into it (no page faults on fresh heap memory) and
// admission moves them to the device without another host copy. Blocks that
// do not fit (arena at kArenaMax, or larger than a chunk) go to the heap.
struct PinnedArena {
    static constexpr size_t kChunk = 256ull << 20;
    static constexpr size_t kArenaMax = 4ull << 30;
    struct Chunk {
        char *p = nullptr;
        size_t head = 0;
        uint32_t live = 0;
    };
    std::mutex mu;
    std::vector<Chunk> chunks;
    int cur = -1;
    char *try_alloc(size_t bytes, int *ci)  // caller holds mu
    {
        bytes = align256(bytes);
        if (cur >= 0 && chunks[cur].head + bytes <= kChunk) return take(cur, bytes, ci);
        for (int c = 0; c < (int)chunks.size(); c++)
            if (chunks[c].live == 0) {
                chunks[c].head = 0;
                cur = c;
                return take(c, bytes, ci);
            }
        return nullptr;
    }
    char *take(int c, size_t bytes, int *ci)
    {
        char *p = chunks[c].p + chunks[c].head;
        chunks[c].head += bytes;
        chunks[c].live++;
        *ci = c;
        return p;
    }
    char *alloc(size_t bytes, int *ci)
    {
        if (align256(bytes) > kChunk) return nullptr;
        std::lock_guard<std::mutex> lk(mu);
        if (char *p = try_alloc(bytes, ci)) return p;
        if ((chunks.size() + 1) * kChunk > kArenaMax) return nullptr;
        Chunk c;
        if (cudaHostAlloc((void **)&c.p, kChunk, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        chunks.push_back(c);
        cur = (int)chunks.size() - 1;
        return take(cur, align256(bytes), ci);
    }
    void release(int c)
    {
        std::lock_guard<std::mutex> lk(mu);
        if (--chunks[c].live == 0 && c != cur) chunks[c].head = 0;
    }
    ~PinnedArena()
    {
        for (Chunk &c : chunks) cudaFreeHost(c.p);
    }
};

struct umapcu_server {
    Stream own;                  // ticks
    Stream own2[kAdmitThreads] = {Stream(true), Stream(true)};
    Stream own3;                 // completions
    cudaStream_t s = nullptr;
    int device = 0;
    uint64_t budget = 0;
    uint32_t max_jobs = 0, tick_epochs = 0, n_dim = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_admit, cv_fin;
    std::deque<ServeJob *> pending;
    std::vector<ServeJob *> ready;     // admitted, waiting for the next tick boundary
    std::vector<ServeJob *> active;    // owned by the tick thread
    std::deque<ServeJob *> finishing;  // computed, waiting for read-back
    uint32_t live = 0;                 // admitting + ready + active + finishing
    int tick_ctas = kTickCtasPerSm;
    std::thread th, finisher;
    std::thread admitters[kAdmitThreads];
    PinnedStage stage[kAdmitThreads];  // group headers
    PinnedStage fin_stage;
    PinnedArena arena;
    std::map<uint64_t, std::unique_ptr<ServeJob>> jobs;
    uint64_t next_id = 1, used = 0, peak_used = 0, ticks = 0, completed = 0, groups = 0;
    uint32_t peak_jobs = 0;
    bool stop = false;
    // wall-time totals, printed at shutdown when UMAPCU_TIMING is set
    double t_build = 0, t_tick = 0;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    DevBuf<BatchProblem> probs;
    DevBuf<uint32_t> seg_prob, ctr;
    std::vector<BatchProblem> hp;  // host tables of the tick in flight
    std::vector<uint32_t> segs;
    uint32_t err_h = 0;
    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
    void loop();
    void admit_loop(int k);
    void finish_loop();
    void admit_group(std::vector<ServeJob *> &g, int k);
    void group_job_done(ServeJob *j);  // caller holds mu
    void free_block(ServeJob *j);
    void tick_launch();
    umapcu_status tick_finish();
    void answer_snapshots(const std::vector<ServeJob *> &done);
    void release_snapshot(ServeJob *j, umapcu_status rc);  // caller holds mu
};

// Ends a job's snapshot request with `rc`. Caller holds mu.
void umapcu_server::release_snapshot(ServeJob *j, umapcu_status rc)
{
    if (!j->snap) return;
    j->snap->rc = rc;
    j->snap->done = true;
    j->snap = nullptr;
    cv_done.notify_all();
}

// Between two ticks (tick thread, nothing in flight on s): copies the state
// of every running job with a snapshot request -- the embedding buffer its
// next epoch reads, its moments, its epoch count -- to the requester; jobs
// that finished in the last tick answer UMAPCU_BAD_ARG (nothing left to
// resume).
void umapcu_server::answer_snapshots(const std::vector<ServeJob *> &done)
{
    std::vector<ServeJob *> req;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (ServeJob *j : done) release_snapshot(j, UMAPCU_BAD_ARG);
        for (ServeJob *j : active)
            if (j->snap) req.push_back(j);
    }
    for (ServeJob *j : req) {
        umapcu_status rc = UMAPCU_OK;
        try {
            const uint64_t nt = (uint64_t)j->n * j->n_dim;
            const AdmitGroup &G = *j->grp;
            const float *y = ((j->epochs_done & 1) ? G.y1.p : G.y0.p) + j->y_off;
            d2h(j->snap->y, y, nt, s);
            if (j->snap->m) d2h(j->snap->m, G.m.p + j->y_off, nt, s);
            if (j->snap->v) d2h(j->snap->v, G.v.p + j->y_off, nt, s);
            sync(s);
        } catch (const Error &e) {
            rc = e.status;
        }
        std::lock_guard<std::mutex> lk(mu);
        j->snap->epochs = j->epochs_done;
        release_snapshot(j, rc);
    }
}

// Moves a group of pending jobs to the device (per job, straight from its
// submit block), builds their graphs in one multi-graph build and their state
// in shared buffers (stream of admission thread k).
void umapcu_server::admit_group(std::vector<ServeJob *> &g, int k)
{
    NvtxRange r("umapcu admit group");
    cudaStream_t s = own2[k].s;
    const uint32_t J = (uint32_t)g.size();
    uint64_t n_tot = 0, nnz = 0, y_tot = 0, sc_tot = 0;
    for (ServeJob *j : g) {
        j->node_base = (uint32_t)n_tot;
        j->y_off = y_tot;
        j->sc_off = sc_tot;
        n_tot += j->n;
        nnz += j->nnz;
        y_tot += align256(4ull * j->n * j->n_dim) / 4;
        sc_tot += j->params.n_epochs;
    }
    if (n_tot + J >= (1ull << 32)) fail(UMAPCU_BAD_ARG, "group too large");
    const double ta = now();
    // group header: node_base [J + 1] | job_entry_base [J + 1]
    const size_t o_jb = align256(4ull * (J + 1)), hdr = o_jb + 8ull * (J + 1);
    char *h = stage[k].ensure(hdr);
    uint32_t *nb = (uint32_t *)h;
    uint64_t *jb = (uint64_t *)(h + o_jb);
    uint64_t e0 = 0;
    for (uint32_t t = 0; t < J; t++) {
        nb[t] = g[t]->node_base;
        jb[t] = e0;
        e0 += g[t]->nnz;
    }
    nb[J] = (uint32_t)n_tot;
    jb[J] = e0;
    auto grp = std::make_shared<AdmitGroup>();
    grp->y0.alloc(y_tot, s);
    grp->y1.alloc(y_tot, s);
    grp->m.alloc(y_tot, s);
    grp->v.alloc(y_tot, s);
    grp->scal.alloc(sc_tot, s);
    std::vector<uint64_t> edges(J);
    {
        const size_t d_lp = align256(hdr), d_col = d_lp + align256(8 * (n_tot + J)), d_w = d_col + align256(4 * nnz),
                     total = d_w + 4 * nnz;
        DevBuf<char> d(total, s);
        check_cuda(cudaMemcpyAsync(d.p, h, hdr, cudaMemcpyHostToDevice, s), "h2d");
        uint64_t e = 0;
        for (uint32_t t = 0; t < J; t++) {
            const ServeJob *j = g[t];
            const uint64_t nt = (uint64_t)j->n * j->n_dim;
            check_cuda(cudaMemcpyAsync(d.p + d_lp + 8ull * (j->node_base + t), j->blk, 8ull * (j->n + 1),
                                       cudaMemcpyHostToDevice, s), "h2d");
            if (j->nnz) {
                check_cuda(cudaMemcpyAsync(d.p + d_col + 4 * e, j->blk + j->o_col, 4 * j->nnz, cudaMemcpyHostToDevice,
                                           s), "h2d");
                check_cuda(cudaMemcpyAsync(d.p + d_w + 4 * e, j->blk + j->o_w, 4 * j->nnz, cudaMemcpyHostToDevice, s),
                           "h2d");
            }
            // the buffer an epoch of this parity reads (a resumed job starts mid-run)
            float *y_start = ((j->start_epoch & 1) ? grp->y1.p : grp->y0.p) + j->y_off;
            check_cuda(cudaMemcpyAsync(y_start, j->blk + j->o_y, 4 * nt, cudaMemcpyHostToDevice, s), "h2d");
            check_cuda(cudaMemcpyAsync(grp->scal.p + j->sc_off, j->blk + j->o_sc, 16ull * j->params.n_epochs,
                                       cudaMemcpyHostToDevice, s), "h2d");
            e += j->nnz;
        }
        const umapcu_status rc = build_csr_multi((uint32_t)n_tot, J, (const uint32_t *)d.p,
                                                 (const uint64_t *)(d.p + o_jb), (const uint64_t *)(d.p + d_lp),
                                                 (const uint32_t *)(d.p + d_col), (const float *)(d.p + d_w), nnz,
                                                 grp->csr, edges.data(), s);
        if (rc != UMAPCU_OK) fail(rc, "csr");
    }
    check_cuda(cudaMemsetAsync(grp->m.p, 0, 4 * y_tot, s), "memset");
    check_cuda(cudaMemsetAsync(grp->v.p, 0, 4 * y_tot, s), "memset");
    {
        // schedule bitmasks of the whole group (from the periods, so valid for
        // resumed jobs too: they are indexed by the job's own epoch)
        uint32_t max_ep = 0;
        for (const ServeJob *j : g) max_ep = std::max(max_ep, j->params.n_epochs);
        const uint64_t entries = 2 * grp->csr.n_edges;
        grp->bits_words = (entries + 31) / 32;
        if (entries) {
            grp->bits.alloc((size_t)grp->bits_words * max_ep, s);
            launch_schedule_bits(grp->csr.sched.p, entries, max_ep, grp->bits.p, s);
        }
    }
    for (uint32_t t = 0; t < J; t++) {
        const ServeJob *j = g[t];
        if (!j->start_epoch && !j->o_m) continue;
        // a resumed job: its moments, and its cursors as the schedule left
        // them after its first start_epoch epochs
        const uint64_t nt = (uint64_t)j->n * j->n_dim;
        if (j->o_m) {
            check_cuda(cudaMemcpyAsync(grp->m.p + j->y_off, j->blk + j->o_m, 4 * nt, cudaMemcpyHostToDevice, s), "h2d");
            check_cuda(cudaMemcpyAsync(grp->v.p + j->y_off, j->blk + j->o_v, 4 * nt, cudaMemcpyHostToDevice, s), "h2d");
        }
        if (j->start_epoch && edges[t])
            materialise_schedule_range(grp->csr, j->node_base, 2 * edges[t], j->start_epoch, s);
    }
    sync(s);  // the submit blocks and the header staging are free after this
    const double tc = now();
    std::lock_guard<std::mutex> lk(mu);
    t_build += tc - ta;
    groups++;
    for (uint32_t t = 0; t < J; t++) {
        ServeJob *j = g[t];
        j->n_edges = edges[t];
        if (edges[t] == 0) {
            j->rc = UMAPCU_NO_GRAPH_EDGES;  // as the single-graph build reports; holds no group share
            continue;
        }
        j->grp = grp;
        grp->bytes += j->bytes;
        grp->remaining++;
    }
}

// Releases a job's submit block (arena chunk or heap).
void umapcu_server::free_block(ServeJob *j)
{
    if (j->chunk >= 0) arena.release(j->chunk);
    j->chunk = -1;
    j->blk = nullptr;
    std::vector<char>().swap(j->heap);
}

// A job leaves its group; the last one out releases the group's buffers and
// its budget. Caller holds mu.
void umapcu_server::group_job_done(ServeJob *j)
{
    std::shared_ptr<AdmitGroup> grp;
    grp.swap(j->grp);
    if (!grp) {
        used -= j->bytes;  // failed at admission: holds no group share
        return;
    }
    if (--grp->remaining) return;
    used -= grp->bytes;
    grp->csr = DeviceCsr();
    grp->y0.release();
    grp->y1.release();
    grp->m.release();
    grp->v.release();
    grp->scal.release();
    grp->bits.release();
}

// Enqueues one tick over the active jobs on stream s (asynchronous).
void umapcu_server::tick_launch()
{
    NvtxRange r("umapcu tick");
    hp.assign(active.size(), BatchProblem{});
    segs.clear();
    bool nr5 = true, all_hash = true;
    for (size_t i = 0; i < active.size(); i++) {
        ServeJob *j = active[i];
        BatchProblem &P = hp[i];
        P = BatchProblem{};
        P.n = j->n;
        P.nseg = ceil_div(j->n, 32);
        P.seg_base = (uint32_t)segs.size();
        P.epoch_base = j->epochs_done;
        P.n_epochs = j->params.n_epochs;
        const AdmitGroup &G = *j->grp;
        P.offsets = G.csr.offsets.p + j->node_base;
        P.other = G.csr.other.p;
        P.sched = G.csr.sched.p;
        P.y0 = G.y0.p + j->y_off;
        P.y1 = G.y1.p + j->y_off;
        P.m = G.m.p + j->y_off;
        P.v = G.v.p + j->y_off;
        P.scal = G.scal.p + j->sc_off;
        P.bits = G.bits.p;
        P.bits_words = G.bits_words;
        // the length of the group's entry arrays: the job's offsets index
        // them group-wide
        P.n_entries = 2 * G.csr.n_edges;
        const umapcu_optim_params &q = j->params;
        P.a = q.a;
        P.b = q.b;
        P.two_a_b = 2.0f * q.a * q.b;
        P.two_gamma_b = 2.0f * q.gamma * q.b;
        P.omb1 = 1.0f - q.beta1;
        P.omb2 = 1.0f - q.beta2;
        P.neg_rate = q.neg_sample_rate;
        nr5 = nr5 && q.neg_sample_rate == 5;
        all_hash = all_hash && j->sampler == UMAPCU_NEG_REF_HASH;
        P.sampler = j->sampler;
        P.seed32 = (uint32_t)j->seed;
        P.seed_lo = (uint32_t)j->seed;
        P.seed_hi = (uint32_t)(j->seed >> 32);
        P.fastmod_M = fastmod_magic(j->n);
        for (uint32_t k = 0; k < P.nseg; k++) segs.push_back((uint32_t)i);
    }
    if (probs.n < hp.size()) probs.alloc(hp.size() * 2, s);
    if (seg_prob.n < segs.size()) seg_prob.alloc(segs.size() * 2, s);
    if (ctr.n < 2 + hp.size()) ctr.alloc(2 * (2 + hp.size()), s);
    h2d(probs.p, hp.data(), hp.size(), s);
    h2d(seg_prob.p, segs.data(), segs.size(), s);
    check_cuda(cudaMemsetAsync(ctr.p, 0, (2 + hp.size()) * sizeof(uint32_t), s), "memset");
    BatchArgs B{};
    B.probs = probs.p;
    B.seg_prob = seg_prob.p;
    B.n_probs = (uint32_t)hp.size();
    B.n_segs = (uint32_t)segs.size();
    B.n_epochs = tick_epochs;
    B.optimiser = UMAPCU_OPT_ADAM;
    B.work = ctr.p;
    B.error = ctr.p + 1;
    B.done = ctr.p + 2;
    B.wait_limit = 1u << 24;
    B.poison = ~0u;
    BatchConfig c;
    c.mode = 1;
    c.ctas_per_sm = tick_ctas;
    switch (n_dim) {
        case 2: nr5 ? launch_batch_kernel<2>(B, c, s, 0, all_hash, true) : launch_batch_kernel_nr0<2>(B, c, s, 0, true); break;
        case 3: nr5 ? launch_batch_kernel<3>(B, c, s, 0, all_hash, true) : launch_batch_kernel_nr0<3>(B, c, s, 0, true); break;
        default: nr5 ? launch_batch_kernel<4>(B, c, s, 0, all_hash, true) : launch_batch_kernel_nr0<4>(B, c, s, 0, true); break;
    }
    d2h(&err_h, ctr.p + 1, 1, s);
}

// Waits for the tick in flight; its status.
umapcu_status umapcu_server::tick_finish()
{
    sync(s);  // hp / segs / err_h stay alive until here
    std::lock_guard<std::mutex> lk(mu);
    ticks++;
    return err_h ? (umapcu_status)err_h : UMAPCU_OK;
}

void umapcu_server::admit_loop(int k)
{
    cudaSetDevice(device);
    for (;;) {
        std::vector<ServeJob *> g;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_admit.wait(lk, [&] {
                return stop ||
                       (!pending.empty() && live < max_jobs && used + pending.front()->bytes <= budget);
            });
            if (stop) return;
            // a group: pending jobs in arrival order while they fit
            uint64_t entries = 0;
            while (!pending.empty() && live < max_jobs && g.size() < kGroupMaxJobs) {
                ServeJob *j = pending.front();
                const uint64_t m = j->nnz;
                if (used + j->bytes > budget || (!g.empty() && entries + m > kGroupMaxEntries)) break;
                pending.pop_front();
                entries += m;
                used += j->bytes;
                live++;
                g.push_back(j);
            }
            peak_used = std::max(peak_used, used);
        }
        umapcu_status rc = UMAPCU_OK;
        try {
            admit_group(g, k);
        } catch (const Error &e) {
            rc = e.status;
        }
        if (rc != UMAPCU_OK) cudaStreamSynchronize(own2[k].s);  // no copy in flight from the blocks
        for (ServeJob *j : g) free_block(j);
        std::lock_guard<std::mutex> lk(mu);
        const double t = now();
        for (ServeJob *j : g) {
            j->t_admit = t;
            if (rc != UMAPCU_OK) j->rc = rc;
            if (j->rc == UMAPCU_OK) {
                ready.push_back(j);
                continue;
            }
            j->state = kFailed;
            j->t_done = t;
            release_snapshot(j, j->rc);
            group_job_done(j);
            live--;
        }
        cv_work.notify_all();
        cv_done.notify_all();
        cv_admit.notify_all();
    }
}

// Reads finished jobs back (through page-locked staging, on its own stream)
// and releases their group share; the tick loop never waits on this.
void umapcu_server::finish_loop()
{
    cudaSetDevice(device);
    for (;;) {
        ServeJob *j = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_fin.wait(lk, [&] { return !finishing.empty() || stop; });
            if (finishing.empty()) return;
            j = finishing.front();
            finishing.pop_front();
        }
        if (j->rc == UMAPCU_OK) {
            const uint64_t nt = (uint64_t)j->n * j->n_dim;
            const AdmitGroup &G = *j->grp;
            try {
                float *h = (float *)fin_stage.ensure(4 * nt);
                d2h(h, ((j->params.n_epochs & 1) ? G.y1.p : G.y0.p) + j->y_off, nt, own3.s);
                sync(own3.s);
                j->result.assign(h, h + nt);
            } catch (const Error &e) {
                j->rc = e.status;
            }
        }
        std::lock_guard<std::mutex> lk(mu);
        group_job_done(j);
        j->t_done = now();
        j->state = j->rc == UMAPCU_OK ? kDone : kFailed;
        release_snapshot(j, UMAPCU_BAD_ARG);  // asked for after its last tick
        live--;
        completed++;
        cv_done.notify_all();
        cv_admit.notify_all();
    }
}

void umapcu_server::loop()
{
    cudaSetDevice(device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return stop || !ready.empty() || !active.empty(); });
            if (stop) break;
            for (ServeJob *j : ready) {
                j->state = kActive;
                active.push_back(j);
            }
            ready.clear();
            peak_jobs = std::max<uint32_t>(peak_jobs, (uint32_t)active.size());
        }
        if (active.empty()) continue;
        umapcu_status tick_rc = UMAPCU_OK;
        const double ta = now();
        try {
            tick_launch();
            tick_rc = tick_finish();
        } catch (const Error &e) {
            tick_rc = e.status;
        }
        const double tb = now();
        if (tick_rc != UMAPCU_OK) cudaStreamSynchronize(s);  // nothing in flight before buffers are released
        std::vector<ServeJob *> still, done;
        for (ServeJob *j : active) {
            if (tick_rc != UMAPCU_OK) {
                j->rc = tick_rc;
            } else {
                j->epochs_done = std::min(j->epochs_done + tick_epochs, j->params.n_epochs);
                if (j->epochs_done < j->params.n_epochs) {
                    still.push_back(j);
                    continue;
                }
            }
            done.push_back(j);
        }
        active.swap(still);
        answer_snapshots(done);
        std::lock_guard<std::mutex> lk(mu);
        for (ServeJob *j : done) finishing.push_back(j);
        if (!done.empty()) cv_fin.notify_all();
        t_tick += tb - ta;
    }
    // shutting down: fail everything that has not finished
    std::lock_guard<std::mutex> lk(mu);
    for (auto *v : {&active, &ready})
        for (ServeJob *j : *v) {
            j->rc = UMAPCU_CANCELLED;
            j->state = kFailed;
            release_snapshot(j, UMAPCU_CANCELLED);
        }
    for (ServeJob *j : pending) {
        j->rc = UMAPCU_CANCELLED;
        j->state = kFailed;
    }
    active.clear();
    ready.clear();
    pending.clear();
    cv_done.notify_all();
}

extern "C" {

umapcu_status umapcu_server_job_bytes(uint32_t n, uint32_t n_dim, uint64_t nnz, uint32_t n_epochs, uint64_t *bytes)
{
    if (!bytes) return UMAPCU_BAD_ARG;
    *bytes = job_bytes(n, n_dim, nnz, n_epochs);
    return UMAPCU_OK;
}

umapcu_status umapcu_server_create(uint64_t device_budget_bytes, uint32_t max_jobs, uint32_t tick_epochs,
                                   uint32_t n_dim, umapcu_server **out)
{
    try {
        if (!out || max_jobs == 0 || tick_epochs == 0 || n_dim < 2 || n_dim > 4) return UMAPCU_BAD_ARG;
        *out = nullptr;
        keep_pool_memory();  // jobs allocate and free continuously
        auto sv = std::make_unique<umapcu_server>();
        sv->s = sv->own.s;
        if (const char *e = getenv("UMAPCU_SERVE_CTAS_PER_SM")) sv->tick_ctas = std::max(1, std::min(8, atoi(e)));
        check_cuda(cudaGetDevice(&sv->device), "cudaGetDevice");
        sv->budget = device_budget_bytes;
        sv->max_jobs = max_jobs;
        sv->tick_epochs = tick_epochs;
        sv->n_dim = n_dim;
        umapcu_server *raw = sv.get();
        sv->th = std::thread([raw] { raw->loop(); });
        sv->finisher = std::thread([raw] { raw->finish_loop(); });
        for (int k = 0; k < kAdmitThreads; k++) sv->admitters[k] = std::thread([raw, k] { raw->admit_loop(k); });
        *out = sv.release();
        return UMAPCU_OK;
    } catch (const Error &e) {
        return e.status;
    } catch (...) {
        return UMAPCU_CUDA_LAUNCH;
    }
}

}  // extern "C"

namespace {

// Submit of a new job (m = v = nullptr, start_epoch = 0) or of a resumed one.
umapcu_status submit_job(umapcu_server *sv, uint32_t n, uint32_t n_dim, const float *embd, const uint64_t *adj_ptr,
                         const uint32_t *adj_col, const float *adj_w, const umapcu_optim_params *params,
                         uint64_t seed, uint32_t sampler, const float *m, const float *v, uint32_t start_epoch,
                         uint64_t *ticket)
{
    if (!sv || !ticket) return UMAPCU_BAD_ARG;
    if (n == 0) return UMAPCU_NO_DATA;
    if (!embd || !adj_ptr || !params || n_dim != sv->n_dim || params->n_epochs == 0 || sampler > UMAPCU_NEG_PHILOX)
        return UMAPCU_BAD_ARG;
    if (start_epoch >= params->n_epochs || (!m) != (!v)) return UMAPCU_BAD_ARG;
    const uint64_t nnz = adj_ptr[n];
    if (nnz && (!adj_col || !adj_w)) return UMAPCU_BAD_ARG;
    if (adj_ptr[0] != 0) return UMAPCU_BAD_ARG;
    for (uint32_t i = 0; i < n; i++)
        if (adj_ptr[i + 1] < adj_ptr[i]) return UMAPCU_BAD_ARG;
    auto j = std::make_unique<ServeJob>();
    j->n = n;
    j->n_dim = n_dim;
    j->params = *params;
    j->seed = seed;
    j->sampler = sampler;
    j->nnz = nnz;
    j->bytes = job_bytes(n, n_dim, nnz, params->n_epochs);
    if (j->bytes > sv->budget) return UMAPCU_CAPACITY;
    const uint64_t nt = (uint64_t)n * n_dim;
    j->o_col = align256(8ull * (n + 1));
    j->o_w = j->o_col + align256(4 * nnz);
    j->o_y = j->o_w + align256(4 * nnz);
    j->o_sc = j->o_y + align256(4 * nt);
    j->blk_bytes = j->o_sc + 16ull * params->n_epochs;
    j->start_epoch = start_epoch;
    j->epochs_done = start_epoch;
    if (m) {
        j->o_m = align256(j->blk_bytes);
        j->o_v = j->o_m + align256(4 * nt);
        j->blk_bytes = j->o_v + 4 * nt;
    }
    j->blk = sv->arena.alloc(j->blk_bytes, &j->chunk);
    if (!j->blk) {
        j->heap.resize(j->blk_bytes);
        j->blk = j->heap.data();
    }
    memcpy(j->blk, adj_ptr, 8ull * (n + 1));
    uint32_t *col = (uint32_t *)(j->blk + j->o_col);
    uint32_t bad = 0;
    for (uint64_t e = 0; e < nnz; e++) {
        const uint32_t c = adj_col[e];
        bad |= c >= n;
        col[e] = c;
    }
    if (bad) {
        sv->free_block(j.get());
        return UMAPCU_BAD_ARG;
    }
    memcpy(j->blk + j->o_w, adj_w, 4 * nnz);
    memcpy(j->blk + j->o_y, embd, 4 * nt);
    if (m) {
        memcpy(j->blk + j->o_m, m, 4 * nt);
        memcpy(j->blk + j->o_v, v, 4 * nt);
    }
    float4 *sc = (float4 *)(j->blk + j->o_sc);
    for (uint32_t e = 0; e < params->n_epochs; e++) {
        float f, ep, lr;
        epoch_scalars(*params, e, &f, &ep, &lr);
        sc[e] = make_float4(f, ep, lr, 0.0f);
    }
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) {
        sv->free_block(j.get());
        return UMAPCU_CANCELLED;
    }
    j->id = sv->next_id++;
    j->t_submit = sv->now();
    *ticket = j->id;
    sv->pending.push_back(j.get());
    sv->jobs[j->id] = std::move(j);
    sv->cv_admit.notify_all();
    return UMAPCU_OK;
}

}  // namespace

extern "C" {

umapcu_status umapcu_server_submit(umapcu_server *sv, uint32_t n, uint32_t n_dim, const float *embd,
                                   const uint64_t *adj_ptr, const uint32_t *adj_col, const float *adj_w,
                                   const umapcu_optim_params *params, uint64_t seed, uint32_t sampler,
                                   uint64_t *ticket)
{
    return submit_job(sv, n, n_dim, embd, adj_ptr, adj_col, adj_w, params, seed, sampler, nullptr, nullptr, 0,
                      ticket);
}

umapcu_status umapcu_server_submit_resume(umapcu_server *sv, uint32_t n, uint32_t n_dim, const float *embd,
                                          const uint64_t *adj_ptr, const uint32_t *adj_col, const float *adj_w,
                                          const umapcu_optim_params *params, uint64_t seed, uint32_t sampler,
                                          const float *m, const float *v, uint32_t epochs_done, uint64_t *ticket)
{
    if (!m || !v) return UMAPCU_BAD_ARG;
    return submit_job(sv, n, n_dim, embd, adj_ptr, adj_col, adj_w, params, seed, sampler, m, v, epochs_done,
                      ticket);
}

umapcu_status umapcu_server_snapshot(umapcu_server *sv, uint64_t ticket, float *embd, float *m, float *v,
                                     uint32_t *epochs_done)
{
    if (!sv || !embd || !epochs_done) return UMAPCU_BAD_ARG;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(ticket);
    if (it == sv->jobs.end()) return UMAPCU_BAD_ARG;
    ServeJob *j = it->second.get();
    if (j->state == kDone || j->state == kFailed || j->snap) return UMAPCU_BAD_ARG;
    const uint64_t nt = (uint64_t)j->n * j->n_dim;
    if (std::find(sv->pending.begin(), sv->pending.end(), j) != sv->pending.end()) {
        // not admitted yet: the state it was submitted with (admission cannot
        // take it from the queue while the lock is held)
        memcpy(embd, j->blk + j->o_y, 4 * nt);
        if (m) j->o_m ? (void)memcpy(m, j->blk + j->o_m, 4 * nt) : (void)memset(m, 0, 4 * nt);
        if (v) j->o_v ? (void)memcpy(v, j->blk + j->o_v, 4 * nt) : (void)memset(v, 0, 4 * nt);
        *epochs_done = j->start_epoch;
        return UMAPCU_OK;
    }
    ServeJob::Snapshot req;
    req.y = embd;
    req.m = m;
    req.v = v;
    j->snap = &req;
    sv->cv_work.notify_all();
    sv->cv_done.wait(lk, [&] { return req.done; });
    *epochs_done = req.epochs;
    return req.rc;
}

umapcu_status umapcu_server_poll(umapcu_server *sv, uint64_t ticket, int *state)
{
    if (!sv || !state) return UMAPCU_BAD_ARG;
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(ticket);
    if (it == sv->jobs.end()) return UMAPCU_BAD_ARG;
    *state = it->second->state;
    return UMAPCU_OK;
}

umapcu_status umapcu_server_cancel(umapcu_server *sv, uint64_t ticket)
{
    if (!sv) return UMAPCU_BAD_ARG;
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(ticket);
    if (it == sv->jobs.end()) return UMAPCU_BAD_ARG;
    ServeJob *j = it->second.get();
    if (j->state != kPending) return UMAPCU_BAD_ARG;  // admitted jobs run to completion
    for (auto q = sv->pending.begin(); q != sv->pending.end(); ++q)
        if (*q == j) {
            sv->pending.erase(q);
            break;
        }
    sv->free_block(j);
    j->rc = UMAPCU_CANCELLED;
    j->state = kFailed;
    j->t_done = sv->now();
    sv->cv_done.notify_all();
    return UMAPCU_OK;
}

umapcu_status umapcu_server_wait(umapcu_server *sv, uint64_t ticket, float *embd_out, double *latency_s,
                                 double *queue_s)
{
    if (!sv) return UMAPCU_BAD_ARG;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(ticket);
    if (it == sv->jobs.end()) return UMAPCU_BAD_ARG;
    ServeJob *j = it->second.get();
    sv->cv_done.wait(lk, [&] { return j->state == kDone || j->state == kFailed; });
    const umapcu_status rc = j->rc;
    if (rc == UMAPCU_OK && embd_out) std::copy(j->result.begin(), j->result.end(), embd_out);
    if (latency_s) *latency_s = j->t_done - j->t_submit;
    if (queue_s) *queue_s = (j->t_admit > 0 ? j->t_admit : j->t_done) - j->t_submit;
    sv->jobs.erase(it);
    return rc;
}

umapcu_status umapcu_server_stats(umapcu_server *sv, uint64_t *completed, uint64_t *ticks, uint64_t *peak_bytes,
                                  uint32_t *peak_jobs)
{
    if (!sv) return UMAPCU_BAD_ARG;
    std::lock_guard<std::mutex> lk(sv->mu);
    if (completed) *completed = sv->completed;
    if (ticks) *ticks = sv->ticks;
    if (peak_bytes) *peak_bytes = sv->peak_used;
    if (peak_jobs) *peak_jobs = sv->peak_jobs;
    return UMAPCU_OK;
}

void umapcu_server_destroy(umapcu_server *sv)
{
    if (!sv) return;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    sv->cv_admit.notify_all();
    if (sv->th.joinable()) sv->th.join();
    for (auto &t : sv->admitters)
        if (t.joinable()) t.join();
    sv->cv_fin.notify_all();
    if (sv->finisher.joinable()) sv->finisher.join();  // drains jobs already computed
    {
        // jobs an admission thread finished after the loop exited
        std::lock_guard<std::mutex> lk(sv->mu);
        for (ServeJob *j : sv->ready) {
            j->rc = UMAPCU_CANCELLED;
            j->state = kFailed;
            sv->release_snapshot(j, UMAPCU_CANCELLED);
        }
        for (auto &kv : sv->jobs) sv->release_snapshot(kv.second.get(), UMAPCU_CANCELLED);
        sv->ready.clear();
        sv->cv_done.notify_all();
        if (getenv("UMAPCU_TIMING"))
            fprintf(stderr,
                    "umapcu server: %llu ticks, %.3f s; %llu admission groups, %.3f s (summed over %d threads)\n",
                    (unsigned long long)sv->ticks, sv->t_tick, (unsigned long long)sv->groups, sv->t_build,
                    kAdmitThreads);
    }
    delete sv;
}

}  // extern "C"
