// Batched form: many independent UMAP layouts of uneven size in one
// persistent launch.
//
// Every problem keeps its own device CSR, embedding buffers and Adam state.
// The 32-node segments of all problems form one segment table; a work item is
// (epoch, segment), numbered epoch-major. In the persistent kernel each warp
// claims items in that order with one atomic counter and, before it runs an
// item of epoch e, waits until every segment of the same problem has finished
// epoch e - 1 (a per-problem completion counter, release/acquire). Problems
// therefore advance independently -- a small problem is never held back by a
// large one, and there is no grid-wide barrier. Because items are claimed in
// epoch order, every item a warp waits for has already been claimed by a
// running warp, so the wait always ends; it is bounded nonetheless: past
// wait_limit polls the warp records UMAPCU_TIMEOUT in the error word and the
// whole launch drains. The whole run (state reset + the persistent kernel) is
// captured in a CUDA graph and replayed.
//
// Inside the persistent kernel the embedding buffers, moments and cursors are
// rewritten every epoch by warps on other SMs, so epoch_segment runs with
// COH = true: those loads bypass L1 and the non-coherent path.
//
// The per-epoch alternative launches one kernel per epoch over all segments
// (the kernel boundary is the barrier), also captured in a graph. The
// autotuner times both, with several CTA counts and super-chunk widths, on
// the batch itself and keeps the fastest.
//
// With the reference hash sampler and neg_rate 5 (the fast kernels) the
// batch precomputes each problem's schedule as per-epoch bitmasks at
// creation (schedule.cu); the kernels scan those in place of the cursors,
// which every run would otherwise stream and rewrite. Results are
// bit-identical either way.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <memory>
#include <vector>

#include "batch_device.cuh"

namespace umapcu {

// Restores every problem's initial state (embedding, zero moments, cursors
// at one period): blockIdx.y = problem.
__global__ void k_batch_reset(const BatchProblem *__restrict__ probs, uint32_t n_dim)
{
    const BatchProblem &P = probs[blockIdx.y];
    const uint64_t nt = (uint64_t)P.n * n_dim;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += stride) {
        P.y0[i] = P.init[i];
        P.m[i] = 0.0f;
        P.v[i] = 0.0f;
    }
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < P.n_entries; q += stride) {
        const float2 v = P.sched[q];
        P.sched[q] = make_float2(v.y, v.y);
    }
}

}  // namespace umapcu

using namespace umapcu;

struct umapcu_batch {
    Stream own;
    cudaStream_t s = nullptr;
    uint32_t n_probs = 0, n_dim = 0, n_epochs = 0, n_segs = 0;
    bool all_nr5 = true;
    uint32_t sampler = UMAPCU_NEG_REF_HASH;
    std::vector<uint32_t> n;
    std::vector<DeviceCsr> csr;
    std::vector<DevBuf<float>> y0, y1, m, v, init;
    std::vector<DevBuf<float4>> scal;
    std::vector<DevBuf<uint32_t>> bits;  // per-problem schedule bitmasks (when use_bits)
    bool use_bits = false;
    std::vector<BatchProblem> hprobs;
    DevBuf<BatchProblem> probs;
    DevBuf<uint32_t> seg_prob;
    DevBuf<uint32_t> ctr;  // [2 + n_probs]: work, error, done[]
    BatchConfig cfg;
    bool tuned = false;
    cudaGraphExec_t exec = nullptr;
    BatchConfig exec_cfg;
    uint32_t exec_epochs = 0;
    ~umapcu_batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
    }
};

namespace {

template <typename F>
umapcu_status guard_b(F &&f)
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

BatchArgs batch_args(umapcu_batch *b, uint32_t epochs, uint32_t wait_limit, uint32_t poison)
{
    BatchArgs B{};
    B.probs = b->probs.p;
    B.seg_prob = b->seg_prob.p;
    B.n_probs = b->n_probs;
    B.n_segs = b->n_segs;
    B.n_epochs = epochs;
    B.optimiser = UMAPCU_OPT_ADAM;
    B.work = b->ctr.p;
    B.error = b->ctr.p + 1;
    B.done = b->ctr.p + 2;
    B.wait_limit = wait_limit;
    B.poison = poison;
    return B;
}

// Enqueues one full run (state reset + all epochs) on b->s.
void enqueue_run(umapcu_batch *b, const BatchConfig &c, uint32_t epochs, uint32_t wait_limit = 1u << 24,
                 uint32_t poison = ~0u)
{
    cudaStream_t s = b->s;
    k_batch_reset<<<dim3(64, b->n_probs), 256, 0, s>>>(b->probs.p, b->n_dim);
    check_launch("k_batch_reset");
    check_cuda(cudaMemsetAsync(b->ctr.p, 0, (2 + b->n_probs) * sizeof(uint32_t), s), "memset counters");
    const BatchArgs B = batch_args(b, epochs, wait_limit, poison);
    const uint32_t launches = c.mode == 1 ? 1 : epochs;
    for (uint32_t e = 0; e < launches; e++) {
        switch (b->n_dim) {
            case 2: b->all_nr5 ? launch_batch_kernel<2>(B, c, s, e, b->sampler == UMAPCU_NEG_REF_HASH, b->use_bits) : launch_batch_kernel_nr0<2>(B, c, s, e); break;
            case 3: b->all_nr5 ? launch_batch_kernel<3>(B, c, s, e, b->sampler == UMAPCU_NEG_REF_HASH, b->use_bits) : launch_batch_kernel_nr0<3>(B, c, s, e); break;
            case 4: b->all_nr5 ? launch_batch_kernel<4>(B, c, s, e, b->sampler == UMAPCU_NEG_REF_HASH, b->use_bits) : launch_batch_kernel_nr0<4>(B, c, s, e); break;
            default: fail(UMAPCU_BAD_ARG, "batched n_dim must be 2, 3 or 4");
        }
    }
}

// Captures enqueue_run in a CUDA graph (cached per config / epoch count).
void run_graph(umapcu_batch *b, const BatchConfig &c, uint32_t epochs)
{
    const bool same = b->exec && b->exec_cfg.mode == c.mode && b->exec_cfg.ctas_per_sm == c.ctas_per_sm &&
                      b->exec_cfg.ku == c.ku && b->exec_epochs == epochs;
    if (!same) {
        if (b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
        }
        cudaGraph_t g;
        check_cuda(cudaStreamBeginCapture(b->s, cudaStreamCaptureModeThreadLocal), "begin capture");
        try {
            enqueue_run(b, c, epochs);
        } catch (...) {
            cudaStreamEndCapture(b->s, &g);
            throw;
        }
        check_cuda(cudaStreamEndCapture(b->s, &g), "end capture");
        check_cuda(cudaGraphInstantiate(&b->exec, g, 0), "graph instantiate");
        cudaGraphDestroy(g);
        b->exec_cfg = c;
        b->exec_epochs = epochs;
    }
    check_cuda(cudaGraphLaunch(b->exec, b->s), "graph launch");
}

uint32_t read_error(umapcu_batch *b)
{
    uint32_t err = 0;
    d2h(&err, b->ctr.p + 1, 1, b->s);
    sync(b->s);
    return err;
}

float timed_run(umapcu_batch *b, const BatchConfig &c, uint32_t epochs)
{
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "event");
    check_cuda(cudaEventCreate(&e1), "event");
    run_graph(b, c, epochs);  // warm-up / instantiate
    sync(b->s);
    check_cuda(cudaEventRecord(e0, b->s), "record");
    run_graph(b, c, epochs);
    check_cuda(cudaEventRecord(e1, b->s), "record");
    sync(b->s);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms;
}

void autotune(umapcu_batch *b)
{
    const uint32_t trial = std::min<uint32_t>(b->n_epochs, 20);
    std::vector<BatchConfig> cands;
    for (int ku : {8, 4}) {
        for (int ctas : {8, 6, 4}) cands.push_back(BatchConfig{1, ctas, ku});
        cands.push_back(BatchConfig{2, 8, ku});
    }
    float best = 1e30f;
    BatchConfig bc = cands[0];
    for (const auto &c : cands) {
        const float ms = timed_run(b, c, trial);
        if (read_error(b) != 0) continue;
        if (getenv("UMAPCU_TIMING"))
            fprintf(stderr, "umapcu autotune: mode %d ctas/SM %d ku %d: %.3f ms / %u epochs\n", c.mode, c.ctas_per_sm,
                    c.ku, ms, trial);
        if (ms < best) {
            best = ms;
            bc = c;
        }
    }
    b->cfg = bc;
    b->tuned = true;
}

}  // namespace

extern "C" {

umapcu_status umapcu_batch_create(uint32_t n_problems, const uint32_t *n, uint32_t n_dim, const float *const *embd,
                                  const uint64_t *const *adj_ptr, const uint32_t *const *adj_col,
                                  const float *const *adj_w, const umapcu_optim_params *params, const uint64_t *seeds,
                                  uint32_t sampler, umapcu_batch **out)
{
    return guard_b([&]() -> umapcu_status {
        if (!out) return UMAPCU_BAD_ARG;
        *out = nullptr;
        if (n_problems == 0) return UMAPCU_NO_DATA;
        if (!n || !embd || !adj_ptr || !adj_col || !adj_w || !params || !seeds) return UMAPCU_BAD_ARG;
        if (n_dim < 2 || n_dim > 4 || sampler > UMAPCU_NEG_PHILOX) return UMAPCU_BAD_ARG;
        keep_pool_memory();
        const uint32_t n_epochs = params[0].n_epochs;
        for (uint32_t p = 0; p < n_problems; p++) {
            if (n[p] == 0) return UMAPCU_NO_DATA;
            if (!embd[p] || !adj_ptr[p] || params[p].n_epochs != n_epochs || n_epochs == 0) return UMAPCU_BAD_ARG;
        }
        auto b = std::make_unique<umapcu_batch>();
        b->s = b->own.s;
        cudaStream_t s = b->s;
        b->n_probs = n_problems;
        b->n_dim = n_dim;
        b->sampler = sampler;
        b->n_epochs = n_epochs;
        b->n.assign(n, n + n_problems);
        b->csr.resize(n_problems);
        b->y0.resize(n_problems);
        b->y1.resize(n_problems);
        b->m.resize(n_problems);
        b->v.resize(n_problems);
        b->init.resize(n_problems);
        b->scal.resize(n_problems);
        b->hprobs.resize(n_problems);
        std::vector<uint32_t> seg_prob;
        for (uint32_t p = 0; p < n_problems; p++) {
            const uint64_t nnz = adj_ptr[p][n[p]];
            {
                DevBuf<uint64_t> dptr(n[p] + 1, s);
                DevBuf<uint32_t> dcol(nnz, s);
                DevBuf<float> dw(nnz, s);
                h2d(dptr.p, adj_ptr[p], n[p] + 1, s);
                h2d(dcol.p, adj_col[p], nnz, s);
                h2d(dw.p, adj_w[p], nnz, s);
                umapcu_status rc = build_csr_dev(n[p], dptr.p, dcol.p, dw.p, nnz, b->csr[p], s);
                if (rc != UMAPCU_OK) return rc;
            }
            const uint64_t nt = (uint64_t)n[p] * n_dim;
            b->y0[p].alloc(nt, s);
            b->y1[p].alloc(nt, s);
            b->m[p].alloc(nt, s);
            b->v[p].alloc(nt, s);
            b->init[p].alloc(nt, s);
            h2d(b->init[p].p, embd[p], nt, s);
            std::vector<float4> sc(n_epochs);
            for (uint32_t e = 0; e < n_epochs; e++) {
                float f, ep, lr;
                epoch_scalars(params[p], e, &f, &ep, &lr);
                sc[e] = make_float4(f, ep, lr, 0.0f);
            }
            b->scal[p].alloc(n_epochs, s);
            h2d(b->scal[p].p, sc.data(), n_epochs, s);
            sync(s);  // sc leaves scope
            BatchProblem &P = b->hprobs[p];
            P.n = n[p];
            P.nseg = ceil_div(n[p], 32);
            P.epoch_base = 0;
            P.n_epochs = n_epochs;
            P.seg_base = (uint32_t)seg_prob.size();
            P.offsets = b->csr[p].offsets.p;
            P.other = b->csr[p].other.p;
            P.sched = b->csr[p].sched.p;
            P.y0 = b->y0[p].p;
            P.y1 = b->y1[p].p;
            P.m = b->m[p].p;
            P.v = b->v[p].p;
            P.scal = b->scal[p].p;
            P.init = b->init[p].p;
            P.n_entries = 2 * b->csr[p].n_edges;
            const umapcu_optim_params &q = params[p];
            P.a = q.a;
            P.b = q.b;
            P.two_a_b = 2.0f * q.a * q.b;
            P.two_gamma_b = 2.0f * q.gamma * q.b;
            P.omb1 = 1.0f - q.beta1;
            P.omb2 = 1.0f - q.beta2;
            P.neg_rate = q.neg_sample_rate;
            if (q.neg_sample_rate != 5) b->all_nr5 = false;
            P.sampler = sampler;
            P.seed32 = (uint32_t)seeds[p];
            P.seed_lo = (uint32_t)seeds[p];
            P.seed_hi = (uint32_t)(seeds[p] >> 32);
            P.fastmod_M = fastmod_magic(n[p]);
            for (uint32_t k = 0; k < P.nseg; k++) seg_prob.push_back(p);
        }
        if ((uint64_t)seg_prob.size() * n_epochs >= (1ull << 32)) return UMAPCU_BAD_ARG;
        // every run starts from the reset schedule and walks epochs 0, 1, ...
        // in order, so the fast kernels can scan per-epoch bitmasks of the
        // active entries in place of the cursors (bit-identical); skipped
        // when they would take more than half the free device memory
        if (b->all_nr5 && sampler == UMAPCU_NEG_REF_HASH && !getenv("UMAPCU_NO_SCHEDULE_LISTS")) {
            uint64_t words_total = 0;
            for (uint32_t p = 0; p < n_problems; p++) words_total += (b->hprobs[p].n_entries + 31) / 32;
            size_t free_b = 0, total_b = 0;
            check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
            if (words_total * n_epochs * sizeof(uint32_t) <= free_b / 2) {
                b->bits.resize(n_problems);
                for (uint32_t p = 0; p < n_problems; p++) {
                    BatchProblem &P = b->hprobs[p];
                    P.bits_words = (P.n_entries + 31) / 32;
                    b->bits[p].alloc((size_t)P.bits_words * n_epochs, s);
                    launch_schedule_bits(b->csr[p].sched.p, P.n_entries, n_epochs, b->bits[p].p, s);
                    P.bits = b->bits[p].p;
                }
                b->use_bits = true;
            }
        }
        b->n_segs = (uint32_t)seg_prob.size();
        b->probs.alloc(n_problems, s);
        h2d(b->probs.p, b->hprobs.data(), n_problems, s);
        b->seg_prob.alloc(seg_prob.size(), s);
        h2d(b->seg_prob.p, seg_prob.data(), seg_prob.size(), s);
        b->ctr.alloc(2 + n_problems, s);
        sync(s);
        *out = b.release();
        return UMAPCU_OK;
    });
}

void umapcu_batch_destroy(umapcu_batch *b) { delete b; }

umapcu_status umapcu_batch_autotune(umapcu_batch *b, uint32_t *mode, uint32_t *ctas_per_sm, uint32_t *ku)
{
    return guard_b([&]() -> umapcu_status {
        if (!b) return UMAPCU_BAD_ARG;
        autotune(b);
        if (mode) *mode = (uint32_t)b->cfg.mode;
        if (ctas_per_sm) *ctas_per_sm = (uint32_t)b->cfg.ctas_per_sm;
        if (ku) *ku = (uint32_t)b->cfg.ku;
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_batch_run(umapcu_batch *b, uint32_t mode, float *ms)
{
    return guard_b([&]() -> umapcu_status {
        if (!b || mode > 2) return UMAPCU_BAD_ARG;
        NvtxRange r("umapcu batch run");
        BatchConfig c = b->cfg;
        if (mode == 0 && !b->tuned) autotune(b);
        if (mode == 0) c = b->cfg;
        else c.mode = (int)mode;
        cudaEvent_t e0, e1;
        check_cuda(cudaEventCreate(&e0), "event");
        check_cuda(cudaEventCreate(&e1), "event");
        check_cuda(cudaEventRecord(e0, b->s), "record");
        run_graph(b, c, b->n_epochs);
        check_cuda(cudaEventRecord(e1, b->s), "record");
        sync(b->s);
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms) *ms = t;
        const uint32_t err = read_error(b);
        return err ? (umapcu_status)err : UMAPCU_OK;
    });
}

umapcu_status umapcu_batch_read(const umapcu_batch *b, uint32_t problem, float *embd)
{
    return guard_b([&]() -> umapcu_status {
        if (!b || !embd || problem >= b->n_probs) return UMAPCU_BAD_ARG;
        const uint64_t nt = (uint64_t)b->n[problem] * b->n_dim;
        const float *src = (b->n_epochs & 1) ? b->y1[problem].p : b->y0[problem].p;
        d2h(embd, src, nt, b->s);
        sync(b->s);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_batch_wait_check(umapcu_batch *b, uint32_t poisoned_problem, uint32_t wait_limit)
{
    return guard_b([&]() -> umapcu_status {
        if (!b || poisoned_problem >= b->n_probs) return UMAPCU_BAD_ARG;
        BatchConfig c = b->cfg;
        c.mode = 1;
        enqueue_run(b, c, b->n_epochs, wait_limit, poisoned_problem);
        sync(b->s);
        return (umapcu_status)read_error(b);
    });
}

}  // extern "C"
