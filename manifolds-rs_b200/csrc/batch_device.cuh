// Multi-problem epoch kernels (batched and served forms). See batch.cu.
#pragma once

#include <algorithm>

#include "epoch_device.cuh"

namespace umapcu {

struct BatchProblem {
    uint32_t n, nseg, seg_base;
    uint32_t epoch_base;  // epochs this problem had completed before the launch
    uint32_t n_epochs;    // the problem's own epoch count (items past it do nothing)
    uint32_t pad0;
    const uint32_t *offsets;
    const uint32_t *other;
    float2 *sched;
    float *y0, *y1, *m, *v;
    const float4 *scal;  // [n_epochs] {fused, epsc, lr_e, 0}
    const float *init;   // [n * n_dim] initial embedding (restored by every run)
    const uint32_t *bits;  // [n_epochs][bits_words] schedule bitmasks (batched form), or nullptr
    uint64_t bits_words;
    uint64_t n_entries;  // 2E
    float a, b, two_a_b, two_gamma_b, omb1, omb2;
    uint32_t neg_rate, sampler, seed32, seed_lo, seed_hi, pad1;
    uint64_t fastmod_M;
};

struct BatchArgs {
    const BatchProblem *probs;
    const uint32_t *seg_prob;  // [n_segs] problem of each segment
    uint32_t n_probs, n_segs, n_epochs, optimiser;
    uint32_t *work;            // [1] next work item
    uint32_t *done;            // [n_probs] segments finished (all epochs so far)
    uint32_t *error;           // [1] 0, or the status that stopped the launch
    uint32_t wait_limit;       // polls before a wait gives up
    uint32_t poison;           // test hook: problem whose barrier never opens (~0u: none)
};

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Arguments of epoch e of problem P (e counts from the problem's own start).
__device__ __forceinline__ void epoch_args_of(const BatchProblem &P, uint32_t e, uint32_t optimiser, uint32_t *err,
                                              EpochArgs &A)
{
    A.n = P.n;
    A.n_entries = P.n_entries;
    A.err = err;  // checked builds report a bad index in the launch's status word
    A.offsets = P.offsets;
    A.other = P.other;
    A.sched = P.sched;
    A.bits = P.bits ? P.bits + (size_t)e * P.bits_words : nullptr;
    A.y_cur = (e & 1) ? P.y1 : P.y0;
    A.y_next = (e & 1) ? P.y0 : P.y1;
    A.m = P.m;
    A.v = P.v;
    const float4 sc = P.scal[e];
    A.fused = sc.x;
    A.epsc = sc.y;
    A.lr_sgd = sc.z;
    A.epoch = e;
    A.epoch_f = (float)e;
    A.a = P.a;
    A.b = P.b;
    A.two_a_b = P.two_a_b;
    A.two_gamma_b = P.two_gamma_b;
    A.omb1 = P.omb1;
    A.omb2 = P.omb2;
    A.neg_rate = P.neg_rate;
    A.sampler = P.sampler;
    A.seed32 = P.seed32;
    A.seed_lo = P.seed_lo;
    A.seed_hi = P.seed_hi;
    A.fastmod_M = P.fastmod_M;
    A.optimiser = optimiser;
}

// BITS: every problem has its schedule bitmasks (P.bits), scanned in place of
// the cursors.
template <int D, int NR, int KU, bool FAST = false, bool BITS = false>
__global__ void __launch_bounds__(kWarps * 32, 8) k_batch_persistent(const BatchArgs B)
{
    __shared__ WarpSmem<D, KU, BITS, false> smem[kWarps];
    __shared__ EpochArgs sargs[kWarps];  // per-warp arguments of the current item (kept out of registers)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t total = B.n_epochs * B.n_segs;
    for (;;) {
        uint32_t w = 0;
        if (lane == 0) w = atomicAdd(B.work, 1u);
        w = __shfl_sync(kFull, w, 0);
        if (w >= total) break;
        const uint32_t e = w / B.n_segs, s = w - e * B.n_segs;
        const uint32_t p = B.seg_prob[s];
        const BatchProblem &P = B.probs[p];
        int ok = 1;
        if (lane == 0) {
            const uint32_t need = e * P.nseg + (p == B.poison ? 1u : 0u);
            uint32_t it = 0;
            while (ld_acquire(&B.done[p]) < need) {
                if (++it > B.wait_limit || *(volatile uint32_t *)B.error) {
                    atomicCAS(B.error, 0u, (uint32_t)UMAPCU_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(128);
            }
        }
        ok = __shfl_sync(kFull, ok, 0);
        if (!ok) break;
        const uint32_t ej = P.epoch_base + e;
        if (ej < P.n_epochs) {
            if (lane == 0) {
                EpochArgs A{};
                epoch_args_of(P, ej, B.optimiser, B.error, A);
                sargs[warp] = A;
            }
            __syncwarp();
            epoch_segment<D, false, NR, true, KU, FAST, false, BITS>(sargs[warp], smem[warp], (s - P.seg_base) * 32u,
                                                                     lane);
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicAdd(&B.done[p], 1u);
    }
}

template <int D, int NR, int KU, bool FAST = false, bool BITS = false>
__global__ void __launch_bounds__(kWarps * 32, 8) k_batch_epoch(const BatchArgs B, uint32_t e)
{
    __shared__ WarpSmem<D, KU, BITS, false> smem[kWarps];
    __shared__ EpochArgs sargs[kWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t s = blockIdx.x * kWarps + warp;
    if (s >= B.n_segs) return;
    const BatchProblem &P = B.probs[B.seg_prob[s]];
    const uint32_t ej = P.epoch_base + e;
    if (ej >= P.n_epochs) return;
    if (lane == 0) {
        EpochArgs A{};
        epoch_args_of(P, ej, B.optimiser, B.error, A);
        sargs[warp] = A;
    }
    __syncwarp();
    epoch_segment<D, false, NR, false, KU, FAST, false, BITS>(sargs[warp], smem[warp], (s - P.seg_base) * 32u, lane);
}

struct BatchConfig {
    int mode = 0;        // 1 persistent, 2 per-epoch graph
    int ctas_per_sm = 8; // persistent grid = ctas_per_sm * SMs
    int ku = 8;          // scan super-chunk width
};

// fast: every problem uses the reference hash sampler (the batched and served
// forms have no injected negatives and no precise mode), so the kernels can
// take the compile-time fast path.
template <int D, bool FAST, bool BITS>
inline void launch_batch_kernel_t(const BatchArgs &B, const BatchConfig &c, cudaStream_t s, uint32_t epoch)
{
    if (c.mode == 1) {
        const unsigned grid = (unsigned)(c.ctas_per_sm * device_sm_count());
        if (c.ku == 4) k_batch_persistent<D, 5, 4, FAST, BITS><<<grid, kWarps * 32, 0, s>>>(B);
        else k_batch_persistent<D, 5, 8, FAST, BITS><<<grid, kWarps * 32, 0, s>>>(B);
    } else {
        const unsigned grid = ceil_div(B.n_segs, kWarps);
        if (c.ku == 4) k_batch_epoch<D, 5, 4, FAST, BITS><<<grid, kWarps * 32, 0, s>>>(B, epoch);
        else k_batch_epoch<D, 5, 8, FAST, BITS><<<grid, kWarps * 32, 0, s>>>(B, epoch);
    }
    check_launch("k_batch");
}

// bits: every problem carries its schedule bitmasks (P.bits), scanned in
// place of the cursors (the batched form with the fast kernels; the served
// form always)
template <int D>
inline void launch_batch_kernel(const BatchArgs &B, const BatchConfig &c, cudaStream_t s, uint32_t epoch,
                                bool fast, bool bits = false)
{
    if (fast && bits) launch_batch_kernel_t<D, true, true>(B, c, s, epoch);
    else if (fast) launch_batch_kernel_t<D, true, false>(B, c, s, epoch);
    else if (bits) launch_batch_kernel_t<D, false, true>(B, c, s, epoch);
    else launch_batch_kernel_t<D, false, false>(B, c, s, epoch);
}

// Problems with other negative sample rates (NR = 0: the rate is a runtime
// value); bits as above.
template <int D>
inline void launch_batch_kernel_nr0(const BatchArgs &B, const BatchConfig &c, cudaStream_t s, uint32_t epoch,
                                    bool bits = false)
{
    if (c.mode == 1) {
        const unsigned grid = (unsigned)(c.ctas_per_sm * device_sm_count());
        if (bits) k_batch_persistent<D, 0, 8, false, true><<<grid, kWarps * 32, 0, s>>>(B);
        else if (c.ku == 4) k_batch_persistent<D, 0, 4><<<grid, kWarps * 32, 0, s>>>(B);
        else k_batch_persistent<D, 0, 8><<<grid, kWarps * 32, 0, s>>>(B);
    } else {
        const unsigned grid = ceil_div(B.n_segs, kWarps);
        if (bits) k_batch_epoch<D, 0, 8, false, true><<<grid, kWarps * 32, 0, s>>>(B, epoch);
        else if (c.ku == 4) k_batch_epoch<D, 0, 4><<<grid, kWarps * 32, 0, s>>>(B, epoch);
        else k_batch_epoch<D, 0, 8><<<grid, kWarps * 32, 0, s>>>(B, epoch);
    }
    check_launch("k_batch");
}

}  // namespace umapcu
