// Per-epoch lists of active CSR entries ("schedule lists").
//
// The edge schedule (umap_edge_schedule_update, umap_optimiser_gpu.rs:
// 940-955) is a fixed function of each entry's period: the cursor starts at
// the period, the entry is active in epoch e when cursor <= e, and an active
// entry's cursor then grows by its period (f32 additions). Simulating that
// recurrence once per state -- with the same f32 arithmetic, so every
// decision is the one the per-epoch scan would make -- yields for every
// epoch the active entries of every 32-node segment, in CSR order. The epoch
// kernel then reads only those records instead of streaming every entry's
// (cursor, period) and other endpoint each epoch.
//
// Layout: rec [R] = (CSR position, other endpoint) of the active entries,
// epoch-major, then segment, then CSR order; seg_ptr [n_epochs * nseg + 1] = exclusive scan of
// the per-(epoch, segment) counts, so epoch e, segment s owns
// rec[seg_ptr[e * nseg + s] .. seg_ptr[e * nseg + s + 1]).
#include <chrono>
#include <cstdlib>

#include <cub/cub.cuh>

#include "internal.cuh"

namespace umapcu {
namespace {

constexpr int kSchedWarps = 4;
// Segments with at most this many CSR entries keep their cursors in shared
// memory and are walked epoch by epoch (each (epoch, segment) cell written
// contiguously by one warp); longer ones walk chunk by chunk.
constexpr uint32_t kSchedCap = 1024;

// One warp per segment. counts [n_epochs][nseg] (pass 1) or, with rec
// non-null, the records written at seg_ptr (pass 2).
__global__ void __launch_bounds__(kSchedWarps * 32) k_sched_lists(const uint32_t *__restrict__ offsets,
                                                                  const uint32_t *__restrict__ other,
                                                                  const float2 *__restrict__ sched, uint32_t n,
                                                                  uint32_t nseg, uint32_t n_epochs,
                                                                  uint32_t *__restrict__ counts,
                                                                  const uint64_t *__restrict__ seg_ptr,
                                                                  uint2 *__restrict__ rec)
{
    extern __shared__ float2 cur[];  // [kSchedWarps][kSchedCap] (cursor, period)
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t s = blockIdx.x * kSchedWarps + warp;
    if (s >= nseg) return;  // warp-uniform
    float2 *my = cur + (size_t)warp * kSchedCap;
    const uint32_t beg = offsets[s * 32u], end = offsets[min(s * 32u + 32u, n)];
    const uint32_t len = end - beg;
    const unsigned lt = (1u << lane) - 1u;
    if (len <= kSchedCap) {
        // epoch-major: cursors in shared memory, one contiguous cell per epoch
        for (uint32_t i = lane; i < len; i += 32) {
            const float per = sched[beg + i].y;
            my[i] = make_float2(per, per);  // reset state: cursor = period
        }
        __syncwarp();
        uint64_t bases = 0;  // lane l: the cell offset of epoch (e & ~31) + l
        for (uint32_t e = 0; e < n_epochs; e++) {
            const float ef = (float)e;
            if (rec && (e & 31) == 0 && e + lane < n_epochs) bases = seg_ptr[(size_t)(e + lane) * nseg + s];
            uint64_t pos = rec ? __shfl_sync(0xFFFFFFFFu, bases, e & 31) : 0;
            uint32_t cnt = 0;
            for (uint32_t i0 = 0; i0 < len; i0 += 32) {
                const uint32_t i = i0 + lane;
                bool a = false;
                if (i < len) {
                    float2 c = my[i];
                    a = c.x <= ef;
                    if (a) my[i].x = c.x + c.y;
                }
                const unsigned m = __ballot_sync(0xFFFFFFFFu, a);
                if (rec && a) rec[pos + __popc(m & lt)] = make_uint2(beg + i, other[beg + i]);
                pos += __popc(m);
                cnt += __popc(m);
            }
            if (!rec && lane == 0) counts[(size_t)e * nseg + s] = cnt;
        }
        return;
    }
    // chunk-major for long segments: per-epoch running counts in global
    // memory order (chunk by chunk, CSR order within each cell)
    uint32_t *run = reinterpret_cast<uint32_t *>(my);  // n_epochs <= 2 * kSchedCap words
    for (uint32_t e = lane; e < n_epochs; e += 32) run[e] = 0;
    __syncwarp();
    for (uint32_t c0 = beg; c0 < end; c0 += 32u) {
        const uint32_t p = c0 + lane;
        const bool live = p < end;
        float c = 0.0f, per = 0.0f;
        uint32_t o = 0;
        if (live) {
            per = sched[p].y;
            c = per;
            if (rec) o = other[p];
        }
        for (uint32_t e = 0; e < n_epochs; e++) {
            const bool a = live && c <= (float)e;
            if (a) c = c + per;
            const unsigned m = __ballot_sync(0xFFFFFFFFu, a);
            if (m) {
                if (rec && a) rec[seg_ptr[(size_t)e * nseg + s] + run[e] + __popc(m & lt)] = make_uint2(p, o);
                __syncwarp();
                if (lane == 0) run[e] += __popc(m);
                __syncwarp();
            }
        }
    }
    if (!rec) {
        __syncwarp();
        for (uint32_t e = lane; e < n_epochs; e += 32) counts[(size_t)e * nseg + s] = run[e];
    }
}

// Cursors after `epochs` epochs of the schedule from the reset state.
__global__ void k_sched_materialise(float2 *__restrict__ sched, uint64_t n_entries, uint32_t epochs)
{
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_entries) return;
    const float per = sched[p].y;
    float c = per;
    for (uint32_t e = 0; e < epochs; e++)
        if (c <= (float)e) c = c + per;
    sched[p].x = c;
}

}  // namespace

bool build_schedule_lists(const DeviceCsr &csr, uint32_t n_epochs, ScheduleLists &out, cudaStream_t s)
{
    out = ScheduleLists();
    const uint32_t n = csr.n, nseg = ceil_div(n, 32);
    if (!n || !n_epochs || n_epochs > 2 * kSchedCap || !csr.n_edges) return false;
    const uint64_t cells = (uint64_t)n_epochs * nseg;
    const size_t smem = (size_t)kSchedWarps * kSchedCap * sizeof(float2);
    const unsigned grid = ceil_div(nseg, kSchedWarps);
    check_cuda(cudaFuncSetAttribute(k_sched_lists, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
               "smem attribute");
    const bool timing = getenv("UMAPCU_TIMING") != nullptr;
    auto t0 = std::chrono::steady_clock::now();
    auto lap = [&](const char *what) {
        if (!timing) return;
        sync(s);
        auto t1 = std::chrono::steady_clock::now();
        fprintf(stderr, "umapcu timing:   lists %-10s %9.3f ms\n", what,
                std::chrono::duration<double, std::milli>(t1 - t0).count());
        t0 = t1;
    };
    DevBuf<uint32_t> counts(cells, s);
    lap("alloc");
    k_sched_lists<<<grid, kSchedWarps * 32, smem, s>>>(csr.offsets.p, csr.other.p, csr.sched.p, n, nseg, n_epochs,
                                                       counts.p, nullptr, nullptr);
    check_launch("k_sched_lists count");
    lap("count");
    DevBuf<uint64_t> ptr(cells + 1, s);
    check_cuda(cudaMemsetAsync(ptr.p + cells, 0, sizeof(uint64_t), s), "memset");
    {
        size_t tb = 0;
        check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, tb, counts.p, ptr.p, (int64_t)cells, s), "scan size");
        DevBuf<char> tmp(tb ? tb : 1, s);
        check_cuda(cub::DeviceScan::ExclusiveSum(tmp.p, tb, counts.p, ptr.p, (int64_t)cells, s), "scan");
    }
    uint64_t last_ptr = 0;
    uint32_t last_cnt = 0;
    d2h(&last_ptr, ptr.p + cells - 1, 1, s);
    d2h(&last_cnt, counts.p + cells - 1, 1, s);
    sync(s);
    const uint64_t R = last_ptr + last_cnt;
    h2d(ptr.p + cells, &R, 1, s);
    // the records must fit comfortably beside everything else
    size_t free_b = 0, total_b = 0;
    check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    if (R * sizeof(uint2) > free_b / 2) {
        sync(s);
        return false;
    }
    lap("scan");
    DevBuf<uint2> rec(R ? R : 1, s);
    lap("alloc rec");
    k_sched_lists<<<grid, kSchedWarps * 32, smem, s>>>(csr.offsets.p, csr.other.p, csr.sched.p, n, nseg, n_epochs,
                                                       nullptr, ptr.p, rec.p);
    check_launch("k_sched_lists fill");
    lap("fill");
    out.rec = std::move(rec);
    out.seg_ptr = std::move(ptr);
    out.n_records = R;
    out.n_epochs = n_epochs;
    out.nseg = nseg;
    return true;
}

void materialise_schedule(DeviceCsr &csr, uint32_t epochs, cudaStream_t s)
{
    const uint64_t tot = 2 * csr.n_edges;
    if (!tot) return;
    k_sched_materialise<<<ceil_div(tot, 256), 256, 0, s>>>(csr.sched.p, tot, epochs);
    check_launch("k_sched_materialise");
}

}  // namespace umapcu
