// The edge schedule precomputed for a whole run, in two forms: per-epoch
// lists of active CSR entries ("schedule lists", resident states) and
// per-epoch bitmasks of them (the one-shot call).
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
// Layout: rec [R] = (packed entry, other endpoint) of the active entries
// (the entry as its node's index in the segment and its offset in the node's
// row, so the epoch kernel needs no search for the node),
// epoch-major, then work unit (units of a segment adjacent), then CSR order;
// ptr [n_epochs * n_units + 1] = exclusive scan of the per-(epoch, unit)
// counts and unit_base [nseg + 1] the segments' first units, so epoch e,
// segment s owns rec[ptr[e * n_units + unit_base[s]] ..
// ptr[e * n_units + unit_base[s + 1]]).
//
// Bitmasks: bits [n_epochs][ceil(2E / 32)], bit p & 31 of word p >> 5 set
// when entry p is active in that epoch; the epoch kernel scans these words
// in place of the (cursor, period) pairs.
#include <chrono>
#include <cstdlib>
#include <mutex>
#include <utility>

#include <cub/cub.cuh>

#include "internal.cuh"

namespace umapcu {
namespace {

constexpr int kSchedWarps = 4;
// A work unit is at most kSchedCap consecutive CSR entries of one segment
// (a segment of L entries has ceil(L / kSchedCap) units, at least one). One
// warp per unit: lane l owns the unit's entries l, l + 32, ..., and keeps
// their (cursor, period) -- and, when filling, their record fields -- in
// registers for the whole walk over the epochs.
constexpr uint32_t kSchedPer = 8;
constexpr uint32_t kSchedCap = 32 * kSchedPer;

__global__ void k_sched_units(const uint32_t *__restrict__ offsets, uint32_t n, uint32_t nseg,
                              uint32_t *__restrict__ units)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const uint32_t len = offsets[min(s * 32u + 32u, n)] - offsets[s * 32u];
    units[s] = len ? (len + kSchedCap - 1) / kSchedCap : 1u;
}

// unit_seg[u] = the segment of work unit u
__global__ void k_sched_unit_seg(const uint32_t *__restrict__ unit_base, uint32_t nseg, uint32_t *__restrict__ unit_seg)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    for (uint32_t u = unit_base[s]; u < unit_base[s + 1]; u++) unit_seg[u] = s;
}

// packed[p] = (node & 31) << kRecNodeShift | (p - offsets[node]) for every
// CSR entry p of node; *too_long set when a row does not fit the offset field
__global__ void k_sched_pack(const uint32_t *__restrict__ offsets, uint32_t n, uint32_t *__restrict__ packed,
                             uint32_t *__restrict__ too_long)
{
    const uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= n) return;
    const uint32_t b = offsets[node], e = offsets[node + 1];
    if (e - b > kRecOffsetMask + 1u) {
        *too_long = 1u;
        return;
    }
    for (uint32_t p = b; p < e; p++) packed[p] = ((node & 31u) << kRecNodeShift) | (p - b);
}

// One warp per unit. FILL = false: counts [n_epochs][n_units]; FILL = true:
// the records, written from ptr.
template <bool FILL>
__global__ void __launch_bounds__(kSchedWarps * 32) k_sched_lists(const uint32_t *__restrict__ offsets,
                                                                  const uint32_t *__restrict__ other,
                                                                  const uint32_t *__restrict__ packed,
                                                                  const float2 *__restrict__ sched, uint32_t n,
                                                                  const uint32_t *__restrict__ unit_seg,
                                                                  const uint32_t *__restrict__ unit_base,
                                                                  uint32_t n_units, uint32_t n_epochs,
                                                                  uint32_t *__restrict__ counts,
                                                                  const uint64_t *__restrict__ ptr,
                                                                  uint2 *__restrict__ rec)
{
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t u = blockIdx.x * kSchedWarps + warp;
    if (u >= n_units) return;  // warp-uniform
    const uint32_t sg = unit_seg[u], piece = u - unit_base[sg];
    const uint32_t sbeg = offsets[sg * 32u], send = offsets[min(sg * 32u + 32u, n)];
    const uint32_t beg = min(send, sbeg + piece * kSchedCap), end = min(send, beg + kSchedCap);
    const unsigned lt = (1u << lane) - 1u;
    float cur[kSchedPer], per[kSchedPer];
    uint2 rv[kSchedPer];
#pragma unroll
    for (uint32_t t = 0; t < kSchedPer; t++) {
        const uint32_t p = beg + 32u * t + lane;
        cur[t] = __int_as_float(0x7f800000);  // beyond the unit: never active
        per[t] = 0.0f;
        rv[t] = make_uint2(0, 0);
        if (p < end) {
            per[t] = sched[p].y;
            cur[t] = per[t];  // reset state: cursor = period
            if (FILL) rv[t] = make_uint2(packed[p], other[p]);
        }
    }
    uint64_t bases = 0;  // lane l: the record offset of epoch (e & ~31) + l
    uint32_t mine = 0;   // lane l: the count of epoch (e & ~31) + l
    for (uint32_t e = 0; e < n_epochs; e++) {
        const float ef = (float)e;
        if (FILL && (e & 31) == 0 && e + lane < n_epochs) bases = ptr[(size_t)(e + lane) * n_units + u];
        uint64_t pos = FILL ? __shfl_sync(0xFFFFFFFFu, bases, e & 31) : 0;
        uint32_t cnt = 0;
#pragma unroll
        for (uint32_t t = 0; t < kSchedPer; t++) {
            const bool a = cur[t] <= ef;
            if (a) cur[t] = cur[t] + per[t];
            const unsigned m = __ballot_sync(0xFFFFFFFFu, a);
            if (FILL) {
                if (a) rec[pos + __popc(m & lt)] = rv[t];
                pos += __popc(m);
            } else {
                cnt += __popc(m);
            }
        }
        if (!FILL) {
            if (lane == (e & 31)) mine = cnt;
            if ((e & 31) == 31 || e + 1 == n_epochs) {
                const uint32_t e0 = e & ~31u;
                if (e0 + lane <= e) counts[(size_t)(e0 + lane) * n_units + u] = mine;
            }
        }
    }
}

// Bitmasks: thread per 32-entry word, the word's cursors and periods in
// registers, one word written per epoch (coalesced across the warp). The
// walk starts from the reset schedule and writes the words of epochs
// [e_begin, n_epochs) only, so a run's epochs can be built in two launches.
__global__ void __launch_bounds__(128) k_sched_bits(const float2 *__restrict__ sched, uint64_t n_entries,
                                                    uint64_t words, uint32_t e_begin, uint32_t n_epochs,
                                                    uint32_t *__restrict__ bits)
{
    const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= words) return;
    float cur[32], per[32];
#pragma unroll
    for (int t = 0; t < 32; t++) {
        const uint64_t p = w * 32 + t;
        per[t] = p < n_entries ? sched[p].y : 0.0f;
        cur[t] = p < n_entries ? per[t] : __int_as_float(0x7f800000);  // reset: cursor = period
    }
    for (uint32_t e = 0; e < n_epochs; e++) {
        const float ef = (float)e;
        uint32_t word = 0;
#pragma unroll
        for (int t = 0; t < 32; t++) {
            const bool a = cur[t] <= ef;
            if (a) cur[t] = cur[t] + per[t];
            word |= (a ? 1u : 0u) << t;
        }
        if (e >= e_begin) bits[(size_t)e * words + w] = word;
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

// Cursors of the entries [offsets[node_lo], offsets[node_lo] + count) after
// `epochs` epochs from the reset schedule.
__global__ void k_sched_materialise_range(const uint32_t *__restrict__ offsets, uint32_t node_lo, uint64_t count,
                                          float2 *__restrict__ sched, uint32_t epochs)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint64_t p = offsets[node_lo] + t;
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
    if (!n || !n_epochs || n_epochs > 4096 || !csr.n_edges) return false;
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
    // work units per segment -> unit_base [nseg + 1]
    DevBuf<uint32_t> units(nseg, s), unit_base(nseg + 1, s);
    k_sched_units<<<ceil_div(nseg, 256), 256, 0, s>>>(csr.offsets.p, n, nseg, units.p);
    check_launch("k_sched_units");
    {
        size_t tb = 0;
        check_cuda(cub::DeviceScan::InclusiveSum(nullptr, tb, units.p, unit_base.p + 1, (int64_t)nseg, s), "scan size");
        DevBuf<char> tmp(tb ? tb : 1, s);
        check_cuda(cub::DeviceScan::InclusiveSum(tmp.p, tb, units.p, unit_base.p + 1, (int64_t)nseg, s), "scan");
    }
    check_cuda(cudaMemsetAsync(unit_base.p, 0, sizeof(uint32_t), s), "memset");
    DevBuf<uint32_t> packed(2 * csr.n_edges, s), too_long(1, s);
    check_cuda(cudaMemsetAsync(too_long.p, 0, sizeof(uint32_t), s), "memset");
    k_sched_pack<<<ceil_div(n, 256), 256, 0, s>>>(csr.offsets.p, n, packed.p, too_long.p);
    check_launch("k_sched_pack");
    uint32_t n_units = 0, long_row = 0;
    d2h(&n_units, unit_base.p + nseg, 1, s);
    d2h(&long_row, too_long.p, 1, s);
    sync(s);
    if (long_row) return false;
    DevBuf<uint32_t> unit_seg(n_units, s);
    k_sched_unit_seg<<<ceil_div(nseg, 256), 256, 0, s>>>(unit_base.p, nseg, unit_seg.p);
    check_launch("k_sched_unit_seg");
    const uint64_t cells = (uint64_t)n_epochs * n_units;
    const unsigned grid = ceil_div(n_units, kSchedWarps);
    DevBuf<uint32_t> counts(cells, s);
    lap("units");
    k_sched_lists<false><<<grid, kSchedWarps * 32, 0, s>>>(csr.offsets.p, csr.other.p, packed.p, csr.sched.p, n,
                                                          unit_seg.p, unit_base.p, n_units, n_epochs, counts.p,
                                                          nullptr, nullptr);
    check_launch("k_sched_lists count");
    lap("count");
    DevBuf<uint64_t> ptr(cells + 1, s);
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
    lap("scan");
    // the records must fit comfortably beside everything else
    size_t free_b = 0, total_b = 0;
    check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    if (R * sizeof(uint2) > free_b / 2) {
        sync(s);
        return false;
    }
    DevBuf<uint2> rec(R ? R : 1, s);
    lap("alloc rec");
    k_sched_lists<true><<<grid, kSchedWarps * 32, 0, s>>>(csr.offsets.p, csr.other.p, packed.p, csr.sched.p, n,
                                                         unit_seg.p, unit_base.p, n_units, n_epochs, nullptr, ptr.p,
                                                         rec.p);
    check_launch("k_sched_lists fill");
    lap("fill");
    out.rec = std::move(rec);
    out.ptr = std::move(ptr);
    out.unit_base = std::move(unit_base);
    out.n_records = R;
    out.n_epochs = n_epochs;
    out.nseg = nseg;
    out.n_units = n_units;
    return true;
}

namespace {

// One cached bitmask block per device (cudaMalloc, outside the stream-ordered
// pool); a call that finds it taken by a concurrent call allocates its own.
std::mutex g_bits_mu;
struct BitsBlock {
    uint32_t *p = nullptr;
    size_t cap = 0;
};
BitsBlock g_bits_cache[64];

}  // namespace

void ScheduleBits::release()
{
    if (!bits) return;
    if (built_on) cudaStreamSynchronize(built_on);
    if (side) {
        cudaStreamSynchronize(side);
        cudaStreamDestroy(side);
        side = nullptr;
    }
    if (rest) {
        cudaEventDestroy(rest);
        rest = nullptr;
    }
    first = 0;
    waited = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_bits_mu);
        if (dev >= 0 && dev < 64 && !g_bits_cache[dev].p) {
            g_bits_cache[dev] = BitsBlock{bits, cap};
        } else {
            cudaFree(bits);  // a concurrent call's block: the cache holds one
        }
    }
    bits = nullptr;
    cap = 0;
    words = 0;
    n_epochs = 0;
    built_on = nullptr;
}

void release_cached_bits()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    BitsBlock blk;
    {
        std::lock_guard<std::mutex> lk(g_bits_mu);
        std::swap(blk, g_bits_cache[dev]);
    }
    if (blk.p) cudaFree(blk.p);
}

void launch_schedule_bits(const float2 *sched, uint64_t n_entries, uint32_t n_epochs, uint32_t *bits,
                          cudaStream_t s, uint32_t e_begin)
{
    const uint64_t words = (n_entries + 31) / 32;
    if (!words || e_begin >= n_epochs) return;
    k_sched_bits<<<ceil_div(words, 128), 128, 0, s>>>(sched, n_entries, words, e_begin, n_epochs, bits);
    check_launch("k_sched_bits");
}

bool build_schedule_bits(const DeviceCsr &csr, uint32_t n_epochs, ScheduleBits &out, cudaStream_t s)
{
    const uint64_t entries = 2 * csr.n_edges;
    if (out.bits || !entries || !n_epochs) return false;
    const uint64_t words = (entries + 31) / 32;
    const size_t need = (size_t)n_epochs * words;
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) return false;
    BitsBlock blk;
    {
        std::lock_guard<std::mutex> lk(g_bits_mu);
        std::swap(blk, g_bits_cache[dev]);
    }
    if (blk.cap < need) {
        if (blk.p) {
            sync(s);  // the stream may still be using device memory; the block itself is idle
            cudaFree(blk.p);
            blk = BitsBlock{};
        }
        size_t free_b = 0, total_b = 0;
        check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
        if (need * sizeof(uint32_t) > free_b / 2) return false;
        if (cudaMalloc((void **)&blk.p, need * sizeof(uint32_t)) != cudaSuccess) {
            cudaGetLastError();  // an allocation failure is not sticky: no bitmasks, the scan runs
            return false;
        }
        blk.cap = need;
    }
    out.bits = blk.p;
    out.cap = blk.cap;
    out.dev = dev;
    out.built_on = s;
    out.words = words;
    out.n_epochs = n_epochs;
    // The first kBitsFirst epochs' words on s, the rest on a side stream
    // that starts after them: the run's first epochs then overlap the build
    // of the later words (run_epoch waits for out.rest before epoch
    // kBitsFirst).
    if (n_epochs <= 2 * kBitsFirst || need < kBitsSplitWords) {
        launch_schedule_bits(csr.sched.p, entries, n_epochs, out.bits, s);
        return true;
    }
    launch_schedule_bits(csr.sched.p, entries, kBitsFirst, out.bits, s);
    check_cuda(cudaStreamCreateWithFlags(&out.side, cudaStreamNonBlocking), "cudaStreamCreate");
    check_cuda(cudaEventCreateWithFlags(&out.rest, cudaEventDisableTiming), "cudaEventCreate");
    check_cuda(cudaEventRecord(out.rest, s), "cudaEventRecord");
    check_cuda(cudaStreamWaitEvent(out.side, out.rest, 0), "cudaStreamWaitEvent");
    launch_schedule_bits(csr.sched.p, entries, n_epochs, out.bits, out.side, kBitsFirst);
    check_cuda(cudaEventRecord(out.rest, out.side), "cudaEventRecord");
    out.first = kBitsFirst;
    return true;
}

void materialise_schedule_range(DeviceCsr &csr, uint32_t node_lo, uint64_t count, uint32_t epochs, cudaStream_t s)
{
    if (!count) return;
    k_sched_materialise_range<<<ceil_div(count, 256), 256, 0, s>>>(csr.offsets.p, node_lo, count, csr.sched.p, epochs);
    check_launch("k_sched_materialise_range");
}

void materialise_schedule(DeviceCsr &csr, uint32_t epochs, cudaStream_t s)
{
    const uint64_t tot = 2 * csr.n_edges;
    if (!tot) return;
    k_sched_materialise<<<ceil_div(tot, 256), 256, 0, s>>>(csr.sched.p, tot, epochs);
    check_launch("k_sched_materialise");
}

}  // namespace umapcu
