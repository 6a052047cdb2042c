// Fuzzy simplicial set construction on the device (sm_100a).
//
// Stage chain of construct_umap_graph (src/lib.rs:296-306):
//   smooth_knn_dist (graph.rs:499-565)   -> k_smooth_knn_dist, one thread per row
//   knn_to_coo      (graph.rs:585-662)   -> k_knn_weights + order-preserving compaction
//   symmetrise_graph(graph.rs:684-694)   -> sort-based transpose + merge: every directed
//                                           entry is emitted as an "out" record keyed
//                                           (row, col) and an "in" record keyed (col, row);
//                                           one stable radix sort groups each (i, j) pair,
//                                           the group head evaluates the fuzzy union
//   filter_weak_edges (graph.rs:776-853) -> fused into the union's compaction (w >= max/N)
// and UmapCsrGraph::from_graph (umap_optimiser_gpu.rs:132-209) -> build_csr_dev.
//
// Arithmetic is evaluated in the reference's order with no FMA contraction
// (the translation unit is compiled with -fmad=false). exp is evaluated as
// (float)exp((double)x), i.e. correctly rounded except in double-rounding
// corner cases; the reference calls glibc expf.
#include <atomic>
#include <cfloat>

#include <cub/cub.cuh>

#include "internal.cuh"

namespace umapcu {

int device_sm_count()
{
    static std::atomic<int> cached{0};  // the same value from every thread
    int sms = cached.load(std::memory_order_relaxed);
    if (!sms) {
        int dev = 0;
        check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
        check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
        cached.store(sms, std::memory_order_relaxed);
    }
    return sms;
}

__device__ __forceinline__ float exp_ref(float x) { return (float)exp((double)x); }

// graph.rs:107-125 local_connectivity_distance
__device__ float local_connectivity_distance(const float *__restrict__ d, uint32_t k, float lc)
{
    if (lc <= 0.0f || k == 0) return 0.0f;
    float offset = fmaxf(lc - 1.0f, 0.0f);
    float whole = floorf(offset);
    float fraction = offset - whole;
    uint64_t idx = (whole >= 0.0f && whole < 1.8e19f) ? (uint64_t)whole : UINT64_MAX;
    if (idx > (uint64_t)(k - 1)) idx = k - 1;
    if (fraction > 0.0f && idx + 1 < k) return d[idx] * (1.0f - fraction) + d[idx + 1] * fraction;
    return d[idx];
}

// graph.rs:499-565: per-row bisection of sigma, sum of exp in f32 (folded
// from -0.0 like Rust's f32 Sum), comparison in f64.
__global__ void k_smooth_knn_dist(const float *__restrict__ dist, uint32_t n, uint32_t k, float lc,
                                  double tol, double target, uint32_t n_iter, float *__restrict__ sigma,
                                  float *__restrict__ rho)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *d = dist + (uint64_t)i * k;
    float r = local_connectivity_distance(d, k, lc);
    float lo = 0.0f, hi = FLT_MAX, mid = 1.0f;
    for (uint32_t it = 0; it < n_iter; it++) {
        float inv_mid = 1.0f / mid;
        float s = -0.0f;
        for (uint32_t t = 0; t < k; t++) s += exp_ref((-fmaxf(d[t] - r, 0.0f)) * inv_mid);
        double val = (double)s;
        if (fabs(val - target) < tol) break;
        if (val > target) {
            hi = mid;
            mid = (lo + hi) / 2.0f;
        } else {
            lo = mid;
            if (hi == FLT_MAX) mid *= 2.0f;
            else mid = (lo + hi) / 2.0f;
        }
    }
    sigma[i] = mid;
    rho[i] = r;
}

void smooth_knn_dist_dev(const float *d_dist, uint32_t n, uint32_t k, float local_connectivity,
                         float bandwidth, uint32_t n_iter, float *d_sigma, float *d_rho, cudaStream_t s)
{
    if (!n) return;
    const double target = log((double)k);
    k_smooth_knn_dist<<<ceil_div(n, 128), 128, 0, s>>>(d_dist, n, k, local_connectivity, (double)bandwidth,
                                                        target, n_iter, d_sigma, d_rho);
    check_launch("k_smooth_knn_dist");
}

// graph.rs:625-653: membership weight of every kNN entry; keep[] marks
// non-self entries.
__global__ void k_knn_weights(const int32_t *__restrict__ idx, const float *__restrict__ dist, uint32_t n,
                              uint32_t k, const float *__restrict__ sigma, const float *__restrict__ rho,
                              float *__restrict__ w_out, uint32_t *__restrict__ keep)
{
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (uint64_t)n * k) return;
    uint32_t i = (uint32_t)(p / k);
    float sg = sigma[i], r = rho[i];
    bool smooth = sg > 0.0f;
    float inv_sigma = smooth ? 1.0f / sg : 0.0f;
    float adjusted = fmaxf(dist[p] - r, 0.0f);
    float w;
    if (smooth) w = exp_ref((-adjusted) * inv_sigma);
    else if (adjusted > 0.0f) w = 0.0f;
    else w = 1.0f;
    w_out[p] = w;
    keep[p] = (uint32_t)idx[p] != i;
}

__global__ void k_compact_coo(const int32_t *__restrict__ idx, const float *__restrict__ w, uint64_t m,
                              uint32_t k, const uint32_t *__restrict__ keep, const uint32_t *__restrict__ pos,
                              uint32_t *__restrict__ row, uint32_t *__restrict__ col, float *__restrict__ val)
{
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m || !keep[p]) return;
    uint32_t o = pos[p];
    row[o] = (uint32_t)(p / k);
    col[o] = (uint32_t)idx[p];
    val[o] = w[p];
}

// Records for the fuzzy union: r < m is the out record of COO entry r
// (key row*n+col), r >= m the in record of entry r-m (key col*n+row).
__global__ void k_sym_records(const uint32_t *__restrict__ row, const uint32_t *__restrict__ col, uint64_t m,
                              uint64_t n, uint64_t *__restrict__ key, uint32_t *__restrict__ rec)
{
    uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= 2 * m) return;
    uint64_t e = r < m ? r : r - m;
    uint64_t a = row[e], b = col[e];
    key[r] = r < m ? a * n + b : b * n + a;
    rec[r] = (uint32_t)r;
}

// graph.rs:321-363 merge_row, one group of equal keys per head. After the
// stable sort a group holds its out records (input order) then its in
// records (input order); duplicates collapse to the last one of each kind.
// Writes the union weight at the head (0 elsewhere).
__global__ void k_sym_union(const uint64_t *__restrict__ key, const uint32_t *__restrict__ rec,
                            const float *__restrict__ val, uint64_t m, float mix_weight,
                            float *__restrict__ wsym, uint32_t *__restrict__ head)
{
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t tot = 2 * m;
    if (t >= tot) return;
    uint64_t kk = key[t];
    if (t > 0 && key[t - 1] == kk) {
        wsym[t] = 0.0f;
        head[t] = 0;
        return;
    }
    float w_ij = 0.0f, w_ji = 0.0f;
    for (uint64_t u = t; u < tot && key[u] == kk; u++) {
        uint32_t r = rec[u];
        if (r < m) w_ij = val[r];
        else w_ji = val[r - m];
    }
    const float directed_weight = 1.0f - mix_weight;
    float uni = (w_ij + w_ji) - w_ij * w_ji;
    float w = mix_weight * uni + directed_weight * w_ij;
    wsym[t] = w;
    head[t] = 1;
}

// filter_weak_edges (graph.rs:786-809) fused with the merge's "> min_weight"
// test: keep heads with w > 0 and w >= max/n_epochs.
__global__ void k_sym_keep(const float *__restrict__ wsym, const uint32_t *__restrict__ head, uint64_t tot,
                           const float *__restrict__ d_max, float n_epochs_f, uint32_t *__restrict__ keep)
{
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tot) return;
    float threshold = *d_max / n_epochs_f;
    float w = wsym[t];
    keep[t] = head[t] && w > 0.0f && w >= threshold;
}

__global__ void k_sym_scatter(const uint64_t *__restrict__ key, const float *__restrict__ wsym,
                              const uint32_t *__restrict__ keep, const uint32_t *__restrict__ pos, uint64_t tot,
                              uint64_t n, uint32_t *__restrict__ row, uint32_t *__restrict__ col,
                              float *__restrict__ val)
{
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tot || !keep[t]) return;
    uint32_t o = pos[t];
    uint64_t kk = key[t];
    row[o] = (uint32_t)(kk / n);
    col[o] = (uint32_t)(kk % n);
    val[o] = wsym[t];
}

struct MaxFrom0 {
    __device__ __forceinline__ float operator()(float a, float b) const { return b > a ? b : a; }
};

static int bits_for(uint64_t v)
{
    int b = 1;
    while (b < 64 && (1ull << b) <= v) b++;
    return b;
}

// Exclusive scan of u32 flags; returns the total. d_word (optional): a
// device word read back in the same synchronisation.
static uint64_t scan_flags(const uint32_t *d_flags, uint32_t *d_pos, uint64_t m, cudaStream_t s,
                           const uint32_t *d_word = nullptr, uint32_t *h_word = nullptr)
{
    if (d_word) d2h(h_word, d_word, 1, s);
    if (!m) {
        if (d_word) sync(s);
        return 0;
    }
    size_t tb = 0;
    check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_flags, d_pos, (int64_t)m, s), "scan size");
    DevBuf<char> tmp(tb ? tb : 1, s);
    check_cuda(cub::DeviceScan::ExclusiveSum(tmp.p, tb, d_flags, d_pos, (int64_t)m, s), "scan");
    uint32_t last_flag = 0, last_pos = 0;
    d2h(&last_flag, d_flags + m - 1, 1, s);
    d2h(&last_pos, d_pos + m - 1, 1, s);
    sync(s);
    return (uint64_t)last_pos + last_flag;
}

static void reduce_max0(const float *d_in, uint64_t m, float *d_out, cudaStream_t s)
{
    size_t tb = 0;
    check_cuda(cub::DeviceReduce::Reduce(nullptr, tb, d_in, d_out, (int64_t)m, MaxFrom0(), 0.0f, s), "max size");
    DevBuf<char> tmp(tb ? tb : 1, s);
    check_cuda(cub::DeviceReduce::Reduce(tmp.p, tb, d_in, d_out, (int64_t)m, MaxFrom0(), 0.0f, s), "max");
}

void construct_graph_dev(const int32_t *d_idx, const float *d_dist, uint32_t n, uint32_t k,
                         const umapcu_graph_params &gp, uint32_t n_epochs, DeviceCoo &out, float *d_sigma,
                         float *d_rho, cudaStream_t s)
{
    const uint64_t nk = (uint64_t)n * k;
    if (nk >= (1ull << 31)) fail(UMAPCU_BAD_ARG, "n*k too large");
    DevBuf<float> sig_own, rho_own;
    if (!d_sigma) { sig_own.alloc(n, s); d_sigma = sig_own.p; }
    if (!d_rho) { rho_own.alloc(n, s); d_rho = rho_own.p; }
    smooth_knn_dist_dev(d_dist, n, k, gp.local_connectivity, gp.bandwidth, 64, d_sigma, d_rho, s);

    // knn_to_coo
    DevBuf<float> w(nk, s);
    DevBuf<uint32_t> keep(nk, s), pos(nk, s);
    k_knn_weights<<<ceil_div(nk, 256), 256, 0, s>>>(d_idx, d_dist, n, k, d_sigma, d_rho, w.p, keep.p);
    check_launch("k_knn_weights");
    uint64_t m = scan_flags(keep.p, pos.p, nk, s);
    DevBuf<uint32_t> row(m, s), col(m, s);
    DevBuf<float> val(m, s);
    if (m) {
        k_compact_coo<<<ceil_div(nk, 256), 256, 0, s>>>(d_idx, w.p, nk, k, keep.p, pos.p, row.p, col.p, val.p);
        check_launch("k_compact_coo");
    }
    w.release(); keep.release(); pos.release();
    out.nnz = 0;
    if (!m) {
        out.row.alloc(0, s); out.col.alloc(0, s); out.val.alloc(0, s);
        return;
    }

    // symmetrise: stable sort of 2m records by (row, col)
    const uint64_t tot = 2 * m;
    DevBuf<uint64_t> key(tot, s), key_s(tot, s);
    DevBuf<uint32_t> rec(tot, s), rec_s(tot, s);
    k_sym_records<<<ceil_div(tot, 256), 256, 0, s>>>(row.p, col.p, m, n, key.p, rec.p);
    check_launch("k_sym_records");
    int end_bit = bits_for((uint64_t)n * n - 1);
    size_t tb = 0;
    check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.p, key_s.p, rec.p, rec_s.p, (int64_t)tot, 0,
                                               end_bit, s), "sort size");
    {
        DevBuf<char> tmp(tb ? tb : 1, s);
        check_cuda(cub::DeviceRadixSort::SortPairs(tmp.p, tb, key.p, key_s.p, rec.p, rec_s.p, (int64_t)tot, 0,
                                                   end_bit, s), "sort");
    }
    key.release(); rec.release();
    DevBuf<float> wsym(tot, s);
    DevBuf<uint32_t> head(tot, s), keep2(tot, s), pos2(tot, s);
    k_sym_union<<<ceil_div(tot, 256), 256, 0, s>>>(key_s.p, rec_s.p, val.p, m, gp.mix_weight, wsym.p, head.p);
    check_launch("k_sym_union");
    DevBuf<float> dmax(1, s);
    reduce_max0(wsym.p, tot, dmax.p, s);
    k_sym_keep<<<ceil_div(tot, 256), 256, 0, s>>>(wsym.p, head.p, tot, dmax.p, (float)n_epochs, keep2.p);
    check_launch("k_sym_keep");
    uint64_t nnz = scan_flags(keep2.p, pos2.p, tot, s);
    out.row.alloc(nnz, s); out.col.alloc(nnz, s); out.val.alloc(nnz, s);
    out.nnz = nnz;
    if (nnz) {
        k_sym_scatter<<<ceil_div(tot, 256), 256, 0, s>>>(key_s.p, wsym.p, keep2.p, pos2.p, tot, n, out.row.p,
                                                         out.col.p, out.val.p);
        check_launch("k_sym_scatter");
    }
}

// ---------------------------------------------------------------- CSR

__device__ __forceinline__ uint32_t row_of(const uint64_t *__restrict__ ptr, uint32_t n, uint64_t p)
{
    // largest i with ptr[i] <= p
    uint32_t lo = 0, hi = n;  // invariant ptr[lo] <= p < ptr[hi]
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (ptr[mid] <= p) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Upper-triangle entries (i < j) become edges. A warp per segment of 32
// rows: lane l holds the first entry of row r0 + l, and each entry of the
// segment finds its row among them by a search over the lanes (the last row
// starting at or before it, as row_of; entries before ptr[0] belong to row
// 0). A column outside [0, n) is reported in *bad and its entry dropped (the
// reference indexes out of range); so are row starts out of order, with
// which the segments would not cover the entries once each.
__global__ void __launch_bounds__(256) k_upper_flags(const uint64_t *__restrict__ adj_ptr,
                                                     const uint32_t *__restrict__ adj_col, uint32_t n, uint64_t nnz,
                                                     uint32_t *__restrict__ src_row, uint32_t *__restrict__ flag,
                                                     uint32_t *__restrict__ bad)
{
    const unsigned full = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t r0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u;
    if (r0 >= n) return;  // warp-uniform
    const uint32_t rows = min(32u, n - r0);
    const uint64_t start = adj_ptr[r0 + min(lane, rows)], seg_end = adj_ptr[r0 + rows];
    const uint64_t next = __shfl_down_sync(full, start, 1);
    const uint64_t row_end = lane + 1 < rows ? next : seg_end;
    if (lane < rows && row_end < start) *bad = 1u;
    const uint64_t b = r0 == 0 ? 0 : __shfl_sync(full, start, 0), e = min(seg_end, nnz);
    for (uint64_t p0 = b; p0 < e; p0 += 32) {  // warp-uniform
        const uint64_t p = p0 + lane;
        uint32_t lo = 0;
#pragma unroll
        for (uint32_t step = 16; step > 0; step >>= 1) {
            const uint64_t s = __shfl_sync(full, start, lo + step);
            if (lo + step < rows && s <= p) lo += step;
        }
        if (p < e) {
            const uint32_t i = r0 + lo, c = adj_col[p];
            src_row[p] = i;
            if (c >= n) *bad = 1u;
            flag[p] = i < c && c < n;
        }
    }
}

__global__ void k_edges(const uint32_t *__restrict__ src_row, const uint32_t *__restrict__ adj_col,
                        const float *__restrict__ adj_w, const uint32_t *__restrict__ flag,
                        const uint32_t *__restrict__ pos, uint64_t nnz, uint32_t *__restrict__ ei,
                        uint32_t *__restrict__ ej, float *__restrict__ ew)
{
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nnz || !flag[p]) return;
    uint32_t e = pos[p];
    ei[e] = src_row[p];
    ej[e] = adj_col[p];
    ew[e] = adj_w[p];
}

// umap_optimiser_gpu.rs:186-196: period = 1 / (w / max_w), 1e8 when the
// normalised weight is not positive. Endpoint records (node, 2e + side).
// node_job (several graphs in one build): the maximum is the edge's own
// graph's, d_max indexed by graph.
__global__ void k_edge_records(const uint32_t *__restrict__ ei, const uint32_t *__restrict__ ej,
                               const float *__restrict__ ew, uint64_t E, const float *__restrict__ d_max,
                               float *__restrict__ eps, uint32_t *__restrict__ key, uint32_t *__restrict__ val,
                               uint32_t *__restrict__ degree, const uint32_t *__restrict__ node_job)
{
    uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    float norm = ew[e] / d_max[node_job ? node_job[ei[e]] : 0];
    eps[e] = norm > 0.0f ? 1.0f / norm : 1e8f;
    key[2 * e] = ei[e];
    val[2 * e] = (uint32_t)(2 * e);
    key[2 * e + 1] = ej[e];
    val[2 * e + 1] = (uint32_t)(2 * e + 1);
    atomicAdd(&degree[ei[e]], 1u);
    atomicAdd(&degree[ej[e]], 1u);
}

// node_job / node_base (several graphs in one build): `other` is written as
// an index local to its graph.
__global__ void k_csr_entries(const uint32_t *__restrict__ val_s, uint64_t tot, const uint32_t *__restrict__ ei,
                              const uint32_t *__restrict__ ej, const float *__restrict__ ew,
                              const float *__restrict__ eps, uint32_t *__restrict__ other,
                              uint32_t *__restrict__ edge_id, float2 *__restrict__ sched,
                              float *__restrict__ mu_entry, const uint32_t *__restrict__ node_job,
                              const uint32_t *__restrict__ node_base)
{
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= tot + 8) return;
    if (p >= tot) {
        // padding behind the last entry, copied (never used) by 16-byte chunk copies
        sched[p] = make_float2(__int_as_float(0x7f800000), 0.0f);
        other[p] = 0;
        return;
    }
    uint32_t v = val_s[p];
    uint32_t e = v >> 1;
    uint32_t o = (v & 1) ? ei[e] : ej[e];
    other[p] = node_job ? o - node_base[node_job[o]] : o;
    edge_id[p] = e;
    float pe = eps[e];
    sched[p] = make_float2(pe, pe);
    mu_entry[p] = ew[e];
}

__global__ void k_reset_sched(float2 *__restrict__ sched, uint64_t tot)
{
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= tot) return;
    float2 s = sched[p];
    sched[p] = make_float2(s.y, s.y);
}

void reset_schedule_dev(DeviceCsr &csr, cudaStream_t s)
{
    uint64_t tot = 2 * csr.n_edges;
    if (!tot) return;
    k_reset_sched<<<ceil_div(tot, 256), 256, 0, s>>>(csr.sched.p, tot);
    check_launch("k_reset_sched");
}

// One graph's CSR in two phases, so that the structure can be built while
// the weights are still on their way to the device.
//
// Structure (row pointers and columns): flags of the i < j entries, their
// scan, the edges' endpoints and adjacency positions, the endpoint records
// (node, 2e + side) stably sorted by node -- each node's entries in
// ascending edge index, as from_graph lists them -- the offsets, and per
// entry its other endpoint and edge.
__global__ void k_edges_struct(const uint32_t *__restrict__ src_row, const uint32_t *__restrict__ adj_col,
                               const uint32_t *__restrict__ flag, const uint32_t *__restrict__ pos, uint64_t nnz,
                               uint32_t *__restrict__ ei, uint32_t *__restrict__ ej, uint32_t *__restrict__ epos)
{
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nnz || !flag[p]) return;
    const uint32_t e = pos[p];
    ei[e] = src_row[p];
    ej[e] = adj_col[p];
    epos[e] = (uint32_t)p;
}

__global__ void k_edge_keys(const uint32_t *__restrict__ ei, const uint32_t *__restrict__ ej, uint64_t E,
                            uint32_t *__restrict__ key, uint32_t *__restrict__ val, uint32_t *__restrict__ degree)
{
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const uint32_t a = ei[e], b = ej[e];
    key[2 * e] = a;
    val[2 * e] = (uint32_t)(2 * e);
    key[2 * e + 1] = b;
    val[2 * e + 1] = (uint32_t)(2 * e + 1);
    atomicAdd(&degree[a], 1u);
    atomicAdd(&degree[b], 1u);
}

__global__ void k_csr_struct(const uint32_t *__restrict__ val_s, uint64_t tot, const uint32_t *__restrict__ ei,
                             const uint32_t *__restrict__ ej, uint32_t *__restrict__ other,
                             uint32_t *__restrict__ edge_id)
{
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= tot + 8) return;
    if (p >= tot) {
        other[p] = 0;  // padding behind the last entry, copied (never used) by 16-byte chunk copies
        return;
    }
    const uint32_t v = val_s[p], e = v >> 1;
    other[p] = (v & 1) ? ei[e] : ej[e];
    edge_id[p] = e;
}

// Weights: each edge's weight from its upper entry (mu), the largest from 0
// (umap_optimiser_gpu.rs:180-184), the periods (:186-196: 1 / (w / max_w),
// 1e8 when the normalised weight is not positive), and per entry its
// schedule (cursor = period) and weight, read from one packed (period,
// weight) pair per edge.
__global__ void k_edge_weight(const uint32_t *__restrict__ epos, const float *__restrict__ adj_w, uint64_t E,
                              float *__restrict__ mu)
{
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < E) mu[e] = adj_w[epos[e]];
}

__global__ void k_edge_period(const float *__restrict__ mu, uint64_t E, const float *__restrict__ d_max,
                              float *__restrict__ eps, float2 *__restrict__ pw)
{
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const float w = mu[e], norm = w / d_max[0];
    const float per = norm > 0.0f ? 1.0f / norm : 1e8f;
    eps[e] = per;
    pw[e] = make_float2(per, w);
}

__global__ void k_csr_weights(const uint32_t *__restrict__ edge_id, uint64_t tot, const float2 *__restrict__ pw,
                              float2 *__restrict__ sched, float *__restrict__ mu_entry)
{
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= tot + 8) return;
    if (p >= tot) {
        sched[p] = make_float2(__int_as_float(0x7f800000), 0.0f);  // padding, never active
        return;
    }
    const float2 q = pw[edge_id[p]];
    sched[p] = make_float2(q.x, q.x);
    mu_entry[p] = q.y;
}

umapcu_status build_csr_structure(uint32_t n, const uint64_t *d_adj_ptr, const uint32_t *d_adj_col, uint64_t nnz,
                                  DeviceCsr &csr, CsrBuild &tmp, cudaStream_t s)
{
    if (n == 0) return UMAPCU_NO_DATA;
    if (nnz >= (1ull << 31)) fail(UMAPCU_BAD_ARG, "graph too large for 32-bit CSR entries");
    csr.n = n;
    DevBuf<uint32_t> src_row(nnz, s), flag(nnz, s), pos(nnz, s), bad(1, s);
    check_cuda(cudaMemsetAsync(bad.p, 0, sizeof(uint32_t), s), "memset");
    if (nnz) {
        k_upper_flags<<<ceil_div(n, 256), 256, 0, s>>>(d_adj_ptr, d_adj_col, n, nnz, src_row.p, flag.p, bad.p);
        check_launch("k_upper_flags");
    }
    uint32_t bad_h = 0;
    const uint64_t E = scan_flags(flag.p, pos.p, nnz, s, bad.p, &bad_h);
    if (bad_h) return UMAPCU_BAD_ARG;
    if (E == 0) return UMAPCU_NO_GRAPH_EDGES;
    csr.n_edges = E;
    DevBuf<uint32_t> ei(E, s), ej(E, s);
    tmp.epos.alloc(E, s);
    k_edges_struct<<<ceil_div(nnz, 256), 256, 0, s>>>(src_row.p, d_adj_col, flag.p, pos.p, nnz, ei.p, ej.p,
                                                      tmp.epos.p);
    check_launch("k_edges_struct");
    src_row.release(); flag.release(); pos.release();
    const uint64_t tot = 2 * E;
    DevBuf<uint32_t> key(tot, s), val(tot, s), key_s(tot, s), val_s(tot, s), degree(n + 1, s);
    check_cuda(cudaMemsetAsync(degree.p, 0, sizeof(uint32_t) * (n + 1), s), "memset");
    k_edge_keys<<<ceil_div(E, 256), 256, 0, s>>>(ei.p, ej.p, E, key.p, val.p, degree.p);
    check_launch("k_edge_keys");
    const int end_bit = bits_for(n);
    size_t tb = 0;
    check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.p, key_s.p, val.p, val_s.p, (int64_t)tot, 0,
                                               end_bit, s), "sort size");
    {
        DevBuf<char> t(tb ? tb : 1, s);
        check_cuda(cub::DeviceRadixSort::SortPairs(t.p, tb, key.p, key_s.p, val.p, val_s.p, (int64_t)tot, 0,
                                                   end_bit, s), "sort");
    }
    key.release(); val.release(); key_s.release();
    csr.offsets.alloc(n + 1, s);
    {
        size_t tb2 = 0;
        check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, tb2, degree.p, csr.offsets.p, (int64_t)(n + 1), s),
                   "scan size");
        DevBuf<char> t(tb2 ? tb2 : 1, s);
        check_cuda(cub::DeviceScan::ExclusiveSum(t.p, tb2, degree.p, csr.offsets.p, (int64_t)(n + 1), s), "scan");
    }
    csr.other.alloc(tot + 8, s);
    csr.edge_id.alloc(tot, s);
    k_csr_struct<<<ceil_div(tot + 8, 256), 256, 0, s>>>(val_s.p, tot, ei.p, ej.p, csr.other.p, csr.edge_id.p);
    check_launch("k_csr_struct");
    return UMAPCU_OK;
}

void build_csr_weights(const float *d_adj_w, DeviceCsr &csr, CsrBuild &tmp, cudaStream_t s)
{
    const uint64_t E = csr.n_edges, tot = 2 * E;
    csr.mu.alloc(E, s);
    csr.eps.alloc(E, s);
    csr.sched.alloc(tot + 8, s);
    csr.mu_entry.alloc(tot, s);
    k_edge_weight<<<ceil_div(E, 256), 256, 0, s>>>(tmp.epos.p, d_adj_w, E, csr.mu.p);
    check_launch("k_edge_weight");
    tmp.epos.release();
    DevBuf<float> dmax(1, s);
    reduce_max0(csr.mu.p, E, dmax.p, s);
    DevBuf<float2> pw(E, s);
    k_edge_period<<<ceil_div(E, 256), 256, 0, s>>>(csr.mu.p, E, dmax.p, csr.eps.p, pw.p);
    check_launch("k_edge_period");
    k_csr_weights<<<ceil_div(tot + 8, 256), 256, 0, s>>>(csr.edge_id.p, tot, pw.p, csr.sched.p, csr.mu_entry.p);
    check_launch("k_csr_weights");
}

umapcu_status build_csr_dev(uint32_t n, const uint64_t *d_adj_ptr, const uint32_t *d_adj_col,
                            const float *d_adj_w, uint64_t nnz, DeviceCsr &csr, cudaStream_t s)
{
    CsrBuild tmp;
    const umapcu_status rc = build_csr_structure(n, d_adj_ptr, d_adj_col, nnz, csr, tmp, s);
    if (rc != UMAPCU_OK) return rc;
    build_csr_weights(d_adj_w, csr, tmp, s);
    return UMAPCU_OK;
}

// ---------------------------------------------- several graphs, one build

__global__ void k_node_job(const uint32_t *__restrict__ node_base, uint32_t n_jobs, uint32_t n_total,
                           uint32_t *__restrict__ node_job)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_total) return;
    uint32_t lo = 0, hi = n_jobs;  // largest t with node_base[t] <= i
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (node_base[mid] <= i) lo = mid;
        else hi = mid;
    }
    node_job[i] = lo;
}

// k_upper_flags over concatenated graphs: the entry's graph by its first
// entry (job_entry_base [J + 1]), its row inside the graph's own local ptr
// (graph t's ptr starts at lptr + node_base[t] + t), the row and column made
// global. Columns outside the graph are reported and dropped.
__global__ void k_upper_flags_multi(const uint64_t *__restrict__ lptr, const uint32_t *__restrict__ adj_col,
                                    const uint32_t *__restrict__ node_base, const uint64_t *__restrict__ job_entry_base,
                                    uint32_t n_jobs, uint64_t nnz, uint32_t *__restrict__ src_row,
                                    uint32_t *__restrict__ gcol, uint32_t *__restrict__ flag, uint32_t *__restrict__ bad)
{
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    uint32_t lo = 0, hi = n_jobs;  // largest t with job_entry_base[t] <= p
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (job_entry_base[mid] <= p) lo = mid;
        else hi = mid;
    }
    const uint32_t nb = node_base[lo], nj = node_base[lo + 1] - nb;
    const uint32_t il = row_of(lptr + nb + lo, nj, p - job_entry_base[lo]);
    const uint32_t c = adj_col[p];
    src_row[p] = nb + il;
    gcol[p] = nb + c;
    if (c >= nj) *bad = 1u;
    flag[p] = il < c && c < nj;
}

// Edges per job from the exclusive scan of the upper flags.
__global__ void k_job_edges(const uint32_t *__restrict__ flag, const uint32_t *__restrict__ pos, uint64_t nnz,
                            const uint64_t *__restrict__ job_entry_base, uint32_t n_jobs,
                            uint64_t *__restrict__ job_edges)
{
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > n_jobs) return;
    // edges before entry a: pos[a] (a < nnz) or the total
    const uint64_t a = job_entry_base[t];
    job_edges[t] = a < nnz ? pos[a] : (uint64_t)pos[nnz - 1] + flag[nnz - 1];
}

// Per-job maximum weight from 0 (the single build's MaxFrom0 reduction):
// non-negative floats order like their bit patterns, NaN never enters.
__global__ void k_job_max(const uint32_t *__restrict__ ei, const float *__restrict__ ew, uint64_t E,
                          const uint32_t *__restrict__ node_job, float *__restrict__ dmax)
{
    uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const float w = ew[e];
    if (w > 0.0f) atomicMax((int *)&dmax[node_job[ei[e]]], __float_as_int(w));
}

umapcu_status build_csr_multi(uint32_t n_total, uint32_t n_jobs, const uint32_t *d_node_base,
                              const uint64_t *d_job_entry_base, const uint64_t *d_lptr, const uint32_t *d_adj_col,
                              const float *d_adj_w, uint64_t nnz, DeviceCsr &csr, uint64_t *h_job_edges,
                              cudaStream_t s)
{
    if (n_total == 0 || n_jobs == 0) return UMAPCU_NO_DATA;
    if (nnz >= (1ull << 31)) fail(UMAPCU_BAD_ARG, "graphs too large for 32-bit CSR entries");
    if (nnz == 0) return UMAPCU_NO_GRAPH_EDGES;
    csr.n = n_total;
    DevBuf<uint32_t> node_job(n_total, s);
    k_node_job<<<ceil_div(n_total, 256), 256, 0, s>>>(d_node_base, n_jobs, n_total, node_job.p);
    check_launch("k_node_job");
    DevBuf<uint32_t> src_row(nnz, s), gcol(nnz, s), flag(nnz, s), pos(nnz, s), bad(1, s);
    check_cuda(cudaMemsetAsync(bad.p, 0, sizeof(uint32_t), s), "memset");
    k_upper_flags_multi<<<ceil_div(nnz, 256), 256, 0, s>>>(d_lptr, d_adj_col, d_node_base, d_job_entry_base, n_jobs,
                                                           nnz, src_row.p, gcol.p, flag.p, bad.p);
    check_launch("k_upper_flags_multi");
    {
        size_t tb = 0;
        check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag.p, pos.p, (int64_t)nnz, s), "scan size");
        DevBuf<char> tmp(tb ? tb : 1, s);
        check_cuda(cub::DeviceScan::ExclusiveSum(tmp.p, tb, flag.p, pos.p, (int64_t)nnz, s), "scan");
    }
    DevBuf<uint64_t> je(n_jobs + 1, s);
    k_job_edges<<<ceil_div(n_jobs + 1, 256), 256, 0, s>>>(flag.p, pos.p, nnz, d_job_entry_base, n_jobs, je.p);
    check_launch("k_job_edges");
    std::vector<uint64_t> cum(n_jobs + 1);
    uint32_t bad_h = 0;
    d2h(cum.data(), je.p, n_jobs + 1, s);
    d2h(&bad_h, bad.p, 1, s);
    sync(s);
    if (bad_h) return UMAPCU_BAD_ARG;
    for (uint32_t t = 0; t < n_jobs; t++) h_job_edges[t] = cum[t + 1] - cum[t];
    const uint64_t E = cum[n_jobs] - cum[0];
    if (E == 0) return UMAPCU_NO_GRAPH_EDGES;
    csr.n_edges = E;
    DevBuf<uint32_t> ei(E, s), ej(E, s);
    csr.mu.alloc(E, s);
    k_edges<<<ceil_div(nnz, 256), 256, 0, s>>>(src_row.p, gcol.p, d_adj_w, flag.p, pos.p, nnz, ei.p, ej.p, csr.mu.p);
    check_launch("k_edges");
    src_row.release(); gcol.release(); flag.release(); pos.release();
    DevBuf<float> dmax(n_jobs, s);
    check_cuda(cudaMemsetAsync(dmax.p, 0, sizeof(float) * n_jobs, s), "memset");
    k_job_max<<<ceil_div(E, 256), 256, 0, s>>>(ei.p, csr.mu.p, E, node_job.p, dmax.p);
    check_launch("k_job_max");
    const uint64_t tot = 2 * E;
    csr.eps.alloc(E, s);
    DevBuf<uint32_t> key(tot, s), val(tot, s), key_s(tot, s), val_s(tot, s), degree(n_total + 1, s);
    check_cuda(cudaMemsetAsync(degree.p, 0, sizeof(uint32_t) * (n_total + 1), s), "memset");
    k_edge_records<<<ceil_div(E, 256), 256, 0, s>>>(ei.p, ej.p, csr.mu.p, E, dmax.p, csr.eps.p, key.p, val.p,
                                                    degree.p, node_job.p);
    check_launch("k_edge_records");
    const int end_bit = bits_for(n_total);
    {
        size_t tb = 0;
        check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.p, key_s.p, val.p, val_s.p, (int64_t)tot, 0,
                                                   end_bit, s), "sort size");
        DevBuf<char> tmp(tb ? tb : 1, s);
        check_cuda(cub::DeviceRadixSort::SortPairs(tmp.p, tb, key.p, key_s.p, val.p, val_s.p, (int64_t)tot, 0,
                                                   end_bit, s), "sort");
    }
    csr.offsets.alloc(n_total + 1, s);
    {
        size_t tb2 = 0;
        check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, tb2, degree.p, csr.offsets.p, (int64_t)(n_total + 1), s),
                   "scan size");
        DevBuf<char> tmp(tb2 ? tb2 : 1, s);
        check_cuda(cub::DeviceScan::ExclusiveSum(tmp.p, tb2, degree.p, csr.offsets.p, (int64_t)(n_total + 1), s),
                   "scan");
    }
    csr.other.alloc(tot + 8, s);
    csr.edge_id.alloc(tot, s);
    csr.sched.alloc(tot + 8, s);
    csr.mu_entry.alloc(tot, s);
    k_csr_entries<<<ceil_div(tot + 8, 256), 256, 0, s>>>(val_s.p, tot, ei.p, ej.p, csr.mu.p, csr.eps.p, csr.other.p,
                                                         csr.edge_id.p, csr.sched.p, csr.mu_entry.p, node_job.p,
                                                         d_node_base);
    check_launch("k_csr_entries");
    return UMAPCU_OK;
}

// ------------------------------------------------------- densMAP state

// density.rs:286-334: squared high-dimensional distance per COO entry.
__global__ void k_edge_dsq(const uint32_t *__restrict__ row, const uint32_t *__restrict__ col, uint64_t nnz,
                           const int32_t *__restrict__ idx, const float *__restrict__ dist, uint32_t k,
                           int distances_squared, float *__restrict__ out)
{
    uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    uint32_t i = row[e], j = col[e];
    float raw = 0.0f;
    bool found = false;
    for (uint32_t t = 0; t < k && !found; t++)
        if ((uint32_t)idx[(uint64_t)i * k + t] == j) { raw = dist[(uint64_t)i * k + t]; found = true; }
    for (uint32_t t = 0; t < k && !found; t++)
        if ((uint32_t)idx[(uint64_t)j * k + t] == i) { raw = dist[(uint64_t)j * k + t]; found = true; }
    out[e] = distances_squared ? raw : raw * raw;
}

// density.rs:358-398: per-node f64 sums in COO order (rows are contiguous
// and ascending), then the log radius.
__global__ void k_orig_radii(const uint32_t *__restrict__ row, const float *__restrict__ val,
                             const float *__restrict__ dsq, uint64_t nnz, uint32_t n, double *__restrict__ ro,
                             double *__restrict__ ms)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t lo = 0, hi = nnz;  // first entry with row >= i
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if (row[mid] < i) lo = mid + 1;
        else hi = mid;
    }
    double a = 0.0, b = 0.0;
    for (uint64_t e = lo; e < nnz && row[e] == i; e++) {
        double mu = (double)val[e];
        a += mu * (double)dsq[e];
        b += mu;
    }
    ms[i] = b;
    double denom = fmax(b, DBL_EPSILON);
    ro[i] = log(1e-8 + a / denom);
}

// Deterministic single-block f64 reductions (fixed thread count and order).
template <int MODE>
__global__ void k_block_sum(const double *__restrict__ x, const float *__restrict__ xf, uint64_t n,
                            const double *__restrict__ mean_in, double *__restrict__ out)
{
    __shared__ double sh[1024];
    double acc = 0.0;
    double mean = MODE == 1 ? *mean_in : 0.0;
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
        if (MODE == 0) acc += x[i];
        else if (MODE == 1) { double d = x[i] - mean; acc += d * d; }
        else acc += (double)xf[i];
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = MODE == 0 ? sh[0] / (double)n : (MODE == 1 ? sh[0] : sh[0]);
}

__global__ void k_standardise(const double *__restrict__ ro, const double *__restrict__ ms, uint32_t n,
                              const double *__restrict__ mean, const double *__restrict__ ss,
                              float *__restrict__ r, float *__restrict__ mu_sum)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double sd = sqrt(*ss / (double)(n - 1));
    r[i] = (float)((ro[i] - *mean) / sd);
    mu_sum[i] = (float)ms[i];
}

umapcu_status dens_state_dev(uint32_t n, uint64_t nnz, const uint32_t *d_row, const uint32_t *d_col,
                             const float *d_val, const int32_t *d_idx, const float *d_dist, uint32_t k,
                             int distances_squared, float *d_r, float *d_mu_sum, float *h_mu_tot, cudaStream_t s)
{
    if (n == 0) return UMAPCU_NO_DATA;
    if (n < 2) return UMAPCU_DEGENERATE_LOCAL_RADII;
    DevBuf<float> dsq(nnz, s);
    if (nnz) {
        k_edge_dsq<<<ceil_div(nnz, 256), 256, 0, s>>>(d_row, d_col, nnz, d_idx, d_dist, k, distances_squared, dsq.p);
        check_launch("k_edge_dsq");
    }
    DevBuf<double> ro(n, s), ms(n, s), scal(3, s);
    k_orig_radii<<<ceil_div(n, 256), 256, 0, s>>>(d_row, d_val, dsq.p, nnz, n, ro.p, ms.p);
    check_launch("k_orig_radii");
    k_block_sum<0><<<1, 1024, 0, s>>>(ro.p, nullptr, n, nullptr, scal.p);
    k_block_sum<1><<<1, 1024, 0, s>>>(ro.p, nullptr, n, scal.p, scal.p + 1);
    check_launch("k_block_sum");
    double h[2];
    d2h(h, scal.p, 2, s);
    sync(s);
    double sd = sqrt(h[1] / (double)(n - 1));
    if (std::isnan(sd) || sd <= DBL_EPSILON) return UMAPCU_DEGENERATE_LOCAL_RADII;
    k_standardise<<<ceil_div(n, 256), 256, 0, s>>>(ro.p, ms.p, n, scal.p, scal.p + 1, d_r, d_mu_sum);
    check_launch("k_standardise");
    k_block_sum<2><<<1, 1024, 0, s>>>(nullptr, d_mu_sum, n, nullptr, scal.p + 2);
    check_launch("k_block_sum");
    double t = 0.0;
    d2h(&t, scal.p + 2, 1, s);
    sync(s);
    *h_mu_tot = (float)t;
    return UMAPCU_OK;
}

}  // namespace umapcu
