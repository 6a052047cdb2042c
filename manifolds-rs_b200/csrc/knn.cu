// Exact k-nearest neighbours and embedding-quality metrics on the device.
//
// The reference delegates kNN to ann-search-rs 0.5.2 (run_ann_search,
// src/data/nearest_neighbours.rs:225-364; AnnSearch::Exhaustive queries k+1
// and drops the first, i.e. self) and takes the neighbours' squared Euclidean
// distances as they come (src/lib.rs:435). It has no quality metrics. Here:
//
//  * k_knn_tile<EUC, EPI>: a CTA owns 64 queries and streams every point in
//    tiles of 128, the coordinates staged 16 dimensions at a time through
//    shared memory by cp.async (double-buffered). Warp w computes queries
//    8w..8w+7 against the tile, lane l points 4l..4l+3: 32 distances per
//    thread, each a sequential FMA chain over the dimensions in order
//    (d += (q-p)^2, or d += q*p for cosine), so every distance equals the
//    one-line C loop with fmaf bit for bit. The warp then folds its
//    distances into per-query state held in registers:
//      EPI_TOPK: the k best (distance, index) pairs, one per lane, kept
//        sorted by warp ballots (ties broken by the smaller index, self
//        excluded) -- the exact kNN, unique under that total order;
//      EPI_RANK: per lane m < k, the number of points strictly better than
//        threshold m -- the ranks trustworthiness needs.
//    Few queries (the metrics' subsample) split the point range into slices
//    (partial lists merged by k_knn_merge, rank counts added atomically).
//  * trustworthiness (sklearn.manifold.trustworthiness's definition) over a
//    query subsample, kNN preservation, fuzzy cross-entropy (f64).
//
// This is CUDA-core (FP32 FMA) work on purpose: the tensor-core expansion
// |q|^2 + |p|^2 - 2 q.p changes distances in their last bits and with them
// near-tied neighbour sets; the exact path stays bit-reproducible.
#include <cfloat>

#include "internal.cuh"

namespace umapcu {
namespace {

constexpr int kQT = 64;       // queries per CTA
constexpr int kPT = 128;      // points per tile
constexpr int kDC = 16;       // dimensions per staged chunk
constexpr int kThreads = 256;
constexpr int kQS = kQT + 4;  // shared-memory row strides (16-byte aligned rows)
constexpr int kPS = kPT + 4;
constexpr uint32_t kMaxK = 32;
constexpr unsigned kFull = 0xffffffffu;

enum { EPI_TOPK = 0, EPI_RANK = 1 };

struct __align__(16) TileSmem {
    float q[2][kDC][kQS];
    float p[2][kDC][kPS];
    uint32_t qrow[kQT];
};

__device__ __forceinline__ void cp_async4(float *smem, const float *gmem, bool ok)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(ok ? 4 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// (d, i) strictly before (td, ti): smaller distance, ties by smaller index.
__device__ __forceinline__ bool better(float d, uint32_t i, float td, uint32_t ti)
{
    return d < td || (d == td && i < ti);
}

struct TileArgs {
    const float *x;          // [n, dim] points (cosine: unit rows)
    uint32_t n, dim, k;
    const uint32_t *qidx;    // [nq] query rows, nullptr: query q is row q
    uint32_t nq;
    uint32_t tiles_per_slice;
    // EPI_TOPK
    uint32_t *out_idx;       // [slices][nq][k]
    float *out_dist;
    // EPI_RANK
    const float *thr_d;      // [nq][k]
    const uint32_t *thr_j;   // [nq][k]
    uint32_t *counts;        // [nq][k], added to
};

// Sorted insertion of (cd, ci) into the warp's list (lane l holds entry l,
// lanes >= k hold (+inf, ~0)).
__device__ __forceinline__ void list_insert(float &ld, uint32_t &li, float cd, uint32_t ci, uint32_t k,
                                            uint32_t lane)
{
    const int pos = __popc(__ballot_sync(kFull, better(ld, li, cd, ci)));
    const float ud = __shfl_up_sync(kFull, ld, 1);
    const uint32_t ui = __shfl_up_sync(kFull, li, 1);
    if (lane < k) {
        if ((int)lane > pos) {
            ld = ud;
            li = ui;
        } else if ((int)lane == pos) {
            ld = cd;
            li = ci;
        }
    }
}

// Offers the lane's pending candidates (bit j of pend: cand_d[j], cand_i[j])
// to the list, best-first across lanes is not needed: every candidate better
// than the current k-th is inserted, the threshold re-read after each.
template <int NC>
__device__ __forceinline__ void list_offer(float &ld, uint32_t &li, const float (&cd)[NC], const uint32_t (&ci)[NC],
                                           unsigned pend, uint32_t k, uint32_t lane)
{
    for (;;) {
        const unsigned m = __ballot_sync(kFull, pend != 0);
        if (!m) break;
        const int src = __ffs(m) - 1;
        float myd = 0.0f;
        uint32_t myi = 0;
        bool found = false;
#pragma unroll
        for (int j = 0; j < NC; j++)
            if (!found && ((pend >> j) & 1u)) {
                myd = cd[j];
                myi = ci[j];
                found = true;
            }
        const float d = __shfl_sync(kFull, myd, src);
        const uint32_t i = __shfl_sync(kFull, myi, src);
        if ((int)lane == src) pend &= pend - 1;
        list_insert(ld, li, d, i, k, lane);
        const float td = __shfl_sync(kFull, ld, k - 1);
        const uint32_t ti = __shfl_sync(kFull, li, k - 1);
#pragma unroll
        for (int j = 0; j < NC; j++)
            if (((pend >> j) & 1u) && !better(cd[j], ci[j], td, ti)) pend &= ~(1u << j);
    }
}

template <bool EUC, int EPI>
__global__ void __launch_bounds__(kThreads, 2) k_knn_tile(const TileArgs A)
{
    __shared__ TileSmem S;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t q0 = blockIdx.x * kQT;
    const uint32_t slice = blockIdx.y;
    const uint32_t n_tiles = (A.n + kPT - 1) / kPT;
    const uint32_t t_beg = slice * A.tiles_per_slice;
    const uint32_t t_end = min(n_tiles, t_beg + A.tiles_per_slice);
    const uint32_t n_chunks = (A.dim + kDC - 1) / kDC;
    if (tid < kQT) {
        const uint32_t q = q0 + tid;
        S.qrow[tid] = q < A.nq ? (A.qidx ? A.qidx[q] : q) : 0u;
    }
    __syncthreads();

    // per-query state of this warp's 8 queries
    float ld[8];
    uint32_t li[8];
    uint32_t cnt[8];
    float td[8];
    uint32_t tj[8];
    uint32_t gq[8];
    bool qok[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const uint32_t ql = warp * 8 + i;
        qok[i] = q0 + ql < A.nq;
        gq[i] = S.qrow[ql];
        ld[i] = __int_as_float(0x7f800000);
        li[i] = ~0u;
        cnt[i] = 0;
        td[i] = 0.0f;
        tj[i] = 0;
        if (EPI == EPI_RANK && qok[i] && lane < A.k) {
            td[i] = A.thr_d[(size_t)(q0 + ql) * A.k + lane];
            tj[i] = A.thr_j[(size_t)(q0 + ql) * A.k + lane];
        }
    }

    auto stage = [&](uint32_t it, int b) {
        const uint32_t t = t_beg + it / n_chunks, c = it % n_chunks;
        const uint32_t p0 = t * kPT, d0 = c * kDC;
        for (uint32_t e = tid; e < kPT * kDC; e += kThreads) {
            const uint32_t r = e / kDC, dd = e % kDC, gp = p0 + r, gd = d0 + dd;
            const bool ok = gp < A.n && gd < A.dim;
            cp_async4(&S.p[b][dd][r], ok ? A.x + (size_t)gp * A.dim + gd : A.x, ok);
        }
        for (uint32_t e = tid; e < kQT * kDC; e += kThreads) {
            const uint32_t r = e / kDC, dd = e % kDC, gd = d0 + dd;
            const bool ok = q0 + r < A.nq && gd < A.dim;
            cp_async4(&S.q[b][dd][r], ok ? A.x + (size_t)S.qrow[r] * A.dim + gd : A.x, ok);
        }
        cp_async_commit();
    };

    const uint32_t n_it = (t_end > t_beg ? t_end - t_beg : 0) * n_chunks;
    float acc[8][4];
    if (n_it) stage(0, 0);
    for (uint32_t it = 0; it < n_it; it++) {
        const uint32_t c = it % n_chunks;
        const int b = it & 1;
        if (c == 0) {
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = 0.0f;
        }
        if (it + 1 < n_it) {
            stage(it + 1, b ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int dd = 0; dd < kDC; dd++) {
            const float4 qa = *reinterpret_cast<const float4 *>(&S.q[b][dd][warp * 8]);
            const float4 qb = *reinterpret_cast<const float4 *>(&S.q[b][dd][warp * 8 + 4]);
            const float4 pv = *reinterpret_cast<const float4 *>(&S.p[b][dd][lane * 4]);
            const float qv[8] = {qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z, qb.w};
            const float pp[4] = {pv.x, pv.y, pv.z, pv.w};
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    if (EUC) {
                        const float df = qv[i] - pp[j];
                        acc[i][j] = __fmaf_rn(df, df, acc[i][j]);
                    } else {
                        acc[i][j] = __fmaf_rn(qv[i], pp[j], acc[i][j]);
                    }
                }
        }
        __syncthreads();  // buffer b is restaged two iterations on
        if (c + 1 != n_chunks) continue;

        // ---- epilogue of one point tile
        const uint32_t p0 = (t_beg + it / n_chunks) * kPT;
        uint32_t pidx[4];
#pragma unroll
        for (int j = 0; j < 4; j++) pidx[j] = p0 + lane * 4 + j;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            if (!qok[i]) continue;  // warp-uniform
            float dv[4];
#pragma unroll
            for (int j = 0; j < 4; j++) dv[j] = EUC ? acc[i][j] : 1.0f - acc[i][j];
            if (EPI == EPI_TOPK) {
                const float thd = __shfl_sync(kFull, ld[i], A.k - 1);
                const uint32_t thi = __shfl_sync(kFull, li[i], A.k - 1);
                unsigned pend = 0;
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (pidx[j] < A.n && pidx[j] != gq[i] && better(dv[j], pidx[j], thd, thi)) pend |= 1u << j;
                list_offer<4>(ld[i], li[i], dv, pidx, pend, A.k, lane);
            } else {
                uint32_t c_i = 0;
                for (int src = 0; src < 32; src++) {
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const float d = __shfl_sync(kFull, dv[j], src);
                        const uint32_t p = p0 + src * 4 + j;
                        c_i += (p < A.n && p != gq[i] && better(d, p, td[i], tj[i])) ? 1u : 0u;
                    }
                }
                cnt[i] += c_i;
            }
        }
    }

#pragma unroll
    for (int i = 0; i < 8; i++) {
        if (!qok[i] || lane >= A.k) continue;
        const size_t q = q0 + warp * 8 + i;
        if (EPI == EPI_TOPK) {
            const size_t o = ((size_t)slice * A.nq + q) * A.k + lane;
            A.out_idx[o] = li[i];
            A.out_dist[o] = ld[i];
        } else if (cnt[i]) {
            atomicAdd(&A.counts[q * A.k + lane], cnt[i]);
        }
    }
}

// Merges the slices' partial lists: one warp per query.
__global__ void k_knn_merge(const uint32_t *__restrict__ pidx, const float *__restrict__ pdist, uint32_t slices,
                            uint32_t nq, uint32_t k, uint32_t *__restrict__ out_idx, float *__restrict__ out_dist)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (q >= nq) return;  // warp-uniform
    float ld = __int_as_float(0x7f800000);
    uint32_t li = ~0u;
    for (uint32_t s = 0; s < slices; s++) {
        const size_t o = ((size_t)s * nq + q) * k + lane;
        float cd[1] = {lane < k ? pdist[o] : __int_as_float(0x7f800000)};
        uint32_t ci[1] = {lane < k ? pidx[o] : ~0u};
        const float td = __shfl_sync(kFull, ld, k - 1);
        const uint32_t ti = __shfl_sync(kFull, li, k - 1);
        const unsigned pend = (lane < k && ci[0] != ~0u && better(cd[0], ci[0], td, ti)) ? 1u : 0u;
        list_offer<1>(ld, li, cd, ci, pend, k, lane);
    }
    if (lane < k) {
        out_idx[(size_t)q * k + lane] = li;
        out_dist[(size_t)q * k + lane] = ld;
    }
}

// Unit rows for the cosine metric: x / sqrt(sum x^2) (sequential FMA chain,
// IEEE sqrt and division); zero rows stay zero.
__global__ void k_unit_rows(const float *__restrict__ x, uint32_t n, uint32_t dim, float *__restrict__ xn)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *r = x + (size_t)i * dim;
    float s = 0.0f;
    for (uint32_t d = 0; d < dim; d++) s = __fmaf_rn(r[d], r[d], s);
    const float nrm = sqrtf(s);
    for (uint32_t d = 0; d < dim; d++) xn[(size_t)i * dim + d] = nrm > 0.0f ? r[d] / nrm : 0.0f;
}

// The distance of each query to each of its given neighbours, by the same
// chain as k_knn_tile (so a neighbour's own threshold compares equal).
template <bool EUC>
__global__ void k_pair_dist(const float *__restrict__ x, uint32_t dim, const uint32_t *__restrict__ qidx,
                            uint32_t nq, const uint32_t *__restrict__ nbr, uint32_t k, float *__restrict__ out)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint64_t)nq * k) return;
    const uint32_t q = (uint32_t)(t / k);
    const float *a = x + (size_t)(qidx ? qidx[q] : q) * dim;
    const float *b = x + (size_t)nbr[t] * dim;
    float s = 0.0f;
    for (uint32_t d = 0; d < dim; d++) {
        if (EUC) {
            const float df = a[d] - b[d];
            s = __fmaf_rn(df, df, s);
        } else {
            s = __fmaf_rn(a[d], b[d], s);
        }
    }
    out[t] = EUC ? s : 1.0f - s;
}

// |kNN_X(i)[:k] & kNN_Y(i)| per query, summed: one warp per query.
__global__ void k_knn_overlap(const int32_t *__restrict__ knn_x, uint32_t kx, const uint32_t *__restrict__ qidx,
                              uint32_t nq, const uint32_t *__restrict__ knn_y, uint32_t k,
                              unsigned long long *__restrict__ total)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (q >= nq) return;
    const uint32_t row = qidx ? qidx[q] : q;
    const int32_t mine = lane < k ? (int32_t)knn_y[(size_t)q * k + lane] : -1;
    uint32_t hits = 0;
    for (uint32_t m = 0; m < k; m++) {
        const int32_t xm = knn_x[(size_t)row * kx + m];
        hits += __ballot_sync(kFull, lane < k && mine == xm) ? 1u : 0u;
    }
    if (lane == 0) atomicAdd(total, (unsigned long long)hits);
}

// Fuzzy cross-entropy terms per edge (f64), summed per block in a fixed
// order; the host adds the block sums in order.
__global__ void k_fuzzy_ce(const uint32_t *__restrict__ row, const uint32_t *__restrict__ col,
                           const float *__restrict__ w, uint64_t nnz, const float *__restrict__ y, uint32_t dim,
                           double a, double b, double *__restrict__ block_sum)
{
    __shared__ double part[256];
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double term = 0.0;
    if (e < nnz) {
        double d2 = 0.0;
        for (uint32_t d = 0; d < dim; d++) {
            const double df = (double)y[(size_t)row[e] * dim + d] - (double)y[(size_t)col[e] * dim + d];
            d2 += df * df;
        }
        double q = 1.0 / (1.0 + a * pow(d2, b));
        q = fmin(fmax(q, 1e-12), 1.0 - 1e-12);
        const double ww = fmin(fmax((double)w[e], 1e-12), 1.0 - 1e-12);
        term = ww * log(ww / q) + (1.0 - ww) * log((1.0 - ww) / (1.0 - q));
    }
    part[threadIdx.x] = term;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) block_sum[blockIdx.x] = part[0];
}

// Point-range slices so that few queries still fill the device.
uint32_t slices_for(uint32_t nq, uint32_t n)
{
    const uint32_t qtiles = ceil_div(nq, kQT), n_tiles = ceil_div(n, kPT);
    const uint32_t want = 2u * 2u * (uint32_t)device_sm_count();
    uint32_t s = qtiles >= want ? 1u : ceil_div(want, qtiles);
    return std::max(1u, std::min({s, n_tiles, 256u}));
}

}  // namespace

void knn_dev(const float *d_x, uint32_t n, uint32_t dim, const uint32_t *d_qidx, uint32_t nq, uint32_t k,
             uint32_t metric, uint32_t *d_idx, float *d_dist, cudaStream_t s)
{
    if (k == 0 || k > kMaxK || n <= k || dim == 0) fail(UMAPCU_BAD_ARG, "knn: need 0 < k <= 32 and n > k");
    if (metric > UMAPCU_METRIC_COSINE) fail(UMAPCU_BAD_ARG, "knn: metric");
    if (nq == 0) return;
    DevBuf<float> xn;
    const float *x = d_x;
    if (metric == UMAPCU_METRIC_COSINE) {
        xn.alloc((size_t)n * dim, s);
        k_unit_rows<<<ceil_div(n, 256), 256, 0, s>>>(d_x, n, dim, xn.p);
        check_launch("k_unit_rows");
        x = xn.p;
    }
    const uint32_t S = slices_for(nq, n), n_tiles = ceil_div(n, kPT);
    TileArgs A{};
    A.x = x;
    A.n = n;
    A.dim = dim;
    A.k = k;
    A.qidx = d_qidx;
    A.nq = nq;
    A.tiles_per_slice = ceil_div(n_tiles, S);
    const uint32_t S_eff = ceil_div(n_tiles, A.tiles_per_slice);
    DevBuf<uint32_t> pidx;
    DevBuf<float> pdist;
    if (S_eff > 1) {
        pidx.alloc((size_t)S_eff * nq * k, s);
        pdist.alloc((size_t)S_eff * nq * k, s);
        A.out_idx = pidx.p;
        A.out_dist = pdist.p;
    } else {
        A.out_idx = d_idx;
        A.out_dist = d_dist;
    }
    const dim3 grid(ceil_div(nq, kQT), S_eff);
    if (metric == UMAPCU_METRIC_EUCLIDEAN_SQ) k_knn_tile<true, EPI_TOPK><<<grid, kThreads, 0, s>>>(A);
    else k_knn_tile<false, EPI_TOPK><<<grid, kThreads, 0, s>>>(A);
    check_launch("k_knn_tile");
    if (S_eff > 1) {
        k_knn_merge<<<ceil_div((uint64_t)nq * 32, 256), 256, 0, s>>>(pidx.p, pdist.p, S_eff, nq, k, d_idx, d_dist);
        check_launch("k_knn_merge");
    }
}

// counts[q][m] = #points strictly better than (distance to nbr[q][m],
// nbr[q][m]) for query q, self excluded (rank - 1 of that neighbour).
void knn_rank_dev(const float *d_x, uint32_t n, uint32_t dim, const uint32_t *d_qidx, uint32_t nq,
                  const uint32_t *d_nbr, uint32_t k, uint32_t metric, uint32_t *d_counts, cudaStream_t s)
{
    if (k == 0 || k > kMaxK || n <= k || dim == 0 || metric > UMAPCU_METRIC_COSINE) fail(UMAPCU_BAD_ARG, "rank");
    if (nq == 0) return;
    DevBuf<float> xn;
    const float *x = d_x;
    if (metric == UMAPCU_METRIC_COSINE) {
        xn.alloc((size_t)n * dim, s);
        k_unit_rows<<<ceil_div(n, 256), 256, 0, s>>>(d_x, n, dim, xn.p);
        check_launch("k_unit_rows");
        x = xn.p;
    }
    DevBuf<float> thr((size_t)nq * k, s);
    const bool euc = metric == UMAPCU_METRIC_EUCLIDEAN_SQ;
    const unsigned pg = ceil_div((uint64_t)nq * k, 256);
    if (euc) k_pair_dist<true><<<pg, 256, 0, s>>>(x, dim, d_qidx, nq, d_nbr, k, thr.p);
    else k_pair_dist<false><<<pg, 256, 0, s>>>(x, dim, d_qidx, nq, d_nbr, k, thr.p);
    check_launch("k_pair_dist");
    check_cuda(cudaMemsetAsync(d_counts, 0, sizeof(uint32_t) * nq * k, s), "memset");
    const uint32_t S = slices_for(nq, n), n_tiles = ceil_div(n, kPT);
    TileArgs A{};
    A.x = x;
    A.n = n;
    A.dim = dim;
    A.k = k;
    A.qidx = d_qidx;
    A.nq = nq;
    A.tiles_per_slice = ceil_div(n_tiles, S);
    A.thr_d = thr.p;
    A.thr_j = d_nbr;
    A.counts = d_counts;
    const dim3 grid(ceil_div(nq, kQT), ceil_div(n_tiles, A.tiles_per_slice));
    if (euc) k_knn_tile<true, EPI_RANK><<<grid, kThreads, 0, s>>>(A);
    else k_knn_tile<false, EPI_RANK><<<grid, kThreads, 0, s>>>(A);
    check_launch("k_knn_tile rank");
}

}  // namespace umapcu

using namespace umapcu;

namespace {

template <typename F>
umapcu_status guard_k(F &&f)
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

}  // namespace

extern "C" {

umapcu_status umapcu_knn_exact(const float *x, uint32_t n, uint32_t dim, uint32_t k, uint32_t metric,
                               int32_t *knn_idx, float *knn_dist)
{
    return guard_k([&]() -> umapcu_status {
        if (n == 0) return UMAPCU_NO_DATA;
        if (!x || !knn_idx || !knn_dist || dim == 0 || k == 0 || k > kMaxK || n <= k ||
            metric > UMAPCU_METRIC_COSINE)
            return UMAPCU_BAD_ARG;
        if (n >= (1u << 31)) return UMAPCU_BAD_ARG;
        keep_pool_memory();
        Stream st;
        cudaStream_t s = st.s;
        DevBuf<float> dx((size_t)n * dim, s), dd((size_t)n * k, s);
        DevBuf<uint32_t> di((size_t)n * k, s);
        h2d(dx.p, x, (size_t)n * dim, s);
        knn_dev(dx.p, n, dim, nullptr, n, k, metric, di.p, dd.p, s);
        d2h((uint32_t *)knn_idx, di.p, (size_t)n * k, s);
        d2h(knn_dist, dd.p, (size_t)n * k, s);
        sync(s);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_knn_exact_dev(const float *d_x, uint32_t n, uint32_t dim, const uint32_t *d_queries,
                                   uint32_t n_queries, uint32_t k, uint32_t metric, uint32_t *d_idx, float *d_dist,
                                   void *stream)
{
    return guard_k([&]() -> umapcu_status {
        if (n == 0) return UMAPCU_NO_DATA;
        if (!d_x || !d_idx || !d_dist || n >= (1u << 31)) return UMAPCU_BAD_ARG;
        knn_dev(d_x, n, dim, d_queries, n_queries, k, metric, d_idx, d_dist, (cudaStream_t)stream);
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_embedding_quality(const float *x, uint32_t n, uint32_t dim, const float *y, uint32_t n_dim,
                                       const int32_t *knn_idx, uint32_t knn_k, uint32_t k, const uint32_t *queries,
                                       uint32_t n_queries, uint32_t metric, double *trust, double *knn_preservation)
{
    return guard_k([&]() -> umapcu_status {
        if (n == 0) return UMAPCU_NO_DATA;
        if (!x || !y || dim == 0 || n_dim == 0 || k == 0 || k > kMaxK || metric > UMAPCU_METRIC_COSINE)
            return UMAPCU_BAD_ARG;
        if (2ull * k >= n || n >= (1u << 31)) return UMAPCU_BAD_ARG;  // sklearn: n_neighbors < n_samples / 2
        if (knn_preservation && (!knn_idx || knn_k < k)) return UMAPCU_BAD_ARG;
        const uint32_t nq = queries ? n_queries : n;
        if (nq == 0) return UMAPCU_BAD_ARG;
        if (queries)
            for (uint32_t q = 0; q < nq; q++)
                if (queries[q] >= n) return UMAPCU_BAD_ARG;
        keep_pool_memory();
        Stream st;
        cudaStream_t s = st.s;
        DevBuf<float> dx((size_t)n * dim, s), dy((size_t)n * n_dim, s), ydist((size_t)nq * k, s);
        DevBuf<uint32_t> dq(queries ? nq : 0, s), ynbr((size_t)nq * k, s), counts((size_t)nq * k, s);
        h2d(dx.p, x, (size_t)n * dim, s);
        h2d(dy.p, y, (size_t)n * n_dim, s);
        if (queries) h2d(dq.p, queries, nq, s);
        const uint32_t *qp = queries ? dq.p : nullptr;
        knn_dev(dy.p, n, n_dim, qp, nq, k, UMAPCU_METRIC_EUCLIDEAN_SQ, ynbr.p, ydist.p, s);
        if (trust) {
            knn_rank_dev(dx.p, n, dim, qp, nq, ynbr.p, k, metric, counts.p, s);
            std::vector<uint32_t> hc((size_t)nq * k);
            d2h(hc.data(), counts.p, hc.size(), s);
            sync(s);
            // sklearn.manifold.trustworthiness: ranks are 1-based positions
            // in the ordering of X-distances; penalty max(0, rank - k)
            double t = 0.0;
            for (uint32_t c : hc) t += c + 1 > k ? (double)(c + 1 - k) : 0.0;
            *trust = 1.0 - t * (2.0 / ((double)nq * k * (2.0 * n - 3.0 * k - 1.0)));
        }
        if (knn_preservation) {
            DevBuf<int32_t> dk((size_t)n * knn_k, s);
            DevBuf<unsigned long long> tot(1, s);
            h2d(dk.p, knn_idx, (size_t)n * knn_k, s);
            check_cuda(cudaMemsetAsync(tot.p, 0, sizeof(unsigned long long), s), "memset");
            k_knn_overlap<<<ceil_div((uint64_t)nq * 32, 256), 256, 0, s>>>(dk.p, knn_k, qp, nq, ynbr.p, k, tot.p);
            check_launch("k_knn_overlap");
            unsigned long long h = 0;
            d2h(&h, tot.p, 1, s);
            sync(s);
            *knn_preservation = (double)h / ((double)nq * k);
        }
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_fuzzy_cross_entropy(const uint32_t *row, const uint32_t *col, const float *w, uint64_t nnz,
                                         const float *y, uint32_t n, uint32_t n_dim, float a, float b, double *out)
{
    return guard_k([&]() -> umapcu_status {
        if (n == 0) return UMAPCU_NO_DATA;
        if (!y || !out || n_dim == 0 || (nnz && (!row || !col || !w))) return UMAPCU_BAD_ARG;
        for (uint64_t e = 0; e < nnz; e++)
            if (row[e] >= n || col[e] >= n) return UMAPCU_BAD_ARG;
        *out = 0.0;
        if (!nnz) return UMAPCU_OK;
        keep_pool_memory();
        Stream st;
        cudaStream_t s = st.s;
        DevBuf<uint32_t> dr(nnz, s), dc(nnz, s);
        DevBuf<float> dw(nnz, s), dy((size_t)n * n_dim, s);
        h2d(dr.p, row, nnz, s);
        h2d(dc.p, col, nnz, s);
        h2d(dw.p, w, nnz, s);
        h2d(dy.p, y, (size_t)n * n_dim, s);
        const unsigned blocks = ceil_div(nnz, 256);
        DevBuf<double> part(blocks, s);
        k_fuzzy_ce<<<blocks, 256, 0, s>>>(dr.p, dc.p, dw.p, nnz, dy.p, n_dim, (double)a, (double)b, part.p);
        check_launch("k_fuzzy_ce");
        std::vector<double> hp(blocks);
        d2h(hp.data(), part.p, blocks, s);
        sync(s);
        double t = 0.0;
        for (double v : hp) t += v;
        *out = t;
        return UMAPCU_OK;
    });
}

}  // extern "C"
