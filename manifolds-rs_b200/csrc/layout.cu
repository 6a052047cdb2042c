// UMAP layout epochs on the device (sm_100a): the "adam_gpu" optimiser.
//
// Reference kernels (src/training/umap_optimiser_gpu.rs):
//   umap_grad_accum      :682-860  \
//   umap_adam_update     :887-923   > fused into k_epoch
//   umap_edge_schedule_update :940-955 /
//   gpu_hash_neg         :611-624  -> sample_neg (bit-exact), or Philox4x32-10
//   umap_dens_radii      :487-544  \
//   umap_dens_weights    :568-586   > k_dens_update, one launch (radii, f64 statistics in
//   correlation_stats (density.rs:464-508) /  its last block); the weight is evaluated
//                                     inside k_epoch
//
// k_epoch: one warp owns a segment of 32 consecutive nodes and walks the CSR
// entries of those nodes (edges sorted by head vertex) in chunks of 32. Each
// entry keeps its own copy of its edge's (cursor, period) schedule, so the
// two endpoints of an edge advance identical copies without any
// cross-thread dependency. Active entries are compacted into a per-warp
// queue; every 32 queued entries form a batch in which each lane evaluates
// one entry: the attractive term, the densMAP term and neg_rate repulsive
// terms, with all row gathers of the entry (2-D coordinates as float2)
// issued before any is consumed. The entry's terms are summed in the
// reference's order into one partial; the node's own lane then adds the
// partials of its entries in CSR order. The gradient of a node is therefore
// formed without atomics and deterministically, and the node's lane applies
// the Adam (or SGD) step and writes the next embedding buffer (the embedding
// is double-buffered: every gather of an epoch reads the pre-step positions,
// as the reference's separate gradient and Adam kernels do).
//
// With the schedule precomputed (schedule.cu) the kernel either scans the
// epoch's active-entry bitmask in place of the (cursor, period) pairs (BITS),
// or reads the epoch's active-entry records without any scan (LIST). On
// small problems both give each segment a whole block (k_epoch_split_bits,
// k_epoch_split). All pick the same entries in the same order and form the
// same batches, so their results are bit-identical.
//
// Arithmetic follows the reference expression by expression with no FMA
// contraction (compiled with -fmad=false). x^b is evaluated by pow_pos
// (below) unless the state asks for CUDA's powf; logf/expf are evaluated in
// double precision and rounded.
#include <cfloat>

#include "epoch_device.cuh"

namespace umapcu {

// Resident blocks per SM the register budget is set for: 10 (48 registers,
// 40 warps) for the fast path in one or two dimensions without the density
// term, whose gathers then keep more misses in flight; 6 elsewhere, where 48
// registers would spill.
template <int D, bool DENS, bool FAST>
constexpr int epoch_min_blocks() { return FAST && !DENS && D <= 2 ? 10 : 6; }
// Entries per lane of the bitmask scan's groups: 16 in the kernels run at 10
// blocks per SM (7.3 KB of shared memory per block at 8, 11.4 KB at 16, so
// that L1 keeps ~130 KB), 32 -- a bit word per lane, the fewest groups on
// long segments -- elsewhere.
template <int D, bool DENS, bool FAST>
constexpr int bits_piece() { return FAST && !DENS && D <= 2 ? 16 : 32; }

template <int D, bool DENS, int NR, bool FAST = false, bool LIST = false, bool BITS = false>
__global__ void __launch_bounds__(kWarps * 32, epoch_min_blocks<D, DENS, FAST>()) k_epoch(const EpochArgs A)
{
    constexpr int KU = LIST ? 1 : kU;  // the list path keeps no scan queue
    __shared__ WarpSmem<D, KU, BITS, DENS, bits_piece<D, DENS, FAST>()> smem[kWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t node0 = (blockIdx.x * kWarps + warp) * 32u;
    if (node0 >= A.n) return;
    epoch_segment<D, DENS, NR, false, KU, FAST, LIST, BITS>(A, smem[warp], node0, lane);
}

// Schedule lists on a problem too small to fill the GPU with one warp per
// segment: one block (kWarps warps) per segment, see epoch_segment_split.
template <int D, bool DENS, int NR, bool FAST>
__global__ void __launch_bounds__(kWarps * 32) k_epoch_split(const EpochArgs A)
{
    __shared__ WarpSmem<D, 1, false, DENS> seg;
    __shared__ float part[kWarps][32][D];
    __shared__ unsigned has_w[kWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    epoch_segment_split<D, DENS, NR, FAST>(A, seg, part, has_w, blockIdx.x * 32u, warp, lane);
}

// The bitmask form on a small problem: one block per segment, see
// epoch_segment_split_bits.
template <int D, bool DENS, int NR, bool FAST>
__global__ void __launch_bounds__(kSplitBitsWarps * 32) k_epoch_split_bits(const EpochArgs A)
{
    __shared__ WarpSmem<D, kU, true, DENS> seg;
    __shared__ float part[kSplitBitsWarps][32][D];
    __shared__ unsigned has_w[kSplitBitsWarps];
    __shared__ uint32_t wm[kSplitWords], pre[kSplitWords + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    epoch_segment_split_bits<D, DENS, NR, FAST, kSplitBitsWarps>(A, seg, part, has_w, wm, pre, blockIdx.x * 32u, warp, lane);
}

// ------------------------------------------------------------ densMAP

constexpr int kDensBlock = 128;
// Consecutive CSR entries a lane takes per window: 8 for 1-2 dimensions, 4
// above (the coordinate gathers of a piece are held in registers together).
template <int D>
struct DensPiece {
    static constexpr int P = D <= 2 ? 8 : 4;
};

struct DensSums {
    double s_re, s_re2, s_rer, s_r;
};

__device__ __forceinline__ void dens_sums_add(DensSums &a, const DensSums &b)
{
    a.s_re += b.s_re;
    a.s_re2 += b.s_re2;
    a.s_rer += b.s_rer;
    a.s_r += b.s_r;
}

__device__ __forceinline__ DensSums dens_sums_warp(DensSums v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        v.s_re += __shfl_down_sync(kFull, v.s_re, off);
        v.s_re2 += __shfl_down_sync(kFull, v.s_re2, off);
        v.s_rer += __shfl_down_sync(kFull, v.s_rer, off);
        v.s_r += __shfl_down_sync(kFull, v.s_r, off);
    }
    return v;
}

// The `other` endpoints of CSR entries [a, a + P) into o[]: two (P = 8) or
// one (P = 4) 16-byte loads where the array is 16-byte aligned and the
// piece lies inside it, else entry by entry inside [lo, hi).
template <int P>
__device__ __forceinline__ void dens_load_piece(const uint32_t *__restrict__ other, uint64_t n_entries, bool vec,
                                                uint32_t a, uint32_t lo, uint32_t hi, uint32_t (&o)[P])
{
    if (vec && (uint64_t)a + P <= n_entries) {
#pragma unroll
        for (int h = 0; h < P / 4; h++) {
            const uint4 q = __ldcs(reinterpret_cast<const uint4 *>(other + a) + h);
            o[4 * h] = q.x;
            o[4 * h + 1] = q.y;
            o[4 * h + 2] = q.z;
            o[4 * h + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int u = 0; u < P; u++) {
            const uint32_t p = a + u;
            o[u] = (p >= lo && p < hi) ? __ldcs(other + p) : 0u;
        }
    }
}

// One densMAP update in one launch: umap_dens_radii (umap_optimiser_gpu.rs:
// 503-543) per node -- over all its CSR entries, phi = 1 / (1 + a d^2b),
// sums of phi and phi * d^2, re = log(1e-8 + sum_sq / max(sum_phi, eps)) --
// then correlation_stats (density.rs:464-508) and the weight scalars of
// launch_dens_update (umap_optimiser_gpu.rs:1123-1142) for the whole
// embedding.
// Radii: a warp per 32-node segment, walked in windows of 32 P consecutive
// CSR entries (P = DensPiece<D>::P, windows aligned to P): lane l takes the
// window's piece [w0 + l P, w0 + (l + 1) P). A lane loads its piece's
// endpoints with 16-byte loads (the next window's while the current one
// computes), gathers their coordinates together, then walks the piece in
// CSR order, its node found once by a search of the row starts and
// advanced at each row start it passes. A piece yields a partial (sum of
// phi * d^2, sum of phi) per node it touches: the first node's (h) and the
// last node's (t) stay in the lane's registers, those of nodes wholly
// inside the piece go to the node's shared slot C. The h of consecutive
// pieces that start in the same node are summed by a segmented warp scan,
// and node lane j adds its row's part of the window -- t of its first
// piece plus the run sum, or one partial -- to its sums. Every addition
// has a fixed order.
// Statistics: each block writes f64 sums of re, re^2, re * r and r over its
// nodes (a fixed warp-tree order); the last block to finish (atomic ticket
// after a fence) adds the blocks' sums in a fixed order and forms
// mean = S_re / n, var = (S_re2 - S_re^2 / n) / (n - 1),
// cov = (S_rer - mean * S_r) / (n - 1) -- the reference's two-pass f64
// moments in one pass, equal to them to f64 rounding -- then writes
// stats = {mean, std, cov, 1 / std^2, lambda * mu_tot / (std * (n - 1))} in
// f32 and re-arms the ticket for the next launch.
template <int D, bool PRECISE>
__global__ void __launch_bounds__(kDensBlock) k_dens_update(const DensArgs A)
{
    constexpr int kW = kDensBlock / 32;
    constexpr int P = DensPiece<D>::P;
    constexpr uint32_t kWin = 32u * P;
    struct Seg {
        uint32_t beg[33];
        float ys[32][D];
        float2 C[32];  // partials of nodes wholly inside one piece
    };
    __shared__ Seg sm[kW];
    __shared__ DensSums shw[kW];
    __shared__ bool is_last;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t n = A.n;
    Seg &S = sm[warp];
    const uint32_t node0 = blockIdx.x * kDensBlock + warp * 32u;
    const uint32_t node = node0 + lane;
    const bool valid = node < n;
    const uint32_t nc = min(node0, n);
    S.beg[lane] = A.offsets[valid ? node : n];
    if (lane == 31) S.beg[32] = A.offsets[min(nc + 32u, n)];
    if (valid) {
        float ys[D];
        load_row<D>(A.y, node, ys);
#pragma unroll
        for (int d = 0; d < D; d++) S.ys[lane][d] = ys[d];
    }
    __syncwarp();
#ifdef UMAPCU_CHECKED
    {
        const bool bad = S.beg[lane + 1] < S.beg[lane] || S.beg[lane + 1] > A.n_entries;
        if (__any_sync(kFull, bad)) {
            if (lane == 0) checked_ok(false, A.err);
            __syncwarp();
            S.beg[lane] = 0;
            if (lane == 31) S.beg[32] = 0;
        }
        __syncwarp();
    }
#endif
    const uint32_t seg_beg = S.beg[0], seg_end = S.beg[32];
    const uint32_t my_beg = S.beg[lane], my_end = S.beg[lane + 1];
    const bool vec = (reinterpret_cast<uintptr_t>(A.other) & 15u) == 0;
    const uint64_t pol = l2_keep_policy();
    float sum_sq = 0.0f, sum_phi = 0.0f;  // node lane's sums
    uint32_t w0 = seg_beg & ~(uint32_t)(P - 1);
    uint32_t o[P];
    if (w0 < seg_end) dens_load_piece<P>(A.other, A.n_entries, vec, w0 + lane * P, seg_beg, seg_end, o);
    for (; w0 < seg_end; w0 += kWin) {
        const uint32_t a = w0 + (uint32_t)lane * P;
        // this piece's coordinate gathers, all in flight together
        float yo[P][D];
        bool in[P];
#pragma unroll
        for (int u = 0; u < P; u++) {
            const uint32_t p = a + u;
            in[u] = p >= seg_beg && p < seg_end;
            in[u] = in[u] && checked_ok(o[u] < n, A.err);
#pragma unroll
            for (int d = 0; d < D; d++) yo[u][d] = 0.0f;
            if (in[u]) load_row_keep<D>(A.y, o[u], yo[u], pol);
        }
        // the next window's endpoints, in flight while this one computes
        if (w0 + kWin < seg_end)
            dens_load_piece<P>(A.other, A.n_entries, vec, a + kWin, seg_beg, seg_end, o);
        // the piece in CSR order: each entry's node (jj) and that node's
        // position (ys read when the node changes) ...
        uint32_t j = local_node(S.beg, a);
        const uint32_t j_first = j;
        uint32_t jj[P];
        float yv[P][D];
        {
            uint32_t nxt = S.beg[j + 1];
            float yj[D];
#pragma unroll
            for (int d = 0; d < D; d++) yj[d] = S.ys[j][d];
#pragma unroll
            for (int u = 0; u < P; u++) {
                const uint32_t p = a + u;
                if (in[u] && p >= nxt) {  // a later node's row starts here
                    do j++;
                    while (p >= S.beg[j + 1]);
                    nxt = S.beg[j + 1];
#pragma unroll
                    for (int d = 0; d < D; d++) yj[d] = S.ys[j][d];
                }
                jj[u] = j;
#pragma unroll
                for (int d = 0; d < D; d++) yv[u][d] = yj[d];
            }
        }
        // ... then phi and phi * d^2 of all entries, independent of each other
        // (no branch: entries outside the segment give 0, which leaves the sums
        // below unchanged) ...
        float ph[P], pq[P];
#pragma unroll
        for (int u = 0; u < P; u++) {
            float dist_sq = 0.0f;
#pragma unroll
            for (int d = 0; d < D; d++) {
                const float diff = yv[u][d] - yo[u][d];
                dist_sq += diff * diff;
            }
            const float dist_sq_b = pow_pos(dist_sq, A.b, PRECISE);
            const float phi = div_k(1.0f, 1.0f + A.a * dist_sq_b, PRECISE);
            ph[u] = in[u] ? phi : 0.0f;
            pq[u] = in[u] ? phi * dist_sq : 0.0f;
        }
        // ... and the sums per node in CSR order
        float ps = 0.0f, pp = 0.0f;
        float2 hf = make_float2(0.0f, 0.0f);  // the first node's partial, once closed
        bool first = true;
        uint32_t jc = j_first;
#pragma unroll
        for (int u = 0; u < P; u++) {
            if (jj[u] != jc) {
                if (first) hf = make_float2(ps, pp);
                else S.C[jc] = make_float2(ps, pp);
                first = false;
                ps = pp = 0.0f;
                jc = jj[u];
            }
            ps += pq[u];
            pp += ph[u];
        }
        // this piece's first node's partial (h), and its last node's (t) when
        // that is another node
        float hx = ps, hy = pp, tx = 0.0f, ty = 0.0f;
        if (!first) {
            hx = hf.x;
            hy = hf.y;
            tx = ps;
            ty = pp;
        }
        // h summed over each run of pieces that start in the same node
        // (a segmented inclusive scan over the lanes; the first nodes do not
        // decrease with the lane, so equal keys at lane - off mean one run)
        float sx = hx, sy = hy;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const float ux = __shfl_up_sync(kFull, sx, off), uy = __shfl_up_sync(kFull, sy, off);
            const uint32_t uk = __shfl_up_sync(kFull, j_first, off);
            if (lane >= off && uk == j_first) {
                sx = ux + sx;
                sy = uy + sy;
            }
        }
        __syncwarp();  // the C slots written above
        // node lane: its row's part of this window. Pieces l0 .. l1 hold it:
        // one piece -- that piece's h, t or the node's C slot; several -- the
        // last node's t of piece l0 (unless the node starts piece l0) and the
        // run sum at piece l1
        const uint32_t lo = max(my_beg, w0), hi = min(my_end, w0 + kWin);
        const bool mine = lo < hi;
        const uint32_t l0 = mine ? (lo - w0) / P : (uint32_t)lane, l1 = mine ? (hi - 1 - w0) / P : (uint32_t)lane;
        const uint32_t f0 = __shfl_sync(kFull, j_first, l0), e0 = __shfl_sync(kFull, j, l0);
        const float h0x = __shfl_sync(kFull, hx, l0), h0y = __shfl_sync(kFull, hy, l0);
        const float t0x = __shfl_sync(kFull, tx, l0), t0y = __shfl_sync(kFull, ty, l0);
        const float s1x = __shfl_sync(kFull, sx, l1), s1y = __shfl_sync(kFull, sy, l1);
        if (mine) {
            float vx, vy;
            if (l0 == l1) {
                if (f0 == (uint32_t)lane) {
                    vx = h0x;
                    vy = h0y;
                } else if (e0 == (uint32_t)lane) {
                    vx = t0x;
                    vy = t0y;
                } else {
                    const float2 c = S.C[lane];
                    vx = c.x;
                    vy = c.y;
                }
            } else if (f0 == (uint32_t)lane) {
                vx = s1x;
                vy = s1y;
            } else {
                vx = t0x + s1x;
                vy = t0y + s1y;
            }
            sum_sq += vx;
            sum_phi += vy;
        }
        __syncwarp();
    }
    DensSums v{0.0, 0.0, 0.0, 0.0};
    if (valid) {
        float denom = sum_phi;
        if (denom < FLT_EPSILON) denom = FLT_EPSILON;
        const float re = (float)log((double)(1e-8f + sum_sq / denom));
        const float r = A.r[node];
        A.dens_node[node] = make_float4(sum_phi, (float)exp((double)re), r, re);
        const double red_ = (double)re, rd = (double)r;
        v = DensSums{red_, red_ * red_, red_ * rd, rd};
    }
    // block sums, fixed order: warp tree, then the block's warps in order
    v = dens_sums_warp(v);
    if (lane == 0) shw[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        DensSums acc{0.0, 0.0, 0.0, 0.0};
        for (int w = 0; w < kW; w++) dens_sums_add(acc, shw[w]);
        double *pp = A.part + 4ull * blockIdx.x;
        pp[0] = acc.s_re;
        pp[1] = acc.s_re2;
        pp[2] = acc.s_rer;
        pp[3] = acc.s_r;
        __threadfence();
        is_last = atomicAdd(A.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    // the last block: every block's sums, a fixed order per thread, then the
    // warp tree and the warps in order
    DensSums acc{0.0, 0.0, 0.0, 0.0};
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += kDensBlock) {
        const double *pp = A.part + 4ull * b;
        acc.s_re += __ldcg(pp);
        acc.s_re2 += __ldcg(pp + 1);
        acc.s_rer += __ldcg(pp + 2);
        acc.s_r += __ldcg(pp + 3);
    }
    acc = dens_sums_warp(acc);
    if (lane == 0) shw[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        DensSums t{0.0, 0.0, 0.0, 0.0};
        for (int w = 0; w < kW; w++) dens_sums_add(t, shw[w]);
        const double nn = (double)(n > 1 ? n : 1);
        const double denom = (double)(n > 2 ? n - 1 : 1);
        const double mean = t.s_re / nn;
        const double var = (t.s_re2 - t.s_re * t.s_re / nn) / denom;
        const double cov = (t.s_rer - mean * t.s_r) / denom;
        const double sd = sqrt(var + (double)A.var_shift);
        const float mean_f = (float)mean, std_f = (float)sd, cov_f = (float)cov;
        const float inv_var = 1.0f / (std_f * std_f);
        const float dn = (float)(n > 1 ? n - 1 : 1);
        A.stats[0] = mean_f;
        A.stats[1] = std_f;
        A.stats[2] = cov_f;
        A.stats[3] = inv_var;
        A.stats[4] = A.lambda * A.mu_tot / (std_f * dn);
        *A.ticket = 0u;
    }
}

// ------------------------------------------------------------ launchers

// Below this many segments (about 9 blocks of one warp per segment on each
// of the 148 SMs) the list path gives each segment a whole block.
constexpr uint32_t kSplitSegments = 148 * 9;

template <int D, bool DENS>
static void launch_epoch_t(const EpochArgs &A, cudaStream_t s)
{
    const uint32_t nseg = ceil_div(A.n, 32);
    const bool fast = !A.injected && A.sampler == UMAPCU_NEG_REF_HASH && !A.precise_pow;
    const unsigned grid = ceil_div(nseg, kWarps);
    if (A.rec && nseg < kSplitSegments) {
        if (A.neg_rate == 5 && fast) k_epoch_split<D, DENS, 5, true><<<nseg, kWarps * 32, 0, s>>>(A);
        else if (A.neg_rate == 5) k_epoch_split<D, DENS, 5, false><<<nseg, kWarps * 32, 0, s>>>(A);
        else k_epoch_split<D, DENS, 0, false><<<nseg, kWarps * 32, 0, s>>>(A);
    } else if (A.rec) {
        if (A.neg_rate == 5 && fast) k_epoch<D, DENS, 5, true, true><<<grid, kWarps * 32, 0, s>>>(A);
        else if (A.neg_rate == 5) k_epoch<D, DENS, 5, false, true><<<grid, kWarps * 32, 0, s>>>(A);
        else k_epoch<D, DENS, 0, false, true><<<grid, kWarps * 32, 0, s>>>(A);
    } else if (A.bits && nseg < kSplitSegments) {
        if (A.neg_rate == 5 && fast) k_epoch_split_bits<D, DENS, 5, true><<<nseg, kSplitBitsWarps * 32, 0, s>>>(A);
        else if (A.neg_rate == 5) k_epoch_split_bits<D, DENS, 5, false><<<nseg, kSplitBitsWarps * 32, 0, s>>>(A);
        else k_epoch_split_bits<D, DENS, 0, false><<<nseg, kSplitBitsWarps * 32, 0, s>>>(A);
    } else if (A.bits) {
        if (A.neg_rate == 5 && fast) k_epoch<D, DENS, 5, true, false, true><<<grid, kWarps * 32, 0, s>>>(A);
        else if (A.neg_rate == 5) k_epoch<D, DENS, 5, false, false, true><<<grid, kWarps * 32, 0, s>>>(A);
        else k_epoch<D, DENS, 0, false, false, true><<<grid, kWarps * 32, 0, s>>>(A);
    } else {
        if (A.neg_rate == 5 && fast) k_epoch<D, DENS, 5, true><<<grid, kWarps * 32, 0, s>>>(A);
        else if (A.neg_rate == 5) k_epoch<D, DENS, 5><<<grid, kWarps * 32, 0, s>>>(A);
        else k_epoch<D, DENS, 0><<<grid, kWarps * 32, 0, s>>>(A);
    }
}

void launch_epoch(const EpochArgs &A, uint32_t n_dim, bool dens, cudaStream_t s)
{
#define UMAPCU_CASE(DD)                                          \
    case DD:                                                     \
        if (dens) launch_epoch_t<DD, true>(A, s);                \
        else launch_epoch_t<DD, false>(A, s);                    \
        break;
    switch (n_dim) {
        UMAPCU_CASE(1) UMAPCU_CASE(2) UMAPCU_CASE(3) UMAPCU_CASE(4)
        UMAPCU_CASE(5) UMAPCU_CASE(6) UMAPCU_CASE(7) UMAPCU_CASE(8)
        default: fail(UMAPCU_BAD_ARG, "n_dim must be in 1..8");
    }
#undef UMAPCU_CASE
    check_launch("k_epoch");
}

void launch_dens_update(const DensArgs &Dn, uint32_t n_dim, cudaStream_t s)
{
    const uint32_t nb = ceil_div(Dn.n, kDensBlock);
#define UMAPCU_CASE(DD)                                                   \
    case DD:                                                              \
        if (Dn.precise_pow) k_dens_update<DD, true><<<nb, kDensBlock, 0, s>>>(Dn); \
        else k_dens_update<DD, false><<<nb, kDensBlock, 0, s>>>(Dn);       \
        break;
    switch (n_dim) {
        UMAPCU_CASE(1) UMAPCU_CASE(2) UMAPCU_CASE(3) UMAPCU_CASE(4)
        UMAPCU_CASE(5) UMAPCU_CASE(6) UMAPCU_CASE(7) UMAPCU_CASE(8)
        default: fail(UMAPCU_BAD_ARG, "n_dim must be in 1..8");
    }
#undef UMAPCU_CASE
    check_launch("k_dens_update");
}

uint32_t dens_partials(uint32_t n) { return ceil_div(n, kDensBlock); }

// ------------------------------------------------------ test-hook kernels

__global__ void k_adam_apply(const float *__restrict__ grad, const uint32_t *__restrict__ has_update,
                             float *__restrict__ m, float *__restrict__ v, float *__restrict__ y, uint64_t n_total,
                             uint32_t n_dim, float fused, float epsc, float omb1, float omb2)
{
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_total) return;
    if (has_update[i / n_dim] == 0u) return;
    float mm = m[i], vv = v[i];
    y[i] = adam_coord(grad[i], mm, vv, y[i], fused, epsc, omb1, omb2);
    m[i] = mm;
    v[i] = vv;
}

void launch_adam_apply(const float *grad, const uint32_t *hu, float *m, float *v, float *y, uint64_t n_total,
                       uint32_t n_dim, float fused, float epsc, float omb1, float omb2, cudaStream_t s)
{
    if (!n_total) return;
    k_adam_apply<<<ceil_div(n_total, 256), 256, 0, s>>>(grad, hu, m, v, y, n_total, n_dim, fused, epsc, omb1, omb2);
    check_launch("k_adam_apply");
}

__global__ void k_schedule(const float *__restrict__ eps, float *__restrict__ cursor, uint64_t ne, float epoch_f)
{
    uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    if (cursor[e] <= epoch_f) cursor[e] += eps[e];
}

void launch_schedule(const float *eps, float *cursor, uint64_t ne, uint32_t epoch, cudaStream_t s)
{
    if (!ne) return;
    k_schedule<<<ceil_div(ne, 256), 256, 0, s>>>(eps, cursor, ne, (float)epoch);
    check_launch("k_schedule");
}

__global__ void k_sample(uint32_t sampler, uint32_t seed32, uint32_t seed_lo, uint32_t seed_hi, uint64_t M,
                         uint32_t node, uint32_t entry, uint32_t epoch, uint32_t edge_local, uint32_t count,
                         uint32_t n, uint32_t *__restrict__ out)
{
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    if (sampler == UMAPCU_NEG_PHILOX) {
        uint4 ph = philox4x32_10(make_uint4(entry, epoch, t >> 2, 0x554D4150u), seed_lo, seed_hi);
        uint32_t r = (t & 3) == 0 ? ph.x : (t & 3) == 1 ? ph.y : (t & 3) == 2 ? ph.z : ph.w;
        out[t] = range32(r, n);
    } else {
        out[t] = fastmod_u32(hash_neg_raw(seed32, node, epoch, edge_local, t), M, n);
    }
}

__global__ void k_eval_pow(const float *__restrict__ x, uint32_t n, float b, bool precise, float *__restrict__ out)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = pow_pos(x[i], b, precise);
}

void launch_eval_pow(const float *x, uint32_t n, float b, bool precise, float *out, cudaStream_t s)
{
    if (!n) return;
    k_eval_pow<<<ceil_div(n, 256), 256, 0, s>>>(x, n, b, precise, out);
    check_launch("k_eval_pow");
}

// L2 random-gather probe: every thread issues rounds x 8 independent 8-byte
// row gathers in the epoch kernel's load form (ld.global.nc, evict_last L2
// policy, float2 rows) at pseudo-random rows of a table small enough to stay
// in L2. The row of each gather comes from an integer hash chain (Wellons'
// "lowbias32" finaliser), independent of the loaded values.
__global__ void __launch_bounds__(256) k_l2_gather_probe(const float *__restrict__ table, uint32_t rows,
                                                         uint32_t rounds, float *__restrict__ out)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t pol = l2_keep_policy();
    uint32_t h = t * 0x9E3779B1u + 0x7F4A7C15u;
    float acc = 0.0f;
    for (uint32_t r = 0; r < rounds; r++) {
        float v[8][2];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            h ^= h >> 16;
            h *= 0x7FEB352Du;
            h ^= h >> 15;
            h *= 0x846CA68Bu;
            h ^= h >> 16;
            load_row_keep<2>(table, __umulhi(h, rows), v[u], pol);
        }
#pragma unroll
        for (int u = 0; u < 8; u++) acc += v[u][0] + v[u][1];
    }
    out[t] = acc;
}

float probe_l2_gather(uint64_t table_bytes, cudaStream_t s)
{
    const uint32_t rows = (uint32_t)(table_bytes / 8);
    const uint32_t threads = 256, blocks = (uint32_t)device_sm_count() * 8, rounds = 64;
    DevBuf<float> table((size_t)rows * 2, s), out((size_t)threads * blocks, s);
    check_cuda(cudaMemsetAsync(table.p, 0, (size_t)rows * 8, s), "memset");
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    float best = 1e30f;
    for (int it = 0; it < 6; it++) {  // the first launch warms L2
        check_cuda(cudaEventRecord(e0, s), "record");
        k_l2_gather_probe<<<blocks, threads, 0, s>>>(table.p, rows, rounds, out.p);
        check_launch("k_l2_gather_probe");
        check_cuda(cudaEventRecord(e1, s), "record");
        sync(s);
        float ms = 0.0f;
        check_cuda(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        if (it > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double bytes = 8.0 * 8.0 * rounds * (double)threads * blocks;
    return (float)(bytes / (best * 1e-3) / 1e9);
}

void launch_sample(uint32_t sampler, uint64_t seed, uint32_t node, uint32_t entry, uint32_t epoch,
                   uint32_t edge_local, uint32_t count, uint32_t n, uint32_t *out, cudaStream_t s)
{
    if (!count) return;
    k_sample<<<ceil_div(count, 128), 128, 0, s>>>(sampler, (uint32_t)seed, (uint32_t)seed, (uint32_t)(seed >> 32),
                                                  fastmod_magic(n), node, entry, epoch, edge_local, count, n, out);
    check_launch("k_sample");
}

}  // namespace umapcu
