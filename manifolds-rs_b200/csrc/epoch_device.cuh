// Device code of one layout epoch, shared by the single-problem kernel
// (layout.cu) and the multi-problem kernels (batch.cu). See layout.cu for the
// design of the warp-segment epoch.
#pragma once

#include <cfloat>

#include "internal.cuh"
#include "layout.cuh"

namespace umapcu {

constexpr int kWarps = 4;
// CSR entries are scanned in super-chunks of KU x 32 entries (default kU);
// the queue of active entries holds one super-chunk plus the carried partial
// batch.
constexpr int kU = 8;
// Negatives per chunk: exactly NR when the kernel is specialised on the
// negative sample rate (NR > 0), else 4 (one Philox block = 4 draws).
template <int NR>
constexpr int neg_chunk() { return NR > 0 ? NR : 4; }
constexpr unsigned kFull = 0xFFFFFFFFu;

// ------------------------------------------------------------ samplers

// umap_optimiser_gpu.rs:611-624 gpu_hash_neg, with h % n evaluated by
// Lemire's exact fastmod (Lemire, Kaser & Kurz 2019): M = 2^64 / n + 1.
__device__ __forceinline__ uint32_t hash_neg_raw(uint32_t seed, uint32_t node, uint32_t epoch,
                                                 uint32_t edge_local, uint32_t neg)
{
    uint32_t h = seed ^ (node * 0x9E3779B1u) ^ (epoch * 0x85EBCA77u) ^ (edge_local * 0xC2B2AE3Du) ^
                 (neg * 0x27D4EB2Fu);
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return h;
}

__device__ __forceinline__ uint32_t fastmod_u32(uint32_t a, uint64_t M, uint32_t d)
{
    // lowbits = (M * a) mod 2^64, then floor(lowbits * d / 2^64) with d < 2^32:
    // high word of (lowbits_hi * d + umulhi(lowbits_lo, d)).
    const uint64_t lowbits = M * a;
    const uint32_t lo = (uint32_t)lowbits, hi = (uint32_t)(lowbits >> 32);
    return (uint32_t)(((uint64_t)hi * d + __umulhi(lo, d)) >> 32);
}

// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ uint32_t range32(uint32_t x, uint32_t n) { return __umulhi(x, n); }

// ------------------------------------------------------------ helpers

// Checked builds (compiled with UMAPCU_CHECKED): an index that would take an
// access outside its array -- a CSR offset past the entries or out of order,
// an other endpoint, injected negative or list record beyond the nodes -- is
// reported (the error word becomes UMAPCU_BAD_ARG unless it already holds a
// status) and the access is skipped, never performed. Other builds compile
// every check away: checked_ok() is then the constant true.
__device__ __forceinline__ bool checked_ok(bool ok, uint32_t *err)
{
#ifdef UMAPCU_CHECKED
    if (!ok && err) atomicCAS(err, 0u, (uint32_t)UMAPCU_BAD_ARG);
    return ok;
#else
    (void)ok;
    (void)err;
    return true;
#endif
}

// L2 residency: the embedding (gathered at random every epoch) is loaded
// with an evict_last policy; the CSR arrays (streamed once per epoch) with
// the streaming (evict-first) qualifier, so they do not push the embedding
// out of L2. The random gathers do not allocate in L1 (they almost never
// hit there), which leaves L1 to the segment's streamed lines (1M points:
// 26.5 -> 26.1 ms per 200-epoch run).
__device__ __forceinline__ uint64_t l2_keep_policy()
{
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// COH = true: loads of data that other SMs rewrite while the kernel runs
// (the persistent multi-problem kernel: the embedding buffers, moments and
// cursors change roles every epoch). They go through L2 (ld.global.cg)
// instead of the non-coherent read-only path / L1.
template <int D, bool COH = false>
__device__ __forceinline__ void load_row_keep(const float *__restrict__ y, uint32_t i, float (&out)[D], uint64_t pol)
{
    if constexpr (D == 2) {
        const float *a = y + 2ull * i;
        if constexpr (COH)
            asm volatile("ld.global.cg.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
                         : "=f"(out[0]), "=f"(out[1])
                         : "l"(a), "l"(pol));
        else
            asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
                         : "=f"(out[0]), "=f"(out[1])
                         : "l"(a), "l"(pol));
    } else if constexpr (D == 4) {
        const float *a = y + 4ull * i;
        if constexpr (COH)
            asm volatile("ld.global.cg.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                         : "=f"(out[0]), "=f"(out[1]), "=f"(out[2]), "=f"(out[3])
                         : "l"(a), "l"(pol));
        else
            asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                         : "=f"(out[0]), "=f"(out[1]), "=f"(out[2]), "=f"(out[3])
                         : "l"(a), "l"(pol));
    } else {
#pragma unroll
        for (int d = 0; d < D; d++) {
            const float *a = y + (uint64_t)i * D + d;
            if constexpr (COH)
                asm volatile("ld.global.cg.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(out[d]) : "l"(a), "l"(pol));
            else
                asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(out[d]) : "l"(a), "l"(pol));
        }
    }
}

template <int D, bool COH = false>
__device__ __forceinline__ void load_row(const float *__restrict__ y, uint32_t i, float (&out)[D])
{
    if constexpr (D == 2) {
        const float2 *a = reinterpret_cast<const float2 *>(y) + i;
        float2 v = COH ? __ldcg(a) : __ldg(a);
        out[0] = v.x;
        out[1] = v.y;
    } else if constexpr (D == 4) {
        const float4 *a = reinterpret_cast<const float4 *>(y) + i;
        float4 v = COH ? __ldcg(a) : __ldg(a);
        out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
    } else {
#pragma unroll
        for (int d = 0; d < D; d++) out[d] = COH ? __ldcg(y + (uint64_t)i * D + d) : __ldg(y + (uint64_t)i * D + d);
    }
}

template <int D>
__device__ __forceinline__ void store_row(float *__restrict__ y, uint32_t i, const float (&v)[D])
{
    if constexpr (D == 2) {
        reinterpret_cast<float2 *>(y)[i] = make_float2(v[0], v[1]);
    } else if constexpr (D == 4) {
        reinterpret_cast<float4 *>(y)[i] = make_float4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
        for (int d = 0; d < D; d++) y[(uint64_t)i * D + d] = v[d];
    }
}

// x^b for the strictly positive x of the UMAP kernels (dist_sq >= 1e-8,
// dist_sq + 0.001): 2^(b * log2 x) on the MUFU units (lg2.approx /
// ex2.approx, no subnormal inputs occur). Relative error about 1e-6 over
// x in [1e-8, 1e6] against the correctly rounded power (checked on the device
// by the test suite), a few ulp; CUDA's full-range powf costs ~30x the
// instructions. `precise` selects CUDA's powf instead.
__device__ __forceinline__ float pow_pos(float x, float b, bool precise)
{
    if (precise) return powf(x, b);
    float l, r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l) : "f"(x));
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b * l));
    return r;
}

// a / b for the kernels' positive denominators (>= 1e-11): IEEE division
// when `precise`, else a * rcp.approx(b) (2 ulp).
__device__ __forceinline__ float div_k(float a, float b, bool precise)
{
    return precise ? a / b : __fdividef(a, b);
}

__device__ __forceinline__ float clip4(float x)
{
    if (x > 4.0f) x = 4.0f;
    if (x < -4.0f) x = -4.0f;
    return x;
}

// umap_adam_update (umap_optimiser_gpu.rs:912-922) for one coordinate.
__device__ __forceinline__ float adam_coord(float g, float &m, float &v, float y, float fused, float epsc,
                                           float omb1, float omb2)
{
    float m_new = m + omb1 * (g - m);
    m = m_new;
    float v_new = v + omb2 * (g * g - v);
    v = v_new;
    return y + fused * m_new / (sqrtf(v_new) + epsc);
}

// densMAP per-node weight (umap_dens_weights, umap_optimiser_gpu.rs:584-585).
__device__ __forceinline__ float dens_weight(float r, float re, const float *__restrict__ st)
{
    // st = {mean, std, cov, inv_var, coeff}
    return r - st[2] * (re - st[0]) * st[3];
}

// Per-warp shared memory of the segment walk. The queue holds the CSR
// positions (and, for the cursor scan, the other endpoints) of active
// entries not yet evaluated: one super-chunk plus the carried partial batch
// for the cursor scan; for the bitmask scan, a group of 32 x BP entries (a
// lane per BP) plus the carried partial batch. The densMAP node records only
// in the densMAP kernels.
// Shared memory is sized with care: the random coordinate gathers hold their
// in-flight misses in L1, which gets what the blocks' shared memory leaves of
// each SM's 256 KB; at 8 resident blocks, 22.6 KB of shared memory per block
// (a 1024-entry queue) left 60 KB of L1 and 25.8 KB left 28 KB, and the epoch
// took 141 and 243 us at 1M points. Larger groups cost less per entry on
// long segments, smaller ones leave more L1 (bits_piece).
template <int D, int KU = kU, bool BITS = false, bool DENS = true, int BP = 32>
struct WarpSmem {
    static constexpr int kQ = BITS ? BP * 32 + 32 : 32 * KU + 32;
    uint32_t beg[33];
    uint32_t qp[kQ];
    uint32_t qo[BITS ? 1 : kQ];
    float ys[32][D];
    float part[32][D];
    float4 dn[DENS ? 32 : 1];
};

__device__ __forceinline__ uint32_t local_node(const uint32_t *beg, uint32_t p)
{
    // largest j in [0, 31] with beg[j] <= p
    uint32_t j = 0;
#pragma unroll
    for (uint32_t step = 16; step > 0; step >>= 1)
        if (beg[j + step] <= p) j += step;
    return j;
}

// One batch of up to 32 active entries, lane t = entry t (`live` lanes
// only): CSR position p, other endpoint o, the entry's node as an index j
// into the segment, and its offset el within the node's row. The other
// endpoint's row and the first chunk of negatives' rows are gathered
// together, so a batch waits on L2 once.
// FAST: the common configuration resolved at compile time (reference hash
// sampler, no injected negatives, MUFU x^b and approximate division), which
// removes the per-negative and per-term uniform branches of the general path.
// The batch's per-node sums go to part[j] for the nodes in the returned
// mask; unless SPLIT, the node's lane then adds them to g (and sets act).
template <int D, bool DENS, int NR, bool COH, int KU, bool FAST, bool SPLIT = false, class Smem = WarpSmem<D, KU>>
__device__ __forceinline__ unsigned process_batch(const EpochArgs &A, Smem &S, bool live, uint32_t p,
                                                  uint32_t o, uint32_t j, uint32_t edge_local, uint32_t node0,
                                                  int lane, float (&g)[D], bool &act, const float *dstat,
                                                  float (*part)[D])
{
    if (live && !checked_ok(o < A.n && p < A.n_entries, A.err)) live = false;
    if (!live) j = 32;  // dead lanes: a node of their own, contributing zero
    float c[D];
#pragma unroll
    for (int d = 0; d < D; d++) c[d] = 0.0f;
    if (live) {
        const uint32_t self = node0 + j;
        float ys[D], yo[D];
#pragma unroll
        for (int d = 0; d < D; d++) ys[d] = S.ys[j][d];
        const uint64_t pol = l2_keep_policy();
        constexpr int kNegChunk = neg_chunk<NR>();
        const uint32_t neg_rate = NR > 0 ? (uint32_t)NR : A.neg_rate;
        uint32_t kk[kNegChunk];
        float yk[kNegChunk][D];
        // negatives of chunk k0 (umap_optimiser_gpu.rs:801-816): indices and
        // gathers issued before any of them is used
        auto issue = [&](uint32_t k0) {
            uint4 ph = make_uint4(0, 0, 0, 0);
#pragma unroll
            for (int t = 0; t < kNegChunk; t++) {
                const uint32_t neg = k0 + t;
                uint32_t kn = self;
                if (neg < neg_rate) {
                    if (!FAST && A.injected) {
                        kn = A.injected[(uint64_t)p * neg_rate + neg];
                        if (!checked_ok(kn < A.n, A.err)) kn = self;  // skipped like a self sample
                    } else if (!FAST && A.sampler == UMAPCU_NEG_PHILOX) {
                        if ((t & 3) == 0) ph = philox4x32_10(make_uint4(p, A.epoch, neg >> 2, 0x554D4150u), A.seed_lo,
                                                             A.seed_hi);
                        uint32_t r = (t & 3) == 0 ? ph.x : (t & 3) == 1 ? ph.y : (t & 3) == 2 ? ph.z : ph.w;
                        kn = range32(r, A.n);
                    } else {
                        kn = fastmod_u32(hash_neg_raw(A.seed32, self, A.epoch, edge_local, neg), A.fastmod_M, A.n);
                    }
                }
                kk[t] = kn;
                if (neg < neg_rate) load_row_keep<D, COH>(A.y_cur, kn, yk[t], pol);
            }
        };
        load_row_keep<D, COH>(A.y_cur, o, yo, pol);
        // (wider rows: registers for all gathers at once would spill)
        if constexpr (D <= 2) issue(0);
        float4 dno;
        float mu_e = 1.0f;
        if constexpr (DENS) {
            dno = __ldg(A.dens_node + o);
            mu_e = __ldg(A.mu_entry + p);
        }
        // attractive (umap_optimiser_gpu.rs:746-762)
        float dist_sq = 0.0f;
#pragma unroll
        for (int d = 0; d < D; d++) {
            float diff = ys[d] - yo[d];
            dist_sq += diff * diff;
        }
        if (dist_sq >= 1e-8f) {
            float dist_sq_b = pow_pos(dist_sq, A.b, (!FAST && A.precise_pow));
            float denom = 1.0f + A.a * dist_sq_b;
            float grad_coeff = div_k(A.two_a_b * dist_sq_b, dist_sq * denom, (!FAST && A.precise_pow));
            if (A.optimiser == UMAPCU_OPT_SGD) {
#pragma unroll
                for (int d = 0; d < D; d++) c[d] += 2.0f * clip4(grad_coeff * (yo[d] - ys[d]));
            } else {
                const float gc2 = 2.0f * grad_coeff;
#pragma unroll
                for (int d = 0; d < D; d++) c[d] += gc2 * (yo[d] - ys[d]);
            }
            if constexpr (DENS) {
                // umap_optimiser_gpu.rs:769-798
                const float4 dns = S.dn[j];
                const bool pr = !FAST && A.precise_pow;
                float phi = div_k(1.0f, denom, pr);
                float dphi_term = div_k(A.a * A.b * dist_sq_b, dist_sq, pr) * phi;
                float common = 1.0f - A.b * (1.0f - phi);
                float dr_self = div_k(phi, dns.x, pr) * (div_k(common, dns.y, pr) + dphi_term);
                float dr_other = div_k(phi, dno.x, pr) * (div_k(common, dno.y, pr) + dphi_term);
                float w_s = dens_weight(dns.z, dns.w, dstat), w_o = dens_weight(dno.z, dno.w, dstat);
                float cor = div_k(dstat[4] * (w_s * dr_self + w_o * dr_other), mu_e, pr);
                float two_cor = 2.0f * cor;
#pragma unroll
                for (int d = 0; d < D; d++) c[d] += 2.0f * clip4(two_cor * (ys[d] - yo[d]));
            }
        }
        // negatives (umap_optimiser_gpu.rs:817-849)
        for (uint32_t k0 = 0; k0 < neg_rate; k0 += kNegChunk) {
            if (k0 || D > 2) issue(k0);
#pragma unroll
            for (int t = 0; t < kNegChunk; t++) {
                if (k0 + t < neg_rate && kk[t] != self) {
                    float diff[D], dsk = 0.0f;
#pragma unroll
                    for (int d = 0; d < D; d++) {
                        diff[d] = ys[d] - yk[t][d];
                        dsk += diff[d] * diff[d];
                    }
                    float dist_sq_safe = dsk + 0.001f;
                    float dist_sq_b = pow_pos(dist_sq_safe, A.b, (!FAST && A.precise_pow));
                    float denom = dist_sq_safe * (1.0f + A.a * dist_sq_b);
                    float gc = clip4(div_k(A.two_gamma_b, denom, (!FAST && A.precise_pow)));
#pragma unroll
                    for (int d = 0; d < D; d++) c[d] += gc * diff[d];
                }
            }
        }
    }
    // Per-node sums of the lanes' partials: the slots are sorted by node, so
    // each node's slots form a run; a segmented inclusive scan over the warp
    // leaves each run's sum on its last lane, which hands it to the node's
    // lane through shared memory.
    const uint32_t jprev = __shfl_up_sync(kFull, j, 1);
    const uint32_t jnext = __shfl_down_sync(kFull, j, 1);
    const unsigned heads = __ballot_sync(kFull, lane == 0 || jprev != j);
    const int start = 31 - __clz(heads & (lane == 31 ? kFull : ((2u << lane) - 1u)));
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
        for (int d = 0; d < D; d++) {
            const float v = __shfl_up_sync(kFull, c[d], off);
            if (lane - off >= start) c[d] += v;
        }
    }
    const bool tail = live && (lane == 31 || jnext != j);
    if (tail) {
#pragma unroll
        for (int d = 0; d < D; d++) part[j][d] = c[d];
    }
    const unsigned has = __reduce_or_sync(kFull, tail ? (1u << j) : 0u);
    if constexpr (!SPLIT) {
        __syncwarp();
        if ((has >> lane) & 1u) {
            act = true;
#pragma unroll
            for (int d = 0; d < D; d++) g[d] += part[lane][d];
        }
        __syncwarp();
    }
    return has;
}

// The segment's row starts, positions (and densMAP node data) into shared
// memory; ys = the lane's node's position (zeros beyond n).
template <int D, bool DENS, bool COH, class Smem>
__device__ __forceinline__ void load_segment(const EpochArgs &A, Smem &S, uint32_t node0, int lane, float (&ys)[D])
{
    const uint32_t node = node0 + lane;
    const bool valid = node < A.n;
    S.beg[lane] = A.offsets[valid ? node : A.n];
    if (lane == 31) S.beg[32] = A.offsets[min(node0 + 32u, A.n)];
    if (valid) load_row<D, COH>(A.y_cur, node, ys);
    else {
#pragma unroll
        for (int d = 0; d < D; d++) ys[d] = 0.0f;
    }
#pragma unroll
    for (int d = 0; d < D; d++) S.ys[lane][d] = ys[d];
    if constexpr (DENS) {
        if (valid) S.dn[lane] = __ldg(A.dens_node + node);
    }
#ifdef UMAPCU_CHECKED
    // the segment's row starts must be in order and within the entries; a
    // segment that breaks that is walked as empty
    __syncwarp();
    const bool bad = S.beg[lane + 1] < S.beg[lane] || S.beg[lane + 1] > A.n_entries;
    if (__any_sync(kFull, bad)) {
        if (lane == 0) checked_ok(false, A.err);
        __syncwarp();
        S.beg[lane] = 0;
        if (lane == 31) S.beg[32] = 0;
    }
    __syncwarp();
#endif
}

// The node's step (umap_adam_update, umap_optimiser_gpu.rs:887-923, or the
// SGD step) from its gradient g, and the next embedding buffer's row.
template <int D, bool COH>
__device__ __forceinline__ void finish_node(const EpochArgs &A, uint32_t node, const float (&ys)[D],
                                            const float (&g)[D], bool act)
{
    float yn[D];
    if (act) {
        if (A.optimiser == UMAPCU_OPT_SGD) {
#pragma unroll
            for (int d = 0; d < D; d++) yn[d] = ys[d] + A.lr_sgd * g[d];
        } else {
            float m[D], v[D];
            load_row<D, COH>(A.m, node, m);
            load_row<D, COH>(A.v, node, v);
#pragma unroll
            for (int d = 0; d < D; d++) yn[d] = adam_coord(g[d], m[d], v[d], ys[d], A.fused, A.epsc, A.omb1, A.omb2);
            store_row<D>(A.m, node, m);
            store_row<D>(A.v, node, v);
        }
    } else {
#pragma unroll
        for (int d = 0; d < D; d++) yn[d] = ys[d];
    }
    store_row<D>(A.y_next, node, yn);
    if (A.dbg_grad) store_row<D>(A.dbg_grad, node, g);
    if (A.dbg_active) A.dbg_active[node] = act ? 1u : 0u;
}

// One epoch of one 32-node segment [node0, node0 + 32) of problem A, run by
// one warp (see the file comment).
// LIST: the segment's active entries come from the epoch's schedule lists
// (A.rec / A.seg_ptr) instead of a scan of its CSR range.
// BITS: the scan reads the epoch's active-entry bitmask (A.bits) in place of
// the entries' (cursor, period) and writes no cursor.
template <int D, bool DENS, int NR, bool COH, int KU = kU, bool FAST = false, bool LIST = false,
          bool BITS = false, int BP = 32>
__device__ __forceinline__ void epoch_segment(const EpochArgs &A, WarpSmem<D, KU, BITS, DENS, BP> &S, uint32_t node0,
                                              int lane)
{
    __syncwarp();  // the warp's shared memory may still be read by its previous segment
    const uint32_t node = node0 + lane;
    const bool valid = node < A.n;
    float ys[D];
    load_segment<D, DENS, COH>(A, S, node0, lane, ys);
    const float *dstat = A.dens_stats;
    // Degenerate self beyond the last beg (beg[32] read by the search only
    // through j + step <= 31 + 1).
    float g[D];
#pragma unroll
    for (int d = 0; d < D; d++) g[d] = 0.0f;
    bool act = false;
    __syncwarp();
    if constexpr (LIST) {
        // records in CSR order, 32 per batch; the next chunk's records are
        // loaded while the current batch runs
        const uint32_t sg = node0 >> 5;
        const uint64_t r0 = A.seg_ptr[A.seg_unit[sg]], r1 = A.seg_ptr[A.seg_unit[sg + 1]];
        uint2 nx = make_uint2(0, 0);
        if (r0 + lane < r1) nx = __ldcs(A.rec + r0 + lane);
        for (uint64_t q = r0; q < r1; q += 32) {
            const bool live = q + lane < r1;
            const uint32_t j = nx.x >> kRecNodeShift, el = nx.x & kRecOffsetMask, o = nx.y;
            uint32_t p = live ? S.beg[j] + el : 0u;  // unused (and not loaded) on the fast path
#ifdef UMAPCU_CHECKED
            if (live && !checked_ok(p < S.beg[j + 1], A.err)) p = ~0u;  // refused in process_batch
#endif
            if (q + 32 + lane < r1) nx = __ldcs(A.rec + q + 32 + lane);
            process_batch<D, DENS, NR, COH, KU, FAST>(A, S, live, p, o, j, el, node0, lane, g, act, dstat, S.part);
        }
    } else if constexpr (BITS) {
        // The epoch's bit words in pieces of BP CSR entries, a lane per piece,
        // 32 x BP entries at a time: the pieces are masked to the segment, an
        // exclusive warp prefix of their popcounts gives each lane its first
        // queue slot, and each lane writes the positions of its set bits in
        // ascending order -- so the queue holds the active entries in CSR
        // order, and every 32 of them form a batch exactly as in the cursor
        // scan below. The other endpoint is loaded for active entries only,
        // one batch ahead.
        const uint32_t seg_beg = S.beg[0], seg_end = S.beg[32];
        uint32_t count = 0;
        static_assert(BP == 8 || BP == 16 || BP == 32, "pieces of 8, 16 or 32 entries");
        for (uint64_t e0 = seg_beg & ~(uint32_t)(BP - 1); e0 < seg_end; e0 += 32u * BP) {
            const uint64_t wb = e0 + (uint32_t)BP * (uint32_t)lane;
            uint32_t m = 0;
            if (wb < seg_end) {
                // the piece lies inside one word: wb is a multiple of BP
                const uint32_t word = __ldg(A.bits + (wb >> 5));
                m = BP == 32 ? word : (word >> ((uint32_t)wb & 31u)) & ((1u << (BP & 31)) - 1u);
                if (wb < seg_beg) m &= ~0u << (seg_beg - (uint32_t)wb);
                if (seg_end - wb < (uint32_t)BP) m &= (1u << (uint32_t)(seg_end - wb)) - 1u;
            }
            const uint32_t c = __popc(m);
            uint32_t x = c;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t y = __shfl_up_sync(kFull, x, off);
                if (lane >= off) x += y;
            }
            uint32_t slot = count + x - c;
            while (m) {
                S.qp[slot++] = (uint32_t)wb + (uint32_t)(__ffs(m) - 1);
                m &= m - 1u;
            }
            count += __shfl_sync(kFull, x, 31);
            __syncwarp();
            const bool last = e0 + 32u * BP >= seg_end;
            const uint32_t upto = last ? count : (count & ~31u);
            uint32_t p = 0, o = 0;
            if ((uint32_t)lane < upto) {
                p = S.qp[lane];
                o = __ldcs(A.other + p);
            }
            for (uint32_t q0 = 0; q0 < upto; q0 += 32) {
                const bool live = q0 + lane < upto;
                uint32_t pn = 0, on = 0;
                if (q0 + 32u + lane < upto) {
                    pn = S.qp[q0 + 32u + lane];
                    on = __ldcs(A.other + pn);
                }
                uint32_t j = 0, el = 0;
                if (live) {
                    j = local_node(S.beg, p);
                    el = p - S.beg[j];
                }
                process_batch<D, DENS, NR, COH, KU, FAST>(A, S, live, p, o, j, el, node0, lane, g, act, dstat, S.part);
                p = pn;
                o = on;
            }
            const uint32_t rem = count - upto;
            if (upto && rem) {
                const uint32_t tp = (uint32_t)lane < rem ? S.qp[upto + lane] : 0u;
                __syncwarp();
                if ((uint32_t)lane < rem) S.qp[lane] = tp;
            }
            __syncwarp();
            count = rem;
        }
    } else {
    const uint32_t seg_beg = S.beg[0], seg_end = S.beg[32];
    const unsigned lt_mask = (1u << lane) - 1u;
    uint32_t count = 0;
    float *cursor = reinterpret_cast<float *>(A.sched);
    // Scan in super-chunks of kU x 32 entries: all loads of a super-chunk are
    // issued before the first is used.
    for (uint32_t c0 = seg_beg; c0 < seg_end; c0 += 32u * KU) {
        float2 sv[KU];
        uint32_t ov[KU];
#pragma unroll
        for (int u = 0; u < KU; u++) {
            const uint32_t p = c0 + 32u * u + lane;
            sv[u] = make_float2(__int_as_float(0x7f800000), 0.0f);
            ov[u] = 0;
            if (p < seg_end) {
                sv[u] = COH ? __ldcg(A.sched + p) : __ldcs(A.sched + p);
                ov[u] = __ldcs(A.other + p);
            }
        }
#pragma unroll
        for (int u = 0; u < KU; u++) {
            const uint32_t p = c0 + 32u * u + lane;
            const bool a = sv[u].x <= A.epoch_f;  // out-of-range lanes hold +inf
            if (a) __stcs(cursor + 2 * (uint64_t)p, sv[u].x + sv[u].y);  // umap_edge_schedule_update
            const unsigned mask = __ballot_sync(kFull, a);
            if (a) {
                const uint32_t slot = count + __popc(mask & lt_mask);
                S.qp[slot] = p;
                S.qo[slot] = ov[u];
            }
            count += __popc(mask);
        }
        __syncwarp();
        const bool more = c0 + 32u * KU < seg_end;
        // every full batch, and at the end of the segment the remainder too
        const bool last = !more;
        const uint32_t upto = last ? count : (count & ~31u);
        for (uint32_t q0 = 0; q0 < upto; q0 += 32) {
            const bool live = (uint32_t)lane < min(32u, upto - q0);
            uint32_t p = 0, o = 0, j = 0, el = 0;
            if (live) {
                p = S.qp[q0 + lane];
                o = S.qo[q0 + lane];
                j = local_node(S.beg, p);
                el = p - S.beg[j];
            }
            process_batch<D, DENS, NR, COH, KU, FAST>(A, S, live, p, o, j, el, node0, lane, g, act, dstat, S.part);
        }
        const uint32_t rem = count - upto;
        if (upto && rem) {
            uint32_t tp = 0, to = 0;
            if ((uint32_t)lane < rem) { tp = S.qp[upto + lane]; to = S.qo[upto + lane]; }
            __syncwarp();
            if ((uint32_t)lane < rem) { S.qp[lane] = tp; S.qo[lane] = to; }
            __syncwarp();
        }
        count = rem;
    }
    }
    if (!valid) return;
    finish_node<D, COH>(A, node, ys, g, act);
}

// One epoch of one 32-node segment run by all kWarps warps of a block, for
// problems too small to fill the GPU with one warp per segment (schedule
// lists only). The segment's batches are the same 32-record slices of its
// list as in epoch_segment; in each round warp w evaluates batch
// round * kWarps + w into its own part[w], and warp 0's node lanes add the
// round's partials in batch order -- the order epoch_segment adds them in, so
// the result is bit-identical.
template <int D, bool DENS, int NR, bool FAST>
__device__ __forceinline__ void epoch_segment_split(const EpochArgs &A, WarpSmem<D, 1, false, DENS> &S,
                                                    float (*part)[32][D],
                                                    unsigned *has_w, uint32_t node0, int warp, int lane)
{
    const uint32_t node = node0 + lane;
    const bool valid = node < A.n;
    float ys[D];
    if (warp == 0) load_segment<D, DENS, false>(A, S, node0, lane, ys);
    __syncthreads();
    const float *dstat = A.dens_stats;
    float g[D];
#pragma unroll
    for (int d = 0; d < D; d++) g[d] = 0.0f;
    bool act = false;
    const uint32_t sg = node0 >> 5;
    const uint64_t r0 = A.seg_ptr[A.seg_unit[sg]], r1 = A.seg_ptr[A.seg_unit[sg + 1]];
    const uint64_t stride = 32u * kWarps;
    uint2 nx = make_uint2(0, 0);
    if (r0 + 32u * warp + lane < r1) nx = __ldcs(A.rec + r0 + 32u * warp + lane);
    for (uint64_t q0 = r0; q0 < r1; q0 += stride) {  // block-uniform
        const uint64_t q = q0 + 32u * warp;
        unsigned has = 0;
        if (q < r1) {  // warp-uniform
            const bool live = q + lane < r1;
            const uint32_t j = nx.x >> kRecNodeShift, el = nx.x & kRecOffsetMask, o = nx.y;
            uint32_t p = live ? S.beg[j] + el : 0u;
#ifdef UMAPCU_CHECKED
            if (live && !checked_ok(p < S.beg[j + 1], A.err)) p = ~0u;
#endif
            if (q + stride + lane < r1) nx = __ldcs(A.rec + q + stride + lane);
            float gd[D];
            bool ad = false;
            has = process_batch<D, DENS, NR, false, 1, FAST, true>(A, S, live, p, o, j, el, node0, lane, gd, ad,
                                                                   dstat, part[warp]);
        }
        if (lane == 0) has_w[warp] = has;
        __syncthreads();
        if (warp == 0) {
#pragma unroll
            for (int w = 0; w < kWarps; w++) {
                if ((has_w[w] >> lane) & 1u) {
                    act = true;
#pragma unroll
                    for (int d = 0; d < D; d++) g[d] += part[w][lane][d];
                }
            }
        }
        __syncthreads();
    }
    if (warp != 0 || !valid) return;
    finish_node<D, false>(A, node, ys, g, act);
}

// Position of the k-th set bit (k from 0) of m, which has more than k set
// bits: a binary search on popcounts.
__device__ __forceinline__ uint32_t select_bit(uint32_t m, uint32_t k)
{
    uint32_t pos = 0;
#pragma unroll
    for (uint32_t w = 16; w > 0; w >>= 1) {
        const uint32_t c = __popc(m & ((1u << w) - 1u));
        if (k >= c) {
            k -= c;
            m >>= w;
            pos += w;
        }
    }
    return pos;
}

// Words of a segment's bitmask one block of epoch_segment_split_bits holds;
// a longer segment runs on warp 0 alone with the sequential scan.
constexpr uint32_t kSplitWords = 256;
// Warps of a k_epoch_split_bits block: a small problem's segment has a few
// batches per epoch, and each warp takes one batch per round, so more warps
// mean fewer dependent rounds of gathers per epoch.
constexpr int kSplitBitsWarps = 8;

// The bitmask form of epoch_segment_split: the block reads the segment's
// words of the epoch's bitmask, masks them to the segment's entries, and
// forms prefix counts; batch b is then the active entries of rank 32 b ..
// 32 b + 31 in CSR order -- the batches the sequential scan forms -- and
// lane t finds its entry by searching the prefix counts and selecting the
// bit. Partials are added in batch order as in epoch_segment_split, so the
// result is bit-identical to the scan.
template <int D, bool DENS, int NR, bool FAST, int W = kWarps>
__device__ __forceinline__ void epoch_segment_split_bits(const EpochArgs &A, WarpSmem<D, kU, true, DENS, 32> &S,
                                                         float (*part)[32][D],
                                                         unsigned *has_w, uint32_t *wm, uint32_t *pre,
                                                         uint32_t node0, int warp, int lane)
{
    uint32_t sbeg = A.offsets[node0], send = A.offsets[min(node0 + 32u, A.n)];
#ifdef UMAPCU_CHECKED
    if (!checked_ok(sbeg <= send && send <= A.n_entries, A.err)) sbeg = send = 0;
#endif
    const uint32_t w0 = sbeg >> 5, nw = send > sbeg ? ((send - 1) >> 5) - w0 + 1 : 0;
    if (nw > kSplitWords) {  // block-uniform
        if (warp == 0) epoch_segment<D, DENS, NR, false, kU, FAST, false, true>(A, S, node0, lane);
        return;
    }
    const uint32_t node = node0 + lane;
    const bool valid = node < A.n;
    float ys[D];
    if (warp == 0) load_segment<D, DENS, false>(A, S, node0, lane, ys);
    // masked words and their popcounts; exclusive prefix by warp 0
    for (uint32_t t = threadIdx.x; t < nw; t += blockDim.x) {
        const uint32_t wi = w0 + t;
        uint32_t m = __ldg(A.bits + wi);
        if (wi * 32u < sbeg) m &= ~0u << (sbeg - wi * 32u);
        if (wi * 32u + 32u > send) m &= (send - wi * 32u >= 32u) ? ~0u : ((1u << (send - wi * 32u)) - 1u);
        wm[t] = m;
    }
    __syncthreads();
    if (warp == 0) {
        uint32_t carry = 0;
        for (uint32_t t0 = 0; t0 < nw; t0 += 32) {
            const uint32_t t = t0 + lane;
            const uint32_t c = t < nw ? __popc(wm[t]) : 0u;
            uint32_t x = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(kFull, x, o);
                if (lane >= o) x += y;
            }
            if (t < nw) pre[t] = carry + x - c;
            carry += __shfl_sync(kFull, x, 31);
        }
        if (lane == 0) pre[kSplitWords] = carry;  // total active entries
    }
    __syncthreads();
    const uint32_t total = pre[kSplitWords];
    const float *dstat = A.dens_stats;
    float g[D];
#pragma unroll
    for (int d = 0; d < D; d++) g[d] = 0.0f;
    bool act = false;
    for (uint32_t r0 = 0; r0 < total; r0 += 32u * W) {  // block-uniform
        const uint32_t rb = r0 + 32u * warp;
        unsigned has = 0;
        if (rb < total) {  // warp-uniform
            const uint32_t r = rb + lane;
            const bool live = r < total;
            uint32_t p = 0, o = 0, j = 0, el = 0;
            if (live) {
                uint32_t lo = 0, hi = nw;  // last word with pre <= r
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (pre[mid] <= r) lo = mid;
                    else hi = mid;
                }
                p = (w0 + lo) * 32u + select_bit(wm[lo], r - pre[lo]);
                o = __ldg(A.other + p);
                j = local_node(S.beg, p);
                el = p - S.beg[j];
            }
            float gd[D];
            bool ad = false;
            has = process_batch<D, DENS, NR, false, kU, FAST, true>(A, S, live, p, o, j, el, node0, lane, gd, ad,
                                                                    dstat, part[warp]);
        }
        if (lane == 0) has_w[warp] = has;
        __syncthreads();
        if (warp == 0) {
#pragma unroll
            for (int w = 0; w < W; w++) {
                if ((has_w[w] >> lane) & 1u) {
                    act = true;
#pragma unroll
                    for (int d = 0; d < D; d++) g[d] += part[w][lane][d];
                }
            }
        }
        __syncthreads();
    }
    if (warp != 0 || !valid) return;
    finish_node<D, false>(A, node, ys, g, act);
}

}  // namespace umapcu
