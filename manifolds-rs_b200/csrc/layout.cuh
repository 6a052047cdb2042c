// Layout-epoch kernel interfaces (see layout.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace umapcu {

// Arguments of one epoch of one embedding problem.
struct EpochArgs {
    uint32_t n;
    const uint32_t *offsets;   // [n + 1] CSR offsets
    const uint32_t *other;     // [2E + 8] other endpoint per CSR entry
    float2 *sched;             // [2E + 8] per-entry (cursor, period), advanced in place
    const float *mu_entry;     // [2E] edge weight per entry (densMAP only)
    const float *y_cur;        // [n * D] embedding read this epoch
    float *y_next;             // [n * D] embedding written this epoch
    float *m;                  // [n * D] Adam first moment
    float *v;                  // [n * D] Adam second moment
    const float4 *dens_node;   // [n] {phi_sum, exp(re), r, re} (densMAP only)
    const float *dens_stats;   // {mean, std, cov, inv_var, coeff} (densMAP only)
    const uint2 *rec;          // schedule lists: (CSR position, other) of active entries, or nullptr (scan)
    const uint64_t *seg_ptr;   // schedule lists: this epoch's record offsets per work unit
    const uint32_t *seg_unit;  // schedule lists: [nseg + 1] each segment's first work unit
    const uint32_t *bits;      // schedule bitmask of this epoch (bit p: entry p active), or nullptr
    const uint32_t *injected;  // [2E * neg_rate] injected negatives or nullptr
    float *dbg_grad;           // [n * D] gradient output or nullptr
    uint32_t *dbg_active;      // [n] has_update output or nullptr
    uint32_t epoch;
    float epoch_f;
    float fused;               // lr * (1 - e/N) * ad_scale
    float epsc;                // sqrt(1 - beta2^t) * eps
    float lr_sgd;              // lr * (1 - e/N) (SGD)
    float a, b, two_a_b, two_gamma_b, omb1, omb2;
    uint32_t neg_rate;
    uint32_t sampler;
    uint32_t seed32, seed_lo, seed_hi;
    uint64_t fastmod_M;
    uint32_t optimiser;
    bool precise_pow;          // CUDA powf instead of pow_pos
    uint64_t n_entries;        // CSR entries (2E): the length of other / sched / mu_entry
    uint32_t *err;             // checked builds: error word (UMAPCU_BAD_ARG on a bad index), or nullptr
};

// Arguments of one densMAP radius/statistics update.
struct DensArgs {
    uint32_t n;
    const uint32_t *offsets;
    const uint32_t *other;
    const float *y;
    float a, b;
    const float *r;       // [n] z-scored original log radii
    float4 *dens_node;    // [n] output
    double *part;         // [4 * dens_partials(n)] per-block f64 sums
    uint32_t *ticket;     // [1] zero between launches (the last block re-arms it)
    float *stats;         // [5]
    float var_shift, lambda, mu_tot;
    bool precise_pow;
    uint64_t n_entries;   // CSR entries: the length of other
    uint32_t *err;        // checked builds: error word, or nullptr
};

inline uint64_t fastmod_magic(uint32_t n) { return n ? (~0ull / n) + 1 : 0; }

void launch_epoch(const EpochArgs &A, uint32_t n_dim, bool dens, cudaStream_t s);
void launch_dens_update(const DensArgs &D, uint32_t n_dim, cudaStream_t s);
uint32_t dens_partials(uint32_t n);
void launch_adam_apply(const float *grad, const uint32_t *hu, float *m, float *v, float *y, uint64_t n_total,
                       uint32_t n_dim, float fused, float epsc, float omb1, float omb2, cudaStream_t s);
void launch_schedule(const float *eps, float *cursor, uint64_t ne, uint32_t epoch, cudaStream_t s);
void launch_eval_pow(const float *x, uint32_t n, float b, bool precise, float *out, cudaStream_t s);
// GB/s (8 bytes per gather) of random float2 gathers from an L2-resident
// table of table_bytes, best of five timed launches.
float probe_l2_gather(uint64_t table_bytes, cudaStream_t s);
void launch_sample(uint32_t sampler, uint64_t seed, uint32_t node, uint32_t entry, uint32_t epoch,
                   uint32_t edge_local, uint32_t count, uint32_t n, uint32_t *out, cudaStream_t s);

}  // namespace umapcu
