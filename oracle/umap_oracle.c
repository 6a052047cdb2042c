/*
 * umap_oracle.c -- CPU restatement of manifolds-rs's UMAP hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the parity checker: only the test
 * suite, the smoke check and the CPU-baseline leg of the benchmark load it.
 * The product path (the CUDA library) never links, calls or falls back to it.
 *
 * Every function restates one reference function in the same operation order
 * and the same floating-point types (T = f32 where the reference runs the GPU
 * path in f32, f64 where the reference widens). Build with
 * -ffp-contract=off: Rust never contracts a*b+c into an FMA, so neither may
 * this file. glibc's expf/powf/logf/sqrtf are what Rust's f32 methods call on
 * Linux, so transcendental results agree bit for bit on the same host.
 *
 * Parity pin: the reference (Rust + cubecl) cannot be built here (no Rust
 * toolchain, crates not vendored). The restatement is pinned to the
 * known-answer tests the reference itself holds (tests/test_oracle_golden.py
 * lists each with its file:line).
 *
 * Stand-ins (documented, parity unpinned by the reference itself):
 *  - rand 0.9 SmallRng (Xoshiro256++ seeded by SplitMix64) is restated from
 *    the published Xoshiro256++ / SplitMix64 algorithms (Blackman & Vigna);
 *    range reduction uses Lemire's multiply-high, not rand's exact sampler.
 *    Only the CPU optimisers (adam_parallel / adam / sgd) use it.
 */
#include <math.h>
#include <float.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_NO_DATA 1
#define ORC_NO_GRAPH_EDGES 2
#define ORC_DEGENERATE_LOCAL_RADII 3
#define ORC_BAD_ARG 7

/* umap_optimiser_gpu.rs:58-70 */
#define GRAD_CLIP_VAL 4.0f
#define GRAD_REP_EPS 0.001f
#define GRAD_DIST_SQ_THRESHOLD 1e-8f
/* density.rs:38 */
#define DENS_EPS 1e-8

/* ------------------------------------------------------------------ */
/* Graph construction                                                   */
/* ------------------------------------------------------------------ */

/* graph.rs:107-125 local_connectivity_distance */
float orc_local_connectivity_distance(const float *dists, uint32_t k, float lc)
{
    if (lc <= 0.0f || k == 0) return 0.0f;
    float offset = fmaxf(lc - 1.0f, 0.0f);
    float whole = floorf(offset);
    float fraction = offset - whole;
    uint64_t idx;
    if (!(whole >= 0.0f) || whole >= 1.8e19f) idx = UINT64_MAX; else idx = (uint64_t)whole;
    if (idx > (uint64_t)(k - 1)) idx = k - 1;
    if (fraction > 0.0f && idx + 1 < k)
        return dists[idx] * (1.0f - fraction) + dists[idx + 1] * fraction;
    return dists[idx];
}

/* The exp of the graph stage (smooth_knn_dist, knn_to_coo). 0 (default):
 * glibc's expf, what the reference's f32::exp calls. 1: exp rounded from
 * double, (float)exp((double)x) -- the device's form; a test switches to it
 * only to attribute a difference from the device to the last bit of expf
 * (glibc's expf and the correctly rounded exp differ for about 0.06 % of
 * arguments). */
static int orc_exp_mode = 0;

void orc_set_exp_mode(int mode) { orc_exp_mode = mode; }

static inline float orc_graph_exp(float x) { return orc_exp_mode ? (float)exp((double)x) : expf(x); }

/* graph.rs:499-565 smooth_knn_dist. Row length k is the reference's `k`
 * argument (lib.rs:298 passes knn_dist[0].len()). */
void orc_smooth_knn_dist(const float *dist, uint32_t n, uint32_t k, float local_connectivity,
                         float bandwidth, uint32_t n_iter, float *sigmas, float *rhos)
{
    const double target = log((double)k);
    const double tol = (double)bandwidth;
#pragma omp parallel
    {
        float *adjusted = (float *)malloc(sizeof(float) * (k ? k : 1));
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; i++) {
            const float *d = dist + (uint64_t)i * k;
            float rho = orc_local_connectivity_distance(d, k, local_connectivity);
            for (uint32_t t = 0; t < k; t++) adjusted[t] = fmaxf(d[t] - rho, 0.0f);
            float lo = 0.0f, hi = FLT_MAX, mid = 1.0f;
            for (uint32_t it = 0; it < n_iter; it++) {
                float inv_mid = 1.0f / mid;
                float s = -0.0f; /* Rust's f32 Sum folds from -0.0 */
                for (uint32_t t = 0; t < k; t++) s += orc_graph_exp((-adjusted[t]) * inv_mid);
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
            sigmas[i] = mid;
            rhos[i] = rho;
        }
        free(adjusted);
    }
}

/* graph.rs:585-662 knn_to_coo. Returns the number of COO entries; rows in
 * kNN order, self entries skipped. */
uint64_t orc_knn_to_coo(const int32_t *knn_idx, const float *knn_dist, uint32_t n, uint32_t k,
                        const float *sigmas, const float *rhos, uint32_t *row, uint32_t *col,
                        float *val)
{
    uint64_t w = 0;
    for (uint32_t i = 0; i < n; i++) {
        float sigma = sigmas[i], rho = rhos[i];
        int smooth = sigma > 0.0f;
        float inv_sigma = smooth ? 1.0f / sigma : 0.0f;
        for (uint32_t t = 0; t < k; t++) {
            int32_t j = knn_idx[(uint64_t)i * k + t];
            if ((uint32_t)j == i) continue;
            float adjusted = fmaxf(knn_dist[(uint64_t)i * k + t] - rho, 0.0f);
            float weight;
            if (smooth) weight = orc_graph_exp((-adjusted) * inv_sigma);
            else if (adjusted > 0.0f) weight = 0.0f;
            else weight = 1.0f;
            row[w] = i;
            col[w] = (uint32_t)j;
            val[w] = weight;
            w++;
        }
    }
    return w;
}

typedef struct { uint32_t c; float w; uint64_t ord; } orc_ent;

/* stable insertion sort by column; rows are short (k to a few hundred) */
static void orc_sort_row(orc_ent *e, uint64_t len)
{
    for (uint64_t a = 1; a < len; a++) {
        orc_ent x = e[a];
        uint64_t b = a;
        while (b > 0 && e[b - 1].c > x.c) { e[b] = e[b - 1]; b--; }
        e[b] = x;
    }
}

/* graph.rs:185-468 (coo_to_sorted_csr, transpose_csr, merge_row,
 * symmetrise_csr) with the fuzzy-union kernel of graph.rs:684-694.
 * Duplicate columns within a row collapse to the last occurrence in input
 * order (the reference's sort_unstable leaves that order unspecified).
 * Output: grouped by row, column ascending. Capacity of the outputs must be
 * at least 2*nnz. Returns the output entry count. */
uint64_t orc_symmetrise(uint32_t n, uint64_t nnz, const uint32_t *row, const uint32_t *col,
                        const float *val, float mix_weight, uint32_t *orow, uint32_t *ocol,
                        float *oval)
{
    if (n == 0 || nnz == 0) return 0;
    const float directed_weight = 1.0f - mix_weight;
    uint64_t *indptr = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    for (uint64_t e = 0; e < nnz; e++) indptr[row[e] + 1]++;
    for (uint32_t i = 0; i < n; i++) indptr[i + 1] += indptr[i];
    orc_ent *out = (orc_ent *)malloc(sizeof(orc_ent) * nnz);
    uint64_t *cur = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)n + 1));
    memcpy(cur, indptr, sizeof(uint64_t) * n);
    for (uint64_t e = 0; e < nnz; e++) {
        orc_ent x = {col[e], val[e], e};
        out[cur[row[e]]++] = x;
    }
    for (uint32_t i = 0; i < n; i++) orc_sort_row(out + indptr[i], indptr[i + 1] - indptr[i]);
    /* transpose (graph.rs:236-263): rows visited ascending, so each output
     * row comes out sorted by source */
    uint64_t *tptr = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    for (uint64_t e = 0; e < nnz; e++) tptr[out[e].c + 1]++;
    for (uint32_t i = 0; i < n; i++) tptr[i + 1] += tptr[i];
    orc_ent *in = (orc_ent *)malloc(sizeof(orc_ent) * nnz);
    memcpy(cur, tptr, sizeof(uint64_t) * n);
    for (uint32_t r = 0; r < n; r++)
        for (uint64_t e = indptr[r]; e < indptr[r + 1]; e++) {
            orc_ent x = {r, out[e].w, out[e].ord};
            in[cur[out[e].c]++] = x;
        }
    /* merge_row (graph.rs:321-363) */
    uint64_t w = 0;
    for (uint32_t i = 0; i < n; i++) {
        uint64_t ia = indptr[i], ea = indptr[i + 1], ib = tptr[i], eb = tptr[i + 1];
        while (ia < ea || ib < eb) {
            uint32_t c;
            if (ia < ea && ib < eb) c = out[ia].c < in[ib].c ? out[ia].c : in[ib].c;
            else if (ia < ea) c = out[ia].c;
            else c = in[ib].c;
            float w_ij = 0.0f, w_ji = 0.0f;
            while (ia < ea && out[ia].c == c) { w_ij = out[ia].w; ia++; }
            while (ib < eb && in[ib].c == c) { w_ji = in[ib].w; ib++; }
            float uni = (w_ij + w_ji) - w_ij * w_ji;
            float w_sym = mix_weight * uni + directed_weight * w_ij;
            if (w_sym > 0.0f) {
                orow[w] = i;
                ocol[w] = c;
                oval[w] = w_sym;
                w++;
            }
        }
    }
    free(indptr); free(out); free(cur); free(tptr); free(in);
    return w;
}

/* graph.rs:776-853 filter_weak_edges (order preserving). Returns kept count;
 * outputs may alias the inputs. */
uint64_t orc_filter_weak_edges(uint64_t nnz, const uint32_t *row, const uint32_t *col,
                               const float *val, uint32_t n_epochs, uint32_t *orow,
                               uint32_t *ocol, float *oval)
{
    float max_weight = 0.0f;
    for (uint64_t e = 0; e < nnz; e++) if (val[e] > max_weight) max_weight = val[e];
    float threshold = max_weight / (float)n_epochs;
    uint64_t w = 0;
    for (uint64_t e = 0; e < nnz; e++) {
        float x = val[e];
        if (x >= threshold) {
            uint32_t r = row[e], c = col[e];
            orow[w] = r; ocol[w] = c; oval[w] = x; w++;
        }
    }
    return w;
}

/* ------------------------------------------------------------------ */
/* CSR for the optimiser                                                */
/* ------------------------------------------------------------------ */

/* umap_optimiser_gpu.rs:132-209 UmapCsrGraph::from_graph. The adjacency list
 * is given in CSR form: row i = (adj_col, adj_w)[adj_ptr[i]..adj_ptr[i+1]).
 * Outputs: offsets[n+1], edge_idx[2E], other[2E], eps[E], mu[E] (capacity
 * for E = adj_ptr[n]/1 entries is always enough). */
int orc_csr_from_graph(uint32_t n, const uint64_t *adj_ptr, const uint32_t *adj_col,
                       const float *adj_w, uint32_t *offsets, uint32_t *edge_idx,
                       uint32_t *other, float *eps, float *mu, uint64_t *n_edges_out)
{
    if (n == 0) return ORC_NO_DATA;
    uint32_t *degree = (uint32_t *)calloc(n, sizeof(uint32_t));
    uint64_t ne = 0;
    for (uint32_t i = 0; i < n; i++)
        for (uint64_t p = adj_ptr[i]; p < adj_ptr[i + 1]; p++) {
            uint32_t j = adj_col[p];
            if (i < j) {
                mu[ne] = adj_w[p];
                other[2 * ne] = i; /* stash endpoints temporarily */
                other[2 * ne + 1] = j;
                degree[i]++;
                degree[j]++;
                ne++;
            }
        }
    if (ne == 0) { free(degree); return ORC_NO_GRAPH_EDGES; }
    uint32_t *ends = (uint32_t *)malloc(sizeof(uint32_t) * 2 * ne);
    memcpy(ends, other, sizeof(uint32_t) * 2 * ne);
    offsets[0] = 0;
    for (uint32_t i = 0; i < n; i++) offsets[i + 1] = offsets[i] + degree[i];
    uint32_t *cursor = (uint32_t *)malloc(sizeof(uint32_t) * n);
    memcpy(cursor, offsets, sizeof(uint32_t) * n);
    for (uint64_t e = 0; e < ne; e++) {
        uint32_t i = ends[2 * e], j = ends[2 * e + 1];
        uint32_t pi = cursor[i]++;
        edge_idx[pi] = (uint32_t)e; other[pi] = j;
        uint32_t pj = cursor[j]++;
        edge_idx[pj] = (uint32_t)e; other[pj] = i;
    }
    float max_weight = 0.0f;
    for (uint64_t e = 0; e < ne; e++) if (mu[e] > max_weight) max_weight = mu[e];
    for (uint64_t e = 0; e < ne; e++) {
        float norm = mu[e] / max_weight;
        eps[e] = norm > 0.0f ? 1.0f / norm : 1e8f;
    }
    *n_edges_out = ne;
    free(degree); free(ends); free(cursor);
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* Optimiser parameters                                                 */
/* ------------------------------------------------------------------ */

/* umap_optimisers.rs:139-209 fit_params, T = f32 */
void orc_fit_params_f32(float min_dist, float spread, uint32_t n_iter, float *a_out, float *b_out)
{
    const int n_points = 300;
    float xv[300], yv[300];
    float max_x = spread * 3.0f;
    float step = max_x / (float)(n_points - 1);
    for (int i = 0; i < n_points; i++) {
        float x = step * (float)i;
        float y = x < min_dist ? 1.0f : expf(-(x - min_dist) / spread);
        xv[i] = x; yv[i] = y;
    }
    float a = 1.0f, b = 1.0f;
    for (uint32_t it = 0; it < n_iter; it++) {
        float grad_a = 0.0f, grad_b = 0.0f;
        float n_points_t = (float)n_points;
        for (int i = 0; i < n_points; i++) {
            float x = xv[i];
            if (x <= 0.0f) continue;
            float y_target = yv[i];
            float x_2b = powf(x, 2.0f * b);
            float denom = 1.0f + a * x_2b;
            float pred = 1.0f / denom;
            float err = pred - y_target;
            grad_a += err * (-x_2b / (denom * denom));
            float log_x = logf(x);
            grad_b += err * (-2.0f * a * x_2b * log_x / (denom * denom));
        }
        grad_a /= n_points_t;
        grad_b /= n_points_t;
        a -= 1.0f * grad_a;
        b -= 1.0f * grad_b;
        a = fminf(fmaxf(a, 0.001f), 10.0f);
        b = fminf(fmaxf(b, 0.1f), 2.0f);
    }
    *a_out = a; *b_out = b;
}

/* umap_optimisers.rs:139-209 fit_params, T = f64 */
void orc_fit_params_f64(double min_dist, double spread, uint32_t n_iter, double *a_out, double *b_out)
{
    const int n_points = 300;
    double xv[300], yv[300];
    double max_x = spread * 3.0;
    double step = max_x / (double)(n_points - 1);
    for (int i = 0; i < n_points; i++) {
        double x = step * (double)i;
        double y = x < min_dist ? 1.0 : exp(-(x - min_dist) / spread);
        xv[i] = x; yv[i] = y;
    }
    double a = 1.0, b = 1.0;
    for (uint32_t it = 0; it < n_iter; it++) {
        double grad_a = 0.0, grad_b = 0.0;
        double n_points_t = (double)n_points;
        for (int i = 0; i < n_points; i++) {
            double x = xv[i];
            if (x <= 0.0) continue;
            double y_target = yv[i];
            double x_2b = pow(x, 2.0 * b);
            double denom = 1.0 + a * x_2b;
            double pred = 1.0 / denom;
            double err = pred - y_target;
            grad_a += err * (-x_2b / (denom * denom));
            double log_x = log(x);
            grad_b += err * (-2.0 * a * x_2b * log_x / (denom * denom));
        }
        grad_a /= n_points_t;
        grad_b /= n_points_t;
        a -= 1.0 * grad_a;
        b -= 1.0 * grad_b;
        a = fmin(fmax(a, 0.001), 10.0);
        b = fmin(fmax(b, 0.1), 2.0);
    }
    *a_out = a; *b_out = b;
}

/* umap_optimiser_gpu.rs:1155-1196 (host scalars of launch_adam_update):
 * returns the fused lr_alpha * ad_scale and epsc for one epoch. */
void orc_adam_epoch_scalars(float lr, float beta1, float beta2, float eps, uint32_t epoch,
                            uint32_t n_epochs, float *fused, float *epsc)
{
    float lr_alpha = lr * (1.0f - (float)epoch / (float)n_epochs);
    float t = (float)(epoch + 1);
    float beta1t = powf(beta1, t);
    float beta2t = powf(beta2, t);
    float sqrt_b2t1 = sqrtf(1.0f - beta2t);
    float ad_scale = sqrt_b2t1 / (1.0f - beta1t);
    *epsc = sqrt_b2t1 * eps;
    *fused = lr_alpha * ad_scale;
}

/* ------------------------------------------------------------------ */
/* adam_gpu kernels, restated from the reference's CPU mirrors          */
/* ------------------------------------------------------------------ */

/* umap_optimiser_gpu.rs:611-624 / 1379-1391 */
uint32_t orc_hash_neg(uint32_t seed, uint32_t node, uint32_t epoch, uint32_t edge_local,
                      uint32_t neg, uint32_t n)
{
    uint32_t h = seed ^ (node * 0x9E3779B1u) ^ (epoch * 0x85EBCA77u) ^
                 (edge_local * 0xC2B2AE3Du) ^ (neg * 0x27D4EB2Fu);
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return h % n;
}

/* Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11), the counter-based
 * sampler the CUDA library offers as its alternative negative sampler.
 * Counter (entry, epoch, block, 0), key (seed lo, seed hi). */
void orc_philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

uint32_t orc_philox_neg(uint64_t seed, uint32_t entry, uint32_t epoch, uint32_t neg, uint32_t n)
{
    uint32_t c[4] = {entry, epoch, neg >> 2, 0x554D4150u};
    orc_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    return (uint32_t)(((uint64_t)c[neg & 3] * n) >> 32);
}

#define ORC_SAMPLER_HASH 0
#define ORC_SAMPLER_PHILOX 1

/* umap_optimiser_gpu.rs:1409-1453 cpu_dens_radii (== kernel :487-544) */
void orc_dens_radii(const float *embd, uint32_t n, uint32_t n_dim, const uint32_t *offsets,
                    const uint32_t *other, float a, float b, float *re, float *phi_sum)
{
    const float dens_eps = (float)DENS_EPS;
    for (uint32_t node = 0; node < n; node++) {
        uint64_t base_self = (uint64_t)node * n_dim;
        float sum_sq = 0.0f, sum_phi = 0.0f;
        for (uint32_t pos = offsets[node]; pos < offsets[node + 1]; pos++) {
            uint64_t base_other = (uint64_t)other[pos] * n_dim;
            float dist_sq = 0.0f;
            for (uint32_t d = 0; d < n_dim; d++) {
                float diff = embd[base_self + d] - embd[base_other + d];
                dist_sq += diff * diff;
            }
            float dist_sq_b = powf(dist_sq, b);
            float phi = 1.0f / (1.0f + a * dist_sq_b);
            sum_sq += phi * dist_sq;
            sum_phi += phi;
        }
        re[node] = logf(dens_eps + sum_sq / fmaxf(sum_phi, FLT_EPSILON));
        phi_sum[node] = sum_phi;
    }
}

/* density.rs:464-508 correlation_stats with T = f32 inputs: f64
 * accumulation in fixed 8192-element chunks summed in index order. */
void orc_correlation_stats(const float *re, const float *r, uint64_t n, float var_shift,
                           float *mean_out, float *std_out, float *cov_out)
{
    const uint64_t CH = 8192;
    double denom = (double)((n > 1 ? n - 1 : 0) > 1 ? n - 1 : 1);
    double mean = -0.0;
    for (uint64_t c0 = 0; c0 < n; c0 += CH) {
        uint64_t c1 = c0 + CH < n ? c0 + CH : n;
        double s = 0.0;
        for (uint64_t i = c0; i < c1; i++) s = s + (double)re[i];
        mean = mean + s;
    }
    mean = mean / (double)(n > 1 ? n : 1);
    double ss = 0.0, cross = 0.0;
    for (uint64_t c0 = 0; c0 < n; c0 += CH) {
        uint64_t c1 = c0 + CH < n ? c0 + CH : n;
        double a = 0.0, b = 0.0;
        for (uint64_t i = c0; i < c1; i++) {
            double d = (double)re[i] - mean;
            a = a + d * d;
            b = b + d * (double)r[i];
        }
        ss = ss + a;
        cross = cross + b;
    }
    double var = ss / denom, cov = cross / denom;
    double sd = sqrt(var + (double)var_shift);
    *mean_out = (float)mean;
    *std_out = (float)sd;
    *cov_out = (float)cov;
}

/* umap_optimiser_gpu.rs:1089-1143 launch_dens_update, host half + the
 * umap_dens_weights kernel (:568-586). Returns dens_coeff. */
float orc_dens_weights(const float *r, const float *re, uint32_t n, float var_shift, float lambda,
                       float mu_tot, float *weight)
{
    float re_mean, re_std, cov;
    orc_correlation_stats(re, r, n, var_shift, &re_mean, &re_std, &cov);
    float inv_var = 1.0f / (re_std * re_std);
    for (uint32_t i = 0; i < n; i++) weight[i] = r[i] - cov * (re[i] - re_mean) * inv_var;
    float denom = (float)(n > 1 ? n - 1 : 1);
    return lambda * mu_tot / (re_std * denom);
}

/* umap_optimiser_gpu.rs:1461-1579 cpu_grad_accum (== kernel :682-860), plus
 * the has_update flag the kernel writes (:737-742, :859). Cursor array is
 * per edge. Negative source: sampler (hash / philox) or, when inj != NULL,
 * inj[pos * neg_rate + neg] for CSR entry pos. dens_* may be NULL.
 * abs_sum (test aid, may be NULL): per node and coordinate, the sum of the
 * absolute values of the terms added into the gradient, in f64 -- the scale
 * of the f32 sum's own rounding (a few units of 2^-24 times it). */
static double *orc_grad_abs_sum = NULL;

void orc_set_grad_abs_sum(double *abs_sum) { orc_grad_abs_sum = abs_sum; }

void orc_grad_accum(const float *embd, uint32_t n, uint32_t n_dim, const uint32_t *offsets,
                    const uint32_t *edge_idx, const uint32_t *other, const float *cursor,
                    uint32_t epoch, uint64_t seed, uint32_t sampler, uint32_t neg_rate, float a,
                    float b, float gamma, const float *mu, const float *dens_re,
                    const float *dens_phi_sum, const float *dens_weight, float dens_coeff,
                    const uint32_t *inj, float *grad, uint32_t *has_update)
{
    double *abs_sum = orc_grad_abs_sum;
    const float two = 2.0f, one = 1.0f;
    const float two_a_b = two * a * b;
    const float two_gamma_b = two * gamma * b;
    const float clip_val = GRAD_CLIP_VAL;
    const float epoch_t = (float)epoch;
    const uint32_t seed_u32 = (uint32_t)seed;
    float g[16];
    double ga[16];
#pragma omp parallel for schedule(dynamic, 256) private(g, ga)
    for (int64_t node_s = 0; node_s < (int64_t)n; node_s++) {
        uint32_t node = (uint32_t)node_s;
        uint64_t base_self = (uint64_t)node * n_dim;
        for (uint32_t d = 0; d < n_dim; d++) g[d] = 0.0f;
        for (uint32_t d = 0; d < n_dim; d++) ga[d] = 0.0;
        uint32_t edge_local = 0, active = 0;
        for (uint32_t pos = offsets[node]; pos < offsets[node + 1]; pos++, edge_local++) {
            uint32_t e = edge_idx[pos];
            if (cursor[e] > epoch_t) continue;
            active = 1;
            uint32_t o = other[pos];
            uint64_t base_other = (uint64_t)o * n_dim;
            float dist_sq = 0.0f;
            for (uint32_t d = 0; d < n_dim; d++) {
                float diff = embd[base_self + d] - embd[base_other + d];
                dist_sq += diff * diff;
            }
            if (dist_sq >= GRAD_DIST_SQ_THRESHOLD) {
                float dist_sq_b = powf(dist_sq, b);
                float denom = one + a * dist_sq_b;
                float grad_coeff = two_a_b * dist_sq_b / (dist_sq * denom);
                for (uint32_t d = 0; d < n_dim; d++) {
                    float delta = embd[base_other + d] - embd[base_self + d];
                    g[d] += two * grad_coeff * delta;
                    ga[d] += fabs((double)(two * grad_coeff * delta));
                }
                if (dens_re) {
                    float phi = one / denom;
                    float dphi_term = a * b * dist_sq_b / dist_sq * phi;
                    float common = one - b * (one - phi);
                    float dr_self = (phi / dens_phi_sum[node]) * (common / expf(dens_re[node]) + dphi_term);
                    float dr_other = (phi / dens_phi_sum[o]) * (common / expf(dens_re[o]) + dphi_term);
                    float cor = dens_coeff * (dens_weight[node] * dr_self + dens_weight[o] * dr_other) / mu[e];
                    float two_cor = two * cor;
                    for (uint32_t d = 0; d < n_dim; d++) {
                        float delta = embd[base_self + d] - embd[base_other + d];
                        float gg = two_cor * delta;
                        if (gg > clip_val) gg = clip_val;
                        if (gg < -clip_val) gg = -clip_val;
                        g[d] += two * gg;
                        ga[d] += fabs((double)(two * gg));
                    }
                }
            }
            for (uint32_t neg = 0; neg < neg_rate; neg++) {
                uint32_t k;
                if (inj) k = inj[(uint64_t)pos * neg_rate + neg];
                else if (sampler == ORC_SAMPLER_PHILOX) k = orc_philox_neg(seed, pos, epoch, neg, n);
                else k = orc_hash_neg(seed_u32, node, epoch, edge_local, neg, n);
                if (k == node) continue;
                uint64_t base_k = (uint64_t)k * n_dim;
                float dist_sq_k = 0.0f;
                for (uint32_t d = 0; d < n_dim; d++) {
                    float diff = embd[base_self + d] - embd[base_k + d];
                    dist_sq_k += diff * diff;
                }
                float dist_sq_safe = dist_sq_k + GRAD_REP_EPS;
                float dist_sq_b = powf(dist_sq_safe, b);
                float denom = dist_sq_safe * (one + a * dist_sq_b);
                float grad_coeff = two_gamma_b / denom;
                if (grad_coeff > clip_val) grad_coeff = clip_val;
                if (grad_coeff < -clip_val) grad_coeff = -clip_val;
                for (uint32_t d = 0; d < n_dim; d++) {
                    float delta = embd[base_self + d] - embd[base_k + d];
                    g[d] += grad_coeff * delta;
                    ga[d] += fabs((double)(grad_coeff * delta));
                }
            }
        }
        for (uint32_t d = 0; d < n_dim; d++) grad[base_self + d] = g[d];
        if (abs_sum)
            for (uint32_t d = 0; d < n_dim; d++) abs_sum[base_self + d] = ga[d];
        if (has_update) has_update[node] = active;
    }
}

/* umap_optimiser_gpu.rs:1584-1627 cpu_adam_update (== kernel :887-923) */
void orc_adam_update(const float *node_grad, const uint32_t *has_update, float *m, float *v,
                     float *embd, uint32_t n, uint32_t n_dim, float fused, float epsc,
                     float beta1, float beta2)
{
    const float one_minus_beta1 = 1.0f - beta1;
    const float one_minus_beta2 = 1.0f - beta2;
    for (uint32_t node = 0; node < n; node++) {
        if (has_update[node] == 0) continue;
        for (uint32_t d = 0; d < n_dim; d++) {
            uint64_t i = (uint64_t)node * n_dim + d;
            float g = node_grad[i];
            float m_new = m[i] + one_minus_beta1 * (g - m[i]);
            m[i] = m_new;
            float v_new = v[i] + one_minus_beta2 * (g * g - v[i]);
            v[i] = v_new;
            embd[i] += fused * m_new / (sqrtf(v_new) + epsc);
        }
    }
}

/* umap_optimiser_gpu.rs:940-955 umap_edge_schedule_update */
void orc_schedule_update(const float *eps, float *cursor, uint64_t n_edges, uint32_t epoch)
{
    const float epoch_f = (float)epoch;
    for (uint64_t e = 0; e < n_edges; e++)
        if (cursor[e] <= epoch_f) cursor[e] += eps[e];
}

/* density.rs:244-250 DensState::is_active with T = f32 */
int orc_dens_is_active(float lambda, float frac, uint32_t epoch, uint32_t n_epochs)
{
    if (lambda <= 0.0f || n_epochs == 0) return 0;
    float progress = (float)(epoch + 1) / (float)n_epochs;
    return progress > 1.0f - frac;
}

/* umap_optimiser_gpu.rs:1302-1369 optimise_embedding_adam_gpu, restated
 * over the CPU mirrors: per epoch [densMAP radii -> stats -> weights] ->
 * grad -> Adam -> schedule. embd [n*n_dim] in/out. dens_r may be NULL
 * (plain UMAP). `epochs_to_run` stops early (0 = all). */
int orc_optimise_adam_gpu(float *embd, uint32_t n, uint32_t n_dim, const uint64_t *adj_ptr,
                          const uint32_t *adj_col, const float *adj_w, float a, float b, float lr,
                          float gamma, uint32_t n_epochs, uint32_t neg_rate, float beta1,
                          float beta2, float eps_adam, const float *dens_r, float dens_lambda,
                          float dens_frac, float dens_var_shift, float dens_mu_tot,
                          uint64_t seed, uint32_t sampler, uint32_t epochs_to_run)
{
    if (n == 0) return ORC_NO_DATA;
    uint64_t cap = adj_ptr[n];
    uint32_t *offsets = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)n + 1));
    uint32_t *edge_idx = (uint32_t *)malloc(sizeof(uint32_t) * (2 * cap + 2));
    uint32_t *other = (uint32_t *)malloc(sizeof(uint32_t) * (2 * cap + 2));
    float *eps = (float *)malloc(sizeof(float) * (cap + 1));
    float *mu = (float *)malloc(sizeof(float) * (cap + 1));
    uint64_t ne = 0;
    int st = orc_csr_from_graph(n, adj_ptr, adj_col, adj_w, offsets, edge_idx, other, eps, mu, &ne);
    if (st != ORC_OK) { free(offsets); free(edge_idx); free(other); free(eps); free(mu); return st; }
    float *cursor = (float *)malloc(sizeof(float) * ne);
    memcpy(cursor, eps, sizeof(float) * ne);
    uint64_t nt = (uint64_t)n * n_dim;
    float *m = (float *)calloc(nt, sizeof(float));
    float *v = (float *)calloc(nt, sizeof(float));
    float *grad = (float *)calloc(nt, sizeof(float));
    uint32_t *hu = (uint32_t *)calloc(n, sizeof(uint32_t));
    float *re = NULL, *phi = NULL, *wt = NULL;
    if (dens_r) {
        re = (float *)calloc(n, sizeof(float));
        phi = (float *)calloc(n, sizeof(float));
        wt = (float *)calloc(n, sizeof(float));
    }
    uint32_t last = epochs_to_run ? epochs_to_run : n_epochs;
    for (uint32_t epoch = 0; epoch < last; epoch++) {
        int dens_on = dens_r && orc_dens_is_active(dens_lambda, dens_frac, epoch, n_epochs);
        float coeff = 0.0f;
        if (dens_on) {
            orc_dens_radii(embd, n, n_dim, offsets, other, a, b, re, phi);
            coeff = orc_dens_weights(dens_r, re, n, dens_var_shift, dens_lambda, dens_mu_tot, wt);
        }
        orc_grad_accum(embd, n, n_dim, offsets, edge_idx, other, cursor, epoch, seed, sampler,
                       neg_rate, a, b, gamma, mu, dens_on ? re : NULL, phi, wt, coeff, NULL,
                       grad, hu);
        float fused, epsc;
        orc_adam_epoch_scalars(lr, beta1, beta2, eps_adam, epoch, n_epochs, &fused, &epsc);
        orc_adam_update(grad, hu, m, v, embd, n, n_dim, fused, epsc, beta1, beta2);
        orc_schedule_update(eps, cursor, ne, epoch);
    }
    free(offsets); free(edge_idx); free(other); free(eps); free(mu); free(cursor);
    free(m); free(v); free(grad); free(hu); free(re); free(phi); free(wt);
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* densMAP constant state                                               */
/* ------------------------------------------------------------------ */

/* density.rs:286-334 lookup_knn_dist + edge_distances_from_knn */
void orc_edge_distances_from_knn(uint64_t nnz, const uint32_t *row, const uint32_t *col,
                                 const int32_t *knn_idx, const float *knn_dist, uint32_t k,
                                 int distances_squared, float *out)
{
    for (uint64_t e = 0; e < nnz; e++) {
        uint32_t i = row[e], j = col[e];
        float raw = 0.0f;
        int found = 0;
        for (uint32_t t = 0; t < k && !found; t++)
            if ((uint32_t)knn_idx[(uint64_t)i * k + t] == j) { raw = knn_dist[(uint64_t)i * k + t]; found = 1; }
        for (uint32_t t = 0; t < k && !found; t++)
            if ((uint32_t)knn_idx[(uint64_t)j * k + t] == i) { raw = knn_dist[(uint64_t)j * k + t]; found = 1; }
        out[e] = distances_squared ? raw : raw * raw;
    }
}

/* density.rs:358-398 original_log_radii + :410-438 standardise. T = f32
 * in/out, f64 inside. Returns ORC_OK or ORC_DEGENERATE_LOCAL_RADII. */
int orc_original_log_radii(uint32_t n, uint64_t nnz, const uint32_t *row, const float *val,
                           const float *edge_d_sq, float *r_out, float *mu_sum_out)
{
    if (n == 0) return ORC_NO_DATA;
    double *ro = (double *)calloc(n, sizeof(double));
    double *ms = (double *)calloc(n, sizeof(double));
    for (uint64_t e = 0; e < nnz; e++) {
        double mu = (double)val[e];
        ro[row[e]] += mu * (double)edge_d_sq[e];
        ms[row[e]] += mu;
    }
    for (uint32_t i = 0; i < n; i++) {
        double denom = fmax(ms[i], DBL_EPSILON);
        ro[i] = log(DENS_EPS + ro[i] / denom);
    }
    int st = ORC_OK;
    if (n < 2) st = ORC_DEGENERATE_LOCAL_RADII;
    else {
        double s = -0.0;
        for (uint32_t i = 0; i < n; i++) s += ro[i];
        double mean = s / (double)n;
        double vs = -0.0;
        for (uint32_t i = 0; i < n; i++) { double d = ro[i] - mean; vs += d * d; }
        double var = vs / (double)(n - 1);
        double sd = sqrt(var);
        if (isnan(sd) || sd <= DBL_EPSILON) st = ORC_DEGENERATE_LOCAL_RADII;
        else for (uint32_t i = 0; i < n; i++) ro[i] = (ro[i] - mean) / sd;
    }
    if (st == ORC_OK)
        for (uint32_t i = 0; i < n; i++) { r_out[i] = (float)ro[i]; mu_sum_out[i] = (float)ms[i]; }
    free(ro); free(ms);
    return st;
}

/* density.rs:181-201 DensState::new (mu_tot = f64 fold over mu_sum, cast) */
int orc_dens_state_new(uint32_t n, uint64_t nnz, const uint32_t *row, const uint32_t *col,
                       const float *val, const int32_t *knn_idx, const float *knn_dist,
                       uint32_t k, int distances_squared, float *r_out, float *mu_sum_out,
                       float *mu_tot_out)
{
    float *dsq = (float *)malloc(sizeof(float) * (nnz ? nnz : 1));
    orc_edge_distances_from_knn(nnz, row, col, knn_idx, knn_dist, k, distances_squared, dsq);
    int st = orc_original_log_radii(n, nnz, row, val, dsq, r_out, mu_sum_out);
    free(dsq);
    if (st != ORC_OK) return st;
    double t = 0.0;
    for (uint32_t i = 0; i < n; i++) t = t + (double)mu_sum_out[i];
    *mu_tot_out = (float)t;
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* CPU optimisers (timed baseline + statistical parity)                 */
/* ------------------------------------------------------------------ */

typedef struct { uint64_t s[4]; } orc_rng;

static inline uint64_t orc_rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

/* SplitMix64 seeding of Xoshiro256++ (Blackman & Vigna), the algorithm the
 * reference's SmallRng::seed_from_u64 uses on 64-bit targets */
static void orc_rng_seed(orc_rng *r, uint64_t state)
{
    for (int i = 0; i < 4; i++) {
        state += 0x9E3779B97F4A7C15ull;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        r->s[i] = z ^ (z >> 31);
    }
}

static inline uint64_t orc_rng_next(orc_rng *r)
{
    uint64_t *s = r->s;
    uint64_t result = orc_rotl(s[0] + s[3], 23) + s[0];
    uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t;
    s[3] = orc_rotl(s[3], 45);
    return result;
}

static inline uint64_t orc_rng_range(orc_rng *r, uint64_t n)
{
    return (uint64_t)(((unsigned __int128)orc_rng_next(r) * n) >> 64);
}

/* umap_optimisers.rs:329-397 FastPowLut, T = f32 */
typedef struct { float b, max_val, inv_step; float *table; uint64_t size; } orc_lut;

static void orc_lut_new(orc_lut *l, float b, double max_val, uint64_t size)
{
    l->table = (float *)malloc(sizeof(float) * size);
    float max_t = (float)max_val;
    float step = max_t / (float)(size - 1);
    for (uint64_t i = 0; i < size; i++) l->table[i] = powf(step * (float)i, b);
    l->b = b; l->max_val = max_t; l->inv_step = 1.0f / step; l->size = size;
}

static inline float orc_lut_get(const orc_lut *l, float x)
{
    if (x >= l->max_val) return powf(x, l->b);
    float idx_f = x * l->inv_step;
    uint64_t idx = (idx_f >= 0.0f && idx_f < 1.8e19f) ? (uint64_t)idx_f : 0;
    if (idx >= l->size - 1) return l->table[l->size - 1];
    float rem = idx_f - (float)idx;
    float y0 = l->table[idx], y1 = l->table[idx + 1];
    return y0 + rem * (y1 - y0);
}

static inline uint64_t orc_floor_to_usize(float x)
{
    float f = floorf(x);
    if (!(f >= 0.0f) || f >= 1.8e19f) return 0;
    return (uint64_t)f;
}

/* umap_optimisers.rs:408-610 densMAP helpers, shared by the CPU optimisers */
typedef struct { float *re_acc, *phi_sum, *re, *weight; float coeff; } orc_dens_scratch;

static void orc_accumulate_umap_radii(uint32_t n, uint32_t n_dim, const uint64_t *adj_ptr,
                                      const uint32_t *adj_col, const float *embd, float a,
                                      int mode, float b, const orc_lut *lut,
                                      orc_dens_scratch *sc)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        uint64_t bi = (uint64_t)i * n_dim;
        float sum_sq = 0.0f, sum_phi = 0.0f;
        for (uint64_t p = adj_ptr[i]; p < adj_ptr[i + 1]; p++) {
            uint64_t bo = (uint64_t)adj_col[p] * n_dim;
            float dist_sq = 0.0f;
            for (uint32_t d = 0; d < n_dim; d++) { float diff = embd[bi + d] - embd[bo + d]; dist_sq += diff * diff; }
            float dsb;
            if (mode == 1) dsb = dist_sq;            /* b == 1 */
            else if (mode == 2) dsb = sqrtf(dist_sq); /* b == 0.5 (sgd/adam fast path) */
            else if (mode == 3) dsb = orc_lut_get(lut, dist_sq);
            else dsb = powf(dist_sq, b);
            float phi = 1.0f / (1.0f + a * dsb);
            sum_sq += phi * dist_sq;
            sum_phi += phi;
        }
        sc->re_acc[i] = sum_sq;
        sc->phi_sum[i] = sum_phi;
    }
    const float e8 = (float)DENS_EPS;
    for (uint32_t i = 0; i < n; i++) sc->re[i] = logf(e8 + sc->re_acc[i] / fmaxf(sc->phi_sum[i], FLT_EPSILON));
}

static void orc_update_density_weights(orc_dens_scratch *sc, const float *r, uint32_t n,
                                       float var_shift, float lambda, float mu_tot)
{
    sc->coeff = orc_dens_weights(r, sc->re, n, var_shift, lambda, mu_tot, sc->weight);
}

static inline float orc_density_edge_coeff(uint32_t i, uint32_t o, float mu_edge, float dist_sq,
                                           float dist_sq_b, float denom, float a, float b,
                                           const orc_dens_scratch *sc)
{
    const float floor_ = FLT_EPSILON;
    float phi = 1.0f / denom;
    float dphi_term = a * b * dist_sq_b / dist_sq * phi;
    float common = 1.0f - b * (1.0f - phi);
    float dr_self = (phi / fmaxf(sc->phi_sum[i], floor_)) * (common / expf(sc->re[i]) + dphi_term);
    float dr_other = (phi / fmaxf(sc->phi_sum[o], floor_)) * (common / expf(sc->re[o]) + dphi_term);
    return sc->coeff * (sc->weight[i] * dr_self + sc->weight[o] * dr_other) / fmaxf(mu_edge, floor_);
}

/* umap_optimisers.rs:1170-1492 (file lines 511-833 of the optimiser body):
 * optimise_embedding_adam_parallel. The timed CPU baseline. n_threads = 0
 * uses the OpenMP default. Runs epochs [first_epoch, first_epoch +
 * epochs_to_run) (epochs_to_run = 0: to the end); the edge schedules are
 * first fast-forwarded through the skipped epochs without gradient work, so
 * a bounded window of a run can be timed. *loop_seconds (if not NULL)
 * receives the wall time of the epoch loop alone, the part the reference's
 * timing harness isolates (tests/umap_gpu_bench.rs:217-252). */
int orc_optimise_adam_parallel(float *embd, uint32_t n, uint32_t n_dim, const uint64_t *adj_ptr,
                               const uint32_t *adj_col, const float *adj_w, float a, float b,
                               float lr, float gamma, uint32_t n_epochs, uint32_t neg_rate,
                               float beta1, float beta2, float eps_adam, const float *dens_r,
                               float dens_lambda, float dens_frac, float dens_var_shift,
                               float dens_mu_tot, uint64_t seed, int n_threads,
                               uint32_t first_epoch, uint32_t epochs_to_run, double *loop_seconds)
{
    if (n == 0) return ORC_NO_DATA;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
    const float two = 2.0f;
    const float two_a_b = two * a * b, two_gamma_b = two * gamma * b;
    const float clip_val = 4.0f, rep_eps = 0.001f;
    int b_is_one = fabsf(b - 1.0f) < 1e-10f;
    orc_lut lut;
    orc_lut_new(&lut, b, 25.0, 65536);
    uint64_t cap = adj_ptr[n];
    uint32_t *ei = (uint32_t *)malloc(sizeof(uint32_t) * (cap + 1));
    uint32_t *ej = (uint32_t *)malloc(sizeof(uint32_t) * (cap + 1));
    float *ew = (float *)malloc(sizeof(float) * (cap + 1));
    uint64_t *degree = (uint64_t *)calloc(n, sizeof(uint64_t));
    uint64_t ne = 0;
    for (uint32_t i = 0; i < n; i++)
        for (uint64_t p = adj_ptr[i]; p < adj_ptr[i + 1]; p++)
            if (i < adj_col[p]) { ei[ne] = i; ej[ne] = adj_col[p]; ew[ne] = adj_w[p]; degree[i]++; degree[adj_col[p]]++; ne++; }
    if (ne == 0) { free(ei); free(ej); free(ew); free(degree); free(lut.table); return ORC_NO_GRAPH_EDGES; }
    float max_weight = 0.0f;
    for (uint64_t e = 0; e < ne; e++) if (ew[e] > max_weight) max_weight = ew[e];
    float *eps = (float *)malloc(sizeof(float) * ne), *nxt = (float *)malloc(sizeof(float) * ne);
    float *eps_neg = (float *)malloc(sizeof(float) * ne), *nxt_neg = (float *)malloc(sizeof(float) * ne);
    for (uint64_t e = 0; e < ne; e++) {
        float norm = ew[e] / max_weight;
        eps[e] = norm > 0.0f ? 1.0f / norm : 1e8f;
        nxt[e] = eps[e];
        eps_neg[e] = eps[e] / (float)neg_rate;
        nxt_neg[e] = eps_neg[e];
    }
    uint64_t nt = (uint64_t)n * n_dim;
    float *m = (float *)calloc(nt, sizeof(float)), *v = (float *)calloc(nt, sizeof(float));
    float *grad = (float *)calloc(nt, sizeof(float));
    uint8_t *hu = (uint8_t *)calloc(n, 1);
    uint64_t *off = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)n + 1));
    off[0] = 0;
    for (uint32_t i = 0; i < n; i++) off[i + 1] = off[i] + degree[i];
    uint64_t *ce = (uint64_t *)malloc(sizeof(uint64_t) * 2 * ne);
    uint8_t *cs = (uint8_t *)malloc(2 * ne);
    uint32_t *co = (uint32_t *)malloc(sizeof(uint32_t) * 2 * ne);
    uint64_t *cur = (uint64_t *)malloc(sizeof(uint64_t) * n);
    memcpy(cur, off, sizeof(uint64_t) * n);
    for (uint64_t e = 0; e < ne; e++) {
        uint64_t pi = cur[ei[e]]++; ce[pi] = e; cs[pi] = 1; co[pi] = ej[e];
        uint64_t pj = cur[ej[e]]++; ce[pj] = e; cs[pj] = 0; co[pj] = ei[e];
    }
    orc_rng *rngs = (orc_rng *)malloc(sizeof(orc_rng) * n);
    for (uint32_t i = 0; i < n; i++) orc_rng_seed(&rngs[i], seed + i);
    orc_dens_scratch sc = {0};
    if (dens_r) {
        sc.re_acc = (float *)calloc(n, sizeof(float)); sc.phi_sum = (float *)calloc(n, sizeof(float));
        sc.re = (float *)calloc(n, sizeof(float)); sc.weight = (float *)calloc(n, sizeof(float));
    }
    const float omb1 = 1.0f - beta1, omb2 = 1.0f - beta2;
    uint32_t last = epochs_to_run ? first_epoch + epochs_to_run : n_epochs;
    if (last > n_epochs) last = n_epochs;
    for (uint32_t epoch = 0; epoch < first_epoch && epoch < n_epochs; epoch++) {
        const float epoch_t = (float)epoch;
        for (uint64_t e = 0; e < ne; e++)
            if (nxt[e] <= epoch_t) {
                nxt[e] += eps[e];
                uint64_t nneg = orc_floor_to_usize((epoch_t - nxt_neg[e]) / eps_neg[e]);
                nxt_neg[e] += (float)nneg * eps_neg[e];
            }
    }
#ifdef _OPENMP
    double t_start = omp_get_wtime();
#endif
    for (uint32_t epoch = first_epoch; epoch < last; epoch++) {
        float lrs = lr * (1.0f - (float)epoch / (float)n_epochs);
        float epoch_t = (float)epoch;
        float t = (float)(epoch + 1);
        float sqrt_b2t1 = sqrtf(1.0f - powf(beta2, t));
        float ad_scale = sqrt_b2t1 / (1.0f - powf(beta1, t));
        float epsc = sqrt_b2t1 * eps_adam;
        memset(hu, 0, n);
        const orc_dens_scratch *dctx = NULL;
        if (dens_r && orc_dens_is_active(dens_lambda, dens_frac, epoch, n_epochs)) {
            orc_accumulate_umap_radii(n, n_dim, adj_ptr, adj_col, embd, a, b_is_one ? 1 : 3, b, &lut, &sc);
            orc_update_density_weights(&sc, dens_r, n, dens_var_shift, dens_lambda, dens_mu_tot);
            dctx = &sc;
        }
#pragma omp parallel for schedule(dynamic, 512)
        for (int64_t is = 0; is < (int64_t)n; is++) {
            uint32_t i = (uint32_t)is;
            float *g = grad + (uint64_t)i * n_dim;
            for (uint32_t d = 0; d < n_dim; d++) g[d] = 0.0f;
            int local = 0;
            uint64_t bi = (uint64_t)i * n_dim;
            for (uint64_t p = off[i]; p < off[i + 1]; p++) {
                uint64_t e = ce[p];
                if (nxt[e] > epoch_t) continue;
                local = 1;
                uint32_t o = co[p];
                uint64_t bo = (uint64_t)o * n_dim;
                float dist_sq = 0.0f;
                for (uint32_t d = 0; d < n_dim; d++) { float diff = embd[bi + d] - embd[bo + d]; dist_sq += diff * diff; }
                if (dist_sq >= 1e-8f) {
                    float dsb = b_is_one ? dist_sq : orc_lut_get(&lut, dist_sq);
                    float denom = 1.0f + a * dsb;
                    float gc = two_a_b * dsb / (dist_sq * denom);
                    for (uint32_t d = 0; d < n_dim; d++) { float delta = embd[bo + d] - embd[bi + d]; g[d] += two * gc * delta; }
                    if (dctx) {
                        float cor = orc_density_edge_coeff(i, o, ew[e], dist_sq, dsb, denom, a, b, dctx);
                        float two_cor = two * cor;
                        for (uint32_t d = 0; d < n_dim; d++) {
                            float delta = embd[bi + d] - embd[bo + d];
                            g[d] += two * fminf(fmaxf(two_cor * delta, -clip_val), clip_val);
                        }
                    }
                }
                if (cs[p]) {
                    uint64_t nneg = orc_floor_to_usize((epoch_t - nxt_neg[e]) / eps_neg[e]);
                    for (uint64_t s = 0; s < nneg; s++) {
                        uint64_t k = orc_rng_range(&rngs[i], n);
                        if (k == i) continue;
                        uint64_t bk = k * n_dim;
                        float dsq = 0.0f;
                        for (uint32_t d = 0; d < n_dim; d++) { float diff = embd[bi + d] - embd[bk + d]; dsq += diff * diff; }
                        float safe = dsq + rep_eps;
                        float dsb = b_is_one ? safe : orc_lut_get(&lut, safe);
                        float denom = safe * (1.0f + a * dsb);
                        float gc = fminf(fmaxf(two_gamma_b / denom, -clip_val), clip_val);
                        for (uint32_t d = 0; d < n_dim; d++) { float delta = embd[bi + d] - embd[bk + d]; g[d] += gc * delta; }
                    }
                }
            }
            if (local) hu[i] = 1;
        }
#pragma omp parallel for schedule(static)
        for (int64_t is = 0; is < (int64_t)n; is++) {
            if (!hu[is]) continue;
            for (uint32_t d = 0; d < n_dim; d++) {
                uint64_t x = (uint64_t)is * n_dim + d;
                float gg = grad[x];
                float m_old = m[x];
                m[x] += omb1 * (gg - m_old);
                float v_old = v[x];
                v[x] += omb2 * (gg * gg - v_old);
                embd[x] += lrs * ad_scale * m[x] / (sqrtf(v[x]) + epsc);
            }
        }
#pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < (int64_t)ne; e++) {
            if (nxt[e] <= epoch_t) {
                nxt[e] += eps[e];
                uint64_t nneg = orc_floor_to_usize((epoch_t - nxt_neg[e]) / eps_neg[e]);
                nxt_neg[e] += (float)nneg * eps_neg[e];
            }
        }
    }
#ifdef _OPENMP
    if (loop_seconds) *loop_seconds = omp_get_wtime() - t_start;
#endif
    free(ei); free(ej); free(ew); free(degree); free(eps); free(nxt); free(eps_neg); free(nxt_neg);
    free(m); free(v); free(grad); free(hu); free(off); free(ce); free(cs); free(co); free(cur);
    free(rngs); free(lut.table);
    free(sc.re_acc); free(sc.phi_sum); free(sc.re); free(sc.weight);
    return ORC_OK;
}

static inline float orc_fast_pow(float x, float b, int b_is_one, int b_is_half)
{
    if (b_is_one) return x;
    if (b_is_half) return sqrtf(x);
    return powf(x, b);
}

/* umap_optimisers.rs:653-865 (sgd, algo=0) and :907-1142 (adam, algo=1):
 * the sequential optimisers over the directed adjacency with immediate
 * updates. */
int orc_optimise_sequential(int algo, float *embd, uint32_t n, uint32_t n_dim,
                            const uint64_t *adj_ptr, const uint32_t *adj_col, const float *adj_w,
                            float a, float b, float lr, float gamma, uint32_t n_epochs,
                            uint32_t neg_rate, float beta1, float beta2, float eps_adam,
                            const float *dens_r, float dens_lambda, float dens_frac,
                            float dens_var_shift, float dens_mu_tot, uint64_t seed)
{
    if (n == 0) return ORC_NO_DATA;
    const float two = 2.0f, one = 1.0f, half = 0.5f;
    const float two_a_b = two * a * b, two_gamma_b = two * gamma * b;
    const float clip_val = 4.0f, rep_eps = 0.001f;
    int b_is_one = fabsf(b - one) < 1e-10f;
    int b_is_half = fabsf(b - half) < 1e-10f;
    uint64_t ne = adj_ptr[n];
    if (ne == 0) return ORC_NO_GRAPH_EDGES;
    uint32_t *ei = (uint32_t *)malloc(sizeof(uint32_t) * ne);
    for (uint32_t i = 0; i < n; i++) for (uint64_t p = adj_ptr[i]; p < adj_ptr[i + 1]; p++) ei[p] = i;
    float max_weight = 0.0f;
    for (uint64_t e = 0; e < ne; e++) if (adj_w[e] > max_weight) max_weight = adj_w[e];
    float *eps = (float *)malloc(sizeof(float) * ne), *nxt = (float *)malloc(sizeof(float) * ne);
    float *eps_neg = (float *)malloc(sizeof(float) * ne), *nxt_neg = (float *)malloc(sizeof(float) * ne);
    float nsr = (float)neg_rate;
    for (uint64_t e = 0; e < ne; e++) {
        float norm = adj_w[e] / max_weight;
        eps[e] = norm > 0.0f ? one / norm : 1e8f;
        nxt[e] = eps[e];
        eps_neg[e] = eps[e] / nsr;
        nxt_neg[e] = eps_neg[e];
    }
    uint64_t nt = (uint64_t)n * n_dim;
    float *m = (float *)calloc(nt, sizeof(float)), *v = (float *)calloc(nt, sizeof(float));
    orc_rng *rngs = (orc_rng *)malloc(sizeof(orc_rng) * n);
    for (uint32_t i = 0; i < n; i++) orc_rng_seed(&rngs[i], seed + i);
    orc_dens_scratch sc = {0};
    if (dens_r) {
        sc.re_acc = (float *)calloc(n, sizeof(float)); sc.phi_sum = (float *)calloc(n, sizeof(float));
        sc.re = (float *)calloc(n, sizeof(float)); sc.weight = (float *)calloc(n, sizeof(float));
    }
    const float beta11 = one - beta1, beta21 = one - beta2;
    float beta1t = beta1, beta2t = beta2;
    const float n_epochs_f = (float)n_epochs;
    int pmode = b_is_one ? 1 : (b_is_half ? 2 : 0);
    for (uint32_t epoch = 0; epoch < n_epochs; epoch++) {
        float lrs = lr * (one - (float)epoch / n_epochs_f);
        float sqrt_b2t1 = sqrtf(one - beta2t);
        float ad_scale = lrs * sqrt_b2t1 / (one - beta1t);
        float epsc = sqrt_b2t1 * eps_adam;
        float epoch_t = (float)epoch;
        const orc_dens_scratch *dctx = NULL;
        if (dens_r && orc_dens_is_active(dens_lambda, dens_frac, epoch, n_epochs)) {
            orc_accumulate_umap_radii(n, n_dim, adj_ptr, adj_col, embd, a, pmode, b, NULL, &sc);
            orc_update_density_weights(&sc, dens_r, n, dens_var_shift, dens_lambda, dens_mu_tot);
            dctx = &sc;
        }
        for (uint64_t e = 0; e < ne; e++) {
            if (nxt[e] > epoch_t) continue;
            uint32_t i = ei[e], j = adj_col[e];
            uint64_t bi = (uint64_t)i * n_dim, bj = (uint64_t)j * n_dim;
            float dist_sq = 0.0f;
            for (uint32_t d = 0; d < n_dim; d++) { float diff = embd[bi + d] - embd[bj + d]; dist_sq += diff * diff; }
            if (dist_sq >= 1e-8f) {
                float dsb = orc_fast_pow(dist_sq, b, b_is_one, b_is_half);
                float denom = one + a * dsb;
                float gc = two_a_b * dsb / (dist_sq * denom);
                float two_cor = 0.0f;
                if (dctx) two_cor = two * orc_density_edge_coeff(i, j, adj_w[e], dist_sq, dsb, denom, a, b, dctx);
                for (uint32_t d = 0; d < n_dim; d++) {
                    float delta = embd[bj + d] - embd[bi + d];
                    if (algo == 0) {
                        float gd = fminf(fmaxf(gc * delta, -clip_val), clip_val);
                        if (dctx) gd += fminf(fmaxf(two_cor * -delta, -clip_val), clip_val);
                        embd[bi + d] += gd * lrs;
                        embd[bj + d] -= gd * lrs;
                    } else {
                        float g = gc * delta;
                        if (dctx) g += fminf(fmaxf(two_cor * -delta, -clip_val), clip_val);
                        uint64_t xi = bi + d;
                        float vo = v[xi], mo = m[xi];
                        v[xi] = vo + beta21 * (g * g - vo);
                        m[xi] = mo + beta11 * (g - mo);
                        embd[xi] += ad_scale * m[xi] / (sqrtf(v[xi]) + epsc);
                        uint64_t xj = bj + d;
                        vo = v[xj]; mo = m[xj];
                        v[xj] = vo + beta21 * (g * g - vo);
                        m[xj] = mo + beta11 * (-g - mo);
                        embd[xj] += ad_scale * m[xj] / (sqrtf(v[xj]) + epsc);
                    }
                }
            }
            nxt[e] += eps[e];
            uint64_t nneg = orc_floor_to_usize((epoch_t - nxt_neg[e]) / eps_neg[e]);
            for (uint64_t s = 0; s < nneg; s++) {
                uint64_t k = orc_rng_range(&rngs[i], n);
                if (k == i) continue;
                uint64_t bk = k * n_dim;
                float dsq = 0.0f;
                for (uint32_t d = 0; d < n_dim; d++) { float diff = embd[bi + d] - embd[bk + d]; dsq += diff * diff; }
                float safe = dsq + rep_eps;
                float dsb = orc_fast_pow(safe, b, b_is_one, b_is_half);
                float denom = safe * (one + a * dsb);
                float gc = fminf(fmaxf(two_gamma_b / denom, -clip_val), clip_val);
                for (uint32_t d = 0; d < n_dim; d++) {
                    float delta = embd[bi + d] - embd[bk + d];
                    float g = gc * delta;
                    uint64_t xi = bi + d;
                    if (algo == 0) embd[xi] += g * lrs;
                    else {
                        float vo = v[xi], mo = m[xi];
                        v[xi] = vo + beta21 * (g * g - vo);
                        m[xi] = mo + beta11 * (g - mo);
                        embd[xi] += ad_scale * m[xi] / (sqrtf(v[xi]) + epsc);
                    }
                }
            }
            nxt_neg[e] += (float)nneg * eps_neg[e];
        }
        beta1t *= beta1;
        beta2t *= beta2;
    }
    free(ei); free(eps); free(nxt); free(eps_neg); free(nxt_neg); free(m); free(v); free(rngs);
    free(sc.re_acc); free(sc.phi_sum); free(sc.re); free(sc.weight);
    return ORC_OK;
}

/* Number of active undirected edges per epoch for the adam_gpu schedule
 * (umap_optimiser_gpu.rs:741, :952): out[e] = #{edges with cursor <= e}. */
void orc_active_edges_per_epoch(const float *eps, uint64_t n_edges, uint32_t n_epochs, uint64_t *out)
{
    for (uint32_t e = 0; e < n_epochs; e++) out[e] = 0;
#pragma omp parallel
    {
        uint64_t *loc = (uint64_t *)calloc(n_epochs ? n_epochs : 1, sizeof(uint64_t));
#pragma omp for schedule(static)
        for (int64_t x = 0; x < (int64_t)n_edges; x++) {
            float c = eps[x];
            for (uint32_t e = 0; e < n_epochs; e++)
                if (c <= (float)e) { loc[e]++; c += eps[x]; }
        }
#pragma omp critical
        for (uint32_t e = 0; e < n_epochs; e++) out[e] += loc[e];
        free(loc);
    }
}

/* ------------------------------------------------ exact kNN and ranks
 * The reference's exact search is ann-search-rs 0.5.2's exhaustive index
 * (third-party, not vendored; called from src/data/nearest_neighbours.rs:
 * 313-316 with k + 1, the first result -- self -- dropped at :352-361). Its
 * published algorithm: every point against every query, the k smallest
 * squared Euclidean (or cosine) distances. Restated here with the
 * arithmetic fixed so that results are reproducible bit for bit: each
 * distance is the sequential f32 FMA chain over dimensions in order, ties are
 * broken by the smaller index, self (the query's own row) is excluded. */

static inline int orc_better(float d, uint32_t i, float td, uint32_t ti)
{
    return d < td || (d == td && i < ti);
}

static void orc_unit_rows(const float *x, uint32_t n, uint32_t dim, float *xn)
{
    for (uint32_t i = 0; i < n; i++) {
        const float *r = x + (size_t)i * dim;
        float s = 0.0f;
        for (uint32_t d = 0; d < dim; d++) s = fmaf(r[d], r[d], s);
        const float nrm = sqrtf(s);
        for (uint32_t d = 0; d < dim; d++) xn[(size_t)i * dim + d] = nrm > 0.0f ? r[d] / nrm : 0.0f;
    }
}

static inline float orc_dist(const float *a, const float *b, uint32_t dim, int metric)
{
    float s = 0.0f;
    if (metric == 0) {
        for (uint32_t d = 0; d < dim; d++) {
            const float df = a[d] - b[d];
            s = fmaf(df, df, s);
        }
        return s;
    }
    for (uint32_t d = 0; d < dim; d++) s = fmaf(a[d], b[d], s);
    return 1.0f - s;
}

/* metric 0: squared Euclidean, 1: cosine (1 - <x/|x|, y/|y|>). qidx NULL:
 * queries are rows 0..nq-1. idx/dist [nq * k], ascending. */
int orc_knn_exact(const float *x, uint32_t n, uint32_t dim, const uint32_t *qidx, uint32_t nq, uint32_t k,
                  int metric, uint32_t *idx, float *dist)
{
    if (n == 0) return ORC_NO_DATA;
    if (k == 0 || n <= k) return ORC_BAD_ARG;
    const float *xs = x;
    float *xn = NULL;
    if (metric == 1) {
        xn = (float *)malloc(sizeof(float) * (size_t)n * dim);
        orc_unit_rows(x, n, dim, xn);
        xs = xn;
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t q = 0; q < (int64_t)nq; q++) {
        const uint32_t gq = qidx ? qidx[q] : (uint32_t)q;
        float *ld = dist + (size_t)q * k;
        uint32_t *li = idx + (size_t)q * k;
        for (uint32_t m = 0; m < k; m++) {
            ld[m] = INFINITY;
            li[m] = UINT32_MAX;
        }
        for (uint32_t p = 0; p < n; p++) {
            if (p == gq) continue;
            const float d = orc_dist(xs + (size_t)gq * dim, xs + (size_t)p * dim, dim, metric);
            if (!orc_better(d, p, ld[k - 1], li[k - 1])) continue;
            uint32_t m = k - 1;
            while (m > 0 && orc_better(d, p, ld[m - 1], li[m - 1])) {
                ld[m] = ld[m - 1];
                li[m] = li[m - 1];
                m--;
            }
            ld[m] = d;
            li[m] = p;
        }
    }
    free(xn);
    return ORC_OK;
}

/* counts[q][m] = #{p != query : (d(q,p), p) strictly before (d(q,nbr), nbr)}
 * for nbr = nbr[q][m] -- the 0-based rank of that neighbour. */
int orc_rank_counts(const float *x, uint32_t n, uint32_t dim, const uint32_t *qidx, uint32_t nq,
                    const uint32_t *nbr, uint32_t k, int metric, uint32_t *counts)
{
    const float *xs = x;
    float *xn = NULL;
    if (metric == 1) {
        xn = (float *)malloc(sizeof(float) * (size_t)n * dim);
        orc_unit_rows(x, n, dim, xn);
        xs = xn;
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t q = 0; q < (int64_t)nq; q++) {
        const uint32_t gq = qidx ? qidx[q] : (uint32_t)q;
        float td[64];
        for (uint32_t m = 0; m < k && m < 64; m++) {
            td[m] = orc_dist(xs + (size_t)gq * dim, xs + (size_t)nbr[(size_t)q * k + m] * dim, dim, metric);
            counts[(size_t)q * k + m] = 0;
        }
        for (uint32_t p = 0; p < n; p++) {
            if (p == gq) continue;
            const float d = orc_dist(xs + (size_t)gq * dim, xs + (size_t)p * dim, dim, metric);
            for (uint32_t m = 0; m < k && m < 64; m++)
                counts[(size_t)q * k + m] += orc_better(d, p, td[m], nbr[(size_t)q * k + m]);
        }
    }
    free(xn);
    return ORC_OK;
}
