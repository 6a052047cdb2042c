// Spectral initialisation on the device: the smallest eigenpairs of a sparse
// symmetric matrix by Lanczos with full reorthogonalisation
// (compute_smallest_eigenpairs_lanczos, src/utils/math.rs:401-616), and the
// layout built on them (spectral_layout, src/data/init.rs:986-1004: the
// negative normalised adjacency -D^-1/2 A D^-1/2 per connected component,
// eigenvectors 1..n_comp, centred, scaled to a range, small noise).
//
// Device side: the normalised adjacency (stable row sort, per-row degree
// sums), connected components (label hooking with pointer jumping), CSR SpMV
// in f64, dot products (fixed-order partial sums), the two-pass classical
// Gram-Schmidt against the whole Krylov basis (basis^T w, then w -= basis c,
// twice, in place of the reference's sequential modified Gram-Schmidt; both
// keep the basis orthogonal to rounding), the back-transformation basis * c;
// alpha and beta stay on the device until the recurrence ends. Host side:
// the small tridiagonal eigenproblem (at most 4 k + 30 rows) by cyclic Jacobi
// rotations, the selection, and the placement of several components. The
// components of a graph are solved together: one Lanczos over the
// block-diagonal whole-graph matrix in which every dot product, recurrence
// coefficient, breakdown test and back-transformation is per component, so
// thirty components cost about as many launches as one.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <numeric>
#include <vector>

#include <cub/cub.cuh>

#include "internal.cuh"

namespace umapcu {
namespace {

constexpr int kBlk = 256;

// y = M x, one warp per row, f64
__global__ void k_spmv(uint32_t n, const uint64_t *__restrict__ ptr, const uint32_t *__restrict__ col,
                       const double *__restrict__ val, const double *__restrict__ x, double *__restrict__ y)
{
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= n) return;
    double acc = 0.0;
    for (uint64_t p = ptr[row] + lane; p < ptr[row + 1]; p += 32) acc += val[p] * x[col[p]];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xFFFFFFFFu, acc, o);
    if (lane == 0) y[row] = acc;
}

// Partial dot products for long vectors: block (b, j) sums a grid-strided
// share of <V_j, w> into part[j * P + b]; k_sum_parts adds each row's P
// partials in order (fixed order: deterministic).
constexpr unsigned kParts = 64;

__global__ void k_basis_dots_part(const double *__restrict__ V, uint32_t n, const double *__restrict__ w,
                                  double *__restrict__ part)
{
    __shared__ double sh[kBlk];
    const uint32_t j = blockIdx.y, b = blockIdx.x;
    const double *v = V + (size_t)j * n;
    double acc = 0.0;
    for (uint32_t i = b * kBlk + threadIdx.x; i < n; i += kParts * kBlk) acc += v[i] * w[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kBlk / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(size_t)j * kParts + b] = sh[0];
}

__global__ void k_sum_parts(const double *__restrict__ part, uint32_t m, double *__restrict__ out)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    double acc = 0.0;
    for (uint32_t b = 0; b < kParts; b++) acc += part[(size_t)j * kParts + b];
    out[j] = acc;
}

// w -= sum_j c_j V_j (sub) or out = sum_j c_j V_j (!sub)
__global__ void k_basis_comb(const double *__restrict__ V, uint32_t n, uint32_t m, const double *__restrict__ c,
                             double *__restrict__ w, bool sub)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc = 0.0;
    for (uint32_t j = 0; j < m; j++) acc += c[j] * V[(size_t)j * n + i];
    w[i] = sub ? w[i] - acc : acc;
}


// dst = x / sqrt(*sq) (x unchanged when the norm is zero)
__global__ void k_scale_by(const double *__restrict__ x, uint32_t n, const double *__restrict__ sq,
                           double *__restrict__ dst)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double nr = sqrt(*sq);
    dst[i] = nr > 0.0 ? x[i] / nr : x[i];
}

// c [0..j] = (0, ..., beta_{j-1}, alpha_j) from ab (alpha_i = ab[2i],
// beta_i^2 = ab[2i + 1])
__global__ void k_recurrence_coef(const double *__restrict__ ab, uint32_t j, double *__restrict__ c)
{
    for (uint32_t i = threadIdx.x; i <= j; i += blockDim.x)
        c[i] = i == j ? ab[2 * j] : (i + 1 == j ? sqrt(ab[2 * i + 1]) : 0.0);
}

// Start vector: uniform in [-0.5, 0.5) from a counter-based SplitMix64
// stream keyed by the seed (the reference draws it from StdRng; any start
// vector with a component along the wanted eigenvectors converges to them).
__global__ void k_random_start(double *__restrict__ v, uint32_t n, uint64_t seed)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    v[i] = (double)(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;
}

// Symmetric eigen-decomposition of a small dense matrix by cyclic Jacobi
// rotations (Golub & Van Loan, Matrix Computations, section 8.5):
// a [m * m] is destroyed; evals [m], evecs [m * m] column-major (column k is
// the eigenvector of evals[k]).
void jacobi_eigen(std::vector<double> &a, uint32_t m, std::vector<double> &evals, std::vector<double> &evecs)
{
    evecs.assign((size_t)m * m, 0.0);
    for (uint32_t i = 0; i < m; i++) evecs[(size_t)i * m + i] = 1.0;
    auto A = [&](uint32_t r, uint32_t c) -> double & { return a[(size_t)r * m + c]; };
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, tot = 0.0;
        for (uint32_t r = 0; r < m; r++)
            for (uint32_t c = 0; c < m; c++) {
                tot += A(r, c) * A(r, c);
                if (r != c) off += A(r, c) * A(r, c);
            }
        if (off <= 1e-30 * (tot > 0 ? tot : 1.0)) break;
        for (uint32_t p = 0; p + 1 < m; p++)
            for (uint32_t q = p + 1; q < m; q++) {
                const double apq = A(p, q);
                if (std::fabs(apq) < 1e-300) continue;
                const double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (uint32_t k = 0; k < m; k++) {  // A := A J (columns p, q)
                    const double akp = A(k, p), akq = A(k, q);
                    A(k, p) = c * akp - s * akq;
                    A(k, q) = s * akp + c * akq;
                }
                for (uint32_t k = 0; k < m; k++) {  // A := J^T A (rows p, q)
                    const double apk = A(p, k), aqk = A(q, k);
                    A(p, k) = c * apk - s * aqk;
                    A(q, k) = s * apk + c * aqk;
                }
                for (uint32_t k = 0; k < m; k++) {  // V := V J
                    double &vp = evecs[(size_t)p * m + k], &vq = evecs[(size_t)q * m + k];
                    const double x = vp, y = vq;
                    vp = c * x - s * y;
                    vq = s * x + c * y;
                }
            }
    }
    evals.resize(m);
    for (uint32_t i = 0; i < m; i++) evals[i] = A(i, i);
}

// out[j] = <V_j, w> for j < m
void basis_dots(const double *V, uint32_t n, uint32_t m, const double *w, double *part, double *out, cudaStream_t s)
{
    k_basis_dots_part<<<dim3(kParts, m), kBlk, 0, s>>>(V, n, w, part);
    k_sum_parts<<<ceil_div(m, 128), 128, 0, s>>>(part, m, out);
    check_launch("basis dots");
}


}  // namespace

// Smallest n_components eigenpairs of a symmetric CSR matrix (f64 values) on
// the device: compute_smallest_eigenpairs_lanczos (src/utils/math.rs:401-616)
// -- min(4 n_components + 30, n) Lanczos steps, early stop when beta < 1e-12,
// the tridiagonal problem on the host, Ritz values ascending, Ritz vectors
// back-transformed through the basis and normalised. evals [k], evecs
// [n * k] (row i = point i, the reference's transposed output); k <=
// n_components (fewer after an early breakdown, as in the reference).
void smallest_eigenpairs_dev(uint32_t n, const uint64_t *d_ptr, const uint32_t *d_col, const double *d_val,
                             uint32_t n_components, uint64_t seed, std::vector<float> &evals,
                             std::vector<float> &evecs, uint32_t &k_out, cudaStream_t s)
{
    if (n == 0) fail(UMAPCU_NO_DATA, "eigenpairs of an empty matrix");
    const uint32_t n_iter = std::min<uint32_t>(n_components * 4 + 30, n);
    // The recurrence runs without host round trips: alpha_j and beta_j stay
    // in device memory (ab[2j], ab[2j + 1] = beta_j^2) and are read back once
    // at the end; a breakdown (beta < 1e-12) truncates the steps there, so
    // whatever the later steps computed is discarded.
    DevBuf<double> V((size_t)n_iter * n, s), w(n, s), c(n_iter, s), ab(2 * (size_t)n_iter + 2, s),
        part((size_t)n_iter * kParts, s);
    const unsigned g = ceil_div(n, kBlk);
    k_random_start<<<g, kBlk, 0, s>>>(V.p, n, seed);
    basis_dots(V.p, n, 1, V.p, part.p, ab.p + 2 * n_iter, s);  // |v0|^2
    k_scale_by<<<g, kBlk, 0, s>>>(V.p, n, ab.p + 2 * n_iter, V.p);
    check_launch("start vector");
    for (uint32_t j = 0; j < n_iter; j++) {
        double *vj = V.p + (size_t)j * n;
        k_spmv<<<ceil_div((uint64_t)n * 32, kBlk), kBlk, 0, s>>>(n, d_ptr, d_col, d_val, vj, w.p);
        basis_dots(vj, n, 1, w.p, part.p, ab.p + 2 * j, s);  // alpha_j
        // w -= alpha_j v_j + beta_{j-1} v_{j-1}
        k_recurrence_coef<<<1, 32, 0, s>>>(ab.p, j, c.p);
        k_basis_comb<<<g, kBlk, 0, s>>>(V.p, n, j + 1, c.p, w.p, true);
        // full reorthogonalisation: two classical Gram-Schmidt passes
        for (int pass = 0; pass < 2; pass++) {
            basis_dots(V.p, n, j + 1, w.p, part.p, c.p, s);
            k_basis_comb<<<g, kBlk, 0, s>>>(V.p, n, j + 1, c.p, w.p, true);
        }
        basis_dots(w.p, n, 1, w.p, part.p, ab.p + 2 * j + 1, s);  // beta_j^2
        if (j + 1 < n_iter) k_scale_by<<<g, kBlk, 0, s>>>(w.p, n, ab.p + 2 * j + 1, V.p + (size_t)(j + 1) * n);
        check_launch("lanczos step");
    }
    std::vector<double> hab(2 * (size_t)n_iter);
    d2h(hab.data(), ab.p, 2 * (size_t)n_iter, s);
    sync(s);
    std::vector<double> alpha, beta;
    uint32_t n_done = 0;
    for (uint32_t j = 0; j < n_iter; j++) {
        alpha.push_back(hab[2 * j]);
        beta.push_back(std::sqrt(std::max(0.0, hab[2 * j + 1])));
        n_done = j + 1;
        if (beta.back() < 1e-12) break;
    }
    const uint32_t m = n_done;
    std::vector<double> T((size_t)m * m, 0.0), tev, tvec;
    for (uint32_t i = 0; i < m; i++) {
        T[(size_t)i * m + i] = alpha[i];
        if (i + 1 < m) T[(size_t)i * m + i + 1] = T[(size_t)(i + 1) * m + i] = beta[i];
    }
    jacobi_eigen(T, m, tev, tvec);
    std::vector<uint32_t> order(m);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return tev[x] < tev[y]; });
    const uint32_t k = std::min(n_components, m);
    evals.resize(k);
    evecs.assign((size_t)n * k, 0.0f);
    std::vector<double> hv(n);
    for (uint32_t q = 0; q < k; q++) {
        const uint32_t idx = order[q];
        h2d(c.p, tvec.data() + (size_t)idx * m, m, s);
        k_basis_comb<<<g, kBlk, 0, s>>>(V.p, n, m, c.p, w.p, false);
        check_launch("k_basis_comb");
        d2h(hv.data(), w.p, n, s);
        sync(s);
        double nrm = 0.0;
        for (double x : hv) nrm += x * x;
        nrm = std::sqrt(nrm);
        for (uint32_t i = 0; i < n; i++) evecs[(size_t)i * k + q] = (float)(nrm > 0 ? hv[i] / nrm : hv[i]);
        evals[q] = (float)tev[idx];
    }
    k_out = k;
}

namespace {

__global__ void k_iota(uint32_t *__restrict__ v, uint64_t m)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) v[i] = (uint32_t)i;
}

__global__ void k_row_count(const uint32_t *__restrict__ row, uint64_t m, unsigned long long *__restrict__ cnt)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) atomicAdd(&cnt[row[i]], 1ull);
}

// CSR (input order within rows) gathered through the stable row sort
__global__ void k_csr_gather(const uint32_t *__restrict__ perm, uint64_t m, const uint32_t *__restrict__ col,
                             const float *__restrict__ w, uint32_t *__restrict__ ccol, double *__restrict__ cw)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t e = perm[i];
    ccol[i] = col[e];
    cw[i] = (double)w[e];
}

// D^-1/2 from the row sums (self loops included), per row in CSR order
__global__ void k_deg_inv_sqrt(uint32_t n, const uint64_t *__restrict__ ptr, const double *__restrict__ cw,
                               double *__restrict__ dis)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = 0.0;
    for (uint64_t p = ptr[i]; p < ptr[i + 1]; p++) d += cw[p];
    dis[i] = d > 1e-8 ? 1.0 / sqrt(d) : 0.0;
}

// values -D^-1/2 w D^-1/2, self loops zero (the matrix has none)
__global__ void k_neg_norm_values(uint32_t n, const uint64_t *__restrict__ ptr, const uint32_t *__restrict__ ccol,
                                  const double *__restrict__ dis, double *__restrict__ cw)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (uint64_t p = ptr[i]; p < ptr[i + 1]; p++) {
        const uint32_t j = ccol[p];
        cw[p] = i == j ? 0.0 : -dis[i] * cw[p] * dis[j];
    }
}

// ---- batched Lanczos: every component's recurrence advances together.
// The normalised adjacency of the whole graph is block-diagonal (no edge
// crosses components), so one SpMV serves all of them; the per-component
// dot products run over each component's member list (mem[seg[s] ..
// seg[s + 1]]) as fixed-order partial sums; sidx[g] is point g's segment
// (~0: not solved, its vector entries stay zero).
// Per-component dot products over the whole index space: every component
// (segment) is cut into chunks of at most kSegChunk of its members, one block
// per (chunk, row); a segment's chunks are consecutive work items
// [pofs[s], pofs[s + 1]) and are summed in order, so the result does not
// depend on scheduling.
constexpr uint32_t kSegChunk = 4096;

// part[r * n_items + t] = <V_r, w> over work item t's members
__global__ void k_seg_dots_part(const double *__restrict__ V, uint64_t n, const double *__restrict__ w,
                                const uint32_t *__restrict__ mem, const uint32_t *__restrict__ item_beg,
                                const uint32_t *__restrict__ item_end, uint32_t n_items, double *__restrict__ part)
{
    __shared__ double sh[kBlk];
    const uint32_t t = blockIdx.x, r = blockIdx.y;
    const double *v = V + (size_t)r * n;
    double acc = 0.0;
    for (uint32_t i = item_beg[t] + threadIdx.x; i < item_end[t]; i += kBlk) {
        const uint32_t g = mem[i];
        acc += v[g] * w[g];
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int h = kBlk / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(size_t)r * n_items + t] = sh[0];
}

// out[r * S + s] = sum of segment s's work items of row r, in order
__global__ void k_seg_sum_parts(const double *__restrict__ part, uint32_t n_items, const uint32_t *__restrict__ pofs,
                                uint32_t S, uint32_t rows, double *__restrict__ out)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint64_t)rows * S) return;
    const uint32_t r = (uint32_t)(t / S), sg = (uint32_t)(t - (uint64_t)r * S);
    double acc = 0.0;
    for (uint32_t q = pofs[sg]; q < pofs[sg + 1]; q++) acc += part[(size_t)r * n_items + q];
    out[t] = acc;
}

// w[g] -= sum_{r < m} c[r * S + s] V_r[g] (sub), or w[g] = that sum, for the
// points of solved segments
__global__ void k_seg_comb(const double *__restrict__ V, uint64_t n, uint32_t m, const double *__restrict__ c,
                           uint32_t S, const uint32_t *__restrict__ sidx, double *__restrict__ w, bool sub)
{
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t sg = sidx[g];
    if (sg == ~0u) return;
    double acc = 0.0;
    for (uint32_t r = 0; r < m; r++) acc += c[(size_t)r * S + sg] * V[(size_t)r * n + g];
    w[g] = sub ? w[g] - acc : acc;
}

// recurrence coefficients of step j: c[r][s] = alpha_j(s) at r = j,
// beta_{j-1}(s) at r = j - 1, else 0; ab = [step][2][S] (alpha, beta^2)
__global__ void k_seg_recurrence(const double *__restrict__ ab, uint32_t j, uint32_t S, double *__restrict__ c)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (j + 1) * S) return;
    const uint32_t r = t / S, sg = t - r * S;
    double v = 0.0;
    if (r == j) v = ab[((size_t)j * 2) * S + sg];
    else if (r + 1 == j) v = sqrt(ab[((size_t)r * 2 + 1) * S + sg]);
    c[t] = v;
}

// v_{j+1}[g] = w[g] / beta_j(s) while segment s still steps (j + 1 < its
// step count and no breakdown so far), else 0
__global__ void k_seg_next(const double *__restrict__ w, uint64_t n, const uint32_t *__restrict__ sidx,
                           const double *__restrict__ ab, uint32_t j, uint32_t S, const uint32_t *__restrict__ iters,
                           double *__restrict__ vnext)
{
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t sg = sidx[g];
    if (sg == ~0u) return;
    bool live = j + 1 < iters[sg];
    for (uint32_t r = 0; live && r <= j; r++) live = sqrt(ab[((size_t)r * 2 + 1) * S + sg]) >= 1e-12;
    vnext[g] = live ? w[g] / sqrt(ab[((size_t)j * 2 + 1) * S + sg]) : 0.0;
}

// start vectors: point g with local index l in component `label` gets the
// same value k_random_start gives index l under seed + label; then scaled by
// its segment's norm (sq = squared norms per segment)
__global__ void k_seg_start(uint64_t n, const uint32_t *__restrict__ sidx, const uint32_t *__restrict__ lidx,
                            const uint32_t *__restrict__ seg_label, uint64_t seed, double *__restrict__ v)
{
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t sg = sidx[g];
    if (sg == ~0u) {
        v[g] = 0.0;
        return;
    }
    uint64_t z = (seed + seg_label[sg]) + 0x9E3779B97F4A7C15ull * (uint64_t)(lidx[g] + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    v[g] = (double)(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;
}

__global__ void k_seg_scale(double *__restrict__ v, uint64_t n, const uint32_t *__restrict__ sidx,
                            const double *__restrict__ sq)
{
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t sg = sidx[g];
    if (sg == ~0u) return;
    const double nr = sqrt(sq[sg]);
    if (nr > 0.0) v[g] /= nr;
}

// -D^-1/2 A D^-1/2 of a COO graph on n nodes (graph_to_negative_normalised_
// adjacency, src/data/init.rs:210-256) built on the device: degrees include
// self loops, self-loop entries carry 0 (the reference drops them), CSR rows
// keep the input order (stable sort by row). Host arrays in, device CSR out.
void neg_normalised_adjacency(uint32_t n, uint64_t nnz, const uint32_t *row, const uint32_t *col, const float *w,
                              DevBuf<uint64_t> &ptr, DevBuf<uint32_t> &cidx, DevBuf<double> &val, cudaStream_t s)
{
    const uint64_t m = nnz ? nnz : 1;
    DevBuf<uint32_t> drow(m, s), dcol(m, s), rs(m, s), perm0(m, s), perm(m, s);
    DevBuf<float> dw(m, s);
    h2d(drow.p, row, nnz, s);
    h2d(dcol.p, col, nnz, s);
    h2d(dw.p, w, nnz, s);
    DevBuf<unsigned long long> cnt(n + 1, s);
    check_cuda(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long) * (n + 1), s), "memset");
    ptr.alloc(n + 1, s);
    cidx.alloc(m, s);
    val.alloc(m, s);
    if (nnz) {
        const unsigned g = ceil_div(nnz, kBlk);
        k_iota<<<g, kBlk, 0, s>>>(perm0.p, nnz);
        size_t tb = 0;
        int bits = 1;
        while (bits < 32 && (1ull << bits) <= n) bits++;
        check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, tb, drow.p, rs.p, perm0.p, perm.p, (int64_t)nnz, 0, bits,
                                                   s), "sort size");
        {
            DevBuf<char> tmp(tb ? tb : 1, s);
            check_cuda(cub::DeviceRadixSort::SortPairs(tmp.p, tb, drow.p, rs.p, perm0.p, perm.p, (int64_t)nnz, 0, bits,
                                                       s), "sort");
        }
        k_row_count<<<g, kBlk, 0, s>>>(drow.p, nnz, cnt.p + 1);
        k_csr_gather<<<g, kBlk, 0, s>>>(perm.p, nnz, dcol.p, dw.p, cidx.p, val.p);
        check_launch("csr gather");
    }
    {
        size_t tb = 0;
        check_cuda(cub::DeviceScan::InclusiveSum(nullptr, tb, cnt.p, (unsigned long long *)ptr.p, (int64_t)(n + 1), s),
                   "scan size");
        DevBuf<char> tmp(tb ? tb : 1, s);
        check_cuda(cub::DeviceScan::InclusiveSum(tmp.p, tb, cnt.p, (unsigned long long *)ptr.p, (int64_t)(n + 1), s),
                   "scan");
    }
    DevBuf<double> dis(n, s);
    k_deg_inv_sqrt<<<ceil_div(n, kBlk), kBlk, 0, s>>>(n, ptr.p, val.p, dis.p);
    k_neg_norm_values<<<ceil_div(n, kBlk), kBlk, 0, s>>>(n, ptr.p, cidx.p, dis.p, val.p);
    check_launch("neg normalised adjacency");
}

// Connected-component labels on the device: every point starts with its own
// index, edges pull both endpoints to the smaller label and labels follow
// their labels' labels until nothing changes; each point ends with the
// smallest index of its component. Host labels out.
__global__ void k_cc_hook(const uint32_t *__restrict__ row, const uint32_t *__restrict__ col, uint64_t m,
                          uint32_t *__restrict__ lab, uint32_t *__restrict__ changed)
{
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const uint32_t a = lab[row[e]], b = lab[col[e]];
    if (a == b) return;
    const uint32_t lo = min(a, b), hi = max(a, b);
    atomicMin(&lab[hi], lo);
    *changed = 1u;
}

__global__ void k_cc_jump(uint32_t *__restrict__ lab, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t l = lab[i];
    while (lab[l] != l) l = lab[l];
    lab[i] = l;
}

void component_labels(uint32_t n, uint64_t nnz, const uint32_t *row, const uint32_t *col,
                      std::vector<uint32_t> &labels, cudaStream_t s)
{
    const uint64_t m = nnz ? nnz : 1;
    DevBuf<uint32_t> drow(m, s), dcol(m, s), lab(n, s), changed(1, s);
    h2d(drow.p, row, nnz, s);
    h2d(dcol.p, col, nnz, s);
    k_iota<<<ceil_div(n, kBlk), kBlk, 0, s>>>(lab.p, n);
    for (uint32_t it = 0; nnz && it < 4096; it++) {
        uint32_t h = 0;
        check_cuda(cudaMemsetAsync(changed.p, 0, sizeof(uint32_t), s), "memset");
        k_cc_hook<<<ceil_div(nnz, kBlk), kBlk, 0, s>>>(drow.p, dcol.p, nnz, lab.p, changed.p);
        k_cc_jump<<<ceil_div(n, kBlk), kBlk, 0, s>>>(lab.p, n);
        check_launch("components");
        d2h(&h, changed.p, 1, s);
        sync(s);
        if (!h) break;
    }
    labels.resize(n);
    d2h(labels.data(), lab.p, n, s);
    sync(s);
}

// Deterministic host stream for the random fallbacks and the noise
// (SplitMix64; the reference's StdRng streams are not reproduced).
struct Mix {
    uint64_t x;
    uint64_t next()
    {
        uint64_t z = (x += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    double normal()  // Box-Muller
    {
        double u1 = uniform(), u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

// single_component_spectral_raw (src/data/init.rs:276-320) for every
// component in `solve` at once (batched Lanczos, see above): raw[c] [n_c *
// n_comp] = eigenvectors 1..n_comp of the component's -D^-1/2 A D^-1/2
// (dimensions Lanczos did not supply: uniform in [-1, 1)), each component
// from its own start vector (seed + label). members[c] ascending.
void batched_component_raw(uint32_t n, const DevBuf<uint64_t> &ptr, const DevBuf<uint32_t> &ci,
                           const DevBuf<double> &val, const std::vector<std::vector<uint32_t>> &members,
                           const std::vector<uint32_t> &solve, uint32_t n_comp, uint64_t seed,
                           std::vector<std::vector<double>> &raw, cudaStream_t s)
{
    const uint32_t S = (uint32_t)solve.size();
    if (!S) return;
    const uint32_t kk = n_comp + 1;
    std::vector<uint32_t> hmem, hsidx(n, ~0u), hlidx(n, 0), hlabel(S), hiters(S), hbeg, hend, hpofs(S + 1, 0);
    uint32_t it_max = 0;
    for (uint32_t q = 0; q < S; q++) {
        const std::vector<uint32_t> &mem = members[solve[q]];
        const uint32_t at = (uint32_t)hmem.size();
        for (uint32_t l = 0; l < mem.size(); l++) {
            hsidx[mem[l]] = q;
            hlidx[mem[l]] = l;
            hmem.push_back(mem[l]);
        }
        for (uint32_t b = 0; b < mem.size(); b += kSegChunk) {
            hbeg.push_back(at + b);
            hend.push_back(at + std::min<uint32_t>(b + kSegChunk, (uint32_t)mem.size()));
        }
        hpofs[q + 1] = (uint32_t)hbeg.size();
        hlabel[q] = solve[q];
        hiters[q] = std::min<uint32_t>(kk * 4 + 30, (uint32_t)mem.size());
        it_max = std::max(it_max, hiters[q]);
    }
    const uint32_t n_items = (uint32_t)hbeg.size();
    DevBuf<uint32_t> mem(hmem.size(), s), ibeg(n_items, s), iend(n_items, s), pofs(S + 1, s), sidx(n, s), lidx(n, s),
        label(S, s), iters(S, s);
    h2d(mem.p, hmem.data(), hmem.size(), s);
    h2d(ibeg.p, hbeg.data(), n_items, s);
    h2d(iend.p, hend.data(), n_items, s);
    h2d(pofs.p, hpofs.data(), S + 1, s);
    h2d(sidx.p, hsidx.data(), n, s);
    h2d(lidx.p, hlidx.data(), n, s);
    h2d(label.p, hlabel.data(), S, s);
    h2d(iters.p, hiters.data(), S, s);
    DevBuf<double> V((size_t)it_max * n, s), w(n, s), c((size_t)it_max * S, s), ab((size_t)it_max * 2 * S, s),
        part((size_t)it_max * n_items, s), sq(S, s);
    check_cuda(cudaMemsetAsync(V.p, 0, sizeof(double) * V.n, s), "memset");  // rows of unsolved points stay 0
    const unsigned g = ceil_div(n, kBlk);
    auto seg_dots = [&](const double *Vrows, uint32_t rows, const double *x, double *out) {
        k_seg_dots_part<<<dim3(n_items, rows), kBlk, 0, s>>>(Vrows, n, x, mem.p, ibeg.p, iend.p, n_items, part.p);
        k_seg_sum_parts<<<ceil_div((uint64_t)rows * S, 128), 128, 0, s>>>(part.p, n_items, pofs.p, S, rows, out);
    };
    k_seg_start<<<g, kBlk, 0, s>>>(n, sidx.p, lidx.p, label.p, seed, V.p);
    seg_dots(V.p, 1, V.p, sq.p);
    k_seg_scale<<<g, kBlk, 0, s>>>(V.p, n, sidx.p, sq.p);
    check_launch("batched start");
    for (uint32_t j = 0; j < it_max; j++) {
        const double *vj = V.p + (size_t)j * n;
        k_spmv<<<ceil_div((uint64_t)n * 32, kBlk), kBlk, 0, s>>>(n, ptr.p, ci.p, val.p, vj, w.p);
        seg_dots(vj, 1, w.p, ab.p + (size_t)j * 2 * S);  // alpha_j per segment
        k_seg_recurrence<<<ceil_div((uint64_t)(j + 1) * S, 128), 128, 0, s>>>(ab.p, j, S, c.p);
        k_seg_comb<<<g, kBlk, 0, s>>>(V.p, n, j + 1, c.p, S, sidx.p, w.p, true);
        for (int pass = 0; pass < 2; pass++) {
            seg_dots(V.p, j + 1, w.p, c.p);
            k_seg_comb<<<g, kBlk, 0, s>>>(V.p, n, j + 1, c.p, S, sidx.p, w.p, true);
        }
        seg_dots(w.p, 1, w.p, ab.p + ((size_t)j * 2 + 1) * S);  // beta_j^2
        if (j + 1 < it_max)
            k_seg_next<<<g, kBlk, 0, s>>>(w.p, n, sidx.p, ab.p, j, S, iters.p, V.p + (size_t)(j + 1) * n);
        check_launch("batched lanczos step");
    }
    std::vector<double> hab((size_t)it_max * 2 * S);
    d2h(hab.data(), ab.p, hab.size(), s);
    sync(s);
    // per component: truncate, tridiagonal eigenproblem; keep the Ritz
    // coefficients of its kk smallest eigenvalues (ritz[q] [e][m_q])
    std::vector<std::vector<double>> ritz(S);
    std::vector<uint32_t> found(S), msteps(S);
    for (uint32_t q = 0; q < S; q++) {
        std::vector<double> alpha, beta;
        for (uint32_t j = 0; j < hiters[q]; j++) {
            alpha.push_back(hab[((size_t)j * 2) * S + q]);
            beta.push_back(std::sqrt(std::max(0.0, hab[((size_t)j * 2 + 1) * S + q])));
            if (beta.back() < 1e-12) break;
        }
        const uint32_t m = (uint32_t)alpha.size();
        std::vector<double> T((size_t)m * m, 0.0), tev, tvec;
        for (uint32_t i = 0; i < m; i++) {
            T[(size_t)i * m + i] = alpha[i];
            if (i + 1 < m) T[(size_t)i * m + i + 1] = T[(size_t)(i + 1) * m + i] = beta[i];
        }
        jacobi_eigen(T, m, tev, tvec);
        std::vector<uint32_t> order(m);
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return tev[x] < tev[y]; });
        found[q] = std::min(kk, m);
        msteps[q] = m;
        ritz[q].resize((size_t)found[q] * m);
        for (uint32_t e = 0; e < found[q]; e++)
            std::copy(tvec.begin() + (size_t)order[e] * m, tvec.begin() + (size_t)(order[e] + 1) * m,
                      ritz[q].begin() + (size_t)e * m);
    }
    // back-transform eigenvector e of every component, normalise per component
    for (uint32_t q = 0; q < S; q++) raw[solve[q]].assign(members[solve[q]].size() * n_comp, 0.0);
    std::vector<double> hv(n), hn(S), coef((size_t)it_max * S);
    for (uint32_t e = 1; e < kk; e++) {
        std::fill(coef.begin(), coef.end(), 0.0);  // [r][s]
        for (uint32_t q = 0; q < S; q++)
            if (e < found[q])
                for (uint32_t r = 0; r < msteps[q]; r++)
                    coef[(size_t)r * S + q] = ritz[q][(size_t)e * msteps[q] + r];
        h2d(c.p, coef.data(), coef.size(), s);
        k_seg_comb<<<g, kBlk, 0, s>>>(V.p, n, it_max, c.p, S, sidx.p, w.p, false);
        seg_dots(w.p, 1, w.p, sq.p);
        check_launch("batched back-transform");
        d2h(hv.data(), w.p, n, s);
        d2h(hn.data(), sq.p, S, s);
        sync(s);
        const uint32_t d = e - 1;
        for (uint32_t q = 0; q < S; q++) {
            const std::vector<uint32_t> &mem = members[solve[q]];
            std::vector<double> &out = raw[solve[q]];
            if (e < found[q]) {
                const double nr = std::sqrt(hn[q]);
                for (uint32_t l = 0; l < mem.size(); l++)
                    out[(size_t)l * n_comp + d] = (double)(float)(nr > 0 ? hv[mem[l]] / nr : hv[mem[l]]);
            } else {
                Mix r{seed + solve[q] + d};
                for (uint32_t l = 0; l < mem.size(); l++) out[(size_t)l * n_comp + d] = 2.0 * r.uniform() - 1.0;
            }
        }
    }
}

double max_abs(const std::vector<double> &v)
{
    double m = 0.0;
    for (double x : v) m = std::max(m, std::fabs(x));
    return m;
}

// centre every dimension, then scale so the largest |coordinate| is range
void centre_and_scale(std::vector<double> &e, uint32_t n, uint32_t n_comp, double range)
{
    for (uint32_t d = 0; d < n_comp; d++) {
        double mean = 0.0;
        for (uint32_t i = 0; i < n; i++) mean += e[(size_t)i * n_comp + d];
        mean /= n;
        for (uint32_t i = 0; i < n; i++) e[(size_t)i * n_comp + d] -= mean;
    }
    const double m = max_abs(e);
    if (m > 1e-8)
        for (double &x : e) x *= range / m;
}


}  // namespace
}  // namespace umapcu

using namespace umapcu;

namespace {

template <typename F>
umapcu_status guard_s(F &&f)
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

umapcu_status umapcu_smallest_eigenpairs(uint32_t n, const uint64_t *ptr, const uint32_t *col, const double *val,
                                         uint32_t n_components, uint64_t seed, float *evals, float *evecs,
                                         uint32_t *n_found)
{
    return guard_s([&]() -> umapcu_status {
        if (n == 0) return UMAPCU_NO_DATA;
        if (!ptr || !evals || !evecs || !n_found || n_components == 0 || n_components > 128) return UMAPCU_BAD_ARG;
        const uint64_t nnz = ptr[n];
        if (nnz && (!col || !val)) return UMAPCU_BAD_ARG;
        for (uint32_t i = 0; i < n; i++)
            if (ptr[i + 1] < ptr[i]) return UMAPCU_BAD_ARG;
        for (uint64_t e = 0; e < nnz; e++)
            if (col[e] >= n) return UMAPCU_BAD_ARG;
        keep_pool_memory();
        Stream st;
        DevBuf<uint64_t> dp(n + 1, st.s);
        DevBuf<uint32_t> dc(nnz ? nnz : 1, st.s);
        DevBuf<double> dv(nnz ? nnz : 1, st.s);
        h2d(dp.p, ptr, n + 1, st.s);
        h2d(dc.p, col, nnz, st.s);
        h2d(dv.p, val, nnz, st.s);
        std::vector<float> ev, vec;
        uint32_t k = 0;
        smallest_eigenpairs_dev(n, dp.p, dc.p, dv.p, n_components, seed, ev, vec, k, st.s);
        std::copy(ev.begin(), ev.end(), evals);
        std::copy(vec.begin(), vec.end(), evecs);  // [n][k]
        *n_found = k;
        return UMAPCU_OK;
    });
}

umapcu_status umapcu_spectral_layout(const uint32_t *row, const uint32_t *col, const float *val, uint64_t nnz,
                                     uint32_t n, uint32_t n_comp, uint64_t seed, float range, float *embd)
{
    return guard_s([&]() -> umapcu_status {
        if (n == 0) return UMAPCU_NO_DATA;
        if (!embd || n_comp == 0 || n_comp > 64 || (nnz && (!row || !col || !val))) return UMAPCU_BAD_ARG;
        for (uint64_t e = 0; e < nnz; e++)
            if (row[e] >= n || col[e] >= n) return UMAPCU_BAD_ARG;
        const double rng = range > 0.0f ? (double)range : 10.0;  // SPECTRAL_RANGE, init.rs:17
        keep_pool_memory();
        Stream st;
        const bool timing = getenv("UMAPCU_TIMING") != nullptr;
        auto t0 = std::chrono::steady_clock::now();
        auto lap = [&](const char *what) {
            if (!timing) return;
            sync(st.s);
            auto t1 = std::chrono::steady_clock::now();
            fprintf(stderr, "umapcu timing: spectral %-12s %9.3f ms\n", what,
                    std::chrono::duration<double, std::milli>(t1 - t0).count());
            t0 = t1;
        };
        lap("validate");
        // connected components (find_connected_components, init.rs:349-391),
        // labelled in order of their smallest point, members ascending
        std::vector<uint32_t> root;
        component_labels(n, nnz, row, col, root, st.s);
        lap("components");
        std::vector<uint32_t> cid(n, ~0u);
        std::vector<std::vector<uint32_t>> members;
        for (uint32_t i = 0; i < n; i++) {
            const uint32_t r = root[i];
            if (cid[r] == ~0u) {
                cid[r] = (uint32_t)members.size();
                members.emplace_back();
            }
            members[cid[r]].push_back(i);
        }
        std::vector<double> out((size_t)n * n_comp, 0.0);
        if (members.size() == 1) {
            // single_component_spectral + finalise_spectral_embedding
            // (init.rs:876-958): centre, scale to range, N(0, 1e-4) noise
            if (n <= n_comp + 1) {
                Mix r{seed};
                for (double &v : out) v = 2.0 * r.uniform() - 1.0;
            } else {
                DevBuf<uint64_t> ptr;
                DevBuf<uint32_t> ci;
                DevBuf<double> av;
                neg_normalised_adjacency(n, nnz, row, col, val, ptr, ci, av, st.s);
                std::vector<std::vector<double>> raw(1);
                batched_component_raw(n, ptr, ci, av, members, {0u}, n_comp, seed, raw, st.s);
                out.swap(raw[0]);
            }
            lap("eigen");
            centre_and_scale(out, n, n_comp, rng);
            Mix r{seed + 9999};
            for (double &x : out) x += 1e-4 * r.normal();
        } else {
            // multi_component_init (init.rs:413-524) without a data matrix:
            // centroids on the simplex (component_simplex_meta, init.rs:614),
            // each component spectral around its centroid within half the
            // largest centroid distance (random when it has fewer than
            // 2 n_comp points), then the whole centred and scaled
            const uint32_t C = (uint32_t)members.size(), half = (C + 1) / 2;
            std::vector<double> meta((size_t)C * n_comp, 0.0);
            for (uint32_t c = 0; c < C; c++) {
                const uint32_t idx = c < half ? c : c - half;
                if (idx < n_comp) meta[(size_t)c * n_comp + idx] = c < half ? 1.0 : -1.0;
            }
            const double mm = max_abs(meta);
            if (mm > 1e-8)
                for (double &x : meta) x /= mm;
            // the components' eigen-solves advance together: one Lanczos
            // over the block-diagonal whole-graph matrix, every operation
            // per component (batched_component_raw), in batches of at most
            // 16384 components
            std::vector<std::vector<double>> subs(C);
            std::vector<uint32_t> solve;
            for (uint32_t c = 0; c < C; c++) {
                const uint32_t nc = (uint32_t)members[c].size();
                if (nc < 2 * n_comp) continue;
                if (nc > n_comp + 1) {
                    solve.push_back(c);
                } else {  // too small for Lanczos (single_component_spectral_raw)
                    Mix r{seed + c};
                    subs[c].resize((size_t)nc * n_comp);
                    for (double &v : subs[c]) v = 2.0 * r.uniform() - 1.0;
                }
            }
            if (!solve.empty()) {
                DevBuf<uint64_t> ptr;
                DevBuf<uint32_t> ci;
                DevBuf<double> av;
                neg_normalised_adjacency(n, nnz, row, col, val, ptr, ci, av, st.s);
                for (size_t b = 0; b < solve.size(); b += 16384) {
                    const std::vector<uint32_t> part(solve.begin() + b,
                                                     solve.begin() + std::min(solve.size(), b + 16384));
                    batched_component_raw(n, ptr, ci, av, members, part, n_comp, seed, subs, st.s);
                }
            }
            lap("eigen");
            Mix r{seed};
            for (uint32_t c = 0; c < C; c++) {
                const double *cen = meta.data() + (size_t)c * n_comp;
                double dr = 0.0;  // meta_data_range (init.rs:768)
                for (uint32_t o = 0; o < C; o++) {
                    double d2 = 0.0;
                    for (uint32_t d = 0; d < n_comp; d++) {
                        const double df = cen[d] - meta[(size_t)o * n_comp + d];
                        d2 += df * df;
                    }
                    dr = std::max(dr, std::sqrt(d2));
                }
                dr /= 2.0;
                const std::vector<uint32_t> &mem = members[c];
                const uint32_t nc = (uint32_t)mem.size();
                if (nc < 2 * n_comp) {
                    for (uint32_t gi : mem)
                        for (uint32_t d = 0; d < n_comp; d++)
                            out[(size_t)gi * n_comp + d] = cen[d] + (2.0 * r.uniform() - 1.0) * dr;
                    continue;
                }
                const std::vector<double> &sub = subs[c];
                const double sm = max_abs(sub);
                const double ex = sm > 1e-8 ? dr / sm : 1.0;
                for (uint32_t li = 0; li < nc; li++)
                    for (uint32_t d = 0; d < n_comp; d++)
                        out[(size_t)mem[li] * n_comp + d] = cen[d] + sub[(size_t)li * n_comp + d] * ex;
            }
            centre_and_scale(out, n, n_comp, rng);
        }
        for (size_t i = 0; i < out.size(); i++) embd[i] = (float)out[i];
        lap("finish");
        return UMAPCU_OK;
    });
}

}  // extern "C"
