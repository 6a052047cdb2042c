// Layout optimisation that allocates no device memory.
//
// Some callers cannot allocate device memory at the moment they want a
// layout: a host framework that has reserved the whole device for its own
// allocator, or a deployment whose device-memory budget is fixed at start-up.
// For them, umapcu_optimise_csr_noalloc runs the same fused epoch kernel as
// the allocating entry points, with every scratch buffer (Adam moments, the
// second embedding buffer, the per-entry schedule cursors) carved out of one
// file-scope device array of fixed size that the library holds on every GPU
// that loads it, until the process exits. It is an ordinary host call: it
// makes CUDA runtime calls (device query, symbol lookup, memset, launches,
// copy), so it must not be called from a stream callback or a host function
// node, where CUDA forbids runtime calls.
#include "internal.cuh"
#include "layout.cuh"

#include <mutex>

using namespace umapcu;

namespace {

// Maximum scratch of one call; problems that need more are rejected.
constexpr size_t kNoAllocScratchBytes = 16u << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch for the current device. In host code
// the symbol names a host-side stand-in, not device memory, so the address
// is looked up once per device with that device current and cached.
void *scratch_address()
{
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) fail(UMAPCU_NO_DEVICE, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void *ptr = nullptr;
        check_cuda(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress");
        g_scratch_addr[dev] = ptr;
    }
    return g_scratch_addr[dev];
}

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

__global__ void k_noalloc_sched_init(const float *__restrict__ period, float2 *__restrict__ sched, uint64_t tot)
{
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= tot) return;
    const float pe = period[p];
    sched[p] = make_float2(pe, pe);  // cursors start one period in (umap_optimiser_gpu.rs:425-430)
}

}  // namespace

extern "C" umapcu_status umapcu_optimise_csr_noalloc(float *d_embd, uint32_t n, uint32_t n_dim,
                                                     const uint32_t *d_offsets, const uint32_t *d_other,
                                                     const float *d_period, uint64_t n_entries,
                                                     const umapcu_optim_params *params, uint64_t seed,
                                                     uint32_t sampler, void *cuda_stream)
{
    try {
        if (n == 0) return UMAPCU_NO_DATA;
        if (n_entries == 0) return UMAPCU_NO_GRAPH_EDGES;
        if (!d_embd || !d_offsets || !d_other || !d_period || !params) return UMAPCU_BAD_ARG;
        if (n_dim < 1 || n_dim > 8 || params->n_epochs == 0 || sampler > UMAPCU_NEG_PHILOX) return UMAPCU_BAD_ARG;
        // The epoch kernel moves a row of the embedding (and of the moments)
        // as one float2 for n_dim = 2 and one float4 for n_dim = 4, and reads
        // the CSR arrays as 32-bit words: refuse pointers those accesses
        // would fault on, before anything is launched.
        const uintptr_t row_align = n_dim == 2 ? 8 : n_dim == 4 ? 16 : 4;
        if ((uintptr_t)d_embd % row_align || (uintptr_t)d_offsets % 4 || (uintptr_t)d_other % 4 ||
            (uintptr_t)d_period % 4)
            return UMAPCU_BAD_ARG;
        const uint64_t nt = (uint64_t)n * n_dim;
        const size_t b_sched = round256(n_entries * sizeof(float2));
        const size_t b_vec = round256(nt * sizeof(float));
        // the last 256 bytes hold the checked build's error word
        if (n_entries >= (1ull << 31) || b_sched + 3 * b_vec > kNoAllocScratchBytes - 256) return UMAPCU_CAPACITY;
        cudaStream_t s = (cudaStream_t)cuda_stream;
        unsigned char *base = (unsigned char *)scratch_address();
        float2 *sched = (float2 *)base;
        float *y_alt = (float *)(base + b_sched);
        float *m = (float *)(base + b_sched + b_vec);
        float *v = (float *)(base + b_sched + 2 * b_vec);
        uint32_t *err = (uint32_t *)(base + kNoAllocScratchBytes - 256);
        // the array keeps the previous call's contents: start every state
        // buffer from its initial value
        check_cuda(cudaMemsetAsync(m, 0, nt * sizeof(float), s), "cudaMemsetAsync");
        check_cuda(cudaMemsetAsync(v, 0, nt * sizeof(float), s), "cudaMemsetAsync");
        check_cuda(cudaMemsetAsync(err, 0, sizeof(uint32_t), s), "cudaMemsetAsync");
        k_noalloc_sched_init<<<ceil_div(n_entries, 256), 256, 0, s>>>(d_period, sched, n_entries);
        check_launch("k_noalloc_sched_init");
        float *y[2] = {d_embd, y_alt};
        int cur = 0;
        for (uint32_t epoch = 0; epoch < params->n_epochs; epoch++) {
            EpochArgs A{};
            A.n = n;
            A.offsets = d_offsets;
            A.other = d_other;
            A.sched = sched;
            A.y_cur = y[cur];
            A.y_next = y[cur ^ 1];
            A.m = m;
            A.v = v;
            A.epoch = epoch;
            A.epoch_f = (float)epoch;
            epoch_scalars(*params, epoch, &A.fused, &A.epsc, &A.lr_sgd);
            A.a = params->a;
            A.b = params->b;
            A.two_a_b = 2.0f * params->a * params->b;
            A.two_gamma_b = 2.0f * params->gamma * params->b;
            A.omb1 = 1.0f - params->beta1;
            A.omb2 = 1.0f - params->beta2;
            A.neg_rate = params->neg_sample_rate;
            A.sampler = sampler;
            A.seed32 = (uint32_t)seed;
            A.seed_lo = (uint32_t)seed;
            A.seed_hi = (uint32_t)(seed >> 32);
            A.fastmod_M = fastmod_magic(n);
            A.optimiser = UMAPCU_OPT_ADAM;
            A.n_entries = n_entries;
            A.err = err;
            launch_epoch(A, n_dim, false, s);
            cur ^= 1;
        }
        if (cur != 0)
            check_cuda(cudaMemcpyAsync(d_embd, y_alt, nt * sizeof(float), cudaMemcpyDeviceToDevice, s),
                       "cudaMemcpyAsync");
#ifdef UMAPCU_CHECKED
        // the checked build waits for the epochs to report their indices
        uint32_t h = 0;
        check_cuda(cudaMemcpyAsync(&h, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
        check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        return (umapcu_status)h;
#else
        return UMAPCU_OK;
#endif
    } catch (const Error &e) {
        return e.status;
    } catch (...) {
        return UMAPCU_CUDA_LAUNCH;
    }
}
