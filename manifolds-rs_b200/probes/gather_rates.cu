// Random-gather rates of one B200, the measurements behind the layout
// kernels' gather design (the coordinate rows of the other endpoint and the
// negatives are fetched with ordinary loads, one row per lane):
//
//   lsu      ordinary loads of random rows (4, 8, 16 bytes) from an 8 MiB
//            table held in L2, on a quarter, half and all of the SMs (one
//            1024-thread block per SM) and with 8 blocks of 256 per SM: rows
//            per SM-clock show whether the limit is per SM or the L2's;
//   dsmem    the same rows held in the shared memory of a thread-block
//            cluster (8 and 16 CTAs) and read across the cluster;
//   bulk16   cp.async.bulk copies of random 16-byte rows into shared memory;
//   gather4  cp.async.bulk.tensor.2d tile::gather4: four random 16-byte rows
//            per request (tensor map box one row high, x coordinate 0).
//
// All on one GPU, local memory only, no cluster multicast. Every row index
// is a hash reduced into the table by a multiply-high; every mbarrier wait is
// bounded (a warp that gives up records it and waits, bounded again, for the
// copies it still has in flight). Prints one line per measurement.
//
// Build: make -C manifolds-rs_b200 probes; run: manifolds-rs_b200/probes/gather_rates
#include <cstdint>
#include <cstdio>

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#define CK(x)                                                                                   \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) {                                                                \
            printf("CUDA error %s at line %d: %s\n", #x, __LINE__, cudaGetErrorString(e_));     \
            return 1;                                                                           \
        }                                                                                       \
    } while (0)

namespace {

__device__ __forceinline__ uint32_t mix(uint32_t h)
{
    // Wellons' lowbias32 finaliser
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return h;
}

// W floats per row (1, 2, 4); 8 independent gathers per thread per round
template <int W>
__global__ void k_lsu(const float *__restrict__ t, uint32_t rows, uint32_t rounds, float *__restrict__ out)
{
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t h = tid * 0x9E3779B1u + 0x7F4A7C15u;
    float acc = 0.0f;
    for (uint32_t r = 0; r < rounds; r++) {
        float v[8][W];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            h = mix(h);
            const uint32_t i = __umulhi(h, rows);
            if constexpr (W == 1) {
                v[u][0] = __ldg(t + i);
            } else if constexpr (W == 2) {
                const float2 q = __ldg(reinterpret_cast<const float2 *>(t) + i);
                v[u][0] = q.x;
                v[u][1] = q.y;
            } else {
                const float4 q = __ldg(reinterpret_cast<const float4 *>(t) + i);
                v[u][0] = q.x;
                v[u][1] = q.y;
                v[u][2] = q.z;
                v[u][3] = q.w;
            }
        }
#pragma unroll
        for (int u = 0; u < 8; u++)
#pragma unroll
            for (int w = 0; w < W; w++) acc += v[u][w];
    }
    out[tid] = acc;
}

// Each CTA of a cluster holds rows_per_cta float2 rows; a gather of row i
// reads CTA i / rows_per_cta's shared memory.
__global__ void k_dsmem(const float2 *__restrict__ t, uint32_t rows_per_cta, uint32_t rounds, float *__restrict__ out)
{
    extern __shared__ float2 sm[];
    uint32_t crank, csize;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(crank));
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(csize));
    for (uint32_t i = threadIdx.x; i < rows_per_cta; i += blockDim.x) sm[i] = t[(uint64_t)crank * rows_per_cta + i];
    asm volatile("barrier.cluster.arrive.aligned; barrier.cluster.wait.aligned;" ::: "memory");
    const uint32_t rows = rows_per_cta * csize;
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(sm);
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t h = tid * 0x9E3779B1u + 0x7F4A7C15u;
    float acc = 0.0f;
    for (uint32_t r = 0; r < rounds; r++) {
        float v[8][2];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            h = mix(h);
            const uint32_t i = __umulhi(h, rows);
            const uint32_t c = i / rows_per_cta, o = i - c * rows_per_cta;
            uint32_t ra;
            asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(base + o * 8u), "r"(c));
            asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v[u][0]), "=f"(v[u][1]) : "r"(ra));
        }
#pragma unroll
        for (int u = 0; u < 8; u++) acc += v[u][0] + v[u][1];
    }
    out[tid] = acc;
    // no CTA leaves while another may still read its shared memory
    asm volatile("barrier.cluster.arrive.aligned; barrier.cluster.wait.aligned;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t cnt)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(cnt) : "memory");
}
__device__ __forceinline__ void mbar_expect(uint32_t a, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
// bounded wait for the phase of the given parity; true when it completed
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity)
{
    for (uint32_t it = 0; it < (1u << 20); it++) {
        uint32_t ok;
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                     : "=r"(ok)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (ok) return true;
    }
    return false;
}

constexpr int kStages = 4;  // requests in flight per lane

// MODE 0: one 16-byte cp.async.bulk per lane and stage; MODE 1: one
// tile::gather4 request (four 16-byte rows) per lane and stage. Each warp
// owns kStages shared-memory stages and mbarriers; lane 0 arms a stage's
// barrier with the stage's bytes, every lane issues into its own slot.
template <int MODE>
__global__ void __launch_bounds__(256) k_tma(const __grid_constant__ CUtensorMap tmap,
                                             const float4 *__restrict__ t, uint32_t rows, uint32_t rounds,
                                             float *__restrict__ out, uint32_t *err)
{
    constexpr uint32_t kSlot = MODE == 0 ? 16 : 128;  // a tensor copy's destination 128-byte aligned
    constexpr uint32_t kBytes = MODE == 0 ? 16 : 64;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[8][kStages];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char *wbuf = smem + (size_t)warp * kStages * 32 * kSlot;
    const uint32_t bar0 = (uint32_t)__cvta_generic_to_shared(&bars[warp][0]);
    if (lane == 0)
        for (int s = 0; s < kStages; s++) mbar_init(bar0 + 8 * s, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncwarp();
    uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) * 0x9E3779B1u + 0x7F4A7C15u;
    float acc = 0.0f;
    bool bad = false;
    auto issue = [&](uint32_t r) {
        const int s = r % kStages;
        const uint32_t bar = bar0 + 8 * s;
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(wbuf + ((size_t)s * 32 + lane) * kSlot);
        if (lane == 0) mbar_expect(bar, 32 * kBytes);
        __syncwarp();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if constexpr (MODE == 0) {
            h = mix(h);
            const float4 *src = t + __umulhi(h, rows);
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], 16, [%2];"
                         ::"r"(dst), "l"(src), "r"(bar)
                         : "memory");
        } else {
            int32_t rr[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                h = mix(h);
                rr[u] = (int32_t)__umulhi(h, rows);
            }
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
                " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
                "l"(&tmap), "r"(0), "r"(rr[0]), "r"(rr[1]), "r"(rr[2]), "r"(rr[3]), "r"(bar)
                : "memory");
        }
    };
    auto consume = [&](uint32_t r) -> bool {
        const int s = r % kStages;
        if (!mbar_wait(bar0 + 8 * s, (r / kStages) & 1u)) return false;
        const float4 *p = reinterpret_cast<const float4 *>(wbuf + ((size_t)s * 32 + lane) * kSlot);
#pragma unroll
        for (uint32_t u = 0; u < kBytes / 16; u++) {
            const float4 v = p[u];
            acc += v.x + v.y + v.z + v.w;
        }
        __syncwarp();
        return true;
    };
    uint32_t issued = 0, done = 0;
    for (uint32_t r = 0; r < rounds; r++) {
        if (r >= kStages) {
            if (!consume(done)) {
                bad = true;
                break;
            }
            done++;
        }
        issue(r);
        issued++;
    }
    while (done < issued) {  // every issued stage is waited for (bounded) before the warp leaves
        if (!consume(done)) {
            bad = true;
            consume(done);
        }
        done++;
    }
    if (bad && lane == 0) atomicAdd(err, 1u);
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

template <class F>
float best_ms(F launch, int reps)
{
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    for (int it = 0; it <= reps; it++) {  // the first launch warms L2
        cudaEventRecord(a);
        launch();
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        if (it && ms < best) best = ms;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best;
}

}  // namespace

int main()
{
    int sms = 0, khz = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
    CK(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, 0));
    const double sm_hz = (double)khz * 1e3;
    printf("gather_rates: %d SMs, max SM clock %.0f MHz, 8 MiB table (L2-resident)\n", sms, sm_hz / 1e6);
    const uint64_t tbytes = 8ull << 20;
    float *t = nullptr, *out = nullptr;
    uint32_t *err = nullptr;
    CK(cudaMalloc(&t, tbytes));
    CK(cudaMemset(t, 0, tbytes));
    CK(cudaMalloc(&out, (size_t)sms * 2048 * sizeof(float)));
    CK(cudaMalloc(&err, sizeof(uint32_t)));
    CK(cudaMemset(err, 0, sizeof(uint32_t)));
    auto report = [&](const char *what, double rows, float ms, int sms_used) {
        const double rate = rows / (ms * 1e-3);
        printf("%-44s %8.3f ms %8.1f G rows/s %6.3f rows per SM-clock\n", what, ms, rate / 1e9,
               rate / (sms_used * sm_hz));
    };

    // lsu: 1024-thread blocks on a quarter, half and all SMs; 8 x 256 per SM
    const uint32_t rounds = 64;
    for (int w : {2, 1, 4}) {
        const int cfg[4] = {sms / 4, sms / 2, sms, 0};
        for (int k : cfg) {
            const uint32_t blocks = k ? (uint32_t)k : 8u * sms, threads = k ? 1024u : 256u;
            const uint32_t rows = (uint32_t)(tbytes / (4u * w));
            const float ms = best_ms([&] {
                if (w == 1) k_lsu<1><<<blocks, threads>>>(t, rows, rounds, out);
                else if (w == 2) k_lsu<2><<<blocks, threads>>>(t, rows, rounds, out);
                else k_lsu<4><<<blocks, threads>>>(t, rows, rounds, out);
            }, 5);
            CK(cudaGetLastError());
            char what[96];
            snprintf(what, sizeof what, "lsu %2d-byte rows, %4u blocks x %4u", 4 * w, blocks, threads);
            report(what, 8.0 * rounds * blocks * threads, ms, k ? k : sms);
        }
    }

    // dsmem: a 1.6 MB table (200k 8-byte rows) spread over clusters of 8 and 16
    for (int c : {8, 16}) {
        const uint32_t rows_total = 204800, rpc = rows_total / c;
        const size_t smem = (size_t)rpc * 8;
        CK(cudaFuncSetAttribute(k_dsmem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        if (c > 8 && cudaFuncSetAttribute(k_dsmem, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
            cudaGetLastError();
            printf("dsmem clusters of %d: not allowed here\n", c);
            continue;
        }
        cudaLaunchConfig_t lc = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = c;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        lc.attrs = at;
        lc.numAttrs = 1;
        lc.blockDim = dim3(1024);
        lc.dynamicSmemBytes = smem;
        lc.gridDim = dim3(c);
        int clusters = 0;
        CK(cudaOccupancyMaxActiveClusters(&clusters, k_dsmem, &lc));
        if (clusters <= 0) continue;
        lc.gridDim = dim3((uint32_t)clusters * c);
        const float2 *t2 = reinterpret_cast<const float2 *>(t);
        const float ms = best_ms([&] { cudaLaunchKernelEx(&lc, k_dsmem, t2, rpc, rounds, out); }, 5);
        CK(cudaGetLastError());
        CK(cudaDeviceSynchronize());
        char what[96];
        snprintf(what, sizeof what, "dsmem 8-byte rows, %d clusters of %d", clusters, c);
        report(what, 8.0 * rounds * clusters * c * 1024.0, ms, clusters * c);
    }

    // bulk16 / gather4 over the table as [rows][4] floats (16-byte rows)
    PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void **)&encode, cudaEnableDefault, &q));
    if (!encode || q != cudaDriverEntryPointSuccess) {
        printf("cuTensorMapEncodeTiled unavailable\n");
        return 1;
    }
    const uint32_t rows16 = (uint32_t)(tbytes / 16);
    CUtensorMap tm;
    cuuint64_t gdim[2] = {4, rows16}, gstride[1] = {16};
    cuuint32_t box[2] = {4, 1}, estride[2] = {1, 1};
    if (encode(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, t, gdim, gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
        printf("tensor map encoding failed\n");
        return 1;
    }
    const uint32_t trounds = 256;
    for (int mode = 0; mode < 2; mode++) {
        const uint32_t threads = mode == 0 ? 256 : 128;
        const size_t smem = (size_t)(threads / 32) * kStages * 32 * (mode == 0 ? 16 : 128);
        if (mode == 0) CK(cudaFuncSetAttribute(k_tma<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        else CK(cudaFuncSetAttribute(k_tma<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        for (int per_sm : {1, 2, 4, 8}) {
            if (smem * per_sm > 200 * 1024) continue;
            const uint32_t blocks = (uint32_t)sms * per_sm;
            const float4 *t4 = reinterpret_cast<const float4 *>(t);
            const float ms = best_ms([&] {
                if (mode == 0) k_tma<0><<<blocks, threads, smem>>>(tm, t4, rows16, trounds, out, err);
                else k_tma<1><<<blocks, threads, smem>>>(tm, t4, rows16, trounds, out, err);
            }, 3);
            CK(cudaGetLastError());
            CK(cudaDeviceSynchronize());
            uint32_t h_err = 0;
            CK(cudaMemcpy(&h_err, err, sizeof h_err, cudaMemcpyDeviceToHost));
            if (h_err) {
                printf("%s: %u warps gave up waiting; stopping\n", mode ? "gather4" : "bulk16", h_err);
                return 2;
            }
            char what[96];
            snprintf(what, sizeof what, "%s 16-byte rows, %d blocks x %u per SM", mode ? "gather4" : "bulk16 ",
                     per_sm, threads);
            report(what, (double)trounds * blocks * threads * (mode ? 4 : 1), ms, sms);
        }
    }
    CK(cudaFree(t));
    CK(cudaFree(out));
    CK(cudaFree(err));
    return 0;
}
