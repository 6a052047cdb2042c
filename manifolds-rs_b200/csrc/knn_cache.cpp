// kNN cache file: precomputed neighbours stored once and reused across
// layouts (the reference keeps them in memory only, PreComputedKnn,
// src/lib.rs:79). Layout (little-endian):
//   header, 48 bytes: char magic[8] = "UMAPKNN\0", u32 version = 1,
//     u32 metric, u64 n, u32 k, u32 flags (bit 0: self excluded),
//     u64 checksum (FNV-1a 64 over the payload bytes), u64 reserved = 0
//   payload: i32 idx [n * k], f32 dist [n * k]
#include <stdint.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "umapcu.h"

namespace {

struct KnnHeader {
    char magic[8];
    uint32_t version;
    uint32_t metric;
    uint64_t n;
    uint32_t k;
    uint32_t flags;
    uint64_t checksum;
    uint64_t reserved;
};
static_assert(sizeof(KnnHeader) == 48, "header layout");

constexpr char kMagic[8] = {'U', 'M', 'A', 'P', 'K', 'N', 'N', '\0'};

bool little_endian()
{
    const uint16_t one = 1;
    unsigned char b;
    memcpy(&b, &one, 1);
    return b == 1;
}

uint64_t fnv1a(uint64_t h, const void *p, size_t bytes)
{
    const unsigned char *c = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i < bytes; i++) {
        h ^= c[i];
        h *= 0x100000001b3ull;
    }
    return h;
}
constexpr uint64_t kFnvBasis = 0xcbf29ce484222325ull;

struct File {
    FILE *f = nullptr;
    File(const char *path, const char *mode) : f(fopen(path, mode)) {}
    ~File()
    {
        if (f) fclose(f);
    }
};

umapcu_status read_header(FILE *f, KnnHeader &h)
{
    if (fread(&h, sizeof h, 1, f) != 1) return UMAPCU_BAD_ARG;
    if (memcmp(h.magic, kMagic, 8) != 0 || h.version != 1 || h.metric > UMAPCU_METRIC_COSINE || h.k == 0 ||
        h.n == 0 || h.n > 0xffffffffull)
        return UMAPCU_BAD_ARG;
    return UMAPCU_OK;
}

}  // namespace

extern "C" {

umapcu_status umapcu_knn_save(const char *path, uint32_t n, uint32_t k, uint32_t metric, const int32_t *knn_idx,
                              const float *knn_dist)
{
    if (!path || !knn_idx || !knn_dist || n == 0 || k == 0 || metric > UMAPCU_METRIC_COSINE) return UMAPCU_BAD_ARG;
    if (!little_endian()) return UMAPCU_BAD_ARG;
    const size_t m = (size_t)n * k;
    KnnHeader h{};
    memcpy(h.magic, kMagic, 8);
    h.version = 1;
    h.metric = metric;
    h.n = n;
    h.k = k;
    h.flags = 1u;
    h.checksum = fnv1a(fnv1a(kFnvBasis, knn_idx, 4 * m), knn_dist, 4 * m);
    File f(path, "wb");
    if (!f.f) return UMAPCU_BAD_ARG;
    if (fwrite(&h, sizeof h, 1, f.f) != 1 || fwrite(knn_idx, 4, m, f.f) != m || fwrite(knn_dist, 4, m, f.f) != m)
        return UMAPCU_BAD_ARG;
    return fflush(f.f) == 0 ? UMAPCU_OK : UMAPCU_BAD_ARG;
}

umapcu_status umapcu_knn_load_header(const char *path, uint32_t *n, uint32_t *k, uint32_t *metric)
{
    if (!path || !n || !k || !metric) return UMAPCU_BAD_ARG;
    File f(path, "rb");
    if (!f.f) return UMAPCU_BAD_ARG;
    KnnHeader h;
    const umapcu_status rc = read_header(f.f, h);
    if (rc != UMAPCU_OK) return rc;
    *n = (uint32_t)h.n;
    *k = h.k;
    *metric = h.metric;
    return UMAPCU_OK;
}

umapcu_status umapcu_knn_load(const char *path, uint32_t n, uint32_t k, int32_t *knn_idx, float *knn_dist)
{
    if (!path || !knn_idx || !knn_dist || !little_endian()) return UMAPCU_BAD_ARG;
    File f(path, "rb");
    if (!f.f) return UMAPCU_BAD_ARG;
    KnnHeader h;
    umapcu_status rc = read_header(f.f, h);
    if (rc != UMAPCU_OK) return rc;
    if (h.n != n || h.k != k) return UMAPCU_BAD_ARG;
    const size_t m = (size_t)n * k;
    if (fread(knn_idx, 4, m, f.f) != m || fread(knn_dist, 4, m, f.f) != m) return UMAPCU_BAD_ARG;
    char extra;
    if (fread(&extra, 1, 1, f.f) != 0) return UMAPCU_BAD_ARG;  // trailing bytes
    if (fnv1a(fnv1a(kFnvBasis, knn_idx, 4 * m), knn_dist, 4 * m) != h.checksum) return UMAPCU_BAD_ARG;
    for (size_t i = 0; i < m; i++)
        if (knn_idx[i] < 0 || (uint32_t)knn_idx[i] >= n) return UMAPCU_BAD_ARG;
    return UMAPCU_OK;
}

}  // extern "C"
