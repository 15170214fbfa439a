// noalloc.cu -- gts_knn_device_noalloc: the tensor-core kNN filter with its
// scratch in a fixed, file-scope device array instead of cudaMalloc'd memory.
//
// Callers that cannot allocate: processes whose device memory is already
// handed to a pool (a PyTorch caching allocator or a serving engine that
// reserves a fixed share of HBM), where a cudaMalloc fails or breaks their
// budget; and latency paths that share the GPU, where the cudaFree behind a
// per-call allocation synchronises the whole device.
//
// Limits: at most kNoAllocMaxQueries queries per call, L2 metric, dim <= 128,
// 1 <= k <= 64; the array is kNoAllocBytes (12 MiB) per device.  Every call
// on a device shares the one array, so calls whose work overlaps on the GPU
// (other host threads, or other streams without ordering between them) race
// on it; calls on one stream, or ordered by events, are safe.  Nothing in the
// array has to start at zero: each call clears the counters it uses (work
// item counter, candidate counts, failure count) on its stream before use.
// Every call looks the array up with cudaGetSymbolAddress on the current
// device (cheap once the module is loaded), so a context that was reset and
// made again gets the new address; the first call on a device loads this
// file's module and should come before any stream capture.
//
// Index size: the fixed array also holds one run's per-tile block lists
// (4 bytes per filter block per tile) and work items, next to the 1,024-slot
// candidate lists of the queries (about 6.3 MiB at 512 queries).  Past about
// 35 million objects (some 270,000 filter blocks) those no longer fit beside
// 512 queries and a call fails with "fixed scratch ... too small"; fewer
// queries per call fit larger indexes.
#include "index.cuh"

namespace {

constexpr int kNoAllocMaxQueries = 512;
constexpr size_t kNoAllocBytes = (size_t)12 << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of the array on the current device.
int noalloc_scratch(unsigned char **out)
{
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        gts_set_error("gts_knn_device_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return GTS_ERR_CUDA;
    }
    *out = (unsigned char *)p;
    return GTS_OK;
}

}  // namespace

extern "C" int gts_knn_device_noalloc(gts_index *idx, const int *d_qids, int qnum, int k, float *d_kth,
                                      int *d_ids, float *d_dists, void *stream)
{
    if (!idx || qnum < 0 || (qnum > 0 && (!d_qids || !d_kth))) {
        gts_set_error("gts_knn_device_noalloc: invalid argument");
        return GTS_ERR_INVALID;
    }
    if (qnum > kNoAllocMaxQueries) {
        gts_set_error("gts_knn_device_noalloc: %d queries exceed the maximum of %d per call", qnum,
                      kNoAllocMaxQueries);
        return GTS_ERR_INVALID;
    }
    if (k < 1 || k > 64) {
        gts_set_error("gts_knn_device_noalloc: k must be in [1, 64], got %d", k);
        return GTS_ERR_INVALID;
    }
    if (qnum == 0) return GTS_OK;
    unsigned char *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    return gts::search_knn_fast_fixed(idx, d_qids, qnum, k, d_kth, d_ids, d_dists, scratch, kNoAllocBytes,
                                      (cudaStream_t)stream);
}
