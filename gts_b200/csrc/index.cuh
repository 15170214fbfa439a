// index.cuh -- the gts_index handle (host side) and internal entry points.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/gts_b200.h"
#include "common.cuh"

struct gts_index {
    gts_params params;
    int num = 0, dim = 0, metric = 0;
    int tree_h = 0, max_node_num = 0;
    cudaStream_t stream = 0;

    float *rows = nullptr, *trows = nullptr;
    char *strs = nullptr, *tstrs = nullptr;
    int *lens = nullptr, *tlens = nullptr;
    uint4 *tsig = nullptr;
    int *id_list = nullptr, *pos_of_id = nullptr;
    int *node_pid = nullptr, *node_size = nullptr, *node_lid = nullptr, *node_pivot = nullptr;
    float *node_min_dis = nullptr;
    uint8_t *node_flags = nullptr;

    // per-call scratch owned by the handle
    int *d_counter = nullptr;   // persistent-kernel work counter
    int *d_status = nullptr;    // kernel status word
    unsigned long long *d_stats = nullptr;   // work counters of the last search (kStatsN)
    bool keep_stats = false;                 // a nested search adds to, not resets, the counters
    size_t device_bytes = 0;

    // tensor-core filter (L2): per-block operand records, built on first use
    unsigned char *fast_recs = nullptr;
    int fast_nb = 0, fast_nsb = 0;   // filter blocks, superblocks
    int last_fast_overflow = 0;
    // device time of the filter kernel (CUDA events around each launch),
    // kept only while timing is on (gts_filter_timing)
    bool time_filter = false;
    cudaEvent_t fev[2] = {nullptr, nullptr};
    double filter_ms = 0.0;
    long long filter_launches = 0;
    // kernels this library launched for searches on this handle (host count)
    long long kernel_launches = 0;
    // autotuned fast-form configuration per k (fast.cu): 0 = not tuned, else
    // 1 | learned << 1 | column groups << 2 | blocks per item << 8
    int fast_cfg[65] = {};
    int range_variant = 1;   // fast range counts: 0 the block-stationary filter where it fits, 1 the tile filter
    // autotuned threads per query CTA of the plain traversal per search mode
    // (kNN, range count, range ids; search.cu), 0 = not tuned
    int plain_nt[3] = {};
    // range counts: objects a query verifies in one CTA before it hands its
    // older stack entries over as (query, node) items (0: never); the item
    // lists, and the items handed over since the last reset
    int plain_split = 32768;
    void *split_buf = nullptr;
    size_t split_bytes = 0;
    long long last_split_items = 0;

    // reusable per-call scratch (grown on demand, freed with the handle)
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    // device copies of host-buffer arguments (gts_knn, gts_range, ...):
    // grown on demand and kept, so those calls allocate nothing in steady state
    void *io = nullptr;
    size_t io_bytes = 0;
    // CUDA graph of the fast form's filter pass (fast.cu), launched on the
    // handle's own stream and replayed while the batch shape stays the same
    cudaStream_t graph_stream = nullptr;
    // up to kGraphSlots captured filter passes, one per batch shape and
    // argument buffers (batches of a few shapes in turn, such as one per k,
    // each replay their own), least recently used replaced
    static constexpr int kGraphSlots = 16;
    cudaGraphExec_t graph_exec[kGraphSlots] = {};
    long long graph_key[kGraphSlots][8] = {};
    long long graph_used[kGraphSlots] = {};
    long long graph_kernels[kGraphSlots] = {};   // this library's kernels in each graph
    cudaEvent_t graph_ev[2] = {nullptr, nullptr};
    bool use_graphs = true;
    long long graph_launches = 0;
    long long graph_clock = 0;

    // learned kNN radius (mlp.cu): parameters, input standardisation,
    // feature pivots; valid for the tree it was trained on
    float *mlp_P = nullptr, *mlp_norm = nullptr;
    int *mlp_piv = nullptr;
    int mlp_npiv = 0;
    float mlp_ymu = 0.f, mlp_ysig = 1.f, mlp_widen = 1.f;
    float mlp_widen_at[65] = {};   // per trained k (0: none; the global factor serves)
    bool mlp_ready = false;

    gts::DevTree dev() const;
};

namespace gts {

// Search work counters (gts_search_stats):
//   [0] plain: leaf objects read          fast: operand blocks streamed
//   [1] plain: pivots evaluated           fast: bytes streamed
//   [2] exact (reference-order) values    [3] plain: queries finished
//   [4] fast: queries answered again on the plain path
//   [5] fast: candidates appended         [6] fast: filter passes
//   [7] fast: (query tile, block) pairs tested by the block bound
constexpr int kStatsN = 8;

// Build the tree for the data already placed in idx->rows / strs / lens.
int build_tree(gts_index *idx, cudaStream_t s);
// Free the tree arrays (not the data).
void free_tree(gts_index *idx);
void free_data(gts_index *idx);

int search_knn(gts_index *idx, const int *d_qids, int qnum, int k, int form,
               float *d_kth, int *d_ids, float *d_dists, cudaStream_t s);
int search_range(gts_index *idx, const int *d_qids, int qnum, float r, int *d_counts,
                 const uint32_t *d_deleted, cudaStream_t s);
int search_range_fast(gts_index *idx, const int *d_qids, int qnum, float r, int *d_counts, cudaStream_t s);
// Range counts at time stamps (the stream-update path): query q is object
// d_qids[q] at operation d_qtime[q]; an object within r adds its entries
// live in the tree (d_tree_counts) and in the cache list (d_cache_counts)
// at that operation (SearchArgs::ents).
int search_range_timed(gts_index *idx, const int *d_qids, const int *d_qtime, int qnum, float r,
                       const int *d_ent_off, const int4 *d_ents, int *d_tree_counts, int *d_cache_counts,
                       cudaStream_t s);
// Queries given as data (rows, or strings with lengths), not ids: no self
// match; the plain traversal.
int search_knn_rows(gts_index *idx, const float *d_qrows, const char *d_qstrs, const int *d_qlens, int qnum, int k,
                    float *d_kth, int *d_ids, float *d_dists, cudaStream_t s);
int search_range_rows(gts_index *idx, const float *d_qrows, const char *d_qstrs, const int *d_qlens, int qnum,
                      float r, int *d_counts, cudaStream_t s);
int search_range_ids(gts_index *idx, const int *d_qids, int qnum, float r, int *d_counts,
                     int *d_ids, float *d_dists, const int *d_offsets, cudaStream_t s);

template <typename T>
int dev_alloc(T **p, size_t n, size_t *acct);

// Device scratch one search call may hold (gts_params.mem_budget_gb; 0 means
// 8 GiB).  The fast form sizes its runs of queries, the seeded plain form its
// chunks and the update path its query batches to fit it.
inline size_t search_budget(const gts_index *idx)
{
    const double gb = idx->params.mem_budget_gb;
    return gb > 0 ? (size_t)(gb * 1073741824.0) : ((size_t)8 << 30);
}

// Grow idx->scratch to at least `bytes`.
int ensure_scratch(gts_index *idx, size_t bytes);
// Grow idx->io to at least `bytes`.
int ensure_io(gts_index *idx, size_t bytes);

bool fast_supported(const gts_index *idx, int k);
int mlp_seed(gts_index *idx, const int *d_qids, int qnum, int k, int *d_r2_bits, cudaStream_t st);
int search_knn_fast(gts_index *idx, const int *d_qids, int qnum, int k, float *d_kth, int *d_ids,
                    float *d_dists, cudaStream_t s);
int search_knn_plain_learned(gts_index *idx, const int *d_qids, int qnum, int k, float *d_kth, int *d_ids,
                             float *d_dists, cudaStream_t s);
int fast_config_get(const gts_index *idx, int k, int *tuned, int *learned, int *cg, int *item, int *variant);
int fast_prepare_now(gts_index *idx, cudaStream_t st, int *done);
// Drop the captured filter graph (its device pointers or parameters changed).
void graph_invalidate(gts_index *idx);
// Unseeded filter with all scratch inside the caller's fixed buffer.
int search_knn_fast_fixed(gts_index *idx, const int *d_qids, int qnum, int k, float *d_kth, int *d_ids,
                          float *d_dists, unsigned char *scratch, size_t bytes, cudaStream_t s);

// A set of device allocations freed together on scope exit.
struct DevVec {
    void *ps[8] = {};
    int n = 0;
    ~DevVec()
    {
        for (int i = 0; i < n; i++)
            if (ps[i]) cudaFree(ps[i]);
    }
    template <typename T>
    int alloc(T **p, size_t cnt)
    {
        int rc = dev_alloc(p, cnt, nullptr);
        if (rc == 0 && n < 8) ps[n++] = *p;
        return rc;
    }
};

}  // namespace gts
