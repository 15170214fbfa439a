// update.cu -- lazy cache-list stream update (updateIndexRnn, update.cuh:449-638).
//
// Semantics kept from the reference:
//   * insert (flag 0): the id names a physical row of the current data
//     array; a copy of that row joins the cache list (update.cuh:481).  When
//     the list holds max_in_size entries the data is compacted -- live tree
//     rows in physical order, then the cached rows -- and the index is rebuilt
//     (update.cuh:484-540);
//   * delete (flag 1): the id is logical -- live tree rows in physical order,
//     then the cache list (findIdx, update.cuh:118-143).  A tree row is
//     marked deleted; a cache entry is removed (update.cuh:561-578).  An id
//     that matches nothing re-applies the previous delete (the reference's
//     delete_id keeps its last value);
//   * query (flag 2): the id is used as a physical row (update.cuh:588); the
//     answer is the number of live tree objects within r plus the number of
//     cache entries within r (search_naive.cuh:208-251).  When the cache is
//     empty the cache count of the previous query is reused, as the
//     reference's rnum is (update.cuh:592-597).
// What is different: the logical->physical map is a Fenwick tree on the
// host (O(log N) per delete instead of a device scan), deletions reach the
// device as a bitmap that the search kernel skips, and each run of
// consecutive queries is one batched launch.
#include <algorithm>
#include <chrono>
#include <vector>
#include "index.cuh"

namespace gts {

__global__ void k_gather_rows(int n_new, int dim, const int *map, const float *src, float *dst)
{
    size_t total = (size_t)n_new * dim;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        size_t r = i / dim, c = i % dim;
        dst[i] = src[(size_t)map[r] * dim + c];
    }
}

__global__ void k_gather_strs(int n_new, const int *map, const char *src, const int *src_len, char *dst,
                              int *dst_len)
{
    size_t total = (size_t)n_new * kStrStride;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        size_t r = i / kStrStride, c = i % kStrStride;
        dst[i] = src[(size_t)map[r] * kStrStride + c];
        if (c == 0) dst_len[r] = src_len[map[r]];
    }
}

// Cache-list scan (searchD / searchS, search_naive.cuh:24-127): F32-site
// distance from every query of the batch to every cached row.
__global__ void k_cache_scan(DevData d, const int *cache, int in_size, const int *qids, int nq, float r,
                             int *counts)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nq * in_size) return;
    int qi = t / in_size, e = t % in_size;
    int a = cache[e], b = qids[qi];
    float res;
    if (d.metric == kEdit) {
        res = (float)edit_dp(d.strs + (size_t)a * kStrStride, d.lens[a], d.strs + (size_t)b * kStrStride,
                             d.lens[b]);
    } else {
        res = dist_row_f32(d.rows + (size_t)a * d.dim, d.rows + (size_t)b * d.dim, d.dim, d.metric);
    }
    if (res <= r) atomicAdd(&counts[qi], 1);
}

namespace {

struct Fenwick {   // counts of live tree rows
    std::vector<int> t;
    int n = 0, log = 0;
    void init_all_live(int n_)
    {
        n = n_;
        t.assign((size_t)n + 1, 0);
        for (int i = 1; i <= n; i++) {
            t[i] += 1;
            int j = i + (i & -i);
            if (j <= n) t[j] += t[i];
        }
        log = 1;
        while ((1 << log) <= n) log++;
    }
    void add(int i, int v)
    {
        for (i++; i <= n; i += i & -i) t[i] += v;
    }
    // physical index of the (u+1)-th live row; caller checks u < live count
    int select(int u) const
    {
        int pos = 0, rem = u + 1;
        for (int b = log; b >= 0; b--) {
            int np = pos + (1 << b);
            if (np <= n && t[np] < rem) {
                pos = np;
                rem -= t[np];
            }
        }
        return pos;   // 0-based index of the row
    }
};

struct DevScratch {
    std::vector<void *> ps;
    ~DevScratch()
    {
        for (void *p : ps)
            if (p) cudaFree(p);
    }
    template <typename T>
    int alloc(T **p, size_t n)
    {
        int rc = dev_alloc(p, n, nullptr);
        if (rc == GTS_OK) ps.push_back(*p);
        return rc;
    }
};

}  // namespace

static int rebuild(gts_index *idx, const std::vector<uint8_t> &deleted, const std::vector<int> &cache,
                   cudaStream_t s)
{
    const int tree_size = idx->num;
    std::vector<int> map;
    map.reserve((size_t)tree_size + cache.size());
    for (int j = 0; j < tree_size; j++)
        if (!deleted[j]) map.push_back(j);
    for (int c : cache) map.push_back(c);
    const int n_new = (int)map.size();
    if (n_new < 1) {
        gts_set_error("update stream deleted every object");
        return GTS_ERR_INVALID;
    }
    DevScratch sc;
    int *d_map = nullptr;
    int rc;
    if ((rc = sc.alloc(&d_map, map.size()))) return rc;
    GTS_CUDA_TRY(cudaMemcpyAsync(d_map, map.data(), sizeof(int) * map.size(), cudaMemcpyHostToDevice, s));
    size_t acct = 0;
    if (idx->metric == kEdit) {
        char *ns = nullptr;
        int *nl = nullptr;
        if ((rc = dev_alloc(&ns, (size_t)n_new * kStrStride, &acct))) return rc;
        if ((rc = dev_alloc(&nl, (size_t)n_new, &acct))) { cudaFree(ns); return rc; }
        k_gather_strs<<<1184, 256, 0, s>>>(n_new, d_map, idx->strs, idx->lens, ns, nl);
        GTS_CUDA_TRY(cudaStreamSynchronize(s));
        cudaFree(idx->strs);
        cudaFree(idx->lens);
        idx->strs = ns;
        idx->lens = nl;
    } else {
        float *nr = nullptr;
        if ((rc = dev_alloc(&nr, (size_t)n_new * idx->dim, &acct))) return rc;
        k_gather_rows<<<1184, 256, 0, s>>>(n_new, idx->dim, d_map, idx->rows, nr);
        GTS_CUDA_TRY(cudaStreamSynchronize(s));
        cudaFree(idx->rows);
        idx->rows = nr;
    }
    free_tree(idx);
    idx->num = n_new;
    idx->device_bytes = acct;
    return build_tree(idx, s);
}

int update_run(gts_index *idx, const int *flags, const int *ids, int nops, float r, int *counts_out,
               int *nq_out, double *search_s, double *update_s)
{
    using clk = std::chrono::high_resolution_clock;
    cudaStream_t s = idx->stream;
    const int max_in = idx->params.max_in_size;
    double t_search = 0, t_update = 0;
    auto t0 = clk::now();

    int tree_size = idx->num, ndel = 0, rnum = 0, delete_id = 0, nq = 0;
    std::vector<int> cache;
    std::vector<uint8_t> deleted((size_t)tree_size, 0);
    std::vector<uint32_t> bitmap(((size_t)tree_size + 31) / 32, 0);
    Fenwick fw;
    fw.init_all_live(tree_size);

    DevScratch sc;
    uint32_t *d_bitmap = nullptr;
    int *d_q = nullptr, *d_cnt = nullptr, *d_ccnt = nullptr, *d_cache = nullptr;
    int rc;
    // query batches are bounded by the number of query ops
    int max_batch = 0;
    for (int i = 0; i < nops; i++) max_batch += flags[i] == 2;
    max_batch = std::max(1, std::min(max_batch, 65536));
    if ((rc = sc.alloc(&d_q, (size_t)max_batch)) || (rc = sc.alloc(&d_cnt, (size_t)max_batch)) ||
        (rc = sc.alloc(&d_ccnt, (size_t)max_batch)) || (rc = sc.alloc(&d_cache, (size_t)max_in + 1)))
        return rc;
    size_t bm_cap = bitmap.size();
    if ((rc = sc.alloc(&d_bitmap, bm_cap + 1))) return rc;
    GTS_CUDA_TRY(cudaMemsetAsync(d_bitmap, 0, sizeof(uint32_t) * (bm_cap + 1), s));
    bool bitmap_dirty = false;
    std::vector<int> qbuf, cbuf, ccbuf;
    t_update += std::chrono::duration<double>(clk::now() - t0).count();

    int i = 0;
    while (i < nops) {
        int f = flags[i];
        if (f == 0) {   // insert
            auto ts = clk::now();
            if (ids[i] >= tree_size) {
                gts_set_error("op %d inserts row %d, data has %d rows", i, ids[i], tree_size);
                return GTS_ERR_INVALID;
            }
            cache.push_back(ids[i]);
            if ((int)cache.size() == max_in) {
                if ((rc = rebuild(idx, deleted, cache, s))) return rc;
                tree_size = idx->num;
                ndel = 0;
                cache.clear();
                deleted.assign((size_t)tree_size, 0);
                bitmap.assign(((size_t)tree_size + 31) / 32, 0);
                fw.init_all_live(tree_size);
                if (bitmap.size() > bm_cap) {
                    cudaFree(d_bitmap);
                    sc.ps.erase(std::find(sc.ps.begin(), sc.ps.end(), (void *)d_bitmap));
                    bm_cap = bitmap.size();
                    if ((rc = sc.alloc(&d_bitmap, bm_cap + 1))) return rc;
                }
                GTS_CUDA_TRY(cudaMemsetAsync(d_bitmap, 0, sizeof(uint32_t) * (bm_cap + 1), s));
                bitmap_dirty = false;
            }
            t_update += std::chrono::duration<double>(clk::now() - ts).count();
            i++;
        } else if (f == 1) {   // delete
            auto ts = clk::now();
            int u = ids[i];
            int live_tree = tree_size - ndel;
            if (u >= 0 && u < live_tree) delete_id = fw.select(u);
            else if (u >= live_tree && u < live_tree + (int)cache.size()) delete_id = tree_size + (u - live_tree);
            if (delete_id < tree_size) {
                if (!deleted[delete_id]) {
                    deleted[delete_id] = 1;
                    bitmap[delete_id >> 5] |= 1u << (delete_id & 31);
                    fw.add(delete_id, -1);
                    ndel++;
                    bitmap_dirty = true;
                }
            } else if (!cache.empty()) {
                size_t e = (size_t)(delete_id - tree_size);
                if (e < cache.size()) cache.erase(cache.begin() + (long)e);
                else cache.pop_back();
            }
            t_update += std::chrono::duration<double>(clk::now() - ts).count();
            i++;
        } else {   // a run of consecutive queries: one batched launch
            auto ts = clk::now();
            qbuf.clear();
            while (i < nops && flags[i] == 2 && (int)qbuf.size() < max_batch) {
                int q = ids[i++];
                if (q < 0 || q >= tree_size) {
                    gts_set_error("update query id %d out of range [0, %d)", q, tree_size);
                    return GTS_ERR_INVALID;
                }
                qbuf.push_back(q);
            }
            const int nb = (int)qbuf.size();
            if (bitmap_dirty) {
                GTS_CUDA_TRY(cudaMemcpyAsync(d_bitmap, bitmap.data(), sizeof(uint32_t) * bitmap.size(),
                                             cudaMemcpyHostToDevice, s));
                bitmap_dirty = false;
            }
            GTS_CUDA_TRY(cudaMemcpyAsync(d_q, qbuf.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
            if ((rc = search_range(idx, d_q, nb, r, d_cnt, d_bitmap, s))) return rc;
            cbuf.resize(nb);
            GTS_CUDA_TRY(cudaMemcpyAsync(cbuf.data(), d_cnt, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
            const int in_size = (int)cache.size();
            if (in_size > 0) {
                GTS_CUDA_TRY(cudaMemcpyAsync(d_cache, cache.data(), sizeof(int) * in_size, cudaMemcpyHostToDevice, s));
                GTS_CUDA_TRY(cudaMemsetAsync(d_ccnt, 0, sizeof(int) * nb, s));
                DevData dd{idx->dim, idx->num, idx->metric, idx->rows, idx->strs, idx->lens};
                int work = nb * in_size;
                k_cache_scan<<<(work + 127) / 128, 128, 0, s>>>(dd, d_cache, in_size, d_q, nb, r, d_ccnt);
                GTS_CUDA_TRY(cudaGetLastError());
                ccbuf.resize(nb);
                GTS_CUDA_TRY(cudaMemcpyAsync(ccbuf.data(), d_ccnt, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
            }
            GTS_CUDA_TRY(cudaStreamSynchronize(s));
            for (int j = 0; j < nb; j++) {
                if (in_size > 0) rnum = ccbuf[j];
                counts_out[nq++] = cbuf[j] + rnum;
            }
            t_search += std::chrono::duration<double>(clk::now() - ts).count();
        }
    }
    if (nq_out) *nq_out = nq;
    if (search_s) *search_s = t_search;
    if (update_s) *update_s = t_update;
    return GTS_OK;
}

}  // namespace gts

extern "C" int gts_update_run(gts_index *idx, const int *flags, const int *ids, int nops, float r,
                              int *counts_out, int *nq_out, double *search_s, double *update_s)
{
    if (!idx || nops < 0 || (nops > 0 && (!flags || !ids || !counts_out))) {
        gts_set_error("gts_update_run: invalid argument");
        return GTS_ERR_INVALID;
    }
    for (int i = 0; i < nops; i++) {
        if (flags[i] < 0 || flags[i] > 2) {
            gts_set_error("op %d has flag %d (expected 0, 1 or 2)", i, flags[i]);
            return GTS_ERR_INVALID;
        }
        if (flags[i] == 0 && ids[i] < 0) {
            gts_set_error("op %d inserts negative id %d", i, ids[i]);
            return GTS_ERR_INVALID;
        }
    }
    return gts::update_run(idx, flags, ids, nops, r, counts_out, nq_out, search_s, update_s);
}
