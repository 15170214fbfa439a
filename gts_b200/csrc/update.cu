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
//
// How it runs here.  An insert copies an existing row, so every object that
// ever exists in the stream is a copy of a row of the data the index was
// built on.  One host pass over the operations (O(log N) each, two Fenwick
// trees) keeps the reference's id bookkeeping and gives every entry -- the
// original rows and every inserted copy -- the operation intervals during
// which it is live in the tree and in the cache list; it gives every query
// its object and operation index.  All queries of the stream then run as ONE
// batched launch of the range traversal over the unchanged tree
// (kModeRangeTimed, search.cu): an object within r adds its entries live at
// the query's operation.  The per-query cache counts, with the reference's
// stale count for an empty cache, are combined on the host.  Physical ids
// follow from store order: the data array after a compaction is exactly the
// entries live at that compaction, in store order (original rows first, then
// the copies in insertion order).  The compactions themselves therefore cost
// no rebuild; one rebuild at the end leaves the handle holding the data of
// the last compaction, as the reference's does.  Results are identical to
// running the rebuilds, since every count is exact.
#include <algorithm>
#include <chrono>
#include <climits>
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

namespace {

// Counts over [0, cap): the first n_live positions start at 1.
struct Fenwick {
    std::vector<int> t;
    int n = 0, log = 0;
    void init(int cap, int n_live)
    {
        n = cap;
        t.assign((size_t)n + 1, 0);
        for (int i = 1; i <= n; i++) {
            if (i <= n_live) t[i] += 1;
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
    // sum over [0, i)
    int prefix(int i) const
    {
        int r = 0;
        for (; i > 0; i -= i & -i) r += t[i];
        return r;
    }
    // position of the (u+1)-th counted position; caller checks u < total
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
        return pos;
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

constexpr int kNever = INT_MAX;

}  // namespace

// The outcome of the host pass over an update stream.
struct StreamPlan {
    std::vector<int> src;      // per entry: the row of the built data it copies
    std::vector<int4> life;    // per entry: (tree_from, tree_to, cache_from, cache_to)
    std::vector<int> q_obj, q_time;
    std::vector<uint8_t> q_cache;   // the cache list was non-empty at the query
    std::vector<int> final_rows;    // data after the last compaction (empty: none)
};

// The reference's bookkeeping of update.cuh:473-623 over entries in store
// order.  fphys counts the entries live at the last compaction (their rank
// is the physical id); flive the tree entries live now (their rank is the
// logical id of a delete).
// new_base < 0: an insert copies physical row ids[i] (the reference);
// otherwise it brings new row ids[i] (0 <= ids[i] < n_new), whose index
// object is new_base + ids[i].
int plan_stream(int n0, const int *flags, const int *ids, int nops, int max_in, int new_base, int n_new,
                StreamPlan *P)
{
    int n_ins = 0;
    for (int i = 0; i < nops; i++) n_ins += flags[i] == 0;
    const int cap = n0 + n_ins;
    P->src.resize((size_t)n0);
    for (int i = 0; i < n0; i++) P->src[i] = i;
    P->src.reserve((size_t)cap);
    P->life.assign((size_t)n0, make_int4(-1, kNever, kNever, kNever));
    P->life.reserve((size_t)cap);
    Fenwick fphys, flive;
    fphys.init(cap, n0);
    flive.init(cap, n0);
    int tree_size = n0, ndel = 0, delete_id = 0;
    bool compacted = false;
    std::vector<int> cache, pending;
    for (int i = 0; i < nops; i++) {
        const int f = flags[i];
        if (f == 0) {   // insert: a copy of physical row ids[i] (or new row ids[i]) joins the cache list
            if (new_base < 0 ? ids[i] >= tree_size : (ids[i] < 0 || ids[i] >= n_new)) {
                gts_set_error("op %d inserts %s %d (%d available)", i, new_base < 0 ? "row" : "new row", ids[i],
                              new_base < 0 ? tree_size : n_new);
                return GTS_ERR_INVALID;
            }
            const int e = (int)P->src.size();
            P->src.push_back(new_base < 0 ? P->src[fphys.select(ids[i])] : new_base + ids[i]);
            P->life.push_back(make_int4(kNever, kNever, i, kNever));
            cache.push_back(e);
            if ((int)cache.size() == max_in) {   // compaction (update.cuh:484-540)
                for (int p : pending) fphys.add(p, -1);
                for (int c : cache) {
                    P->life[c].x = i;   // in the tree from here on
                    P->life[c].w = i;   // out of the cache list
                    fphys.add(c, 1);
                    flive.add(c, 1);
                }
                tree_size = tree_size - ndel + (int)cache.size();
                ndel = 0;
                cache.clear();
                pending.clear();
                compacted = true;
            }
        } else if (f == 1) {   // delete (update.cuh:546-582)
            const int u = ids[i];
            const int live_tree = tree_size - ndel;
            if (u >= 0 && u < live_tree) delete_id = fphys.prefix(flive.select(u));
            else if (u >= live_tree && u < live_tree + (int)cache.size()) delete_id = tree_size + (u - live_tree);
            if (delete_id < tree_size) {
                const int e = fphys.select(delete_id);
                if (P->life[e].y == kNever) {
                    P->life[e].y = i;
                    flive.add(e, -1);
                    pending.push_back(e);
                    ndel++;
                }
            } else if (!cache.empty()) {
                size_t c = (size_t)(delete_id - tree_size);
                if (c >= cache.size()) c = cache.size() - 1;
                P->life[cache[c]].w = i;
                cache.erase(cache.begin() + (long)c);
            }
        } else {   // query: physical row ids[i] (update.cuh:588)
            const int q = ids[i];
            if (q < 0 || q >= tree_size) {
                gts_set_error("update query id %d out of range [0, %d)", q, tree_size);
                return GTS_ERR_INVALID;
            }
            P->q_obj.push_back(P->src[fphys.select(q)]);
            P->q_time.push_back(i);
            P->q_cache.push_back(cache.empty() ? 0 : 1);
        }
    }
    P->final_rows.clear();
    if (compacted) {
        P->final_rows.reserve((size_t)tree_size);
        for (int e = 0; e < (int)P->src.size(); e++)
            if (fphys.prefix(e + 1) - fphys.prefix(e)) P->final_rows.push_back(P->src[e]);
        if (P->final_rows.empty()) {
            gts_set_error("update stream deleted every object");
            return GTS_ERR_INVALID;
        }
    }
    return GTS_OK;
}

// The data after the last compaction (rows `map` of the current data, in
// order), and the index rebuilt on it.
static int rebuild_on(gts_index *idx, const std::vector<int> &map, cudaStream_t s)
{
    const int n_new = (int)map.size();
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

// new_rows (host, n_new x dim floats; nullable): inserts bring these rows.
// They are known before the stream runs, so the index is first rebuilt on
// the data rows followed by the new rows; a new row is an object of that
// index whose only entries are its inserts (none: it never counts).
int update_run(gts_index *idx, const int *flags, const int *ids, int nops, float r, int *counts_out,
               int *nq_out, double *search_s, double *update_s, const float *new_rows, int n_new)
{
    using clk = std::chrono::high_resolution_clock;
    cudaStream_t s = idx->stream;
    auto t0 = clk::now();
    const int n_data = idx->num;
    StreamPlan P;
    int rc = plan_stream(n_data, flags, ids, nops, idx->params.max_in_size, new_rows ? n_data : -1, n_new, &P);
    if (rc) return rc;
    if (new_rows && n_new > 0) {
        // the data rows, then the new rows; the tree over both
        float *all = nullptr;
        size_t acct = 0;
        const size_t dim = (size_t)idx->dim;
        if ((rc = dev_alloc(&all, ((size_t)n_data + n_new) * dim, &acct))) return rc;
        GTS_CUDA_TRY(cudaMemcpyAsync(all, idx->rows, sizeof(float) * n_data * dim, cudaMemcpyDeviceToDevice, s));
        GTS_CUDA_TRY(cudaMemcpyAsync(all + (size_t)n_data * dim, new_rows, sizeof(float) * (size_t)n_new * dim,
                                     cudaMemcpyHostToDevice, s));
        GTS_CUDA_TRY(cudaStreamSynchronize(s));
        cudaFree(idx->rows);
        idx->rows = all;
        free_tree(idx);
        idx->num = n_data + n_new;
        idx->device_bytes = acct;
        if ((rc = build_tree(idx, s))) return rc;
        if (P.final_rows.empty()) {   // no compaction: the handle keeps the data rows
            P.final_rows.resize((size_t)n_data);
            for (int i = 0; i < n_data; i++) P.final_rows[i] = i;
        }
    }
    const int nq = (int)P.q_obj.size();
    double t_update = std::chrono::duration<double>(clk::now() - t0).count();
    double t_search = 0;
    if (nq > 0) {
        auto ts = clk::now();
        // entries grouped by the row they copy (CSR over the built data)
        const int n0 = idx->num;
        const size_t ne = P.src.size();
        std::vector<int> off((size_t)n0 + 1, 0);
        for (size_t e = 0; e < ne; e++) off[(size_t)P.src[e] + 1]++;
        for (int i = 0; i < n0; i++) off[(size_t)i + 1] += off[i];
        std::vector<int4> ents(ne);
        {
            std::vector<int> fill(off.begin(), off.end() - 1);
            for (size_t e = 0; e < ne; e++) ents[(size_t)fill[P.src[e]]++] = P.life[e];
        }
        // the entries stay resident; the queries run in batches of 16 bytes
        // each (id, time, two counts) within the call's budget
        const size_t fixed = sizeof(int) * off.size() + sizeof(int4) * ne + 1024;
        const size_t budget = search_budget(idx);
        if (fixed + 16 > budget) {
            gts_set_error("scratch budget of %zu bytes is below the %zu bytes of the stream's entries", budget,
                          fixed + 16);
            return GTS_ERR_NOMEM;
        }
        const int qc = (int)std::min<size_t>((size_t)nq, (budget - fixed) / 16);
        DevScratch sc;
        int *d_off = nullptr, *d_q = nullptr, *d_t = nullptr, *d_ct = nullptr, *d_cc = nullptr;
        int4 *d_ents = nullptr;
        if ((rc = sc.alloc(&d_off, off.size())) || (rc = sc.alloc(&d_ents, ne)) ||
            (rc = sc.alloc(&d_q, (size_t)qc)) || (rc = sc.alloc(&d_t, (size_t)qc)) ||
            (rc = sc.alloc(&d_ct, (size_t)qc)) || (rc = sc.alloc(&d_cc, (size_t)qc)))
            return rc;
        GTS_CUDA_TRY(cudaMemcpyAsync(d_off, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice, s));
        GTS_CUDA_TRY(cudaMemcpyAsync(d_ents, ents.data(), sizeof(int4) * ne, cudaMemcpyHostToDevice, s));
        std::vector<int> ct((size_t)nq), cc((size_t)nq);
        for (int q0 = 0; q0 < nq; q0 += qc) {
            const int n = std::min(qc, nq - q0);
            GTS_CUDA_TRY(cudaMemcpyAsync(d_q, P.q_obj.data() + q0, sizeof(int) * n, cudaMemcpyHostToDevice, s));
            GTS_CUDA_TRY(cudaMemcpyAsync(d_t, P.q_time.data() + q0, sizeof(int) * n, cudaMemcpyHostToDevice, s));
            if ((rc = search_range_timed(idx, d_q, d_t, n, r, d_off, d_ents, d_ct, d_cc, s))) return rc;
            GTS_CUDA_TRY(cudaMemcpyAsync(ct.data() + q0, d_ct, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
            GTS_CUDA_TRY(cudaMemcpyAsync(cc.data() + q0, d_cc, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
        }
        GTS_CUDA_TRY(cudaStreamSynchronize(s));
        int rnum = 0;   // the cache count of the last query that had a cache (update.cuh:592-597)
        for (int j = 0; j < nq; j++) {
            if (P.q_cache[j]) rnum = cc[j];
            counts_out[j] = ct[j] + rnum;
        }
        t_search = std::chrono::duration<double>(clk::now() - ts).count();
    }
    if (!P.final_rows.empty()) {
        auto tr = clk::now();
        if ((rc = rebuild_on(idx, P.final_rows, s))) return rc;
        t_update += std::chrono::duration<double>(clk::now() - tr).count();
    }
    if (nq_out) *nq_out = nq;
    if (search_s) *search_s = t_search;
    if (update_s) *update_s = t_update;
    return GTS_OK;
}

}  // namespace gts

extern "C" int gts_update_plan(int num, const int *flags, const int *ids, int nops, int max_in_size, int n_new,
                               int *q_obj, int *q_time, int *q_cache, int *n_q, int *ent_src, int *ent_life,
                               int *n_ent, int *final_rows, int *n_final)
{
    if (num < 1 || nops < 0 || max_in_size < 1 || n_new < 0 || (nops > 0 && (!flags || !ids)) || !n_q || !n_ent ||
        !n_final) {
        gts_set_error("gts_update_plan: invalid argument");
        return GTS_ERR_INVALID;
    }
    for (int i = 0; i < nops; i++) {
        if (flags[i] < 0 || flags[i] > 2 || (flags[i] == 0 && ids[i] < 0)) {
            gts_set_error("op %d is (%d, %d)", i, flags[i], ids[i]);
            return GTS_ERR_INVALID;
        }
    }
    gts::StreamPlan P;
    int rc = gts::plan_stream(num, flags, ids, nops, max_in_size, n_new > 0 ? num : -1, n_new, &P);
    if (rc) return rc;
    *n_q = (int)P.q_obj.size();
    *n_ent = (int)P.src.size();
    *n_final = (int)P.final_rows.size();
    for (size_t j = 0; j < P.q_obj.size(); j++) {
        if (q_obj) q_obj[j] = P.q_obj[j];
        if (q_time) q_time[j] = P.q_time[j];
        if (q_cache) q_cache[j] = P.q_cache[j];
    }
    for (size_t e = 0; e < P.src.size(); e++) {
        if (ent_src) ent_src[e] = P.src[e];
        if (ent_life) {
            ent_life[4 * e + 0] = P.life[e].x;
            ent_life[4 * e + 1] = P.life[e].y;
            ent_life[4 * e + 2] = P.life[e].z;
            ent_life[4 * e + 3] = P.life[e].w;
        }
    }
    if (final_rows)
        for (size_t i = 0; i < P.final_rows.size(); i++) final_rows[i] = P.final_rows[i];
    return GTS_OK;
}

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
    return gts::update_run(idx, flags, ids, nops, r, counts_out, nq_out, search_s, update_s, nullptr, 0);
}

extern "C" int gts_update_run_rows(gts_index *idx, const int *flags, const int *ids, int nops, const float *new_rows,
                                   int n_new, float r, int *counts_out, int *nq_out, double *search_s,
                                   double *update_s)
{
    if (!idx || nops < 0 || n_new < 0 || (nops > 0 && (!flags || !ids || !counts_out)) || (n_new > 0 && !new_rows)) {
        gts_set_error("gts_update_run_rows: invalid argument");
        return GTS_ERR_INVALID;
    }
    if (idx->metric == 6) {
        gts_set_error("gts_update_run_rows: new rows need a row metric (not edit distance)");
        return GTS_ERR_INVALID;
    }
    for (int i = 0; i < nops; i++) {
        if (flags[i] < 0 || flags[i] > 2) {
            gts_set_error("op %d has flag %d (expected 0, 1 or 2)", i, flags[i]);
            return GTS_ERR_INVALID;
        }
        if (flags[i] == 0 && (ids[i] < 0 || ids[i] >= n_new)) {
            gts_set_error("op %d inserts new row %d of %d", i, ids[i], n_new);
            return GTS_ERR_INVALID;
        }
    }
    return gts::update_run(idx, flags, ids, nops, r, counts_out, nq_out, search_s, update_s, new_rows, n_new);
}
