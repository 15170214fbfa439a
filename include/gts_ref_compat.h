/*
 * gts_ref_compat.h -- the reference's C++ entry points over the C ABI.
 *
 * A program written against the reference headers (Source Code/GTS/include:
 * tree.cuh, file.cuh, search.cuh, search_v2.cuh, update.cuh, config.cuh)
 * compiles against this header instead and runs on libgts_b200: same
 * function names, argument lists and ownership (every array it returns is a
 * CUDA managed allocation the caller frees with cudaFree, as the
 * reference's are), same globals (res, res_dis, update_list, update_num and
 * the tunables).  include/gts_ref/ holds one-line headers named like the
 * reference's, so the reference's own src/main.cu builds unchanged with
 * `-I include/gts_ref` and links with -lgts_b200.
 *
 * Differences from the reference, by design:
 *   * the tree arrays (id_list, node_list, max_node_num, empty_list) are
 *     copies of the index the library holds; the searches take the index
 *     from node_list (the pointer indexConstru returned), not from the
 *     arrays' contents;
 *   * searches are exact on every tree shape (the reference skips shallow
 *     leaves and oversized last-level nodes); they run the tensor-core form
 *     where the index allows it (L2, dim <= 128), else the plain traversal;
 *   * the v1 searches return their outputs (the reference frees them before
 *     it returns, search.cuh:866-888, 1066-1081);
 *   * errors print the library's message and exit(1), like CHECK
 *     (tree.cuh:19-29).
 *
 * Single-threaded, like the reference.  C++17 (inline variables).
 */
#ifndef GTS_REF_COMPAT_H
#define GTS_REF_COMPAT_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>
#include <cuda_runtime_api.h>
#include "gts_b200.h"

/* TN (tree.cuh:37-44) and UO (update.cuh:18-22). */
struct TN {
    int pid;
    float min_dis;
    int size;
    int lid;
    int is_leaf;
};
struct UO {
    int update_flag;
    int update_id;
};

/* Tunables (tree.cuh:31-35, update.cuh:16): read by indexConstru and
 * updateIndexRnn.  Plain host variables here (the reference's are
 * __managed__); set them before indexConstru. */
inline int TREE_ORDER = 10;
inline int MAX_SIZE = 20;
inline int MAX_H = 3;
inline int DIS_CODE = 100;
inline int INFI_DIS = 10000;
inline int MAX_IN_SIZE = 10;

/* Outputs of the v2 searches (search_v2.cuh:19-20) and the update list
 * loadUpdate fills (update.cuh:23-24). */
inline int *res = nullptr;
inline float *res_dis = nullptr;
inline int update_num = 0;
inline UO *update_list = nullptr;

namespace gts_ref {

inline void die(const char *what)
{
    fprintf(stderr, "%s failed: %s\n", what, gts_last_error());
    exit(1);
}

inline void check(int rc, const char *what)
{
    if (rc != GTS_OK) die(what);
}

template <typename T>
inline T *managed(size_t n)
{
    T *p = nullptr;
    if (cudaMallocManaged((void **)&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) {
        fprintf(stderr, "cudaMallocManaged of %zu bytes failed\n", n * sizeof(T));
        exit(1);
    }
    return p;
}

/* The library index behind each node_list indexConstru returned. */
inline std::map<const void *, gts_index *> &handles()
{
    static std::map<const void *, gts_index *> m;
    return m;
}

inline gts_index *handle_of(const TN *node_list)
{
    auto it = handles().find(node_list);
    if (it == handles().end()) {
        fprintf(stderr, "node_list was not returned by indexConstru\n");
        exit(1);
    }
    return it->second;
}

inline gts_params current_params()
{
    gts_params p;
    gts_params_default(&p);
    p.tree_order = TREE_ORDER;
    p.max_size = MAX_SIZE;
    p.max_h = MAX_H;
    p.dis_code = DIS_CODE;
    p.infi_dis = INFI_DIS;
    p.max_in_size = MAX_IN_SIZE;
    return p;
}

/* The reference-shaped tree arrays of idx, in new managed allocations. */
inline void export_tree(gts_index *idx, int *&id_list, TN *&node_list, int *&max_node_num, int &tree_h,
                        int *&empty_list)
{
    gts_index_info info;
    check(gts_index_info_get(idx, &info), "indexConstru");
    const int m = info.max_node_num, n = info.num;
    std::vector<int> pid(m), size(m), lid(m), leaf(m), exists(m);
    std::vector<float> md(m);
    id_list = managed<int>(n);
    check(gts_index_export(idx, id_list, pid.data(), md.data(), size.data(), lid.data(), leaf.data(),
                           exists.data()),
          "indexConstru");
    node_list = managed<TN>(m);
    empty_list = managed<int>(m);
    for (int i = 0; i < m; i++) {
        node_list[i] = TN{pid[i], md[i], size[i], lid[i], leaf[i]};
        empty_list[i] = exists[i] ? 0 : 0x01010101;   // tree.cuh:347 sets absent nodes' bytes to 1
    }
    max_node_num = managed<int>(1);
    max_node_num[0] = m;
    tree_h = info.tree_h;
}

}  // namespace gts_ref

/* ---------------------------------------------------------------- I/O */

/* load (file.cuh:28): header "dim num metric", then the objects. */
inline void load(char *file, int *&data_info, float *&data_d, char *&data_s, int *&size_s)
{
    int dim = 0, num = 0, metric = 0;
    float *rows = nullptr;
    char *strs = nullptr;
    int *lens = nullptr;
    if (gts_load(file, &dim, &num, &metric, &rows, &strs, &lens) != GTS_OK) {
        fprintf(stderr, "open file error: %s\n", gts_last_error());
        exit(-1);   // file.cuh:33-37
    }
    data_info = gts_ref::managed<int>(3);
    data_info[0] = dim;
    data_info[1] = num;
    data_info[2] = metric;
    data_d = nullptr;
    data_s = nullptr;
    size_s = nullptr;
    if (metric == GTS_METRIC_EDIT) {
        data_s = gts_ref::managed<char>((size_t)num * GTS_STR_STRIDE);
        size_s = gts_ref::managed<int>((size_t)num);
        memcpy(data_s, strs, (size_t)num * GTS_STR_STRIDE);
        memcpy(size_s, lens, sizeof(int) * (size_t)num);
    } else {
        data_d = gts_ref::managed<float>((size_t)num * dim);
        memcpy(data_d, rows, sizeof(float) * (size_t)num * dim);
    }
    gts_free_host(rows);
    gts_free_host(strs);
    gts_free_host(lens);
}

/* loadQuery (file.cuh:112). */
inline void loadQuery(char *file, int *&qid, int &qnum)
{
    int *q = nullptr;
    if (gts_load_queries(file, &q, &qnum) != GTS_OK) {
        fprintf(stderr, "open file error: %s\n", gts_last_error());
        exit(-1);
    }
    qid = gts_ref::managed<int>((size_t)qnum);
    memcpy(qid, q, sizeof(int) * (size_t)qnum);
    gts_free_host(q);
}

/* loadUpdate (update.cuh:43). */
inline void loadUpdate(char *file, UO *&list, int &num)
{
    int *f = nullptr, *i = nullptr;
    if (gts_load_updates(file, &f, &i, &num) != GTS_OK) {
        fprintf(stderr, "open file error: %s\n", gts_last_error());
        exit(-1);
    }
    list = gts_ref::managed<UO>((size_t)num);
    for (int j = 0; j < num; j++) list[j] = UO{f[j], i[j]};
    gts_free_host(f);
    gts_free_host(i);
}

/* saveK (file.cuh:154): k ids / k distances per query line. */
inline void saveK(char *filenamer, char *filenamed, int *res_id, float *dis, int k, int qnum)
{
    FILE *fr = fopen(filenamer, "w"), *fd = fopen(filenamed, "w");
    if (!fr || !fd) gts_ref::die("saveK");
    for (int i = 0; i < qnum; i++) {
        for (int j = 0; j < k; j++) {
            fprintf(fr, "%d ", res_id[(size_t)i * k + j]);
            fprintf(fd, "%f ", dis[(size_t)i * k + j]);
        }
        fprintf(fr, "\n");
        fprintf(fd, "\n");
    }
    fclose(fr);
    fclose(fd);
}

/* saveR (file.cuh:178): appended, one line of hits per query. */
inline void saveR(char *filenamer, char *filenamed, int *res_id, float *dis, int *qresult_count,
                  int *qresult_count_prefix, int qnum)
{
    FILE *fr = fopen(filenamer, "a"), *fd = fopen(filenamed, "a");
    if (!fr || !fd) gts_ref::die("saveR");
    for (int i = 0; i < qnum; i++) {
        for (int j = qresult_count_prefix[i]; j < qresult_count_prefix[i] + qresult_count[i]; j++) {
            fprintf(fr, "%d ", res_id[j]);
            fprintf(fd, "%f ", dis[j]);
        }
        fprintf(fr, "\n");
        fprintf(fd, "\n");
    }
    fclose(fr);
    fclose(fd);
}

/* ---------------------------------------------------------------- index */

/* indexConstru (tree.cuh:332-393). */
inline void indexConstru(float *data_d, char *data_s, int *size_s, int *data_info, int *&id_list,
                         TN *&node_list, int *&max_node_num, int &tree_h, int *&empty_list)
{
    printf("Index construction...\n");
    const gts_params p = gts_ref::current_params();
    gts_index *idx = nullptr;
    gts_ref::check(gts_index_build(data_info[0], data_info[1], data_info[2], data_d, data_s, size_s, &p, &idx),
                   "indexConstru");
    gts_ref::export_tree(idx, id_list, node_list, max_node_num, tree_h, empty_list);
    gts_ref::handles()[node_list] = idx;
}

/* ---------------------------------------------------------------- search v2 */

/* searchIndexKnnV2 (search_v2.cuh:975-1228): res_dis[q] = the k-th
 * distance of query qid_list[q] (allocated here, as the reference does). */
inline void searchIndexKnnV2(float *data_d, TN *node_list, int *id_list, int *max_node_num, int *qid_list,
                             int qnum, int k, int tree_h, int *data_info, int *empty_list, char *data_s,
                             int *size_s)
{
    (void)data_d; (void)id_list; (void)max_node_num; (void)tree_h; (void)data_info; (void)empty_list;
    (void)data_s; (void)size_s;
    printf("Searching...\n");
    res_dis = gts_ref::managed<float>((size_t)qnum);
    gts_ref::check(gts_knn(gts_ref::handle_of(node_list), qid_list, qnum, k, GTS_FORM_FAST, res_dis, nullptr,
                           nullptr),
                   "searchIndexKnnV2");
}

/* searchIndexRnnV2 (search_v2.cuh:780-972): res[q] = the number of objects
 * within r of query qid_list[q]. */
inline void searchIndexRnnV2(float *data_d, TN *node_list, int *id_list, int *max_node_num, int *qid_list,
                             int qnum, float r, int tree_h, int *data_info, int *empty_list, char *data_s,
                             int *size_s)
{
    (void)data_d; (void)id_list; (void)max_node_num; (void)tree_h; (void)data_info; (void)empty_list;
    (void)data_s; (void)size_s;
    printf("Searching...\n");
    res = gts_ref::managed<int>((size_t)qnum);
    gts_ref::check(gts_range_form(gts_ref::handle_of(node_list), qid_list, qnum, r, GTS_FORM_FAST, res),
                   "searchIndexRnnV2");
}

/* ---------------------------------------------------------------- search v1 */

/* searchIndexRnn (search.cuh:749-889): every query's hits.  qresult_count /
 * qresult_count_prefix (qnum each) and result_id / result_dis (the hits of
 * query i at prefix[i] .. prefix[i] + count[i], by (distance, id)) are new
 * managed allocations.  fcost receives the counts ("%d "). */
inline void searchIndexRnn(float *data_d, TN *node_list, int *id_list, int *max_node_num, int *qid_list,
                           int qnum, float r, int tree_h, int *data_info, int *empty_list, int *&qresult_count,
                           int *&qresult_count_prefix, int *&result_id, float *&result_dis, char *data_s,
                           int *size_s, float &time_search, FILE *&fcost)
{
    (void)data_d; (void)id_list; (void)max_node_num; (void)tree_h; (void)data_info; (void)empty_list;
    (void)data_s; (void)size_s;
    printf("Search...\n");
    gts_index *idx = gts_ref::handle_of(node_list);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    qresult_count = gts_ref::managed<int>((size_t)qnum);
    qresult_count_prefix = gts_ref::managed<int>((size_t)qnum);
    gts_ref::check(gts_range(idx, qid_list, qnum, r, qresult_count), "searchIndexRnn");
    size_t total = 0;
    for (int i = 0; i < qnum; i++) total += (size_t)qresult_count[i];
    result_id = gts_ref::managed<int>(total);
    result_dis = gts_ref::managed<float>(total);
    gts_ref::check(gts_range_ids(idx, qid_list, qnum, r, qresult_count, qresult_count_prefix, result_id,
                                 result_dis, total),
                   "searchIndexRnn");
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    time_search += ms / 1e3f;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (fcost)
        for (int i = 0; i < qnum; i++) fprintf(fcost, "%d ", qresult_count[i]);
}

/* searchIndexKnn (search.cuh:891-1081): k ids and distances per query at
 * result_id / result_dis[i*k .. i*k + k) by (distance, id); qresult_count[i]
 * = k and qresult_count_prefix[i] = i*k.  fcost receives the k-th
 * distances ("%f "). */
inline void searchIndexKnn(float *data_d, TN *node_list, int *id_list, int *max_node_num, int *qid_list,
                           int qnum, int k, int tree_h, int *data_info, int *empty_list, int *&result_id,
                           float *&result_dis, int *&qresult_count, int *&qresult_count_prefix, char *data_s,
                           int *size_s, float &time_search, FILE *fcost)
{
    (void)data_d; (void)id_list; (void)max_node_num; (void)tree_h; (void)data_info; (void)empty_list;
    (void)data_s; (void)size_s;
    printf("Search...\n");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    std::vector<float> kth((size_t)qnum);
    result_id = gts_ref::managed<int>((size_t)qnum * k);
    result_dis = gts_ref::managed<float>((size_t)qnum * k);
    gts_ref::check(gts_knn(gts_ref::handle_of(node_list), qid_list, qnum, k, GTS_FORM_FAST, kth.data(),
                           result_id, result_dis),
                   "searchIndexKnn");
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    time_search += ms / 1e3f;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    qresult_count = gts_ref::managed<int>((size_t)qnum);
    qresult_count_prefix = gts_ref::managed<int>((size_t)qnum);
    for (int i = 0; i < qnum; i++) {
        qresult_count[i] = k;
        qresult_count_prefix[i] = i * k;
        if (fcost) fprintf(fcost, "%f ", kth[i]);
    }
}

/* ---------------------------------------------------------------- update */

/* updateIndexRnn (update.cuh:449-638): the operations of update_list
 * (loadUpdate) through the lazy cache list of MAX_IN_SIZE entries; fcost
 * receives every query op's count ("%d ").  Afterwards data_d / data_s /
 * size_s / data_info hold the data after the last compaction and the tree
 * arrays its tree (new managed allocations; the old ones are freed), as in
 * the reference.  time_update_s / time_update_u gain the search and the
 * bookkeeping time, count_update_s / count_update_u the query and the
 * insert / delete ops. */
inline void updateIndexRnn(float *&data_d, TN *&node_list, int *&id_list, int *&max_node_num, int *&qid_list,
                           int qnum, float r, int &tree_h, int *&data_info, int *&empty_list,
                           int *&qresult_count, int *&qresult_count_prefix, int *&result_id,
                           float *&result_dis, char *&data_s, int *&size_s, FILE *fcost, float &time_update_s,
                           float &time_update_u, int &count_update_s, int &count_update_u)
{
    (void)qid_list; (void)qnum; (void)qresult_count; (void)qresult_count_prefix; (void)result_id;
    (void)result_dis;
    printf("Updating...\n");
    gts_index *idx = gts_ref::handle_of(node_list);
    const int n = update_num, num0 = data_info[1];
    std::vector<int> flags((size_t)n), ids((size_t)n);
    int nq = 0;
    for (int i = 0; i < n; i++) {
        flags[i] = update_list[i].update_flag;
        ids[i] = update_list[i].update_id;
        nq += flags[i] == 2;
    }
    // the data after the last compaction, from the stream's bookkeeping
    int n_ent = 0, n_final = 0, n_q = 0;
    std::vector<int> final_rows((size_t)num0 + n);
    gts_ref::check(gts_update_plan(num0, flags.data(), ids.data(), n, MAX_IN_SIZE, 0, nullptr, nullptr, nullptr,
                                   &n_q, nullptr, nullptr, &n_ent, final_rows.data(), &n_final),
                   "updateIndexRnn");
    std::vector<int> counts((size_t)(nq > 0 ? nq : 1));
    double ts = 0, tu = 0;
    gts_ref::check(gts_update_run(idx, flags.data(), ids.data(), n, r, counts.data(), &nq, &ts, &tu),
                   "updateIndexRnn");
    if (fcost) {
        for (int j = 0; j < nq; j++) fprintf(fcost, "%d ", counts[j]);
        fflush(fcost);
    }
    time_update_s += (float)ts;
    time_update_u += (float)tu;
    count_update_s += nq;
    count_update_u += n - nq;
    if (n_final > 0) {
        if (data_info[2] == GTS_METRIC_EDIT) {
            char *ns = gts_ref::managed<char>((size_t)n_final * GTS_STR_STRIDE);
            int *nl = gts_ref::managed<int>((size_t)n_final);
            for (int i = 0; i < n_final; i++) {
                memcpy(ns + (size_t)i * GTS_STR_STRIDE, data_s + (size_t)final_rows[i] * GTS_STR_STRIDE,
                       GTS_STR_STRIDE);
                nl[i] = size_s[final_rows[i]];
            }
            cudaFree(data_s);
            cudaFree(size_s);
            data_s = ns;
            size_s = nl;
        } else {
            const size_t d = (size_t)data_info[0];
            float *nd = gts_ref::managed<float>((size_t)n_final * d);
            for (int i = 0; i < n_final; i++) memcpy(nd + i * d, data_d + (size_t)final_rows[i] * d, d * sizeof(float));
            cudaFree(data_d);
            data_d = nd;
        }
        data_info[1] = n_final;
        gts_ref::handles().erase(node_list);
        cudaFree(id_list);
        cudaFree(node_list);
        cudaFree(max_node_num);
        cudaFree(empty_list);
        gts_ref::export_tree(idx, id_list, node_list, max_node_num, tree_h, empty_list);
        gts_ref::handles()[node_list] = idx;
    }
}

#endif /* GTS_REF_COMPAT_H */
