/*
 * gts_oracle.h -- CPU oracle for the GTS similarity-search path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * implementation in gts_b200/.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline / reference legs may load it.  The product path
 * never calls into it.
 *
 * It has two halves:
 *   1. A restatement of the reference algorithm in plain C, following the
 *      reference's own operation order (file:line cited per function):
 *        - index construction   Source Code/GTS/include/tree.cuh:53-393
 *        - kNN search (v2)      Source Code/GTS/include/search_v2.cuh:975-1228
 *        - range search (v2)    Source Code/GTS/include/search_v2.cuh:780-972
 *        - stream update        Source Code/GTS/include/update.cuh:449-638,
 *                               search.cuh:38-194, search_naive.cuh:24-251
 *   2. Exact brute force (kNN k-th distance, ID lists with ties broken by
 *      ID, range counts) in the reference's per-site arithmetic.  This is
 *      the truth the GPU path is held to.
 *
 * Parity is pinned by fixtures produced by the reference's own CUDA build
 * (see oracle/Makefile target `ref` and tests/golden/).
 */
#ifndef GTS_ORACLE_H
#define GTS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Row stride of string objects in the reference's layout (file.cuh:15). */
#define ORC_STR_STRIDE 109

typedef struct {
    int dim;            /* data_info[0] */
    int num;            /* data_info[1] */
    int metric;         /* data_info[2]: 0 Linf, 1 L1, 2 L2, 5 angle, 6 edit */
    const float *rows;  /* num*dim row-major, metric != 6 */
    const char *strs;   /* num*ORC_STR_STRIDE, metric == 6 */
    const int *lens;    /* num, metric == 6 */
} orc_data;

typedef struct {
    int order;          /* TREE_ORDER (tree.cuh:31) */
    int max_size;       /* MAX_SIZE   (tree.cuh:32) */
    int max_h;          /* MAX_H      (tree.cuh:33) */
    int dis_code;       /* DIS_CODE   (tree.cuh:34) */
    int infi_dis;       /* INFI_DIS   (tree.cuh:35) */
} orc_params;

typedef struct {
    int max_node_num;
    int tree_h;
    int start_idx;      /* value of the build loop's start_idx global after the build */
    int *id_list;       /* num */
    int *pid;           /* max_node_num, TN.pid */
    float *min_dis;     /* TN.min_dis */
    int *size;          /* TN.size */
    int *lid;           /* TN.lid */
    int *is_leaf;       /* TN.is_leaf */
    int *exists;        /* 1 where empty_list == 0 */
} orc_tree;

/* Distance call-site families (reference arithmetic differs per site):
 *   ORC_ACC_F64: double accumulator (tree.cuh:80-155 build key,
 *                search_v2.cuh:664-745 kNN pivot, search_v2.cuh:447-535 kNN leaf)
 *   ORC_ACC_F32: float accumulator  (tree.cuh:205-280 min_dis,
 *                search_v2.cuh:63-129 range node, search_v2.cuh:337-408 range leaf,
 *                update.cuh:246-323 update leaf, search_naive.cuh:31-68 cache scan) */
enum { ORC_ACC_F32 = 0, ORC_ACC_F64 = 1 };

double orc_dist(const orc_data *d, int a, int b, int acc);

int orc_build(const orc_data *d, const orc_params *p, orc_tree *out);
void orc_tree_free(orc_tree *t);

/* Restated reference searches (single list-table batch per level). */
int orc_knn_v2(const orc_data *d, const orc_params *p, const orc_tree *t,
               const int *qids, int qnum, int k, float *kth_out);
int orc_range_v2(const orc_data *d, const orc_params *p, const orc_tree *t,
                 const int *qids, int qnum, float r, int *count_out);

/* Exact brute force.  ids_out / dists_out (qnum*k) may be NULL.  Ties are
 * broken by ascending object id.  Positions beyond the number of objects
 * get id -1 and distance infi_dis. */
int orc_knn_brute(const orc_data *d, const int *qids, int qnum, int k, int infi_dis,
                  float *kth_out, int *ids_out, float *dists_out, int nthreads);
int orc_range_brute(const orc_data *d, const int *qids, int qnum, float r,
                    int *count_out, int nthreads);

/* Stream update (update.cuh:449-638).  flags/ids: the update file's ops.
 * counts_out receives one entry per query op (flag 2); *nq_out their number.
 * The data set is copied internally; `d` is not modified.
 * exact == 0: the reference's v1 tree search restated (it skips last-level
 *             nodes above MAX_SIZE, so it undercounts on non-perfect trees);
 * exact != 0: the tree part of each count is a brute-force scan of the live
 *             rows (the exact answer), everything else unchanged. */
int orc_update_run(const orc_data *d, const orc_params *p, int max_in_size,
                   const int *flags, const int *ids, int nops, float r,
                   int exact, int *counts_out, int *nq_out);

/* Stream update whose flag-0 ops insert new_rows[ids[i]] (n_new rows of
 * dim floats) instead of a copy of a physical row: an extension, not a
 * reference behaviour.  Exact counts; row metrics only (not 6). */
int orc_update_run_rows(const orc_data *d, int max_in_size, const int *flags, const int *ids, int nops,
                        const float *new_rows, int n_new, float r, int *counts_out, int *nq_out);

#ifdef __cplusplus
}
#endif
#endif
