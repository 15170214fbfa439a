/*
 * gts_b200.h -- C ABI of the B200-native GTS similarity-search path.
 *
 * Plain C types only (pointers, sizes, an opaque handle, a cudaStream_t
 * passed as void*).  Every function returns an int status (GTS_OK or a
 * negative GTS_ERR_*); gts_last_error() gives the message of the last
 * failure on the calling thread.  There is no global search state: all of it
 * lives in the gts_index handle, so independent handles may be used from
 * different threads.  One handle must not be used by two threads at once.
 *
 * Each entry point names the reference interface it replaces
 * (paths inside the reference checkout: Source Code/GTS/...).
 */
#ifndef GTS_B200_H
#define GTS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GTS_OK 0
#define GTS_ERR_INVALID -1   /* bad argument (null pointer, k < 1, bad metric, size) */
#define GTS_ERR_CUDA -2      /* CUDA runtime error or no usable device */
#define GTS_ERR_NOMEM -3     /* device or host allocation failed / over budget */
#define GTS_ERR_IO -4        /* file could not be opened or parsed */
#define GTS_ERR_KERNEL -5    /* a kernel reported a bounded failure (status word) */

#define GTS_STR_STRIDE 109   /* row stride of string objects (file.cuh:15) */

/* Metric codes (data_info[2]; tree.cuh:81-154). */
#define GTS_METRIC_LINF 0
#define GTS_METRIC_L1 1
#define GTS_METRIC_L2 2
#define GTS_METRIC_ANGLE 5
#define GTS_METRIC_EDIT 6

/* Search forms. */
#define GTS_FORM_PLAIN 0     /* traversal + FP32 filter + exact recheck */
#define GTS_FORM_FAST 1      /* learned radius + BF16 tensor-core filter + exact recheck (L2) */
#define GTS_FORM_PLAIN_LEARNED 2  /* plain traversal seeded by the learned radius (L2, after
                                     gts_learn_radius; otherwise the plain form) */

typedef struct gts_index gts_index;

/* Tunables.  The reference fixes these at compile time (tree.cuh:31-35,
 * update.cuh:16; the argv overrides in src/main.cu:54-76 are commented out);
 * here they are runtime values with the reference's defaults. */
typedef struct {
    int tree_order;      /* TREE_ORDER, default 10 */
    int max_size;        /* MAX_SIZE,   default 20 */
    int max_h;           /* MAX_H,      default 3 */
    int dis_code;        /* DIS_CODE,   default 100 */
    int infi_dis;        /* INFI_DIS,   default 10000 */
    int max_in_size;     /* MAX_IN_SIZE (cache list), default 10 */
    double mem_budget_gb;/* device scratch one search call may hold, in GiB (0 = 8): the fast
                            form runs its queries in runs whose scratch fits (at most 32,768
                            queries, halved in 128-query tiles), the seeded plain form in
                            chunks, the update path its queries in batches; a call that cannot
                            fit one tile / query returns GTS_ERR_NOMEM.  The plain traversal
                            itself holds no per-query device memory.  Negative: invalid. */
} gts_params;

typedef struct {
    int num, dim, metric;
    int tree_h, max_node_num;
    int tree_order, max_size;
    size_t device_bytes;  /* device memory held by the index */
} gts_index_info;

/* Fill *p with the reference defaults. */
void gts_params_default(gts_params *p);

const char *gts_last_error(void);

/* ---------------------------------------------------------------- I/O */

/* load (file.cuh:28-110): text data file, header "dim num metric".
 * Allocates *rows (num*dim floats) or *strs (num*GTS_STR_STRIDE bytes) and
 * *lens with malloc; free with gts_free_host. */
int gts_load(const char *path, int *dim, int *num, int *metric,
             float **rows, char **strs, int **lens);

/* loadQuery (file.cuh:112-152): count line, then one id per line. */
int gts_load_queries(const char *path, int **qids, int *qnum);

/* loadUpdate (update.cuh:43-95): count line, then "flag id" per line. */
int gts_load_updates(const char *path, int **flags, int **ids, int *nops);

void gts_free_host(void *p);

/* ---------------------------------------------------------------- index */

/* indexConstru (tree.cuh:332-393): build the pivot tree on the device.
 * Host inputs (copied to the device).  rows for metrics 0/1/2/5, strs+lens
 * (num*GTS_STR_STRIDE bytes, lengths <= 108) for metric 6. */
int gts_index_build(int dim, int num, int metric, const float *rows,
                    const char *strs, const int *lens, const gts_params *params,
                    gts_index **out);

/* Same, with inputs already in device memory (not retained; copied). */
int gts_index_build_device(int dim, int num, int metric, const float *d_rows,
                           const char *d_strs, const int *d_lens,
                           const gts_params *params, void *stream, gts_index **out);

int gts_index_info_get(const gts_index *idx, gts_index_info *info);

/* Copy the built tree to host buffers (each may be NULL): id_list[num];
 * per node (max_node_num): pid, min_dis, size, lid, is_leaf, exists
 * (exists = 1 where the reference's empty_list is 0). */
int gts_index_export(const gts_index *idx, int *id_list, int *pid, float *min_dis,
                     int *size, int *lid, int *is_leaf, int *exists);

void gts_index_free(gts_index *idx);

/* No counterpart in the reference (its only index is the tree).  Build
 * what a search form needs beyond the tree now, on `stream`, instead of in
 * the first search of that form: for GTS_FORM_FAST on an L2 index with
 * dim <= 128, the block order, filter records and slot-ordered rows (their
 * bytes join gts_index_info.device_bytes).  *prepared (nullable) = 1 when
 * the index holds them afterwards, 0 when the form needs nothing more on
 * this index.  A rebuild or update drops them again. */
int gts_index_prepare(gts_index *idx, int form, void *stream, int *prepared);

/* Set the stream used by the host-buffer entry points of this handle. */
int gts_index_set_stream(gts_index *idx, void *stream);

/* Work counters of the last search call on this handle (no reference
 * counterpart; the reference prints only wall-clock times, main.cu:106-109).
 * out8[0] plain form: leaf objects read; fast form: operand blocks streamed
 * out8[1] plain form: pivots evaluated;  fast form: bytes streamed
 * out8[2] exact (reference-order) recomputations
 * out8[3] queries finished by the plain traversal
 * out8[4] fast form: queries answered again on the plain path
 * out8[5] fast form: candidates appended
 * out8[6] fast form: filter passes over the blocks
 * out8[7] fast form: (query tile, block) pairs tested by the block bound */
int gts_search_stats(const gts_index *idx, unsigned long long *out8);

/* No counterpart in the reference.  Device time of the fast form's filter
 * kernel, from CUDA events around each launch on the index's stream.
 * reset != 0 zeroes the totals and turns timing on (creating the events);
 * *ms / *launches (nullable) receive the totals since the last reset. */
int gts_filter_timing(gts_index *idx, int reset, double *ms, long long *launches);

/* No counterpart in the reference.  Number of kernels this library has
 * launched for searches on this handle (a host-side count, cumulative). */
int gts_kernel_launches(const gts_index *idx, long long *count);

/* No counterpart in the reference (its launch shapes are compile-time
 * constants, search_v2.cuh: THREAD_NUM).  The GTS_FORM_FAST configuration
 * used for k on this index.  The first batch of at least 2048 queries with a
 * given k is run once per candidate -- learned-radius seed on or off (when a
 * model is trained), and the filter: the block-stationary one (each needed
 * block read once per run and multiplied with the queries that need it;
 * dim <= 128), or the tile one with 4 / 2 / 1 epilogue warps per query
 * lane, 8 / 16 / 32 blocks per work item, block records resident per stage
 * or streamed in 64-wide K chunks (always streamed above dim 128) -- and the
 * fastest that fits the shared memory is kept (every candidate returns the
 * same exact answers).  *variant: 0 tile filter, resident records; 1 tile
 * filter, streamed records; 2 block-stationary filter (*col_groups and
 * *item_blocks then unused).  *tuned = 0 reports the default that smaller
 * batches use.  Any output pointer may be NULL. */
int gts_fast_config(const gts_index *idx, int k, int *tuned, int *learned, int *col_groups, int *item_blocks,
                    int *variant);

/* No counterpart in the reference.  The fast form's starting bound for each
 * query object qids[q] at this k: a certified upper bound on the square of
 * its k-th distance, made with the filter records (the k-th smallest
 * squared distance over the object's own block and the 31 blocks with the
 * nearest centres, widened past FP32 rounding; for k not a power of two the
 * next power of two's; FLT_MAX where those blocks hold fewer objects).  Host
 * buffers; needs the records (gts_index_prepare with GTS_FORM_FAST). */
int gts_fast_seeds(gts_index *idx, const int *qids, int qnum, int k, float *seeds_out);

/* Pin the configuration for k (learned seed 0/1, 1/2/4 column groups with
 * groups * k <= 128, 8/16/32 blocks per item, filter variant 0/1/2 as
 * gts_fast_config reports it) instead of tuning it; GTS_ERR_INVALID when it
 * does not fit this index's shared memory plan. */
int gts_fast_config_set(gts_index *idx, int k, int learned, int col_groups, int item_blocks, int variant);

/* The filter of GTS_FORM_FAST range counts: variant 0 the block-stationary
 * filter where it fits (dim <= 128), 1 the tile filter (the default); -1
 * leaves it.  *current (nullable) receives the setting. */
int gts_fast_range_variant(gts_index *idx, int variant, int *current);

/* Forget the tuned configurations (the next large batch tunes again). */
int gts_fast_autotune_reset(gts_index *idx);

/* No counterpart in the reference (search_v2.cuh: THREAD_NUM per query
 * block).  Threads per query CTA of the plain traversal for one search mode
 * (0 kNN, 1 range count, 2 range ids).  The first batch of a mode with at
 * least twice the tuning sample (four times the most query CTAs resident at
 * once, about 1,800 on a B200) times 128 / 256 / 512 on its leading sample
 * and keeps the fastest (the answers do not depend on it); range ids take
 * the range-count choice.  *threads = 0 means not tuned yet (256 is used).
 * _set pins it (128, 256, 512; 0 = tune again). */
int gts_plain_threads(const gts_index *idx, int mode, int *threads);
int gts_plain_threads_set(gts_index *idx, int mode, int threads);

/* No counterpart in the reference (its list tables hold (query, node) pairs
 * level by level, search_v2.cuh:40-151).  Range counts of the plain
 * traversal run one query per CTA until a query has verified `objects`
 * objects in its CTA; then its older pending subtrees are handed over as
 * (query, node) work items, which the next launch spreads over every CTA
 * (their counts add up), so a few heavy queries do not leave the GPU idle
 * behind them.  objects = 0 turns this off, < 0 leaves it (default 32768).
 * *items_handed (nullable): items handed over since the index was built. */
int gts_plain_split(gts_index *idx, int objects, long long *items_handed);

/* No counterpart in the reference (it launches and synchronises every kernel
 * from the host, search_v2.cuh:868-871).  A GTS_FORM_FAST batch of at most
 * 32,768 queries runs its filter pass as a CUDA graph, captured once per
 * batch shape and argument buffers and replayed on the handle's own stream
 * (ordered after and before the caller's stream by events); a caller whose
 * buffers move from call to call gets direct launches instead.  on = 1 / 0 turns this on (the
 * default) / off, on < 0 leaves it; *replays (nullable) receives the number
 * of graph launches so far. */
int gts_fast_graphs(gts_index *idx, int on, long long *replays);

/* ---------------------------------------------------------------- search */

/* searchIndexKnnV2 (search_v2.cuh:975-1228) -> res_dis.
 * kth_out[q]: the k-th smallest distance of query object qids[q] (the query
 * itself counts, at distance 0), INFI_DIS when fewer than k objects exist.
 * ids_out / dists_out (qnum*k, nullable): the k nearest ids in ascending
 * (distance, id) order.  Host buffers. */
int gts_knn(gts_index *idx, const int *qids, int qnum, int k, int form,
            float *kth_out, int *ids_out, float *dists_out);

/* Same with device buffers, on `stream`. */
int gts_knn_device(gts_index *idx, const int *d_qids, int qnum, int k, int form,
                   float *d_kth, int *d_ids, float *d_dists, void *stream);

/* No counterpart in the reference.  gts_knn_device's GTS_FORM_FAST results
 * (the BF16 filter seeded from the index's seed table, without the learned
 * radius, + exact recheck) without any device allocation:
 * scratch is a fixed 12 MiB file-scope device array per device, so at most
 * 512 queries per call (more -> GTS_ERR_INVALID), L2 only, dim <= 128,
 * 1 <= k <= 64.  The index must already hold its filter records (made by
 * gts_index_prepare or one earlier GTS_FORM_FAST gts_knn / gts_knn_device
 * call); a rebuild or gts_update_run drops them, so one of those must follow
 * every update.  The array also holds the run's per-tile block lists, so
 * past about 35 million objects 512 queries no longer fit ("fixed scratch
 * ... too small"; fewer queries per call do).  Every call looks the array's
 * address up (cudaGetSymbolAddress); the first call on a device loads the
 * module and should come before any stream capture.  All calls on a device
 * share the array: calls that overlap on the GPU race. */
int gts_knn_device_noalloc(gts_index *idx, const int *d_qids, int qnum, int k,
                           float *d_kth, int *d_ids, float *d_dists, void *stream);

/* No counterpart in the reference (its queries are object ids,
 * search_v2.cuh:975 qid_list).  kNN of queries given as data: qrows
 * (qnum x dim floats) for metrics 0/1/2/5, or qstrs (qnum x GTS_STR_STRIDE
 * bytes) and qlens (lengths <= 108) for metric 6.  A query is not an object
 * of the index, so nothing matches it by id (an equal object is found at
 * its distance 0).  Outputs as gts_knn; the plain traversal.  This is what a
 * rank of an object-sharded index runs for queries it does not hold.  Host
 * buffers; _device takes device buffers on `stream`. */
int gts_knn_rows(gts_index *idx, const float *qrows, const char *qstrs, const int *qlens, int qnum, int k,
                 float *kth_out, int *ids_out, float *dists_out);
int gts_knn_rows_device(gts_index *idx, const float *d_qrows, const char *d_qstrs, const int *d_qlens, int qnum,
                        int k, float *d_kth, int *d_ids, float *d_dists, void *stream);

/* No counterpart in the reference.  Range counts of queries given as data
 * (as gts_knn_rows): the number of objects within r of each query row. */
int gts_range_rows(gts_index *idx, const float *qrows, const char *qstrs, const int *qlens, int qnum, float r,
                   int *counts_out);

/* searchIndexRnnV2 (search_v2.cuh:780-972) -> res.
 * counts_out[q]: number of objects within r of qids[q] (itself included). */
int gts_range(gts_index *idx, const int *qids, int qnum, float r, int *counts_out);

int gts_range_device(gts_index *idx, const int *d_qids, int qnum, float r,
                     int *d_counts, void *stream);

/* searchIndexRnnV2 (search_v2.cuh:780-972) -> res, as gts_range, in a
 * chosen form.  GTS_FORM_FAST (L2, dim <= 128; other indexes take the plain
 * form): the tensor-core filter with the bound fixed at r^2; objects whose
 * certified upper bound lies below r^2 (1 - 3e-5) count without a recheck
 * (the reference's FP32-accumulated value is within 8e-6 of the square),
 * those whose lower bound lies above r^2 (1 + 3e-5) do not, and the rest get
 * the reference's value.  The counts equal gts_range's. */
int gts_range_form(gts_index *idx, const int *qids, int qnum, float r, int form, int *counts_out);

int gts_range_form_device(gts_index *idx, const int *d_qids, int qnum, float r, int form,
                          int *d_counts, void *stream);

/* saveR layout (file.cuh:178-199): ids of every object within r.
 * counts_out[q] as above, offsets_out[q] = exclusive prefix of counts,
 * ids_out/dists_out hold up to `capacity` entries grouped by query in
 * ascending (distance, id) order.  Returns GTS_ERR_NOMEM (with counts and
 * offsets filled) if the total exceeds capacity. */
int gts_range_ids(gts_index *idx, const int *qids, int qnum, float r, int *counts_out,
                  int *offsets_out, int *ids_out, float *dists_out, size_t capacity);

/* ---------------------------------------------------------------- learned radius */

/* No reference counterpart (the reference has no learned component).
 * Train the kNN radius predictor of an L2 index: a 33-128-128-1 MLP whose
 * inputs are a query's distances to the first 32 pivots of the tree plus
 * log(k), and whose output is log of the k-th neighbour distance.  Labels are
 * exact radii of n_train random objects (k drawn uniformly from
 * {2, 4, 8, 16, 32, 64} up to k_max, plus k_max itself; k = 1 is not learned:
 * its radius is 0, the query itself) computed by this index's own exact
 * search; training runs on the device (forward, backward and Adam kernels).
 * Afterwards GTS_FORM_FAST searches may start from the predicted radius
 * (the autotuner decides per k; gts_fast_config), widened by the 99.5th
 * percentile of the held-out under-predictions of that k (of all k where a
 * k has fewer than 400 held-out samples; *widen reports the all-k factor),
 * and re-answer any query
 * whose radius held fewer than k objects -- results stay exact.
 * val_rmse_log: RMS error of log(radius) on the held-out 10%; widen: factor
 * applied to predictions (both nullable).  A rebuild discards the model. */
int gts_learn_radius(gts_index *idx, int n_train, int k_max, int epochs, unsigned seed,
                     float *val_rmse_log, float *widen);

/* The trained model: params[20993] (W1[128][33] b1[128] W2[128][128] b2[128]
 * W3[128] b3), norm[66] (input means, input deviations), ymu_ysig_widen[3].
 * Each pointer may be NULL. */
int gts_radius_model_params(const gts_index *idx, float *params, float *norm, float *ymu_ysig_widen);

/* Loss and parameter gradient of the model's mean squared error on a host
 * batch (X[batch][33] raw features, target[batch] standardised log radii),
 * evaluated by the device training kernels. */
int gts_radius_model_grad(const float *X, const float *target, int batch, const float *params,
                          const float *norm, float *grad, float *loss);

/* ---------------------------------------------------------------- update */

/* updateIndexRnn (update.cuh:449-638): replay a stream of operations
 * (flag 0 insert, 1 delete, 2 range query of radius r) through the lazy
 * cache list of params->max_in_size entries with the reference's id rules
 * and answers.  counts_out receives one entry per query op (*nq_out of
 * them; size it to the number of flag-2 ops).  Every query of the stream
 * runs in one batched launch over the index as it was built (an insert
 * copies an existing row, so no compaction needs a rebuild); afterwards the
 * handle holds the data of the last compaction and its rebuilt tree, as the
 * reference's does.  *search_s: the batched search (copies included);
 * *update_s: the host pass and the final rebuild. */
int gts_update_run(gts_index *idx, const int *flags, const int *ids, int nops, float r,
                   int *counts_out, int *nq_out, double *search_s, double *update_s);

/* updateIndexRnn's bookkeeping (update.cuh:473-623) without the device:
 * the host pass of gts_update_run (n_new = 0) and gts_update_run_rows
 * (n_new > 0: a flag-0 op with id j brings new row j, object num + j).
 * Every object the stream ever holds is an entry: the num rows of the data
 * (entries 0..num-1) and one per insert, in insertion order.  ent_src[e] is
 * the object entry e copies (a data row, or num + j for new row j);
 * ent_life[4e..4e+3] = (tree_from, tree_to, cache_from, cache_to): entry e
 * is in the tree at operation t when tree_from < t < tree_to and in the
 * cache list when cache_from < t < cache_to (INT_MAX = never).  Query op j
 * (in stream order) asks about data row q_obj[j] at operation q_time[j];
 * q_cache[j] = 1 when the cache list was not empty then (otherwise the
 * reference reuses the previous query's cache count).  final_rows: the data
 * rows of the array after the last compaction (*n_final = 0: no
 * compaction).  Size q_* to the number of flag-2 ops and ent_* / final_rows
 * to num + the number of flag-0 ops; every output array may be NULL. */
int gts_update_plan(int num, const int *flags, const int *ids, int nops, int max_in_size, int n_new,
                    int *q_obj, int *q_time, int *q_cache, int *n_q,
                    int *ent_src, int *ent_life, int *n_ent, int *final_rows, int *n_final);

/* updateIndexRnn's operations (update.cuh:449-638) with inserts that bring
 * new rows instead of copying a physical row (the reference's insert can
 * only copy, update.cuh:481, 186): a flag-0 op with id j inserts
 * new_rows[j] (n_new rows of dim floats, host memory).  Deletes and queries
 * keep the reference's id rules; the data after a compaction holds the live
 * rows, then the cached new rows.  The handle is rebuilt on the data rows
 * plus the new rows first, searched once for every query op, and ends on
 * the data of the last compaction.  Row metrics only. */
int gts_update_run_rows(gts_index *idx, const int *flags, const int *ids, int nops, const float *new_rows,
                        int n_new, float r, int *counts_out, int *nq_out, double *search_s, double *update_s);

#ifdef __cplusplus
}
#endif

#endif /* GTS_B200_H */
