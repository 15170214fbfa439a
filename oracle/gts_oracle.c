/*
 * gts_oracle.c -- CPU oracle for the GTS similarity-search path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA implementation.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU legs may load it; the
 * product path (gts_b200/) never does.
 *
 * Arithmetic notes (device semantics of the reference expressions, checked
 * with decltype against the reference headers and measured on the device):
 *   - `pow(float_diff, 2)` resolves to a double-returning overload;
 *     `float acc += pow(..)` therefore adds in double and rounds to float.
 *     This oracle uses the exact square and `sqrt` for `pow(x, 0.5)`.  The
 *     device functions differ from those in the last bit of a double for a
 *     few percent of inputs, which reaches a reported float value only when
 *     a sum lies within that bit of a float rounding boundary; tests that
 *     compare with the device allow for that and nothing else.
 *   - `abs(float)` and `acos(float)` are the float overloads; the host
 *     `acosf` / `acos` may differ from the device's in the last bit.
 *   - `s += a * b` on floats is contracted to a fused multiply-add.
 */
#include "gts_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

/* ------------------------------------------------------------------ */
/* Minimal dynamic parallel-for over [0, n) on pthreads                */
/* ------------------------------------------------------------------ */

typedef void (*orc_body)(void *ctx, int i, void *scratch);

typedef struct {
    orc_body body;
    void *ctx;
    int n;
    size_t scratch_bytes;
    int next;
    pthread_mutex_t mu;
} par_job;

static void *par_worker(void *arg)
{
    par_job *j = (par_job *)arg;
    void *scratch = j->scratch_bytes ? malloc(j->scratch_bytes) : NULL;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        int i = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (i >= j->n) break;
        j->body(j->ctx, i, scratch);
    }
    free(scratch);
    return NULL;
}

static int default_threads(void)
{
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

static void par_for(int n, int nthreads, size_t scratch_bytes, orc_body body, void *ctx)
{
    if (nthreads <= 0) nthreads = default_threads();
    if (nthreads > n) nthreads = n > 0 ? n : 1;
    par_job j;
    j.body = body; j.ctx = ctx; j.n = n; j.scratch_bytes = scratch_bytes; j.next = 0;
    pthread_mutex_init(&j.mu, NULL);
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    for (int t = 0; t < nthreads; t++) pthread_create(&th[t], NULL, par_worker, &j);
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    free(th);
    pthread_mutex_destroy(&j.mu);
}

/* ------------------------------------------------------------------ */
/* Distance functions                                                  */
/* ------------------------------------------------------------------ */

static inline double sq_dev(float x) { return (double)x * (double)x; }

/* Levenshtein distance with the reference's DP recurrence
 * (tree.cuh:128-153; identical at every call site). */
static int edit_distance(const char *a, int n, const char *b, int m)
{
    if (n == 0) return m;
    if (m == 0) return n;
    int prev[ORC_STR_STRIDE + 1], cur[ORC_STR_STRIDE + 1];
    for (int k = 0; k <= m; k++) prev[k] = k;
    for (int j = 1; j <= n; j++) {
        cur[0] = j;
        for (int k = 1; k <= m; k++) {
            int cost = (a[j - 1] == b[k - 1]) ? 0 : 1;
            int v = 1 + (prev[k] < cur[k - 1] ? prev[k] : cur[k - 1]);
            int diag = prev[k - 1] + cost;
            cur[k] = diag < v ? diag : v;
        }
        memcpy(prev, cur, sizeof(int) * (size_t)(m + 1));
    }
    return prev[m];
}

/* Angle in degrees, float partial sums (tree.cuh:106-127 and siblings). */
static void angle_sums(const float *a, const float *b, int dim, float *s1, float *s2, float *s3)
{
    float sa1 = 0.f, sa2 = 0.f, sa3 = 0.f;
    for (int j = 0; j < dim; j++) {
        sa1 = fmaf(a[j], a[j], sa1);
        sa2 = fmaf(b[j], b[j], sa2);
        sa3 = fmaf(a[j], b[j], sa3);
    }
    *s1 = (float)sqrt((double)sa1);
    *s2 = (float)sqrt((double)sa2);
    *s3 = sa3;
}

double orc_dist(const orc_data *d, int a, int b, int acc)
{
    const int dim = d->dim;
    if (d->metric == 6) {
        return (double)edit_distance(d->strs + (size_t)a * ORC_STR_STRIDE, d->lens[a],
                                     d->strs + (size_t)b * ORC_STR_STRIDE, d->lens[b]);
    }
    const float *x = d->rows + (size_t)a * dim;
    const float *y = d->rows + (size_t)b * dim;
    if (acc == ORC_ACC_F64) {
        double r = 0.0;
        switch (d->metric) {
        case 2:
            for (int j = 0; j < dim; j++) r = r + sq_dev(x[j] - y[j]);
            return sqrt(r);
        case 1:
            for (int j = 0; j < dim; j++) r = r + (double)fabsf(x[j] - y[j]);
            return r;
        case 0:
            for (int j = 0; j < dim; j++) {
                float t = fabsf(x[j] - y[j]);
                if ((double)t > r) r = t;
            }
            return r;
        case 5: {
            float s1, s2, s3;
            angle_sums(x, y, dim, &s1, &s2, &s3);
            r = (double)(s3 / (s1 * s2));
            if (r > 1) r = 1.0;
            return fabs(acos(r) * 180 / 3.1415926);
        }
        default:
            return NAN;
        }
    } else {
        float r = 0.f;
        switch (d->metric) {
        case 2:
            for (int j = 0; j < dim; j++) r = (float)((double)r + sq_dev(x[j] - y[j]));
            return (double)(float)sqrt((double)r);
        case 1:
            for (int j = 0; j < dim; j++) r = r + fabsf(x[j] - y[j]);
            return r;
        case 0:
            for (int j = 0; j < dim; j++) {
                float t = fabsf(x[j] - y[j]);
                if (t > r) r = t;
            }
            return r;
        case 5: {
            float s1, s2, s3;
            angle_sums(x, y, dim, &s1, &s2, &s3);
            r = s3 / (s1 * s2);
            if (r > 1) r = 1.0f;
            float t = acosf(r) * 180.0f;
            return (double)(float)fabs((double)t / 3.1415926);
        }
        default:
            return NAN;
        }
    }
}

/* ------------------------------------------------------------------ */
/* Index construction: tree.cuh:332-393                                */
/* ------------------------------------------------------------------ */

static long ipow(int b, int e)
{
    long r = 1;
    for (int i = 0; i < e; i++) r *= b;
    return r;
}

/* Stable merge sort of (key, val) pairs by key: thrust::sort_by_key on
 * double keys is a stable radix sort, and every key here is >= +0.0. */
static void stable_sort_kv(double *key, int *val, long n)
{
    double *k2 = (double *)malloc(sizeof(double) * (size_t)n);
    int *v2 = (int *)malloc(sizeof(int) * (size_t)n);
    for (long w = 1; w < n; w *= 2) {
        for (long lo = 0; lo < n; lo += 2 * w) {
            long mid = lo + w < n ? lo + w : n;
            long hi = lo + 2 * w < n ? lo + 2 * w : n;
            long i = lo, j = mid, o = lo;
            while (i < mid && j < hi) {
                if (key[j] < key[i]) { k2[o] = key[j]; v2[o++] = val[j++]; }
                else { k2[o] = key[i]; v2[o++] = val[i++]; }
            }
            while (i < mid) { k2[o] = key[i]; v2[o++] = val[i++]; }
            while (j < hi) { k2[o] = key[j]; v2[o++] = val[j++]; }
        }
        memcpy(key, k2, sizeof(double) * (size_t)n);
        memcpy(val, v2, sizeof(int) * (size_t)n);
    }
    free(k2);
    free(v2);
}

int orc_build(const orc_data *d, const orc_params *p, orc_tree *t)
{
    const int O = p->order, H = p->max_h, N = d->num;
    memset(t, 0, sizeof(*t));
    if (O < 2 || H < 1 || N < 1) return -1;
    /* max_node_num[0] = (pow(TREE_ORDER, MAX_H) - 1) / (TREE_ORDER - 1)  (tree.cuh:339) */
    long mnn = (long)((pow((double)O, (double)H) - 1) / (O - 1));
    if (mnn > 0x7fffffffL) return -2;
    t->max_node_num = (int)mnn;
    t->id_list = (int *)malloc(sizeof(int) * (size_t)N);
    t->pid = (int *)malloc(sizeof(int) * (size_t)mnn);
    t->min_dis = (float *)calloc((size_t)mnn, sizeof(float));
    t->size = (int *)calloc((size_t)mnn, sizeof(int));
    t->lid = (int *)calloc((size_t)mnn, sizeof(int));
    t->is_leaf = (int *)calloc((size_t)mnn, sizeof(int));
    t->exists = (int *)calloc((size_t)mnn, sizeof(int));
    int *split = (int *)calloc((size_t)mnn, sizeof(int));
    int *pid_list = (int *)malloc(sizeof(int) * (size_t)mnn);
    double *key = (double *)calloc((size_t)N, sizeof(double));
    for (long i = 0; i < mnn; i++) { t->pid[i] = -1; pid_list[i] = -1; }

    /* initIndexData (tree.cuh:299-318) */
    for (int i = 0; i < N; i++) t->id_list[i] = i;
    t->size[0] = N; t->lid[0] = 0; t->pid[0] = -1; t->min_dis[0] = 0.f; t->is_leaf[0] = 0;
    split[0] = 1; t->exists[0] = 1;

    int cur_level = 0, start_idx = 0;
    long split_num = 1;
    while (cur_level < H - 1 && split_num > 0) {
        long nb = ipow(O, cur_level);
        /* getPivotDis (tree.cuh:53-171) */
        for (long b = 0; b < nb; b++) {
            long nid = start_idx + b;
            if (!t->exists[nid]) continue;
            int lid = t->lid[nid], size = t->size[nid], rid = lid + size - 1;
            if (split[nid] == 1) {
                int piv = t->id_list[(lid + rid) / 2];
                pid_list[nid] = piv;
                for (int i = lid; i <= rid; i++) {
                    double res = orc_dist(d, t->id_list[i], piv, ORC_ACC_F64);
                    key[i] = (double)(res / p->infi_dis + (double)(int)(b * p->dis_code));
                }
            } else {
                for (int i = lid; i <= rid; i++) key[i] = (double)(int)(b * p->dis_code);
            }
        }
        stable_sort_kv(key, t->id_list, N);
        /* nodeSplit (tree.cuh:173-297) */
        for (long b = 0; b < nb; b++) {
            long nid = start_idx + b;
            if (split[nid] != 1) continue;
            int lid = t->lid[nid], size = t->size[nid];
            split[nid] = 0;
            int avg = size / O;
            for (int i = 0; i < O; i++) {
                long c = nid * O + i + 1;
                int clid = lid + avg * i;
                int csize = (i < O - 1) ? avg : size - (O - 1) * avg;
                t->lid[c] = clid;
                t->pid[c] = pid_list[nid];
                t->size[c] = csize;
                t->min_dis[c] = (float)orc_dist(d, t->id_list[clid], pid_list[nid], ORC_ACC_F32);
                if (csize > p->max_size) { split[c] = 1; t->is_leaf[c] = 0; }
                else { split[c] = 0; t->is_leaf[c] = 1; }
                t->exists[c] = 1;
            }
        }
        start_idx += (int)nb;
        cur_level++;
        split_num = 0;
        for (long i = 0; i < mnn; i++) split_num += split[i];
    }
    t->tree_h = cur_level + 1;
    t->start_idx = start_idx;
    free(split);
    free(pid_list);
    free(key);
    return 0;
}

void orc_tree_free(orc_tree *t)
{
    free(t->id_list); free(t->pid); free(t->min_dis); free(t->size);
    free(t->lid); free(t->is_leaf); free(t->exists);
    memset(t, 0, sizeof(*t));
}

/* ------------------------------------------------------------------ */
/* Restated v2 searches                                                */
/* ------------------------------------------------------------------ */

static long level_offset(int O, int l) { return (ipow(O, l) - 1) / (O - 1); }

/* Ring lower bound of nodeProcessRnn / nodeProcessKnn (search_v2.cuh:131-141,
 * 181-190): float arithmetic, `max(float, 0.0)` is exact. */
static inline float ring_lb(const orc_tree *t, long nid, int O, float dq)
{
    float lb = t->min_dis[nid] - dq;
    if (lb < 0.f) lb = 0.f;
    if (nid % O != 0) {
        float lb2 = dq - t->min_dis[nid + 1];
        if (lb2 > lb) lb = lb2;
    }
    return lb;
}

typedef struct {
    const orc_data *d;
    const orc_params *p;
    const orc_tree *t;
    const int *qids;
    float r;
    int k;
    int update_level;
    int *count_out;
    float *kth_out;
    int *ids_out;
    float *dists_out;
} search_ctx;

/* One range query, v2 semantics (search_v2.cuh:40-151 node level,
 * 319-430 + 547-569 leaf level). */
static void range_v2_body(void *vc, int q, void *scratch)
{
    const search_ctx *c = (const search_ctx *)vc;
    const orc_data *d = c->d;
    const orc_tree *t = c->t;
    const int O = c->p->order, H = t->tree_h;
    unsigned char *flag = (unsigned char *)scratch;
    int qid = c->qids[q];
    memset(flag, 0, (size_t)t->max_node_num);
    flag[0] = 1;
    for (int l = 1; l < H; l++) {
        long off = level_offset(O, l), nn = ipow(O, l), offu = level_offset(O, l - 1);
        for (long j = 0; j < nn; j++) {
            long nid = off + j;
            if (!flag[offu + j / O] || !t->exists[nid]) continue;
            float dq = (float)orc_dist(d, t->pid[nid], qid, ORC_ACC_F32);
            if (ring_lb(t, nid, O, dq) <= c->r) flag[nid] = 1;
        }
    }
    /* leaf stage: only level tree_h-1 (search_v2.cuh:873-919) */
    int cnt = 0;
    long off = level_offset(O, H - 1), nn = ipow(O, H - 1);
    for (long j = 0; j < nn; j++) {
        long nid = off + j;
        if (!flag[nid] || !t->is_leaf[nid]) continue;
        for (int s = 0; s < t->size[nid]; s++) {
            int id = t->id_list[t->lid[nid] + s];
            double res = (id == qid) ? 0.0 : orc_dist(d, id, qid, ORC_ACC_F32);
            if ((float)res <= c->r) cnt++;
        }
    }
    c->count_out[q] = cnt;
}

int orc_range_v2(const orc_data *d, const orc_params *p, const orc_tree *t,
                 const int *qids, int qnum, float r, int *count_out)
{
    search_ctx c;
    memset(&c, 0, sizeof(c));
    c.d = d; c.p = p; c.t = t; c.qids = qids; c.r = r; c.count_out = count_out;
    par_for(qnum, 0, (size_t)t->max_node_num, range_v2_body, &c);
    return 0;
}

typedef struct { double code; int idx; } code_idx;

static int cmp_code_idx(const void *a, const void *b)
{
    const code_idx *x = (const code_idx *)a, *y = (const code_idx *)b;
    if (x->code < y->code) return -1;
    if (x->code > y->code) return 1;
    return (x->idx > y->idx) - (x->idx < y->idx);   /* stability */
}

/* One kNN query, v2 semantics with one list-table batch per level
 * (search_v2.cuh:1039-1222). */
static void knn_v2_body(void *vc, int q, void *scratch)
{
    const search_ctx *c = (const search_ctx *)vc;
    const orc_data *d = c->d;
    const orc_params *p = c->p;
    const orc_tree *t = c->t;
    const int O = p->order, H = t->tree_h, S = p->max_size, k = c->k;
    const double INF = (double)p->infi_dis;
    long npmax = ipow(O, H > 1 ? H - 2 : 0);
    unsigned char *flag = (unsigned char *)scratch;
    code_idx *piv = (code_idx *)malloc(sizeof(code_idx) * (size_t)npmax);
    double *pdis = (double *)malloc(sizeof(double) * (size_t)npmax);
    int qid = c->qids[q];
    float disk = (float)INF;
    memset(flag, 0, (size_t)t->max_node_num);
    flag[0] = 1;
    for (int l = 1; l < H; l++) {
        long off = level_offset(O, l), nn = ipow(O, l), offu = level_offset(O, l - 1);
        if (l < c->update_level) {
            /* labelCNode (search_v2.cuh:612-642) */
            for (long j = 0; j < nn; j++)
                if (flag[offu + j / O] && t->exists[off + j]) flag[off + j] = 1;
            continue;
        }
        /* getDisPQ + sort + updateDisK (search_v2.cuh:645-777, 1084-1107) */
        long np = nn / O;
        for (long j = 0; j < np; j++) {
            long first = off + j * O;
            double dq = INF;
            if (flag[offu + j] && t->exists[first])
                dq = orc_dist(d, t->pid[first], qid, ORC_ACC_F64);
            pdis[j] = dq;
            piv[j].code = (double)(dq / p->infi_dis + (double)(q * p->dis_code));
            piv[j].idx = (int)j;
        }
        if (np >= k) {
            qsort(piv, (size_t)np, sizeof(code_idx), cmp_code_idx);
            double kd = pdis[piv[k - 1].idx];
            if ((double)disk > kd) disk = (float)kd;
        }
        /* nodeProcessKnn (search_v2.cuh:155-196) */
        for (long j = 0; j < nn; j++) {
            long nid = off + j;
            if (!flag[offu + j / O] || !t->exists[nid]) continue;
            float dq = (float)pdis[j / O];
            if (ring_lb(t, nid, O, dq) <= disk) flag[nid] = 1;
        }
    }
    free(piv);
    free(pdis);
    /* dataProcessKnn + sort + mergeResKnn (search_v2.cuh:433-585, 1150-1173) */
    long nleaf = ipow(O, H - 1), npair = 0;
    long off = level_offset(O, H - 1);
    for (long j = 0; j < nleaf; j++) if (flag[off + j]) npair++;
    if (npair * S < k) { c->kth_out[q] = NAN; return; }
    code_idx *slots = (code_idx *)malloc(sizeof(code_idx) * (size_t)(npair * S));
    double *vals = (double *)malloc(sizeof(double) * (size_t)(npair * S));
    long pi = 0;
    for (long j = 0; j < nleaf; j++) {
        long nid = off + j;
        if (!flag[nid]) continue;
        for (int s = 0; s < S; s++) {
            double res = INF;
            if (s < t->size[nid] && t->is_leaf[nid]) {
                int id = t->id_list[t->lid[nid] + s];
                res = (id == qid) ? 0.0 : orc_dist(d, id, qid, ORC_ACC_F64);
                if (res > (double)disk) res = INF;
            }
            long slot = pi * S + s;
            vals[slot] = res;
            slots[slot].code = (double)(res / p->infi_dis + (double)(q * p->dis_code));
            slots[slot].idx = (int)slot;
        }
        pi++;
    }
    qsort(slots, (size_t)(npair * S), sizeof(code_idx), cmp_code_idx);
    c->kth_out[q] = (float)vals[slots[k - 1].idx];
    free(slots);
    free(vals);
}

int orc_knn_v2(const orc_data *d, const orc_params *p, const orc_tree *t,
               const int *qids, int qnum, int k, float *kth_out)
{
    const int O = p->order, H = t->tree_h;
    const long mnn = t->max_node_num;
    /* update_disk is a global that persists across the levels of one call
     * (search_v2.cuh:35, 1071-1078).  With one batch per level it flips at
     * the same level for every query, so that level is found once here.
     * pnum_level reads empty_list from the stale build start_idx
     * (search_v2.cuh:1065, tree.cuh:381); absent nodes hold 0x01010101. */
    int update_level = H;
    for (int l = 1; l < H; l++) {
        long nn = ipow(O, l);
        long long s = 0;
        for (long i = t->start_idx; i < t->start_idx + nn; i++) {
            if (i >= mnn) return -3;
            s += t->exists[i] ? 0 : 0x01010101;
        }
        int pnum = (int)((int32_t)(nn - s)) / O;
        if (!(pnum < k || l <= 2)) { update_level = l; break; }
    }
    search_ctx c;
    memset(&c, 0, sizeof(c));
    c.d = d; c.p = p; c.t = t; c.qids = qids; c.k = k; c.kth_out = kth_out;
    c.update_level = update_level;
    par_for(qnum, 0, (size_t)mnn, knn_v2_body, &c);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Brute force                                                         */
/* ------------------------------------------------------------------ */

typedef struct { double d; int id; } dist_id;

static inline int di_less(dist_id a, dist_id b) { return a.d < b.d || (a.d == b.d && a.id < b.id); }

/* max-heap of the k best (smallest) entries */
static void heap_push(dist_id *h, int *n, int k, dist_id e)
{
    if (*n < k) {
        int i = (*n)++;
        h[i] = e;
        while (i > 0) {
            int pa = (i - 1) / 2;
            if (di_less(h[pa], h[i])) { dist_id tmp = h[pa]; h[pa] = h[i]; h[i] = tmp; i = pa; }
            else break;
        }
    } else if (di_less(e, h[0])) {
        h[0] = e;
        int i = 0;
        for (;;) {
            int l = 2 * i + 1, r = l + 1, m = i;
            if (l < *n && di_less(h[m], h[l])) m = l;
            if (r < *n && di_less(h[m], h[r])) m = r;
            if (m == i) break;
            dist_id tmp = h[m]; h[m] = h[i]; h[i] = tmp; i = m;
        }
    }
}

static int cmp_di(const void *a, const void *b)
{
    dist_id x = *(const dist_id *)a, y = *(const dist_id *)b;
    return di_less(x, y) ? -1 : (di_less(y, x) ? 1 : 0);
}

static void knn_brute_body(void *vc, int q, void *scratch)
{
    const search_ctx *c = (const search_ctx *)vc;
    const orc_data *d = c->d;
    const int k = c->k;
    dist_id *h = (dist_id *)scratch;
    int qid = c->qids[q], n = 0;
    for (int o = 0; o < d->num; o++) {
        dist_id e;
        e.d = (o == qid) ? 0.0 : orc_dist(d, o, qid, ORC_ACC_F64);
        e.id = o;
        heap_push(h, &n, k, e);
    }
    qsort(h, (size_t)n, sizeof(dist_id), cmp_di);
    float inf = (float)c->update_level;   /* carries infi_dis */
    c->kth_out[q] = (n >= k) ? (float)h[k - 1].d : inf;
    for (int j = 0; j < k; j++) {
        if (c->ids_out) c->ids_out[(size_t)q * k + j] = j < n ? h[j].id : -1;
        if (c->dists_out) c->dists_out[(size_t)q * k + j] = j < n ? (float)h[j].d : inf;
    }
}

int orc_knn_brute(const orc_data *d, const int *qids, int qnum, int k, int infi_dis,
                  float *kth_out, int *ids_out, float *dists_out, int nthreads)
{
    if (k < 1) return -1;
    search_ctx c;
    memset(&c, 0, sizeof(c));
    c.d = d; c.qids = qids; c.k = k; c.kth_out = kth_out; c.ids_out = ids_out;
    c.dists_out = dists_out; c.update_level = infi_dis;
    par_for(qnum, nthreads, sizeof(dist_id) * (size_t)k, knn_brute_body, &c);
    return 0;
}

static void range_brute_body(void *vc, int q, void *scratch)
{
    (void)scratch;
    const search_ctx *c = (const search_ctx *)vc;
    const orc_data *d = c->d;
    int qid = c->qids[q], cnt = 0;
    for (int o = 0; o < d->num; o++) {
        double res = (o == qid) ? 0.0 : orc_dist(d, o, qid, ORC_ACC_F32);
        if ((float)res <= c->r) cnt++;
    }
    c->count_out[q] = cnt;
}

int orc_range_brute(const orc_data *d, const int *qids, int qnum, float r,
                    int *count_out, int nthreads)
{
    search_ctx c;
    memset(&c, 0, sizeof(c));
    c.d = d; c.qids = qids; c.r = r; c.count_out = count_out;
    par_for(qnum, nthreads, 0, range_brute_body, &c);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Stream update: update.cuh:449-638                                   */
/* ------------------------------------------------------------------ */

/* v1 range search for one query with deletes skipped
 * (update.cuh:337-447, search.cuh:38-142, 178-194, update.cuh:219-335). */
static int v1_range_count(const orc_data *d, const orc_params *p, const orc_tree *t,
                          const int *is_delete, int qid, float r, unsigned char *flag)
{
    const int O = p->order, H = t->tree_h;
    memset(flag, 0, (size_t)t->max_node_num);
    flag[0] = 1;
    for (int l = 1; l < H; l++) {
        long off = level_offset(O, l), nn = ipow(O, l);
        for (long i = 0; i < nn; i++) {           /* findNextRnn */
            long nid = off + i, par = (nid - 1) / O;
            if (flag[par] != 1 || !t->exists[nid]) continue;
            float dq = (float)orc_dist(d, t->pid[nid], qid, ORC_ACC_F32);
            if (ring_lb(t, nid, O, dq) <= r) flag[nid] = 1;
        }
        for (long i = 0; i < nn; i++) {           /* updatePnodeFlag */
            long nid = off + i, par = (nid - 1) / O;
            if (flag[par] == 1 && t->exists[nid] && (nid - 1) % O == 0) flag[par] = 0;
        }
    }
    int cnt = 0;
    for (long nid = 0; nid < t->max_node_num; nid++) {
        if (flag[nid] != 1 || !t->is_leaf[nid]) continue;
        for (int s = 0; s < t->size[nid]; s++) {
            int id = t->id_list[t->lid[nid] + s];
            if (is_delete[id]) continue;
            double res = (id == qid) ? 0.0 : orc_dist(d, id, qid, ORC_ACC_F32);
            if ((float)res <= r) cnt++;
        }
    }
    return cnt;
}

static int live_range_count(const orc_data *d, const int *is_delete, int qid, float r)
{
    int cnt = 0;
    for (int o = 0; o < d->num; o++) {
        if (is_delete[o]) continue;
        double res = (o == qid) ? 0.0 : orc_dist(d, o, qid, ORC_ACC_F32);
        if ((float)res <= r) cnt++;
    }
    return cnt;
}

int orc_update_run(const orc_data *d0, const orc_params *p, int max_in_size,
                   const int *flags, const int *ids, int nops, float r,
                   int exact, int *counts_out, int *nq_out)
{
    orc_data d = *d0;
    const int dim = d.dim;
    const int is_str = d.metric == 6;
    float *rows = NULL; char *strs = NULL; int *lens = NULL;
    if (is_str) {
        strs = (char *)malloc((size_t)d.num * ORC_STR_STRIDE);
        lens = (int *)malloc(sizeof(int) * (size_t)d.num);
        memcpy(strs, d0->strs, (size_t)d.num * ORC_STR_STRIDE);
        memcpy(lens, d0->lens, sizeof(int) * (size_t)d.num);
        d.strs = strs; d.lens = lens;
    } else {
        rows = (float *)malloc(sizeof(float) * (size_t)d.num * dim);
        memcpy(rows, d0->rows, sizeof(float) * (size_t)d.num * dim);
        d.rows = rows;
    }
    orc_tree t;
    if (orc_build(&d, p, &t) != 0) return -1;
    int tree_size = d.num, in_size = 0, rnum = 0, delete_id = 0, nq = 0;
    int *insert_list = (int *)malloc(sizeof(int) * (size_t)(max_in_size + 1));
    int *is_delete = (int *)calloc((size_t)tree_size, sizeof(int));
    unsigned char *flag = (unsigned char *)malloc((size_t)t.max_node_num);

    for (int i = 0; i < nops; i++) {
        if (flags[i] == 0) {
            insert_list[in_size++] = ids[i];
            if (in_size == max_in_size) {
                /* compact live rows + cached inserts, then rebuild (update.cuh:484-540) */
                int live = 0;
                for (int j = 0; j < tree_size; j++) live += !is_delete[j];
                int nn = live + in_size, o = 0;
                if (is_str) {
                    char *ns = (char *)calloc((size_t)nn, ORC_STR_STRIDE);
                    int *nl = (int *)malloc(sizeof(int) * (size_t)nn);
                    for (int j = 0; j < tree_size; j++) if (!is_delete[j]) {
                        memcpy(ns + (size_t)o * ORC_STR_STRIDE, strs + (size_t)j * ORC_STR_STRIDE, (size_t)lens[j]);
                        nl[o++] = lens[j];
                    }
                    for (int j = 0; j < in_size; j++) {
                        int s = insert_list[j];
                        memcpy(ns + (size_t)o * ORC_STR_STRIDE, strs + (size_t)s * ORC_STR_STRIDE, (size_t)lens[s]);
                        nl[o++] = lens[s];
                    }
                    free(strs); free(lens); strs = ns; lens = nl;
                    d.strs = strs; d.lens = lens;
                } else {
                    float *nr = (float *)malloc(sizeof(float) * (size_t)nn * dim);
                    for (int j = 0; j < tree_size; j++) if (!is_delete[j])
                        memcpy(nr + (size_t)(o++) * dim, rows + (size_t)j * dim, sizeof(float) * (size_t)dim);
                    for (int j = 0; j < in_size; j++)
                        memcpy(nr + (size_t)(o++) * dim, rows + (size_t)insert_list[j] * dim, sizeof(float) * (size_t)dim);
                    free(rows); rows = nr; d.rows = rows;
                }
                d.num = nn;
                orc_tree_free(&t);
                if (orc_build(&d, p, &t) != 0) return -1;
                free(flag);
                flag = (unsigned char *)malloc((size_t)t.max_node_num);
                tree_size = nn;
                free(is_delete);
                is_delete = (int *)calloc((size_t)tree_size, sizeof(int));
                in_size = 0;
            }
        } else if (flags[i] == 1) {
            /* findIdx (update.cuh:118-143): logical id -> physical slot */
            int u = ids[i], del_before = 0, total_del = 0;
            for (int j = 0; j < tree_size; j++) total_del += is_delete[j];
            for (int j = 0; j < tree_size; j++) {
                del_before += is_delete[j];
                if (!is_delete[j] && j - del_before == u) delete_id = j;
            }
            for (int j = tree_size; j < tree_size + in_size; j++)
                if (j - total_del == u) delete_id = j;
            if (delete_id < tree_size) {
                is_delete[delete_id] = 1;
            } else {
                int e = delete_id - tree_size;
                for (int j = e; j + 1 < in_size; j++) insert_list[j] = insert_list[j + 1];
                in_size--;
            }
        } else {
            int qid = ids[i];
            int c = exact ? live_range_count(&d, is_delete, qid, r)
                          : v1_range_count(&d, p, &t, is_delete, qid, r, flag);
            if (in_size > 0) {
                rnum = 0;
                for (int j = 0; j < in_size; j++) {
                    float res = (float)orc_dist(&d, insert_list[j], qid, ORC_ACC_F32);
                    if (res <= r) rnum++;
                }
            }
            counts_out[nq++] = c + rnum;
        }
    }
    *nq_out = nq;
    orc_tree_free(&t);
    free(insert_list); free(is_delete); free(flag);
    free(rows); free(strs); free(lens);
    return 0;
}

/* ------------------------------------------------------------------------
 * Stream update whose inserts bring new rows (an extension: the reference's
 * insert copies an existing physical row, update.cuh:481, 186).  Same op
 * semantics as orc_update_run otherwise; exact counts (live rows scanned).
 * The cache list holds copies of the inserted rows; the compaction appends
 * them after the live rows, as getNewData does (update.cuh:159-217). */

/* F32-site distance of two rows (search_naive.cuh:31-68), through orc_dist
 * on a two-row scratch set: a first (the cached row), then b (the query). */
static float row_pair_dist_f32(int dim, int metric, const float *a, const float *b, float *tmp)
{
    memcpy(tmp, a, sizeof(float) * (size_t)dim);
    memcpy(tmp + dim, b, sizeof(float) * (size_t)dim);
    orc_data two = {dim, 2, metric, tmp, NULL, NULL};
    return (float)orc_dist(&two, 0, 1, ORC_ACC_F32);
}

int orc_update_run_rows(const orc_data *d0, int max_in_size, const int *flags, const int *ids, int nops,
                        const float *new_rows, int n_new, float r, int *counts_out, int *nq_out)
{
    if (d0->metric == 6 || max_in_size < 1) return -1;
    orc_data d = *d0;
    const int dim = d.dim;
    float *rows = (float *)malloc(sizeof(float) * (size_t)d.num * dim);
    memcpy(rows, d0->rows, sizeof(float) * (size_t)d.num * dim);
    d.rows = rows;
    float *cache = (float *)malloc(sizeof(float) * (size_t)max_in_size * dim);
    float *tmp = (float *)malloc(sizeof(float) * 2 * (size_t)dim);
    int tree_size = d.num, in_size = 0, rnum = 0, delete_id = 0, nq = 0, rc = 0;
    int *is_delete = (int *)calloc((size_t)tree_size, sizeof(int));
    for (int i = 0; i < nops && rc == 0; i++) {
        if (flags[i] == 0) {
            if (ids[i] < 0 || ids[i] >= n_new) { rc = -2; break; }
            memcpy(cache + (size_t)(in_size++) * dim, new_rows + (size_t)ids[i] * dim, sizeof(float) * (size_t)dim);
            if (in_size == max_in_size) {
                int live = 0;
                for (int j = 0; j < tree_size; j++) live += !is_delete[j];
                const int nn = live + in_size;
                float *nr = (float *)malloc(sizeof(float) * (size_t)nn * dim);
                int o = 0;
                for (int j = 0; j < tree_size; j++)
                    if (!is_delete[j]) memcpy(nr + (size_t)(o++) * dim, rows + (size_t)j * dim, sizeof(float) * (size_t)dim);
                memcpy(nr + (size_t)o * dim, cache, sizeof(float) * (size_t)in_size * dim);
                free(rows);
                rows = nr;
                d.rows = rows;
                d.num = nn;
                tree_size = nn;
                free(is_delete);
                is_delete = (int *)calloc((size_t)tree_size, sizeof(int));
                in_size = 0;
            }
        } else if (flags[i] == 1) {
            /* findIdx (update.cuh:118-143) */
            int u = ids[i], del_before = 0, total_del = 0;
            for (int j = 0; j < tree_size; j++) total_del += is_delete[j];
            for (int j = 0; j < tree_size; j++) {
                del_before += is_delete[j];
                if (!is_delete[j] && j - del_before == u) delete_id = j;
            }
            for (int j = tree_size; j < tree_size + in_size; j++)
                if (j - total_del == u) delete_id = j;
            if (delete_id < tree_size) {
                is_delete[delete_id] = 1;
            } else if (in_size > 0) {
                int e = delete_id - tree_size;
                if (e >= in_size) e = in_size - 1;
                memmove(cache + (size_t)e * dim, cache + (size_t)(e + 1) * dim,
                        sizeof(float) * (size_t)(in_size - 1 - e) * dim);
                in_size--;
            }
        } else {
            const int qid = ids[i];
            if (qid < 0 || qid >= tree_size) { rc = -3; break; }
            const int c = live_range_count(&d, is_delete, qid, r);
            if (in_size > 0) {
                rnum = 0;
                for (int j = 0; j < in_size; j++)
                    if (row_pair_dist_f32(dim, d.metric, cache + (size_t)j * dim, rows + (size_t)qid * dim, tmp) <= r)
                        rnum++;
            }
            counts_out[nq++] = c + rnum;
        }
    }
    *nq_out = nq;
    free(rows); free(cache); free(tmp); free(is_delete);
    return rc;
}
