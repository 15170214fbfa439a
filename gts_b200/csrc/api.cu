// api.cu -- the C ABI (include/gts_b200.h) over the device index.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <string>
#include <vector>
#include "index.cuh"

static thread_local char g_err[1024] = "";

extern "C" void gts_set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

extern "C" const char *gts_last_error(void) { return g_err; }

extern "C" void gts_params_default(gts_params *p)
{
    if (!p) return;
    p->tree_order = 10;    // tree.cuh:31
    p->max_size = 20;      // tree.cuh:32
    p->max_h = 3;          // tree.cuh:33
    p->dis_code = 100;     // tree.cuh:34
    p->infi_dis = 10000;   // tree.cuh:35
    p->max_in_size = 10;   // update.cuh:16
    p->mem_budget_gb = 0;
}

gts::DevTree gts_index::dev() const
{
    gts::DevTree t;
    t.num = num; t.dim = dim; t.metric = metric;
    t.order = params.tree_order; t.max_size = params.max_size; t.max_h = params.max_h;
    t.tree_h = tree_h; t.max_node_num = max_node_num;
    t.dis_code = params.dis_code; t.infi_dis = params.infi_dis;
    t.rows = rows; t.trows = trows; t.strs = strs; t.tstrs = tstrs; t.lens = lens; t.tlens = tlens;
    t.tsig = tsig;
    t.id_list = id_list; t.pos_of_id = pos_of_id;
    t.node_pid = node_pid; t.node_size = node_size; t.node_lid = node_lid; t.node_pivot = node_pivot;
    t.node_min_dis = node_min_dis; t.node_flags = node_flags;
    return t;
}

// ---------------------------------------------------------------- helpers

static int check_device()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n < 1) {
        cudaGetLastError();
        gts_set_error("no CUDA device available: %s", cudaGetErrorString(e));
        return GTS_ERR_CUDA;
    }
    return GTS_OK;
}

static int check_params(const gts_params *p)
{
    if (p->tree_order < 2 || p->max_size < 1 || p->max_h < 1 || p->dis_code < 1 || p->infi_dis < 1 ||
        p->max_in_size < 1 || !(p->mem_budget_gb >= 0.0)) {
        gts_set_error("invalid parameters (order %d, max_size %d, max_h %d, mem_budget_gb %g)", p->tree_order,
                      p->max_size, p->max_h, p->mem_budget_gb);
        return GTS_ERR_INVALID;
    }
    return GTS_OK;
}

static bool metric_ok(int m) { return m == 0 || m == 1 || m == 2 || m == 5 || m == 6; }

// ---------------------------------------------------------------- I/O
// The text formats of file.cuh:28-152 and update.cuh:43-95.  Parsing is a
// single pass with strtof/strtol over the whole file instead of a
// stringstream per token.

static bool read_file(const char *path, std::string &out)
{
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    out.resize(n > 0 ? (size_t)n : 0);
    size_t got = n > 0 ? fread(&out[0], 1, (size_t)n, f) : 0;
    fclose(f);
    return got == out.size();
}

extern "C" int gts_load(const char *path, int *dim, int *num, int *metric, float **rows, char **strs,
                        int **lens)
{
    if (!path || !dim || !num || !metric) {
        gts_set_error("gts_load: null argument");
        return GTS_ERR_INVALID;
    }
    std::string buf;
    if (!read_file(path, buf)) {
        gts_set_error("open file error: %s", path);
        return GTS_ERR_IO;
    }
    const char *p = buf.c_str();
    char *e = nullptr;
    long h[3];
    for (int i = 0; i < 3; i++) {
        h[i] = strtol(p, &e, 10);
        if (e == p) {
            gts_set_error("%s: bad header", path);
            return GTS_ERR_IO;
        }
        p = e;
    }
    *dim = (int)h[0];
    *num = (int)h[1];
    *metric = (int)h[2];
    if (*num < 0 || *dim < 1 || !metric_ok(*metric)) {
        gts_set_error("%s: bad header values (%ld %ld %ld)", path, h[0], h[1], h[2]);
        return GTS_ERR_IO;
    }
    while (*p && *p != '\n') p++;   // rest of the header line
    if (*p == '\n') p++;
    if (*metric == 6) {
        char *s = (char *)calloc((size_t)*num * GTS_STR_STRIDE + 1, 1);
        int *l = (int *)calloc((size_t)*num + 1, sizeof(int));
        for (int i = 0; i < *num && *p; i++) {
            const char *ls = p;
            while (*p && *p != '\n') p++;
            size_t len = (size_t)(p - ls);
            if (len > GTS_STR_STRIDE - 1) {
                free(s); free(l);
                gts_set_error("%s: string %d longer than %d characters", path, i, GTS_STR_STRIDE - 1);
                return GTS_ERR_IO;
            }
            memcpy(s + (size_t)i * GTS_STR_STRIDE, ls, len);
            l[i] = (int)len;
            if (*p == '\n') p++;
        }
        if (strs) *strs = s; else free(s);
        if (lens) *lens = l; else free(l);
        if (rows) *rows = nullptr;
    } else {
        size_t n = (size_t)*num * *dim;
        float *r = (float *)malloc((n ? n : 1) * sizeof(float));
        for (size_t i = 0; i < n; i++) {
            float v = strtof(p, &e);
            if (e == p) {
                free(r);
                gts_set_error("%s: expected %zu values, found %zu", path, n, i);
                return GTS_ERR_IO;
            }
            r[i] = v;
            p = e;
        }
        if (rows) *rows = r; else free(r);
        if (strs) *strs = nullptr;
        if (lens) *lens = nullptr;
    }
    return GTS_OK;
}

extern "C" int gts_load_queries(const char *path, int **qids, int *qnum)
{
    std::string buf;
    if (!qids || !qnum || !read_file(path, buf)) {
        gts_set_error("open file error: %s", path ? path : "(null)");
        return GTS_ERR_IO;
    }
    const char *p = buf.c_str();
    char *e;
    long n = strtol(p, &e, 10);
    if (e == p || n < 0) {
        gts_set_error("%s: bad query count", path);
        return GTS_ERR_IO;
    }
    p = e;
    int *q = (int *)malloc(sizeof(int) * (size_t)(n ? n : 1));
    for (long i = 0; i < n; i++) {
        long v = strtol(p, &e, 10);
        if (e == p) {
            free(q);
            gts_set_error("%s: expected %ld ids, found %ld", path, n, i);
            return GTS_ERR_IO;
        }
        q[i] = (int)v;
        p = e;
    }
    *qids = q;
    *qnum = (int)n;
    return GTS_OK;
}

extern "C" int gts_load_updates(const char *path, int **flags, int **ids, int *nops)
{
    std::string buf;
    if (!flags || !ids || !nops || !read_file(path, buf)) {
        gts_set_error("open file error: %s", path ? path : "(null)");
        return GTS_ERR_IO;
    }
    const char *p = buf.c_str();
    char *e;
    long n = strtol(p, &e, 10);
    if (e == p || n < 0) {
        gts_set_error("%s: bad op count", path);
        return GTS_ERR_IO;
    }
    p = e;
    int *f = (int *)malloc(sizeof(int) * (size_t)(n ? n : 1));
    int *d = (int *)malloc(sizeof(int) * (size_t)(n ? n : 1));
    for (long i = 0; i < n; i++) {
        long a = strtol(p, &e, 10);
        if (e == p) break;
        p = e;
        long b = strtol(p, &e, 10);
        if (e == p) {
            free(f); free(d);
            gts_set_error("%s: op %ld incomplete", path, i);
            return GTS_ERR_IO;
        }
        p = e;
        f[i] = (int)a;
        d[i] = (int)b;
    }
    *flags = f;
    *ids = d;
    *nops = (int)n;
    return GTS_OK;
}

extern "C" void gts_free_host(void *p) { free(p); }

// ---------------------------------------------------------------- index

static int index_alloc_common(gts_index *idx)
{
    size_t acct = 0;
    int rc;
    if ((rc = gts::dev_alloc(&idx->d_counter, 1, &acct)) != GTS_OK) return rc;
    if ((rc = gts::dev_alloc(&idx->d_status, 1, &acct)) != GTS_OK) return rc;
    if ((rc = gts::dev_alloc(&idx->d_stats, gts::kStatsN, &acct)) != GTS_OK) return rc;
    cudaMemset(idx->d_stats, 0, gts::kStatsN * sizeof(unsigned long long));
    idx->device_bytes += acct;
    return GTS_OK;
}

static int build_common(int dim, int num, int metric, const float *rows, const char *strs,
                        const int *lens, cudaMemcpyKind kind, const gts_params *params,
                        cudaStream_t stream, gts_index **out)
{
    if (!out) {
        gts_set_error("out is null");
        return GTS_ERR_INVALID;
    }
    *out = nullptr;
    int rc;
    gts_params p;
    if (params) p = *params; else gts_params_default(&p);
    if ((rc = check_params(&p))) return rc;
    if (num < 1 || dim < 1 || !metric_ok(metric)) {
        gts_set_error("invalid data shape (dim %d, num %d, metric %d)", dim, num, metric);
        return GTS_ERR_INVALID;
    }
    if (metric == 6 ? (!strs || !lens) : !rows) {
        gts_set_error("missing %s input", metric == 6 ? "string" : "row");
        return GTS_ERR_INVALID;
    }
    if ((rc = check_device())) return rc;
    if (metric == 6 && kind == cudaMemcpyHostToDevice) {
        for (int i = 0; i < num; i++) {
            if (lens[i] < 0 || lens[i] > GTS_STR_STRIDE - 1) {
                gts_set_error("string %d has length %d (allowed 0..%d)", i, lens[i], GTS_STR_STRIDE - 1);
                return GTS_ERR_INVALID;
            }
        }
    }
    gts_index *idx = new gts_index();
    idx->params = p;
    idx->num = num;
    idx->dim = metric == 6 ? 1 : dim;
    idx->metric = metric;
    idx->stream = stream;
    size_t acct = 0;
    if ((rc = index_alloc_common(idx)) != GTS_OK) { gts_index_free(idx); return rc; }
    if (metric == 6) {
        if ((rc = gts::dev_alloc(&idx->strs, (size_t)num * GTS_STR_STRIDE, &acct)) ||
            (rc = gts::dev_alloc(&idx->lens, (size_t)num, &acct))) {
            gts_index_free(idx);
            return rc;
        }
        cudaMemcpyAsync(idx->strs, strs, (size_t)num * GTS_STR_STRIDE, kind, stream);
        cudaMemcpyAsync(idx->lens, lens, sizeof(int) * (size_t)num, kind, stream);
    } else {
        if ((rc = gts::dev_alloc(&idx->rows, (size_t)num * dim, &acct))) {
            gts_index_free(idx);
            return rc;
        }
        cudaMemcpyAsync(idx->rows, rows, sizeof(float) * (size_t)num * dim, kind, stream);
    }
    idx->device_bytes += acct;
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        gts_set_error("copy of the data set failed: %s", cudaGetErrorString(e));
        gts_index_free(idx);
        return GTS_ERR_CUDA;
    }
    if ((rc = gts::build_tree(idx, stream)) != GTS_OK) {
        gts_index_free(idx);
        return rc;
    }
    *out = idx;
    return GTS_OK;
}

extern "C" int gts_index_build(int dim, int num, int metric, const float *rows, const char *strs,
                               const int *lens, const gts_params *params, gts_index **out)
{
    return build_common(dim, num, metric, rows, strs, lens, cudaMemcpyHostToDevice, params, 0, out);
}

extern "C" int gts_index_build_device(int dim, int num, int metric, const float *d_rows,
                                      const char *d_strs, const int *d_lens, const gts_params *params,
                                      void *stream, gts_index **out)
{
    return build_common(dim, num, metric, d_rows, d_strs, d_lens, cudaMemcpyDeviceToDevice, params,
                        (cudaStream_t)stream, out);
}

extern "C" int gts_index_info_get(const gts_index *idx, gts_index_info *info)
{
    if (!idx || !info) {
        gts_set_error("null argument");
        return GTS_ERR_INVALID;
    }
    info->num = idx->num;
    info->dim = idx->dim;
    info->metric = idx->metric;
    info->tree_h = idx->tree_h;
    info->max_node_num = idx->max_node_num;
    info->tree_order = idx->params.tree_order;
    info->max_size = idx->params.max_size;
    info->device_bytes = idx->device_bytes;
    return GTS_OK;
}

extern "C" int gts_index_export(const gts_index *idx, int *id_list, int *pid, float *min_dis, int *size,
                                int *lid, int *is_leaf, int *exists)
{
    if (!idx) {
        gts_set_error("null index");
        return GTS_ERR_INVALID;
    }
    const int m = idx->max_node_num, n = idx->num;
    if (id_list) GTS_CUDA_TRY(cudaMemcpy(id_list, idx->id_list, sizeof(int) * n, cudaMemcpyDeviceToHost));
    if (pid) GTS_CUDA_TRY(cudaMemcpy(pid, idx->node_pid, sizeof(int) * m, cudaMemcpyDeviceToHost));
    if (min_dis) GTS_CUDA_TRY(cudaMemcpy(min_dis, idx->node_min_dis, sizeof(float) * m, cudaMemcpyDeviceToHost));
    if (size) GTS_CUDA_TRY(cudaMemcpy(size, idx->node_size, sizeof(int) * m, cudaMemcpyDeviceToHost));
    if (lid) GTS_CUDA_TRY(cudaMemcpy(lid, idx->node_lid, sizeof(int) * m, cudaMemcpyDeviceToHost));
    if (is_leaf || exists) {
        std::vector<uint8_t> fl(m);
        GTS_CUDA_TRY(cudaMemcpy(fl.data(), idx->node_flags, m, cudaMemcpyDeviceToHost));
        for (int i = 0; i < m; i++) {
            if (is_leaf) is_leaf[i] = (fl[i] & gts::kLeaf) ? 1 : 0;
            if (exists) exists[i] = (fl[i] & gts::kExists) ? 1 : 0;
        }
    }
    return GTS_OK;
}

extern "C" void gts_index_free(gts_index *idx)
{
    if (!idx) return;
    gts::free_tree(idx);
    gts::free_data(idx);
    if (idx->d_counter) cudaFree(idx->d_counter);
    if (idx->d_status) cudaFree(idx->d_status);
    if (idx->d_stats) cudaFree(idx->d_stats);
    if (idx->scratch) cudaFree(idx->scratch);
    if (idx->split_buf) cudaFree(idx->split_buf);
    if (idx->io) cudaFree(idx->io);
    for (int i = 0; i < gts_index::kGraphSlots; i++)
        if (idx->graph_exec[i]) cudaGraphExecDestroy(idx->graph_exec[i]);
    if (idx->graph_stream) cudaStreamDestroy(idx->graph_stream);
    for (int i = 0; i < 2; i++)
        if (idx->graph_ev[i]) cudaEventDestroy(idx->graph_ev[i]);
    if (idx->mlp_P) cudaFree(idx->mlp_P);
    if (idx->mlp_norm) cudaFree(idx->mlp_norm);
    if (idx->mlp_piv) cudaFree(idx->mlp_piv);
    for (int i = 0; i < 2; i++)
        if (idx->fev[i]) cudaEventDestroy(idx->fev[i]);
    delete idx;
}

extern "C" int gts_search_stats(const gts_index *idx, unsigned long long *out8)
{
    if (!idx || !out8) {
        gts_set_error("null argument");
        return GTS_ERR_INVALID;
    }
    GTS_CUDA_TRY(cudaMemcpy(out8, idx->d_stats, gts::kStatsN * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    return GTS_OK;
}

extern "C" int gts_filter_timing(gts_index *idx, int reset, double *ms, long long *launches)
{
    if (!idx) {
        gts_set_error("null argument");
        return GTS_ERR_INVALID;
    }
    if (reset) {
        for (int i = 0; i < 2; i++)
            if (!idx->fev[i]) GTS_CUDA_TRY(cudaEventCreate(&idx->fev[i]));
        idx->filter_ms = 0.0;
        idx->filter_launches = 0;
        idx->time_filter = true;
    }
    if (ms) *ms = idx->filter_ms;
    if (launches) *launches = idx->filter_launches;
    return GTS_OK;
}

extern "C" int gts_kernel_launches(const gts_index *idx, long long *count)
{
    if (!idx || !count) {
        gts_set_error("null argument");
        return GTS_ERR_INVALID;
    }
    *count = idx->kernel_launches;
    return GTS_OK;
}

extern "C" int gts_index_prepare(gts_index *idx, int form, void *stream, int *prepared)
{
    if (!idx || (form != GTS_FORM_PLAIN && form != GTS_FORM_FAST && form != GTS_FORM_PLAIN_LEARNED)) {
        gts_set_error("gts_index_prepare: invalid argument");
        return GTS_ERR_INVALID;
    }
    int done = 0, rc = GTS_OK;
    if (form == GTS_FORM_FAST) rc = gts::fast_prepare_now(idx, (cudaStream_t)stream, &done);
    if (prepared) *prepared = done;
    return rc;
}

extern "C" int gts_index_set_stream(gts_index *idx, void *stream)
{
    if (!idx) {
        gts_set_error("null index");
        return GTS_ERR_INVALID;
    }
    idx->stream = (cudaStream_t)stream;
    return GTS_OK;
}

// ---------------------------------------------------------------- search

namespace {
// Device scratch for the host-buffer entry points, freed on scope exit.
struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    int alloc(size_t bytes)
    {
        if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            gts_set_error("cudaMalloc of %zu bytes failed", bytes);
            return GTS_ERR_NOMEM;
        }
        return GTS_OK;
    }
};

// Carves consecutive 256-byte aligned buffers out of idx->io.
struct IoCarve {
    size_t sizes[6];
    int n = 0;
    void add(size_t b) { sizes[n++] = (b + 255) & ~(size_t)255; }
    int get(gts_index *idx, void **out)
    {
        size_t total = 0;
        for (int i = 0; i < n; i++) total += sizes[i];
        int rc = gts::ensure_io(idx, total);
        if (rc) return rc;
        unsigned char *p = (unsigned char *)idx->io;
        for (int i = 0; i < n; i++) {
            out[i] = p;
            p += sizes[i];
        }
        return GTS_OK;
    }
};

int check_qids(const gts_index *idx, const int *qids, int qnum)
{
    for (int i = 0; i < qnum; i++) {
        if (qids[i] < 0 || qids[i] >= idx->num) {
            gts_set_error("query id %d out of range [0, %d)", qids[i], idx->num);
            return GTS_ERR_INVALID;
        }
    }
    return GTS_OK;
}
}  // namespace

extern "C" int gts_knn_device(gts_index *idx, const int *d_qids, int qnum, int k, int form, float *d_kth,
                              int *d_ids, float *d_dists, void *stream)
{
    if (!idx || (qnum > 0 && (!d_qids || !d_kth)) || qnum < 0) {
        gts_set_error("gts_knn_device: invalid argument");
        return GTS_ERR_INVALID;
    }
    return gts::search_knn(idx, d_qids, qnum, k, form, d_kth, d_ids, d_dists, (cudaStream_t)stream);
}

extern "C" int gts_knn(gts_index *idx, const int *qids, int qnum, int k, int form, float *kth_out,
                       int *ids_out, float *dists_out)
{
    if (!idx || qnum < 0 || (qnum > 0 && (!qids || !kth_out))) {
        gts_set_error("gts_knn: invalid argument");
        return GTS_ERR_INVALID;
    }
    if (qnum == 0) return GTS_OK;
    int rc = check_qids(idx, qids, qnum);
    if (rc) return rc;
    cudaStream_t s = idx->stream;
    IoCarve io;
    io.add(sizeof(int) * (size_t)qnum);
    io.add(sizeof(float) * (size_t)qnum);
    io.add(ids_out ? sizeof(int) * (size_t)qnum * (k > 0 ? k : 1) : 0);
    io.add(dists_out ? sizeof(float) * (size_t)qnum * (k > 0 ? k : 1) : 0);
    void *buf[4];
    if ((rc = io.get(idx, buf))) return rc;
    struct { void *p; } bq{buf[0]}, bk{buf[1]}, bi{ids_out ? buf[2] : nullptr}, bd{dists_out ? buf[3] : nullptr};
    GTS_CUDA_TRY(cudaMemcpyAsync(bq.p, qids, sizeof(int) * (size_t)qnum, cudaMemcpyHostToDevice, s));
    rc = gts::search_knn(idx, (int *)bq.p, qnum, k, form, (float *)bk.p, (int *)bi.p, (float *)bd.p, s);
    if (rc) return rc;
    GTS_CUDA_TRY(cudaMemcpyAsync(kth_out, bk.p, sizeof(float) * (size_t)qnum, cudaMemcpyDeviceToHost, s));
    if (ids_out)
        GTS_CUDA_TRY(cudaMemcpyAsync(ids_out, bi.p, sizeof(int) * (size_t)qnum * k, cudaMemcpyDeviceToHost, s));
    if (dists_out)
        GTS_CUDA_TRY(cudaMemcpyAsync(dists_out, bd.p, sizeof(float) * (size_t)qnum * k, cudaMemcpyDeviceToHost, s));
    GTS_CUDA_TRY(cudaStreamSynchronize(s));
    return GTS_OK;
}

extern "C" int gts_range_device(gts_index *idx, const int *d_qids, int qnum, float r, int *d_counts,
                                void *stream)
{
    if (!idx || qnum < 0 || (qnum > 0 && (!d_qids || !d_counts))) {
        gts_set_error("gts_range_device: invalid argument");
        return GTS_ERR_INVALID;
    }
    return gts::search_range(idx, d_qids, qnum, r, d_counts, nullptr, (cudaStream_t)stream);
}

extern "C" int gts_range(gts_index *idx, const int *qids, int qnum, float r, int *counts_out)
{
    if (!idx || qnum < 0 || (qnum > 0 && (!qids || !counts_out))) {
        gts_set_error("gts_range: invalid argument");
        return GTS_ERR_INVALID;
    }
    if (qnum == 0) return GTS_OK;
    int rc = check_qids(idx, qids, qnum);
    if (rc) return rc;
    cudaStream_t s = idx->stream;
    IoCarve io;
    io.add(sizeof(int) * (size_t)qnum);
    io.add(sizeof(int) * (size_t)qnum);
    void *buf[2];
    if ((rc = io.get(idx, buf))) return rc;
    struct { void *p; } bq{buf[0]}, bc{buf[1]};
    GTS_CUDA_TRY(cudaMemcpyAsync(bq.p, qids, sizeof(int) * (size_t)qnum, cudaMemcpyHostToDevice, s));
    rc = gts::search_range(idx, (int *)bq.p, qnum, r, (int *)bc.p, nullptr, s);
    if (rc) return rc;
    GTS_CUDA_TRY(cudaMemcpyAsync(counts_out, bc.p, sizeof(int) * (size_t)qnum, cudaMemcpyDeviceToHost, s));
    GTS_CUDA_TRY(cudaStreamSynchronize(s));
    return GTS_OK;
}

extern "C" int gts_range_form_device(gts_index *idx, const int *d_qids, int qnum, float r, int form,
                                     int *d_counts, void *stream)
{
    if (!idx || qnum < 0 || (qnum > 0 && (!d_qids || !d_counts)) ||
        (form != GTS_FORM_PLAIN && form != GTS_FORM_FAST)) {
        gts_set_error("gts_range_form_device: invalid argument (form must be GTS_FORM_PLAIN or GTS_FORM_FAST)");
        return GTS_ERR_INVALID;
    }
    if (form == GTS_FORM_FAST) return gts::search_range_fast(idx, d_qids, qnum, r, d_counts, (cudaStream_t)stream);
    return gts::search_range(idx, d_qids, qnum, r, d_counts, nullptr, (cudaStream_t)stream);
}

extern "C" int gts_range_form(gts_index *idx, const int *qids, int qnum, float r, int form, int *counts_out)
{
    if (!idx || qnum < 0 || (qnum > 0 && (!qids || !counts_out)) ||
        (form != GTS_FORM_PLAIN && form != GTS_FORM_FAST)) {
        gts_set_error("gts_range_form: invalid argument (form must be GTS_FORM_PLAIN or GTS_FORM_FAST)");
        return GTS_ERR_INVALID;
    }
    if (qnum == 0) return GTS_OK;
    int rc = check_qids(idx, qids, qnum);
    if (rc) return rc;
    cudaStream_t s = idx->stream;
    IoCarve io;
    io.add(sizeof(int) * (size_t)qnum);
    io.add(sizeof(int) * (size_t)qnum);
    void *buf[2];
    if ((rc = io.get(idx, buf))) return rc;
    GTS_CUDA_TRY(cudaMemcpyAsync(buf[0], qids, sizeof(int) * (size_t)qnum, cudaMemcpyHostToDevice, s));
    rc = form == GTS_FORM_FAST ? gts::search_range_fast(idx, (int *)buf[0], qnum, r, (int *)buf[1], s)
                               : gts::search_range(idx, (int *)buf[0], qnum, r, (int *)buf[1], nullptr, s);
    if (rc) return rc;
    GTS_CUDA_TRY(cudaMemcpyAsync(counts_out, buf[1], sizeof(int) * (size_t)qnum, cudaMemcpyDeviceToHost, s));
    GTS_CUDA_TRY(cudaStreamSynchronize(s));
    return GTS_OK;
}

extern "C" int gts_range_ids(gts_index *idx, const int *qids, int qnum, float r, int *counts_out,
                             int *offsets_out, int *ids_out, float *dists_out, size_t capacity)
{
    if (!idx || qnum < 0 || (qnum > 0 && (!qids || !counts_out || !offsets_out))) {
        gts_set_error("gts_range_ids: invalid argument");
        return GTS_ERR_INVALID;
    }
    if (qnum == 0) return GTS_OK;
    int rc = gts_range(idx, qids, qnum, r, counts_out);
    if (rc) return rc;
    size_t total = 0;
    for (int i = 0; i < qnum; i++) {
        offsets_out[i] = (int)total;
        total += (size_t)counts_out[i];
    }
    if (total > capacity || total > 0x7fffffff) {
        gts_set_error("range result needs %zu entries, capacity %zu", total, capacity);
        return GTS_ERR_NOMEM;
    }
    if (total == 0) return GTS_OK;
    cudaStream_t s = idx->stream;
    DevBuf bq, bc, bo, bi, bd;
    if ((rc = bq.alloc(sizeof(int) * (size_t)qnum)) || (rc = bc.alloc(sizeof(int) * (size_t)qnum)) ||
        (rc = bo.alloc(sizeof(int) * (size_t)qnum)) || (rc = bi.alloc(sizeof(int) * total)) ||
        (rc = bd.alloc(sizeof(float) * total)))
        return rc;
    GTS_CUDA_TRY(cudaMemcpyAsync(bq.p, qids, sizeof(int) * (size_t)qnum, cudaMemcpyHostToDevice, s));
    GTS_CUDA_TRY(cudaMemcpyAsync(bo.p, offsets_out, sizeof(int) * (size_t)qnum, cudaMemcpyHostToDevice, s));
    rc = gts::search_range_ids(idx, (int *)bq.p, qnum, r, (int *)bc.p, (int *)bi.p, (float *)bd.p,
                               (int *)bo.p, s);
    if (rc) return rc;
    std::vector<int> ids(total);
    std::vector<float> ds(total);
    GTS_CUDA_TRY(cudaMemcpyAsync(ids.data(), bi.p, sizeof(int) * total, cudaMemcpyDeviceToHost, s));
    GTS_CUDA_TRY(cudaMemcpyAsync(ds.data(), bd.p, sizeof(float) * total, cudaMemcpyDeviceToHost, s));
    GTS_CUDA_TRY(cudaStreamSynchronize(s));
    // order each query's hits by (distance, id) for a deterministic layout
    for (int qi = 0; qi < qnum; qi++) {
        size_t b = (size_t)offsets_out[qi], n = (size_t)counts_out[qi];
        std::vector<std::pair<float, int>> v(n);
        for (size_t j = 0; j < n; j++) v[j] = {ds[b + j], ids[b + j]};
        std::sort(v.begin(), v.end());
        for (size_t j = 0; j < n; j++) {
            if (ids_out) ids_out[b + j] = v[j].second;
            if (dists_out) dists_out[b + j] = v[j].first;
        }
    }
    return GTS_OK;
}

// ---------------------------------------------------------------- queries given as data

static int check_rows_args(const gts_index *idx, const void *qrows, const char *qstrs, const int *qlens, int qnum,
                           const char *fn)
{
    if (!idx || qnum < 0) {
        gts_set_error("%s: invalid argument", fn);
        return GTS_ERR_INVALID;
    }
    if (qnum > 0 && (idx->metric == 6 ? (!qstrs || !qlens) : !qrows)) {
        gts_set_error("%s: the index's metric takes query %s", fn, idx->metric == 6 ? "strings and lengths" : "rows");
        return GTS_ERR_INVALID;
    }
    return GTS_OK;
}

extern "C" int gts_knn_rows_device(gts_index *idx, const float *d_qrows, const char *d_qstrs, const int *d_qlens,
                                   int qnum, int k, float *d_kth, int *d_ids, float *d_dists, void *stream)
{
    int rc = check_rows_args(idx, d_qrows, d_qstrs, d_qlens, qnum, "gts_knn_rows_device");
    if (rc) return rc;
    if (qnum > 0 && !d_kth) {
        gts_set_error("gts_knn_rows_device: kth output is null");
        return GTS_ERR_INVALID;
    }
    if (qnum == 0) return GTS_OK;
    return gts::search_knn_rows(idx, idx->metric == 6 ? nullptr : d_qrows, idx->metric == 6 ? d_qstrs : nullptr,
                                idx->metric == 6 ? d_qlens : nullptr, qnum, k, d_kth, d_ids, d_dists,
                                (cudaStream_t)stream);
}

// Host query data copied into idx->io: rows, or strings and their lengths.
static int stage_query_data(gts_index *idx, const float *qrows, const char *qstrs, const int *qlens, int qnum,
                            size_t out_bytes, size_t out2_bytes, void **bufs)
{
    const bool str = idx->metric == 6;
    if (str) {
        for (int i = 0; i < qnum; i++)
            if (qlens[i] < 0 || qlens[i] > GTS_STR_STRIDE - 1) {
                gts_set_error("query string %d has length %d (allowed 0..%d)", i, qlens[i], GTS_STR_STRIDE - 1);
                return GTS_ERR_INVALID;
            }
    }
    IoCarve io;
    io.add(str ? (size_t)qnum * GTS_STR_STRIDE : sizeof(float) * (size_t)qnum * idx->dim);
    io.add(str ? sizeof(int) * (size_t)qnum : 0);
    io.add(out_bytes);
    io.add(out2_bytes);
    io.add(out2_bytes);
    int rc = io.get(idx, bufs);
    if (rc) return rc;
    cudaStream_t s = idx->stream;
    if (str) {
        GTS_CUDA_TRY(cudaMemcpyAsync(bufs[0], qstrs, (size_t)qnum * GTS_STR_STRIDE, cudaMemcpyHostToDevice, s));
        GTS_CUDA_TRY(cudaMemcpyAsync(bufs[1], qlens, sizeof(int) * (size_t)qnum, cudaMemcpyHostToDevice, s));
    } else {
        GTS_CUDA_TRY(cudaMemcpyAsync(bufs[0], qrows, sizeof(float) * (size_t)qnum * idx->dim, cudaMemcpyHostToDevice,
                                     s));
    }
    return GTS_OK;
}

extern "C" int gts_knn_rows(gts_index *idx, const float *qrows, const char *qstrs, const int *qlens, int qnum, int k,
                            float *kth_out, int *ids_out, float *dists_out)
{
    int rc = check_rows_args(idx, qrows, qstrs, qlens, qnum, "gts_knn_rows");
    if (rc) return rc;
    if (qnum > 0 && !kth_out) {
        gts_set_error("gts_knn_rows: kth output is null");
        return GTS_ERR_INVALID;
    }
    if (qnum == 0) return GTS_OK;
    const size_t kk = (size_t)(k > 0 ? k : 1) * (size_t)qnum;
    void *b[5];
    if ((rc = stage_query_data(idx, qrows, qstrs, qlens, qnum, sizeof(float) * (size_t)qnum, sizeof(int) * kk, b)))
        return rc;
    const bool str = idx->metric == 6;
    cudaStream_t s = idx->stream;
    rc = gts::search_knn_rows(idx, str ? nullptr : (const float *)b[0], str ? (const char *)b[0] : nullptr,
                              str ? (const int *)b[1] : nullptr, qnum, k, (float *)b[2],
                              ids_out ? (int *)b[3] : nullptr, dists_out ? (float *)b[4] : nullptr, s);
    if (rc) return rc;
    GTS_CUDA_TRY(cudaMemcpyAsync(kth_out, b[2], sizeof(float) * (size_t)qnum, cudaMemcpyDeviceToHost, s));
    if (ids_out) GTS_CUDA_TRY(cudaMemcpyAsync(ids_out, b[3], sizeof(int) * kk, cudaMemcpyDeviceToHost, s));
    if (dists_out) GTS_CUDA_TRY(cudaMemcpyAsync(dists_out, b[4], sizeof(float) * kk, cudaMemcpyDeviceToHost, s));
    GTS_CUDA_TRY(cudaStreamSynchronize(s));
    return GTS_OK;
}

extern "C" int gts_range_rows(gts_index *idx, const float *qrows, const char *qstrs, const int *qlens, int qnum,
                              float r, int *counts_out)
{
    int rc = check_rows_args(idx, qrows, qstrs, qlens, qnum, "gts_range_rows");
    if (rc) return rc;
    if (qnum > 0 && !counts_out) {
        gts_set_error("gts_range_rows: counts output is null");
        return GTS_ERR_INVALID;
    }
    if (qnum == 0) return GTS_OK;
    void *b[5];
    if ((rc = stage_query_data(idx, qrows, qstrs, qlens, qnum, sizeof(int) * (size_t)qnum, 0, b))) return rc;
    const bool str = idx->metric == 6;
    cudaStream_t s = idx->stream;
    rc = gts::search_range_rows(idx, str ? nullptr : (const float *)b[0], str ? (const char *)b[0] : nullptr,
                                str ? (const int *)b[1] : nullptr, qnum, r, (int *)b[2], s);
    if (rc) return rc;
    GTS_CUDA_TRY(cudaMemcpyAsync(counts_out, b[2], sizeof(int) * (size_t)qnum, cudaMemcpyDeviceToHost, s));
    GTS_CUDA_TRY(cudaStreamSynchronize(s));
    return GTS_OK;
}

extern "C" int gts_plain_split(gts_index *idx, int objects, long long *items_handed)
{
    if (!idx) {
        gts_set_error("null index");
        return GTS_ERR_INVALID;
    }
    if (objects >= 0) idx->plain_split = objects;
    if (items_handed) *items_handed = idx->last_split_items;
    return GTS_OK;
}
