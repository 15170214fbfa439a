// build.cu -- parallel pivot-tree construction on the device.
//
// Restates indexConstru (tree.cuh:332-393) level by level:
//   1. k_select_pivots: for every node split at this level the pivot is the
//      object at the middle rank of the node's range, id_list[(lid+rid)/2]
//      (tree.cuh:73), and the node's range becomes one sort segment;
//   2. k_keys: every object of a split node gets the reference's double key
//      dist/INFI_DIS + b*DIS_CODE (tree.cuh:155), distance in the
//      F64-accumulated build arithmetic;
//   3. a stable segmented sort of (key, id) inside each split node.  The
//      reference sorts all N keys globally (tree.cuh:372); node codes keep
//      the segments apart and the sort is stable, so for every tree in which
//      each level's objects all sit in split nodes the order is identical;
//   4. k_split: O children per split node with the equal-count split, the
//      last child taking the remainder, min_dis = dist(first object of the
//      child, pivot) in F32-accumulated arithmetic, is_leaf = size <= MAX_SIZE
//      (tree.cuh:191-295);
//   5. k_node_of_pos: each position learns its child, so the next level can
//      run one thread per object instead of one block per node.
// One 4-byte device->host read per level (the number of nodes still to
// split) decides whether to continue, as the reference's reduce does.
#include <cub/device/device_segmented_sort.cuh>
#include <cstdio>
#include <vector>
#include "index.cuh"

namespace gts {

template <typename T>
int dev_alloc(T **p, size_t n, size_t *acct)
{
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        gts_set_error("cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
        return GTS_ERR_NOMEM;
    }
    if (acct) *acct += n * sizeof(T);
    return GTS_OK;
}
template int dev_alloc<float>(float **, size_t, size_t *);
template int dev_alloc<int>(int **, size_t, size_t *);
template int dev_alloc<char>(char **, size_t, size_t *);
template int dev_alloc<uint8_t>(uint8_t **, size_t, size_t *);
template int dev_alloc<double>(double **, size_t, size_t *);
template int dev_alloc<uint32_t>(uint32_t **, size_t, size_t *);
template int dev_alloc<unsigned short>(unsigned short **, size_t, size_t *);
template int dev_alloc<unsigned long long>(unsigned long long **, size_t, size_t *);
template int dev_alloc<int4>(int4 **, size_t, size_t *);
template int dev_alloc<uint4>(uint4 **, size_t, size_t *);

// Build-time distance between two objects (by id), F64 or F32 site.
__device__ __forceinline__ double obj_dist(const DevData &d, int a, int b, int acc)
{
    if (d.metric == kEdit) {
        return (double)edit_dp(d.strs + (size_t)a * kStrStride, d.lens[a],
                               d.strs + (size_t)b * kStrStride, d.lens[b]);
    }
    const float *x = d.rows + (size_t)a * d.dim;
    const float *y = d.rows + (size_t)b * d.dim;
    return acc == kAccF64 ? dist_row_f64(x, y, d.dim, d.metric)
                          : (double)dist_row_f32(x, y, d.dim, d.metric);
}

__global__ void k_init(int n, int mnn, int *id_list, int *node_of_pos, int *node_pid,
                       int *node_size, int *node_lid, int *node_pivot, float *node_min_dis,
                       uint8_t *node_flags, uint8_t *split)
{
    size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = tid; i < (size_t)n; i += stride) {
        id_list[i] = (int)i;
        node_of_pos[i] = 0;
    }
    for (size_t i = tid; i < (size_t)mnn; i += stride) {
        node_pid[i] = -1;
        node_size[i] = 0;
        node_lid[i] = 0;
        node_pivot[i] = -1;
        node_min_dis[i] = 0.f;
        node_flags[i] = 0;
        split[i] = 0;
    }
    if (tid == 0) {   // initIndexData (tree.cuh:308-317)
        node_size[0] = n;
        node_lid[0] = 0;
        node_pid[0] = -1;
        node_min_dis[0] = 0.f;
        node_flags[0] = kExists;
        split[0] = 1;
    }
}

__global__ void k_select_pivots(int start, int nb, const int *id_list, const int *node_size,
                                const int *node_lid, const uint8_t *split, int *node_pivot,
                                int *seg_begin, int *seg_end)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    int nid = start + b;
    if (split[nid]) {
        int lid = node_lid[nid], size = node_size[nid];
        int rid = lid + size - 1;
        node_pivot[nid] = id_list[(lid + rid) / 2];
        seg_begin[b] = lid;
        seg_end[b] = lid + size;
    } else {
        seg_begin[b] = 0;
        seg_end[b] = 0;
    }
}

__global__ void k_keys(DevData d, int n, int start, int nb, int dis_code, int infi_dis,
                       const int *id_list, const int *node_of_pos, const uint8_t *split,
                       const int *node_pivot, double *key)
{
    size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x; pos < (size_t)n; pos += stride) {
        int nid = node_of_pos[pos];
        int b = nid - start;
        if (b < 0 || b >= nb || !split[nid]) continue;
        double res = obj_dist(d, id_list[pos], node_pivot[nid], kAccF64);
        key[pos] = (double)(res / infi_dis + b * dis_code);
    }
}

__global__ void k_split(DevData d, int start, int nb, int order, int max_size, const int *id_list,
                        const uint8_t *split_in, int *node_pid, int *node_size, int *node_lid,
                        const int *node_pivot, float *node_min_dis, uint8_t *node_flags,
                        uint8_t *split, int *nsplit)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)nb * order) return;
    int b = (int)(t / order), i = (int)(t % order);
    int nid = start + b;
    if (!split_in[nid]) return;
    int lid = node_lid[nid], size = node_size[nid];
    int avg = size / order;
    long c = (long)nid * order + i + 1;
    int clid = lid + avg * i;
    int csize = (i < order - 1) ? avg : size - (order - 1) * avg;
    int piv = node_pivot[nid];
    node_lid[c] = clid;
    node_pid[c] = piv;
    node_size[c] = csize;
    node_min_dis[c] = (float)obj_dist(d, id_list[clid], piv, kAccF32);
    bool leaf = csize <= max_size;
    node_flags[c] = kExists | (leaf ? kLeaf : 0);
    split[c] = leaf ? 0 : 1;
    if (!leaf) atomicAdd(nsplit, 1);
}

__global__ void k_node_of_pos(int n, int start, int nb, int order, const uint8_t *split,
                              const int *node_size, const int *node_lid, int *node_of_pos)
{
    size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x; pos < (size_t)n; pos += stride) {
        int nid = node_of_pos[pos];
        int b = nid - start;
        if (b < 0 || b >= nb || !split[nid]) continue;
        int avg = node_size[nid] / order;
        int off = (int)pos - node_lid[nid];
        int ci = avg > 0 ? min(off / avg, order - 1) : order - 1;
        node_of_pos[pos] = nid * order + 1 + ci;
    }
}

__global__ void k_clear_level(int start, int nb, uint8_t *split)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb) split[start + b] = 0;
}

// Tree-order copies of the data so that a leaf's objects are contiguous.
// Character-class signatures of the strings in tree order (edit lower bounds).
__global__ void k_str_sig(int n, const char *tstrs, const int *tlens, uint4 *tsig)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += (size_t)gridDim.x * blockDim.x)
        tsig[i] = str_sig(tstrs + i * kStrStride, tlens[i]);
}

__global__ void k_permute(int n, int dim, int metric, const int *id_list, const float *rows,
                          float *trows, const char *strs, char *tstrs, const int *lens, int *tlens,
                          int *pos_of_id)
{
    size_t stride = (size_t)gridDim.x * blockDim.x;
    size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (metric == kEdit) {
        for (size_t i = tid; i < (size_t)n * kStrStride; i += stride) {
            size_t pos = i / kStrStride, c = i % kStrStride;
            tstrs[i] = strs[(size_t)id_list[pos] * kStrStride + c];
        }
    } else {
        for (size_t i = tid; i < (size_t)n * dim; i += stride) {
            size_t pos = i / dim, c = i % dim;
            trows[i] = rows[(size_t)id_list[pos] * dim + c];
        }
    }
    for (size_t pos = tid; pos < (size_t)n; pos += stride) {
        int id = id_list[pos];
        pos_of_id[id] = (int)pos;
        if (metric == kEdit) tlens[pos] = lens[id];
    }
}

static inline unsigned grid_for(size_t n, int block, unsigned cap = 148u * 32u)
{
    size_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    return (unsigned)(g > cap ? cap : g);
}

int ensure_scratch(gts_index *idx, size_t bytes)
{
    if (idx->scratch_bytes >= bytes) return GTS_OK;
    if (idx->scratch) cudaFree(idx->scratch);
    idx->scratch = nullptr;
    idx->scratch_bytes = 0;
    if (cudaMalloc(&idx->scratch, bytes) != cudaSuccess) {
        cudaGetLastError();
        idx->scratch = nullptr;
        gts_set_error("cudaMalloc of %zu bytes of search scratch failed", bytes);
        return GTS_ERR_NOMEM;
    }
    idx->scratch_bytes = bytes;
    return GTS_OK;
}

int ensure_io(gts_index *idx, size_t bytes)
{
    if (bytes <= idx->io_bytes) return GTS_OK;
    if (idx->io) cudaFree(idx->io);
    idx->io = nullptr;
    idx->io_bytes = 0;
    size_t want = bytes + bytes / 4 + 4096;
    if (cudaMalloc(&idx->io, want) != cudaSuccess) {
        cudaGetLastError();
        idx->io = nullptr;
        gts_set_error("cudaMalloc of %zu bytes of argument buffers failed", want);
        return GTS_ERR_NOMEM;
    }
    idx->io_bytes = want;
    return GTS_OK;
}

void free_tree(gts_index *idx)
{
    if (idx->fast_recs) cudaFree(idx->fast_recs);
    idx->fast_recs = nullptr;
    idx->fast_nb = 0;
    idx->fast_nsb = 0;
    for (int &c : idx->fast_cfg) c = 0;
    for (int &c : idx->plain_nt) c = 0;
    graph_invalidate(idx);
    idx->mlp_ready = false;   // its feature pivots belong to the old tree
    void *ps[] = {idx->trows, idx->tstrs, idx->tlens, idx->tsig, idx->id_list, idx->pos_of_id, idx->node_pid,
                  idx->node_size, idx->node_lid, idx->node_pivot, idx->node_min_dis,
                  idx->node_flags};
    for (void *p : ps)
        if (p) cudaFree(p);
    idx->trows = nullptr; idx->tstrs = nullptr; idx->tlens = nullptr; idx->tsig = nullptr;
    idx->id_list = nullptr; idx->pos_of_id = nullptr; idx->node_pid = nullptr;
    idx->node_size = nullptr; idx->node_lid = nullptr; idx->node_pivot = nullptr;
    idx->node_min_dis = nullptr; idx->node_flags = nullptr;
}

void free_data(gts_index *idx)
{
    graph_invalidate(idx);   // the captured filter pass reads the rows
    if (idx->rows) cudaFree(idx->rows);
    if (idx->strs) cudaFree(idx->strs);
    if (idx->lens) cudaFree(idx->lens);
    idx->rows = nullptr; idx->strs = nullptr; idx->lens = nullptr;
}

namespace {
// Build-time scratch, released on every exit path.
struct BuildScratch {
    int *node_of_pos = nullptr, *ids_alt = nullptr, *seg_b = nullptr, *seg_e = nullptr, *nsplit = nullptr;
    double *key = nullptr, *key_alt = nullptr;
    uint8_t *split = nullptr;
    void *temp = nullptr;
    ~BuildScratch()
    {
        void *ps[] = {node_of_pos, ids_alt, seg_b, seg_e, nsplit, key, key_alt, split, temp};
        for (void *p : ps)
            if (p) cudaFree(p);
    }
};
}  // namespace

static int build_tree_impl(gts_index *idx, cudaStream_t s)
{
    const gts_params &p = idx->params;
    const int n = idx->num, O = p.tree_order, H = p.max_h;
    double mnn_d = (pow((double)O, (double)H) - 1) / (O - 1);   // tree.cuh:339
    if (mnn_d > 2.0e9) {
        gts_set_error("max_node_num too large (order %d, max_h %d)", O, H);
        return GTS_ERR_INVALID;
    }
    const int mnn = (int)mnn_d;
    idx->max_node_num = mnn;
    int maxnb = 1;   // nodes at the deepest level that can split: O^(H-2)
    for (int l = 0; l + 2 < H; l++) maxnb *= O;

    size_t acct = 0;
    int rc;
#define ALLOC(ptr, cnt) \
    if ((rc = dev_alloc(&(ptr), (cnt), &acct)) != GTS_OK) return rc;
    ALLOC(idx->id_list, n);
    ALLOC(idx->pos_of_id, n);
    ALLOC(idx->node_pid, mnn);
    ALLOC(idx->node_size, mnn);
    ALLOC(idx->node_lid, mnn);
    ALLOC(idx->node_pivot, mnn);
    ALLOC(idx->node_min_dis, mnn);
    ALLOC(idx->node_flags, mnn);
    if (idx->metric == kEdit) {
        ALLOC(idx->tstrs, (size_t)n * kStrStride);
        ALLOC(idx->tlens, n);
        ALLOC(idx->tsig, n);
    } else {
        ALLOC(idx->trows, (size_t)n * idx->dim);
    }
    idx->device_bytes += acct;

    BuildScratch sc;
    ALLOC(sc.node_of_pos, n);
    ALLOC(sc.ids_alt, n);
    ALLOC(sc.key, n);
    ALLOC(sc.key_alt, n);
    ALLOC(sc.split, mnn);
    ALLOC(sc.seg_b, maxnb);
    ALLOC(sc.seg_e, maxnb);
    ALLOC(sc.nsplit, 1);
#undef ALLOC
    size_t temp_bytes = 0;
    GTS_CUDA_TRY(cub::DeviceSegmentedSort::StableSortPairs(nullptr, temp_bytes, sc.key, sc.key_alt,
                                                           idx->id_list, sc.ids_alt, n, maxnb,
                                                           sc.seg_b, sc.seg_e, s));
    if (cudaMalloc(&sc.temp, temp_bytes ? temp_bytes : 1) != cudaSuccess) {
        cudaGetLastError();
        gts_set_error("cudaMalloc of sort scratch (%zu bytes) failed", temp_bytes);
        return GTS_ERR_NOMEM;
    }

    DevData dd{idx->dim, n, idx->metric, idx->rows, idx->strs, idx->lens};
    k_init<<<grid_for(std::max(n, mnn), 256), 256, 0, s>>>(
        n, mnn, idx->id_list, sc.node_of_pos, idx->node_pid, idx->node_size, idx->node_lid,
        idx->node_pivot, idx->node_min_dis, idx->node_flags, sc.split);
    int cur_level = 0, start = 0, split_num = 1;
    while (cur_level < H - 1 && split_num > 0) {   // tree.cuh:360
        int nb = 1;
        for (int l = 0; l < cur_level; l++) nb *= O;
        k_select_pivots<<<(nb + 255) / 256, 256, 0, s>>>(start, nb, idx->id_list, idx->node_size,
                                                         idx->node_lid, sc.split, idx->node_pivot,
                                                         sc.seg_b, sc.seg_e);
        k_keys<<<grid_for(n, 256), 256, 0, s>>>(dd, n, start, nb, p.dis_code, p.infi_dis,
                                                 idx->id_list, sc.node_of_pos, sc.split,
                                                 idx->node_pivot, sc.key);
        GTS_CUDA_TRY(cudaMemcpyAsync(sc.ids_alt, idx->id_list, sizeof(int) * (size_t)n,
                                     cudaMemcpyDeviceToDevice, s));
        size_t tb = temp_bytes;
        GTS_CUDA_TRY(cub::DeviceSegmentedSort::StableSortPairs(sc.temp, tb, sc.key, sc.key_alt,
                                                               idx->id_list, sc.ids_alt, n, nb,
                                                               sc.seg_b, sc.seg_e, s));
        std::swap(idx->id_list, sc.ids_alt);
        GTS_CUDA_TRY(cudaMemsetAsync(sc.nsplit, 0, sizeof(int), s));
        long nthreads = (long)nb * O;
        k_split<<<(unsigned)((nthreads + 255) / 256), 256, 0, s>>>(
            dd, start, nb, O, p.max_size, idx->id_list, sc.split, idx->node_pid, idx->node_size,
            idx->node_lid, idx->node_pivot, idx->node_min_dis, idx->node_flags, sc.split, sc.nsplit);
        k_node_of_pos<<<grid_for(n, 256), 256, 0, s>>>(n, start, nb, O, sc.split, idx->node_size,
                                                        idx->node_lid, sc.node_of_pos);
        k_clear_level<<<(nb + 255) / 256, 256, 0, s>>>(start, nb, sc.split);
        GTS_CUDA_TRY(cudaMemcpyAsync(&split_num, sc.nsplit, sizeof(int), cudaMemcpyDeviceToHost, s));
        GTS_CUDA_TRY(cudaStreamSynchronize(s));
        GTS_CUDA_TRY(cudaGetLastError());
        start += nb;
        cur_level++;
    }
    idx->tree_h = cur_level + 1;   // tree.cuh:386
    size_t work = (size_t)n * (idx->metric == kEdit ? kStrStride : idx->dim);
    k_permute<<<grid_for(work, 256), 256, 0, s>>>(n, idx->dim, idx->metric, idx->id_list, idx->rows,
                                                  idx->trows, idx->strs, idx->tstrs, idx->lens,
                                                  idx->tlens, idx->pos_of_id);
    if (idx->metric == kEdit) k_str_sig<<<grid_for((size_t)n, 256), 256, 0, s>>>(n, idx->tstrs, idx->tlens, idx->tsig);
    GTS_CUDA_TRY(cudaStreamSynchronize(s));
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

int build_tree(gts_index *idx, cudaStream_t s)
{
    int rc = build_tree_impl(idx, s);
    if (rc != GTS_OK) free_tree(idx);
    return rc;
}

}  // namespace gts
