// search.cu -- exact kNN / range traversal of the GTS pivot tree ("plain" form).
//
// Restates the results of searchIndexKnnV2 / searchIndexRnnV2
// (search_v2.cuh:780-1228) and of the update path's range search
// (update.cuh:337-447) with one persistent kernel:
//
//   * work queue: each CTA pulls the next query index from a device counter
//     (atomicAdd) until the batch is exhausted, so queries with very uneven
//     candidate counts balance themselves over the 148 SMs;
//   * traversal: a depth-first walk over the implicit O-ary node numbering
//     (child = nid*O+i+1, search_v2.cuh:53) that pops up to 32 stack entries
//     per step.  For every internal node the query-to-pivot distance gives
//     the ring lower bound of each child, exactly the rule of nodeProcessRnn /
//     nodeProcessKnn (search_v2.cuh:131-141, 181-192):
//         lb = max(min_dis_i - dq, 0, dq - min_dis_{i+1})
//     and a child survives when lb <= radius (range) or <= the current k-th
//     distance (kNN) -- both widened by a rounding slack so the pruning never
//     drops an object the reference arithmetic would report;
//   * leaf verification: one warp per object row (coalesced 512-byte row
//     reads for d = 128) computes an FP32 distance with a rounding bound;
//     objects whose bound can matter are recomputed by one thread in the
//     reference's own operation order (metric.cuh), so every reported value
//     is bit-identical to the reference's leaf value;
//   * kNN merge: exact (distance, id) candidates in shared memory, compacted
//     with a bitonic sort that keeps the k best and tightens the radius.
//
// The query object itself is at distance 0 (search_v2.cuh:338-340,
// 454-456).  Deleted objects (a deletion bitmap) are skipped
// (update.cuh:244).  The stream-update path counts with time stamps instead
// (kModeRangeTimed): an object within r adds the number of its entries that
// are live in the tree, and separately in the cache list, at the query's
// operation index.  Objects of every childless node are verified, at any
// depth, so results equal the exact answer for every tree shape.
#include <algorithm>
#include <cfloat>
#include <cstdio>
#include "index.cuh"

namespace gts {

// threads per query CTA: 128, 256 or 512, picked per search mode by the
// autotuner in run_search (warps per query)
constexpr int kBatch = 32;            // stack entries popped per step (one warp lane each)
constexpr int kRows = 8;              // leaf rows per warp in flight
constexpr int kStackCap = 2048;
constexpr int kLeafObjCap = 1024;     // objects verified per step
constexpr int kMaxK = 256;
constexpr int kCandCap = kLeafObjCap + kMaxK;
constexpr int kSortCap = 2048;        // next power of two >= kCandCap
constexpr int kMaxDimSmem = 1024;
constexpr int kLaneRowDim = 8;        // up to this dimension a lane filters a whole row

enum SearchMode { kModeKnn = 0, kModeRangeCount = 1, kModeRangeIds = 2, kModeRangeTimed = 3 };

struct SearchArgs {
    DevTree t;
    const int *qids;
    int qnum;
    int mode;
    int k;
    float r;
    float *kth;
    int *ids;
    float *dists;
    int *counts;
    const int *offsets;
    int *rids;
    float *rdists;
    const uint32_t *deleted;
    int *counter;
    int *status;
    // kNN seeded by the learned radius (nullable): squared radius per query
    // (float bits); a query with fewer than k objects inside is listed in
    // fail / n_fail instead of answered
    const int *seed_r2_bits;
    int *fail, *n_fail;
    unsigned long long *stats;   // [objects filtered, pivots evaluated, exact values, queries]
    // kModeRangeTimed: the query's operation index; per object id its
    // entries ents[ent_off[id] .. ent_off[id + 1]) as (tree_from, tree_to,
    // cache_from, cache_to), live in the tree at t when tree_from < t <
    // tree_to and in the cache list when cache_from < t < cache_to; counts
    // receives the tree part, counts2 the cache part
    const int *qtime;
    const int *ent_off;
    const int4 *ents;
    int *counts2;
    // queries given as data instead of ids (nullable): rows [qnum][dim], or
    // strings [qnum][109] with lengths; such a query is no object of the
    // index (no self match)
    const float *qrows;
    const char *qstrs;
    const int *qlens;
    // (query, node) work items, range counts only (count and timed modes):
    // items_in (nullable) are (query, node, first unverified object, lower
    // bound bits) handed over by an earlier launch; n_items_in of them are
    // the work units instead of the queries.  A query that has verified more
    // than split_objs objects in one CTA since its last hand-over gives all
    // but its kBatch newest stack entries to items_out (capacity items_cap,
    // count in *n_items_out; entries with query -1 are unused), so the next
    // launch spreads its subtrees over every CTA.  With splitting on, counts
    // are added atomically (the caller zeroes them first).
    const int4 *items_in;
    int4 *items_out;
    int *n_items_out;
    int items_cap;
    int split_objs;   // 0: no hand-over
    float rel_eps;   // relative pruning slack
    float abs_eps;   // absolute pruning slack
};

struct __align__(16) SearchSmem {
    float qrow[kMaxDimSmem];
    uint64_t peq[256];
    char qstr[kStrStride + 3];
    int qlen;
    uint4 qsig;   // the query string's character-class signature
    int stack_node[kStackCap];
    int stack_off[kStackCap];  // first unverified object of a leaf entry
    float stack_lb[kStackCap];
    double cd[kSortCap];
    int cid[kSortCap];
    int bnode[kBatch];
    float bdq_lo[kBatch], bdq_hi[kBatch];
    int bint[kBatch];          // internal nodes of the step
    int bleaf[kBatch];         // leaves of the step
    int bleaf_off[kBatch];     // their first object this step
    int leaf_pre[kBatch + 1];  // prefix of their sizes
    int cpos[kLeafObjCap];     // positions needing an exact value
    int nint, nleaf, ncpos;
    int top, ncand, q, qid, cnt, cnt2, tq, overflow;
    const float *qsrc;         // the query row in global memory
    unsigned long long n_obj, n_piv, n_exact, obj_mark;
    double R;
};

// ---------------------------------------------------------------------------

__device__ __forceinline__ bool is_deleted(const uint32_t *bm, int id)
{
    return bm && ((bm[id >> 5] >> (id & 31)) & 1u);
}

// kModeRangeTimed: adds object id's entries live in the tree / in the cache
// list at operation t to the query's two counts.
__device__ __forceinline__ void add_timed(const SearchArgs &a, SearchSmem &s, int id)
{
    const int t = s.tq;
    int wt = 0, wc = 0;
    for (int e = a.ent_off[id], e1 = a.ent_off[id + 1]; e < e1; e++) {
        const int4 v = a.ents[e];
        wt += (v.x < t && t < v.y) ? 1 : 0;
        wc += (v.z < t && t < v.w) ? 1 : 0;
    }
    if (wt) atomicAdd(&s.cnt, wt);
    if (wc) atomicAdd(&s.cnt2, wc);
}

// Exact leaf value, in the reference's arithmetic for the call site.
__device__ __forceinline__ double exact_obj(const SearchArgs &a, const SearchSmem &s, int pos,
                                            int acc)
{
    const DevTree &t = a.t;
    if (t.metric == kEdit) {
        const char *txt = t.tstrs + (size_t)pos * kStrStride;
        int n = t.tlens[pos];
        if (s.qlen <= 64) return (double)edit_myers64(s.peq, s.qlen, txt, n);
        return (double)edit_dp(txt, n, s.qstr, s.qlen);
    }
    const float *row = t.trows + (size_t)pos * t.dim;
    const float *q = t.dim <= kMaxDimSmem ? s.qrow : s.qsrc;
    return acc == kAccF64 ? dist_row_f64(row, q, t.dim, t.metric)
                          : (double)dist_row_f32(row, q, t.dim, t.metric);
}

// Exact query-to-object value by object id (pivots).
__device__ __forceinline__ double exact_id(const SearchArgs &a, const SearchSmem &s, int id, int acc)
{
    const DevTree &t = a.t;
    if (t.metric == kEdit) {
        const char *txt = t.strs + (size_t)id * kStrStride;
        int n = t.lens[id];
        if (s.qlen <= 64) return (double)edit_myers64(s.peq, s.qlen, txt, n);
        return (double)edit_dp(txt, n, s.qstr, s.qlen);
    }
    const float *row = t.rows + (size_t)id * t.dim;
    const float *q = t.dim <= kMaxDimSmem ? s.qrow : s.qsrc;
    return acc == kAccF64 ? dist_row_f64(row, q, t.dim, t.metric)
                          : (double)dist_row_f32(row, q, t.dim, t.metric);
}

// Warp-cooperative FP32 partial value of a row against the query:
// L2 -> sum of squares, L1 -> sum of |diff|, Linf -> max |diff| (exact).
__device__ __forceinline__ float warp_row_value(const float *__restrict__ row,
                                                const float *__restrict__ q, int dim, int metric,
                                                int lane)
{
    float acc = 0.f;
    if ((dim & 3) == 0) {
        const float4 *r4 = reinterpret_cast<const float4 *>(row);
        const float4 *q4 = reinterpret_cast<const float4 *>(q);
        for (int j = lane; j < (dim >> 2); j += 32) {
            float4 x = __ldg(r4 + j), y = q4[j];
            float d0 = x.x - y.x, d1 = x.y - y.y, d2 = x.z - y.z, d3 = x.w - y.w;
            if (metric == kL2) {
                acc = fmaf(d0, d0, acc); acc = fmaf(d1, d1, acc);
                acc = fmaf(d2, d2, acc); acc = fmaf(d3, d3, acc);
            } else if (metric == kL1) {
                acc += fabsf(d0) + fabsf(d1) + fabsf(d2) + fabsf(d3);
            } else {
                acc = fmaxf(acc, fmaxf(fmaxf(fabsf(d0), fabsf(d1)), fmaxf(fabsf(d2), fabsf(d3))));
            }
        }
    } else {
        for (int j = lane; j < dim; j += 32) {
            float d0 = __ldg(row + j) - q[j];
            if (metric == kL2) acc = fmaf(d0, d0, acc);
            else if (metric == kL1) acc += fabsf(d0);
            else acc = fmaxf(acc, fabsf(d0));
        }
    }
    return metric == kLinf ? warp_max(acc) : warp_sum(acc);
}

// R rows at once (independent loads in flight): out[u] as warp_row_value.
template <int R>
__device__ __forceinline__ void warp_row_values(const float *const (&rows)[R], const float *__restrict__ q,
                                                int dim, int metric, int lane, float (&out)[R])
{
    float acc[R];
#pragma unroll
    for (int u = 0; u < R; u++) acc[u] = 0.f;
    if ((dim & 3) == 0) {
        const float4 *q4 = reinterpret_cast<const float4 *>(q);
        for (int j = lane; j < (dim >> 2); j += 32) {
            float4 x[R];
#pragma unroll
            for (int u = 0; u < R; u++) x[u] = __ldg(reinterpret_cast<const float4 *>(rows[u]) + j);
            const float4 y = q4[j];
#pragma unroll
            for (int u = 0; u < R; u++) {
                float d0 = x[u].x - y.x, d1 = x[u].y - y.y, d2 = x[u].z - y.z, d3 = x[u].w - y.w;
                if (metric == kL2) {
                    acc[u] = fmaf(d0, d0, acc[u]); acc[u] = fmaf(d1, d1, acc[u]);
                    acc[u] = fmaf(d2, d2, acc[u]); acc[u] = fmaf(d3, d3, acc[u]);
                } else if (metric == kL1) {
                    acc[u] += fabsf(d0) + fabsf(d1) + fabsf(d2) + fabsf(d3);
                } else {
                    acc[u] = fmaxf(acc[u], fmaxf(fmaxf(fabsf(d0), fabsf(d1)), fmaxf(fabsf(d2), fabsf(d3))));
                }
            }
        }
    } else {
        for (int j = lane; j < dim; j += 32) {
            float x[R];
#pragma unroll
            for (int u = 0; u < R; u++) x[u] = __ldg(rows[u] + j);
            const float y = q[j];
#pragma unroll
            for (int u = 0; u < R; u++) {
                float d0 = x[u] - y;
                if (metric == kL2) acc[u] = fmaf(d0, d0, acc[u]);
                else if (metric == kL1) acc[u] += fabsf(d0);
                else acc[u] = fmaxf(acc[u], fabsf(d0));
            }
        }
    }
#pragma unroll
    for (int u = 0; u < R; u++) out[u] = metric == kLinf ? warp_max(acc[u]) : warp_sum(acc[u]);
}

// Interval [lo, hi] that contains both exact leaf values (F32 and F64
// sites) given the FP32 warp value v.
__device__ __forceinline__ void value_bounds(int metric, int dim, float v, double &lo, double &hi)
{
    if (metric == kLinf) {   // max of exactly rounded |diff|: exact
        lo = hi = (double)v;
        return;
    }
    double g = 2.0 * (double)f32_sum_rel_bound(dim + 32) + 4.0 * 5.9604645e-8;
    double vl = (double)v * (1.0 - g), vh = (double)v * (1.0 + g);
    if (metric == kL2) {
        lo = sqrt(vl > 0 ? vl : 0.0) * (1.0 - 1e-7);
        hi = sqrt(vh) * (1.0 + 1e-7);
    } else {
        lo = vl;
        hi = vh;
    }
}

// Index of the leaf holding step object o: the last li < nleaf with
// leaf_pre[li] <= o (leaf_pre ascending, at most kBatch + 1 entries).
__device__ __forceinline__ int leaf_of(const int *leaf_pre, int nleaf, int o)
{
    int lo = 0, hi = nleaf - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (leaf_pre[mid] <= o) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// value_bounds in FP32: the products and square roots add at most a few
// ulps, covered by the extra 4e-7 / 2e-7 relative margins.
__device__ __forceinline__ void value_bounds_f(int metric, int dim, float v, float &lo, float &hi)
{
    if (metric == kLinf) {   // max of exactly rounded |diff|: exact
        lo = hi = v;
        return;
    }
    const float g = 2.f * f32_sum_rel_bound(dim + 32) + 4.f * 5.9604645e-8f;
    const float vl = v * (1.f - g), vh = v * (1.f + g);
    if (metric == kL2) {
        lo = sqrtf(fmaxf(vl, 0.f)) * (1.f - 4e-7f);
        hi = sqrtf(vh) * (1.f + 4e-7f);
    } else {
        lo = vl * (1.f - 2e-7f);
        hi = vh * (1.f + 2e-7f);
    }
}

// Bitonic sort of the candidate buffer by (distance, id), n entries padded
// to the next power of two; keeps the first min(n, k).
template <int NT>
__device__ void compact_candidates(SearchSmem &s, int k)
{
    int n = s.ncand;
    int p2 = 1;
    while (p2 < n) p2 <<= 1;
    for (int i = n + threadIdx.x; i < p2; i += NT) {
        s.cd[i] = DBL_MAX;
        s.cid[i] = 0x7fffffff;
    }
    __syncthreads();
    for (int size = 2; size <= p2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < p2 / 2; i += NT) {
                int lo = 2 * i - (i & (stride - 1));
                int hi = lo + stride;
                bool up = ((lo & size) == 0);
                double dl = s.cd[lo], dh = s.cd[hi];
                int il = s.cid[lo], ih = s.cid[hi];
                bool gt = (dl > dh) || (dl == dh && il > ih);
                if (gt == up) {
                    s.cd[lo] = dh; s.cd[hi] = dl;
                    s.cid[lo] = ih; s.cid[hi] = il;
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        s.ncand = n < k ? n : k;
        if (n >= k) s.R = s.cd[k - 1];
    }
    __syncthreads();
}

template <int NT>
__global__ void __launch_bounds__(NT, 1) k_search(SearchArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SearchSmem &s = *reinterpret_cast<SearchSmem *>(smem_raw);
    const DevTree &t = a.t;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int O = t.order;
    const bool knn = a.mode == kModeKnn;
    const bool timed = a.mode == kModeRangeTimed;
    const bool count_only = a.mode == kModeRangeCount || timed;
    const int acc = knn ? kAccF64 : kAccF32;
    const bool warp_filter = (t.metric == kL2 || t.metric == kL1 || t.metric == kLinf);

    for (;;) {
        if (tid == 0) s.q = atomicAdd(a.counter, 1);
        __syncthreads();
        const int w = s.q;   // work unit: a query, or a handed-over (query, node) item
        if (w >= a.qnum) break;
        const int4 item = a.items_in ? a.items_in[w] : make_int4(w, 0, 0, 0);
        const int q = item.x;
        if (q < 0) {   // an unused item slot
            __syncthreads();
            continue;
        }
        const bool by_data = a.qrows || a.qstrs;
        const int qid = by_data ? -1 : a.qids[q];
        if (!by_data && (qid < 0 || qid >= t.num)) {   // device-API ids are checked here
            if (tid == 0) {
                atomicMax(a.status, (int)kKsBadQuery);
                if (a.mode == kModeKnn) a.kth[q] = __int_as_float(0x7fc00000);
                else if (count_only) a.counts[q] = -1;
                if (timed) a.counts2[q] = -1;
            }
            __syncthreads();
            continue;
        }
        // ---- per-query set-up
        if (tid == 0) {
            s.qid = qid;
            s.top = 1;
            s.stack_node[0] = item.y;
            s.stack_off[0] = item.z;
            s.stack_lb[0] = __int_as_float(item.w);
            s.ncand = 0;
            s.cnt = 0;
            s.cnt2 = 0;
            s.tq = timed ? a.qtime[q] : 0;
            s.overflow = 0;
            s.n_obj = s.n_piv = s.n_exact = s.obj_mark = 0;
            s.R = !knn ? (double)a.r
                       : (a.seed_r2_bits ? sqrt((double)__int_as_float(a.seed_r2_bits[q])) : DBL_MAX);
        }
        if (t.metric == kEdit) {
            int m = min(max(by_data ? a.qlens[q] : t.lens[qid], 0), kStrStride - 1);
            const char *src = by_data ? a.qstrs + (size_t)q * kStrStride : t.strs + (size_t)qid * kStrStride;
            for (int i = tid; i < kStrStride; i += NT) s.qstr[i] = src[i];
            for (int c = tid; c < 256; c += NT) {
                uint64_t bits = 0;
                for (int i = 0; i < m && i < 64; i++)
                    if ((unsigned char)src[i] == (unsigned)c) bits |= 1ull << i;
                s.peq[c] = bits;
            }
            if (tid == 0) s.qlen = m;
        } else {
            const float *src = by_data ? a.qrows + (size_t)q * t.dim : t.rows + (size_t)qid * t.dim;
            if (tid == 0) s.qsrc = src;
            if (t.dim <= kMaxDimSmem)
                for (int i = tid; i < t.dim; i += NT) s.qrow[i] = src[i];
        }
        __syncthreads();
        if (t.metric == kEdit) {
            if (tid == 0) s.qsig = str_sig(s.qstr, s.qlen);
            __syncthreads();
        }
        const float *qrow = t.dim <= kMaxDimSmem ? s.qrow : s.qsrc;

        // ---- traversal
        for (;;) {
            if (warp == 0 && a.split_objs > 0 && s.top > kBatch && s.n_obj - s.obj_mark > (unsigned long long)a.split_objs) {
                // hand the older stack entries over as (query, node) items
                const int top = s.top, nd = top - kBatch;
                int base = 0;
                if (lane == 0) base = atomicAdd(a.n_items_out, nd);
                base = __shfl_sync(0xffffffffu, base, 0);
                if (base + nd <= a.items_cap) {
                    for (int i = lane; i < nd; i += 32)
                        a.items_out[base + i] = make_int4(q, s.stack_node[i], s.stack_off[i], __float_as_int(s.stack_lb[i]));
                    // the kBatch newest entries move to the bottom (one per lane)
                    const int kn = s.stack_node[nd + lane], ko = s.stack_off[nd + lane];
                    const float kl = s.stack_lb[nd + lane];
                    __syncwarp();
                    s.stack_node[lane] = kn;
                    s.stack_off[lane] = ko;
                    s.stack_lb[lane] = kl;
                    if (lane == 0) s.top = kBatch;
                } else {
                    // no room: keep them; mark this reservation's slots below the capacity unused
                    for (int i = base + lane; i < a.items_cap && i < base + nd; i += 32)
                        a.items_out[i] = make_int4(-1, 0, 0, 0);
                }
                if (lane == 0) s.obj_mark = s.n_obj;
                __syncwarp();
            }
            if (warp == 0) {
                // pop, in parallel, the top kBatch (= 32) entries: lane i looks
                // at entry top-1-i.  Entries whose bound no longer admits
                // results are dropped; internal nodes are taken; leaves are
                // taken in stack order while their objects fit in
                // kLeafObjCap (the first leaf that does not fit is taken in
                // part and stays on the stack with its offset advanced, and
                // nothing below it is popped this step).
                const double R = s.R;
                const int top = s.top;
                const int n = top < kBatch ? top : kBatch;
                const int e = top - 1 - lane;
                const bool valid = lane < n;
                int node = 0, off = 0, piv = -1, sz = 0;
                bool alive = false;
                if (valid) {
                    node = s.stack_node[e];
                    off = s.stack_off[e];
                    const float lb = s.stack_lb[e];
                    const double slack = a.abs_eps + a.rel_eps * ((double)lb + (R < 1e300 ? R : 0.0));
                    alive = !((double)lb > R + slack);
                }
                if (alive) {
                    piv = t.node_pivot[node];
                    if (piv < 0) sz = t.node_size[node] - off;
                }
                const bool leaf = alive && piv < 0;
                int incl = sz;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                const int excl = incl - sz;
                const unsigned over = __ballot_sync(0xffffffffu, leaf && incl > kLeafObjCap);
                const int stop = over ? __ffs(over) - 1 : n;   // first leaf that does not fit
                const bool take_int = alive && !leaf && lane < stop;
                const bool take_leaf = leaf && (lane < stop || (lane == stop && excl < kLeafObjCap));
                const unsigned mi = __ballot_sync(0xffffffffu, take_int);
                const unsigned ml = __ballot_sync(0xffffffffu, take_leaf);
                const unsigned below = (1u << lane) - 1u;
                if (take_int) s.bint[__popc(mi & below)] = node;
                if (take_leaf) {
                    const int li = __popc(ml & below);
                    s.bleaf[li] = node;
                    s.bleaf_off[li] = off;
                    s.leaf_pre[li] = excl;
                    if (lane == stop) s.stack_off[e] = off + (kLeafObjCap - excl);   // the rest stays
                }
                const int nint = __popc(mi), nleaf = __popc(ml);
                int nobj = 0;
                if (nleaf > 0) {
                    const int last = 31 - __clz(ml);   // the last taken leaf lane
                    const int lincl = __shfl_sync(0xffffffffu, incl, last);
                    nobj = lincl < kLeafObjCap ? lincl : kLeafObjCap;
                }
                if (lane == 0) {
                    s.top = top - stop;
                    s.leaf_pre[nleaf] = nobj;
                    s.nint = nint;
                    s.nleaf = nleaf;
                    s.ncpos = 0;
                    s.n_obj += nobj;
                    s.n_piv += nint;
                }
            }
            __syncthreads();
            const int nint = s.nint, nleaf = s.nleaf;
            if (nint == 0 && nleaf == 0) break;
            const int nobj = s.leaf_pre[nleaf];

            // ---- leaves: filter every object, collect those needing exact values
            if (nleaf > 0) {
                if (warp_filter && t.dim <= kLaneRowDim) {
                    // few dimensions: one lane per row, 32 rows per warp step
                    // (the value bounds hold for any summation order)
                    const int nl = s.nleaf;
                    for (int o = warp * 32 + lane; o - lane < nobj; o += NT) {
                        if (o >= nobj) continue;
                        const int li = leaf_of(s.leaf_pre, nl, o);
                        const int pos = t.node_lid[s.bleaf[li]] + s.bleaf_off[li] + (o - s.leaf_pre[li]);
                        const int id = t.id_list[pos];
                        if (is_deleted(a.deleted, id)) continue;
                        const float *row = t.trows + (size_t)pos * t.dim;
                        float v = 0.f;
                        for (int j = 0; j < t.dim; j++) {
                            const float d0 = __ldg(row + j) - qrow[j];
                            if (t.metric == kL2) v = fmaf(d0, d0, v);
                            else if (t.metric == kL1) v += fabsf(d0);
                            else v = fmaxf(v, fabsf(d0));
                        }
                        float lo, hi;
                        value_bounds_f(t.metric, t.dim, v, lo, hi);
                        if (id == qid) lo = hi = 0.f;
                        if (knn) {
                            if ((double)lo <= s.R) s.cpos[atomicAdd(&s.ncpos, 1)] = pos;
                        } else if (count_only && (double)hi < (double)a.r * (1.0 - 2.4e-7)) {
                            if (timed) add_timed(a, s, id);
                            else atomicAdd(&s.cnt, 1);
                        } else if ((double)lo <= (double)a.r * (1.0 + 2.4e-7)) {
                            s.cpos[atomicAdd(&s.ncpos, 1)] = pos;
                        }
                    }
                } else if (warp_filter) {
                    // kRows rows per warp step: their loads are in flight
                    // together.  Lane u < kRows finds row u's leaf (binary
                    // search of the step's leaf prefix) and, after the
                    // warp-split distances, tests row u; rows run in parallel.
                    const int nl = s.nleaf;
                    for (int o0 = warp * kRows; o0 < nobj; o0 += (NT / 32) * kRows) {
                        int my_pos = 0, my_id = -1;
                        if (lane < kRows) {
                            const int o = min(o0 + lane, nobj - 1);
                            const int li = leaf_of(s.leaf_pre, nl, o);
                            my_pos = t.node_lid[s.bleaf[li]] + s.bleaf_off[li] + (o - s.leaf_pre[li]);
                            my_id = t.id_list[my_pos];
                        }
                        const float *rp[kRows];
#pragma unroll
                        for (int u = 0; u < kRows; u++)
                            rp[u] = t.trows + (size_t)__shfl_sync(0xffffffffu, my_pos, u) * t.dim;
                        float v4[kRows];
                        warp_row_values<kRows>(rp, qrow, t.dim, t.metric, lane, v4);
                        float v = 0.f;
#pragma unroll
                        for (int u = 0; u < kRows; u++)
                            if (lane == u) v = v4[u];
                        if (lane < kRows && o0 + lane < nobj && !is_deleted(a.deleted, my_id)) {
                            float lo, hi;
                            value_bounds_f(t.metric, t.dim, v, lo, hi);
                            if (my_id == qid) lo = hi = 0.f;
                            if (knn) {
                                if ((double)lo <= s.R) s.cpos[atomicAdd(&s.ncpos, 1)] = my_pos;
                            } else if (count_only && (double)hi < (double)a.r * (1.0 - 2.4e-7)) {
                                if (timed) add_timed(a, s, my_id);
                                else atomicAdd(&s.cnt, 1);
                            } else if ((double)lo <= (double)a.r * (1.0 + 2.4e-7)) {
                                s.cpos[atomicAdd(&s.ncpos, 1)] = my_pos;
                            }
                        }
                    }
                } else {
                    // edit distance: objects whose length difference or
                    // character-class bound already exceeds the bound are
                    // out without their edit distance (metric.cuh)
                    const bool sig = t.metric == kEdit && t.tsig;
                    const double bnd = knn ? s.R : (double)a.r;
                    for (int o = tid; o < nobj; o += NT) {
                        const int li = leaf_of(s.leaf_pre, s.nleaf, o);
                        int pos = t.node_lid[s.bleaf[li]] + s.bleaf_off[li] + (o - s.leaf_pre[li]);
                        if (is_deleted(a.deleted, t.id_list[pos])) continue;
                        if (sig && (double)edit_lower_bound(t.tsig[pos], t.tlens[pos], s.qsig, s.qlen) > bnd) continue;
                        int c = atomicAdd(&s.ncpos, 1);
                        s.cpos[c] = pos;
                    }
                }
                __syncthreads();
                // exact values for the collected positions
                const int ncpos = s.ncpos;
                if (tid == 0) s.n_exact += ncpos;
                if (knn && s.ncand + ncpos > kCandCap) compact_candidates<NT>(s, a.k);
                for (int c = tid; c < ncpos; c += NT) {
                    int pos = s.cpos[c];
                    int id = t.id_list[pos];
                    double d = (id == qid) ? 0.0 : exact_obj(a, s, pos, acc);
                    if (knn) {
                        if (d <= s.R) {
                            int slot = atomicAdd(&s.ncand, 1);
                            s.cd[slot] = d;
                            s.cid[slot] = id;
                        }
                    } else if ((float)d <= a.r && timed) {
                        add_timed(a, s, id);
                    } else if ((float)d <= a.r) {
                        int slot = atomicAdd(&s.cnt, 1);
                        if (a.mode == kModeRangeIds) {
                            a.rids[a.offsets[q] + slot] = id;
                            a.rdists[a.offsets[q] + slot] = (float)d;
                        }
                    }
                }
                __syncthreads();
                if (knn && s.ncand > kCandCap - kLeafObjCap) compact_candidates<NT>(s, a.k);
            }

            // ---- internal nodes: pivot distance bounds, then ring pruning of children
            if (nint > 0) {
                if (warp_filter && t.dim <= kLaneRowDim) {
                    // few dimensions: one thread per pivot
                    for (int b = tid; b < nint; b += NT) {
                        const int piv = t.node_pivot[s.bint[b]];
                        const float *row = t.rows + (size_t)piv * t.dim;
                        float v = 0.f;
                        for (int j = 0; j < t.dim; j++) {
                            const float d0 = __ldg(row + j) - qrow[j];
                            if (t.metric == kL2) v = fmaf(d0, d0, v);
                            else if (t.metric == kL1) v += fabsf(d0);
                            else v = fmaxf(v, fabsf(d0));
                        }
                        double lo, hi;
                        value_bounds(t.metric, t.dim, v, lo, hi);
                        if (piv == qid) lo = hi = 0.0;
                        s.bdq_lo[b] = (float)lo;
                        s.bdq_hi[b] = (float)hi;
                    }
                } else if (warp_filter) {
                    for (int b = warp; b < nint; b += (NT / 32)) {
                        int piv = t.node_pivot[s.bint[b]];
                        float v = warp_row_value(t.rows + (size_t)piv * t.dim, qrow, t.dim, t.metric, lane);
                        if (lane == 0) {
                            double lo, hi;
                            value_bounds(t.metric, t.dim, v, lo, hi);
                            if (piv == qid) lo = hi = 0.0;
                            s.bdq_lo[b] = (float)lo;
                            s.bdq_hi[b] = (float)hi;
                        }
                    }
                } else {
                    for (int b = tid; b < nint; b += NT) {
                        int piv = t.node_pivot[s.bint[b]];
                        double d = (piv == qid) ? 0.0 : exact_id(a, s, piv, kAccF64);
                        s.bdq_lo[b] = (float)d;
                        s.bdq_hi[b] = (float)d;
                    }
                }
                __syncthreads();
                const double R = s.R;
                for (int w = tid; w < nint * O; w += NT) {
                    int b = w / O, i = w % O;
                    int node = s.bint[b];
                    long c = (long)node * O + i + 1;
                    if (c >= t.max_node_num) continue;
                    uint8_t fl = t.node_flags[c];
                    if (!(fl & kExists) || t.node_size[c] == 0) continue;
                    float dlo = s.bdq_lo[b], dhi = s.bdq_hi[b];
                    float md = t.node_min_dis[c];
                    float lb = fmaxf(md - dhi, 0.f);
                    if (c % O != 0) lb = fmaxf(lb, dlo - t.node_min_dis[c + 1]);
                    double slack = a.abs_eps + a.rel_eps * ((double)dhi + fabs((double)md) + (R < 1e300 ? R : 0.0));
                    if ((double)lb > R + slack) continue;
                    int slot = atomicAdd(&s.top, 1);
                    if (slot < kStackCap) {
                        s.stack_node[slot] = (int)c;
                        s.stack_off[slot] = 0;
                        s.stack_lb[slot] = lb;
                    } else {
                        s.overflow = 1;
                    }
                }
                __syncthreads();
                if (tid == 0 && s.top > kStackCap) s.top = kStackCap;
                __syncthreads();
            }
        }

        // ---- outputs
        if (knn) {
            compact_candidates<NT>(s, a.k);
            int k = a.k;
            if (a.seed_r2_bits && s.ncand < k) {   // the learned radius held fewer than k objects
                if (tid == 0) a.fail[atomicAdd(a.n_fail, 1)] = q;
                k = 0;
            }
            for (int j = tid; j < k; j += NT) {
                bool have = j < s.ncand;
                if (a.ids) a.ids[(size_t)q * k + j] = have ? s.cid[j] : -1;
                if (a.dists) a.dists[(size_t)q * k + j] = have ? (float)s.cd[j] : (float)t.infi_dis;
            }
            if (tid == 0 && k > 0) a.kth[q] = s.ncand >= k ? (float)s.cd[k - 1] : (float)t.infi_dis;
        } else if (tid == 0) {
            const bool add = a.split_objs > 0 || a.items_in;
            if (count_only) {
                if (add) atomicAdd(&a.counts[q], s.cnt);
                else a.counts[q] = s.cnt;
            }
            if (timed) {
                if (add) atomicAdd(&a.counts2[q], s.cnt2);
                else a.counts2[q] = s.cnt2;
            }
        }
        if (tid == 0) {
            if (s.overflow) atomicMax(a.status, (int)kKsStackOverflow);
            if (a.stats) {
                atomicAdd(&a.stats[0], s.n_obj);
                atomicAdd(&a.stats[1], s.n_piv);
                atomicAdd(&a.stats[2], s.n_exact);
                if (!a.items_in) atomicAdd(&a.stats[3], 1ull);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------

constexpr int kPlainDefaultThreads = 256;

// Persistent CTAs of k_search<NT> that fit on the device at once.
template <int NT>
static int search_resident()
{
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_search<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SearchSmem));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_search<NT>, NT, sizeof(SearchSmem));
    return nsm * (per_sm < 1 ? 1 : per_sm);
}

template <int NT>
static int launch_search_nt(gts_index *idx, const SearchArgs &a, cudaStream_t st)
{
    const size_t smem = sizeof(SearchSmem);
    GTS_CUDA_TRY(cudaFuncSetAttribute(k_search<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int grid = search_resident<NT>();
    if (grid > a.qnum) grid = a.qnum;
    k_search<NT><<<grid, NT, smem, st>>>(a);
    idx->kernel_launches++;
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

static int launch_search(gts_index *idx, const SearchArgs &a, int nt, cudaStream_t st)
{
    switch (nt) {
    case 128: return launch_search_nt<128>(idx, a, st);
    case 512: return launch_search_nt<512>(idx, a, st);
    default: return launch_search_nt<256>(idx, a, st);
    }
}

// Times 128 / 256 / 512 threads per query CTA on the batch's leading queries
// (results identical; the full batch then runs with the fastest).  The
// sample is four times the most CTAs any candidate keeps resident, so the
// timing is throughput rather than the latency of a few queries; batches
// below twice the sample are not tuned (*best_nt = 0: the default runs).
// Each candidate is warmed on one query first.  Range-id mode is not tuned
// (its output offsets belong to the whole batch): it takes the range-count
// choice.  A seeded kNN batch is timed unseeded (the seeds' failure list
// belongs to the real run).
static int plain_autotune(gts_index *idx, const SearchArgs &a, cudaStream_t st, int *best_nt)
{
    *best_nt = 0;
    if (a.mode == kModeRangeIds) {
        *best_nt = idx->plain_nt[kModeRangeCount];
        return GTS_OK;
    }
    const int sample = 4 * std::max(search_resident<128>(), std::max(search_resident<256>(), search_resident<512>()));
    if (a.qnum < 2 * sample) return GTS_OK;
    SearchArgs t = a;
    t.seed_r2_bits = nullptr;
    t.split_objs = 0;
    t.items_in = nullptr;
    cudaEvent_t e0, e1;
    GTS_CUDA_TRY(cudaEventCreate(&e0));
    GTS_CUDA_TRY(cudaEventCreate(&e1));
    float best = 3.0e38f;
    int rc = GTS_OK;
    const int cand[3] = {128, 256, 512};
    for (int rep = 0; rep < 2 && rc == GTS_OK; rep++)   // rep 0: one query per candidate (module load, caches)
        for (int c : cand) {
            t.qnum = rep == 0 ? 1 : sample;
            cudaMemsetAsync(idx->d_counter, 0, sizeof(int), st);
            cudaEventRecord(e0, st);
            if ((rc = launch_search(idx, t, c, st))) break;
            cudaEventRecord(e1, st);
            float ms = 0.f;
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                gts_set_error("plain autotune: CUDA event failed");
                rc = GTS_ERR_CUDA;
                break;
            }
            if (rep == 1 && ms < best) {
                best = ms;
                *best_nt = c;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaMemsetAsync(idx->d_counter, 0, sizeof(int), st);
    cudaMemsetAsync(idx->d_stats, 0, kStatsN * sizeof(unsigned long long), st);
    return rc;
}

extern "C" int gts_plain_threads(const gts_index *idx, int mode, int *threads)
{
    if (!idx || mode < 0 || mode > 2 || !threads) {
        gts_set_error("gts_plain_threads: null index / output or mode outside 0..2");
        return GTS_ERR_INVALID;
    }
    *threads = idx->plain_nt[mode];
    return GTS_OK;
}

extern "C" int gts_plain_threads_set(gts_index *idx, int mode, int threads)
{
    if (!idx || mode < 0 || mode > 2 || (threads != 0 && threads != 128 && threads != 256 && threads != 512)) {
        gts_set_error("gts_plain_threads_set: null index, mode outside 0..2 or threads not 0/128/256/512");
        return GTS_ERR_INVALID;
    }
    idx->plain_nt[mode] = threads;
    return GTS_OK;
}

// Range counts with (query, node) hand-over: the queries run, then the items
// heavy queries handed over run as their own launch, spread over every CTA,
// until none are handed over (at most kSplitPhases launches; the last one
// hands nothing over).  Counts are added atomically from zero.  The two item
// lists live in the handle's own buffer (not the search scratch, which a
// caller such as the fast form's overflow path may hold).
constexpr int kSplitPhases = 8;

static int run_split_phases(gts_index *idx, const SearchArgs &a0, int nt, cudaStream_t st)
{
    const size_t budget = search_budget(idx);
    const int cap = (int)std::max<size_t>(1024, std::min<size_t>((size_t)1 << 20, budget / 64));
    const size_t list_bytes = ((sizeof(int4) * (size_t)cap) + 255) & ~(size_t)255;
    const size_t need = 2 * list_bytes + 256;
    if (idx->split_bytes < need) {
        if (idx->split_buf) cudaFree(idx->split_buf);
        idx->split_buf = nullptr;
        idx->split_bytes = 0;
        if (cudaMalloc(&idx->split_buf, need) != cudaSuccess) {
            cudaGetLastError();
            gts_set_error("cudaMalloc of %zu bytes for the work-item lists failed", need);
            return GTS_ERR_NOMEM;
        }
        idx->split_bytes = need;
    }
    unsigned char *B = (unsigned char *)idx->split_buf;
    int4 *lists[2] = {(int4 *)B, (int4 *)(B + list_bytes)};
    int *nout = (int *)(B + 2 * list_bytes);
    GTS_CUDA_TRY(cudaMemsetAsync(a0.counts, 0, sizeof(int) * (size_t)a0.qnum, st));
    if (a0.counts2) GTS_CUDA_TRY(cudaMemsetAsync(a0.counts2, 0, sizeof(int) * (size_t)a0.qnum, st));
    SearchArgs a = a0;
    a.split_objs = idx->plain_split;
    a.items_cap = cap;
    int cur = 0, n = a0.qnum, rc;
    for (int phase = 0; phase < kSplitPhases && n > 0; phase++) {
        a.items_in = phase == 0 ? nullptr : lists[cur];
        a.qnum = n;
        a.items_out = lists[cur ^ 1];
        a.n_items_out = nout + (cur ^ 1);
        if (phase == kSplitPhases - 1) a.split_objs = 0;
        GTS_CUDA_TRY(cudaMemsetAsync(a.n_items_out, 0, sizeof(int), st));
        GTS_CUDA_TRY(cudaMemsetAsync(idx->d_counter, 0, sizeof(int), st));
        if ((rc = launch_search(idx, a, nt, st))) return rc;
        int handed = 0;
        GTS_CUDA_TRY(cudaMemcpyAsync(&handed, a.n_items_out, sizeof(int), cudaMemcpyDeviceToHost, st));
        GTS_CUDA_TRY(cudaStreamSynchronize(st));
        n = std::min(handed, cap);
        idx->last_split_items += n;
        cur ^= 1;
    }
    return GTS_OK;
}

static int run_search(gts_index *idx, SearchArgs &a, cudaStream_t st)
{
    if (a.qnum <= 0) return GTS_OK;
    a.t = idx->dev();
    a.counter = idx->d_counter;
    a.stats = idx->d_stats;
    a.status = idx->d_status;
    if (idx->metric == kAngle) {
        a.rel_eps = 1e-5f;
        a.abs_eps = 0.05f;
    } else if (idx->metric == kEdit) {
        a.rel_eps = 0.f;
        a.abs_eps = 0.f;
    } else {
        a.rel_eps = 4e-6f;
        // build keys are quantised at dist/INFI_DIS + b*DIS_CODE
        double kmax = 1.0;
        for (int l = 0; l + 2 < idx->tree_h; l++) kmax *= idx->params.tree_order;
        double quantum = 4.0 * 2.220446e-16 * (kmax * idx->params.dis_code + 2.0) * idx->params.infi_dis;
        a.abs_eps = (float)(quantum + 1e-6);
    }
    GTS_CUDA_TRY(cudaMemsetAsync(idx->d_counter, 0, sizeof(int), st));
    GTS_CUDA_TRY(cudaMemsetAsync(idx->d_status, 0, sizeof(int), st));
    if (!idx->keep_stats) GTS_CUDA_TRY(cudaMemsetAsync(idx->d_stats, 0, kStatsN * sizeof(unsigned long long), st));
    // threads per query CTA: tuned per search mode on the first batch large
    // enough for plain_autotune's sample, else the tuned or default value
    const int slot = a.mode == kModeRangeTimed ? kModeRangeCount : a.mode;
    int nt = idx->plain_nt[slot];
    if (!nt && !idx->keep_stats) {
        int rc = plain_autotune(idx, a, st, &nt);
        if (rc) return rc;
        if (a.mode != kModeRangeIds) idx->plain_nt[slot] = nt;
    }
    if (!nt) nt = kPlainDefaultThreads;
    const bool split = (a.mode == kModeRangeCount || a.mode == kModeRangeTimed) && idx->plain_split > 0;
    int rc = split ? run_split_phases(idx, a, nt, st) : launch_search(idx, a, nt, st);
    if (rc) return rc;
    int status = 0;
    GTS_CUDA_TRY(cudaMemcpyAsync(&status, idx->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    if (status != 0) {
        gts_set_error("search kernel reported status %d (%s)", status,
                      status == kKsBadQuery ? "query id out of range" : "traversal stack overflow");
        return GTS_ERR_KERNEL;
    }
    return GTS_OK;
}

__global__ void k_gather_q(const int *src, const int *idx, int n, int *dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}

__global__ void k_scatter_q(const int *idx, int n, int k, const float *kth_s, const int *ids_s, const float *dis_s,
                            float *kth, int *ids, float *dists)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q = idx[i];
    kth[q] = kth_s[i];
    for (int j = 0; j < k; j++) {
        if (ids) ids[(size_t)q * k + j] = ids_s[(size_t)i * k + j];
        if (dists) dists[(size_t)q * k + j] = dis_s[(size_t)i * k + j];
    }
}

// Scratch of one seeded chunk of qn queries (offsets in the handle's region).
struct LearnedPlan {
    size_t seed, fail, n, q, kth, ids, dis, end;
};

static LearnedPlan plan_learned(int qn, int k)
{
    LearnedPlan p;
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~(size_t)255; return o; };
    p.seed = take(4 * (size_t)qn);
    p.fail = take(4 * (size_t)qn);
    p.n = take(16);
    p.q = take(4 * (size_t)qn);
    p.kth = take(4 * (size_t)qn);
    p.ids = take(4 * (size_t)qn * k);
    p.dis = take(4 * (size_t)qn * k);
    p.end = off;
    return p;
}

static int search_knn_plain_learned_chunk(gts_index *idx, const int *d_qids, int qnum, int k, float *d_kth,
                                          int *d_ids, float *d_dists, cudaStream_t st);

// The plain traversal seeded by the learned radius (GTS_FORM_PLAIN_LEARNED):
// every query starts pruning from its predicted k-th distance instead of
// from infinity; queries whose radius held fewer than k objects are answered
// again by the unseeded traversal, so the results are the plain form's.
// Queries run in chunks whose scratch fits the call's budget.
int search_knn_plain_learned(gts_index *idx, const int *d_qids, int qnum, int k, float *d_kth, int *d_ids,
                             float *d_dists, cudaStream_t st)
{
    const size_t budget = search_budget(idx);
    int qc = std::max(qnum, 1);
    while (qc > 1 && plan_learned(qc, k).end > budget) qc = (qc + 1) / 2;
    if (plan_learned(qc, k).end > budget) {
        gts_set_error("scratch budget of %zu bytes is below the %zu bytes of one seeded query", budget,
                      plan_learned(qc, k).end);
        return GTS_ERR_NOMEM;
    }
    idx->last_fast_overflow = 0;
    for (int q0 = 0; q0 < qnum; q0 += qc) {
        const int n = std::min(qc, qnum - q0);
        int rc = search_knn_plain_learned_chunk(idx, d_qids + q0, n, k, d_kth + q0,
                                                d_ids ? d_ids + (size_t)q0 * k : nullptr,
                                                d_dists ? d_dists + (size_t)q0 * k : nullptr, st);
        if (rc) return rc;
    }
    return GTS_OK;
}

static int search_knn_plain_learned_chunk(gts_index *idx, const int *d_qids, int qnum, int k, float *d_kth,
                                          int *d_ids, float *d_dists, cudaStream_t st)
{
    const LearnedPlan lp = plan_learned(qnum, k);
    const size_t o_seed = lp.seed, o_fail = lp.fail, o_n = lp.n, o_q = lp.q, o_kth = lp.kth, o_ids = lp.ids,
                 o_dis = lp.dis, off = lp.end;
    int rc;
    if ((rc = ensure_scratch(idx, off))) return rc;
    unsigned char *S = (unsigned char *)idx->scratch;
    int *seed = (int *)(S + o_seed), *fail = (int *)(S + o_fail), *n_fail = (int *)(S + o_n);
    int *sub_q = (int *)(S + o_q), *sub_ids = d_ids ? (int *)(S + o_ids) : nullptr;
    float *sub_kth = (float *)(S + o_kth), *sub_dis = d_dists ? (float *)(S + o_dis) : nullptr;
    if ((rc = mlp_seed(idx, d_qids, qnum, k, seed, st))) return rc;
    GTS_CUDA_TRY(cudaMemsetAsync(n_fail, 0, sizeof(int), st));
    SearchArgs a{};
    a.qids = d_qids;
    a.qnum = qnum;
    a.mode = kModeKnn;
    a.k = k;
    a.kth = d_kth;
    a.ids = d_ids;
    a.dists = d_dists;
    a.seed_r2_bits = seed;
    a.fail = fail;
    a.n_fail = n_fail;
    if ((rc = run_search(idx, a, st))) return rc;
    int nf = 0;
    GTS_CUDA_TRY(cudaMemcpyAsync(&nf, n_fail, sizeof(int), cudaMemcpyDeviceToHost, st));
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    idx->last_fast_overflow += nf;
    if (nf == 0) return GTS_OK;
    k_gather_q<<<(nf + 255) / 256, 256, 0, st>>>(d_qids, fail, nf, sub_q);
    idx->kernel_launches++;
    SearchArgs b{};
    b.qids = sub_q;
    b.qnum = nf;
    b.mode = kModeKnn;
    b.k = k;
    b.kth = sub_kth;
    b.ids = sub_ids;
    b.dists = sub_dis;
    idx->keep_stats = true;
    rc = run_search(idx, b, st);
    idx->keep_stats = false;
    if (rc) return rc;
    k_scatter_q<<<(nf + 255) / 256, 256, 0, st>>>(fail, nf, k, sub_kth, sub_ids, sub_dis, d_kth, d_ids, d_dists);
    idx->kernel_launches++;
    GTS_CUDA_TRY(cudaGetLastError());
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    return GTS_OK;
}

int search_knn(gts_index *idx, const int *d_qids, int qnum, int k, int form, float *d_kth, int *d_ids,
               float *d_dists, cudaStream_t st)
{
    if (k < 1 || k > kMaxK) {
        gts_set_error("k must be in [1, %d], got %d", kMaxK, k);
        return GTS_ERR_INVALID;
    }
    if (form == 1 && qnum > 0 && fast_supported(idx, k))
        return search_knn_fast(idx, d_qids, qnum, k, d_kth, d_ids, d_dists, st);
    if (form == 2 && qnum > 0 && idx->mlp_ready && idx->metric == kL2)
        return search_knn_plain_learned(idx, d_qids, qnum, k, d_kth, d_ids, d_dists, st);
    SearchArgs a{};
    a.qids = d_qids;
    a.qnum = qnum;
    a.mode = kModeKnn;
    a.k = k;
    a.kth = d_kth;
    a.ids = d_ids;
    a.dists = d_dists;
    return run_search(idx, a, st);
}

int search_range(gts_index *idx, const int *d_qids, int qnum, float r, int *d_counts,
                 const uint32_t *d_deleted, cudaStream_t st)
{
    SearchArgs a{};
    a.qids = d_qids;
    a.qnum = qnum;
    a.mode = kModeRangeCount;
    a.r = r;
    a.counts = d_counts;
    a.deleted = d_deleted;
    return run_search(idx, a, st);
}

int search_knn_rows(gts_index *idx, const float *d_qrows, const char *d_qstrs, const int *d_qlens, int qnum, int k,
                    float *d_kth, int *d_ids, float *d_dists, cudaStream_t st)
{
    if (k < 1 || k > kMaxK) {
        gts_set_error("k must be in [1, %d], got %d", kMaxK, k);
        return GTS_ERR_INVALID;
    }
    SearchArgs a{};
    a.qnum = qnum;
    a.mode = kModeKnn;
    a.k = k;
    a.kth = d_kth;
    a.ids = d_ids;
    a.dists = d_dists;
    a.qrows = d_qrows;
    a.qstrs = d_qstrs;
    a.qlens = d_qlens;
    return run_search(idx, a, st);
}

int search_range_rows(gts_index *idx, const float *d_qrows, const char *d_qstrs, const int *d_qlens, int qnum,
                      float r, int *d_counts, cudaStream_t st)
{
    SearchArgs a{};
    a.qnum = qnum;
    a.mode = kModeRangeCount;
    a.r = r;
    a.counts = d_counts;
    a.qrows = d_qrows;
    a.qstrs = d_qstrs;
    a.qlens = d_qlens;
    return run_search(idx, a, st);
}

int search_range_timed(gts_index *idx, const int *d_qids, const int *d_qtime, int qnum, float r,
                       const int *d_ent_off, const int4 *d_ents, int *d_tree_counts, int *d_cache_counts,
                       cudaStream_t st)
{
    SearchArgs a{};
    a.qids = d_qids;
    a.qnum = qnum;
    a.mode = kModeRangeTimed;
    a.r = r;
    a.counts = d_tree_counts;
    a.counts2 = d_cache_counts;
    a.qtime = d_qtime;
    a.ent_off = d_ent_off;
    a.ents = d_ents;
    return run_search(idx, a, st);
}

int search_range_ids(gts_index *idx, const int *d_qids, int qnum, float r, int *d_counts, int *d_ids,
                     float *d_dists, const int *d_offsets, cudaStream_t st)
{
    SearchArgs a{};
    a.qids = d_qids;
    a.qnum = qnum;
    a.mode = kModeRangeIds;
    a.r = r;
    a.counts = d_counts;
    a.offsets = d_offsets;
    a.rids = d_ids;
    a.rdists = d_dists;
    return run_search(idx, a, st);
}

}  // namespace gts
