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
// 454-456).  Deleted objects (update path) are skipped
// (update.cuh:244).  Objects of every childless node are verified, at any
// depth, so results equal the exact answer for every tree shape.
#include <cfloat>
#include <cstdio>
#include "index.cuh"

namespace gts {

constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;
constexpr int kBatch = 32;
constexpr int kStackCap = 2048;
constexpr int kLeafObjCap = 1024;     // objects verified per step
constexpr int kMaxK = 256;
constexpr int kCandCap = kLeafObjCap + kMaxK;
constexpr int kSortCap = 2048;        // next power of two >= kCandCap
constexpr int kMaxDimSmem = 1024;

enum SearchMode { kModeKnn = 0, kModeRangeCount = 1, kModeRangeIds = 2 };

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
    unsigned long long *stats;   // [objects filtered, pivots evaluated, exact values, queries]
    float rel_eps;   // relative pruning slack
    float abs_eps;   // absolute pruning slack
};

struct __align__(16) SearchSmem {
    float qrow[kMaxDimSmem];
    uint64_t peq[256];
    char qstr[kStrStride + 3];
    int qlen;
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
    int top, ncand, q, qid, cnt, overflow;
    unsigned long long n_obj, n_piv, n_exact;
    double R;
};

// ---------------------------------------------------------------------------

__device__ __forceinline__ bool is_deleted(const uint32_t *bm, int id)
{
    return bm && ((bm[id >> 5] >> (id & 31)) & 1u);
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
    const float *q = t.dim <= kMaxDimSmem ? s.qrow : t.rows + (size_t)s.qid * t.dim;
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
    const float *q = t.dim <= kMaxDimSmem ? s.qrow : t.rows + (size_t)s.qid * t.dim;
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

// Four rows at once (independent loads in flight): out[u] as warp_row_value.
__device__ __forceinline__ void warp_row_value4(const float *const (&rows)[4], const float *__restrict__ q,
                                                int dim, int metric, int lane, float (&out)[4])
{
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    if ((dim & 3) == 0) {
        const float4 *q4 = reinterpret_cast<const float4 *>(q);
        for (int j = lane; j < (dim >> 2); j += 32) {
            float4 x[4];
#pragma unroll
            for (int u = 0; u < 4; u++) x[u] = __ldg(reinterpret_cast<const float4 *>(rows[u]) + j);
            const float4 y = q4[j];
#pragma unroll
            for (int u = 0; u < 4; u++) {
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
            float x[4];
#pragma unroll
            for (int u = 0; u < 4; u++) x[u] = __ldg(rows[u] + j);
            const float y = q[j];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                float d0 = x[u] - y;
                if (metric == kL2) acc[u] = fmaf(d0, d0, acc[u]);
                else if (metric == kL1) acc[u] += fabsf(d0);
                else acc[u] = fmaxf(acc[u], fabsf(d0));
            }
        }
    }
#pragma unroll
    for (int u = 0; u < 4; u++) out[u] = metric == kLinf ? warp_max(acc[u]) : warp_sum(acc[u]);
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

// Bitonic sort of the candidate buffer by (distance, id), n entries padded
// to the next power of two; keeps the first min(n, k).
__device__ void compact_candidates(SearchSmem &s, int k)
{
    int n = s.ncand;
    int p2 = 1;
    while (p2 < n) p2 <<= 1;
    for (int i = n + threadIdx.x; i < p2; i += kThreads) {
        s.cd[i] = DBL_MAX;
        s.cid[i] = 0x7fffffff;
    }
    __syncthreads();
    for (int size = 2; size <= p2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < p2 / 2; i += kThreads) {
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

__global__ void __launch_bounds__(kThreads) k_search(SearchArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SearchSmem &s = *reinterpret_cast<SearchSmem *>(smem_raw);
    const DevTree &t = a.t;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int O = t.order;
    const bool knn = a.mode == kModeKnn;
    const int acc = knn ? kAccF64 : kAccF32;
    const bool warp_filter = (t.metric == kL2 || t.metric == kL1 || t.metric == kLinf);

    for (;;) {
        if (tid == 0) s.q = atomicAdd(a.counter, 1);
        __syncthreads();
        const int q = s.q;
        if (q >= a.qnum) break;
        const int qid = a.qids[q];
        if (qid < 0 || qid >= t.num) {   // device-API ids are checked here
            if (tid == 0) {
                atomicMax(a.status, (int)kKsBadQuery);
                if (a.mode == kModeKnn) a.kth[q] = __int_as_float(0x7fc00000);
                else if (a.mode == kModeRangeCount) a.counts[q] = -1;
            }
            __syncthreads();
            continue;
        }
        // ---- per-query set-up
        if (tid == 0) {
            s.qid = qid;
            s.top = 1;
            s.stack_node[0] = 0;
            s.stack_off[0] = 0;
            s.stack_lb[0] = 0.f;
            s.ncand = 0;
            s.cnt = 0;
            s.overflow = 0;
            s.n_obj = s.n_piv = s.n_exact = 0;
            s.R = knn ? DBL_MAX : (double)a.r;
        }
        if (t.metric == kEdit) {
            int m = min(max(t.lens[qid], 0), kStrStride - 1);
            const char *src = t.strs + (size_t)qid * kStrStride;
            for (int i = tid; i < kStrStride; i += kThreads) s.qstr[i] = src[i];
            for (int c = tid; c < 256; c += kThreads) {
                uint64_t bits = 0;
                for (int i = 0; i < m && i < 64; i++)
                    if ((unsigned char)src[i] == (unsigned)c) bits |= 1ull << i;
                s.peq[c] = bits;
            }
            if (tid == 0) s.qlen = m;
        } else if (t.dim <= kMaxDimSmem) {
            const float *src = t.rows + (size_t)qid * t.dim;
            for (int i = tid; i < t.dim; i += kThreads) s.qrow[i] = src[i];
        }
        __syncthreads();
        const float *qrow = t.dim <= kMaxDimSmem ? s.qrow : t.rows + (size_t)qid * t.dim;

        // ---- traversal
        for (;;) {
            if (tid == 0) {
                // pop up to kBatch entries whose bound still admits results,
                // stopping early when the leaves would exceed kLeafObjCap
                int nint = 0, nleaf = 0, nobj = 0;
                double R = s.R;
                while (s.top > 0 && nint + nleaf < kBatch) {
                    int node = s.stack_node[s.top - 1];
                    float lb = s.stack_lb[s.top - 1];
                    double slack = a.abs_eps + a.rel_eps * ((double)lb + (R < 1e300 ? R : 0.0));
                    if ((double)lb > R + slack) { s.top--; continue; }
                    if (t.node_pivot[node] >= 0) {
                        s.bint[nint++] = node;
                        s.top--;
                    } else {
                        int off = s.stack_off[s.top - 1];
                        int sz = t.node_size[node] - off;
                        int room = kLeafObjCap - nobj;
                        if (room <= 0) break;
                        int take = sz < room ? sz : room;
                        s.leaf_pre[nleaf] = nobj;
                        s.bleaf_off[nleaf] = off;
                        s.bleaf[nleaf++] = node;
                        nobj += take;
                        if (take < sz) {   // the rest of a large leaf stays on the stack
                            s.stack_off[s.top - 1] = off + take;
                            break;
                        }
                        s.top--;
                    }
                }
                s.leaf_pre[nleaf] = nobj;
                s.nint = nint;
                s.nleaf = nleaf;
                s.ncpos = 0;
                s.n_obj += nobj;
                s.n_piv += nint;
            }
            __syncthreads();
            const int nint = s.nint, nleaf = s.nleaf;
            if (nint == 0 && nleaf == 0) break;
            const int nobj = s.leaf_pre[nleaf];

            // ---- leaves: filter every object, collect those needing exact values
            if (nleaf > 0) {
                if (warp_filter) {
                    // four rows per warp step: their loads are in flight together
                    for (int o0 = warp * 4; o0 < nobj; o0 += kWarps * 4) {
                        int pos[4], id[4];
                        const float *rp[4];
#pragma unroll
                        for (int u = 0; u < 4; u++) {
                            int o = min(o0 + u, nobj - 1);
                            int li = 0;
                            while (s.leaf_pre[li + 1] <= o) li++;
                            pos[u] = t.node_lid[s.bleaf[li]] + s.bleaf_off[li] + (o - s.leaf_pre[li]);
                            id[u] = t.id_list[pos[u]];
                            rp[u] = t.trows + (size_t)pos[u] * t.dim;
                        }
                        float v4[4];
                        warp_row_value4(rp, qrow, t.dim, t.metric, lane, v4);
                        if (lane == 0) {
                            for (int u = 0; u < 4 && o0 + u < nobj; u++) {
                                if (is_deleted(a.deleted, id[u])) continue;
                                double lo, hi;
                                value_bounds(t.metric, t.dim, v4[u], lo, hi);
                                if (id[u] == qid) lo = hi = 0.0;
                                if (knn) {
                                    if (lo <= s.R) {
                                        int c = atomicAdd(&s.ncpos, 1);
                                        s.cpos[c] = pos[u];
                                    }
                                } else if (a.mode == kModeRangeCount && hi < (double)a.r * (1.0 - 2.4e-7)) {
                                    atomicAdd(&s.cnt, 1);
                                } else if (lo <= (double)a.r * (1.0 + 2.4e-7)) {
                                    int c = atomicAdd(&s.ncpos, 1);
                                    s.cpos[c] = pos[u];
                                }
                            }
                        }
                    }
                } else {
                    for (int o = tid; o < nobj; o += kThreads) {
                        int li = 0;
                        while (s.leaf_pre[li + 1] <= o) li++;
                        int pos = t.node_lid[s.bleaf[li]] + s.bleaf_off[li] + (o - s.leaf_pre[li]);
                        if (is_deleted(a.deleted, t.id_list[pos])) continue;
                        int c = atomicAdd(&s.ncpos, 1);
                        s.cpos[c] = pos;
                    }
                }
                __syncthreads();
                // exact values for the collected positions
                const int ncpos = s.ncpos;
                if (tid == 0) s.n_exact += ncpos;
                if (knn && s.ncand + ncpos > kCandCap) compact_candidates(s, a.k);
                for (int c = tid; c < ncpos; c += kThreads) {
                    int pos = s.cpos[c];
                    int id = t.id_list[pos];
                    double d = (id == qid) ? 0.0 : exact_obj(a, s, pos, acc);
                    if (knn) {
                        if (d <= s.R) {
                            int slot = atomicAdd(&s.ncand, 1);
                            s.cd[slot] = d;
                            s.cid[slot] = id;
                        }
                    } else if ((float)d <= a.r) {
                        int slot = atomicAdd(&s.cnt, 1);
                        if (a.mode == kModeRangeIds) {
                            a.rids[a.offsets[q] + slot] = id;
                            a.rdists[a.offsets[q] + slot] = (float)d;
                        }
                    }
                }
                __syncthreads();
                if (knn && s.ncand > kCandCap - kLeafObjCap) compact_candidates(s, a.k);
            }

            // ---- internal nodes: pivot distance bounds, then ring pruning of children
            if (nint > 0) {
                if (warp_filter) {
                    for (int b = warp; b < nint; b += kWarps) {
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
                    for (int b = tid; b < nint; b += kThreads) {
                        int piv = t.node_pivot[s.bint[b]];
                        double d = (piv == qid) ? 0.0 : exact_id(a, s, piv, kAccF64);
                        s.bdq_lo[b] = (float)d;
                        s.bdq_hi[b] = (float)d;
                    }
                }
                __syncthreads();
                const double R = s.R;
                for (int w = tid; w < nint * O; w += kThreads) {
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
            compact_candidates(s, a.k);
            const int k = a.k;
            for (int j = tid; j < k; j += kThreads) {
                bool have = j < s.ncand;
                if (a.ids) a.ids[(size_t)q * k + j] = have ? s.cid[j] : -1;
                if (a.dists) a.dists[(size_t)q * k + j] = have ? (float)s.cd[j] : (float)t.infi_dis;
            }
            if (tid == 0) a.kth[q] = s.ncand >= k ? (float)s.cd[k - 1] : (float)t.infi_dis;
        } else if (tid == 0) {
            if (a.mode == kModeRangeCount) a.counts[q] = s.cnt;
        }
        if (tid == 0) {
            if (s.overflow) atomicMax(a.status, (int)kKsStackOverflow);
            if (a.stats) {
                atomicAdd(&a.stats[0], s.n_obj);
                atomicAdd(&a.stats[1], s.n_piv);
                atomicAdd(&a.stats[2], s.n_exact);
                atomicAdd(&a.stats[3], 1ull);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------

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
    size_t smem = sizeof(SearchSmem);
    GTS_CUDA_TRY(cudaFuncSetAttribute(k_search, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_search, kThreads, smem);
    if (per_sm < 1) per_sm = 1;
    int grid = nsm * per_sm;
    if (grid > a.qnum) grid = a.qnum;
    k_search<<<grid, kThreads, smem, st>>>(a);
    idx->kernel_launches++;
    GTS_CUDA_TRY(cudaGetLastError());
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

int search_knn(gts_index *idx, const int *d_qids, int qnum, int k, int form, float *d_kth, int *d_ids,
               float *d_dists, cudaStream_t st)
{
    if (k < 1 || k > kMaxK) {
        gts_set_error("k must be in [1, %d], got %d", kMaxK, k);
        return GTS_ERR_INVALID;
    }
    if (form == 1 && qnum > 0 && fast_supported(idx, k))
        return search_knn_fast(idx, d_qids, qnum, k, d_kth, d_ids, d_dists, st);
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
