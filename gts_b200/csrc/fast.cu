// fast.cu -- exact L2 kNN with a BF16 tensor-core filter ("fast" form).
//
// Same answers as searchIndexKnnV2 (search_v2.cuh:975-1228): the k-th
// distance of every query in the reference's F64 leaf arithmetic
// (search_v2.cuh:447-463) and the k nearest ids with ties broken by id.
// How it gets there is B200-specific:
//
//  * layout: objects are grouped into blocks of 128 consecutive tree
//    positions.  Each block is stored once in HBM as a record that a single
//    bulk copy drops into shared memory in the exact operand layout tcgen05
//    reads (K-major, 128-byte swizzle): 128 rows of BF16 residuals r = o - c
//    against the block mean c, 3 rows holding c split into three BF16 parts
//    (c = c_hi + c_mid + c_lo exactly), 13 zero rows, then per object
//    |o|^2 and |r| as floats (|o|^2 accumulated in FP64);
//  * filter: a CTA owns 128 queries (sorted by tree position, so a tile's
//    queries sit in the same region of the tree).  Their rows, split into
//    BF16 q_hi + q_lo, are the A operand; each block is one 128 x 144 x K
//    MMA chain into TMEM giving q.r for the 128 objects and q.c from the
//    centre rows.  One thread per query turns its TMEM row into
//        d^2 ~ |q|^2 + |o|^2 - 2 (q.c + q.r)
//    with a certified bound E (BF16 rounding of r, the hi/lo split of q,
//    FP32 accumulation, FP32 evaluation), keeps the k smallest upper bounds
//    (a running k-th radius R) and appends every object whose lower bound
//    is <= R to the query's candidate list;
//  * recheck: every candidate whose lower bound is <= the final R gets its
//    reference-arithmetic distance; the k best (distance, id) are the answer.
// No object whose reference distance can rank in the top k is ever dropped,
// so the result is exact.  Queries whose candidate list overflows are
// answered by the plain path.
#include <cub/device/device_radix_sort.cuh>
#include <cfloat>
#include <cstdio>
#include <vector>
#include "index.cuh"
#include "sm100.cuh"

namespace gts {

using namespace sm100;

constexpr int kFB = 128;              // objects per block
constexpr int kFN = 144;              // B rows per block: objects + centre rows + padding
constexpr int kFT = 128;              // queries per tile (A rows, TMEM lanes)
constexpr int kFMaxKp = 128;          // padded dimension limit of this path (shared-memory budget)
constexpr int kFMaxK = 64;
constexpr int kFCand = 2048;          // candidate slots per query
constexpr long long kFWait = 1ll << 24;   // bounded mbarrier polls

// Filter error-bound constants (see header comment).
constexpr float kKappa = 0.004f;      // >= 2^-8 + 2^-16 + 2 * 256 * 2^-24
constexpr float kEpsC = 5e-5f;        // >= 2^-16 + 2 * 256 * 2^-24

struct FastShape {
    int kp, nk;              // padded dim, number of 64-wide K chunks
    uint32_t btile_bytes;    // nk * kFN * 128
    uint32_t rec_bytes;      // btile_bytes + 1024 (o2, rn) + 16 (|c|, pad)
    uint32_t atile_bytes;    // nk * kFT * 128
};

__host__ __device__ inline FastShape fast_shape(int dim)
{
    FastShape s;
    s.kp = (dim + 63) / 64 * 64;
    s.nk = s.kp / 64;
    s.btile_bytes = (uint32_t)s.nk * kFN * 128u;
    s.rec_bytes = s.btile_bytes + 1024u + 1024u;   // o2[128], rn[128], then |c|, valid count, padding
    s.atile_bytes = (uint32_t)s.nk * kFT * 128u;
    return s;
}

__device__ __forceinline__ unsigned short f2bf(float x)
{
    return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
__device__ __forceinline__ float bf2f(unsigned short b) { return __bfloat162float(__ushort_as_bfloat16(b)); }

// ---------------------------------------------------------------- prep

// One CTA per block of 128 tree positions; thread t = object t of the block.
__global__ void __launch_bounds__(128) k_fast_prep(int n, int dim, const float *__restrict__ trows,
                                                   unsigned char *__restrict__ recs, FastShape fs)
{
    __shared__ double csum[kFMaxKp];
    __shared__ float cen[kFMaxKp];
    const int b = blockIdx.x, t = threadIdx.x;
    const int base = b * kFB;
    const int cnt = min(kFB, n - base);
    unsigned char *rec = recs + (size_t)b * fs.rec_bytes;
    for (int j = t; j < fs.kp; j += 128) {
        double s = 0.0;
        if (j < dim)
            for (int i = 0; i < cnt; i++) s += (double)trows[(size_t)(base + i) * dim + j];
        csum[j] = s;
        cen[j] = j < dim ? (float)(s / cnt) : 0.f;
    }
    __syncthreads();
    // centre rows 128..130: c = hi + mid + lo; rows 131..143 zero
    if (t < 16) {
        for (int j = 0; j < fs.kp; j++) {
            float c = cen[j];
            unsigned short hi = f2bf(c);
            float r1 = c - bf2f(hi);
            unsigned short mid = f2bf(r1);
            unsigned short lo = f2bf(r1 - bf2f(mid));
            unsigned short v = t == 0 ? hi : (t == 1 ? mid : (t == 2 ? lo : 0));
            *reinterpret_cast<unsigned short *>(rec + sw128_offset(kFB + t, j, kFN)) = v;
        }
    }
    if (t == 0) {
        double c2 = 0.0;
        for (int j = 0; j < dim; j++) c2 += (double)cen[j] * cen[j];
        reinterpret_cast<float *>(rec + fs.btile_bytes + 1024)[0] = (float)sqrt(c2);
        reinterpret_cast<int *>(rec + fs.btile_bytes + 1024)[1] = cnt;
    }
    // residual rows
    const bool valid = t < cnt;
    const float *row = trows + (size_t)(base + t) * dim;
    double o2 = 0.0, r2 = 0.0;
    for (int j = 0; j < fs.kp; j++) {
        float r = 0.f;
        if (valid && j < dim) {
            float o = row[j];
            o2 += (double)o * o;
            r = o - cen[j];
            r2 += (double)r * r;
        }
        *reinterpret_cast<unsigned short *>(rec + sw128_offset(t, j, kFN)) = f2bf(r);
    }
    float *tail = reinterpret_cast<float *>(rec + fs.btile_bytes);
    tail[t] = valid ? (float)o2 : 3.0e38f;
    tail[128 + t] = valid ? (float)sqrt(r2) : 0.f;
}

// ---------------------------------------------------------------- tile

struct FastTileArgs {
    const float *rows;          // id-order rows
    const int *qids;            // caller's query ids
    const int *order;           // query indices sorted by tree position
    const int *pos_of_id;
    const unsigned char *recs;
    int qnum, dim, nb, k, splits;
    FastShape fs;
    int *cand_pos;              // [qnum][kFCand]
    float *cand_lb;             // [qnum][kFCand]
    int *cand_cnt;              // [qnum]
    int *r2_bits;               // [qnum] radius^2 bound as int bits (the append pass's seed)
    float *hbuf;                // bound pass: [qnum][splits][CG][k] smallest upper bounds
    int *item_counter;          // persistent-CTA work queue over (tile, split) items
    int ntiles;
    int *status;
    unsigned long long *stats;
};

constexpr int kFS = 3;   // B stages: copies run two blocks ahead of the MMAs

struct __align__(8) FastCtl {
    uint64_t full[kFS];
    uint64_t mmad[2];
    uint32_t tmem;
    int item;
    int err;
    int pend[kFS];     // copies issued per stage
    int done[kFS];     // copy completions observed per stage (by the MMA issuer)
    int qis[kFT];      // query index of each TMEM lane
    float q2s[kFT];    // |q|^2 (from FP64)
    float qns[kFT];    // |q|
};

// Persistent filter kernel, one CTA per SM.  Work items are (tile, split):
// the 128 queries of a tile (sorted by tree position) against the blocks
// b = split (mod splits).  MODE 0: bound pass -- every thread keeps its
// k smallest upper bounds and writes them to hbuf; MODE 2: the same while
// also appending objects within the running bound capped by a seed (one
// pass for a seeded run); MODE 1: append pass --
// objects whose lower bound is within the query's seed are appended.
//
// CG column groups of 4 warps: warps w, w+4, ... share TMEM lanes
// 32*(w%4)..+31 (the same 32 queries) and split the 128 object columns, so an
// SM runs 4*CG warps of epilogue.
//
// Pipeline per CTA (global block counter gi, barrier parities follow it):
// bulk copy of block gi into B[gi % 3] -> MMA chain into D[gi % 2] (TMEM
// columns 0 / 256) -> epilogue on D[gi % 2].  The MMA of block gi+1 is
// issued before the epilogue of block gi; the copy of block gi+3 after it.
template <int CG, int MODE>
__global__ void __launch_bounds__(128 * CG, 1) k_fast_tile(FastTileArgs a)
{
    constexpr int NT = 128 * CG;
    constexpr int CW = 128 / CG;   // object columns per thread
    extern __shared__ __align__(1024) unsigned char fsm[];
    // 1024-aligned carve-up: A_hi | A_lo | B0 | B1 | B2 | heap | ctl
    unsigned char *base = (unsigned char *)(((uintptr_t)fsm + 1023) & ~(uintptr_t)1023);
    const FastShape fs = a.fs;
    unsigned char *A_hi = base;
    unsigned char *A_lo = A_hi + fs.atile_bytes;
    const uint32_t rec_pad = (fs.rec_bytes + 1023u) & ~1023u;
    unsigned char *B0 = A_lo + fs.atile_bytes;
    float *heap = reinterpret_cast<float *>(B0 + kFS * rec_pad);
    FastCtl &ctl = *reinterpret_cast<FastCtl *>(heap + (MODE == 1 ? 0 : NT * a.k));

    const int t = threadIdx.x, warp = t >> 5;
    const int lq = t & 127, g = t >> 7;   // query lane, column group
    const int k = a.k, splits = a.splits;

    if (t == 0) {
        for (int s = 0; s < kFS; s++) {
            mbar_init(&ctl.full[s], 1);
            ctl.pend[s] = 0;
            ctl.done[s] = 0;
        }
        for (int s = 0; s < 2; s++) mbar_init(&ctl.mmad[s], 1);
        ctl.err = 0;
        fence_mbar_init();
    }
    if (warp == 0) {
        tmem_alloc(&ctl.tmem, 512);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = ctl.tmem;
    const uint32_t idesc = idesc_bf16_f32(kFT, kFN);
    const uint32_t a_hi_s = smem_u32(A_hi), a_lo_s = smem_u32(A_lo);
    long long gblk = 0;   // blocks this CTA has run through the pipeline
    unsigned long long blocks_done = 0, appended = 0;

    for (;;) {
        if (t == 0) ctl.item = atomicAdd(a.item_counter, 1);
        __syncthreads();
        const int item = ctl.item;
        if (item >= a.ntiles * splits || ctl.err) break;
        const int tile = item / splits, split = item % splits;

        // ---- A operand (first column group): the query, split into BF16 hi + lo
        if (g == 0) {
            const int slot = tile * kFT + lq;
            const int qi = slot < a.qnum ? a.order[slot] : -1;
            const int qid = qi >= 0 ? a.qids[qi] : -1;
            const float *row = qid >= 0 ? a.rows + (size_t)qid * a.dim : nullptr;
            double acc = 0.0;
            for (int j0 = 0; j0 < fs.kp; j0 += 8) {
                unsigned short hi[8], lo[8];
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    int j = j0 + u;
                    float x = (row && j < a.dim) ? row[j] : 0.f;
                    acc += (double)x * x;
                    hi[u] = f2bf(x);
                    lo[u] = f2bf(x - bf2f(hi[u]));
                }
                uint4 vh, vl;
                vh.x = hi[0] | ((uint32_t)hi[1] << 16); vh.y = hi[2] | ((uint32_t)hi[3] << 16);
                vh.z = hi[4] | ((uint32_t)hi[5] << 16); vh.w = hi[6] | ((uint32_t)hi[7] << 16);
                vl.x = lo[0] | ((uint32_t)lo[1] << 16); vl.y = lo[2] | ((uint32_t)lo[3] << 16);
                vl.z = lo[4] | ((uint32_t)lo[5] << 16); vl.w = lo[6] | ((uint32_t)lo[7] << 16);
                uint32_t off = sw128_offset(lq, j0, kFT);
                *reinterpret_cast<uint4 *>(A_hi + off) = vh;
                *reinterpret_cast<uint4 *>(A_lo + off) = vl;
            }
            ctl.qis[lq] = qi;
            ctl.q2s[lq] = (float)acc;
            ctl.qns[lq] = (float)sqrt(acc);
        }
        if (MODE != 1)
            for (int i = 0; i < k; i++) heap[i * NT + t] = FLT_MAX;
        fence_proxy_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        const int qi = ctl.qis[lq];
        const float q2 = ctl.q2s[lq], qn = ctl.qns[lq];
        const float cq = 2.f * kKappa * qn;
        const float seed = (MODE != 0 && qi >= 0) ? __int_as_float(a.r2_bits[qi]) : FLT_MAX;
        float R2 = seed;
        int hidx = 0;
        const int n = (a.nb - split + splits - 1) / splits;   // blocks of this item

        auto issue_copy = [&](int j) {
            const long long gi = gblk + j;
            const int s = (int)(gi % kFS);
            const unsigned char *src = a.recs + (size_t)(split + (size_t)j * splits) * fs.rec_bytes;
            mbar_arrive_expect_tx(&ctl.full[s], fs.rec_bytes);
            bulk_g2s(B0 + (size_t)s * rec_pad, src, fs.rec_bytes, &ctl.full[s]);
            ctl.pend[s]++;
        };
        auto issue_mma = [&](int j) -> bool {
            const long long gi = gblk + j;
            const int s = (int)(gi % kFS), d = (int)(gi & 1);
            if (!mbar_wait(&ctl.full[s], (uint32_t)((gi / kFS) & 1), kFWait)) return false;
            ctl.done[s]++;
            tc_fence_after();
            const uint32_t b_s = smem_u32(B0 + (size_t)s * rec_pad);
            const uint32_t dt = tmem + (uint32_t)(d * 256);
            const int ksteps = fs.kp / 16;
            for (int kk = 0; kk < ksteps; kk++) {
                uint32_t off = (uint32_t)(kk >> 2) * (kFT * 128u) + (uint32_t)(kk & 3) * 32u;
                uint32_t boff = (uint32_t)(kk >> 2) * (kFN * 128u) + (uint32_t)(kk & 3) * 32u;
                mma_bf16(dt, smem_desc_sw128(a_hi_s + off, 1024), smem_desc_sw128(b_s + boff, 1024), idesc,
                         kk > 0 ? 1u : 0u);
            }
            for (int kk = 0; kk < ksteps; kk++) {
                uint32_t off = (uint32_t)(kk >> 2) * (kFT * 128u) + (uint32_t)(kk & 3) * 32u;
                uint32_t boff = (uint32_t)(kk >> 2) * (kFN * 128u) + (uint32_t)(kk & 3) * 32u;
                mma_bf16(dt, smem_desc_sw128(a_lo_s + off, 1024), smem_desc_sw128(b_s + boff, 1024), idesc, 1u);
            }
            mma_commit(&ctl.mmad[d]);
            return true;
        };

        if (t == 0) {
            for (int j = 0; j < kFS && j < n; j++) issue_copy(j);
            if (n > 0 && !issue_mma(0)) ctl.err = 1;
        }
        __syncthreads();
        for (int j = 0; j < n; j++) {
            const long long gi = gblk + j;
            const int s = (int)(gi % kFS), d = (int)(gi & 1);
            if (t == 0 && !ctl.err && j + 1 < n) {
                if (!issue_mma(j + 1)) ctl.err = 2;
            }
            if (!mbar_wait(&ctl.mmad[d], (uint32_t)((gi >> 1) & 1), kFWait)) ctl.err = 3;
            tc_fence_after();
            __syncthreads();
            if (ctl.err) break;
            // make the record's tail visible to every thread
            mbar_wait(&ctl.full[s], (uint32_t)((gi / kFS) & 1), kFWait);
            const unsigned char *Bs = B0 + (size_t)s * rec_pad;
            const int blk = split + j * splits;
            const float *o2 = reinterpret_cast<const float *>(Bs + fs.btile_bytes);
            const float *rn = o2 + 128;
            const float cn = o2[256];
            const int nvalid = reinterpret_cast<const int *>(o2)[257];
            const uint32_t taddr = tmem + ((uint32_t)(warp & 3) * 32u << 16) + (uint32_t)(d * 256);
            float v[16];
            tmem_ld16(taddr + 128, v);
            const float qc = v[0] + v[1] + v[2];
            const float ec = 2.f * kEpsC * qn * cn + 1e-6f;
            // lb = (|q|^2 - 2 q.c - ec - 2e-6 |q|^2) + |o|^2 (1 - 2e-6) - cq |r| - 2 q.r
            const float t0 = q2 - 2.f * qc - ec - 2e-6f * q2;
#pragma unroll 1
            for (int c = g * CW; c < (g + 1) * CW; c += 16) {
                tmem_ld16(taddr + (uint32_t)c, v);
                if (qi < 0) continue;
#pragma unroll
                for (int u = 0; u < 16; u++) {
                    const int jj = c + u;
                    if (jj >= nvalid) break;
                    const float oo = o2[jj], rr = rn[jj];
                    const float lb = fmaf(-2.f, v[u], fmaf(-cq, rr, fmaf(oo, 0.999998f, t0)));
                    if (lb <= R2) {
                        if (MODE != 0) {
                            int sl = atomicAdd(&a.cand_cnt[qi], 1);
                            if (sl < kFCand) {
                                a.cand_pos[(size_t)qi * kFCand + sl] = blk * kFB + jj;
                                a.cand_lb[(size_t)qi * kFCand + sl] = lb;
                            }
                            appended++;
                        }
                        if (MODE != 1) {
                            const float ub = lb + 2.f * fmaf(cq, rr, ec + 2e-6f * (q2 + oo));
                            if (ub < R2) {   // replace the largest of the k kept bounds
                                heap[hidx * NT + t] = ub;
                                float mx = -1.f;
                                for (int h = 0; h < k; h++) {
                                    float hv = heap[h * NT + t];
                                    if (hv > mx) { mx = hv; hidx = h; }
                                }
                                R2 = fminf(mx, seed);
                            }
                        }
                    }
                }
            }
            blocks_done++;
            tc_fence_before();
            __syncthreads();
            if (t == 0 && j + kFS < n) issue_copy(j + kFS);
        }
        gblk += n;
        if (MODE != 1 && qi >= 0) {
            float *dst = a.hbuf + (((size_t)qi * splits + split) * CG + g) * k;
            for (int h = 0; h < k; h++) dst[h] = heap[h * NT + t];
        }
        tc_fence_before();
        __syncthreads();
    }
    if (a.stats && appended) atomicAdd(&a.stats[5], appended);
    if (a.stats && blocks_done && t == 0) {
        atomicAdd(&a.stats[0], blocks_done);
        atomicAdd(&a.stats[1], (unsigned long long)fs.rec_bytes * blocks_done);
    }
    if (t == 0 && ctl.err) {
        atomicMax(a.status, 16 + ctl.err);
        // let copies still in flight land before the CTA leaves (bounded)
        for (int s = 0; s < kFS; s++)
            for (int m = ctl.done[s]; m < ctl.pend[s]; m++) mbar_wait(&ctl.full[s], (uint32_t)(m & 1), kFWait);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 512);
}

// Bound merge: the k-th smallest of every upper bound a query's threads kept
// in the bound pass (no object appears twice: each block belongs to one
// split and each column to one group), capped by any seed already there.
__global__ void __launch_bounds__(128) k_fast_merge(const float *__restrict__ hbuf, int per_query, int k,
                                                    int *__restrict__ r2_bits)
{
    __shared__ float v[1024];
    const int q = blockIdx.x, t = threadIdx.x;
    int p2 = 1;
    while (p2 < per_query) p2 <<= 1;
    for (int i = t; i < p2; i += 128) v[i] = i < per_query ? hbuf[(size_t)q * per_query + i] : FLT_MAX;
    __syncthreads();
    for (int size = 2; size <= p2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = t; i < p2 / 2; i += 128) {
                int lo = 2 * i - (i & (stride - 1)), hi = lo + stride;
                bool up = (lo & size) == 0;
                float a = v[lo], b = v[hi];
                if ((a > b) == up) {
                    v[lo] = b;
                    v[hi] = a;
                }
            }
            __syncthreads();
        }
    }
    if (t == 0) {
        float kth = v[k - 1];
        atomicMin(&r2_bits[q], __float_as_int(kth > 0.f ? kth : 0.f));
    }
}

// ---------------------------------------------------------------- finalize

constexpr int kFinSort = kFCand;

// One CTA per query: exact values of the surviving candidates, de-duplicated,
// top k by (distance, id).  Sets overflow[q] when the list was truncated.
__global__ void __launch_bounds__(128) k_fast_final(const float *__restrict__ rows, int dim, int num,
                                                    const int *__restrict__ id_list,
                                                    const int *__restrict__ qids, int qnum, int k,
                                                    int infi_dis, const int *__restrict__ cand_pos,
                                                    const float *__restrict__ cand_lb,
                                                    const int *__restrict__ cand_cnt,
                                                    const int *__restrict__ r2_bits, float *kth, int *ids,
                                                    float *dists, int *overflow, int *n_overflow,
                                                    unsigned long long *stats)
{
    __shared__ double cd[kFinSort];
    __shared__ int cid[kFinSort];
    __shared__ int ns;
    const int q = blockIdx.x, t = threadIdx.x;
    const int qid = qids[q];
    const int cnt = cand_cnt[q];
    if (cnt > kFCand) {
        if (t == 0) {
            overflow[atomicAdd(n_overflow, 1)] = q;
        }
        return;
    }
    const float R2 = __int_as_float(r2_bits[q]);
    if (t == 0) ns = 0;
    __syncthreads();
    const float *qrow = rows + (size_t)qid * dim;
    for (int i = t; i < cnt; i += 128) {
        if (cand_lb[(size_t)q * kFCand + i] > R2) continue;
        int pos = cand_pos[(size_t)q * kFCand + i];
        if (pos < 0 || pos >= num) continue;
        int id = id_list[pos];
        double d = (id == qid) ? 0.0 : dist_row_f64(rows + (size_t)id * dim, qrow, dim, kL2);
        int sl = atomicAdd(&ns, 1);
        cd[sl] = d;
        cid[sl] = id;
    }
    __syncthreads();
    const int n = ns;
    if (t == 0 && stats) atomicAdd(&stats[2], (unsigned long long)n);
    int p2 = 1;
    while (p2 < n) p2 <<= 1;
    for (int i = n + t; i < p2; i += 128) {
        cd[i] = DBL_MAX;
        cid[i] = 0x7fffffff;
    }
    __syncthreads();
    for (int size = 2; size <= p2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = t; i < p2 / 2; i += 128) {
                int lo = 2 * i - (i & (stride - 1)), hi = lo + stride;
                bool up = (lo & size) == 0;
                double dl = cd[lo], dh = cd[hi];
                int il = cid[lo], ih = cid[hi];
                bool gt = (dl > dh) || (dl == dh && il > ih);
                if (gt == up) {
                    cd[lo] = dh; cd[hi] = dl;
                    cid[lo] = ih; cid[hi] = il;
                }
            }
            __syncthreads();
        }
    }
    if (t == 0) {   // distinct ids in order (CTAs of one tile can share a block)
        int m = 0, within = 0;
        for (int i = 0; i < n && m < k; i++) {
            if (m > 0 && cid[i] == cid[m - 1] && cd[i] == cd[m - 1]) continue;
            cd[m] = cd[i];
            cid[m] = cid[i];
            within += cd[m] * cd[m] <= (double)R2;
            m++;
        }
        // every object within the bound is a candidate, so the answer is
        // exact once k distinct candidates lie within it; a seeded bound that
        // was too small leaves fewer, and the query is answered again
        if (within < k && within < num) {
            overflow[atomicAdd(n_overflow, 1)] = q;
            return;
        }
        kth[q] = m >= k ? (float)cd[k - 1] : (float)infi_dis;
        for (int j = 0; j < k; j++) {
            if (ids) ids[(size_t)q * k + j] = j < m ? cid[j] : -1;
            if (dists) dists[(size_t)q * k + j] = j < m ? (float)cd[j] : (float)infi_dis;
        }
    }
}

__global__ void k_fast_keys(const int *qids, int qnum, const int *pos_of_id, int *keys, int *vals)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < qnum) {
        keys[i] = pos_of_id[qids[i]];
        vals[i] = i;
    }
}

__global__ void k_fast_init(int qnum, int *cand_cnt, int *r2_bits)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < qnum) {
        cand_cnt[i] = 0;
        r2_bits[i] = __float_as_int(FLT_MAX);
    }
}

__global__ void k_add_stat(unsigned long long *p, unsigned long long v) { *p += v; }

__global__ void k_gather_i(const int *src, const int *idx, int n, int *dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}

__global__ void k_scatter_results(const int *idx, int n, int k, const float *kth_s, const int *ids_s,
                                  const float *dis_s, float *kth, int *ids, float *dists)
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

// ---------------------------------------------------------------- host

// Column groups per query lane: as many warps as the bound heaps
// (threads x k floats, at most 32 KB of shared memory) allow.
static int fast_cg(int k) { return k <= 16 ? 4 : (k <= 32 ? 2 : 1); }

template <int CG, int MODE>
static int launch_fast_tile_cg(const FastTileArgs &a, int grid, cudaStream_t st)
{
    const uint32_t rec_pad = (a.fs.rec_bytes + 1023u) & ~1023u;
    size_t smem = 1024 + 2 * (size_t)a.fs.atile_bytes + kFS * (size_t)rec_pad +
                  (MODE == 1 ? 0 : sizeof(float) * 128 * CG * (size_t)a.k) + sizeof(FastCtl) + 64;
    GTS_CUDA_TRY(cudaFuncSetAttribute(k_fast_tile<CG, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    GTS_CUDA_TRY(cudaMemsetAsync(a.item_counter, 0, sizeof(int), st));
    k_fast_tile<CG, MODE><<<grid, 128 * CG, smem, st>>>(a);
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

template <int MODE>
static int launch_fast_tile(const FastTileArgs &a, int grid, cudaStream_t st)
{
    switch (fast_cg(a.k)) {
    case 4: return launch_fast_tile_cg<4, MODE>(a, grid, st);
    case 2: return launch_fast_tile_cg<2, MODE>(a, grid, st);
    default: return launch_fast_tile_cg<1, MODE>(a, grid, st);
    }
}

bool fast_supported(const gts_index *idx, int k)
{
    return idx->metric == kL2 && idx->dim <= kFMaxKp && k >= 1 && k <= kFMaxK && idx->num >= 1;
}

static int fast_prepare(gts_index *idx, cudaStream_t st)
{
    if (idx->fast_recs) return GTS_OK;
    FastShape fs = fast_shape(idx->dim);
    int nb = (idx->num + kFB - 1) / kFB;
    size_t bytes = (size_t)nb * fs.rec_bytes;
    unsigned char *recs = nullptr;
    int rc = dev_alloc(&recs, bytes, nullptr);
    if (rc) return rc;
    GTS_CUDA_TRY(cudaMemsetAsync(recs, 0, bytes, st));
    k_fast_prep<<<nb, 128, 0, st>>>(idx->num, idx->dim, idx->trows, recs, fs);
    GTS_CUDA_TRY(cudaGetLastError());
    idx->fast_recs = recs;
    idx->fast_nb = nb;
    idx->device_bytes += bytes;
    return GTS_OK;
}

// One filter run over a query batch.  seeded: take each query's starting
// bound from the learned radius model and make a single appending pass;
// otherwise a bound-only pass first.  Queries the run cannot answer (a
// seed below the k-th distance, or a full candidate list) are written to
// d_fail (owned by the caller) and counted in *n_fail.
// fixed (optional): caller-owned device scratch of fixed_bytes used instead
// of the index's growable scratch.
static int fast_run(gts_index *idx, const int *d_qids, int qnum, int k, bool seeded, float *d_kth, int *d_ids,
                    float *d_dists, int *d_fail, int *n_fail, cudaStream_t st, unsigned char *fixed = nullptr,
                    size_t fixed_bytes = 0)
{
    const FastShape fs = fast_shape(idx->dim);
    const int ntiles = (qnum + kFT - 1) / kFT;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // items = tiles x splits, about four per SM for balance; the bound merge
    // holds splits * CG * k <= 1024 values per query
    const int cg = fast_cg(k);
    int splits = (4 * nsm + ntiles - 1) / ntiles;
    if (splits < 1) splits = 1;
    if (splits > 1024 / (cg * k)) splits = 1024 / (cg * k);
    if (splits > idx->fast_nb) splits = idx->fast_nb;
    const int grid = std::min(nsm, ntiles * splits);

    size_t cub_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (int *)nullptr, (int *)nullptr, (int *)nullptr,
                                    (int *)nullptr, qnum, 0, 32, st);
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~(size_t)255; return o; };
    size_t o_keys = take(sizeof(int) * qnum), o_vals = take(sizeof(int) * qnum);
    size_t o_skeys = take(sizeof(int) * qnum), o_order = take(sizeof(int) * qnum);
    size_t o_cpos = take(sizeof(int) * (size_t)qnum * kFCand), o_clb = take(sizeof(float) * (size_t)qnum * kFCand);
    size_t o_ccnt = take(sizeof(int) * qnum), o_r2 = take(sizeof(int) * qnum);
    size_t o_novf = take(sizeof(int)), o_items = take(sizeof(int));
    size_t o_hbuf = take(sizeof(float) * (size_t)qnum * splits * cg * k);
    size_t o_cub = take(cub_bytes);
    int rc;
    unsigned char *S = fixed;
    if (fixed) {
        if (off > fixed_bytes) {
            gts_set_error("filter run needs %zu bytes of scratch, the fixed array holds %zu", off, fixed_bytes);
            return GTS_ERR_INVALID;
        }
    } else {
        if ((rc = ensure_scratch(idx, off))) return rc;
        S = (unsigned char *)idx->scratch;
    }
    int *keys = (int *)(S + o_keys), *vals = (int *)(S + o_vals), *skeys = (int *)(S + o_skeys);
    int *order = (int *)(S + o_order), *cpos = (int *)(S + o_cpos), *ccnt = (int *)(S + o_ccnt);
    float *clb = (float *)(S + o_clb);
    int *r2 = (int *)(S + o_r2), *novf = (int *)(S + o_novf);

    k_fast_keys<<<(qnum + 255) / 256, 256, 0, st>>>(d_qids, qnum, idx->pos_of_id, keys, vals);
    size_t cb = cub_bytes;
    GTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(S + o_cub, cb, keys, skeys, vals, order, qnum, 0, 32, st));
    k_fast_init<<<(qnum + 255) / 256, 256, 0, st>>>(qnum, ccnt, r2);
    if (seeded && (rc = mlp_seed(idx, d_qids, qnum, k, r2, st))) return rc;
    GTS_CUDA_TRY(cudaMemsetAsync(novf, 0, sizeof(int), st));

    FastTileArgs a;
    a.rows = idx->rows;
    a.qids = d_qids;
    a.order = order;
    a.pos_of_id = idx->pos_of_id;
    a.recs = idx->fast_recs;
    a.qnum = qnum;
    a.dim = idx->dim;
    a.nb = idx->fast_nb;
    a.k = k;
    a.splits = splits;
    a.fs = fs;
    a.cand_pos = cpos;
    a.cand_lb = clb;
    a.cand_cnt = ccnt;
    a.r2_bits = r2;
    a.hbuf = (float *)(S + o_hbuf);
    a.item_counter = (int *)(S + o_items);
    a.ntiles = ntiles;
    a.status = idx->d_status;
    a.stats = idx->d_stats;
    // seeded: one pass that appends within min(seed, running k-th bound) and
    // keeps the bounds; otherwise a bound pass first, then an appending one.
    // The merge lowers each query's bound to the k-th smallest kept bound.
    if ((rc = seeded ? launch_fast_tile<2>(a, grid, st) : launch_fast_tile<0>(a, grid, st))) return rc;
    k_fast_merge<<<qnum, 128, 0, st>>>(a.hbuf, splits * cg * k, k, r2);
    GTS_CUDA_TRY(cudaGetLastError());
    if (!seeded && (rc = launch_fast_tile<1>(a, grid, st))) return rc;
    k_add_stat<<<1, 1, 0, st>>>(idx->d_stats + 6, seeded ? 1ull : 2ull);
    k_fast_final<<<qnum, 128, 0, st>>>(idx->rows, idx->dim, idx->num, idx->id_list, d_qids, qnum, k,
                                        idx->params.infi_dis, cpos, clb, ccnt, r2, d_kth, d_ids, d_dists,
                                        d_fail, novf, idx->d_stats);
    GTS_CUDA_TRY(cudaGetLastError());
    int status = 0;
    GTS_CUDA_TRY(cudaMemcpyAsync(&status, idx->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    GTS_CUDA_TRY(cudaMemcpyAsync(n_fail, novf, sizeof(int), cudaMemcpyDeviceToHost, st));
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    if (status != 0) {
        gts_set_error("tensor-core filter kernel reported status %d (barrier wait gave up)", status);
        return GTS_ERR_KERNEL;
    }
    return GTS_OK;
}

// Queries listed in d_fail (indices into d_qids) answered again: unseeded
// filter first when the first run was seeded, the plain traversal last.
static int rerun_failed(gts_index *idx, const int *d_qids, int k, bool was_seeded, const int *d_fail, int n_fail,
                        float *d_kth, int *d_ids, float *d_dists, cudaStream_t st)
{
    int *sub_q = nullptr, *sub_ids = nullptr, *sub_fail = nullptr, *fail_copy = nullptr;
    float *sub_kth = nullptr, *sub_dis = nullptr;
    DevVec keep;
    int rc;
    if ((rc = keep.alloc(&sub_q, n_fail)) || (rc = keep.alloc(&sub_kth, n_fail)) ||
        (rc = keep.alloc(&fail_copy, n_fail)) || (rc = keep.alloc(&sub_fail, n_fail)) ||
        (d_ids && (rc = keep.alloc(&sub_ids, (size_t)n_fail * k))) ||
        (d_dists && (rc = keep.alloc(&sub_dis, (size_t)n_fail * k))))
        return rc;
    GTS_CUDA_TRY(cudaMemcpyAsync(fail_copy, d_fail, sizeof(int) * n_fail, cudaMemcpyDeviceToDevice, st));
    k_gather_i<<<(n_fail + 255) / 256, 256, 0, st>>>(d_qids, fail_copy, n_fail, sub_q);
    if (was_seeded) {
        int n2 = 0;
        if ((rc = fast_run(idx, sub_q, n_fail, k, false, sub_kth, sub_ids, sub_dis, sub_fail, &n2, st))) return rc;
        if (n2 > 0 && (rc = rerun_failed(idx, sub_q, k, false, sub_fail, n2, sub_kth, sub_ids, sub_dis, st)))
            return rc;
    } else {
        k_add_stat<<<1, 1, 0, st>>>(idx->d_stats + 4, (unsigned long long)n_fail);
        idx->keep_stats = true;
        rc = search_knn(idx, sub_q, n_fail, k, 0, sub_kth, sub_ids, sub_dis, st);
        idx->keep_stats = false;
        if (rc) return rc;
    }
    k_scatter_results<<<(n_fail + 255) / 256, 256, 0, st>>>(fail_copy, n_fail, k, sub_kth, sub_ids, sub_dis, d_kth,
                                                           d_ids, d_dists);
    GTS_CUDA_TRY(cudaGetLastError());
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    return GTS_OK;
}

int search_knn_fast(gts_index *idx, const int *d_qids, int qnum, int k, float *d_kth, int *d_ids,
                    float *d_dists, cudaStream_t st)
{
    int rc = fast_prepare(idx, st);
    if (rc) return rc;
    GTS_CUDA_TRY(cudaMemsetAsync(idx->d_status, 0, sizeof(int), st));
    GTS_CUDA_TRY(cudaMemsetAsync(idx->d_stats, 0, kStatsN * sizeof(unsigned long long), st));
    const bool seeded = idx->mlp_ready;
    DevVec keep;
    int *fail = nullptr;
    if ((rc = keep.alloc(&fail, qnum))) return rc;
    int n_fail = 0;
    if ((rc = fast_run(idx, d_qids, qnum, k, seeded, d_kth, d_ids, d_dists, fail, &n_fail, st))) return rc;
    idx->last_fast_overflow = n_fail;
    if (n_fail > 0) return rerun_failed(idx, d_qids, k, seeded, fail, n_fail, d_kth, d_ids, d_dists, st);
    return GTS_OK;
}

// The unseeded filter run with every buffer carved out of `scratch`
// (bytes long, 256-byte aligned): no device allocation on any path.  The
// filter records must already exist.  Queries the run could not answer
// (a full candidate list) go to the plain traversal, which uses only the
// index's own counters.
int search_knn_fast_fixed(gts_index *idx, const int *d_qids, int qnum, int k, float *d_kth, int *d_ids,
                          float *d_dists, unsigned char *scratch, size_t bytes, cudaStream_t st)
{
    if (!fast_supported(idx, k)) {
        gts_set_error("fixed-scratch kNN supports the L2 metric with dim <= %d and 1 <= k <= %d", kFMaxKp, kFMaxK);
        return GTS_ERR_INVALID;
    }
    if (!idx->fast_recs) {
        gts_set_error("the index has no filter records yet: one GTS_FORM_FAST kNN call on it must come first");
        return GTS_ERR_INVALID;
    }
    if (qnum <= 0) return GTS_OK;
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~(size_t)255; return o; };
    const size_t o_fail = take(sizeof(int) * qnum), o_subq = take(sizeof(int) * qnum);
    const size_t o_kth = take(sizeof(float) * qnum);
    const size_t o_ids = take(sizeof(int) * (size_t)qnum * k), o_dis = take(sizeof(float) * (size_t)qnum * k);
    if (off > bytes) {
        gts_set_error("fixed scratch of %zu bytes is too small for %d queries", bytes, qnum);
        return GTS_ERR_INVALID;
    }
    int *fail = (int *)(scratch + o_fail), *sub_q = (int *)(scratch + o_subq);
    float *sub_kth = (float *)(scratch + o_kth), *sub_dis = (float *)(scratch + o_dis);
    int *sub_ids = (int *)(scratch + o_ids);
    GTS_CUDA_TRY(cudaMemsetAsync(idx->d_status, 0, sizeof(int), st));
    GTS_CUDA_TRY(cudaMemsetAsync(idx->d_stats, 0, kStatsN * sizeof(unsigned long long), st));
    int n_fail = 0, rc;
    if ((rc = fast_run(idx, d_qids, qnum, k, false, d_kth, d_ids, d_dists, fail, &n_fail, st, scratch + off,
                       bytes - off)))
        return rc;
    idx->last_fast_overflow = n_fail;
    if (n_fail == 0) return GTS_OK;
    k_gather_i<<<(n_fail + 255) / 256, 256, 0, st>>>(d_qids, fail, n_fail, sub_q);
    k_add_stat<<<1, 1, 0, st>>>(idx->d_stats + 4, (unsigned long long)n_fail);
    idx->keep_stats = true;
    rc = search_knn(idx, sub_q, n_fail, k, 0, sub_kth, d_ids ? sub_ids : nullptr, d_dists ? sub_dis : nullptr, st);
    idx->keep_stats = false;
    if (rc) return rc;
    k_scatter_results<<<(n_fail + 255) / 256, 256, 0, st>>>(fail, n_fail, k, sub_kth, d_ids ? sub_ids : nullptr,
                                                           d_dists ? sub_dis : nullptr, d_kth, d_ids, d_dists);
    GTS_CUDA_TRY(cudaGetLastError());
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    return GTS_OK;
}

}  // namespace gts
