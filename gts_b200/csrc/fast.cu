// fast.cu -- exact L2 kNN with block pruning and a BF16 tensor-core filter
// ("fast" form).
//
// Same answers as searchIndexKnnV2 (search_v2.cuh:975-1228): the k-th
// distance of every query in the reference's F64 leaf arithmetic
// (search_v2.cuh:447-463) and the k nearest ids with ties broken by id.
// How it gets there is B200-specific:
//
//  * layout: objects are grouped into blocks of 128 consecutive tree
//    positions (the pivot tree keeps near objects near each other).  Each
//    block is stored once in HBM as a record that a single bulk copy drops
//    into shared memory in the operand layout tcgen05 reads (K-major,
//    128-byte swizzle): 128 rows of BF16 residuals r = o - c against the block
//    mean c, 3 rows holding c split into three BF16 parts, 13 zero rows, then
//    per object w = |o|^2 + 2 c.d and |d| (d = bf16(r) - r).  A block summary
//    (c in FP32, |c|^2, radius max |o - c|) sits beside the records.
//  * seeds: every query's k-th distance is bounded before any filtering by
//    the k-th smallest distance inside its own block (the query is a data
//    object), and by the learned radius model when one is trained.
//  * pruning: queries are sorted by tree position into tiles of 128; for
//    every (tile, block) pair the triangle inequality |q - c| - radius gives
//    a lower bound per query, and a block no query of the tile can reach
//    within its seed is never copied or multiplied (GTS's pivot pruning,
//    done with block balls instead of rings).
//  * filter: a persistent CTA per SM takes (tile, 64-block chunk) items.
//    One producer warp streams the tile's query operand and the needed block
//    records with bulk copies and issues a 128 x 144 x K MMA chain per block
//    into one of two TMEM accumulators; 4 x CG epilogue warps turn each TMEM
//    row into certified bounds lb <= d^2 <= ub for the 128 objects, keep the
//    k smallest ub (a running k-th bound shared through global memory) and
//    append every object with lb <= bound to the query's candidate list.
//    Producer and epilogue meet only on mbarriers.
//  * recheck: the final bound is the k-th smallest candidate ub; candidates
//    with lb <= bound get their reference-arithmetic distance and the k best
//    (distance, id) are the answer.
// No object whose reference distance can rank in the top k is ever dropped,
// so the result is exact.  Queries whose candidate list overflows, or whose
// learned seed turns out too small, are answered again.
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
constexpr int kFCand = 1024;          // candidate slots per query
constexpr int kFChunk = 64;           // blocks per work item (two mask words)
constexpr long long kFWait = 1ll << 24;   // bounded mbarrier polls

// Error-bound constants.  Relative error of a q.x product out of the MMA:
// the hi/lo split of q (2^-16), FP32 accumulation over 2 x 128 products
// (taken as 2^-23 per add for margin), the FP32 rounding of r (2^-24).
constexpr float kEpsC = 5e-5f;        // q.c rows:  >= 2^-16 + 2 * 256 * 2^-24
constexpr float kEpsR = 8e-5f;        // q.r rows:  >= 2^-16 + 2 * 256 * 2^-23 + 2^-23

// Record tail, after the BF16 operand rows (floats): w[128], dn[128], then
// |c|, the valid-object count (int), max |bf16(r)|, max |w|.
constexpr int kTailW = 0, kTailDn = 128, kTailC = 256, kTailCnt = 257, kTailRb = 258, kTailWb = 259;

struct FastShape {
    int kp, nk;              // padded dim, number of 64-wide K chunks
    uint32_t btile_bytes;    // nk * kFN * 128
    uint32_t rec_bytes;      // btile_bytes + 1024 (w, dn) + 16 (block scalars)
    uint32_t atile_bytes;    // nk * kFT * 128
    uint32_t arec_bytes;     // query tile: hi + lo operands + 128 x int4 lane info
};

__host__ __device__ inline FastShape fast_shape(int dim)
{
    FastShape s;
    s.kp = (dim + 63) / 64 * 64;
    s.nk = s.kp / 64;
    s.btile_bytes = (uint32_t)s.nk * kFN * 128u;
    s.rec_bytes = s.btile_bytes + 1024u + 16u;
    s.atile_bytes = (uint32_t)s.nk * kFT * 128u;
    s.arec_bytes = 2u * s.atile_bytes + 16u * kFT;
    return s;
}

// After the records: block summaries (centres [nb][kp], |c|^2 [nb], radius
// [nb]), then the filter's object order: ids[pos] (filter position -> id)
// and pos[id].
struct FastSummary {
    float *cen, *c2, *rad;
    int *ids, *pos;
};

static size_t fast_rec_region(const FastShape &fs, int nb) { return ((size_t)nb * fs.rec_bytes + 255) & ~(size_t)255; }
static size_t fast_bytes(const FastShape &fs, int nb, int n)
{
    return fast_rec_region(fs, nb) + sizeof(float) * (size_t)nb * (fs.kp + 2) + sizeof(int) * 2 * (size_t)n;
}
static FastSummary fast_summary(unsigned char *recs, const FastShape &fs, int nb, int n)
{
    float *cen = (float *)(recs + fast_rec_region(fs, nb));
    int *ids = (int *)(cen + (size_t)nb * (fs.kp + 2));
    return {cen, cen + (size_t)nb * fs.kp, cen + (size_t)nb * (fs.kp + 1), ids, ids + n};
}

__device__ __forceinline__ unsigned short f2bf(float x)
{
    return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
__device__ __forceinline__ float bf2f(unsigned short b) { return __bfloat162float(__ushort_as_bfloat16(b)); }

// ---------------------------------------------------------------- prep

// One CTA per block of 128 filter positions; thread t = object t of the block.
__global__ void __launch_bounds__(128) k_fast_prep(int n, int dim, const float *__restrict__ rows,
                                                   unsigned char *__restrict__ recs, FastShape fs, FastSummary bs)
{
    __shared__ float cen[kFMaxKp];
    __shared__ int bid[kFB];
    __shared__ unsigned int mx_rb, mx_w, mx_rad;
    const int b = blockIdx.x, t = threadIdx.x;
    const int base = b * kFB;
    const int cnt = min(kFB, n - base);
    unsigned char *rec = recs + (size_t)b * fs.rec_bytes;
    bid[t] = t < cnt ? bs.ids[base + t] : 0;
    __syncthreads();
    for (int j = t; j < fs.kp; j += 128) {
        double s = 0.0;
        if (j < dim)
            for (int i = 0; i < cnt; i++) s += (double)rows[(size_t)bid[i] * dim + j];
        cen[j] = j < dim ? (float)(s / cnt) : 0.f;
        bs.cen[(size_t)b * fs.kp + j] = cen[j];
    }
    if (t == 0) mx_rb = mx_w = mx_rad = 0u;
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
    float *tail = reinterpret_cast<float *>(rec + fs.btile_bytes);
    if (t == 0) {
        double c2 = 0.0;
        for (int j = 0; j < dim; j++) c2 += (double)cen[j] * cen[j];
        tail[kTailC] = __double2float_ru(sqrt(c2));
        reinterpret_cast<int *>(tail)[kTailCnt] = cnt;
        bs.c2[b] = (float)c2;
    }
    // residual rows r = o - c (FP32), stored as BF16; d = bf16(r) - r exactly
    // (in FP64).  c.d is known per object, so the filter corrects for it and
    // only (q - c).d is left to the error bound.
    const bool valid = t < cnt;
    const float *row = rows + (size_t)bid[t] * dim;
    double o2 = 0.0, cd = 0.0, d2 = 0.0, rb2 = 0.0, oc2 = 0.0;
    for (int j = 0; j < fs.kp; j++) {
        float r = 0.f;
        if (valid && j < dim) {
            float o = row[j];
            o2 += (double)o * o;
            r = o - cen[j];
            const double e = (double)o - (double)cen[j];
            oc2 += e * e;
        }
        const unsigned short rb = f2bf(r);
        const double rbd = (double)bf2f(rb), d = rbd - (double)r;
        cd += (double)cen[j] * d;
        d2 += d * d;
        rb2 += rbd * rbd;
        *reinterpret_cast<unsigned short *>(rec + sw128_offset(t, j, kFN)) = rb;
    }
    const double w = o2 + 2.0 * cd;
    tail[kTailW + t] = valid ? (float)w : INFINITY;
    tail[kTailDn + t] = valid ? __double2float_ru(sqrt(d2) * (1.0 + 1e-12)) : 0.f;
    // block maxima (non-negative floats order like their bit patterns)
    if (valid) {
        atomicMax(&mx_rb, __float_as_uint(__double2float_ru(sqrt(rb2) * (1.0 + 1e-12))));
        atomicMax(&mx_w, __float_as_uint(__double2float_ru(fabs(w))));
        atomicMax(&mx_rad, __float_as_uint(__double2float_ru(sqrt(oc2) * (1.0 + 1e-12))));
    }
    __syncthreads();
    if (t == 0) {
        tail[kTailRb] = __uint_as_float(mx_rb);
        tail[kTailWb] = __uint_as_float(mx_w);
        bs.rad[b] = __uint_as_float(mx_rad);
    }
}

// ---------------------------------------------------------------- object order

// The filter's own object order: a ball tree cut into 128-object blocks.
// Every level splits each segment of more than 128 objects at a multiple of
// 128 after sorting it by the projection on the line through two far-apart
// members (p1 = farthest from the segment's first object, p2 = farthest from
// p1), so blocks come out as tight balls and the block bound prunes.

// Squared FP32 distance between two rows, one warp, lanes over dimensions.
__device__ __forceinline__ float warp_d2(const float *__restrict__ a, const float *__restrict__ b, int dim, int lane)
{
    float s = 0.f;
    for (int j = lane; j < dim; j += 32) {
        const float e = a[j] - b[j];
        s = fmaf(e, e, s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

__global__ void k_ord_init(int n, int *perm, int *sid, int *seg_l, int *seg_r)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        perm[i] = i;
        sid[i] = 0;
    }
    if (i == 0) {
        seg_l[0] = 0;
        seg_r[0] = n;
    }
}

// One warp per position: distance to the segment's reference object; the
// farthest position of every segment that still splits (packed max).
__global__ void k_ord_far(const float *__restrict__ rows, int dim, int n, const int *__restrict__ perm,
                          const int *__restrict__ sid, const int *__restrict__ seg_l, const int *__restrict__ seg_r,
                          const unsigned long long *__restrict__ ref, unsigned long long *__restrict__ best)
{
    const int pos = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (pos >= n) return;
    const int s = sid[pos];
    if (seg_r[s] - seg_l[s] <= kFB) return;
    const int rp = ref ? (int)(ref[s] & 0xffffffffu) : seg_l[s];
    const float d = warp_d2(rows + (size_t)perm[pos] * dim, rows + (size_t)perm[rp] * dim, dim, lane);
    if (lane == 0) atomicMax(&best[s], ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)pos);
}

// Sort key of every position: segment id, then |x - p1|^2 - |x - p2|^2
// (monotone in the projection on p2 - p1) for segments that split.
__global__ void k_ord_key(const float *__restrict__ rows, int dim, int n, const int *__restrict__ perm,
                          const int *__restrict__ sid, const int *__restrict__ seg_l, const int *__restrict__ seg_r,
                          const unsigned long long *__restrict__ p1, const unsigned long long *__restrict__ p2,
                          unsigned long long *__restrict__ keys)
{
    const int pos = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (pos >= n) return;
    const int s = sid[pos];
    float key = 0.f;
    if (seg_r[s] - seg_l[s] > kFB) {
        const float *x = rows + (size_t)perm[pos] * dim;
        const float a = warp_d2(x, rows + (size_t)perm[(int)(p1[s] & 0xffffffffu)] * dim, dim, lane);
        const float b = warp_d2(x, rows + (size_t)perm[(int)(p2[s] & 0xffffffffu)] * dim, dim, lane);
        key = a - b;
    }
    if (lane == 0) {
        uint32_t u = __float_as_uint(key);
        u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);   // order-preserving bits
        keys[pos] = ((unsigned long long)s << 32) | u;
    }
}

// Children of every segment: a segment of nb > 1 blocks keeps ceil(nb / 2)
// blocks on the left; others pass through as child 2s.
__global__ void k_ord_segs(int nseg, const int *__restrict__ seg_l, const int *__restrict__ seg_r,
                           int *__restrict__ nl, int *__restrict__ nr)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const int l = seg_l[s], r = seg_r[s];
    const int nbk = (r - l + kFB - 1) / kFB;
    const int m = nbk > 1 ? l + (nbk + 1) / 2 * kFB : r;
    nl[2 * s] = l;
    nr[2 * s] = m;
    nl[2 * s + 1] = m;
    nr[2 * s + 1] = r;
}

__global__ void k_ord_relabel(int n, int *__restrict__ sid, const int *__restrict__ nr)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const int s = sid[pos];
    sid[pos] = pos < nr[2 * s] ? 2 * s : 2 * s + 1;
}

__global__ void k_ord_finish(int n, const int *__restrict__ perm, int *__restrict__ ids, int *__restrict__ pos_of)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    ids[pos] = perm[pos];
    pos_of[perm[pos]] = pos;
}

// ---------------------------------------------------------------- per call

// One CTA per tile: the A operand of the tile's 128 queries (sorted by tree
// position), split into BF16 hi + lo, in the swizzled layout, and per lane
// (query index, |q|^2, |q|).  A tile record is one bulk copy.
__global__ void __launch_bounds__(128) k_fast_arec(const float *__restrict__ rows, const int *__restrict__ qids,
                                                   const int *__restrict__ order, int qnum, int dim, FastShape fs,
                                                   unsigned char *__restrict__ arec)
{
    const int tile = blockIdx.x, lq = threadIdx.x;
    unsigned char *A_hi = arec + (size_t)tile * fs.arec_bytes, *A_lo = A_hi + fs.atile_bytes;
    int4 *info = reinterpret_cast<int4 *>(A_lo + fs.atile_bytes);
    const int slot = tile * kFT + lq;
    const int qi = slot < qnum ? order[slot] : -1;
    const float *row = qi >= 0 ? rows + (size_t)qids[qi] * dim : nullptr;
    double acc = 0.0;
    for (int j0 = 0; j0 < fs.kp; j0 += 8) {
        unsigned short hi[8], lo[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            int j = j0 + u;
            float x = (row && j < dim) ? row[j] : 0.f;
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
    info[lq] = make_int4(qi, __float_as_int((float)acc), __float_as_int((float)sqrt(acc)), 0);
}

// One CTA per query: the k-th smallest FP32 squared distance inside the
// query's own block (the query is one of its objects), widened past every
// rounding difference to the reference's value, lowers the query's bound.
__global__ void __launch_bounds__(128) k_fast_seed(const float *__restrict__ rows, const int *__restrict__ qids,
                                                   FastSummary bs, int num, int dim, int k, int *__restrict__ r2_bits)
{
    __shared__ float qs[kFMaxKp];
    __shared__ float v[kFB];
    const int q = blockIdx.x, t = threadIdx.x;
    const int qid = qids[q];
    const int base = bs.pos[qid] / kFB * kFB;
    const int cnt = min(kFB, num - base);
    if (cnt < k) return;
    for (int j = t; j < dim; j += 128) qs[j] = rows[(size_t)qid * dim + j];
    __syncthreads();
    float s = FLT_MAX;
    if (t < cnt) {
        const float *o = rows + (size_t)bs.ids[base + t] * dim;
        s = 0.f;
        for (int j = 0; j < dim; j++) {
            const float e = o[j] - qs[j];
            s = fmaf(e, e, s);
        }
    }
    v[t] = s;
    __syncthreads();
    for (int size = 2; size <= kFB; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            if (t < kFB / 2) {
                int lo = 2 * t - (t & (stride - 1)), hi = lo + stride;
                bool up = (lo & size) == 0;
                float x = v[lo], y = v[hi];
                if ((x > y) == up) { v[lo] = y; v[hi] = x; }
            }
            __syncthreads();
        }
    }
    // FP32 sum of 128 non-negative terms: relative error < 2^-17 against the
    // reference's FP64 sum of the same FP32 differences
    if (t == 0) atomicMin(&r2_bits[q], __float_as_int(v[k - 1] * (1.f + 3e-5f)));
}

// Block pruning.  CTA (tile, y) loads the tile's 128 query rows once and
// walks chunks of 64 blocks; each of 256 threads computes 8 queries x 4
// blocks of FP32 q.c, then per pair a certified lower bound
//   |q - o| >= |q - c|_lo - radius.
// A block is needed when some query of the tile can reach it within its
// bound; each chunk with a needed block becomes one filter work item.
constexpr int kNeedGridY = 8;

__global__ void __launch_bounds__(256) k_fast_need(const float *__restrict__ rows, const int *__restrict__ qids,
                                                   const unsigned char *__restrict__ arec, FastShape fs, int dim,
                                                   int nb, FastSummary bs, const int *__restrict__ r2_bits,
                                                   uint32_t *__restrict__ mask, int nbw, int nchunk,
                                                   int *__restrict__ items, int *__restrict__ n_items,
                                                   unsigned long long *stats)
{
    extern __shared__ __align__(16) float nsm[];
    const int kp = fs.kp;
    float *Qs = nsm;               // [kp][128]
    float *Cs = Qs + kp * kFT;     // [kp][64]
    __shared__ float q2s[kFT], qns[kFT], seeds[kFT];
    __shared__ float c2s[kFChunk], cns[kFChunk], rads[kFChunk];
    __shared__ unsigned int flags[2];
    const int tile = blockIdx.x, t = threadIdx.x;
    const int4 *info = reinterpret_cast<const int4 *>(arec + (size_t)tile * fs.arec_bytes + 2 * fs.atile_bytes);
    if (t < kFT) {
        const int4 in = info[t];
        q2s[t] = __int_as_float(in.y);
        qns[t] = __int_as_float(in.z);
        seeds[t] = in.x >= 0 ? __int_as_float(r2_bits[in.x]) : -1.f;
    }
    for (int i = t; i < kp * kFT; i += 256) {
        const int j = i / kFT, l = i % kFT;
        const int qi = info[l].x;
        Qs[i] = (qi >= 0 && j < dim) ? rows[(size_t)qids[qi] * dim + j] : 0.f;
    }
    const int tq = t & 15, tb = t >> 4;
    unsigned long long tested = 0;
    for (int chunk = blockIdx.y; chunk < nchunk; chunk += gridDim.y) {
        const int b0 = chunk * kFChunk;
        __syncthreads();   // previous chunk's Cs / flags consumed
        for (int i = t; i < kp * kFChunk; i += 256) {
            const int j = i / kFChunk, bb = i % kFChunk;
            Cs[i] = (b0 + bb < nb) ? bs.cen[(size_t)(b0 + bb) * kp + j] : 0.f;
        }
        if (t < kFChunk) {
            const bool ok = b0 + t < nb;
            c2s[t] = ok ? bs.c2[b0 + t] : 0.f;
            cns[t] = ok ? sqrtf(bs.c2[b0 + t]) * 1.000001f : 0.f;
            rads[t] = ok ? bs.rad[b0 + t] : -1.f;
        }
        if (t < 2) flags[t] = 0u;
        __syncthreads();
        float acc[8][4];
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
            for (int c = 0; c < 4; c++) acc[i][c] = 0.f;
        for (int j = 0; j < kp; j++) {
            const float4 qa = *reinterpret_cast<const float4 *>(Qs + j * kFT + tq * 8);
            const float4 qb = *reinterpret_cast<const float4 *>(Qs + j * kFT + tq * 8 + 4);
            const float4 cc = *reinterpret_cast<const float4 *>(Cs + j * kFChunk + tb * 4);
            const float qv[8] = {qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z, qb.w};
            const float cv[4] = {cc.x, cc.y, cc.z, cc.w};
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[i][c] = fmaf(qv[i], cv[c], acc[i][c]);
        }
        // FP32 dot of kp products: error <= kp 2^-23 |q||c|; the three-term
        // sum adds <= 4e-7 (|q|^2 + |c|^2)
        const float gam = 2.f * (float)kp * 1.2e-7f;
        unsigned int need = 0;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int bb = tb * 4 + c;
            const float rad = rads[bb];
            bool nd = false;
            if (rad >= 0.f) {
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int l = tq * 8 + i;
                    const float sd = seeds[l];
                    if (sd < 0.f) continue;
                    const float q2 = q2s[l], c2 = c2s[bb];
                    const float e = gam * qns[l] * cns[bb] + 4e-7f * (q2 + c2) + 1e-30f;
                    const float d2lo = q2 - 2.f * acc[i][c] + c2 - e;
                    const float lo = sqrtf(fmaxf(d2lo, 0.f)) * 0.999999f - rad;
                    nd |= lo <= 0.f || lo * lo * 0.999999f <= sd;
                }
            }
            need |= (nd ? 1u : 0u) << c;
        }
        // the 16 threads of a half-warp share their 4 blocks
        need |= __shfl_xor_sync(0xffffffffu, need, 1);
        need |= __shfl_xor_sync(0xffffffffu, need, 2);
        need |= __shfl_xor_sync(0xffffffffu, need, 4);
        need |= __shfl_xor_sync(0xffffffffu, need, 8);
        if (tq == 0 && need) atomicOr(&flags[(tb * 4) >> 5], need << ((tb * 4) & 31));
        __syncthreads();
        if (t == 0) {
            const int w0 = 2 * chunk;
            mask[(size_t)tile * nbw + w0] = flags[0];
            if (w0 + 1 < nbw) mask[(size_t)tile * nbw + w0 + 1] = flags[1];
            if (flags[0] | flags[1]) items[atomicAdd(n_items, 1)] = tile * nchunk + chunk;
            tested += (unsigned long long)min(kFChunk, nb - b0);
        }
    }
    if (t == 0 && stats) atomicAdd(&stats[7], tested);
}

// ---------------------------------------------------------------- filter

struct FastTileArgs {
    const unsigned char *recs;   // block records
    const unsigned char *arec;   // query tile records
    const uint32_t *mask;        // [ntiles][nbw] needed blocks
    const int *items;            // tile * nchunk + chunk, for chunks with a needed block
    const int *n_items;
    int nbw, nchunk, k;
    FastShape fs;
    int *cand_pos;               // [qnum][kFCand] tree positions
    float *cand_lb, *cand_ub;    // [qnum][kFCand] bounds on d^2
    int *cand_cnt;               // [qnum]
    int *r2_bits;                // [qnum] bound on the k-th d^2 (float bits), shared by all threads
    int *item_counter;           // persistent-CTA work queue
    int *status;
    unsigned long long *stats;
};

constexpr int kFS = 3;   // block stages

struct __align__(8) FastCtl {
    uint64_t full[kFS];    // block copy landed
    uint64_t efree[kFS];   // epilogue of the block in this stage done (one arrive per epilogue warp)
    uint64_t mmad[2];      // MMA chain into TMEM accumulator d done
    uint64_t afull;        // query tile copy landed
    uint32_t tmem;
    int item;
    int err;
};

// Persistent filter kernel, one CTA per SM, 4 x CG epilogue warps + one
// producer warp.  CG column groups: warps w, w+4, ... share TMEM lanes
// 32*(w%4)..+31 (the same 32 queries) and split the 128 object columns.
//
// Per item (a tile and a chunk of 64 blocks, of which nblk are needed), with
// gi counting blocks over the CTA's life (barrier phases follow it):
//   producer:  copy A; copy blocks 0..2 into stages gi%3; for each block:
//              wait its copy, wait the epilogue of block gi-2 (frees TMEM
//              accumulator gi%2 and stage (gi-2)%3 = (gi+1)%3), MMA chain into
//              accumulator gi%2, commit, copy block gi+1 into the freed stage.
//   epilogue:  wait the MMA of block gi, bound the 128 x 128 pairs, arrive
//              on efree[gi%3].
// The CTA synchronises only between items.
template <int CG>
__global__ void __launch_bounds__(128 * CG + 32, 1) k_fast_tile(FastTileArgs a)
{
    constexpr int NT = 128 * CG;   // epilogue threads
    constexpr int NEW = NT / 32;   // epilogue warps
    constexpr int CW = 128 / CG;   // object columns per thread
    extern __shared__ __align__(1024) unsigned char fsm[];
    unsigned char *base = (unsigned char *)(((uintptr_t)fsm + 1023) & ~(uintptr_t)1023);
    const FastShape fs = a.fs;
    const uint32_t arec_pad = (fs.arec_bytes + 1023u) & ~1023u;
    const uint32_t rec_pad = (fs.rec_bytes + 1023u) & ~1023u;
    unsigned char *B0 = base + arec_pad;
    float *heap = reinterpret_cast<float *>(B0 + kFS * rec_pad);
    FastCtl &ctl = *reinterpret_cast<FastCtl *>(heap + NT * a.k);

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const bool producer = warp == NEW;
    const int lq = t & 127, g = t >> 7;
    const int k = a.k;

    if (t == 0) {
        for (int s = 0; s < kFS; s++) {
            mbar_init(&ctl.full[s], 1);
            mbar_init(&ctl.efree[s], NEW);
        }
        for (int s = 0; s < 2; s++) mbar_init(&ctl.mmad[s], 1);
        mbar_init(&ctl.afull, 1);
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
    const uint32_t a_hi_s = smem_u32(base), a_lo_s = smem_u32(base + fs.atile_bytes);
    long long gblk = 0;   // blocks this CTA has run through the pipeline
    // producer bookkeeping (lane 0 of the producer warp): copies issued /
    // waited per stage, A copies issued / waited, MMA commits per accumulator
    int c_iss[kFS] = {0, 0, 0}, c_wait[kFS] = {0, 0, 0}, a_iss = 0, a_wait = 0, m_iss[2] = {0, 0};
    unsigned long long blocks_done = 0, appended = 0;

    for (;;) {
        if (t == 0) {
            const int it = atomicAdd(a.item_counter, 1);
            ctl.item = it < *a.n_items ? a.items[it] : -1;
        }
        __syncthreads();
        const int item = ctl.item;
        if (item < 0 || ctl.err) break;
        const int tile = item / a.nchunk, chunk = item % a.nchunk;
        const uint32_t *mw = a.mask + (size_t)tile * a.nbw + 2 * chunk;
        const uint64_t M0 = (uint64_t)mw[0] | ((2 * chunk + 1 < a.nbw) ? (uint64_t)mw[1] << 32 : 0ull);
        const int nblk = __popcll(M0);

        if (producer) {
            if (lane == 0) {
                uint64_t Mp = M0;
                auto issue_copy = [&](long long gi) {
                    const int s = (int)(gi % kFS);
                    const int blk = chunk * kFChunk + __ffsll((long long)Mp) - 1;
                    Mp &= Mp - 1;
                    mbar_arrive_expect_tx(&ctl.full[s], fs.rec_bytes);
                    bulk_g2s(B0 + (size_t)s * rec_pad, a.recs + (size_t)blk * fs.rec_bytes, fs.rec_bytes,
                             &ctl.full[s]);
                    c_iss[s]++;
                };
                mbar_arrive_expect_tx(&ctl.afull, fs.arec_bytes);
                bulk_g2s(base, a.arec + (size_t)tile * fs.arec_bytes, fs.arec_bytes, &ctl.afull);
                a_iss++;
                for (int j = 0; j < kFS && j < nblk; j++) issue_copy(gblk + j);
                int err = 0;
                if (!mbar_wait(&ctl.afull, (uint32_t)(a_wait & 1), kFWait)) err = 1;
                else a_wait++;
                for (int j = 0; j < nblk && !err; j++) {
                    const long long gi = gblk + j;
                    const int s = (int)(gi % kFS), d = (int)(gi & 1);
                    if (!mbar_wait(&ctl.full[s], (uint32_t)((gi / kFS) & 1), kFWait)) { err = 2; break; }
                    c_wait[s]++;
                    if (j >= 2) {
                        const long long gp = gi - 2;
                        if (!mbar_wait(&ctl.efree[gp % kFS], (uint32_t)((gp / kFS) & 1), kFWait)) {
                            err = 3;
                            break;
                        }
                    }
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
                        mma_bf16(dt, smem_desc_sw128(a_lo_s + off, 1024), smem_desc_sw128(b_s + boff, 1024), idesc,
                                 1u);
                    }
                    mma_commit(&ctl.mmad[d]);
                    m_iss[d]++;
                    if (j >= 2 && j + 1 < nblk) issue_copy(gi + 1);
                }
                if (err) atomicMax(&ctl.err, err);
                blocks_done += nblk;
            }
            __syncwarp();
        } else {
            // ---- epilogue: one query lane, CW object columns
            const int4 inf =
                reinterpret_cast<const int4 *>(a.arec + (size_t)tile * fs.arec_bytes + 2 * fs.atile_bytes)[lq];
            const int qi = inf.x;
            const float q2 = __int_as_float(inf.y), qn = __int_as_float(inf.z);
            const float cr = 2.f * kEpsR * qn;
            for (int i = 0; i < k; i++) heap[i * NT + t] = FLT_MAX;
            const float seed = qi >= 0 ? __int_as_float(a.r2_bits[qi]) : FLT_MAX;
            float R2 = seed, pub = seed;   // bound in use, last bound published
            float hmx = FLT_MAX;           // largest of this thread's k kept upper bounds
            int hidx = 0;
            uint64_t Me = M0;
            const uint32_t trow = (uint32_t)(warp & 3) * 32u << 16;
            for (int j = 0; j < nblk; j++) {
                const long long gi = gblk + j;
                const int s = (int)(gi % kFS), d = (int)(gi & 1);
                const int blk = chunk * kFChunk + __ffsll((long long)Me) - 1;
                Me &= Me - 1;
                // the query's bound as published by every thread working on it
                float shr = FLT_MAX;
                if (qi >= 0) shr = __int_as_float(*(volatile const int *)(a.r2_bits + qi));
                if (!mbar_wait(&ctl.mmad[d], (uint32_t)((gi >> 1) & 1), kFWait)) {
                    atomicMax(&ctl.err, 4);
                    break;
                }
                tc_fence_after();
                mbar_wait(&ctl.full[s], (uint32_t)((gi / kFS) & 1), kFWait);   // record tail visible here
                R2 = fminf(R2, shr);
                const unsigned char *Bs = B0 + (size_t)s * rec_pad;
                const float *tail = reinterpret_cast<const float *>(Bs + fs.btile_bytes);
                const float *wv = tail + kTailW, *dn = tail + kTailDn;
                const float cn = tail[kTailC], rb = tail[kTailRb], wb = tail[kTailWb];
                const uint32_t taddr = tmem + trow + (uint32_t)(d * 256);
                float v[16];
                tmem_ld16(taddr + 128, v);
                const float qc = v[0] + v[1] + v[2];
                // d^2 = |q|^2 - 2 q.c + w - 2 v - 2 (q - c).d + (rounding), so with
                //   ec >= 2 |q.c error|                       (centre rows)
                //   eb =  ec + 2e-6 |q|^2 + 2 kEpsR |q| max|bf16 r| + 2e-6 max|w|
                //   A  >= 2 |q - c|                           (from the centre product)
                // every object has |d^2 - (T + w - 2 v)| <= A |d| + eb,  T = |q|^2 - 2 q.c
                const float ec = 2.f * kEpsC * qn * cn + 1e-6f;
                const float c2 = cn * cn;
                const float qmc2 = q2 - 2.f * qc + c2 + ec + 4e-6f * (q2 + c2);
                const float A = 2.000004f * sqrtf(fmaxf(qmc2, 0.f)) + 2e-6f * cn;
                const float eb = ec + 2e-6f * q2 + cr * rb + 2e-6f * wb;
                const float T = q2 - 2.f * qc - eb;
#pragma unroll 1
                for (int c = g * CW; c < (g + 1) * CW; c += 16) {
                    tmem_ld16(taddr + (uint32_t)c, v);
                    if (qi < 0) continue;
#pragma unroll
                    for (int u = 0; u < 16; u++) {
                        const int jj = c + u;
                        const float dj = dn[jj];
                        // padding objects have w = +inf and never pass
                        const float lb = fmaf(-2.f, v[u], fmaf(-A, dj, T + wv[jj]));
                        if (lb <= R2) {
                            const float ub = lb + 2.f * fmaf(A, dj, eb);
                            const int sl = atomicAdd(&a.cand_cnt[qi], 1);
                            if (sl < kFCand) {
                                a.cand_pos[(size_t)qi * kFCand + sl] = blk * kFB + jj;
                                a.cand_lb[(size_t)qi * kFCand + sl] = lb;
                                a.cand_ub[(size_t)qi * kFCand + sl] = ub;
                            }
                            appended++;
                            if (ub < R2) {   // replace the largest of the k kept bounds
                                heap[hidx * NT + t] = ub;
                                float mx = -1.f;
                                for (int h = 0; h < k; h++) {
                                    const float hv = heap[h * NT + t];
                                    if (hv > mx) { mx = hv; hidx = h; }
                                }
                                hmx = mx;
                                R2 = fminf(R2, mx);
                            }
                        }
                    }
                }
                // k distinct objects' upper bounds bound the query's k-th d^2
                if (qi >= 0 && hmx < pub) {
                    atomicMin(a.r2_bits + qi, __float_as_int(fmaxf(hmx, 0.f)));
                    pub = hmx;
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&ctl.efree[s]);
            }
        }
        gblk += nblk;
        tc_fence_before();
        __syncthreads();   // item done: every MMA consumed, stages and A free
        tc_fence_after();
    }
    if (producer && lane == 0 && ctl.err) {
        // let copies and MMAs still in flight finish before the CTA leaves (bounded)
        for (int s = 0; s < kFS; s++)
            if (c_wait[s] < c_iss[s]) mbar_wait(&ctl.full[s], (uint32_t)((c_iss[s] - 1) & 1), kFWait);
        if (a_wait < a_iss) mbar_wait(&ctl.afull, (uint32_t)((a_iss - 1) & 1), kFWait);
        for (int d = 0; d < 2; d++)
            if (m_iss[d] > 0) mbar_wait(&ctl.mmad[d], (uint32_t)((m_iss[d] - 1) & 1), kFWait);
    }
    if (a.stats && appended) atomicAdd(&a.stats[5], appended);
    if (a.stats && producer && lane == 0 && blocks_done) {
        atomicAdd(&a.stats[0], blocks_done);
        atomicAdd(&a.stats[1], (unsigned long long)fs.rec_bytes * blocks_done);
    }
    if (t == 0 && ctl.err) atomicMax(a.status, 16 + ctl.err);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 512);
}

// ---------------------------------------------------------------- finalize

constexpr int kFinSort = kFCand;

// One CTA per query.  The bound drops to the k-th smallest candidate upper
// bound (the candidates are distinct objects); every candidate whose lower
// bound is within it gets its reference-arithmetic distance; top k by
// (distance, id).  Queries that cannot be answered from their list (it
// overflowed, or fewer than k exact values lie inside the bound because a
// learned seed was too small) are listed in overflow.
__global__ void __launch_bounds__(128) k_fast_final(const float *__restrict__ rows, int dim, int num,
                                                    const int *__restrict__ ids_of_pos,
                                                    const int *__restrict__ qids, int qnum, int k,
                                                    int infi_dis, const int *__restrict__ cand_pos,
                                                    const float *__restrict__ cand_lb,
                                                    const float *__restrict__ cand_ub,
                                                    const int *__restrict__ cand_cnt,
                                                    const int *__restrict__ r2_bits, float *kth, int *ids,
                                                    float *dists, int *overflow, int *n_overflow,
                                                    unsigned long long *stats)
{
    __shared__ double cd[kFinSort];
    __shared__ int cid[kFinSort];
    __shared__ float ubs[kFinSort];
    __shared__ int ns;
    const int q = blockIdx.x, t = threadIdx.x;
    const int qid = qids[q];
    const int cnt = cand_cnt[q];
    if (cnt > kFCand) {
        if (t == 0) overflow[atomicAdd(n_overflow, 1)] = q;
        return;
    }
    float R2 = __int_as_float(r2_bits[q]);
    if (cnt >= k) {
        int p2 = 1;
        while (p2 < cnt) p2 <<= 1;
        for (int i = t; i < p2; i += 128) ubs[i] = i < cnt ? cand_ub[(size_t)q * kFCand + i] : FLT_MAX;
        __syncthreads();
        for (int size = 2; size <= p2; size <<= 1) {
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int i = t; i < p2 / 2; i += 128) {
                    int lo = 2 * i - (i & (stride - 1)), hi = lo + stride;
                    bool up = (lo & size) == 0;
                    float x = ubs[lo], y = ubs[hi];
                    if ((x > y) == up) { ubs[lo] = y; ubs[hi] = x; }
                }
                __syncthreads();
            }
        }
        R2 = fminf(R2, ubs[k - 1]);
    }
    if (t == 0) ns = 0;
    __syncthreads();
    const float *qrow = rows + (size_t)qid * dim;
    for (int i = t; i < cnt; i += 128) {
        if (cand_lb[(size_t)q * kFCand + i] > R2) continue;
        int pos = cand_pos[(size_t)q * kFCand + i];
        if (pos < 0 || pos >= num) continue;
        int id = ids_of_pos[pos];
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
    if (t == 0) {
        // every object whose d^2 is within the bound is a candidate, and the
        // reference value differs from d^2 by < 1e-6 relative: the answer is
        // exact once k candidates have reference values inside R2 (1 - 1e-6)
        const double lim = (double)R2 * (1.0 - 1e-6);
        int within = 0;
        for (int i = 0; i < n && i < k; i++) within += cd[i] * cd[i] <= lim;
        if (within < k && within < num) {
            overflow[atomicAdd(n_overflow, 1)] = q;
            return;
        }
        kth[q] = n >= k ? (float)cd[k - 1] : (float)infi_dis;
        for (int j = 0; j < k; j++) {
            if (ids) ids[(size_t)q * k + j] = j < n ? cid[j] : -1;
            if (dists) dists[(size_t)q * k + j] = j < n ? (float)cd[j] : (float)infi_dis;
        }
    }
}

__global__ void k_fast_keys(const int *qids, int qnum, const int *pos_of, int *keys, int *vals)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < qnum) {
        keys[i] = pos_of[qids[i]];
        vals[i] = i;
    }
}

__global__ void k_fast_init(int qnum, int *cand_cnt, int *r2_bits, const int *carry)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < qnum) {
        cand_cnt[i] = 0;
        r2_bits[i] = carry ? carry[i] : __float_as_int(FLT_MAX);
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

// Column groups per query lane: as many epilogue warps as the bound heaps
// (threads x k floats, at most 32 KB of shared memory) allow.
static int fast_cg(int k) { return k <= 16 ? 4 : (k <= 32 ? 2 : 1); }

template <int CG>
static int launch_fast_tile_cg(const FastTileArgs &a, int grid, cudaStream_t st)
{
    const uint32_t arec_pad = (a.fs.arec_bytes + 1023u) & ~1023u;
    const uint32_t rec_pad = (a.fs.rec_bytes + 1023u) & ~1023u;
    size_t smem = 1024 + (size_t)arec_pad + kFS * (size_t)rec_pad + sizeof(float) * 128 * CG * (size_t)a.k +
                  sizeof(FastCtl) + 64;
    GTS_CUDA_TRY(cudaFuncSetAttribute(k_fast_tile<CG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_fast_tile<CG><<<grid, 128 * CG + 32, smem, st>>>(a);
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

static int launch_fast_tile(const FastTileArgs &a, int grid, cudaStream_t st)
{
    switch (fast_cg(a.k)) {
    case 4: return launch_fast_tile_cg<4>(a, grid, st);
    case 2: return launch_fast_tile_cg<2>(a, grid, st);
    default: return launch_fast_tile_cg<1>(a, grid, st);
    }
}

bool fast_supported(const gts_index *idx, int k)
{
    return idx->metric == kL2 && idx->dim <= kFMaxKp && k >= 1 && k <= kFMaxK && idx->num >= 1;
}

// The filter order (ball tree, see k_ord_*) into bs.ids / bs.pos; scratch
// from the index's growable scratch.
static int fast_order(gts_index *idx, const FastSummary &bs, int nb, cudaStream_t st)
{
    const int n = idx->num, dim = idx->dim;
    int L = 0;
    while ((1 << L) < nb) L++;
    const int smax = 1 << L;
    size_t cub_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (unsigned long long *)nullptr, (unsigned long long *)nullptr,
                                    (int *)nullptr, (int *)nullptr, n, 0, 64, st);
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~(size_t)255; return o; };
    const size_t o_perm = take(sizeof(int) * n), o_perm2 = take(sizeof(int) * n), o_sid = take(sizeof(int) * n);
    const size_t o_keys = take(8 * (size_t)n), o_keys2 = take(8 * (size_t)n);
    const size_t o_sl = take(sizeof(int) * smax), o_sr = take(sizeof(int) * smax);
    const size_t o_nl = take(sizeof(int) * smax), o_nr = take(sizeof(int) * smax);
    const size_t o_p1 = take(8 * (size_t)smax), o_p2 = take(8 * (size_t)smax);
    const size_t o_cub = take(cub_bytes);
    int rc;
    if ((rc = ensure_scratch(idx, off))) return rc;
    unsigned char *S = (unsigned char *)idx->scratch;
    int *perm = (int *)(S + o_perm), *perm2 = (int *)(S + o_perm2), *sid = (int *)(S + o_sid);
    unsigned long long *keys = (unsigned long long *)(S + o_keys), *keys2 = (unsigned long long *)(S + o_keys2);
    int *sl = (int *)(S + o_sl), *sr = (int *)(S + o_sr), *nl = (int *)(S + o_nl), *nr = (int *)(S + o_nr);
    unsigned long long *p1 = (unsigned long long *)(S + o_p1), *p2 = (unsigned long long *)(S + o_p2);
    const int wblocks = (int)(((size_t)n * 32 + 255) / 256);
    k_ord_init<<<(n + 255) / 256, 256, 0, st>>>(n, perm, sid, sl, sr);
    int nseg = 1;
    for (int lev = 0; lev < L; lev++) {
        GTS_CUDA_TRY(cudaMemsetAsync(p1, 0, 8 * (size_t)nseg, st));
        GTS_CUDA_TRY(cudaMemsetAsync(p2, 0, 8 * (size_t)nseg, st));
        k_ord_far<<<wblocks, 256, 0, st>>>(idx->rows, dim, n, perm, sid, sl, sr, nullptr, p1);
        k_ord_far<<<wblocks, 256, 0, st>>>(idx->rows, dim, n, perm, sid, sl, sr, p1, p2);
        k_ord_key<<<wblocks, 256, 0, st>>>(idx->rows, dim, n, perm, sid, sl, sr, p1, p2, keys);
        size_t cb = cub_bytes;
        GTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(S + o_cub, cb, keys, keys2, perm, perm2, n, 0, 32 + lev + 1, st));
        std::swap(perm, perm2);
        k_ord_segs<<<(nseg + 255) / 256, 256, 0, st>>>(nseg, sl, sr, nl, nr);
        k_ord_relabel<<<(n + 255) / 256, 256, 0, st>>>(n, sid, nr);
        std::swap(sl, nl);
        std::swap(sr, nr);
        nseg *= 2;
    }
    k_ord_finish<<<(n + 255) / 256, 256, 0, st>>>(n, perm, bs.ids, bs.pos);
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

static int fast_prepare(gts_index *idx, cudaStream_t st)
{
    if (idx->fast_recs) return GTS_OK;
    FastShape fs = fast_shape(idx->dim);
    int nb = (idx->num + kFB - 1) / kFB;
    size_t bytes = fast_bytes(fs, nb, idx->num);
    unsigned char *recs = nullptr;
    int rc = dev_alloc(&recs, bytes, nullptr);
    if (rc) return rc;
    GTS_CUDA_TRY(cudaMemsetAsync(recs, 0, bytes, st));
    const FastSummary bs = fast_summary(recs, fs, nb, idx->num);
    if ((rc = fast_order(idx, bs, nb, st))) {
        cudaFree(recs);
        return rc;
    }
    k_fast_prep<<<nb, 128, 0, st>>>(idx->num, idx->dim, idx->rows, recs, fs, bs);
    GTS_CUDA_TRY(cudaGetLastError());
    idx->fast_recs = recs;
    idx->fast_nb = nb;
    idx->device_bytes += bytes;
    return GTS_OK;
}

// One filter run over a query batch.  learned: also seed each query's bound
// from the learned radius model.  carry (nullable): certified starting bounds
// (float bits, one per query).  Queries the run cannot answer (a learned
// seed below the k-th distance, or a full candidate list) are written to
// d_fail (owned by the caller) and counted in *n_fail; *r2_out (nullable)
// receives the run's final bounds (valid until the next run).
// fixed (optional): caller-owned device scratch of fixed_bytes used instead
// of the index's growable scratch.
static int fast_run(gts_index *idx, const int *d_qids, int qnum, int k, bool learned, const int *carry,
                    float *d_kth, int *d_ids, float *d_dists, int *d_fail, int *n_fail, int **r2_out,
                    cudaStream_t st, unsigned char *fixed = nullptr, size_t fixed_bytes = 0)
{
    const FastShape fs = fast_shape(idx->dim);
    const int ntiles = (qnum + kFT - 1) / kFT;
    const int nb = idx->fast_nb, nbw = (nb + 31) / 32, nchunk = (nb + kFChunk - 1) / kFChunk;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);

    size_t cub_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (int *)nullptr, (int *)nullptr, (int *)nullptr,
                                    (int *)nullptr, qnum, 0, 32, st);
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~(size_t)255; return o; };
    const size_t o_keys = take(sizeof(int) * qnum), o_vals = take(sizeof(int) * qnum);
    const size_t o_skeys = take(sizeof(int) * qnum), o_order = take(sizeof(int) * qnum);
    const size_t o_cpos = take(sizeof(int) * (size_t)qnum * kFCand);
    const size_t o_clb = take(sizeof(float) * (size_t)qnum * kFCand);
    const size_t o_cub_ = take(sizeof(float) * (size_t)qnum * kFCand);
    const size_t o_ccnt = take(sizeof(int) * qnum), o_r2 = take(sizeof(int) * qnum);
    const size_t o_ctr = take(4 * sizeof(int));   // novf, item counter, item count
    const size_t o_arec = take((size_t)ntiles * fs.arec_bytes);
    const size_t o_mask = take(sizeof(uint32_t) * (size_t)ntiles * nbw);
    const size_t o_items = take(sizeof(int) * (size_t)ntiles * nchunk);
    const size_t o_cub = take(cub_bytes);
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
    float *clb = (float *)(S + o_clb), *cub_ = (float *)(S + o_cub_);
    int *r2 = (int *)(S + o_r2), *ctr = (int *)(S + o_ctr);
    unsigned char *arec = S + o_arec;
    uint32_t *mask = (uint32_t *)(S + o_mask);
    int *items = (int *)(S + o_items);
    const FastSummary bs = fast_summary(idx->fast_recs, fs, nb, idx->num);

    k_fast_keys<<<(qnum + 255) / 256, 256, 0, st>>>(d_qids, qnum, bs.pos, keys, vals);
    size_t cb = cub_bytes;
    GTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(S + o_cub, cb, keys, skeys, vals, order, qnum, 0, 32, st));
    k_fast_init<<<(qnum + 255) / 256, 256, 0, st>>>(qnum, ccnt, r2, carry);
    if (learned && (rc = mlp_seed(idx, d_qids, qnum, k, r2, st))) return rc;
    GTS_CUDA_TRY(cudaMemsetAsync(ctr, 0, 4 * sizeof(int), st));
    k_fast_arec<<<ntiles, 128, 0, st>>>(idx->rows, d_qids, order, qnum, idx->dim, fs, arec);
    k_fast_seed<<<qnum, 128, 0, st>>>(idx->rows, d_qids, bs, idx->num, idx->dim, k, r2);
    const size_t need_smem = sizeof(float) * (size_t)fs.kp * (kFT + kFChunk);
    GTS_CUDA_TRY(cudaFuncSetAttribute(k_fast_need, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need_smem));
    k_fast_need<<<dim3(ntiles, std::min(nchunk, kNeedGridY)), 256, need_smem, st>>>(
        idx->rows, d_qids, arec, fs, idx->dim, nb, bs, r2, mask, nbw, nchunk, items, ctr + 2, idx->d_stats);
    GTS_CUDA_TRY(cudaGetLastError());

    FastTileArgs a;
    a.recs = idx->fast_recs;
    a.arec = arec;
    a.mask = mask;
    a.items = items;
    a.n_items = ctr + 2;
    a.nbw = nbw;
    a.nchunk = nchunk;
    a.k = k;
    a.fs = fs;
    a.cand_pos = cpos;
    a.cand_lb = clb;
    a.cand_ub = cub_;
    a.cand_cnt = ccnt;
    a.r2_bits = r2;
    a.item_counter = ctr + 1;
    a.status = idx->d_status;
    a.stats = idx->d_stats;
    const bool timed = idx->time_filter && idx->fev[0];
    if (timed) GTS_CUDA_TRY(cudaEventRecord(idx->fev[0], st));
    if ((rc = launch_fast_tile(a, nsm, st))) return rc;
    if (timed) GTS_CUDA_TRY(cudaEventRecord(idx->fev[1], st));
    k_add_stat<<<1, 1, 0, st>>>(idx->d_stats + 6, 1ull);
    k_fast_final<<<qnum, 128, 0, st>>>(idx->rows, idx->dim, idx->num, bs.ids, d_qids, qnum, k,
                                        idx->params.infi_dis, cpos, clb, cub_, ccnt, r2, d_kth, d_ids, d_dists,
                                        d_fail, ctr, idx->d_stats);
    GTS_CUDA_TRY(cudaGetLastError());
    int status = 0;
    GTS_CUDA_TRY(cudaMemcpyAsync(&status, idx->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    GTS_CUDA_TRY(cudaMemcpyAsync(n_fail, ctr, sizeof(int), cudaMemcpyDeviceToHost, st));
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    if (status != 0) {
        gts_set_error("tensor-core filter kernel reported status %d (barrier wait gave up)", status);
        return GTS_ERR_KERNEL;
    }
    if (timed) {
        float ms = 0.f;
        GTS_CUDA_TRY(cudaEventElapsedTime(&ms, idx->fev[0], idx->fev[1]));
        idx->filter_ms += ms;
        idx->filter_launches++;
    }
    if (r2_out) *r2_out = r2;
    return GTS_OK;
}

// Queries listed in d_fail (indices into d_qids) answered again, in stages:
// 0 -> after a learned run: the filter without the learned seed;
// 1 -> after a run from certified seeds (its list overflowed): the filter
//      again, starting from the bound that run reached (r2_prev);
// 2 -> the plain traversal.
static int rerun_failed(gts_index *idx, const int *d_qids, int k, int stage, const int *d_fail, int n_fail,
                        const int *r2_prev, float *d_kth, int *d_ids, float *d_dists, cudaStream_t st)
{
    int *sub_q = nullptr, *sub_ids = nullptr, *sub_fail = nullptr, *fail_copy = nullptr, *sub_r2 = nullptr;
    float *sub_kth = nullptr, *sub_dis = nullptr;
    DevVec keep;
    int rc;
    if ((rc = keep.alloc(&sub_q, n_fail)) || (rc = keep.alloc(&sub_kth, n_fail)) ||
        (rc = keep.alloc(&fail_copy, n_fail)) || (rc = keep.alloc(&sub_fail, n_fail)) ||
        (rc = keep.alloc(&sub_r2, n_fail)) || (d_ids && (rc = keep.alloc(&sub_ids, (size_t)n_fail * k))) ||
        (d_dists && (rc = keep.alloc(&sub_dis, (size_t)n_fail * k))))
        return rc;
    GTS_CUDA_TRY(cudaMemcpyAsync(fail_copy, d_fail, sizeof(int) * n_fail, cudaMemcpyDeviceToDevice, st));
    k_gather_i<<<(n_fail + 255) / 256, 256, 0, st>>>(d_qids, fail_copy, n_fail, sub_q);
    if (stage == 1) k_gather_i<<<(n_fail + 255) / 256, 256, 0, st>>>(r2_prev, fail_copy, n_fail, sub_r2);
    if (stage < 2) {
        int n2 = 0, *r2 = nullptr;
        if ((rc = fast_run(idx, sub_q, n_fail, k, false, stage == 1 ? sub_r2 : nullptr, sub_kth, sub_ids, sub_dis,
                           sub_fail, &n2, &r2, st)))
            return rc;
        if (n2 > 0 &&
            (rc = rerun_failed(idx, sub_q, k, stage + 1, sub_fail, n2, r2, sub_kth, sub_ids, sub_dis, st)))
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
    const bool learned = idx->mlp_ready;
    DevVec keep;
    int *fail = nullptr, *r2 = nullptr;
    if ((rc = keep.alloc(&fail, qnum))) return rc;
    int n_fail = 0;
    if ((rc = fast_run(idx, d_qids, qnum, k, learned, nullptr, d_kth, d_ids, d_dists, fail, &n_fail, &r2, st)))
        return rc;
    idx->last_fast_overflow = n_fail;
    if (n_fail > 0) return rerun_failed(idx, d_qids, k, learned ? 0 : 1, fail, n_fail, r2, d_kth, d_ids, d_dists, st);
    return GTS_OK;
}

// The filter without the learned seed, with every buffer carved out of
// `scratch` (bytes long, 256-byte aligned): no device allocation on any
// path.  The filter records must already exist.  Queries the run could not
// answer (a full candidate list) go to the plain traversal, which uses only
// the index's own counters.
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
    if ((rc = fast_run(idx, d_qids, qnum, k, false, nullptr, d_kth, d_ids, d_dists, fail, &n_fail, nullptr, st,
                       scratch + off,
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
