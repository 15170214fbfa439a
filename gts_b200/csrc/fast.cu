// fast.cu -- exact L2 kNN with block pruning and a BF16 tensor-core filter
// ("fast" form).
//
// Same answers as searchIndexKnnV2 (search_v2.cuh:975-1228): the k-th
// distance of every query in the reference's F64 leaf arithmetic
// (search_v2.cuh:447-463) and the k nearest ids with ties broken by id.
// How it gets there is B200-specific:
//
//  * layout: objects are grouped into blocks of at most 128 by a
//    hierarchical k-means (fast_order.cu), and blocks into superblocks.
//    Each block is stored once in HBM as a record that a single bulk copy
//    drops into shared memory in the operand layout tcgen05 reads (K-major,
//    128-byte swizzle): 128 rows of BF16 residuals r = o - c against the
//    block mean c, 3 rows holding c split into three BF16 parts, 13 zero
//    rows, then per object w = |o|^2 + 2 c.d and |d| (d = bf16(r) - r).
//    Block and superblock summaries (centre in FP32, |c|^2, radius max
//    |o - c|) sit beside the records.
//  * seeds: every query's k-th distance is bounded before any filtering by
//    the k-th smallest distance inside its own block (the query is a data
//    object), and by the learned radius model when one is trained.
//  * pruning: queries are sorted by block order into tiles of 128; the
//    triangle inequality |q - c| - radius gives a lower bound per query and
//    ball, first for superblocks, then for the blocks of the superblocks
//    some query of the tile can reach.  Blocks no query of the tile can
//    reach within its seed are never copied or multiplied (GTS's pivot
//    pruning, done with balls instead of rings).  The needed blocks of a
//    tile become work items of up to 8-32 blocks (autotuned).
//  * filter: a persistent CTA per SM takes work items.  One producer warp
//    streams the tile's query operand and the item's block records with
//    bulk copies and issues a 128 x 144 x K MMA chain per block into one of
//    two TMEM accumulators; 4 x CG epilogue warps turn each TMEM row into
//    certified bounds lb <= d^2 <= ub for the 128 objects, keep the k
//    smallest ub (a running k-th bound shared through global memory) and
//    append every object with lb <= bound to the query's candidate list.
//    Producer and epilogue meet only on mbarriers.
//  * recheck: the final bound is the k-th smallest candidate ub; candidates
//    with lb <= bound get their reference-arithmetic distance (one warp per
//    candidate) and the k best (distance, id) are the answer.
// No object whose reference distance can rank in the top k is ever dropped,
// so the result is exact.  Queries whose candidate list overflows, or whose
// learned seed turns out too small, are answered again.  Nothing here
// allocates device memory per call: all buffers come from one scratch
// region planned up front.
#include <cub/device/device_radix_sort.cuh>
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#include "fast.cuh"
#include "fast_blk.cuh"
#include "sm100.cuh"

namespace gts {

using namespace sm100;

constexpr int kFItemMax = 32;         // blocks per filter work item at most (autotuned: 8, 16 or 32)
constexpr int kFItemMin = 8;
constexpr int kFChunk = 64;           // balls tested per pruning step
constexpr int kNeedBlkY = 8;          // block-pruning CTAs per tile
constexpr int kFMaxBatch = 32768;     // queries per filter run (bounds the candidate lists)

__device__ __forceinline__ unsigned short f2bf(float x)
{
    return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
__device__ __forceinline__ float bf2f(unsigned short b) { return __bfloat162float(__ushort_as_bfloat16(b)); }

// ---------------------------------------------------------------- layout

// Slots of every block from the order: block b holds the objects at
// positions [bl[b], br[b]) in slots b*128 .. b*128 + size - 1.
__global__ void __launch_bounds__(kFB) k_fast_layout(const int *__restrict__ perm, const int *__restrict__ bl,
                                                     const int *__restrict__ br, int *__restrict__ ids,
                                                     int *__restrict__ pos)
{
    const int b = blockIdx.x, t = threadIdx.x;
    const int l = bl[b], size = br[b] - l;
    const int slot = b * kFB + t;
    if (t < size) {
        const int id = perm[l + t];
        ids[slot] = id;
        pos[id] = slot;
    } else {
        ids[slot] = -1;
    }
}

// One CTA per block: the FP32 rows of its slots, in slot order (row stride
// kp, zeros past dim and in padding slots), so the seed and the exact
// recheck read a block's rows from one contiguous range.
__global__ void __launch_bounds__(kFB) k_fast_prows(int dim, int kp, const float *__restrict__ rows,
                                                   const int *__restrict__ ids, float *__restrict__ prow)
{
    const int b = blockIdx.x, t = threadIdx.x;
    for (int r = 0; r < kFB; r++) {
        const int slot = b * kFB + r;
        const int id = ids[slot];
        for (int j = t; j < kp; j += kFB)
            prow[(size_t)slot * kp + j] = (id >= 0 && j < dim) ? rows[(size_t)id * dim + j] : 0.f;
    }
}

// One CTA per block; thread t = slot t of the block.
__global__ void __launch_bounds__(kFB) k_fast_prep(int dim, const float *__restrict__ rows,
                                                   unsigned char *__restrict__ recs, FastShape fs, FastSummary bs)
{
    __shared__ float cen[kFMaxKp];
    __shared__ int bid[kFB];
    __shared__ unsigned int mx_rb, mx_w, mx_rad;
    const int b = blockIdx.x, t = threadIdx.x;
    const int myid = bs.ids[b * kFB + t];
    const bool valid = myid >= 0;
    bid[t] = valid ? myid : 0;
    const int cnt = __syncthreads_count(valid);   // valid slots come first
    unsigned char *rec = recs + (size_t)b * fs.rec_bytes;
    for (int j = t; j < fs.kp; j += kFB) {
        double s = 0.0;
        if (j < dim)
            for (int i = 0; i < cnt; i++) s += (double)rows[(size_t)bid[i] * dim + j];
        cen[j] = (j < dim && cnt > 0) ? (float)(s / cnt) : 0.f;
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
        tail[kTailRad] = __uint_as_float(mx_rad);
        bs.rad[b] = cnt > 0 ? __uint_as_float(mx_rad) : -1.f;
    }
}

// One CTA per superblock: centre (mean of its objects, FP64 sums) and
// radius max |o - c| rounded up.
__global__ void __launch_bounds__(256) k_fast_sbprep(int dim, const float *__restrict__ rows, FastShape fs,
                                                     FastSummary bs)
{
    __shared__ float cen[kFMaxKp];
    __shared__ unsigned int mx;
    const int s = blockIdx.x, t = threadIdx.x;
    const int b0 = bs.sb_b0[s], b1 = bs.sb_b0[s + 1];
    const int nslot = (b1 - b0) * kFB;
    for (int j = t; j < fs.kp; j += blockDim.x) {
        double acc = 0.0;
        int c = 0;
        if (j < dim)
            for (int i = 0; i < nslot; i++) {
                const int id = bs.ids[(size_t)b0 * kFB + i];
                if (id < 0) continue;
                acc += (double)rows[(size_t)id * dim + j];
                c++;
            }
        cen[j] = (j < dim && c > 0) ? (float)(acc / c) : 0.f;
        bs.sb_cen[(size_t)s * fs.kp + j] = cen[j];
    }
    if (t == 0) mx = 0u;
    __syncthreads();
    if (t == 0) {
        double c2 = 0.0;
        for (int j = 0; j < dim; j++) c2 += (double)cen[j] * cen[j];
        bs.sb_c2[s] = (float)c2;
    }
    for (int i = t; i < nslot; i += blockDim.x) {
        const int id = bs.ids[(size_t)b0 * kFB + i];
        if (id < 0) continue;
        const float *o = rows + (size_t)id * dim;
        double e2 = 0.0;
        for (int j = 0; j < dim; j++) {
            const double e = (double)o[j] - (double)cen[j];
            e2 += e * e;
        }
        atomicMax(&mx, __float_as_uint(__double2float_ru(sqrt(e2) * (1.0 + 1e-12))));
    }
    __syncthreads();
    if (t == 0) bs.sb_rad[s] = __uint_as_float(mx);
}

// ---------------------------------------------------------------- per call

// One CTA per tile: the A operand of the tile's 128 queries (sorted by block
// order), split into BF16 hi + lo, in the swizzled layout, and per lane
// (query index, |q|^2, |q|).  A tile record is one bulk copy.  With qt, beside
// it an FP32 copy of the rows ([kp][128], zero padding) for the FP32 pruning
// kernels.  The tile's rows pass through shared memory 64 columns at a time:
// the CTA reads them coalesced (a warp reads 32 consecutive values of one
// row, all of a thread's loads in flight at once), then each thread converts
// its own query's row; |q|^2 is summed in column order as before.
__global__ void __launch_bounds__(128) k_fast_arec(const float *__restrict__ rows, const int *__restrict__ qids,
                                                   const int *__restrict__ order, int qnum, int dim, FastShape fs,
                                                   unsigned char *__restrict__ arec, float *__restrict__ qt)
{
    __shared__ float sx[kFT][64 + 1];
    __shared__ int rid[kFT];
    const int tile = blockIdx.x, lq = threadIdx.x;
    float *qtt = qt ? qt + (size_t)blockIdx.x * fs.kp * kFT : nullptr;
    unsigned char *A_hi = arec + (size_t)tile * fs.arec_bytes, *A_lo = A_hi + fs.atile_bytes;
    int4 *info = reinterpret_cast<int4 *>(A_lo + fs.atile_bytes);
    const int slot = tile * kFT + lq;
    const int qi = slot < qnum ? order[slot] : -1;
    rid[lq] = qi >= 0 ? qids[qi] : -1;
    __syncthreads();
    double acc = 0.0;
    for (int c0 = 0; c0 < fs.kp; c0 += 64) {
        float v[64];
#pragma unroll
        for (int m = 0; m < 64; m++) {
            const int i = lq + 128 * m, r = i >> 6, j = c0 + (i & 63);
            const int id = rid[r];
            v[m] = (id >= 0 && j < dim) ? rows[(size_t)id * dim + j] : 0.f;
        }
#pragma unroll
        for (int m = 0; m < 64; m++) {
            const int i = lq + 128 * m;
            sx[i >> 6][i & 63] = v[m];
        }
        __syncthreads();
        for (int j0 = 0; j0 < 64; j0 += 8) {
            unsigned short hi[8], lo[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const float x = sx[lq][j0 + u];
                if (qtt) qtt[(size_t)(c0 + j0 + u) * kFT + lq] = x;
                acc += (double)x * x;
                hi[u] = f2bf(x);
                lo[u] = f2bf(x - bf2f(hi[u]));
            }
            uint4 vh, vl;
            vh.x = hi[0] | ((uint32_t)hi[1] << 16); vh.y = hi[2] | ((uint32_t)hi[3] << 16);
            vh.z = hi[4] | ((uint32_t)hi[5] << 16); vh.w = hi[6] | ((uint32_t)hi[7] << 16);
            vl.x = lo[0] | ((uint32_t)lo[1] << 16); vl.y = lo[2] | ((uint32_t)lo[3] << 16);
            vl.z = lo[4] | ((uint32_t)lo[5] << 16); vl.w = lo[6] | ((uint32_t)lo[7] << 16);
            const uint32_t off = sw128_offset(lq, c0 + j0, kFT);
            *reinterpret_cast<uint4 *>(A_hi + off) = vh;
            *reinterpret_cast<uint4 *>(A_lo + off) = vl;
        }
        __syncthreads();
    }
    info[lq] = make_int4(qi, __float_as_int((float)acc), __float_as_int((float)sqrt(acc)), 0);
}

// Seeds made once with the records.  Queries are objects, so a bound on a
// query's k-th distance can be computed per object ahead of any call: the
// k-th smallest distance from the object to the objects of its own block
// and of the kSeedNbr blocks whose centres lie nearest to its block's (the
// object itself counts, at distance 0).  Any k of those objects bound the
// query's k-th distance, and 32 blocks (4,096 objects) hold nearly all of
// a query's close neighbours, so the seed sits next to the answer: at
// 1,000,000 x 128 and k = 8 the filter lists 9.1 candidates per query
// against 97 from the own-block k-th distance.  Stored for k = 1, 2, 4, ..,
// 64 (a call with another k reads the next power of two: a bound for the
// larger k bounds every smaller k).

// The kSeedNbr blocks with the nearest centres (FP32, ties by block id),
// -1 where there are fewer blocks.  One warp per block b, eight per CTA;
// the CTA stages 32 centres at a time in shared memory and lane l measures
// centre l of the stage against its warp's centre.
constexpr int kNbrWarps = 8;
__global__ void __launch_bounds__(32 * kNbrWarps) k_fast_nbrs(FastSummary bs, int nb, int kp,
                                                              int *__restrict__ nbr)
{
    extern __shared__ float nsm[];   // [kNbrWarps][kp] own centres, then [32][kp + 4] staged centres
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int ks = kp + 4;
    float *own = nsm + warp * kp;
    float *stg = nsm + kNbrWarps * kp;
    const int b = blockIdx.x * kNbrWarps + warp;
    for (int d = lane; d < kp; d += 32) own[d] = b < nb ? bs.cen[(size_t)b * kp + d] : 0.f;
    float bd[kSeedNbr];
    int bi[kSeedNbr];
#pragma unroll
    for (int i = 0; i < kSeedNbr; i++) {
        bd[i] = FLT_MAX;
        bi[i] = -1;
    }
    for (int j0 = 0; j0 < nb; j0 += 32) {
        __syncthreads();
        for (int e = t; e < 32 * kp; e += blockDim.x) {
            const int r = e / kp, d = e - r * kp;
            stg[r * ks + d] = j0 + r < nb ? bs.cen[(size_t)(j0 + r) * kp + d] : 0.f;
        }
        __syncthreads();
        const int j = j0 + lane;
        if (b >= nb || j >= nb || j == b) continue;
        float acc = 0.f;
        for (int d = 0; d < kp; d += 4) {
            const float4 c4 = *reinterpret_cast<const float4 *>(stg + lane * ks + d);
            const float4 o4 = *reinterpret_cast<const float4 *>(own + d);
            const float e0 = c4.x - o4.x, e1 = c4.y - o4.y, e2 = c4.z - o4.z, e3 = c4.w - o4.w;
            acc = fmaf(e3, e3, fmaf(e2, e2, fmaf(e1, e1, fmaf(e0, e0, acc))));
        }
        if (acc < bd[kSeedNbr - 1]) {   // sorted insertion (j grows, so ties keep the smaller id)
            float v = acc;
            int vi = j;
#pragma unroll
            for (int i = 0; i < kSeedNbr; i++) {
                if (v < bd[i]) {
                    const float tv = bd[i];
                    const int ti = bi[i];
                    bd[i] = v;
                    bi[i] = vi;
                    v = tv;
                    vi = ti;
                }
            }
        }
    }
    if (b >= nb) return;
    // the kSeedNbr smallest of the 32 lanes' lists: each round the lane
    // holding the smallest head (ties: smaller id) pops it
    int head = 0;
    for (int r = 0; r < kSeedNbr; r++) {
        float v = FLT_MAX;
        int vi = INT_MAX;
#pragma unroll
        for (int i = 0; i < kSeedNbr; i++)
            if (i == head) {
                v = bd[i];
                vi = bi[i] < 0 ? INT_MAX : bi[i];
            }
        float mv = v;
        int mi = vi;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, mv, o);
            const int oi = __shfl_xor_sync(0xffffffffu, mi, o);
            if (ov < mv || (ov == mv && oi < mi)) {
                mv = ov;
                mi = oi;
            }
        }
        if (vi == mi && vi != INT_MAX) head++;
        if (lane == 0) nbr[(size_t)b * kSeedNbr + r] = mi == INT_MAX ? -1 : mi;
    }
}

// The seed table: one CTA per block b, warp w taking objects w, w + 4, ...
// For each of the blocks (b, then its neighbours) the block's FP32 rows are
// staged in shared memory ([128][kp + 4]); lane l sums the squared FP32
// differences of rows l, l + 32, l + 64, l + 96 against the object's row in
// dimension order (fused multiply-adds, as the reference's leaf loop runs
// them), and the object's 64 smallest values so far (in shared memory,
// ascending) are merged with the new values below the 64th by ranking.
// A sum of at most 320 non-negative FP32 terms is within 322 * 2^-24 <
// 2e-5 relative of the exact sum of the same FP32 differences squared, the
// value the reference's FP64 sum rounds, so widening by (1 + 4e-5) gives a
// certified bound on the reference's k-th squared distance.  FLT_MAX where
// the blocks hold fewer than k objects (no seed).
__global__ void __launch_bounds__(128) k_fast_selfk(FastSummary bs, int kp, const int *__restrict__ nbr)
{
    extern __shared__ float ssm[];
    const int b = blockIdx.x, t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int ks = kp + 4;
    float *srow = ssm;                                  // [128][ks] the staged block's rows
    float *best = srow + (size_t)kFB * ks;              // [128][kSeedBest] per object, ascending
    float *obuf = best + (size_t)kFB * kSeedBest + warp * (kp + 3 * kSeedBest);   // [kp] object row
    float *sc = obuf + kp;                              // [3 * kSeedBest] merge scratch
    __shared__ unsigned vmask[kFB / 32], omask[kFB / 32];
    const unsigned own_valid = __ballot_sync(0xffffffffu, bs.ids[b * kFB + t] >= 0);
    if (lane == 0) omask[warp] = own_valid;
    for (int i = t; i < kFB * kSeedBest; i += blockDim.x) best[i] = FLT_MAX;
    int cnt = 0;   // objects in the blocks used so far
    for (int s = 0; s <= kSeedNbr; s++) {
        const int j = s == 0 ? b : nbr[(size_t)b * kSeedNbr + s - 1];
        if (j < 0) break;
        __syncthreads();
        // stage block j's rows and validity
        const float4 *src = reinterpret_cast<const float4 *>(bs.prow + (size_t)j * kFB * kp);
        for (int e = t; e < kFB * kp / 4; e += blockDim.x) {
            const int r = e / (kp / 4), d4 = e - r * (kp / 4);
            *reinterpret_cast<float4 *>(srow + (size_t)r * ks + 4 * d4) = src[e];
        }
        const bool jv = bs.ids[j * kFB + t] >= 0;
        const unsigned jm = __ballot_sync(0xffffffffu, jv);
        if (lane == 0) vmask[warp] = jm;   // valid rows of block j
        cnt += __syncthreads_count(jv);    // also: rows and masks visible
        for (int m = warp; m < kFB; m += 4) {
            if (!((omask[m >> 5] >> (m & 31)) & 1u)) continue;
            const float *orow = bs.prow + ((size_t)b * kFB + m) * kp;
            for (int d = lane; d < kp; d += 32) obuf[d] = orow[d];
            __syncwarp();
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            for (int d = 0; d < kp; d += 4) {
                const float4 q4 = *reinterpret_cast<const float4 *>(obuf + d);
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    const float4 o4 = *reinterpret_cast<const float4 *>(srow + (size_t)(lane + 32 * h) * ks + d);
                    const float e0 = o4.x - q4.x, e1 = o4.y - q4.y, e2 = o4.z - q4.z, e3 = o4.w - q4.w;
                    acc[h] = fmaf(e3, e3, fmaf(e2, e2, fmaf(e1, e1, fmaf(e0, e0, acc[h]))));
                }
            }
            float *bm = best + (size_t)m * kSeedBest;
            const float thr = bm[kSeedBest - 1];
            // survivors (below the current 64th smallest) after the 64 kept values
            sc[lane] = bm[lane];
            sc[lane + 32] = bm[lane + 32];
            int n = kSeedBest;
#pragma unroll
            for (int h = 0; h < 4; h++) {
                const bool rv = (vmask[h] >> lane) & 1u;
                const bool keep = rv && acc[h] < thr;
                const unsigned km = __ballot_sync(0xffffffffu, keep);
                if (keep) sc[n + __popc(km & ((1u << lane) - 1u))] = acc[h];
                n += __popc(km);
            }
            __syncwarp();
            if (n > kSeedBest) {
                for (int i = lane; i < n; i += 32) {
                    const float v = sc[i];
                    int rank = 0;
                    for (int q = 0; q < n; q++) {
                        const float y = sc[q];
                        rank += (y < v || (y == v && q < i)) ? 1 : 0;
                    }
                    if (rank < kSeedBest) bm[rank] = v;
                }
            }
            __syncwarp();
        }
    }
    __syncthreads();
    for (int m = warp; m < kFB; m += 4) {
        int *out = bs.selfk + ((size_t)b * kFB + m) * kSelfK;
        const float *bm = best + (size_t)m * kSeedBest;
        if (lane < kSelfK) {
            int v = __float_as_int(FLT_MAX);
            if (lane < kSelfKN && ((omask[m >> 5] >> (m & 31)) & 1u) && cnt >= (1 << lane))
                v = __float_as_int(bm[(1 << lane) - 1] * (1.f + 4e-5f));
            out[lane] = v;
        }
    }
}

// Seeds from the table: one thread per query (jk: the smallest power of two
// 2^jk >= k).
__global__ void k_fast_seed_tab(const int *__restrict__ qids, int qnum, const int *__restrict__ pos_of,
                                const int *__restrict__ selfk, int jk, int *__restrict__ r2_bits)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < qnum) atomicMin(&r2_bits[i], selfk[(size_t)pos_of[qids[i]] * kSelfK + jk]);
}

// ---------------------------------------------------------------- pruning

// Shared state of a pruning CTA: the tile's 128 query rows (FP32,
// [kp][128]), their |q|^2, |q| and seeds, and one chunk of up to 64 balls.
struct NeedSmem {
    float q2s[kFT], qns[kFT], seeds[kFT];
    float c2s[kFChunk], cns[kFChunk], rads[kFChunk];
    unsigned int flags[2];
    uint32_t lmask[kFChunk][4];   // per ball: the tile's lanes (queries) that need it
};

// The tile's query rows come from the FP32 copy k_fast_arec wrote in this
// layout ([kp][128], zero padding): one contiguous 64 KB read.
__device__ __forceinline__ void need_load_tile(const float *__restrict__ qt, const unsigned char *__restrict__ arec,
                                               const FastShape &fs, int tile, const int *__restrict__ r2_bits,
                                               float *Qs, NeedSmem &sm)
{
    const int t = threadIdx.x;
    const int4 *info = reinterpret_cast<const int4 *>(arec + (size_t)tile * fs.arec_bytes + 2 * fs.atile_bytes);
    if (t < kFT) {
        const int4 in = info[t];
        sm.q2s[t] = __int_as_float(in.y);
        sm.qns[t] = __int_as_float(in.z);
        sm.seeds[t] = in.x >= 0 ? __int_as_float(r2_bits[in.x]) : -1.f;
    }
    const float4 *src = reinterpret_cast<const float4 *>(qt + (size_t)tile * fs.kp * kFT);
    float4 *dst = reinterpret_cast<float4 *>(Qs);
#pragma unroll 4
    for (int i = t; i < fs.kp * (kFT / 4); i += 256) dst[i] = src[i];
}

// Dimensions of the ball centres a pruning CTA holds at once: all of them up
// to kp = 128, 64 at a time above (the tile's rows stay whole).
__host__ __device__ __forceinline__ int need_kc(int kp) { return kp <= kFResKp ? kp : 64; }

// Shared memory of a pruning CTA: the tile's rows [kp][128] and one chunk
// of ball centres [need_kc][64] (FP32).
__host__ __device__ __forceinline__ size_t need_smem_bytes(int kp)
{
    return sizeof(float) * ((size_t)kp * kFT + (size_t)need_kc(kp) * kFChunk);
}

// Balls c0 .. c0+63 (those below cend; with a list, balls list[0 .. cend-1]
// and c0 = 0) against the tile: bit i of the result is set when some query
// of the tile can reach ball i of the chunk within its seed:
// |q - c|_lo - radius <= sqrt(seed).  masks: also sm.lmask[i], the lanes of
// the queries that reach ball i.  256 threads: each computes
// 8 queries (4tq..4tq+3 and 64+4tq..64+4tq+3, so a quarter warp reads 128
// consecutive bytes: no bank conflicts) x 4 balls of FP32 q.c, over the
// centre dimensions need_kc(kp) at a time.
__device__ __forceinline__ uint64_t need_chunk(const float *__restrict__ cen, const float *__restrict__ c2, const float *__restrict__ rad,
                               int c0, int cend, const int *list, int kp, const float *Qs, float *Cs, NeedSmem &sm,
                               bool masks = false)
{
    const int t = threadIdx.x;
    const int kc = need_kc(kp);
    __syncthreads();   // previous chunk's Cs / flags consumed, list written
    if (t < kFChunk) {
        const bool ok = c0 + t < cend;
        const int ball = ok ? (list ? list[t] : c0 + t) : 0;
        sm.c2s[t] = ok ? c2[ball] : 0.f;
        sm.cns[t] = ok ? sqrtf(c2[ball]) * 1.000001f : 0.f;
        sm.rads[t] = ok ? rad[ball] : -1.f;
    }
    if (t < 2) sm.flags[t] = 0u;
    if (masks) sm.lmask[t >> 2][t & 3] = 0u;   // 256 threads, 64 x 4 words
    const int tq = t & 15, tb = t >> 4;
    float acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[i][c] = 0.f;
    for (int k0 = 0; k0 < kp; k0 += kc) {
        if (k0 > 0) __syncthreads();   // the previous centre dimensions consumed
        // thread (bb, j4): 4 dimensions of ball bb; consecutive threads take
        // consecutive balls, so the shared-memory writes do not conflict
        for (int i = t; i < (kc / 4) * kFChunk; i += 256) {
            const int bb = i % kFChunk, j4 = i / kFChunk;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (c0 + bb < cend) {
                const int ball = list ? list[bb] : c0 + bb;
                v = *reinterpret_cast<const float4 *>(cen + (size_t)ball * kp + k0 + 4 * j4);
            }
            Cs[(4 * j4 + 0) * kFChunk + bb] = v.x;
            Cs[(4 * j4 + 1) * kFChunk + bb] = v.y;
            Cs[(4 * j4 + 2) * kFChunk + bb] = v.z;
            Cs[(4 * j4 + 3) * kFChunk + bb] = v.w;
        }
        __syncthreads();
        // kc is a multiple of 64: unrolled so the shared loads of later j are
        // in flight while the FMAs of earlier ones run
#pragma unroll 4
        for (int j = 0; j < kc; j++) {
            const float4 qa = *reinterpret_cast<const float4 *>(Qs + (k0 + j) * kFT + tq * 4);
            const float4 qb = *reinterpret_cast<const float4 *>(Qs + (k0 + j) * kFT + 64 + tq * 4);
            const float4 cc = *reinterpret_cast<const float4 *>(Cs + j * kFChunk + tb * 4);
            const float qv[8] = {qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z, qb.w};
            const float cv[4] = {cc.x, cc.y, cc.z, cc.w};
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[i][c] = fmaf(qv[i], cv[c], acc[i][c]);
        }
    }
    // FP32 dot of kp products: error <= kp 2^-23 |q||c|; the three-term
    // sum adds <= 4e-7 (|q|^2 + |c|^2)
    const float gam = 2.f * (float)kp * 1.2e-7f;
    unsigned int need = 0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int bb = tb * 4 + c;
        const float rd = sm.rads[bb];
        uint32_t qb = 0;   // bit i: query i of this thread's eight reaches the ball
        if (rd >= 0.f) {
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int l = (i < 4 ? 0 : 64 - 4) + tq * 4 + i;
                const float sd = sm.seeds[l];
                if (sd < 0.f) continue;
                const float q2 = sm.q2s[l], cc2 = sm.c2s[bb];
                const float e = gam * sm.qns[l] * sm.cns[bb] + 4e-7f * (q2 + cc2) + 1e-30f;
                const float d2lo = q2 - 2.f * acc[i][c] + cc2 - e;
                const float lo = sqrtf(fmaxf(d2lo, 0.f)) * 0.999999f - rd;
                qb |= (lo <= 0.f || lo * lo * 0.999999f <= sd ? 1u : 0u) << i;
            }
        }
        // lanes 4tq..4tq+3 (bits 0-3) and 64+4tq.. (bits 4-7)
        if (masks && qb) {
            const int sh = (4 * tq) & 31;
            if (qb & 15u) atomicOr(&sm.lmask[bb][tq >> 3], (qb & 15u) << sh);
            if (qb >> 4) atomicOr(&sm.lmask[bb][2 + (tq >> 3)], (qb >> 4) << sh);
        }
        need |= (qb ? 1u : 0u) << c;
    }
    // the 16 threads of a half-warp share their 4 balls
    need |= __shfl_xor_sync(0xffffffffu, need, 1);
    need |= __shfl_xor_sync(0xffffffffu, need, 2);
    need |= __shfl_xor_sync(0xffffffffu, need, 4);
    need |= __shfl_xor_sync(0xffffffffu, need, 8);
    if (tq == 0 && need) atomicOr(&sm.flags[(tb * 4) >> 5], need << ((tb * 4) & 31));
    __syncthreads();
    return (uint64_t)sm.flags[0] | ((uint64_t)sm.flags[1] << 32);
}

// Superblocks the tile needs: CTA (tile, y) tests superblock chunk y and
// writes its two mask words sb_mask[tile][2y .. 2y+1].
__global__ void __launch_bounds__(256) k_need_sb(const float *__restrict__ qt,
                                                 const unsigned char *__restrict__ arec, FastShape fs,
                                                 FastSummary bs, int nsb, const int *__restrict__ r2_bits,
                                                 uint32_t *__restrict__ sb_mask, int nsbw)
{
    extern __shared__ __align__(16) float nsm[];
    __shared__ NeedSmem sm;
    float *Qs = nsm, *Cs = nsm + fs.kp * kFT;
    const int tile = blockIdx.x, ch = blockIdx.y;
    need_load_tile(qt, arec, fs, tile, r2_bits, Qs, sm);
    const uint64_t m = need_chunk(bs.sb_cen, bs.sb_c2, bs.sb_rad, ch * kFChunk, nsb, nullptr, fs.kp, Qs, Cs, sm);
    if (threadIdx.x == 0) {
        sb_mask[(size_t)tile * nsbw + 2 * ch] = (uint32_t)m;
        if (2 * ch + 1 < nsbw) sb_mask[(size_t)tile * nsbw + 2 * ch + 1] = (uint32_t)(m >> 32);
    }
}

// Blocks the tile needs, inside the superblocks it needs: CTA (tile, y)
// takes every gridDim.y-th needed superblock, gathers their blocks into
// full chunks of kFChunk (superblocks hold 1..32 blocks) and appends the
// needed ones to blist[tile][nbcap] (count in bcnt[tile]).
__global__ void __launch_bounds__(256) k_need_blk(const float *__restrict__ qt,
                                                  const unsigned char *__restrict__ arec, FastShape fs,
                                                  FastSummary bs, const int *__restrict__ r2_bits,
                                                  const uint32_t *__restrict__ sb_mask, int nsbw,
                                                  int *__restrict__ blist, int *__restrict__ bcnt, int nbcap,
                                                  unsigned long long *stats, uint4 *__restrict__ bmask,
                                                  int *__restrict__ bq_cnt)
{
    extern __shared__ __align__(16) float nsm[];
    __shared__ NeedSmem sm;
    // two chunk lists: thread 0 reads chunk p's while chunk p + 1's is written
    __shared__ int cblk[2][kFChunk];
    float *Qs = nsm, *Cs = nsm + fs.kp * kFT;
    const int tile = blockIdx.x, t = threadIdx.x;
    // the superblocks of this CTA first, so a CTA with none returns early
    int mine = 0, seen = 0;
    for (int w = 0; w < nsbw; w++) {
        const int c = __popc(sb_mask[(size_t)tile * nsbw + w]);
        mine += (seen + c + (int)gridDim.y - 1 - (int)blockIdx.y) / (int)gridDim.y -
                (seen + (int)gridDim.y - 1 - (int)blockIdx.y) / (int)gridDim.y;
        seen += c;
    }
    if (mine == 0) return;
    need_load_tile(qt, arec, fs, tile, r2_bits, Qs, sm);
    unsigned long long tested = 0;
    int fill = 0, p = 0;
    int *dst = blist + (size_t)tile * nbcap;
    auto run_chunk = [&]() {
        const uint64_t m0 = need_chunk(bs.cen, bs.c2, bs.rad, 0, fill, cblk[p], fs.kp, Qs, Cs, sm, bmask != nullptr);
        if (t == 0) {
            tested += (unsigned long long)fill;
            uint64_t m = m0;
            const int cnt = __popcll(m);
            if (cnt) {
                int at = atomicAdd(&bcnt[tile], cnt);
                while (m) {
                    const int i = __ffsll((long long)m) - 1;
                    m &= m - 1;
                    if (at < nbcap) {
                        dst[at] = cblk[p][i];
                        if (bmask) {
                            const uint4 lm = make_uint4(sm.lmask[i][0], sm.lmask[i][1], sm.lmask[i][2], sm.lmask[i][3]);
                            bmask[(size_t)tile * nbcap + at] = lm;
                            atomicAdd(&bq_cnt[cblk[p][i]], __popc(lm.x) + __popc(lm.y) + __popc(lm.z) + __popc(lm.w));
                        }
                    }
                    at++;
                }
            }
        }
        fill = 0;
        p ^= 1;
    };
    seen = 0;
    for (int w = 0; w < nsbw; w++) {
        uint32_t word = sb_mask[(size_t)tile * nsbw + w];
        while (word) {
            const int s = w * 32 + __ffs(word) - 1;
            word &= word - 1;
            if (seen++ % gridDim.y != blockIdx.y) continue;
            const int b1 = bs.sb_b0[s + 1];
            for (int b = bs.sb_b0[s]; b < b1;) {
                const int take = min(b1 - b, kFChunk - fill);
                if (t < take) cblk[p][fill + t] = b + t;
                fill += take;
                b += take;
                if (fill == kFChunk) run_chunk();
            }
        }
    }
    if (fill > 0) run_chunk();
    if (t == 0 && stats && tested) atomicAdd(&stats[7], tested);
}

// Work items: (tile, first list entry) per `item` needed blocks of a tile.
// Longest first: the full items from the front of the array (count in
// n_items[0]), each tile's partial last item from the back (count in
// n_items[1]), so the persistent CTAs end on the short ones.
__global__ void k_items(int ntiles, const int *__restrict__ bcnt, int nbcap, int item, int2 *__restrict__ items,
                        int *__restrict__ n_items, int items_cap)
{
    const int tile = blockIdx.x * blockDim.x + threadIdx.x;
    if (tile >= ntiles) return;
    const int cnt = min(bcnt[tile], nbcap);
    const int full = cnt / item, rem = cnt - full * item;
    if (full > 0) {
        const int base = atomicAdd(&n_items[0], full);
        for (int i = 0; i < full; i++) items[base + i] = make_int2(tile, i * item);
    }
    if (rem > 0) items[items_cap - 1 - atomicAdd(&n_items[1], 1)] = make_int2(tile, full * item);
}

// ---------------------------------------------------------------- filter

struct FastTileArgs {
    const unsigned char *recs;   // block records
    const unsigned char *arec;   // query tile records
    const int *blist;            // [ntiles][nbcap] needed blocks per tile
    const int *bcnt;             // [ntiles]
    const int2 *items;           // (tile, first entry): n_items[0] full ones from the front,
    const int *n_items;          // n_items[1] partial ones from the back of items_cap
    int items_cap;
    int nbcap, k;
    int item;                    // blocks per work item (<= kFItemMax)
    int st_cap;                  // staged candidates per item (shared memory)
    FastShape fs;
    int *cand_pos;               // [qnum][kFCand] slots
    float *cand_lb, *cand_ub;    // [qnum][kFCand] bounds on d^2
    int *cand_cnt;               // [qnum]
    int *r2_bits;                // [qnum] bound on the k-th d^2 (float bits), shared by all threads
    int *item_counter;           // persistent-CTA work queue
    int *status;
    unsigned long long *stats;
    // range counts (k_fast_tile<.., true>): objects whose upper bound is
    // below r2lo are counted in rcnt[query] without a list entry
    float r2lo;
    int *rcnt;
    int nsc;                     // streamed form: K-chunk stages
    int stream;                  // streamed form also at kp <= kFResKp (autotuned)
};

constexpr int kFS = 3;         // block stages, each with its own TMEM accumulator
constexpr int kFAccCols = 160; // TMEM columns between accumulators (kFN = 144 used)
// Streamed form (kp > kFResKp): K-chunk stages (a.nsc of them, at most
// kFSCMax) and, per accumulator, the block's record tail in its own buffer.
constexpr int kFSCMax = 6;
constexpr uint32_t kFTailBytes = 1024u + 32u;   // w, dn, block scalars
constexpr uint32_t kFTailPad = 1088u;

// Candidates are staged in shared memory during an item; the capacity
// (a.st_cap) is what the shared memory left after the operands holds.
constexpr int kFStageMax = 8192;

struct __align__(16) FastCtl {
    uint64_t full[kFS];    // block copy landed
    uint64_t efree[kFS];   // epilogue of the block in this stage done (one arrive per epilogue warp)
    uint64_t mmad[kFS];    // MMA chain into TMEM accumulator s (one per stage) done
    uint64_t tfull[kFS];   // streamed form: the block's record tail landed in tail buffer s
    uint64_t cfull[kFSCMax];   // streamed form: K chunk landed in chunk stage c
    uint64_t cfree[kFSCMax];   // streamed form: the MMAs reading chunk stage c done
    uint64_t afull;        // query tile copy landed
    uint32_t tmem;
    int tile, nblk;
    int err;
    int blk[kFItemMax];    // the item's blocks
    int th_cnt[4 * kFT];   // at the flush: staged candidates per epilogue thread
    int qbase[kFT];        // at the flush: list offset per query lane
    int r2s[kFT];          // per query lane: the smallest bound its column groups reached (float bits)
};

// A staged candidate: its slot, its lower bound and the margin ub - lb as a
// half rounded up (so lb + margin >= ub), in three arrays.
constexpr size_t kStagedBytes = sizeof(int) + sizeof(float) + sizeof(unsigned short);

// Persistent filter kernel, one CTA per SM, 4 x CG epilogue warps + one
// producer warp.  CG column groups: warps w, w+4, ... share TMEM lanes
// 32*(w%4)..+31 (the same 32 queries) and split the 128 object columns.
//
// Per item (a tile and up to a.item of its needed blocks), with gi counting
// blocks over the CTA's life (barrier phases follow it):
//   producer:  copy A (unless this CTA's previous item had the same tile);
//              copy blocks 0..2 into stages gi%3; for each block:
//              wait its copy, wait the epilogue of block gi-2 (frees TMEM
//              accumulator gi%2 and stage (gi-2)%3 = (gi+1)%3), MMA chain into
//              accumulator gi%2, commit, copy block gi+1 into the freed stage.
//   epilogue:  wait the MMA of block gi, bound the 128 x 128 pairs, arrive
//              on efree[gi%3].  Passing objects are staged in shared memory
//              (shared-memory atomics only) and written to the queries'
//              candidate lists once per item, one global atomic per query.
// The CTA synchronises only between items.
//
// KH > 0 (k <= KH): each epilogue thread keeps its k smallest upper bounds in
// registers (slots k..KH-1 hold -FLT_MAX and are never the largest); KH = 0:
// as a binary max-heap in shared memory, k per thread, each bound stored as
// the upper 16 bits of its float rounded up (a bound again, 2 bytes).
//
// RANGE: range counts instead of kNN.  The bound stays the query's (r^2 with
// the reference-arithmetic margin); objects certainly inside are counted per
// thread, only the uncertain ones are listed; no bound heap.
//
// KS (kp > kFResKp, where a whole record does not fit a stage beside the
// query tile; below it an autotuner choice): the producer streams each block's operand rows in 64-wide K
// chunks through a.nsc chunk stages -- a stage is refilled as soon as the
// MMAs reading it are done (tcgen05.commit on cfree), one unit behind the
// MMA issue -- and copies the block's record tail (w, dn, scalars) into the
// tail buffer of its accumulator once the epilogue of the block three back
// has freed both.  The epilogue is the same, reading the tail buffer.
template <int CG, int KH, bool RANGE, bool KS>
__global__ void __launch_bounds__(128 * CG + 32, 1) k_fast_tile(FastTileArgs a)
{
    constexpr int NT = 128 * CG;   // epilogue threads
    constexpr int NEW = NT / 32;   // epilogue warps
    constexpr int CW = 128 / CG;   // object columns per thread
    extern __shared__ __align__(1024) unsigned char fsm[];
    // 1024-byte aligned start (the swizzled operand layout needs it), as an
    // offset from the shared array so every access stays a shared-memory one
    unsigned char *base = fsm + ((1024u - (smem_u32(fsm) & 1023u)) & 1023u);
    const FastShape fs = a.fs;
    const uint32_t arec_pad = (fs.arec_bytes + 1023u) & ~1023u;
    const uint32_t rec_pad = (fs.rec_bytes + 1023u) & ~1023u;
    unsigned char *B0 = base + arec_pad;
    // KS: chunk stages at B0 (1024-aligned), then the tail buffers
    unsigned char *T0 = B0 + (KS ? (size_t)a.nsc * kFChunkBytes : 0);
    unsigned short *heap = reinterpret_cast<unsigned short *>(KS ? T0 + kFS * kFTailPad : B0 + kFS * rec_pad);
    FastCtl &ctl = *reinterpret_cast<FastCtl *>(heap + (KH > 0 ? 0 : NT * a.k));
    // staging area: a.st_cap entries (slot, lower bound, margin), pcap per
    // epilogue thread
    const int st_cap = a.st_cap, pcap = st_cap / NT;
    int *stg_slot = reinterpret_cast<int *>(&ctl + 1);
    float *stg_lb = reinterpret_cast<float *>(stg_slot + st_cap);
    unsigned short *stg_m = reinterpret_cast<unsigned short *>(stg_lb + st_cap);

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const bool producer = warp == NEW;
    const int lq = t & 127, g = t >> 7;
    const int k = a.k;

    if (t == 0) {
        for (int s = 0; s < kFS; s++) {
            mbar_init(&ctl.full[s], 1);
            mbar_init(&ctl.efree[s], NEW);
        }
        for (int s = 0; s < kFS; s++) mbar_init(&ctl.mmad[s], 1);
        for (int s = 0; s < kFS; s++) mbar_init(&ctl.tfull[s], 1);
        for (int s = 0; s < kFSCMax; s++) {
            mbar_init(&ctl.cfull[s], 1);
            mbar_init(&ctl.cfree[s], 1);
        }
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
    // producer bookkeeping (lane 0 of the producer warp), for the bounded
    // drain on error: last block whose copy was issued / waited, last block
    // whose MMA chain was committed, tile copies issued / waited
    long long c_iss = -1, c_wait = -1, m_iss = -1;
    int a_iss = 0, a_wait = 0;
    // streamed form: K-chunk units run through the pipeline, last chunk copy
    // issued / waited, last unit whose MMAs were committed, last tail issued
    long long gunit = 0, u_iss = -1, u_wait = -1, u_mma = -1, t_iss = -1;
    unsigned long long blocks_done = 0, appended = 0;

    // guided self-scheduling (thread 0): a CTA claims a run of consecutive
    // items, about half the remaining items over twice the CTAs (one item at
    // the end); consecutive items mostly belong to one tile, whose query
    // operand then stays in shared memory
    int c_next = 0, c_end = 0;
    // producer lane 0: the tile whose query operand is in shared memory
    int a_tile = -1;
    for (;;) {
        if (t == 0) {
            const int nfull = a.n_items[0], total = nfull + a.n_items[1];
            if (c_next >= c_end) {
                const int done = *(volatile const int *)a.item_counter;
                const int chunk = max(1, (total - done) / (2 * (int)gridDim.x));
                c_next = atomicAdd(a.item_counter, chunk);
                c_end = min(c_next + chunk, total);
            }
            const int it = c_next++;
            int tile = -1, nblk = 0;
            if (it < total) {
                const int2 e = it < nfull ? a.items[it] : a.items[a.items_cap - 1 - (it - nfull)];
                tile = e.x;
                nblk = min(a.item, min(a.bcnt[tile], a.nbcap) - e.y);
                for (int j = 0; j < nblk; j++) ctl.blk[j] = a.blist[(size_t)tile * a.nbcap + e.y + j];
            }
            ctl.tile = tile;
            ctl.nblk = nblk;
        }
        if (t < kFT) ctl.r2s[t] = __float_as_int(FLT_MAX);
        __syncthreads();
        const int tile = ctl.tile, nblk = ctl.nblk;
        int nst = 0;   // candidates this (epilogue) thread staged in this item
        if (tile < 0 || ctl.err) break;
        const int4 *tinfo = reinterpret_cast<const int4 *>(a.arec + (size_t)tile * fs.arec_bytes + 2 * fs.atile_bytes);

        if (producer && KS) {
            if (lane == 0) {
                const int nk = fs.nk, SC = a.nsc, total = nblk * nk;
                auto issue_chunk = [&](int u) {   // unit u: chunk u % nk of the item's block u / nk
                    const long long gu = gunit + u;
                    const int s = (int)(gu % SC);
                    const int blk = ctl.blk[u / nk];
                    mbar_arrive_expect_tx(&ctl.cfull[s], (uint32_t)kFChunkBytes);
                    bulk_g2s(B0 + (size_t)s * kFChunkBytes,
                             a.recs + (size_t)blk * fs.rec_bytes + (size_t)(u % nk) * kFChunkBytes,
                             (uint32_t)kFChunkBytes, &ctl.cfull[s]);
                    u_iss = gu;
                };
                // the query operand, unless this tile's is in shared memory already
                const bool need_a = tile != a_tile;
                if (need_a) {
                    mbar_arrive_expect_tx(&ctl.afull, fs.arec_bytes);
                    bulk_g2s(base, a.arec + (size_t)tile * fs.arec_bytes, fs.arec_bytes, &ctl.afull);
                    a_iss++;
                }
                // chunk stages are free at an item start (the CTA synchronised
                // after every MMA of the last item was consumed)
                for (int u = 0; u < SC && u < total; u++) issue_chunk(u);
                int err = 0;
                if (need_a) {
                    if (!mbar_wait(&ctl.afull, (uint32_t)(a_wait & 1), kFWait)) err = 1;
                    else {
                        a_wait++;
                        a_tile = tile;
                    }
                }
                const uint64_t dah = smem_desc_sw128(a_hi_s, 1024), dal = smem_desc_sw128(a_lo_s, 1024);
                for (int j = 0; j < nblk && !err; j++) {
                    const long long gi = gblk + j;
                    const int acc = (int)(gi % kFS);
                    const int blk = ctl.blk[j];
                    // accumulator and tail buffer acc: free once the epilogue of
                    // block gi - 3 is done
                    if (gi >= kFS) {
                        const long long gp = gi - kFS;
                        if (!mbar_wait(&ctl.efree[acc], (uint32_t)((gp / kFS) & 1), kFWait)) { err = 3; break; }
                    }
                    mbar_arrive_expect_tx(&ctl.tfull[acc], kFTailBytes);
                    bulk_g2s(T0 + (size_t)acc * kFTailPad, a.recs + (size_t)blk * fs.rec_bytes + fs.btile_bytes,
                             kFTailBytes, &ctl.tfull[acc]);
                    t_iss = gi;
                    const uint32_t dt = tmem + (uint32_t)(acc * kFAccCols);
                    for (int c = 0; c < nk; c++) {
                        const int u = j * nk + c;
                        const long long gu = gunit + u;
                        const int s = (int)(gu % SC);
                        if (!mbar_wait(&ctl.cfull[s], (uint32_t)((gu / SC) & 1), kFWait)) { err = 2; break; }
                        u_wait = gu;
                        tc_fence_after();
                        const uint64_t db = smem_desc_sw128(smem_u32(B0 + (size_t)s * kFChunkBytes), 1024);
#pragma unroll
                        for (int kk = 0; kk < 4; kk++) {
                            const uint64_t ao = ((uint64_t)c * (kFT * 128u) + (uint64_t)kk * 32u) >> 4;
                            mma_bf16(dt, dah + ao, db + (((uint64_t)kk * 32u) >> 4), idesc, (c | kk) ? 1u : 0u);
                        }
#pragma unroll
                        for (int kk = 0; kk < 4; kk++) {
                            const uint64_t ao = ((uint64_t)c * (kFT * 128u) + (uint64_t)kk * 32u) >> 4;
                            mma_bf16(dt, dal + ao, db + (((uint64_t)kk * 32u) >> 4), idesc, 1u);
                        }
                        mma_commit(&ctl.cfree[s]);
                        u_mma = gu;
                        // refill the previous unit's stage (its MMAs retire first)
                        if (u >= 1 && u - 1 + SC < total) {
                            const long long gp = gu - 1;
                            if (!mbar_wait(&ctl.cfree[gp % SC], (uint32_t)((gp / SC) & 1), kFWait)) {
                                err = 5;
                                break;
                            }
                            issue_chunk(u - 1 + SC);
                        }
                    }
                    if (err) break;
                    mma_commit(&ctl.mmad[acc]);
                    m_iss = gi;
                }
                if (err) atomicMax(&ctl.err, err);
                blocks_done += nblk;
            }
            __syncwarp();
        } else if (producer) {
            if (lane == 0) {
                // block gi uses stage gi % 3 and TMEM accumulator gi % 3; its
                // copy waits for the epilogue of block gi - 3 (which frees both)
                auto issue_copy = [&](long long gi) {
                    const int s = (int)(gi % kFS);
                    const int blk = ctl.blk[(int)(gi - gblk)];
                    mbar_arrive_expect_tx(&ctl.full[s], fs.rec_bytes);
                    bulk_g2s(B0 + (size_t)s * rec_pad, a.recs + (size_t)blk * fs.rec_bytes, fs.rec_bytes,
                             &ctl.full[s]);
                    c_iss = gi;
                };
                const bool need_a = tile != a_tile;
                if (need_a) {
                    mbar_arrive_expect_tx(&ctl.afull, fs.arec_bytes);
                    bulk_g2s(base, a.arec + (size_t)tile * fs.arec_bytes, fs.arec_bytes, &ctl.afull);
                    a_iss++;
                }
                // stages are free at an item start (the CTA synchronised)
                for (int j = 0; j < 2 && j < nblk; j++) issue_copy(gblk + j);
                int err = 0;
                if (need_a) {
                    if (!mbar_wait(&ctl.afull, (uint32_t)(a_wait & 1), kFWait)) err = 1;
                    else {
                        a_wait++;
                        a_tile = tile;
                    }
                }
                // operand descriptors: the start-address field (address >> 4,
                // 14 bits; shared memory is below 256 KB) advances by adding
                const uint64_t dah = smem_desc_sw128(a_hi_s, 1024), dal = smem_desc_sw128(a_lo_s, 1024);
                const int ksteps = fs.kp / 16;
                for (int j = 0; j < nblk && !err; j++) {
                    const long long gi = gblk + j;
                    const int s = (int)(gi % kFS);
                    if (!mbar_wait(&ctl.full[s], (uint32_t)((gi / kFS) & 1), kFWait)) { err = 2; break; }
                    c_wait = gi;
                    tc_fence_after();
                    const uint64_t db = smem_desc_sw128(smem_u32(B0 + (size_t)s * rec_pad), 1024);
                    const uint32_t dt = tmem + (uint32_t)(s * kFAccCols);
                    for (int kk = 0; kk < ksteps; kk++) {
                        const uint64_t ao = ((uint64_t)(kk >> 2) * (kFT * 128u) + (uint64_t)(kk & 3) * 32u) >> 4;
                        const uint64_t bo = ((uint64_t)(kk >> 2) * (kFN * 128u) + (uint64_t)(kk & 3) * 32u) >> 4;
                        mma_bf16(dt, dah + ao, db + bo, idesc, kk > 0 ? 1u : 0u);
                    }
                    for (int kk = 0; kk < ksteps; kk++) {
                        const uint64_t ao = ((uint64_t)(kk >> 2) * (kFT * 128u) + (uint64_t)(kk & 3) * 32u) >> 4;
                        const uint64_t bo = ((uint64_t)(kk >> 2) * (kFN * 128u) + (uint64_t)(kk & 3) * 32u) >> 4;
                        mma_bf16(dt, dal + ao, db + bo, idesc, 1u);
                    }
                    mma_commit(&ctl.mmad[s]);
                    m_iss = gi;
                    if (j + 2 < nblk) {
                        // stage (gi + 2) % 3 was last used by block gi - 1
                        if (j >= 1) {
                            const long long gp = gi - 1;
                            if (!mbar_wait(&ctl.efree[gp % kFS], (uint32_t)((gp / kFS) & 1), kFWait)) {
                                err = 3;
                                break;
                            }
                        }
                        issue_copy(gi + 2);
                    }
                }
                if (err) atomicMax(&ctl.err, err);
                blocks_done += nblk;
            }
            __syncwarp();
        } else {
            // ---- epilogue: one query lane, CW object columns
            const int4 inf = tinfo[lq];
            const int qi = inf.x;
            const float q2 = __int_as_float(inf.y), qn = __int_as_float(inf.z);
            const float cr = 2.f * kEpsR * eps_scale(fs.kp) * qn;
            float hreg[KH > 0 ? KH : 1];
            if constexpr (KH > 0) {
#pragma unroll
                for (int h = 0; h < KH; h++) hreg[h] = h < k ? FLT_MAX : -FLT_MAX;
            } else {
                for (int i = 0; i < k; i++) heap[i * NT + t] = 0x7f80u;   // +inf
            }
            // the query's bound as published so far (its seed, tightened by
            // items of the same tile that finished earlier)
            const float seed = qi >= 0 ? __int_as_float(*(volatile const int *)(a.r2_bits + qi)) : FLT_MAX;
            float R2 = seed, pub = seed;   // bound in use, last bound published
            float hmx = FLT_MAX;           // largest of this thread's k kept upper bounds
            int certain = 0;               // range: objects certainly within r
            int hidx = 0;
            const uint32_t trow = (uint32_t)(warp & 3) * 32u << 16;
            for (int j = 0; j < nblk; j++) {
                const long long gi = gblk + j;
                const int s = (int)(gi % kFS);
                const int blk = ctl.blk[j];
                // one verdict per warp: the TMEM loads below are warp-collective
                if (!__all_sync(0xffffffffu, mbar_wait(&ctl.mmad[s], (uint32_t)((gi / kFS) & 1), kFWait))) {
                    atomicMax(&ctl.err, 4);
                    break;
                }
                tc_fence_after();
                // record tail visible here (KS: in the accumulator's tail buffer)
                mbar_wait(KS ? &ctl.tfull[s] : &ctl.full[s], (uint32_t)((gi / kFS) & 1), kFWait);
                // the bound the query's other column groups have reached
                R2 = fminf(R2, __int_as_float(*(volatile const int *)&ctl.r2s[lq]));
                const float *tail = reinterpret_cast<const float *>(
                    KS ? T0 + (size_t)s * kFTailPad : B0 + (size_t)s * rec_pad + fs.btile_bytes);
                const float *wv = tail + kTailW, *dn = tail + kTailDn;
                const float cn = tail[kTailC], rb = tail[kTailRb], wb = tail[kTailWb], brad = tail[kTailRad];
                const uint32_t taddr = tmem + trow + (uint32_t)(s * kFAccCols);
                // d^2 = |q|^2 - 2 q.c + w - 2 v - 2 (q - c).d + (rounding), so with
                //   ec >= 2 |q.c error|                       (centre rows)
                //   eb =  ec + 2e-6 |q|^2 + 2 kEpsR |q| max|bf16 r| + 2e-6 max|w|
                //   A  >= 2 |q - c|                           (from the centre product)
                // every object has |d^2 - (T + w - 2 v)| <= A |d| + eb,  T = |q|^2 - 2 q.c
                uint32_t cv[4];
                __syncwarp();
                tmem_ld4_nowait(taddr + 128, cv);
                tmem_wait_ld(cv);
                const float qc = __uint_as_float(cv[0]) + __uint_as_float(cv[1]) + __uint_as_float(cv[2]);
                const float ec = 2.f * kEpsC * eps_scale(fs.kp) * qn * cn + 1e-6f;
                const float c2 = cn * cn;
                const float qmc2 = q2 - 2.f * qc + c2;
                const float A = 2.000004f * sqrtf(fmaxf(qmc2 + ec + 4e-6f * (q2 + c2), 0.f)) + 2e-6f * cn;
                const float eb = ec + 2e-6f * q2 + cr * rb + 2e-6f * wb;
                const float T = q2 - 2.f * qc - eb;
                // ball test: |q - o| >= |q - c| - radius for every object, so a
                // block entirely beyond the bound is skipped for this query (and
                // by the whole warp when no lane of it needs the block)
                const float dlo = sqrtf(fmaxf(qmc2 - ec - 4e-6f * (q2 + c2), 0.f)) * 0.999999f - brad;
                const bool skip = qi < 0 || (dlo > 0.f && dlo * dlo * 0.999999f > R2);
                const bool warp_skip = __all_sync(0xffffffffu, skip);
#pragma unroll 1
                for (int c = g * CW; c < (g + 1) * CW && !warp_skip; c += 16) {
                    uint32_t r[16];
                    __syncwarp();   // tcgen05.ld is warp-collective: reconverge after the appends
                    tmem_ld16_nowait(taddr + (uint32_t)c, r);
                    tmem_wait_ld(r);
                    uint32_t pass = 0, inside = 0;
                    const float RT = R2 - T;
                    // range: ub < r2lo, with the comparison's own rounding covered
                    const float RLT = a.r2lo - T - 2e-6f * q2;
#pragma unroll
                    for (int u4 = 0; u4 < 4; u4++) {
                        const float4 w4 = *reinterpret_cast<const float4 *>(wv + c + 4 * u4);
                        const float4 d4 = *reinterpret_cast<const float4 *>(dn + c + 4 * u4);
                        const float wq[4] = {w4.x, w4.y, w4.z, w4.w}, dq[4] = {d4.x, d4.y, d4.z, d4.w};
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            const int u = 4 * u4 + e;
                            // lb - T; padding objects have w = +inf and never pass
                            const float x = fmaf(-2.f, __uint_as_float(r[u]), fmaf(-A, dq[e], wq[e]));
                            pass |= (x <= RT ? 1u : 0u) << u;
                            if constexpr (RANGE) inside |= (x + 2.f * fmaf(A, dq[e], eb) < RLT ? 1u : 0u) << u;
                        }
                    }
                    if (skip) pass = inside = 0;
                    if constexpr (RANGE) {
                        pass &= ~inside;
                        certain += __popc(inside);
                    }
                    // staging: each thread appends to its own slice of the
                    // staging area (entry e of thread t at e * NT + t), no
                    // atomics; past its slice, straight to the query's list
                    if (!__any_sync(0xffffffffu, pass != 0)) continue;
                    if (!pass) continue;
                    appended += __popc(pass);
#pragma unroll
                    for (int u = 0; u < 16; u++) {
                        if (!((pass >> u) & 1u)) continue;
                        const int jj = c + u;
                        const float dj = dn[jj];
                        const float lb = T + fmaf(-2.f, __uint_as_float(r[u]), fmaf(-A, dj, wv[jj]));
                        const float ub = lb + 2.f * fmaf(A, dj, eb);
                        const int slot = blk * kFB + jj;
                        if (nst < pcap) {
                            const int e = nst * NT + t;
                            stg_slot[e] = slot;
                            stg_lb[e] = lb;
                            stg_m[e] = __half_as_ushort(__float2half_ru(ub - lb));
                            nst++;
                        } else {
                            const int gsl = atomicAdd(&a.cand_cnt[qi], 1);
                            if (gsl < kFCand) {
                                a.cand_pos[(size_t)qi * kFCand + gsl] = slot;
                                a.cand_lb[(size_t)qi * kFCand + gsl] = lb;
                                a.cand_ub[(size_t)qi * kFCand + gsl] = ub;
                            }
                        }
                        if (!RANGE && ub < R2) {   // replace the largest of the k kept bounds
                            float mx = -FLT_MAX;
                            if constexpr (KH > 0) {
                                int mi = 0;
#pragma unroll
                                for (int h = 0; h < KH; h++) {
                                    if (h == hidx) hreg[h] = ub;
                                    if (hreg[h] > mx) { mx = hreg[h]; mi = h; }
                                }
                                hidx = mi;
                            } else {
                                // binary max-heap in shared memory: the root
                                // (the largest kept bound) is replaced and
                                // sifted down, log2(k) levels
                                // (non-negative floats order like their
                                // bit patterns)
                                const uint32_t ubits = __float_as_uint(fmaxf(ub, 0.f));
                                const unsigned short v = (unsigned short)((ubits + 0xffffu) >> 16);
                                int i = 0;
                                for (;;) {
                                    const int l = 2 * i + 1;
                                    if (l >= k) break;
                                    unsigned short cv = heap[l * NT + t];
                                    int c = l;
                                    if (l + 1 < k) {
                                        const unsigned short rv = heap[(l + 1) * NT + t];
                                        if (rv > cv) { cv = rv; c = l + 1; }
                                    }
                                    if (cv <= v) break;
                                    heap[i * NT + t] = cv;
                                    i = c;
                                }
                                heap[i * NT + t] = v;
                                mx = __uint_as_float((uint32_t)heap[t] << 16);
                            }
                            hmx = mx;
                            R2 = fminf(R2, mx);
                        }
                    }
                }
                // k distinct objects' upper bounds bound the query's k-th d^2
                if (!RANGE && qi >= 0 && hmx < pub) {
                    atomicMin(a.r2_bits + qi, __float_as_int(fmaxf(hmx, 0.f)));
                    if (CG > 1) atomicMin(&ctl.r2s[lq], __float_as_int(fmaxf(hmx, 0.f)));
                    pub = hmx;
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&ctl.efree[s]);
            }
            if (RANGE && qi >= 0 && certain) atomicAdd(a.rcnt + qi, certain);
        }
        gblk += nblk;
        if (KS) gunit += (long long)nblk * fs.nk;
        tc_fence_before();
        __syncthreads();   // item done: every MMA consumed, stages and A free
        tc_fence_after();
        // flush the staged candidates: one list reservation per query lane,
        // then each thread writes its own slice after its lane's earlier
        // column groups
        if (t < NT) ctl.th_cnt[t] = nst;
        __syncthreads();
        if (t < kFT) {
            int c = 0;
#pragma unroll
            for (int g2 = 0; g2 < CG; g2++) c += ctl.th_cnt[t + kFT * g2];
            const int qi = tinfo[t].x;
            ctl.qbase[t] = (c > 0 && qi >= 0) ? atomicAdd(&a.cand_cnt[qi], c) : 0;
        }
        __syncthreads();
        if (t < NT && nst > 0) {
            const int qi = tinfo[lq].x;
            int at = ctl.qbase[lq];
            for (int g2 = 0; g2 < g; g2++) at += ctl.th_cnt[lq + kFT * g2];
            for (int e = 0; e < nst && at < kFCand; e++, at++) {
                const int x = e * NT + t;
                const float lb = stg_lb[x];
                const float margin = __half2float(__ushort_as_half(stg_m[x]));
                a.cand_pos[(size_t)qi * kFCand + at] = stg_slot[x];
                a.cand_lb[(size_t)qi * kFCand + at] = lb;
                a.cand_ub[(size_t)qi * kFCand + at] = __fadd_ru(lb, margin);
            }
        }
        __syncthreads();
    }
    if (producer && lane == 0 && ctl.err) {
        // let copies and MMAs still in flight finish before the CTA leaves (bounded)
        for (long long gi = c_wait + 1; gi <= c_iss; gi++)
            mbar_wait(&ctl.full[gi % kFS], (uint32_t)((gi / kFS) & 1), kFWait);
        if (a_wait < a_iss) mbar_wait(&ctl.afull, (uint32_t)((a_iss - 1) & 1), kFWait);
        if (m_iss >= 0) mbar_wait(&ctl.mmad[m_iss % kFS], (uint32_t)((m_iss / kFS) & 1), kFWait);
        if (KS) {
            const int SC = a.nsc;
            for (long long gu = u_wait + 1; gu <= u_iss; gu++)
                mbar_wait(&ctl.cfull[gu % SC], (uint32_t)((gu / SC) & 1), kFWait);
            if (u_mma >= 0) mbar_wait(&ctl.cfree[u_mma % SC], (uint32_t)((u_mma / SC) & 1), kFWait);
            for (long long gi = t_iss - kFS + 1 > 0 ? t_iss - kFS + 1 : 0; gi <= t_iss; gi++)
                mbar_wait(&ctl.tfull[gi % kFS], (uint32_t)((gi / kFS) & 1), kFWait);
        }
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

// One CTA (4 warps) per query.  The bound drops to the k-th smallest
// candidate upper bound (the candidates are distinct objects); every
// candidate whose lower bound is within it gets its reference-arithmetic
// distance; top k by (distance, id).  Queries that cannot be answered from
// their list (it overflowed, or fewer than k exact values lie inside the
// bound because a learned seed was too small) are listed in overflow.
//
// The reference value of a candidate is a sequential F64 sum of
// pow(o_j - q_j, 2) over j: in batches of kFinB candidates, the four warps
// evaluate the terms (coalesced rows) into shared memory and lane c of warp 0
// adds candidate c's terms in j order, so the sums of a batch run side by
// side, each in the sequential order.
constexpr int kFinB = 16;

// KPM: the widest row the term buffer holds (kFResKp or kFMaxKp); FINB
// candidates per batch (the buffer, FINB x (KPM + 1) doubles, stays within
// the static shared memory).  CAP: the candidates one CTA holds.  Most
// queries list fewer than 128, so a light variant (CAP = 128, a fraction of
// the shared memory: twice the CTAs per SM to hide the row loads) runs
// first over every query and lists the queries with more in `heavy`; the
// full variant (CAP = kFCand) then runs over that list (`only`, *n_only of
// them, a persistent grid walking the list).
template <int KPM, int FINB, int CAP>
__global__ void __launch_bounds__(128) k_fast_final(const float *__restrict__ rows, int dim, int num,
                                                    const float *__restrict__ prow, int kp,
                                                    const int *__restrict__ ids_of_slot, int nslots,
                                                    const int *__restrict__ qids, int k, int infi_dis,
                                                    const int *__restrict__ cand_pos,
                                                    const float *__restrict__ cand_lb,
                                                    const float *__restrict__ cand_ub,
                                                    const int *__restrict__ cand_cnt,
                                                    const int *__restrict__ r2_bits, float *kth, int *ids,
                                                    float *dists, int *overflow, int *n_overflow,
                                                    int *heavy, int *n_heavy, const int *only,
                                                    const int *n_only, unsigned long long *stats)
{
    __shared__ double cd[CAP];
    __shared__ int cid[CAP];
    __shared__ int cl[CAP];
    // the upper bounds (dead once the bound is set) share their space with the
    // pow terms; +1 double per row: lane c's reads of column j miss each
    // other's banks
    constexpr int kTermsBytes = FINB * (KPM + 1) * 8;
    __shared__ __align__(16) unsigned char scratch[kTermsBytes > 4 * CAP ? kTermsBytes : 4 * CAP];
    float *ubs = reinterpret_cast<float *>(scratch);
    double(*terms)[KPM + 1] = reinterpret_cast<double(*)[KPM + 1]>(scratch);
    __shared__ int ns;
    __shared__ float kub;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int nwork = only ? *n_only : (int)gridDim.x;
    for (int wi = blockIdx.x; wi < nwork; wi += gridDim.x) {
    __syncthreads();   // the previous query's shared state is consumed
    const int q = only ? only[wi] : wi;
    const int qid = qids[q];
    const int cnt = cand_cnt[q];
    if (cnt > CAP) {
        if (t == 0) {
            if (CAP < kFCand && cnt <= kFCand) heavy[atomicAdd(n_heavy, 1)] = q;
            else overflow[atomicAdd(n_overflow, 1)] = q;
        }
        continue;
    }
    float R2 = __int_as_float(r2_bits[q]);
    if (cnt >= k && cnt <= 128) {
        // k-th smallest upper bound: warp 0 holds four per lane and takes
        // out the smallest k - 1 times (one occurrence each)
        if (warp == 0) {
            float v[4];
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const int i = lane + 32 * m;
                v[m] = i < cnt ? cand_ub[(size_t)q * kFCand + i] : INFINITY;
            }
            float mn = INFINITY;
            for (int it = 0; it < k; it++) {
                const float lm = fminf(fminf(v[0], v[1]), fminf(v[2], v[3]));
                mn = lm;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
                if (it == k - 1) break;
                const unsigned own = __ballot_sync(0xffffffffu, lm == mn);
                if (lane == __ffs(own) - 1) {
                    if (v[0] == mn) v[0] = INFINITY;
                    else if (v[1] == mn) v[1] = INFINITY;
                    else if (v[2] == mn) v[2] = INFINITY;
                    else v[3] = INFINITY;
                }
            }
            if (lane == 0) kub = mn;
        }
        __syncthreads();
        R2 = fminf(R2, kub);
    } else if (cnt >= k) {
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
    for (int i = t; i < cnt; i += 128) {
        if (cand_lb[(size_t)q * kFCand + i] > R2) continue;
        const int slot = cand_pos[(size_t)q * kFCand + i];
        if (slot < 0 || slot >= nslots) continue;
        const int id = ids_of_slot[slot];
        if (id < 0 || id >= num) continue;
        cl[atomicAdd(&ns, 1)] = slot;
    }
    __syncthreads();
    const int n = ns;
    const float *qrow = rows + (size_t)qid * dim;
    // every object whose d^2 is within the bound is a candidate, and the
    // reference value differs from d^2 by < 1e-6 relative: the answer is
    // exact once k candidates have reference values inside R2 (1 - 1e-6)
    const double lim = (double)R2 * (1.0 - 1e-6);
    // Pass 0 sums exact squares e * e (a float difference squared
    // is exact in FP64) instead of pow(e, 2).  pow is within 2 ulp of the
    // square, so over dim <= 320 terms the sequential sums differ by less
    // than 7.2e-14 relative and the distances by less than 3.6e-14; with the
    // margin delta = 1e-13 v the pass-0 values give the reference's float
    // values, order and bound tests unless some value lies within delta of a
    // float rounding midpoint, of another candidate's value or of the bound.
    // Then pass 1 evaluates pow itself.  More than 32 candidates are sorted
    // by (distance, id) here (bitonic), so near-ties are neighbours.
    __shared__ int risky;
    if (t == 0) risky = 0;
    int p2 = 1;
    while (p2 < n) p2 <<= 1;
    for (int pass = 0; pass < 2; pass++) {
        for (int b0 = 0; b0 < n; b0 += FINB) {
            const int nb = min(FINB, n - b0);
            for (int c = warp; c < nb; c += 4) {
                const float *orow = prow + (size_t)cl[b0 + c] * kp;
                if (pass == 0) {
                    for (int j = lane; j < dim; j += 32) {
                        const double e = (double)(orow[j] - qrow[j]);
                        terms[c][j] = e * e;
                    }
                } else {
                    for (int j = lane; j < dim; j += 32) terms[c][j] = pow(orow[j] - qrow[j], 2);
                }
            }
            __syncthreads();
            if (warp == 0 && lane < nb) {
                const int id = ids_of_slot[cl[b0 + lane]];
                double r = 0.0;
#pragma unroll 4
                for (int j = 0; j < dim; j++) r += terms[lane][j];
                const double v = id == qid ? 0.0 : pow(r, 0.5);
                cd[b0 + lane] = v;
                cid[b0 + lane] = id;
                if (pass == 0 && v != 0.0) {
                    // the float midpoints around (float)v must stay beyond delta
                    const float f = __double2float_rn(v);
                    const double fd = f;
                    const double mhi = 0.5 * (fd + (double)__int_as_float(__float_as_int(f) + 1));
                    const double mlo = 0.5 * (fd + (double)__int_as_float(__float_as_int(f) - 1));
                    const double dl = v * 1e-13;
                    const double v2 = v * v;
                    if (!(f > 0.f && v - dl > mlo && v + dl < mhi) || fabs(v2 - lim) <= 3e-13 * lim) risky = 1;
                }
            }
            __syncthreads();
        }
        // near-ties: two values closer than their margins (exact zeros are
        // exact in both sums)
        if (n <= 32) {
            if (pass == 0 && warp == 0) {
                const double d = lane < n ? cd[lane] : 0.0;
                bool rk = false;
                for (int j = 0; j < n; j++) {
                    const double dj = __shfl_sync(0xffffffffu, d, j);
                    if (lane < n && j != lane && !(d == 0.0 && dj == 0.0) && fabs(dj - d) <= (d + dj) * 1e-13) rk = true;
                }
                if (__any_sync(0xffffffffu, rk) && lane == 0) risky = 1;
            }
        } else {
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
            if (pass == 0)
                for (int i = t; i + 1 < n; i += 128) {
                    const double d = cd[i], dj = cd[i + 1];
                    if (!(d == 0.0 && dj == 0.0) && dj - d <= (d + dj) * 1e-13) risky = 1;
                }
        }
        __syncthreads();
        if (pass == 1 || !risky) break;
    }
    if (t == 0 && stats) atomicAdd(&stats[2], (unsigned long long)n);
    if (n <= 32) {
        // rank of each candidate by (distance, id) within warp 0
        if (warp == 0) {
            const double d = lane < n ? cd[lane] : DBL_MAX;
            const int id = lane < n ? cid[lane] : 0x7fffffff;
            int rank = 0;
            for (int j = 0; j < n; j++) {
                const double dj = __shfl_sync(0xffffffffu, d, j);
                const int ij = __shfl_sync(0xffffffffu, id, j);
                rank += (dj < d) || (dj == d && ij < id);
            }
            const bool top = lane < n && rank < k;
            const int within = __popc(__ballot_sync(0xffffffffu, top && d * d <= lim));
            if (within < k && within < num) {
                if (lane == 0) overflow[atomicAdd(n_overflow, 1)] = q;
            } else {
                if (top) {
                    if (ids) ids[(size_t)q * k + rank] = id;
                    if (dists) dists[(size_t)q * k + rank] = (float)d;
                    if (rank == k - 1) kth[q] = (float)d;
                }
                for (int j = n + lane; j < k; j += 32) {
                    if (ids) ids[(size_t)q * k + j] = -1;
                    if (dists) dists[(size_t)q * k + j] = (float)infi_dis;
                }
                if (n < k && lane == 0) kth[q] = (float)infi_dis;
            }
        }
        continue;
    }
    // sorted above
    if (t == 0) {
        int within = 0;
        for (int i = 0; i < n && i < k; i++) within += cd[i] * cd[i] <= lim;
        if (within < k && within < num) overflow[atomicAdd(n_overflow, 1)] = q;
        else kth[q] = n >= k ? (float)cd[k - 1] : (float)infi_dis;
        ns = within < k && within < num ? -1 : 0;
    }
    __syncthreads();
    if (ns < 0) continue;
    for (int j = t; j < k; j += 128) {
        if (ids) ids[(size_t)q * k + j] = j < n ? cid[j] : -1;
        if (dists) dists[(size_t)q * k + j] = j < n ? (float)cd[j] : (float)infi_dis;
    }
    }   // for wi
}

// Sort keys of the queries: the block of their slot (tiles group queries
// by block order; the order inside a block does not matter).
// Light recheck, one warp per query, for small k (where nearly every query
// lists at most 32 candidates), so a query needs no CTA barrier and a CTA
// runs kFinWarps queries side by side.  The tests and the arithmetic are
// k_fast_final's: the bound drops to the k-th smallest upper bound; each
// candidate within it gets its reference value (exact squares first; pow
// where a value lies near a float rounding midpoint, another value or the
// bound); ranks by (distance, id).  FB candidates at a time, the warp reads
// their rows coalesced (all loads in flight at once) and keeps the FP32
// differences o_j - q_j in shared memory; lane p then sums candidate p's
// terms in j order.  Queries with more than 32 candidates go to `heavy`
// (the full variant of k_fast_final), those whose list overflowed to
// `overflow`.
constexpr int kFinWarps = 4;
constexpr int kFinWarpK = 8;   // k up to which the warp variant runs first
template <int KPM, int FB>
__global__ void __launch_bounds__(32 * kFinWarps) k_fast_final_warp(
    const float *__restrict__ rows, int dim, int num, const float *__restrict__ prow, int kp,
    const int *__restrict__ ids_of_slot, int nslots, const int *__restrict__ qids, int qnum, int k, int infi_dis,
    const int *__restrict__ cand_pos, const float *__restrict__ cand_lb, const float *__restrict__ cand_ub,
    const int *__restrict__ cand_cnt, const int *__restrict__ r2_bits, float *kth, int *ids, float *dists,
    int *overflow, int *n_overflow, int *heavy, int *n_heavy, unsigned long long *stats)
{
    __shared__ float ew_all[kFinWarps][FB][KPM + 1];   // +1: lane p's reads of column j miss each other's banks
    __shared__ int wslot[kFinWarps][32], wid[kFinWarps][32];
    __shared__ unsigned long long nrechk;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float(*ew)[KPM + 1] = ew_all[warp];
    if (threadIdx.x == 0) nrechk = 0;
    __syncthreads();
    const int q = blockIdx.x * kFinWarps + warp;
    const int cnt = q < qnum ? cand_cnt[q] : 0;
    if (q < qnum && cnt > 32) {
        if (lane == 0) {
            if (cnt <= kFCand) heavy[atomicAdd(n_heavy, 1)] = q;
            else overflow[atomicAdd(n_overflow, 1)] = q;
        }
    } else if (q < qnum) {
        const int qid = qids[q];
        float R2 = __int_as_float(r2_bits[q]);
        const bool have = lane < cnt;
        const size_t cb = (size_t)q * kFCand + lane;
        const float ub = have ? cand_ub[cb] : INFINITY;
        const float lb = have ? cand_lb[cb] : INFINITY;
        const int slot = have ? cand_pos[cb] : -1;
        // the query's row, lane l holding columns l, l + 32, ..
        const float *qrow = rows + (size_t)qid * dim;
        float qv[KPM / 32];
#pragma unroll
        for (int m = 0; m < KPM / 32; m++) {
            const int j = lane + 32 * m;
            qv[m] = j < dim ? qrow[j] : 0.f;
        }
        if (cnt >= k) {
            // k-th smallest upper bound (with multiplicity): the lane of rank k - 1
            int rank = 0;
            for (int j = 0; j < 32; j++) {
                const float uj = __shfl_sync(0xffffffffu, ub, j);
                rank += (uj < ub) || (uj == ub && j < lane);
            }
            const unsigned who = __ballot_sync(0xffffffffu, have && rank == k - 1);
            R2 = fminf(R2, __shfl_sync(0xffffffffu, ub, __ffs(who) - 1));
        }
        bool c = have && !(lb > R2) && slot >= 0 && slot < nslots;
        int id = -1;
        if (c) {
            id = ids_of_slot[slot];
            c = id >= 0 && id < num;
        }
        // candidates packed: lane p < n holds the p-th
        const unsigned cm = __ballot_sync(0xffffffffu, c);
        const int n = __popc(cm);
        if (c) {
            const int p = __popc(cm & ((1u << lane) - 1u));
            wslot[warp][p] = slot;
            wid[warp][p] = id;
        }
        __syncwarp();
        const bool mine = lane < n;
        const int pid = mine ? wid[warp][lane] : 0x7fffffff;
        const double lim = (double)R2 * (1.0 - 1e-6);
        double d = DBL_MAX;
        for (int pass = 0; pass < 2; pass++) {
            double r = 0.0;
            for (int b0 = 0; b0 < n; b0 += FB) {
                const int nbat = min(FB, n - b0);
                float e[FB][KPM / 32];
#pragma unroll
                for (int cc = 0; cc < FB; cc++) {
                    const float *orow = prow + (size_t)(cc < nbat ? wslot[warp][b0 + cc] : 0) * kp;
#pragma unroll
                    for (int m = 0; m < KPM / 32; m++) {
                        const int j = lane + 32 * m;
                        e[cc][m] = (cc < nbat && j < dim) ? orow[j] : 0.f;
                    }
                }
#pragma unroll
                for (int cc = 0; cc < FB; cc++)
#pragma unroll
                    for (int m = 0; m < KPM / 32; m++) ew[cc][lane + 32 * m] = e[cc][m] - qv[m];
                __syncwarp();
                if (lane >= b0 && lane < b0 + nbat) {
                    const float *er = ew[lane - b0];
                    if (pass == 0) {
                        // a float difference squared is exact in FP64
#pragma unroll 8
                        for (int j = 0; j < dim; j++) {
                            const double x = (double)er[j];
                            r += x * x;
                        }
                    } else {
                        for (int j = 0; j < dim; j++) {
                            const double tj = pow(er[j], 2);
                            r += tj;
                        }
                    }
                }
                __syncwarp();
            }
            if (mine) d = pid == qid ? 0.0 : pow(r, 0.5);
            if (pass == 1) break;
            bool rk = false;
            if (mine && d != 0.0) {
                // the float midpoints around (float)d must stay beyond delta
                const float f = __double2float_rn(d);
                const double fd = f;
                const double mhi = 0.5 * (fd + (double)__int_as_float(__float_as_int(f) + 1));
                const double mlo = 0.5 * (fd + (double)__int_as_float(__float_as_int(f) - 1));
                const double dl = d * 1e-13;
                const double v2 = d * d;
                if (!(f > 0.f && d - dl > mlo && d + dl < mhi) || fabs(v2 - lim) <= 3e-13 * lim) rk = true;
            }
            // near-ties: two values closer than their margins (exact zeros are
            // exact in both sums)
            for (int j = 0; j < n; j++) {
                const double dj = __shfl_sync(0xffffffffu, d, j);
                if (mine && j != lane && !(d == 0.0 && dj == 0.0) && fabs(dj - d) <= (d + dj) * 1e-13) rk = true;
            }
            if (!__any_sync(0xffffffffu, rk)) break;
        }
        if (lane == 0 && n) atomicAdd(&nrechk, (unsigned long long)n);
        int rank = 0;
        for (int j = 0; j < n; j++) {
            const double dj = __shfl_sync(0xffffffffu, d, j);
            const int ij = __shfl_sync(0xffffffffu, pid, j);
            rank += (dj < d) || (dj == d && ij < pid);
        }
        const bool top = mine && rank < k;
        const int within = __popc(__ballot_sync(0xffffffffu, top && d * d <= lim));
        if (within < k && within < num) {
            if (lane == 0) overflow[atomicAdd(n_overflow, 1)] = q;
        } else {
            if (top) {
                if (ids) ids[(size_t)q * k + rank] = pid;
                if (dists) dists[(size_t)q * k + rank] = (float)d;
                if (rank == k - 1) kth[q] = (float)d;
            }
            for (int j = n + lane; j < k; j += 32) {
                if (ids) ids[(size_t)q * k + j] = -1;
                if (dists) dists[(size_t)q * k + j] = (float)infi_dis;
            }
            if (n < k && lane == 0) kth[q] = (float)infi_dis;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && stats && nrechk) atomicAdd(&stats[2], nrechk);
}

__global__ void k_fast_keys(const int *qids, int qnum, const int *pos_of, int *keys, int *vals)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < qnum) {
        keys[i] = pos_of[qids[i]] / kFB;
        vals[i] = i;
    }
}

// Query order of a filter run in one CTA (nb <= kOrderMaxNb): the queries
// sorted by the block of their slot (keys), ties by query index -- the order
// a stable sort gives.  A counting sort in shared memory: per-block counts,
// their exclusive scan, a scatter through shared-memory cursors; then the
// queries of each block (a few per block) put in index order by insertion
// sort.  A block with more than kOrderSortMax queries keeps their arrival
// order: the order only groups the queries into tiles, the answers do not
// depend on it.
constexpr int kOrderThreads = 1024;
constexpr int kOrderMaxNb = 24576;   // 2 x 4 bytes per block of shared memory
constexpr int kOrderSortMax = 64;
__global__ void __launch_bounds__(kOrderThreads) k_fast_order(const int *__restrict__ keys, int qnum, int nb,
                                                              int *__restrict__ order)
{
    extern __shared__ int osm[];
    int *start = osm, *cur = osm + nb;
    __shared__ int wsum[kOrderThreads / 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int b = t; b < nb; b += kOrderThreads) cur[b] = 0;
    __syncthreads();
    for (int i = t; i < qnum; i += kOrderThreads) atomicAdd(&cur[keys[i]], 1);
    __syncthreads();
    // exclusive scan of the counts: thread t sums its contiguous range of
    // blocks, the CTA scans the sums, each thread writes its range's starts
    const int per = (nb + kOrderThreads - 1) / kOrderThreads;
    const int b0 = min(nb, t * per), b1 = min(nb, b0 + per);
    int local = 0;
    for (int b = b0; b < b1; b++) local += cur[b];
    int x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int v = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        wsum[lane] = v;
    }
    __syncthreads();
    int run = (warp > 0 ? wsum[warp - 1] : 0) + x - local;
    for (int b = b0; b < b1; b++) {
        const int c = cur[b];
        start[b] = run;
        cur[b] = run;
        run += c;
    }
    __syncthreads();
    for (int i = t; i < qnum; i += kOrderThreads) order[atomicAdd(&cur[keys[i]], 1)] = i;
    __syncthreads();   // the CTA's writes to order are visible to all its threads
    for (int b = t; b < nb; b += kOrderThreads) {
        const int s0 = start[b], s1 = cur[b];
        if (s1 - s0 < 2 || s1 - s0 > kOrderSortMax) continue;
        for (int p = s0 + 1; p < s1; p++) {
            const int v = order[p];
            int q = p - 1;
            while (q >= s0 && order[q] > v) {
                order[q + 1] = order[q];
                q--;
            }
            order[q + 1] = v;
        }
    }
}

// The start of a kNN filter run in one launch.  Per query i: an empty
// candidate list, the starting bound (carry, else FLT_MAX; with selfk, the
// smaller of that and the seed table's bound for the k at column jk) and the
// sort key (the block of the query's slot) with its index; over the grid:
// the run's counters, the tiles' block counts and the superblock mask words
// cleared, and the run counted in stats[6].
__global__ void k_fast_begin(int qnum, const int *__restrict__ qids, const int *__restrict__ pos_of,
                             const int *__restrict__ selfk, int jk, const int *__restrict__ carry, int *cand_cnt,
                             int *r2_bits, int *keys, int *vals, int *ctr, int nctr, int *bcnt, int ntiles,
                             uint32_t *sb_mask, int nmask, unsigned long long *stats)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    if (i < qnum) {
        const int pos = pos_of[qids[i]];
        int r2 = carry ? carry[i] : __float_as_int(FLT_MAX);
        if (selfk) r2 = min(r2, selfk[(size_t)pos * kSelfK + jk]);   // non-negative floats order as ints
        cand_cnt[i] = 0;
        r2_bits[i] = r2;
        keys[i] = pos / kFB;
        vals[i] = i;
    }
    if (i < nctr) ctr[i] = 0;
    for (int j = i; j < ntiles; j += stride) bcnt[j] = 0;
    for (int j = i; j < nmask; j += stride) sb_mask[j] = 0u;
    if (i == 0 && stats) stats[6] += 1ull;
}

__global__ void k_add_stat(unsigned long long *p, unsigned long long v) { *p += v; }

__global__ void k_scatter_i(const int *idx, int n, const int *src, int *dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[idx[i]] = src[i];
}

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
// (k <= 16 in registers; above, threads x k 2-byte entries, at most 32 KB of
// shared memory) allow.
static int fast_cg(int k) { return k <= 32 ? 4 : 2; }

// One configuration of the fast form: seed with the learned radius or not,
// epilogue column groups (warps per query lane), blocks per work item,
// records streamed in K chunks (forced above kp = kFResKp) or resident --
// or the block-stationary filter (blk; fast_blk.cu), which has no column
// groups or items.  wfin: the light recheck one warp per query
// (k_fast_final_warp, k <= kFinWarpK) instead of one CTA per query.
struct FastCfg {
    bool learned;
    int cg, item;
    bool stream;
    bool blk;
    bool wfin;
};

static int cfg_pack(const FastCfg &c)
{
    return 1 | (c.learned ? 2 : 0) | (c.cg << 2) | (c.item << 8) | (c.stream ? 1 << 14 : 0) | (c.blk ? 1 << 15 : 0) |
           (c.wfin ? 1 << 16 : 0);
}
static FastCfg cfg_unpack(int v)
{
    return FastCfg{(v & 2) != 0, (v >> 2) & 7, (v >> 8) & 63, (v & (1 << 14)) != 0, (v & (1 << 15)) != 0,
                   (v & (1 << 16)) != 0};
}

// Filter variant of a configuration as the ABI reports it.
static int cfg_variant(const FastCfg &c) { return c.blk ? 2 : (c.stream ? 1 : 0); }

static bool fast_tile_fits(const FastShape &fs, int cg, int k, bool stream);

static FastCfg fast_default_cfg(const gts_index *idx, int k)
{
    // measured on clustered data: the own-block seed is tight for small k,
    // the learned radius pays for its re-answers from k = 16 on; the column
    // groups are the most whose shared memory fits this dimension
    const FastShape fs = fast_shape(idx->dim);
    const bool stream = fs.kp > kFResKp;
    int cg = fast_cg(k);
    while (cg > 1 && !fast_tile_fits(fs, cg, k, stream)) cg >>= 1;
    return FastCfg{idx->mlp_ready && k >= 16, cg, 16, stream};
}

// Shared memory of the filter kernel before candidate staging: the query
// tile, the block stages (whole records, or for kp > kFResKp nsc K-chunk
// stages and three tail buffers), the bound heaps (k > 16) and the control
// block.  nsc = 0 for the resident form.
static size_t fast_tile_fixed_smem(const FastShape &fs, int cg, int k, bool heap_in_smem, int nsc, bool stream)
{
    const uint32_t arec_pad = (fs.arec_bytes + 1023u) & ~1023u;
    const uint32_t rec_pad = (fs.rec_bytes + 1023u) & ~1023u;
    const size_t heap = heap_in_smem ? sizeof(unsigned short) * 128 * cg * (size_t)k : 0;
    const size_t stages = (fs.kp > kFResKp || stream) ? (size_t)nsc * kFChunkBytes + kFS * (size_t)kFTailPad
                                                      : kFS * (size_t)rec_pad;
    return 1024 + (size_t)arec_pad + stages + heap + sizeof(FastCtl) + 64;
}

static int smem_optin()
{
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return optin;
}

// K-chunk stages of the streamed form that fit beside candidate staging of
// at least two entries per epilogue thread (at most kFSCMax); 0 when not
// even two fit.
static int fast_tile_stages(const FastShape &fs, int cg, int k, bool heap_in_smem)
{
    const size_t optin = (size_t)smem_optin();
    for (int nsc = kFSCMax; nsc >= 2; nsc--)
        if (fast_tile_fixed_smem(fs, cg, k, heap_in_smem, nsc, true) + 2 * kFT * cg * kStagedBytes <= optin)
            return nsc;
    return 0;
}

// The filter configuration (column groups cg, bound heap in shared memory
// for k > 16) fits this index's shared-memory plan.
static bool fast_tile_fits(const FastShape &fs, int cg, int k, bool stream)
{
    const bool heap = k > 16;
    if (fs.kp > kFResKp || stream) return fast_tile_stages(fs, cg, k, heap) >= 2;
    return fast_tile_fixed_smem(fs, cg, k, heap, 0, false) + 2 * kFT * cg * kStagedBytes <= (size_t)smem_optin();
}

template <int CG, int KH, bool RANGE = false, bool KS = false>
static int launch_fast_tile_cg(const FastTileArgs &a, int grid, cudaStream_t st)
{
    FastTileArgs b = a;
    b.nsc = KS ? fast_tile_stages(a.fs, CG, a.k, KH == 0) : 0;
    if (KS && b.nsc < 2) {
        gts_set_error("tensor-core filter: kp %d leaves no room for two K-chunk stages (%d column groups, k %d)",
                      a.fs.kp, CG, a.k);
        return GTS_ERR_INVALID;
    }
    const size_t fixed = fast_tile_fixed_smem(a.fs, CG, a.k, KH == 0, b.nsc, KS);
    const int optin = smem_optin();
    b.st_cap = (int)std::min<size_t>(kFStageMax, optin > (int)fixed ? ((size_t)optin - fixed) / kStagedBytes : 0);
    b.st_cap -= b.st_cap % (kFT * CG);   // whole slices per epilogue thread
    if (b.st_cap < kFT * CG) {
        gts_set_error("tensor-core filter: %zu bytes of shared memory leave no room for candidate staging", fixed);
        return GTS_ERR_INVALID;
    }
    const size_t smem = fixed + kStagedBytes * (size_t)b.st_cap;
    GTS_CUDA_TRY(cudaFuncSetAttribute(k_fast_tile<CG, KH, RANGE, KS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    k_fast_tile<CG, KH, RANGE, KS><<<grid, 128 * CG + 32, smem, st>>>(b);
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

template <int CG, int KH, bool RANGE = false>
static int launch_fast_tile_ks(const FastTileArgs &a, int grid, cudaStream_t st)
{
    return (a.fs.kp > kFResKp || a.stream) ? launch_fast_tile_cg<CG, KH, RANGE, true>(a, grid, st)
                                           : launch_fast_tile_cg<CG, KH, RANGE, false>(a, grid, st);
}

static int launch_fast_tile(const FastTileArgs &a, int cg, int grid, cudaStream_t st)
{
    // k <= 16: the k kept bounds live in registers
    if (a.k <= 8) {
        switch (cg) {
        case 4: return launch_fast_tile_ks<4, 8>(a, grid, st);
        case 2: return launch_fast_tile_ks<2, 8>(a, grid, st);
        default: return launch_fast_tile_ks<1, 8>(a, grid, st);
        }
    }
    if (a.k <= 16) {
        switch (cg) {
        case 4: return launch_fast_tile_ks<4, 16>(a, grid, st);
        case 2: return launch_fast_tile_ks<2, 16>(a, grid, st);
        default: return launch_fast_tile_ks<1, 16>(a, grid, st);
        }
    }
    switch (cg) {
    case 4: return launch_fast_tile_ks<4, 0>(a, grid, st);
    case 2: return launch_fast_tile_ks<2, 0>(a, grid, st);
    default: return launch_fast_tile_ks<1, 0>(a, grid, st);
    }
}

bool fast_supported(const gts_index *idx, int k)
{
    return idx->metric == kL2 && idx->dim <= kFMaxKp && k >= 1 && k <= kFMaxK && idx->num >= 1;
}

static int fast_prepare(gts_index *idx, cudaStream_t st)
{
    if (idx->fast_recs) return GTS_OK;
    const FastShape fs = fast_shape(idx->dim);
    FastOrder ord;
    int rc = fast_block_order(idx, &ord, st);
    if (rc) return rc;
    const int nb = ord.nb, nsb = ord.nsb;
    if ((long long)nb * kFB >= (1ll << 25)) {   // staged candidates carry the slot in 25 bits
        gts_set_error("tensor-core filter: %d blocks exceed the %d slots of the candidate format", nb, 1 << 25);
        return GTS_ERR_INVALID;
    }
    const size_t bytes = fast_bytes(fs, nb, nsb, idx->num);
    unsigned char *recs = nullptr;
    if ((rc = dev_alloc(&recs, bytes, nullptr))) return rc;
    GTS_CUDA_TRY(cudaMemsetAsync(recs, 0, bytes, st));
    const FastSummary bs = fast_summary(recs, fs, nb, nsb, idx->num);
    k_fast_layout<<<nb, kFB, 0, st>>>(ord.perm, ord.blk_l, ord.blk_r, bs.ids, bs.pos);
    GTS_CUDA_TRY(cudaMemcpyAsync(bs.sb_b0, ord.sb_b0, sizeof(int) * (nsb + 1), cudaMemcpyDeviceToDevice, st));
    k_fast_prep<<<nb, kFB, 0, st>>>(idx->dim, idx->rows, recs, fs, bs);
    k_fast_prows<<<nb, kFB, 0, st>>>(idx->dim, fs.kp, idx->rows, bs.ids, bs.prow);
    k_fast_sbprep<<<nsb, 256, 0, st>>>(idx->dim, idx->rows, fs, bs);
    // the seed table: neighbour blocks by centre, then per object the k-th
    // distances over its block and those
    const size_t nbrs_smem = sizeof(float) * ((size_t)kNbrWarps * fs.kp + 32 * (size_t)(fs.kp + 4));
    const size_t selfk_smem =
        sizeof(float) * ((size_t)kFB * (fs.kp + 4) + (size_t)kFB * kSeedBest + 4 * (size_t)(fs.kp + 3 * kSeedBest));
    cudaError_t e = cudaFuncSetAttribute(k_fast_nbrs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)nbrs_smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_fast_selfk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)selfk_smem);
    if (e == cudaSuccess) {
        k_fast_nbrs<<<(nb + kNbrWarps - 1) / kNbrWarps, 32 * kNbrWarps, nbrs_smem, st>>>(bs, nb, fs.kp, bs.nbr);
        k_fast_selfk<<<nb, kFB, selfk_smem, st>>>(bs, fs.kp, bs.nbr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && (prune_cop_build(bs.cen, nb, fs, bs.cop, st) || prune_cop_build(bs.sb_cen, nsb, fs, bs.scop, st)))
        e = cudaErrorUnknown;
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaFree(recs);
        gts_set_error("filter records: %s", cudaGetErrorString(e));
        return GTS_ERR_CUDA;
    }
    idx->fast_recs = recs;
    idx->fast_nb = nb;
    idx->fast_nsb = nsb;
    idx->device_bytes += bytes;
    return GTS_OK;
}

// Buffers of one filter run over qnum queries, carved from a region.
struct RunBufs {
    int *keys, *vals, *skeys, *order, *cpos, *ccnt, *r2, *ctr, *blist, *bcnt, *heavy;
    unsigned char *pbufs;   // tensor-core pruning: the block pass's items and result words
    float *clb, *cub_;
    float *qt;   // [ntiles][kp][128] FP32 query rows of each tile
    unsigned char *arec;
    uint32_t *sb_mask;
    int2 *items;
    void *cub;
    size_t cub_bytes;
    // block-stationary filter (kp <= kFResKp): per (tile, needed block) the
    // tile's lanes that need it, per block its pairs, the items and their records
    uint4 *bmask;
    int *bq_cnt, *bq_off, *bq_fill, *bq;
    int4 *bitems;
    unsigned char *irec;
    int pairs_cap;
};

// Work items of a run at most: every tile's needed blocks in items of the
// smallest size.
static size_t plan_items_cap(int ntiles, int nb)
{
    return std::max<size_t>((size_t)ntiles * ((nb + kFItemMin - 1) / kFItemMin), 1);
}

// blk: also the block-stationary filter's buffers (kp <= kFResKp only).
static size_t plan_run(const gts_index *idx, int qnum, unsigned char *base, RunBufs *b, bool blk)
{
    const FastShape fs = fast_shape(idx->dim);
    const int ntiles = (qnum + kFT - 1) / kFT;
    const int nb = idx->fast_nb, nsbw = (idx->fast_nsb + 31) / 32;
    const size_t itemcap = plan_items_cap(ntiles, nb);
    size_t cub_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (int *)nullptr, (int *)nullptr, (int *)nullptr,
                                    (int *)nullptr, qnum, 0, 32, (cudaStream_t)0);
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~(size_t)255; return base + o; };
    RunBufs r;
    r.keys = (int *)take(4 * (size_t)qnum);
    r.vals = (int *)take(4 * (size_t)qnum);
    r.skeys = (int *)take(4 * (size_t)qnum);
    r.order = (int *)take(4 * (size_t)qnum);
    r.cpos = (int *)take(4 * (size_t)qnum * kFCand);
    r.clb = (float *)take(4 * (size_t)qnum * kFCand);
    r.cub_ = (float *)take(4 * (size_t)qnum * kFCand);
    r.ccnt = (int *)take(4 * (size_t)qnum);
    r.r2 = (int *)take(4 * (size_t)qnum);
    r.ctr = (int *)take(8 * sizeof(int));   // failures, item counter, full and partial item counts, heavy rechecks
    r.heavy = (int *)take(4 * (size_t)qnum);
    r.arec = take((size_t)ntiles * fs.arec_bytes);
    r.sb_mask = (uint32_t *)take(4 * (size_t)ntiles * std::max(nsbw, 1));
    // the FP32 tile rows serve only the FP32 pruning kernels (no tensor-core pruning)
    const bool tc_prune = prune_cop_bytes(fs, nb) && prune_cop_bytes(fs, idx->fast_nsb);
    r.qt = tc_prune ? nullptr : (float *)take(4 * (size_t)ntiles * fs.kp * kFT);
    r.blist = (int *)take(4 * (size_t)ntiles * std::max(nb, 1));
    r.bcnt = (int *)take(4 * (size_t)ntiles);
    r.items = (int2 *)take(sizeof(int2) * std::max(itemcap, (size_t)1));
    const bool lanes = blk && fast_blk_stages(fs) >= 2;   // the block-stationary filter's lane masks
    r.pbufs = tc_prune ? take(prune_block_bufs(ntiles, nb, lanes)) : nullptr;
    r.cub = take(cub_bytes);
    r.cub_bytes = cub_bytes;
    r.bmask = nullptr;
    r.bq_cnt = r.bq_off = r.bq_fill = r.bq = nullptr;
    r.bitems = nullptr;
    r.irec = nullptr;
    r.pairs_cap = 0;
    if (blk && fast_blk_stages(fs) >= 2) {
        r.pairs_cap = (int)std::min<long long>((long long)qnum * kBPairs, 1ll << 30);
        r.bmask = (uint4 *)take(sizeof(uint4) * (size_t)ntiles * std::max(nb, 1));
        r.bq_cnt = (int *)take(4 * (size_t)std::max(nb, 1));
        r.bq_off = (int *)take(4 * (size_t)std::max(nb, 1));
        r.bq_fill = (int *)take(4 * (size_t)std::max(nb, 1));
        r.bq = (int *)take(4 * (size_t)r.pairs_cap);
        r.bitems = (int4 *)take(sizeof(int4) * fast_blk_items_cap(nb, r.pairs_cap));
        r.irec = take(fast_blk_irec_bytes(nb, r.pairs_cap));
    }
    if (b) *b = r;
    return off;
}

// The tiles' needed superblocks, then their needed blocks (blist, bcnt;
// bmask and bq_cnt for the block-stationary filter): on the tensor cores up
// to kFResKp (fast_prune.cu), else with the FP32 pruning kernels.  cleared:
// the superblock masks are zero already.  item > 0: the tensor-core path
// also makes the tile filter's work items of `item` blocks (*listed = true);
// otherwise the caller runs k_items.
static int prune_enqueue(gts_index *idx, const FastShape &fs, const FastSummary &bs, const RunBufs &r, int ntiles,
                         bool blk, bool cleared, int item, bool *listed, cudaStream_t st)
{
    const int nb = idx->fast_nb, nsb = idx->fast_nsb, nsbw = (nsb + 31) / 32;
    *listed = false;
    if (bs.cop && bs.scop && r.pbufs) {
        int rc = prune_superblocks(r.arec, fs, bs, nsb, ntiles, r.r2, r.sb_mask, nsbw, !cleared, idx->d_status, st);
        if (!rc)
            rc = prune_blocks(r.arec, fs, bs, nb, ntiles, r.r2, r.sb_mask, nsbw, r.pbufs, r.ctr + 5, r.blist, r.bcnt,
                              blk ? r.bmask : nullptr, blk ? r.bq_cnt : nullptr, item, item > 0 ? r.items : nullptr,
                              r.ctr + 2, (int)plan_items_cap(ntiles, nb), idx->d_stats, idx->d_status, st);
        idx->kernel_launches += 4;
        *listed = item > 0;
        return rc;
    }
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const size_t need_smem = need_smem_bytes(fs.kp);
    GTS_CUDA_TRY(cudaFuncSetAttribute(k_need_sb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need_smem));
    GTS_CUDA_TRY(cudaFuncSetAttribute(k_need_blk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need_smem));
    k_need_sb<<<dim3(ntiles, (nsb + kFChunk - 1) / kFChunk), 256, need_smem, st>>>(r.qt, r.arec, fs, bs, nsb, r.r2,
                                                                                    r.sb_mask, nsbw);
    // CTAs per tile: at least kNeedBlkY, more for small batches so that
    // about four CTAs per SM share the needed superblocks
    const int need_y = std::max(kNeedBlkY, std::min(32, (4 * nsm + ntiles - 1) / ntiles));
    k_need_blk<<<dim3(ntiles, need_y), 256, need_smem, st>>>(r.qt, r.arec, fs, bs, r.r2, r.sb_mask, nsbw, r.blist,
                                                               r.bcnt, nb, idx->d_stats, blk ? r.bmask : nullptr,
                                                               blk ? r.bq_cnt : nullptr);
    idx->kernel_launches += 2;
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

// One filter run over a query batch.  learned: also seed each query's bound
// from the learned radius model.  carry (nullable): certified starting bounds
// (float bits, one per query).  Queries the run cannot answer (a learned
// seed below the k-th distance, or a full candidate list) are written to
// d_fail and counted in *n_fail; *r2_out (nullable) receives the run's final
// bounds (valid until the region is reused).  region: scratch of at least
// plan_run(qnum) bytes.
// The kernels of one filter run over a query batch, enqueued on `st` with no
// host synchronisation (so the sequence can be captured in a CUDA graph).
// learned: also seed each query's bound from the learned radius model.
// carry (nullable): certified starting bounds (float bits, one per query).
// Queries the run cannot answer (a learned seed below the k-th distance, or
// a full candidate list) are written to d_fail, their count to r.ctr[0].
static int fast_run_enqueue(gts_index *idx, const RunBufs &r, const int *d_qids, int qnum, int k, const FastCfg &cfg,
                            bool learned, const int *carry, float *d_kth, int *d_ids, float *d_dists, int *d_fail,
                            bool timed, bool capturing, cudaStream_t st)
{
    const FastShape fs = fast_shape(idx->dim);
    const int ntiles = (qnum + kFT - 1) / kFT;
    const int nb = idx->fast_nb, nsb = idx->fast_nsb;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int rc;
    const FastSummary bs = fast_summary(idx->fast_recs, fs, nb, nsb, idx->num);

    int jk = 0;   // the table's k: the smallest power of two >= k (k <= kFMaxK = 2^(kSelfKN - 1))
    while ((1 << jk) < k) jk++;
    // per-query start, counters and masks cleared, in one launch; with a
    // learned radius its prediction replaces the start bound and the table's
    // bound is applied after it (the smaller of the two is used, and queries
    // it under-predicts are answered again)
    const int nsbw = (idx->fast_nsb + 31) / 32;
    k_fast_begin<<<(qnum + 255) / 256, 256, 0, st>>>(qnum, d_qids, bs.pos, learned ? nullptr : bs.selfk, jk, carry,
                                                     r.ccnt, r.r2, r.keys, r.vals, r.ctr, 8, r.bcnt, ntiles, r.sb_mask,
                                                     ntiles * nsbw, idx->d_stats);
    idx->kernel_launches++;
    if (learned) {
        if ((rc = mlp_seed(idx, d_qids, qnum, k, r.r2, st))) return rc;
        k_fast_seed_tab<<<(qnum + 255) / 256, 256, 0, st>>>(d_qids, qnum, bs.pos, bs.selfk, jk, r.r2);
        idx->kernel_launches++;
    }
    if (nb <= kOrderMaxNb) {
        const size_t osmem = 2 * sizeof(int) * (size_t)nb;
        GTS_CUDA_TRY(cudaFuncSetAttribute(k_fast_order, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)osmem));
        k_fast_order<<<1, kOrderThreads, osmem, st>>>(r.keys, qnum, nb, r.order);
        idx->kernel_launches++;
    } else {
        // block ids are below nb: sort only the bits they use
        int key_bits = 1;
        while (key_bits < 32 && (1ll << key_bits) < (long long)nb) key_bits++;
        size_t cb = r.cub_bytes;
        GTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(r.cub, cb, r.keys, r.skeys, r.vals, r.order, qnum, 0, key_bits,
                                                     st));
    }
    const bool blk = cfg.blk && r.bmask && fast_blk_stages(fs) >= 2;
    if (blk) {
        GTS_CUDA_TRY(cudaMemsetAsync(r.bq_cnt, 0, sizeof(int) * nb, st));
        GTS_CUDA_TRY(cudaMemsetAsync(r.bq_fill, 0, sizeof(int) * nb, st));
    }
    k_fast_arec<<<ntiles, 128, 0, st>>>(idx->rows, d_qids, r.order, qnum, idx->dim, fs, r.arec, r.qt);
    idx->kernel_launches++;
    bool listed = false;   // the filter's work items already made by the pruning
    if ((rc = prune_enqueue(idx, fs, bs, r, ntiles, blk, true, blk ? 0 : cfg.item, &listed, st))) return rc;
    if (!blk && !listed) {
        k_items<<<(ntiles + 127) / 128, 128, 0, st>>>(ntiles, r.bcnt, nb, cfg.item, r.items, r.ctr + 2,
                                                      (int)plan_items_cap(ntiles, nb));
        idx->kernel_launches++;
    }
    GTS_CUDA_TRY(cudaGetLastError());

    FastTileArgs a;
    a.recs = idx->fast_recs;
    a.arec = r.arec;
    a.blist = r.blist;
    a.bcnt = r.bcnt;
    a.items = r.items;
    a.n_items = r.ctr + 2;
    a.items_cap = (int)plan_items_cap(ntiles, nb);
    a.nbcap = nb;
    a.k = k;
    a.item = cfg.item;
    a.stream = cfg.stream ? 1 : 0;
    a.fs = fs;
    a.cand_pos = r.cpos;
    a.cand_lb = r.clb;
    a.cand_ub = r.cub_;
    a.cand_cnt = r.ccnt;
    a.r2_bits = r.r2;
    a.item_counter = r.ctr + 1;
    a.status = idx->d_status;
    a.stats = idx->d_stats;
    a.r2lo = 0.f;
    a.rcnt = nullptr;
    // events inside a captured graph must be external records to time it
    if (blk) {
        // pairs, items and item records, then the filter (the timed part)
        FastBlkRun br;
        br.args.recs = idx->fast_recs;
        br.args.fs = fs;
        br.args.k = k;
        br.args.cand_pos = r.cpos;
        br.args.cand_lb = r.clb;
        br.args.cand_ub = r.cub_;
        br.args.cand_cnt = r.ccnt;
        br.args.r2_bits = r.r2;
        br.args.status = idx->d_status;
        br.args.stats = idx->d_stats;
        br.args.r2lo = 0.f;
        br.args.rcnt = nullptr;
        br.cen = bs.cen;
        br.arec = r.arec;
        br.blist = r.blist;
        br.bmask = r.bmask;
        br.bcnt = r.bcnt;
        br.order = r.order;
        br.bq_cnt = r.bq_cnt;
        br.bq_off = r.bq_off;
        br.bq_fill = r.bq_fill;
        br.bq = r.bq;
        br.irec = r.irec;
        br.items = r.bitems;
        br.n_items = r.ctr + 2;
        br.nb = nb;
        br.nbcap = nb;
        br.ntiles = ntiles;
        br.qnum = qnum;
        br.pairs_cap = r.pairs_cap;
        br.nsm = nsm;
        br.range = false;
        br.timed_begin = timed ? idx->fev[0] : nullptr;
        br.timed_end = timed ? idx->fev[1] : nullptr;
        br.capturing = capturing;
        if ((rc = fast_blk_enqueue(br, st, &idx->kernel_launches))) return rc;
    } else {
        if (timed)
            GTS_CUDA_TRY(cudaEventRecordWithFlags(idx->fev[0], st, capturing ? cudaEventRecordExternal : 0));
        if ((rc = launch_fast_tile(a, cfg.cg, nsm, st))) return rc;
        idx->kernel_launches++;
        if (timed)
            GTS_CUDA_TRY(cudaEventRecordWithFlags(idx->fev[1], st, capturing ? cudaEventRecordExternal : 0));
    }
    // light recheck over every query, then the full one over those with more
    // than 128 candidates: a persistent grid, as many CTAs as fit on the SMs,
    // walking their list
    auto full_grid = [&](const void *fn) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 128, 0) != cudaSuccess || per_sm < 1)
            per_sm = 4;
        return std::min(qnum, per_sm * nsm);
    };
    if (cfg.wfin && k <= kFinWarpK) {
        // one warp per query; lists over 32 candidates to the full variant
        if (fs.kp <= kFResKp)
            k_fast_final_warp<kFResKp, 8><<<(qnum + kFinWarps - 1) / kFinWarps, 32 * kFinWarps, 0, st>>>(
                idx->rows, idx->dim, idx->num, bs.prow, fs.kp, bs.ids, nb * kFB, d_qids, qnum, k,
                idx->params.infi_dis, r.cpos, r.clb, r.cub_, r.ccnt, r.r2, d_kth, d_ids, d_dists, d_fail, r.ctr,
                r.heavy, r.ctr + 4, idx->d_stats);
        else
            k_fast_final_warp<kFMaxKp, 2><<<(qnum + kFinWarps - 1) / kFinWarps, 32 * kFinWarps, 0, st>>>(
                idx->rows, idx->dim, idx->num, bs.prow, fs.kp, bs.ids, nb * kFB, d_qids, qnum, k,
                idx->params.infi_dis, r.cpos, r.clb, r.cub_, r.ccnt, r.r2, d_kth, d_ids, d_dists, d_fail, r.ctr,
                r.heavy, r.ctr + 4, idx->d_stats);
        if (fs.kp <= kFResKp)
            k_fast_final<kFResKp, kFinB, kFCand><<<full_grid((const void *)k_fast_final<kFResKp, kFinB, kFCand>), 128,
                                                    0, st>>>(
                idx->rows, idx->dim, idx->num, bs.prow, fs.kp, bs.ids, nb * kFB, d_qids, k, idx->params.infi_dis,
                r.cpos, r.clb, r.cub_, r.ccnt, r.r2, d_kth, d_ids, d_dists, d_fail, r.ctr, nullptr, nullptr, r.heavy,
                r.ctr + 4, idx->d_stats);
        else
            k_fast_final<kFMaxKp, kFinB / 2, kFCand><<<
                full_grid((const void *)k_fast_final<kFMaxKp, kFinB / 2, kFCand>), 128, 0, st>>>(
                idx->rows, idx->dim, idx->num, bs.prow, fs.kp, bs.ids, nb * kFB, d_qids, k, idx->params.infi_dis,
                r.cpos, r.clb, r.cub_, r.ccnt, r.r2, d_kth, d_ids, d_dists, d_fail, r.ctr, nullptr, nullptr, r.heavy,
                r.ctr + 4, idx->d_stats);
    } else if (fs.kp <= kFResKp) {
        k_fast_final<kFResKp, kFinB, 128><<<qnum, 128, 0, st>>>(
            idx->rows, idx->dim, idx->num, bs.prow, fs.kp, bs.ids, nb * kFB, d_qids, k, idx->params.infi_dis, r.cpos,
            r.clb, r.cub_, r.ccnt, r.r2, d_kth, d_ids, d_dists, d_fail, r.ctr, r.heavy, r.ctr + 4, nullptr, nullptr,
            idx->d_stats);
        k_fast_final<kFResKp, kFinB, kFCand><<<full_grid((const void *)k_fast_final<kFResKp, kFinB, kFCand>), 128, 0,
                                                st>>>(
            idx->rows, idx->dim, idx->num, bs.prow, fs.kp, bs.ids, nb * kFB, d_qids, k, idx->params.infi_dis, r.cpos,
            r.clb, r.cub_, r.ccnt, r.r2, d_kth, d_ids, d_dists, d_fail, r.ctr, nullptr, nullptr, r.heavy, r.ctr + 4,
            idx->d_stats);
    } else {
        k_fast_final<kFMaxKp, kFinB / 2, 128><<<qnum, 128, 0, st>>>(
            idx->rows, idx->dim, idx->num, bs.prow, fs.kp, bs.ids, nb * kFB, d_qids, k, idx->params.infi_dis, r.cpos,
            r.clb, r.cub_, r.ccnt, r.r2, d_kth, d_ids, d_dists, d_fail, r.ctr, r.heavy, r.ctr + 4, nullptr, nullptr,
            idx->d_stats);
        k_fast_final<kFMaxKp, kFinB / 2, kFCand><<<full_grid((const void *)k_fast_final<kFMaxKp, kFinB / 2, kFCand>),
                                                    128, 0, st>>>(
            idx->rows, idx->dim, idx->num, bs.prow, fs.kp, bs.ids, nb * kFB, d_qids, k, idx->params.infi_dis, r.cpos,
            r.clb, r.cub_, r.ccnt, r.r2, d_kth, d_ids, d_dists, d_fail, r.ctr, nullptr, nullptr, r.heavy, r.ctr + 4,
            idx->d_stats);
    }
    idx->kernel_launches += 2;
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

// After a run: kernel status and failure count back on the host.
static int fast_run_finish(gts_index *idx, const RunBufs &r, int *n_fail, int **r2_out, bool timed, cudaStream_t st)
{
    int status = 0;
    GTS_CUDA_TRY(cudaMemcpyAsync(&status, idx->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    GTS_CUDA_TRY(cudaMemcpyAsync(n_fail, r.ctr, sizeof(int), cudaMemcpyDeviceToHost, st));
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
    if (r2_out) *r2_out = r.r2;
    return GTS_OK;
}

// One filter run, launched directly.  region: scratch of at least
// plan_run(qnum) bytes.
static int fast_run(gts_index *idx, unsigned char *region, size_t region_bytes, const int *d_qids, int qnum, int k,
                    const FastCfg &cfg, bool learned, const int *carry, float *d_kth, int *d_ids, float *d_dists,
                    int *d_fail, int *n_fail, int **r2_out, cudaStream_t st)
{
    RunBufs r;
    const size_t need = plan_run(idx, qnum, region, &r, cfg.blk);
    if (need > region_bytes) {
        gts_set_error("filter run needs %zu bytes of scratch, the region holds %zu", need, region_bytes);
        return GTS_ERR_INVALID;
    }
    const bool timed = idx->time_filter && idx->fev[0];
    int rc = fast_run_enqueue(idx, r, d_qids, qnum, k, cfg, learned, carry, d_kth, d_ids, d_dists, d_fail, timed,
                              false, st);
    if (rc) return rc;
    return fast_run_finish(idx, r, n_fail, r2_out, timed, st);
}

// Bookkeeping of one re-answer stage: the failed queries' positions in the
// parent batch (fail), their ids, carried bounds and results.
struct Book {
    int *fail, *sub_q, *sub_r2, *sub_ids;
    float *sub_kth, *sub_dis;
};

static size_t plan_book(int qnum, int k, unsigned char *base, Book *b)
{
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~(size_t)255; return base + o; };
    Book r;
    r.fail = (int *)take(4 * (size_t)qnum);
    r.sub_q = (int *)take(4 * (size_t)qnum);
    r.sub_r2 = (int *)take(4 * (size_t)qnum);
    r.sub_kth = (float *)take(4 * (size_t)qnum);
    r.sub_ids = (int *)take(4 * (size_t)qnum * k);
    r.sub_dis = (float *)take(4 * (size_t)qnum * k);
    if (b) *b = r;
    return off;
}

struct FastCall {
    unsigned char *region;
    size_t region_bytes;
    Book book[3];   // stage 0: filter on table seeds (no learned radius), 1: filter from the bound reached,
                    // 2: plain traversal
};

void graph_invalidate(gts_index *idx)
{
    for (int i = 0; i < gts_index::kGraphSlots; i++) {
        if (idx->graph_exec[i]) cudaGraphExecDestroy(idx->graph_exec[i]);
        idx->graph_exec[i] = nullptr;
        for (long long &v : idx->graph_key[i]) v = 0;
        idx->graph_used[i] = 0;
    }
}

// Queries listed in book[stage].fail (indices into parent_q) answered again:
// 0 -> after a learned run: the filter without the learned seed;
// 1 -> after a run from certified seeds (its list overflowed): the filter
//      again, starting from the bound that run reached (r2_prev);
// 2 -> the plain traversal.
static int rerun_failed(gts_index *idx, FastCall &fc, const FastCfg &cfg, int stage, const int *parent_q, int n,
                        const int *r2_prev, int k, float *d_kth, int *d_ids, float *d_dists, cudaStream_t st)
{
    Book &b = fc.book[stage];
    int *sub_ids = d_ids ? b.sub_ids : nullptr;
    float *sub_dis = d_dists ? b.sub_dis : nullptr;
    k_gather_i<<<(n + 255) / 256, 256, 0, st>>>(parent_q, b.fail, n, b.sub_q);
    idx->kernel_launches++;
    if (stage == 1 && r2_prev) {
        k_gather_i<<<(n + 255) / 256, 256, 0, st>>>(r2_prev, b.fail, n, b.sub_r2);
        idx->kernel_launches++;
    }
    int rc;
    if (stage < 2) {
        int n2 = 0, *r2 = nullptr;
        // lists that overflowed (or pairs a block-stationary run could not
        // store) go through the tile filter, whose running bound tightens
        FastCfg c = cfg;
        if (stage == 1) c.blk = false;
        if ((rc = fast_run(idx, fc.region, fc.region_bytes, b.sub_q, n, k, c, false,
                           stage == 1 && r2_prev ? b.sub_r2 : nullptr, b.sub_kth, sub_ids, sub_dis,
                           fc.book[stage + 1].fail, &n2, &r2, st)))
            return rc;
        if (n2 > 0 &&
            (rc = rerun_failed(idx, fc, c, stage + 1, b.sub_q, n2, r2, k, b.sub_kth, sub_ids, sub_dis, st)))
            return rc;
    } else {
        k_add_stat<<<1, 1, 0, st>>>(idx->d_stats + 4, (unsigned long long)n);
        idx->kernel_launches++;
        idx->keep_stats = true;
        rc = search_knn(idx, b.sub_q, n, k, 0, b.sub_kth, sub_ids, sub_dis, st);
        idx->keep_stats = false;
        if (rc) return rc;
    }
    k_scatter_results<<<(n + 255) / 256, 256, 0, st>>>(b.fail, n, k, b.sub_kth, sub_ids, sub_dis, d_kth, d_ids,
                                                       d_dists);
    idx->kernel_launches++;
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

// Captures of one batch shape (with different argument buffers) kept at most.
constexpr int kGraphShapeMax = 4;

// One batch (at most one filter run) through the CUDA graph of the filter
// pass: the pass (sort, seeds, pruning, filter, recheck: 11-12 kernels and
// the CUB sort) is captured once per batch shape and argument buffers and
// replayed on the handle's own stream.  The host then reads the failure
// count and runs any re-answer stage directly.  Returns 1 (nothing done)
// when this shape was captured kGraphShapeMax times with other buffers
// already: such callers are better served by direct launches.  The caller has reset
// status and counters on st.
static int fast_search_graph(gts_index *idx, FastCall &fc, const FastCfg &cfg, const int *d_qids, int qnum, int k,
                             float *d_kth, int *d_ids, float *d_dists, cudaStream_t st)
{
    if (!idx->graph_stream) {
        GTS_CUDA_TRY(cudaStreamCreateWithFlags(&idx->graph_stream, cudaStreamNonBlocking));
        for (int i = 0; i < 2; i++) GTS_CUDA_TRY(cudaEventCreateWithFlags(&idx->graph_ev[i], cudaEventDisableTiming));
    }
    cudaStream_t gs = idx->graph_stream;
    const bool learned = cfg.learned && idx->mlp_ready;
    const bool timed = idx->time_filter && idx->fev[0];
    const int first = learned ? 0 : 1;
    RunBufs r;
    plan_run(idx, qnum, fc.region, &r, cfg.blk);
    const long long key[8] = {qnum, k,
                              cfg_pack(cfg) | (learned ? 1 << 16 : 0) | (timed ? 1 << 19 : 0),
                              (long long)(uintptr_t)fc.region, (long long)(uintptr_t)idx->fast_recs,
                              (long long)(uintptr_t)d_qids, (long long)(uintptr_t)d_kth,
                              (long long)(uintptr_t)d_ids ^ ((long long)(uintptr_t)d_dists << 1)};
    constexpr int NS = gts_index::kGraphSlots;
    int slot = -1, same_shape = 0;
    for (int s = 0; s < NS; s++) {
        if (!idx->graph_exec[s]) continue;
        bool same = true, shape = true;
        for (int i = 0; i < 8; i++) same = same && idx->graph_key[s][i] == key[i];
        for (int i = 0; i < 5; i++) shape = shape && idx->graph_key[s][i] == key[i];
        if (same) slot = s;
        else if (shape) same_shape++;
    }
    if (slot < 0) {
        // a caller whose buffers keep moving (four captures of this shape
        // with other buffers already) is better served by direct launches
        if (same_shape >= kGraphShapeMax) return 1;
        // capture into a free slot, else the least recently used one
        for (int s = 0; s < NS && slot < 0; s++)
            if (!idx->graph_exec[s]) slot = s;
        if (slot < 0) {
            slot = 0;
            for (int s = 1; s < NS; s++)
                if (idx->graph_used[s] < idx->graph_used[slot]) slot = s;
        }
        if (idx->graph_exec[slot]) cudaGraphExecDestroy(idx->graph_exec[slot]);
        idx->graph_exec[slot] = nullptr;
        const long long l0 = idx->kernel_launches;
        GTS_CUDA_TRY(cudaStreamBeginCapture(gs, cudaStreamCaptureModeRelaxed));
        int rc = fast_run_enqueue(idx, r, d_qids, qnum, k, cfg, learned, nullptr, d_kth, d_ids, d_dists,
                                  fc.book[first].fail, timed, true, gs);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(gs, &g);
        // this library's kernels in the graph (CUB's and memsets not
        // counted), counted at every replay instead
        const long long in_graph = idx->kernel_launches - l0;
        idx->kernel_launches = l0;
        if (rc || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            if (!rc) gts_set_error("filter graph capture failed: %s", cudaGetErrorString(e));
            cudaGetLastError();
            return rc ? rc : GTS_ERR_CUDA;
        }
        e = cudaGraphInstantiate(&idx->graph_exec[slot], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            idx->graph_exec[slot] = nullptr;
            gts_set_error("filter graph instantiation failed: %s", cudaGetErrorString(e));
            return GTS_ERR_CUDA;
        }
        for (int i = 0; i < 8; i++) idx->graph_key[slot][i] = key[i];
        idx->graph_kernels[slot] = in_graph;
    }
    idx->graph_used[slot] = ++idx->graph_clock;
    GTS_CUDA_TRY(cudaEventRecord(idx->graph_ev[0], st));
    GTS_CUDA_TRY(cudaStreamWaitEvent(gs, idx->graph_ev[0], 0));
    GTS_CUDA_TRY(cudaGraphLaunch(idx->graph_exec[slot], gs));
    idx->kernel_launches += idx->graph_kernels[slot];
    idx->graph_launches++;
    int n_fail = 0, *r2 = nullptr, rc;
    if ((rc = fast_run_finish(idx, r, &n_fail, &r2, timed, gs))) return rc;
    if (n_fail > 0 && (rc = rerun_failed(idx, fc, cfg, first, d_qids, n_fail, r2, k, d_kth, d_ids, d_dists, gs)))
        return rc;
    idx->last_fast_overflow = n_fail;
    GTS_CUDA_TRY(cudaEventRecord(idx->graph_ev[1], gs));
    GTS_CUDA_TRY(cudaStreamWaitEvent(st, idx->graph_ev[1], 0));
    return GTS_OK;
}

// The whole batch with one configuration: filter runs of at most qc
// queries, each followed by the re-answer stages its failures need.
static int fast_search_cfg(gts_index *idx, FastCall &fc, int qc, const FastCfg &cfg, const int *d_qids, int qnum,
                           int k, float *d_kth, int *d_ids, float *d_dists, cudaStream_t st)
{
    GTS_CUDA_TRY(cudaMemsetAsync(idx->d_status, 0, sizeof(int), st));
    GTS_CUDA_TRY(cudaMemsetAsync(idx->d_stats, 0, kStatsN * sizeof(unsigned long long), st));
    const bool learned = cfg.learned && idx->mlp_ready;
    const int first = learned ? 0 : 1;
    int total_fail = 0, rc;
    if (idx->use_graphs && qnum <= qc) {
        rc = fast_search_graph(idx, fc, cfg, d_qids, qnum, k, d_kth, d_ids, d_dists, st);
        if (rc < 0) return rc;
        if (rc == 0) {
            GTS_CUDA_TRY(cudaStreamSynchronize(st));
            return GTS_OK;
        }
    }
    for (int q0 = 0; q0 < qnum; q0 += qc) {
        const int qn = std::min(qc, qnum - q0);
        int n_fail = 0, *r2 = nullptr;
        float *kth = d_kth + q0;
        int *ids = d_ids ? d_ids + (size_t)q0 * k : nullptr;
        float *dis = d_dists ? d_dists + (size_t)q0 * k : nullptr;
        if ((rc = fast_run(idx, fc.region, fc.region_bytes, d_qids + q0, qn, k, cfg, learned, nullptr, kth, ids,
                           dis, fc.book[first].fail, &n_fail, &r2, st)))
            return rc;
        total_fail += n_fail;
        if (n_fail > 0 && (rc = rerun_failed(idx, fc, cfg, first, d_qids + q0, n_fail, r2, k, kth, ids, dis, st)))
            return rc;
    }
    idx->last_fast_overflow = total_fail;
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    return GTS_OK;
}

// Autotuner.  The first batch of at least kTuneMinQueries queries with a
// given k runs once per candidate configuration (learned seed on / off when
// a model is trained, 4 / 2 / 1 epilogue column groups as the heap fits, 8 /
// 16 / 32 blocks per work item), timed with CUDA events; every candidate
// returns the same exact answers, so the fastest is kept for this k and
// index (until the index is rebuilt or the model retrained).  Smaller batches
// use the default configuration without tuning.
constexpr int kTuneMinQueries = 2048;

static int fast_autotune(gts_index *idx, FastCall &fc, int qc, const int *d_qids, int qnum, int k, float *d_kth,
                         int *d_ids, float *d_dists, cudaStream_t st, FastCfg *best_out)
{
    cudaEvent_t e0, e1;
    GTS_CUDA_TRY(cudaEventCreate(&e0));
    GTS_CUDA_TRY(cudaEventCreate(&e1));
    FastCfg best = fast_default_cfg(idx, k);
    float best_ms = 3.0e38f;
    int rc = GTS_OK;
    // candidates: per seed choice, the block-stationary filter, then the tile
    // filter's column groups, item sizes and record forms
    const FastShape fs = fast_shape(idx->dim);
    std::vector<FastCfg> cands;
    for (int learned = 0; learned <= (idx->mlp_ready ? 1 : 0); learned++) {
        if (fast_blk_stages(fs) >= 2) cands.push_back(FastCfg{learned != 0, fast_cg(k), 16, false, true});
        for (int cg = 4; cg >= 1; cg >>= 1) {
            if (k > 16 && cg * k > 128) continue;   // heaps: 128 cg threads x k x 2 bytes <= 32 KB
            for (int item = 8; item <= kFItemMax; item *= 2)
                for (int stream = fs.kp > kFResKp ? 1 : 0; stream <= 1; stream++)
                    if (fast_tile_fits(fs, cg, k, stream != 0))
                        cands.push_back(FastCfg{learned != 0, cg, item, stream != 0, false});
        }
    }
    for (size_t ci = 0; ci < cands.size(); ci++) {
        const FastCfg c = cands[ci];
        if (cudaEventRecord(e0, st) != cudaSuccess) {
            rc = GTS_ERR_CUDA;
            break;
        }
        if ((rc = fast_search_cfg(idx, fc, qc, c, d_qids, qnum, k, d_kth, d_ids, d_dists, st))) break;
        float ms = 0.f;
        if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            rc = GTS_ERR_CUDA;
            break;
        }
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
        // after the filter configurations, the best one with the other light recheck
        if (ci + 1 == cands.size() && k <= kFinWarpK && !best.wfin) {
            FastCfg w = best;
            w.wfin = true;
            cands.push_back(w);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc == GTS_ERR_CUDA) gts_set_error("autotune: CUDA event failed");
    *best_out = best;
    return rc;
}

// Build the tensor-core form's block order and filter records now instead of
// on the first fast search.  *done = 1 when the index holds them afterwards,
// 0 when the form does not apply to this index (nothing to build).
int fast_prepare_now(gts_index *idx, cudaStream_t st, int *done)
{
    *done = 0;
    if (!fast_supported(idx, 1)) return GTS_OK;
    int rc = fast_prepare(idx, st);
    if (rc == GTS_OK) *done = 1;
    return rc;
}

// Queries per filter run: at most kFMaxBatch, halved (in whole tiles) until
// the scratch of one run, per_run(q) bytes, fits the call's budget; a run of
// one tile that does not fit is an error.
template <typename F>
static int run_queries_for_budget(const gts_index *idx, int qnum, F per_run, int *qc)
{
    const size_t budget = search_budget(idx);
    int q = std::min(qnum, kFMaxBatch);
    while (q > kFT && per_run(q) > budget) q = std::max(kFT, (q / 2 + kFT - 1) / kFT * kFT);
    if (per_run(q) > budget) {
        gts_set_error("scratch budget of %zu bytes is below the %zu bytes of one %d-query filter run", budget,
                      per_run(q), q);
        return GTS_ERR_NOMEM;
    }
    *qc = q;
    return GTS_OK;
}

int search_knn_fast(gts_index *idx, const int *d_qids, int qnum, int k, float *d_kth, int *d_ids,
                    float *d_dists, cudaStream_t st)
{
    int rc = fast_prepare(idx, st);
    if (rc) return rc;
    // one scratch region for a run of at most kFMaxBatch queries (fewer when
    // the call's budget is smaller), reused by the re-answer stages, plus
    // their bookkeeping
    auto rbytes_of = [&](int q) { return (plan_run(idx, q, nullptr, nullptr, true) + 255) & ~(size_t)255; };
    auto bbytes_of = [&](int q) { return (plan_book(q, k, nullptr, nullptr) + 255) & ~(size_t)255; };
    int qc = 0;
    if ((rc = run_queries_for_budget(idx, qnum, [&](int q) { return rbytes_of(q) + 3 * bbytes_of(q); }, &qc)))
        return rc;
    const size_t rbytes = rbytes_of(qc);
    const size_t bbytes = bbytes_of(qc);
    if ((rc = ensure_scratch(idx, rbytes + 3 * bbytes))) return rc;
    FastCall fc;
    fc.region = (unsigned char *)idx->scratch;
    fc.region_bytes = rbytes;
    for (int s = 0; s < 3; s++) plan_book(qc, k, fc.region + rbytes + s * bbytes, &fc.book[s]);
    FastCfg cfg;
    if (idx->fast_cfg[k]) {
        cfg = cfg_unpack(idx->fast_cfg[k]);
    } else if (qnum >= kTuneMinQueries) {
        if ((rc = fast_autotune(idx, fc, qc, d_qids, qnum, k, d_kth, d_ids, d_dists, st, &cfg))) return rc;
        idx->fast_cfg[k] = cfg_pack(cfg);
    } else {
        cfg = fast_default_cfg(idx, k);
    }
    return fast_search_cfg(idx, fc, qc, cfg, d_qids, qnum, k, d_kth, d_ids, d_dists, st);
}

// The filter without the learned seed, with every buffer carved out of
// `scratch` (bytes long, 256-byte aligned): no device allocation on any
// path.  The filter records must already exist.  Queries the run could not
// answer (a full candidate list) go to the plain traversal, which uses only
// the index's own counters.
int search_knn_fast_fixed(gts_index *idx, const int *d_qids, int qnum, int k, float *d_kth, int *d_ids,
                          float *d_dists, unsigned char *scratch, size_t bytes, cudaStream_t st)
{
    if (!fast_supported(idx, k) || idx->dim > kFResKp) {
        gts_set_error("fixed-scratch kNN supports the L2 metric with dim <= %d and 1 <= k <= %d", kFResKp, kFMaxK);
        return GTS_ERR_INVALID;
    }
    if (!idx->fast_recs) {
        gts_set_error("the index has no filter records (none built yet, or a rebuild or update dropped them): one "
                      "GTS_FORM_FAST kNN call or gts_index_prepare on it must come first");
        return GTS_ERR_INVALID;
    }
    if (qnum <= 0) return GTS_OK;
    Book b;
    const size_t bbytes = (plan_book(qnum, k, scratch, &b) + 255) & ~(size_t)255;
    if (bbytes > bytes) {
        gts_set_error("fixed scratch of %zu bytes is too small for %d queries", bytes, qnum);
        return GTS_ERR_INVALID;
    }
    GTS_CUDA_TRY(cudaMemsetAsync(idx->d_status, 0, sizeof(int), st));
    GTS_CUDA_TRY(cudaMemsetAsync(idx->d_stats, 0, kStatsN * sizeof(unsigned long long), st));
    int n_fail = 0, rc;
    const FastCfg cfg{false, fast_cg(k), 16};
    if ((rc = fast_run(idx, scratch + bbytes, bytes - bbytes, d_qids, qnum, k, cfg, false, nullptr, d_kth, d_ids, d_dists,
                       b.fail, &n_fail, nullptr, st)))
        return rc;
    idx->last_fast_overflow = n_fail;
    if (n_fail == 0) return GTS_OK;
    int *sub_ids = d_ids ? b.sub_ids : nullptr;
    float *sub_dis = d_dists ? b.sub_dis : nullptr;
    k_gather_i<<<(n_fail + 255) / 256, 256, 0, st>>>(d_qids, b.fail, n_fail, b.sub_q);
    idx->kernel_launches++;
    k_add_stat<<<1, 1, 0, st>>>(idx->d_stats + 4, (unsigned long long)n_fail);
    idx->kernel_launches++;
    idx->keep_stats = true;
    rc = search_knn(idx, b.sub_q, n_fail, k, 0, b.sub_kth, sub_ids, sub_dis, st);
    idx->keep_stats = false;
    if (rc) return rc;
    k_scatter_results<<<(n_fail + 255) / 256, 256, 0, st>>>(b.fail, n_fail, k, b.sub_kth, sub_ids, sub_dis, d_kth,
                                                           d_ids, d_dists);
    idx->kernel_launches++;
    GTS_CUDA_TRY(cudaGetLastError());
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    return GTS_OK;
}

// ---------------------------------------------------------------- range counts

__global__ void k_fast_range_init(int qnum, int *cand_cnt, int *r2_bits, int *rcnt, int r2hi_bits)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < qnum) {
        cand_cnt[i] = 0;
        r2_bits[i] = r2hi_bits;
        rcnt[i] = 0;
    }
}

// One CTA per query: the listed (uncertain) objects get the reference's
// range value (searchIndexRnnV2's leaf: FP32 accumulation of pow terms, then
// pow(., 0.5); the query itself at 0) and count when it is within r; the
// count adds to the objects the filter found certainly inside.  A query
// whose list overflowed goes to the overflow list.
//
// One thread per listed object.  The accumulation uses exact squares (a
// float difference squared is exact in FP64) in place of pow(e, 2), which
// is within 2 ulp of it: each step's double sum then differs from the
// reference's by at most 4.4e-16 (term + sum), so both round to the same
// float unless the sum lies within that of a float rounding midpoint.  A
// step that comes that close sends the object through the pow terms.
__global__ void __launch_bounds__(128) k_fast_range_final(const float *__restrict__ rows, int dim, int num,
                                                          const float *__restrict__ prow, int kp,
                                                          const int *__restrict__ ids_of_slot, int nslots,
                                                          const int *__restrict__ qids, float r,
                                                          const int *__restrict__ cand_pos,
                                                          const int *__restrict__ cand_cnt,
                                                          const int *__restrict__ rcnt, int *counts, int *overflow,
                                                          int *n_overflow, unsigned long long *stats)
{
    __shared__ int c;
    __shared__ float qs[kFMaxKp];
    const int q = blockIdx.x, t = threadIdx.x;
    const int cnt = cand_cnt[q];
    if (cnt > kFCand) {
        if (t == 0) overflow[atomicAdd(n_overflow, 1)] = q;
        return;
    }
    const int qid = qids[q];
    if (t == 0) c = 0;
    for (int j = t; j < dim; j += 128) qs[j] = rows[(size_t)qid * dim + j];
    __syncthreads();
    for (int i = t; i < cnt; i += 128) {
        const int slot = cand_pos[(size_t)q * kFCand + i];
        if (slot < 0 || slot >= nslots) continue;
        const int id = ids_of_slot[slot];
        if (id < 0 || id >= num) continue;
        float d = 0.f;
        if (id != qid) {
            const float *orow = prow + (size_t)slot * kp;
            float res = 0.f;
            bool risky = false;
#pragma unroll 8
            for (int j = 0; j < dim; j++) {
                const double e = (double)(orow[j] - qs[j]);
                const double tt = e * e;
                const double s2 = (double)res + tt;
                const float f = __double2float_rn(s2);
                const double fd = f;
                const double nb = (double)__int_as_float(__float_as_int(f) + (s2 > fd ? 1 : -1));
                const double mid = 0.5 * (fd + nb);
                if (s2 != fd && fabs(s2 - mid) <= tt * 8.9e-16 + s2 * 4.5e-16) risky = true;
                res = f;
            }
            if (risky) {
                res = 0.f;
                for (int j = 0; j < dim; j++) res += pow(orow[j] - qs[j], 2);
            }
            d = pow(res, 0.5);
        }
        if (d <= r) atomicAdd(&c, 1);
    }
    __syncthreads();
    if (t == 0) {
        counts[q] = rcnt[q] + c;
        if (stats) atomicAdd(&stats[2], (unsigned long long)cnt);
    }
}

// Range counts on the tensor cores (L2, dim <= 128): the fast form's block
// order, pruning and filter with the bound fixed at r^2.  The reference's
// value is an FP32 accumulation (relative error below (dim + 2) 2^-24 on the
// square, under 8e-6 at dim 128), so an object whose certified upper bound
// on d^2 is below r^2 (1 - 3e-5) is within r in the reference's arithmetic
// too and is counted directly; one whose lower bound is above r^2 (1 + 3e-5)
// is not; the rest get the reference's value.  Queries whose list of
// uncertain objects overflowed are counted by the plain traversal.
int search_range_fast(gts_index *idx, const int *d_qids, int qnum, float r, int *d_counts, cudaStream_t st)
{
    if (!fast_supported(idx, 1) || !(r >= 0.f)) return search_range(idx, d_qids, qnum, r, d_counts, nullptr, st);
    if (qnum <= 0) return GTS_OK;
    int rc = fast_prepare(idx, st);
    if (rc) return rc;
    const FastShape fs = fast_shape(idx->dim);
    const int nb = idx->fast_nb, nsb = idx->fast_nsb;
    const bool blk = idx->range_variant == 0 && fast_blk_stages(fs) >= 2;
    auto rbytes_of = [&](int q) { return (plan_run(idx, q, nullptr, nullptr, blk) + 255) & ~(size_t)255; };
    auto ib_of = [&](int q) { return ((size_t)q * sizeof(int) + 255) & ~(size_t)255; };
    int qc = 0;
    if ((rc = run_queries_for_budget(idx, qnum, [&](int q) { return rbytes_of(q) + 4 * ib_of(q); }, &qc)))
        return rc;
    const size_t rbytes = rbytes_of(qc);
    const size_t ib = ib_of(qc);
    if ((rc = ensure_scratch(idx, rbytes + 4 * ib))) return rc;
    unsigned char *region = (unsigned char *)idx->scratch;
    int *rcnt = (int *)(region + rbytes), *fail = (int *)(region + rbytes + ib);
    int *sub_q = (int *)(region + rbytes + 2 * ib), *sub_c = (int *)(region + rbytes + 3 * ib);
    const double rr = (double)r * (double)r;
    // r^2 (1 + 3e-5) rounded up and r^2 (1 - 3e-5) rounded down to float
    float r2hi = (float)(rr * (1.0 + 3e-5)), r2lo = (float)(rr * (1.0 - 3e-5));
    if ((double)r2hi < rr * (1.0 + 3e-5)) r2hi = std::nextafter(r2hi, INFINITY);
    if ((double)r2lo > rr * (1.0 - 3e-5)) r2lo = std::nextafter(r2lo, 0.f);
    int r2hi_bits;
    std::memcpy(&r2hi_bits, &r2hi, sizeof(int));
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const FastSummary bs = fast_summary(idx->fast_recs, fs, nb, nsb, idx->num);
    GTS_CUDA_TRY(cudaMemsetAsync(idx->d_status, 0, sizeof(int), st));
    if (!idx->keep_stats) GTS_CUDA_TRY(cudaMemsetAsync(idx->d_stats, 0, kStatsN * sizeof(unsigned long long), st));
    int key_bits = 1;
    while (key_bits < 32 && (1ll << key_bits) < (long long)nb) key_bits++;
    for (int q0 = 0; q0 < qnum; q0 += qc) {
        const int n = std::min(qc, qnum - q0);
        const int *dq = d_qids + q0;
        const int ntiles = (n + kFT - 1) / kFT;
        RunBufs rb;
        plan_run(idx, n, region, &rb, blk);
        k_fast_keys<<<(n + 255) / 256, 256, 0, st>>>(dq, n, bs.pos, rb.keys, rb.vals);
        size_t cb = rb.cub_bytes;
        GTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(rb.cub, cb, rb.keys, rb.skeys, rb.vals, rb.order, n, 0,
                                                     key_bits, st));
        k_fast_range_init<<<(n + 255) / 256, 256, 0, st>>>(n, rb.ccnt, rb.r2, rcnt, r2hi_bits);
        GTS_CUDA_TRY(cudaMemsetAsync(rb.ctr, 0, 8 * sizeof(int), st));
        GTS_CUDA_TRY(cudaMemsetAsync(rb.bcnt, 0, sizeof(int) * ntiles, st));
        if (blk) {
            GTS_CUDA_TRY(cudaMemsetAsync(rb.bq_cnt, 0, sizeof(int) * nb, st));
            GTS_CUDA_TRY(cudaMemsetAsync(rb.bq_fill, 0, sizeof(int) * nb, st));
        }
        k_fast_arec<<<ntiles, 128, 0, st>>>(idx->rows, dq, rb.order, n, idx->dim, fs, rb.arec, rb.qt);
        bool listed = false;
        if ((rc = prune_enqueue(idx, fs, bs, rb, ntiles, blk, false, blk ? 0 : 16, &listed, st))) return rc;
        if (!blk && !listed)
            k_items<<<(ntiles + 127) / 128, 128, 0, st>>>(ntiles, rb.bcnt, nb, 16, rb.items, rb.ctr + 2,
                                                          (int)plan_items_cap(ntiles, nb));
        GTS_CUDA_TRY(cudaGetLastError());
        FastTileArgs a;
        a.recs = idx->fast_recs;
        a.arec = rb.arec;
        a.blist = rb.blist;
        a.bcnt = rb.bcnt;
        a.items = rb.items;
        a.n_items = rb.ctr + 2;
        a.items_cap = (int)plan_items_cap(ntiles, nb);
        a.nbcap = nb;
        a.k = 1;
        a.item = 16;
        a.stream = 0;
        a.fs = fs;
        a.cand_pos = rb.cpos;
        a.cand_lb = rb.clb;
        a.cand_ub = rb.cub_;
        a.cand_cnt = rb.ccnt;
        a.r2_bits = rb.r2;
        a.item_counter = rb.ctr + 1;
        a.status = idx->d_status;
        a.stats = idx->d_stats;
        a.r2lo = r2lo;
        a.rcnt = rcnt;
        const bool timed = idx->time_filter && idx->fev[0];
        if (blk) {
            FastBlkRun br;
            br.args.recs = idx->fast_recs;
            br.args.fs = fs;
            br.args.k = 1;
            br.args.cand_pos = rb.cpos;
            br.args.cand_lb = rb.clb;
            br.args.cand_ub = rb.cub_;
            br.args.cand_cnt = rb.ccnt;
            br.args.r2_bits = rb.r2;
            br.args.status = idx->d_status;
            br.args.stats = idx->d_stats;
            br.args.r2lo = r2lo;
            br.args.rcnt = rcnt;
            br.cen = bs.cen;
            br.arec = rb.arec;
            br.blist = rb.blist;
            br.bmask = rb.bmask;
            br.bcnt = rb.bcnt;
            br.order = rb.order;
            br.bq_cnt = rb.bq_cnt;
            br.bq_off = rb.bq_off;
            br.bq_fill = rb.bq_fill;
            br.bq = rb.bq;
            br.irec = rb.irec;
            br.items = rb.bitems;
            br.n_items = rb.ctr + 2;
            br.nb = nb;
            br.nbcap = nb;
            br.ntiles = ntiles;
            br.qnum = n;
            br.pairs_cap = rb.pairs_cap;
            br.nsm = nsm;
            br.range = true;
            br.timed_begin = timed ? idx->fev[0] : nullptr;
            br.timed_end = timed ? idx->fev[1] : nullptr;
            br.capturing = false;
            if ((rc = fast_blk_enqueue(br, st, &idx->kernel_launches))) return rc;
            idx->kernel_launches += 7;   // keys, init, arec, need_sb, need_blk, stat, final
        } else {
            if (timed) GTS_CUDA_TRY(cudaEventRecord(idx->fev[0], st));
            if ((rc = launch_fast_tile_ks<4, 8, true>(a, nsm, st))) return rc;
            if (timed) GTS_CUDA_TRY(cudaEventRecord(idx->fev[1], st));
            idx->kernel_launches += 9;   // keys, init, arec, need_sb, need_blk, items, tile, stat, final
        }
        k_add_stat<<<1, 1, 0, st>>>(idx->d_stats + 6, 1ull);
        k_fast_range_final<<<n, 128, 0, st>>>(idx->rows, idx->dim, idx->num, bs.prow, fs.kp, bs.ids, nb * kFB, dq, r,
                                              rb.cpos, rb.ccnt, rcnt, d_counts + q0, fail, rb.ctr, idx->d_stats);
        GTS_CUDA_TRY(cudaGetLastError());
        int status = 0, n_fail = 0;
        GTS_CUDA_TRY(cudaMemcpyAsync(&status, idx->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
        GTS_CUDA_TRY(cudaMemcpyAsync(&n_fail, rb.ctr, sizeof(int), cudaMemcpyDeviceToHost, st));
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
        if (n_fail > 0) {
            // overflowed lists: the plain traversal counts those queries
            k_gather_i<<<(n_fail + 255) / 256, 256, 0, st>>>(dq, fail, n_fail, sub_q);
            idx->keep_stats = true;
            rc = search_range(idx, sub_q, n_fail, r, sub_c, nullptr, st);
            idx->keep_stats = false;
            if (rc) return rc;
            k_scatter_i<<<(n_fail + 255) / 256, 256, 0, st>>>(fail, n_fail, sub_c, d_counts + q0);
            idx->kernel_launches += 2;
            GTS_CUDA_TRY(cudaGetLastError());
        }
    }
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    return GTS_OK;
}

int fast_config_get(const gts_index *idx, int k, int *tuned, int *learned, int *cg, int *item, int *variant)
{
    if (k < 1 || k > kFMaxK) {
        gts_set_error("k must be in [1, %d], got %d", kFMaxK, k);
        return GTS_ERR_INVALID;
    }
    const int v = idx->fast_cfg[k];
    const FastCfg c = v ? cfg_unpack(v) : fast_default_cfg(idx, k);
    if (tuned) *tuned = v ? 1 : 0;
    if (learned) *learned = c.learned ? 1 : 0;
    if (cg) *cg = c.cg;
    if (item) *item = c.item;
    if (variant) *variant = cfg_variant(c);
    return GTS_OK;
}

}  // namespace gts

extern "C" int gts_fast_config(const gts_index *idx, int k, int *tuned, int *learned, int *col_groups, int *item_blocks,
                               int *variant)
{
    if (!idx) {
        gts_set_error("null index");
        return GTS_ERR_INVALID;
    }
    return gts::fast_config_get(idx, k, tuned, learned, col_groups, item_blocks, variant);
}

extern "C" int gts_fast_config_set(gts_index *idx, int k, int learned, int col_groups, int item_blocks, int variant)
{
    if (!idx || k < 1 || k > gts::kFMaxK || (col_groups != 1 && col_groups != 2 && col_groups != 4) ||
        col_groups * k > 128 || (item_blocks != 8 && item_blocks != 16 && item_blocks != 32) || variant < 0 ||
        variant > 2) {
        gts_set_error("gts_fast_config_set: k in [1, 64], column groups 1/2/4 with groups * k <= 128, "
                      "8/16/32 blocks per item, filter variant 0/1/2");
        return GTS_ERR_INVALID;
    }
    const gts::FastShape fs = gts::fast_shape(idx->dim);
    const bool l2 = idx->metric == gts::kL2 && idx->dim <= gts::kFMaxKp;
    const bool blk = variant == 2;
    if (blk && l2 && gts::fast_blk_stages(fs) < 2) {
        gts_set_error("gts_fast_config_set: the block-stationary filter needs dim <= %d (got %d)", gts::kFResKp,
                      idx->dim);
        return GTS_ERR_INVALID;
    }
    const bool stream = !blk && (variant == 1 || fs.kp > gts::kFResKp);
    if (!blk && l2 && !gts::fast_tile_fits(fs, col_groups, k, stream)) {
        gts_set_error("gts_fast_config_set: %d column groups at k %d do not fit the shared memory at dim %d",
                      col_groups, k, idx->dim);
        return GTS_ERR_INVALID;
    }
    idx->fast_cfg[k] = gts::cfg_pack(gts::FastCfg{learned != 0, col_groups, item_blocks, stream, blk});
    return GTS_OK;
}

extern "C" int gts_fast_range_variant(gts_index *idx, int variant, int *current)
{
    if (!idx || variant < -1 || variant > 1) {
        gts_set_error("gts_fast_range_variant: variant -1, 0 or 1");
        return GTS_ERR_INVALID;
    }
    if (variant >= 0) idx->range_variant = variant;
    if (current) *current = idx->range_variant;
    return GTS_OK;
}

extern "C" int gts_fast_graphs(gts_index *idx, int on, long long *replays)
{
    if (!idx) {
        gts_set_error("null index");
        return GTS_ERR_INVALID;
    }
    if (on >= 0) {
        idx->use_graphs = on != 0;
        if (!idx->use_graphs) gts::graph_invalidate(idx);
    }
    if (replays) *replays = idx->graph_launches;
    return GTS_OK;
}

namespace gts {
__global__ void k_fast_seed_get(const int *__restrict__ qids, int qnum, const int *__restrict__ pos_of,
                                const int *__restrict__ selfk, int jk, int *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < qnum) out[i] = selfk[(size_t)pos_of[qids[i]] * kSelfK + jk];
}
}  // namespace gts

extern "C" int gts_fast_seeds(gts_index *idx, const int *qids, int qnum, int k, float *seeds_out)
{
    if (!idx || qnum < 0 || (qnum > 0 && (!qids || !seeds_out)) || k < 1 || k > gts::kFMaxK) {
        gts_set_error("gts_fast_seeds: invalid argument (k in [1, %d])", gts::kFMaxK);
        return GTS_ERR_INVALID;
    }
    if (!idx->fast_recs) {
        gts_set_error("gts_fast_seeds: the index holds no filter records (gts_index_prepare with GTS_FORM_FAST)");
        return GTS_ERR_INVALID;
    }
    for (int i = 0; i < qnum; i++)
        if (qids[i] < 0 || qids[i] >= idx->num) {
            gts_set_error("gts_fast_seeds: query id %d out of range", qids[i]);
            return GTS_ERR_INVALID;
        }
    if (qnum == 0) return GTS_OK;
    const gts::FastShape fs = gts::fast_shape(idx->dim);
    const gts::FastSummary bs = gts::fast_summary(idx->fast_recs, fs, idx->fast_nb, idx->fast_nsb, idx->num);
    int jk = 0;
    while ((1 << jk) < k) jk++;
    int *d = nullptr;
    GTS_CUDA_TRY(cudaMalloc(&d, 2 * sizeof(int) * (size_t)qnum));
    cudaError_t e = cudaMemcpy(d, qids, sizeof(int) * (size_t)qnum, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        gts::k_fast_seed_get<<<(qnum + 255) / 256, 256>>>(d, qnum, bs.pos, bs.selfk, jk, d + qnum);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(seeds_out, d + qnum, sizeof(int) * (size_t)qnum, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        gts_set_error("gts_fast_seeds: %s", cudaGetErrorString(e));
        return GTS_ERR_CUDA;
    }
    return GTS_OK;
}

extern "C" int gts_fast_autotune_reset(gts_index *idx)
{
    if (!idx) {
        gts_set_error("null index");
        return GTS_ERR_INVALID;
    }
    for (int &c : idx->fast_cfg) c = 0;
    return GTS_OK;
}
