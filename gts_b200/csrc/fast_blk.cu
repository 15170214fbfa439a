// fast_blk.cu -- the block-stationary form of the tensor-core filter.
//
// The tile filter (k_fast_tile, fast.cu) multiplies every block a query tile
// needs with all 128 queries of the tile.  When the queries are sparse
// against the data -- 10,000 queries over the 7,813 blocks of a 1,000,000 x
// 128 set -- a block that a tile needs is needed by one to three of its
// queries, and nearly all of that product is thrown away.  This form turns
// the product around: each needed block is read once per run and multiplied
// with just the queries that need it (up to kBQ at a time), the block's 128
// objects on the M side of the MMA (TMEM lanes) and the queries on the N
// side (16 or 32 columns).  The pass is then bound by the HBM stream of the
// block records, not by the tensor cores or the epilogue.
//
// Per (query, object) pair the arithmetic and the certified bounds are the
// tile filter's: d^2 = |q|^2 - 2 q.c + w - 2 q.bf16(r) - 2 (q - c).d with
// the same error terms; q.c comes from CUDA cores (FP32, from the same BF16
// hi + lo split of q that the MMA reads), inside the error term the tile
// filter allows for it.  No object whose reference distance can rank in the
// top k (or lie within the radius) is dropped.
//
// The run:
//   k_need_blk (fast.cu)  per (tile, needed block) a 128-bit mask of the
//                         tile's queries that need it; per block a count
//   k_bq_items            exclusive scan of the counts: each block's pairs
//                         get a range, split into items of <= kBQ queries
//   k_bq_fill             the pairs' query slots into their block's range
//   k_bq_build            per item, its header: per column the query's bound
//                         terms against this block and its tile slot
//   k_fast_blk            persistent CTAs stream (block record, item header)
//                         pairs through shared memory, gather the item's
//                         query rows from the tile records (L2), MMA, and
//                         list every object whose lower bound is within the
//                         query's bound (range: count the certain ones)
// Pairs beyond the run's capacity (qnum * kBPairs) are not listed; their
// queries are marked (kFListDropped) and answered again by the re-answer
// stages, so the answers stay exact.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include "fast.cuh"
#include "fast_blk.cuh"
#include "sm100.cuh"

namespace gts {

using namespace sm100;

namespace {

constexpr int kBSMax = 6;         // record stages at most
constexpr int kBAcc = 32;         // TMEM columns per accumulator (kBQ)
constexpr int kBRing = 16;        // item descriptor slots
constexpr int kBPre = 8;          // descriptors in flight ahead of the one in use
constexpr int kBEG = 3;           // epilogue warpgroups (at most the stages: the phase waits rely on it)
constexpr int kGRing = 8;         // query-slot ring of the gather warp (items)

// One column of an item: the query's bound terms against the item's block.
// x = w - A |d| - 2 v is lb - T for an object (v its MMA product):
//   pass (listed)    x <= RT  (RT = R2 - T)
//   range: certain   x + 2 (A |d| + eb) < RLT
struct __align__(16) BlkCol {
    float A, RT, T, eb;
    float RLT;
    int qi;       // query index in the run; -1: unused column or ball beyond the bound
    int slot;     // the query's tile slot (tile * 128 + lane)
    int pad;
};
static_assert(sizeof(BlkCol) * kBQ == kBHead, "item header size");

struct __align__(16) BlkCtl {
    uint64_t full[kBSMax];    // record + item header landed in stage s
    uint64_t gfull[kBSMax];   // the item's query rows gathered into stage s
    uint64_t mmad[kBSMax];    // MMA chain into accumulator s done
    uint64_t rfree[kBSMax];   // epilogue read the record tail of stage s (one arrive per warp)
    uint64_t efree[kBSMax];   // epilogue of accumulator s done (one arrive per warp)
    uint32_t tmem;
    int err;
    int blk[kBSMax];          // item in stage s: its block and query count
    int ncol[kBSMax];
};

__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
// this thread's completed generic-proxy shared-memory writes, visible to the
// async proxy (the tensor core's operand reads)
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void cp_async4(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ float bfl(uint32_t v) { return __uint_as_float(v << 16); }   // low bf16 of a word
__device__ __forceinline__ float bfh(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }

}  // namespace

// ---------------------------------------------------------------- pairs

// One CTA: exclusive scan of the per-block pair counts (clamped so that no
// range passes pairs_cap), each block's items (kBQ queries each, the last
// one the rest) in block order.  Items: (block, first pair, queries, item
// index); an item's record sits at item * kBHead + first pair * 4 kp bytes.
__global__ void __launch_bounds__(1024) k_bq_items(int nb, const int *__restrict__ cnt, int *__restrict__ off,
                                                   int4 *__restrict__ items, int *__restrict__ n_items,
                                                   int pairs_cap, unsigned long long *stats)
{
    __shared__ int wsum[2][32];
    __shared__ int carry[2];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) carry[0] = carry[1] = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nb; b0 += 1024) {
        const int b = b0 + t;
        const int c = b < nb ? cnt[b] : 0;
        // inclusive warp scans of (pairs, items); items are clamped below
        int p = c, it = 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, p, o);
            if (lane >= o) p += y;
        }
        if (lane == 31) wsum[0][warp] = p;
        __syncthreads();
        if (warp == 0) {
            int v = wsum[0][lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += y;
            }
            wsum[0][lane] = v;
        }
        __syncthreads();
        const int pex = carry[0] + (warp > 0 ? wsum[0][warp - 1] : 0) + p - c;   // exclusive
        const int ce = pex >= pairs_cap ? 0 : min(c, pairs_cap - pex);
        const int ni = (ce + kBQ - 1) / kBQ;
        it = ni;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, it, o);
            if (lane >= o) it += y;
        }
        if (lane == 31) wsum[1][warp] = it;
        __syncthreads();
        if (warp == 0) {
            int v = wsum[1][lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += y;
            }
            wsum[1][lane] = v;
        }
        __syncthreads();
        const int iex = carry[1] + (warp > 0 ? wsum[1][warp - 1] : 0) + it - ni;
        if (b < nb) {
            off[b] = pex;
            for (int i = 0; i < ni; i++)
                items[iex + i] = make_int4(b, pex + i * kBQ, min(kBQ, ce - i * kBQ), iex + i);
        }
        __syncthreads();
        if (t == 1023) {
            carry[0] += wsum[0][31];
            carry[1] += wsum[1][31];
        }
        __syncthreads();
    }
    if (t == 0) {
        *n_items = carry[1];
        if (stats) atomicAdd(&stats[3], (unsigned long long)carry[0]);   // pairs, before the cap
    }
}

// One CTA per tile: each (tile, needed block) entry's queries into the
// block's pair range (query slot = tile * 128 + lane).  A pair beyond
// pairs_cap is not stored; its query is marked in cand_cnt.
__global__ void __launch_bounds__(256) k_bq_fill(const int *__restrict__ blist, const uint4 *__restrict__ bmask,
                                                 const int *__restrict__ bcnt, int nbcap, const int *__restrict__ off,
                                                 int *__restrict__ fill, int *__restrict__ bq, int pairs_cap,
                                                 const int *__restrict__ order, int qnum, int *__restrict__ cand_cnt)
{
    const int tile = blockIdx.x;
    const int n = min(bcnt[tile], nbcap);
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const size_t at = (size_t)tile * nbcap + e;
        const int blk = blist[at];
        const uint4 m = bmask[at];
        const uint32_t w[4] = {m.x, m.y, m.z, m.w};
        const int c = __popc(w[0]) + __popc(w[1]) + __popc(w[2]) + __popc(w[3]);
        if (c == 0) continue;
        int p = off[blk] + atomicAdd(&fill[blk], c);
        for (int wi = 0; wi < 4; wi++) {
            uint32_t x = w[wi];
            while (x) {
                const int lane = wi * 32 + __ffs(x) - 1;
                x &= x - 1;
                const int slot = tile * kFT + lane;
                if (p < pairs_cap) {
                    bq[p] = slot;
                } else if (slot < qnum) {
                    atomicOr(&cand_cnt[order[slot]], kFListDropped);
                }
                p++;
            }
        }
    }
}

// One warp per item: the item's header, kBQ columns (BlkCol) of the bound
// terms of its queries against its block.  q.c comes from the query's BF16
// hi + lo operand rows in its tile record (what the MMA multiplies) and the
// block's FP32 centre: lane l holds one 16-byte unit (8 dimensions) of the
// hi or lo rows.
__global__ void __launch_bounds__(256) k_bq_build(const int4 *__restrict__ items, const int *__restrict__ n_items,
                                                  const int *__restrict__ bq, const unsigned char *__restrict__ arec,
                                                  const unsigned char *__restrict__ recs, const float *__restrict__ cen,
                                                  FastShape fs, const int *__restrict__ r2_bits, float r2lo,
                                                  unsigned char *__restrict__ irec)
{
    const int lane = threadIdx.x & 31;
    const int nit = *n_items;
    const int nk = fs.nk, units = 2 * nk * 8;   // 16-byte units of a query's hi + lo rows
    // this lane's unit: part p, chunk c, logical unit u (dimensions c * 64 + 8u .. +7)
    const int p = lane / (nk * 8), c = (lane / 8) % nk, u = lane & 7;
    const bool act = lane < units;
    for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < nit; it += (gridDim.x * blockDim.x) >> 5) {
        const int4 d = items[it];
        const int blk = d.x, p0 = d.y, nq = d.z;
        BlkCol *cols = reinterpret_cast<BlkCol *>(irec + (size_t)it * kBHead);
        // the centre values of this lane's eight dimensions
        float cv[8];
        {
            const float4 *cp = reinterpret_cast<const float4 *>(cen + (size_t)blk * fs.kp + c * 64 + 8 * u);
            const float4 a0 = act ? cp[0] : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 a1 = act ? cp[1] : make_float4(0.f, 0.f, 0.f, 0.f);
            cv[0] = a0.x; cv[1] = a0.y; cv[2] = a0.z; cv[3] = a0.w;
            cv[4] = a1.x; cv[5] = a1.y; cv[6] = a1.z; cv[7] = a1.w;
        }
        const int myslot = lane < nq ? bq[p0 + lane] : -1;
        float myqc = 0.f;
        for (int n = 0; n < nq; n++) {
            const int slot = __shfl_sync(0xffffffffu, myslot, n);
            const int tile = slot >> 7, L = slot & 127;
            float part = 0.f;
            if (act) {
                const uint4 v = *reinterpret_cast<const uint4 *>(arec + (size_t)tile * fs.arec_bytes +
                                                                 (size_t)p * fs.atile_bytes + (size_t)c * (kFT * 128) +
                                                                 (size_t)L * 128 + ((u ^ (L & 7)) << 4));
                part = fmaf(bfl(v.x), cv[0], part);
                part = fmaf(bfh(v.x), cv[1], part);
                part = fmaf(bfl(v.y), cv[2], part);
                part = fmaf(bfh(v.y), cv[3], part);
                part = fmaf(bfl(v.z), cv[4], part);
                part = fmaf(bfh(v.z), cv[5], part);
                part = fmaf(bfl(v.w), cv[6], part);
                part = fmaf(bfh(v.w), cv[7], part);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
            if (lane == n) myqc = part;
        }
        // column lane: the query's terms against this block (the tile
        // filter's epilogue terms, with q.c from the sum above: FP32 over
        // at most 16 products per lane and a 5-level tree, inside kEpsC)
        float4 f0 = make_float4(0.f, 0.f, 0.f, 0.f);   // A, RT, T, eb
        int4 f1 = make_int4(0, -1, 0, 0);               // RLT (bits), qi, query slot
        if (lane < nq) {
            const int tile = myslot >> 7, L = myslot & 127;
            const int4 inf = *reinterpret_cast<const int4 *>(arec + (size_t)tile * fs.arec_bytes + 2 * fs.atile_bytes +
                                                             (size_t)L * 16);
            const int qi = inf.x;
            if (qi >= 0) {
                const float q2 = __int_as_float(inf.y), qn = __int_as_float(inf.z);
                const float R2 = __int_as_float(*(volatile const int *)(r2_bits + qi));
                const float *tail = reinterpret_cast<const float *>(recs + (size_t)blk * fs.rec_bytes + fs.btile_bytes);
                const float cn = tail[kTailC], rb = tail[kTailRb], wb = tail[kTailWb], brad = tail[kTailRad];
                const float es = eps_scale(fs.kp);
                const float cr = 2.f * kEpsR * es * qn;
                const float ec = 2.f * kEpsC * es * qn * cn + 1e-6f;
                const float c2 = cn * cn;
                const float qmc2 = q2 - 2.f * myqc + c2;
                const float A = 2.000004f * sqrtf(fmaxf(qmc2 + ec + 4e-6f * (q2 + c2), 0.f)) + 2e-6f * cn;
                const float eb = ec + 2e-6f * q2 + cr * rb + 2e-6f * wb;
                const float T = q2 - 2.f * myqc - eb;
                const float dlo = sqrtf(fmaxf(qmc2 - ec - 4e-6f * (q2 + c2), 0.f)) * 0.999999f - brad;
                const bool skip = dlo > 0.f && dlo * dlo * 0.999999f > R2;
                f0 = make_float4(A, R2 - T, T, eb);
                f1 = make_int4(__float_as_int(r2lo - T - 2e-6f * q2), skip ? -1 : qi, myslot, 0);
            }
        }
        reinterpret_cast<float4 *>(cols + lane)[0] = f0;
        reinterpret_cast<int4 *>(cols + lane)[1] = f1;
    }
}

// ---------------------------------------------------------------- filter

// Persistent filter, one CTA per SM: 4 epilogue warps (warp w: TMEM lanes
// and block objects 32w .. 32w + 31), one producer warp and one gather
// warp.  CTA b takes items b, b + G, b + 2G, ...  Per item j (stage s =
// j % S, accumulator s, header slot j % 2S):
//   producer: copy the block record and the item header into stage s with
//             bulk copies (S - 1 items ahead; stage s is reused once the
//             epilogue of item j - S has read its record tail, its MMAs being
//             done), wait for them and for the gathered query rows, wait for
//             the epilogue of item j - S (frees accumulator s), then the MMA
//             chain objects x queries into accumulator s, hi and lo parts.
//   gather:   once the MMAs of item j - S are done, copy the item's query
//             rows (hi, lo) from their tile records, which stay in L2, into
//             the stage's operand area: 16-byte cp.async copies, row n's
//             units re-swizzled from the tile row's position to row n's;
//             one item behind, wait for the copies, fence them for the
//             tensor core's proxy and arrive on gfull.
//   epilogue: wait the MMA, read the objects' w and |d| (then the stage is
//             free), bound every (object, column) pair, list the passing
//             objects in their query's candidate list (one atomic per warp
//             and column), arrive on efree[s].
// The header of item j stays in its own slot until the epilogue of item
// j + S - 1 starts (2S slots), so the stage can be refilled early.
template <int EG, bool RANGE>
__global__ void __launch_bounds__(128 * EG + 64, 1) k_fast_blk(FastBlkArgs a)
{
    extern __shared__ __align__(1024) unsigned char bsm[];
    unsigned char *base = bsm + ((1024u - (smem_u32(bsm) & 1023u)) & 1023u);
    const FastShape fs = a.fs;
    const int S = a.nst;
    const uint32_t rec_pad = (fs.rec_bytes + 1023u) & ~1023u;
    const uint32_t part_bytes = (uint32_t)fs.nk * kBQ * 128u;
    const uint32_t stage_bytes = rec_pad + 2u * part_bytes;
    BlkCol *heads = reinterpret_cast<BlkCol *>(base + (size_t)S * stage_bytes);   // [2S][kBQ]
    BlkCtl &ctl = *reinterpret_cast<BlkCtl *>(heads + (size_t)2 * S * kBQ);
    int4 *ring = reinterpret_cast<int4 *>(&ctl + 1);     // producer's item descriptors
    int4 *gring = ring + kBRing;                          // gather warp's item descriptors
    int (*sring)[kBQ] = reinterpret_cast<int (*)[kBQ]>(gring + kBRing);   // gather warp's query slots

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int G = gridDim.x;
    const int nit = *a.n_items;
    const int n_local = (int)blockIdx.x < nit ? (nit - (int)blockIdx.x + G - 1) / G : 0;

    if (t == 0) {
        for (int s = 0; s < kBSMax; s++) {
            mbar_init(&ctl.full[s], 1);
            mbar_init(&ctl.gfull[s], 1);
            mbar_init(&ctl.mmad[s], 1);
            mbar_init(&ctl.rfree[s], 4);
            mbar_init(&ctl.efree[s], 4);
        }
        ctl.err = 0;
        fence_mbar_init();
    }
    const uint32_t tcols = S * kBAcc <= 32 ? 32u : (S * kBAcc <= 64 ? 64u : (S * kBAcc <= 128 ? 128u : 256u));
    if (warp == 0) {
        tmem_alloc(&ctl.tmem, tcols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = ctl.tmem;
    unsigned long long appended = 0;

    constexpr int PW = 4 * EG;   // producer warp; the gather warp follows it
    if (warp == PW) {
        if (lane == 0) {
            // producer bookkeeping for the bounded drain on error: last item
            // whose copies were issued / waited, last whose MMAs were committed
            int c_iss = -1, c_wait = -1, m_iss = -1, err = 0;
            // descriptor of item j into ring slot j % kBRing, one copy group
            // per item (empty past the last), kBPre items ahead; the slot it
            // overwrites was read kBRing - kBPre items earlier
            auto prefetch = [&](int j) {
                if (j < n_local) cp_async16(ring + j % kBRing, a.items + (size_t)blockIdx.x + (size_t)j * G);
                cp_async_commit();
            };
            for (int j = 0; j < kBPre; j++) prefetch(j);
            auto issue = [&](int j) {   // copies of item j into stage j % S
                const int s = j % S;
                cp_async_wait<kBPre - 1>();   // j + kBPre groups committed: descriptor j landed
                const int4 d = ring[j % kBRing];
                prefetch(j + kBPre);
                const int blk = d.x, nq = d.z, it = d.w;
                ctl.blk[s] = blk;
                ctl.ncol[s] = nq;
                unsigned char *st = base + (size_t)s * stage_bytes;
                mbar_arrive_expect_tx(&ctl.full[s], fs.rec_bytes + (uint32_t)kBHead);
                bulk_g2s(st, a.recs + (size_t)blk * fs.rec_bytes, fs.rec_bytes, &ctl.full[s]);
                bulk_g2s(heads + (size_t)(j % (2 * S)) * kBQ, a.irec + (size_t)it * kBHead, (uint32_t)kBHead,
                         &ctl.full[s]);
                c_iss = j;
            };
            for (int j = 0; j < S - 1 && j < n_local; j++) issue(j);
            const uint32_t kpart = (uint32_t)fs.nk * kBQ * 128u;
            for (int j = 0; j < n_local; j++) {
                const int s = j % S;
                if (*(volatile int *)&ctl.err) break;
                if (j + S - 1 < n_local) {
                    // stage (j - 1) % S: free once the epilogue of item j - 1 read its tail
                    if (j >= 1 && !mbar_wait(&ctl.rfree[(j - 1) % S], (uint32_t)(((j - 1) / S) & 1), kFWait)) {
                        err = 3;
                        break;
                    }
                    issue(j + S - 1);
                }
                if (!mbar_wait(&ctl.full[s], (uint32_t)((j / S) & 1), kFWait)) { err = 1; break; }
                c_wait = j;
                if (!mbar_wait(&ctl.gfull[s], (uint32_t)((j / S) & 1), kFWait)) { err = 5; break; }
                // accumulator s: the epilogue of item j - S is done
                if (j >= S && !mbar_wait(&ctl.efree[s], (uint32_t)(((j - S) / S) & 1), kFWait)) { err = 2; break; }
                tc_fence_after();
                const int nq = ctl.ncol[s];
                const int N = (nq + 15) & ~15;
                const uint32_t idesc = idesc_bf16_f32(128, N);
                const uint32_t rs = smem_u32(base + (size_t)s * stage_bytes);
                const uint64_t da = smem_desc_sw128(rs, 1024);
                const uint64_t dbh = smem_desc_sw128(rs + rec_pad, 1024), dbl = smem_desc_sw128(rs + rec_pad + kpart, 1024);
                const uint32_t dt = tmem + (uint32_t)(s * kBAcc);
                const int ksteps = fs.kp / 16;
                for (int kk = 0; kk < ksteps; kk++) {
                    const uint64_t ao = ((uint64_t)(kk >> 2) * kFChunkBytes + (uint64_t)(kk & 3) * 32u) >> 4;
                    const uint64_t bo = ((uint64_t)(kk >> 2) * (kBQ * 128u) + (uint64_t)(kk & 3) * 32u) >> 4;
                    mma_bf16(dt, da + ao, dbh + bo, idesc, kk > 0 ? 1u : 0u);
                }
                for (int kk = 0; kk < ksteps; kk++) {
                    const uint64_t ao = ((uint64_t)(kk >> 2) * kFChunkBytes + (uint64_t)(kk & 3) * 32u) >> 4;
                    const uint64_t bo = ((uint64_t)(kk >> 2) * (kBQ * 128u) + (uint64_t)(kk & 3) * 32u) >> 4;
                    mma_bf16(dt, da + ao, dbl + bo, idesc, 1u);
                }
                mma_commit(&ctl.mmad[s]);
                m_iss = j;
            }
            if (err) atomicMax(&ctl.err, err);
            if (*(volatile int *)&ctl.err) {
                // copies and MMAs still in flight finish before the CTA leaves (bounded)
                for (int j = c_wait + 1; j <= c_iss; j++)
                    mbar_wait(&ctl.full[j % S], (uint32_t)((j / S) & 1), kFWait);
                if (m_iss >= 0) mbar_wait(&ctl.mmad[m_iss % S], (uint32_t)((m_iss / S) & 1), kFWait);
            }
            cp_async_wait_all();
            if (a.stats && c_wait >= 0) {
                atomicAdd(&a.stats[0], (unsigned long long)(c_wait + 1));
                atomicAdd(&a.stats[1], (unsigned long long)fs.rec_bytes * (c_wait + 1));
            }
        }
        __syncwarp();
    } else if (warp == PW + 1) {
        // gather: lane l copies one 16-byte unit (part p, K chunk c, unit u)
        // of every query row of the item.  Nothing on its path waits for a
        // global load: item descriptors come kBPre items ahead and the
        // items' query slots kGSlot items ahead, both by cp.async into rings
        // (copy group j of this warp: item j's rows, descriptor j + kBPre,
        // slots j + kGSlot).
        constexpr int kGSlot = 4;
        const int nk = fs.nk, units = 2 * nk * 8;
        const int p = lane / (nk * 8), c = (lane / 8) % nk, u = lane & 7;
        const bool act = lane < units;
        const size_t src_off = (size_t)p * fs.atile_bytes + (size_t)c * (kFT * 128);
        const uint32_t dst_off = rec_pad + (uint32_t)p * part_bytes + (uint32_t)c * (kBQ * 128u);
        auto desc_of = [&](int j) { return a.items + (size_t)blockIdx.x + (size_t)j * G; };
        auto fetch_slots = [&](int j) {   // query slots of item j (its descriptor is in gring)
            const int4 d = gring[j % kBRing];
            if (lane < d.z) cp_async4(&sring[j % kGRing][lane], a.bq + d.y + lane);
        };
        // prologue, synchronous: descriptors 0 .. kBPre - 1, slots 0 .. kGSlot - 1
        if (lane == 0)
            for (int j = 0; j < kBPre && j < n_local; j++) cp_async16(gring + j % kBRing, desc_of(j));
        cp_async_commit();
        cp_async_wait_all();
        __syncwarp();
        for (int j = 0; j < kGSlot && j < n_local; j++) fetch_slots(j);
        cp_async_commit();
        cp_async_wait_all();
        __syncwarp();
        bool ok = true;
        for (int j = 0; j < n_local; j++) {
            const int s = j % S;
            // the operand area of stage s: free once the MMAs of item j - S are done
            if (j >= S &&
                !__all_sync(0xffffffffu, mbar_wait(&ctl.mmad[s], (uint32_t)(((j - S) / S) & 1), kFWait))) {
                ok = false;
                break;
            }
            if (__any_sync(0xffffffffu, *(volatile int *)&ctl.err != 0)) {
                ok = false;
                break;
            }
            // descriptor j and slots j landed: copy groups up to j - 2 are done
            const int nq = gring[j % kBRing].z;
            const int slot = lane < nq ? sring[j % kGRing][lane] : 0;
            unsigned char *dst = base + (size_t)s * stage_bytes + dst_off;
            for (int n = 0; n < nq; n++) {
                const int sl = __shfl_sync(0xffffffffu, slot, n);
                if (act) {
                    const int tile = sl >> 7, L = sl & 127;
                    cp_async16(dst + (size_t)n * 128 + ((u ^ (n & 7)) << 4),
                               a.arec + (size_t)tile * fs.arec_bytes + src_off + (size_t)L * 128 + ((u ^ (L & 7)) << 4));
                }
            }
            if (lane == 0 && j + kBPre < n_local) cp_async16(gring + (j + kBPre) % kBRing, desc_of(j + kBPre));
            if (j + kGSlot < n_local) fetch_slots(j + kGSlot);
            cp_async_commit();
            if (j >= 1) {   // group j - 1 done: item j - 1's rows landed, hand them to the producer
                cp_async_wait<1>();
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(&ctl.gfull[(j - 1) % S]);
            }
        }
        cp_async_wait_all();
        if (ok && n_local > 0) {
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&ctl.gfull[(n_local - 1) % S]);
        }
        __syncwarp();
    } else {
        // epilogue warpgroup g takes items g, g + EG, ...; warp w of a group
        // owns TMEM lanes and block objects 32 (w % 4) .. + 31
        const int g = warp >> 2, wq = warp & 3;
        const int m = wq * 32 + lane;   // block object, TMEM lane
        const uint32_t trow = (uint32_t)(wq * 32) << 16;
        const unsigned lt = (1u << lane) - 1u;
        const int k = a.k;
        for (int j = g; j < n_local; j += EG) {
            const int s = j % S;
            const uint32_t ph = (uint32_t)((j / S) & 1);
            // the copies of item j landed (record tail, header): visible here
            mbar_wait(&ctl.full[s], ph, kFWait);
            const BlkCol *cols = heads + (size_t)(j % (2 * S)) * kBQ;
            // column lane (kBQ = 32 columns): the query's bound now -- other
            // items may have lowered it since the header was built -- as
            // r2c and as rtc = min(RT, r2c - T), read while the MMA runs
            float r2c = 0.f, rtc = 0.f;
            {
                const BlkCol cl = cols[lane];
                if (cl.qi >= 0) {
                    r2c = RANGE ? cl.RT + cl.T : __int_as_float(*(volatile const int *)(a.r2_bits + cl.qi));
                    rtc = RANGE ? cl.RT : fminf(cl.RT, r2c - cl.T);
                }
            }
            // one verdict per warp: the TMEM loads below are warp-collective
            if (!__all_sync(0xffffffffu, mbar_wait(&ctl.mmad[s], ph, kFWait))) {
                atomicMax(&ctl.err, 4);
                break;
            }
            tc_fence_after();
            const float *tail = reinterpret_cast<const float *>(base + (size_t)s * stage_bytes + fs.btile_bytes);
            const float w = tail[kTailW + m], dn = tail[kTailDn + m];
            const int blk = ctl.blk[s], nq = ctl.ncol[s];
            __syncwarp();
            if (lane == 0) mbar_arrive(&ctl.rfree[s]);
            const int slot = blk * kFB + m;
            for (int c0 = 0; c0 < nq; c0 += 16) {
                uint32_t v[16];
                __syncwarp();
                tmem_ld16_nowait(tmem + trow + (uint32_t)(s * kBAcc + c0), v);
                tmem_wait_ld(v);
                uint32_t pass = 0, inside = 0;
#pragma unroll
                for (int u = 0; u < 16; u++) {
                    const BlkCol cc = cols[c0 + u];
                    const float rt = __shfl_sync(0xffffffffu, rtc, c0 + u);
                    const float x = fmaf(-2.f, __uint_as_float(v[u]), fmaf(-cc.A, dn, w));
                    const bool ok = cc.qi >= 0 && c0 + u < nq;
                    pass |= (ok && x <= rt ? 1u : 0u) << u;
                    if constexpr (RANGE) inside |= (ok && x + 2.f * fmaf(cc.A, dn, cc.eb) < cc.RLT ? 1u : 0u) << u;
                }
                if constexpr (RANGE) {
                    pass &= ~inside;
                    // certain objects: one count per (warp, column)
                    int mine = 0;
#pragma unroll
                    for (int u = 0; u < 16; u++) {
                        const int cnt = __popc(__ballot_sync(0xffffffffu, (inside >> u) & 1u));
                        if (lane == u) mine = cnt;
                    }
                    if (mine) atomicAdd(a.rcnt + cols[c0 + lane].qi, mine);
                }
                if (!__any_sync(0xffffffffu, pass != 0)) continue;
                // one list reservation per (warp, column): lane u for column c0 + u
                uint32_t bal[16];
                int mine = 0;
#pragma unroll
                for (int u = 0; u < 16; u++) {
                    bal[u] = __ballot_sync(0xffffffffu, (pass >> u) & 1u);
                    if (lane == u) mine = __popc(bal[u]);
                }
                int mybase = 0;
                if (mine) mybase = atomicAdd(&a.cand_cnt[cols[c0 + lane].qi], mine);
                appended += __popc(pass);
#pragma unroll
                for (int u = 0; u < 16; u++) {
                    const int b = __shfl_sync(0xffffffffu, mybase, u);
                    float ub = INFINITY;
                    if ((pass >> u) & 1u) {
                        const BlkCol cc = cols[c0 + u];
                        const float lb = cc.T + fmaf(-2.f, __uint_as_float(v[u]), fmaf(-cc.A, dn, w));
                        ub = lb + 2.f * fmaf(cc.A, dn, cc.eb);
                        const int at = b + __popc(bal[u] & lt);
                        if (at < kFCand) {
                            const size_t o = (size_t)cc.qi * kFCand + at;
                            a.cand_pos[o] = slot;
                            a.cand_lb[o] = lb;
                            a.cand_ub[o] = ub;
                        }
                    }
                    if constexpr (!RANGE) {
                        // k distinct objects of this warp with upper bounds
                        // below the query's bound: their k-th smallest upper
                        // bound is a bound on its k-th distance (the tile
                        // filter's running bound, per warp and block)
                        const float r2u = __shfl_sync(0xffffffffu, r2c, c0 + u);
                        const unsigned below = __ballot_sync(0xffffffffu, ub < r2u);
                        if (k <= 32 && __popc(below) >= k) {
                            float x = ub < r2u ? ub : INFINITY, mn = x;
                            for (int it = 0; it < k; it++) {
                                mn = x;
#pragma unroll
                                for (int o = 16; o > 0; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
                                if (it == k - 1) break;
                                const unsigned own = __ballot_sync(0xffffffffu, x == mn);
                                if (lane == __ffs(own) - 1) x = INFINITY;
                            }
                            const BlkCol cc = cols[c0 + u];
                            if (lane == 0) atomicMin(a.r2_bits + cc.qi, __float_as_int(fmaxf(mn, 0.f)));
                            if (lane == c0 + u) {
                                r2c = fminf(r2c, mn);
                                rtc = fminf(rtc, mn - cc.T);
                            }
                        }
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&ctl.efree[s]);
        }
    }
    if (a.stats && appended) atomicAdd(&a.stats[5], appended);
    if (t == 0 && ctl.err) atomicMax(a.status, 32 + ctl.err);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, tcols);
}

// ---------------------------------------------------------------- host

size_t fast_blk_smem(const FastShape &fs, int nst)
{
    const size_t rec_pad = (fs.rec_bytes + 1023u) & ~1023u;
    const size_t stage = rec_pad + 2 * (size_t)fs.nk * kBQ * 128;
    return 1024 + (size_t)nst * stage + (size_t)2 * nst * kBHead + sizeof(BlkCtl) + 2 * kBRing * sizeof(int4) +
           (size_t)kGRing * kBQ * sizeof(int);
}

int fast_blk_stages(const FastShape &fs)
{
    if (fs.kp > kFResKp) return 0;
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // at least one stage per epilogue warpgroup
    for (int s = kBSMax; s >= std::max(2, kBEG); s--)
        if (fast_blk_smem(fs, s) <= (size_t)optin) return s;
    return 0;
}

size_t fast_blk_items_cap(int nb, int pairs_cap) { return (size_t)nb + (size_t)pairs_cap / kBQ + 1; }

size_t fast_blk_irec_bytes(int nb, int pairs_cap) { return fast_blk_items_cap(nb, pairs_cap) * kBHead; }

int fast_blk_enqueue(const FastBlkRun &r, cudaStream_t st, long long *launches)
{
    const FastShape fs = r.args.fs;
    k_bq_items<<<1, 1024, 0, st>>>(r.nb, r.bq_cnt, r.bq_off, r.items, r.n_items, r.pairs_cap, r.args.stats);
    k_bq_fill<<<r.ntiles, 256, 0, st>>>(r.blist, r.bmask, r.bcnt, r.nbcap, r.bq_off, r.bq_fill, r.bq, r.pairs_cap,
                                        r.order, r.qnum, r.args.cand_cnt);
    const int build_grid = (int)std::min<size_t>((fast_blk_items_cap(r.nb, r.pairs_cap) + 7) / 8, (size_t)8 * r.nsm);
    k_bq_build<<<build_grid, 256, 0, st>>>(r.items, r.n_items, r.bq, r.arec, r.args.recs, r.cen, fs, r.args.r2_bits,
                                           r.args.r2lo, r.irec);
    FastBlkArgs a = r.args;
    a.irec = r.irec;
    a.items = r.items;
    a.bq = r.bq;
    a.arec = r.arec;
    a.n_items = r.n_items;
    a.nst = fast_blk_stages(fs);
    if (a.nst < 2) {
        gts_set_error("block-stationary filter: kp %d leaves no room for two stages", fs.kp);
        return GTS_ERR_INVALID;
    }
    const size_t smem = fast_blk_smem(fs, a.nst);
    const unsigned rec_flags = r.capturing ? cudaEventRecordExternal : 0;
    if (r.timed_begin) GTS_CUDA_TRY(cudaEventRecordWithFlags(r.timed_begin, st, rec_flags));
    // kBEG epilogue warpgroups take turns on the items, so that many items'
    // list reservations (global atomics) are in flight per SM
    if (r.range) {
        GTS_CUDA_TRY(cudaFuncSetAttribute(k_fast_blk<kBEG, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        k_fast_blk<kBEG, true><<<r.nsm, 128 * kBEG + 64, smem, st>>>(a);
    } else {
        GTS_CUDA_TRY(cudaFuncSetAttribute(k_fast_blk<kBEG, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        k_fast_blk<kBEG, false><<<r.nsm, 128 * kBEG + 64, smem, st>>>(a);
    }
    if (r.timed_end) GTS_CUDA_TRY(cudaEventRecordWithFlags(r.timed_end, st, rec_flags));
    if (launches) *launches += 4;
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

}  // namespace gts
