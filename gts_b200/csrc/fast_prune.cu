// fast_prune.cu -- the fast form's ball pruning on the tensor cores.
//
// Before the filter streams any block, each 128-query tile finds the
// superblocks, then the blocks, that some of its queries can reach within
// their seeds: a ball (centre c, radius rad) is needed by query q when
// |q - c|_lo - rad <= sqrt(seed(q)), with |q - c|^2 = |q|^2 - 2 q.c + |c|^2.
// The q.c products of a tile against a group of 32 balls are one
// 128 x 96 x kp tcgen05.mma pair: the A operand is the tile's query operand
// (BF16 hi + lo, the same tile record the filter reads) and the B operand
// holds each centre as three BF16 rows hi + mid + lo (an exact split of the
// FP32 centre, the layout of the centre rows in the filter's block records).
// The epilogue sums the three columns of a ball and applies a certified ball
// test that skips less than the filter's own (the skip test of
// k_fast_tile), so the blocks kept are a superset of those the filter would
// not skip.  Up to a padded dimension of 128 (kFResKp); wider indexes use
// the FP32 pruning kernels in fast.cu.
//
// Centre operands: all superblocks (or blocks) in id order, 3 rows per ball,
// in the K-major 128-byte swizzled layout of an operand of R = 3 * n32 rows
// (n32: the ball count rounded up to 32); a group of 32 balls is one
// contiguous 12 KB range per 64-wide K chunk, copied with one bulk copy each.
#include <cuda_bf16.h>
#include <algorithm>
#include "fast.cuh"
#include "sm100.cuh"

namespace gts {

using namespace sm100;

namespace {

constexpr int kPG = 32;                 // balls per group
constexpr int kPN = 3 * kPG;            // B rows per group (MMA N)
constexpr uint32_t kPlane = kPN * 128u; // bytes of one group per 64-wide K chunk
constexpr int kPS = 4;                  // group stages, each with its own TMEM accumulator
constexpr uint32_t kPAccCols = 128u;    // TMEM columns between accumulators (kPN used)
constexpr int kPEpi = 512;              // epilogue threads: sixteen warps, four per TMEM lane quarter
constexpr int kPThreads = kPEpi + 64;   // and two producer warps (copies; MMAs)
constexpr int kPBW = kPG / 4;           // balls per epilogue warp
// Shared memory of a pruning CTA at least this large: one CTA per SM, whose
// 512 TMEM columns are then the SM's (two such CTAs exceed 228 KB).
constexpr size_t kPMinSmem = (size_t)116 << 10;

__device__ __forceinline__ unsigned short pr_f2bf(float x)
{
    return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
__device__ __forceinline__ float pr_bf2f(unsigned short b) { return __bfloat162float(__ushort_as_bfloat16(b)); }

// One thread per ball: its centre split into three BF16 rows.
__global__ void k_prune_cop(const float *__restrict__ cen, int n, int kp, int rows, unsigned char *__restrict__ cop)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int j = 0; j < kp; j++) {
        const float c = cen[(size_t)i * kp + j];
        const unsigned short hi = pr_f2bf(c);
        const float r1 = c - pr_bf2f(hi);
        const unsigned short mid = pr_f2bf(r1);
        const unsigned short lo = pr_f2bf(r1 - pr_bf2f(mid));
        *reinterpret_cast<unsigned short *>(cop + sw128_offset(3 * i, j, rows)) = hi;
        *reinterpret_cast<unsigned short *>(cop + sw128_offset(3 * i + 1, j, rows)) = mid;
        *reinterpret_cast<unsigned short *>(cop + sw128_offset(3 * i + 2, j, rows)) = lo;
    }
}

// Block groups the tile has to test: the groups of 32 blocks that hold
// blocks of its needed superblocks, with those blocks as a bit mask.  One
// CTA per tile; its items (tile, group, mask) in group order, appended as
// one contiguous range (one reservation per tile: tfirst, tcnt), so the
// pruning CTAs, which take contiguous item ranges, mostly stay on one tile.
// The items' result words (pword) start at zero.
__global__ void k_prune_items(const uint32_t *__restrict__ sb_mask, int nsbw, const int *__restrict__ sb_b0,
                              int ngroups, int4 *__restrict__ items, uint32_t *__restrict__ pword,
                              int *__restrict__ n_items, int items_cap, int *__restrict__ tfirst,
                              int *__restrict__ tcnt)
{
    extern __shared__ uint32_t gm[];   // [ngroups]
    const int tile = blockIdx.x, t = threadIdx.x, lane = t & 31;
    for (int g = t; g < ngroups; g += blockDim.x) gm[g] = 0u;
    __syncthreads();
    // a needed superblock's blocks are the contiguous range [b0, b1): one
    // shared atomicOr per 32-block word it touches
    for (int s = t; s < nsbw * 32; s += blockDim.x) {
        if (!((sb_mask[(size_t)tile * nsbw + (s >> 5)] >> (s & 31)) & 1u)) continue;
        const int b0 = sb_b0[s], b1 = sb_b0[s + 1];
        for (int w = b0 >> 5; w <= (b1 - 1) >> 5 && b1 > b0; w++) {
            const int lo = max(b0, w * 32) - w * 32, hi = min(b1, w * 32 + 32) - w * 32;   // bits [lo, hi)
            const uint32_t m = (hi - lo == 32) ? 0xffffffffu : (((1u << (hi - lo)) - 1u) << lo);
            atomicOr(&gm[w], m);
        }
    }
    __syncthreads();
    if (t < 32) {
        int cnt = 0;
        for (int g0 = 0; g0 < ngroups; g0 += 32) {
            const int g = g0 + lane;
            cnt += __popc(__ballot_sync(0xffffffffu, g < ngroups && gm[g] != 0u));
        }
        int at = 0;
        if (lane == 0 && cnt) at = atomicAdd(n_items, cnt);
        at = __shfl_sync(0xffffffffu, at, 0);
        if (lane == 0) {
            tfirst[tile] = at;
            tcnt[tile] = max(0, min(cnt, items_cap - at));
        }
        for (int g0 = 0; g0 < ngroups; g0 += 32) {
            const int g = g0 + lane;
            const uint32_t m = g < ngroups ? gm[g] : 0u;
            const uint32_t bal = __ballot_sync(0xffffffffu, m != 0u);
            if (m) {
                const int p = at + __popc(bal & ((1u << lane) - 1u));
                if (p < items_cap) {
                    items[p] = make_int4(tile, g, (int)m, 0);
                    pword[p] = 0u;
                }
            }
            at += __popc(bal);
        }
    }
}

struct PruneArgs {
    const unsigned char *arec;   // tile records (query operand hi + lo, lane info)
    const unsigned char *cop;    // centre operand of the balls
    int rows;                    // its rows (3 * n32)
    const float *c2, *rad;       // per ball: |c|^2, radius (< 0: empty ball)
    int nball;
    FastShape fs;
    const int *r2_bits;          // per query: the seed (float bits)
    int ntiles, ngroups;
    // superblock pass: mask words sb_mask[tile][group]
    uint32_t *sb_mask;
    int nsbw;
    // block pass: items from k_prune_items; per item the needed blocks of its
    // group as a bit mask (pword), and with plm the lanes of each quarter of
    // the tile that need each block (plm[item][ball][quarter])
    const int4 *items;
    const int *n_items;
    int items_cap;
    uint32_t *pword;
    uint32_t *plm;
    int *status;
};

struct PruneCtl {
    uint64_t bfull[kPS];   // the group operand of the stage's item landed
    uint64_t mmad[kPS];    // the MMA pair into the stage's accumulator is done
    uint64_t efree[kPS];   // the epilogue warps are done with the stage's accumulator (one arrive each)
    uint64_t afull;        // the tile's query operand landed
    uint32_t tmem;
    int err;               // a wait gave up (producer or epilogue): the rest skips its waits
    float4 bd[kPEpi / 32][kPBW];   // per epilogue warp: its balls' |c|, |c|^2 (1 - 5e-6), radius, usable
};

// Item it of the pass: its tile, ball group and the balls to test.
template <bool BLK>
__device__ __forceinline__ void prune_item(const PruneArgs &a, int it, int &tile, int &grp, uint32_t &elig)
{
    if (BLK) {
        const int4 e = a.items[it];
        tile = e.x;
        grp = e.y;
        elig = (uint32_t)e.z;
    } else {
        tile = it / a.ngroups;
        grp = it - tile * a.ngroups;
        elig = 0xffffffffu;
    }
}

// Bounded wait that also gives up as soon as the CTA's error flag is set.
__device__ __forceinline__ bool prune_wait(uint64_t *bar, uint32_t parity, const volatile int *err)
{
    for (long long i = 0; i < kFWait; i++) {
        if (mbar_try_wait_sleep(bar, parity, 1000u)) return true;
        if (*err) return false;
    }
    return false;
}

// Persistent CTAs (one per SM), each over a contiguous range of (tile,
// group) items (consecutive items mostly share the tile, whose operand then
// stays in shared memory).  Item j of the CTA uses stage and accumulator
// j % kPS.
//   copy thread (warp 16): the groups' centre operands, up to kPS items ahead
//     (a stage is refilled as soon as the epilogue of its previous item is
//     done).
//   MMA thread (warp 17): the tile's operand when the tile changes (after
//     every MMA reading the old one), and per item one 128 x 96 x kp MMA
//     pair (query hi, then lo) into the item's accumulator.
//   epilogue (sixteen warps; warp w reads TMEM lanes 32 (w % 4) .. + 31 and
//     tests the balls 8 (w / 4) .. + 7 of the group): per item and ball a
//     ballot of its 32 query lanes; the balls some lane needs are ORed into
//     the item's result word (sb_mask for superblocks, pword for blocks) with
//     a fire-and-forget atomicOr, so the warps never wait for each other.
//   The test skips a ball when X (1 - 3e-6) > (radius + sqrt(seed) (1 +
//     1e-6))^2, X = |q|^2 (1 - 5e-6) + |c|^2 (1 - 5e-6) - 2 q.c - ec: in exact
//     arithmetic it skips less than the filter's own ball test (k_fast_tile),
//     whose margins are wider than this form's rounding, so the blocks kept
//     are a superset of those the filter would not skip.
// A wait that gives up sets the error flag; every later wait then returns
// at once, so all warps still run through every item and barrier and the
// CTA leaves (the results are not used: the status reports the error).
template <bool BLK>
__global__ void __launch_bounds__(kPThreads, 1) k_prune(PruneArgs a)
{
    extern __shared__ __align__(1024) unsigned char psm[];
    unsigned char *base = psm + ((1024u - (smem_u32(psm) & 1023u)) & 1023u);
    const FastShape fs = a.fs;
    const uint32_t arec_pad = (fs.arec_bytes + 1023u) & ~1023u;
    const uint32_t bstage = (uint32_t)fs.nk * kPlane;
    unsigned char *B = base + arec_pad;
    __shared__ PruneCtl ctl;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    constexpr int kEW = kPEpi / 32;   // epilogue warps
    if (t == 0) {
        for (int s = 0; s < kPS; s++) {
            mbar_init(&ctl.bfull[s], 1);
            mbar_init(&ctl.mmad[s], 1);
            mbar_init(&ctl.efree[s], kEW);
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
    volatile int *err = &ctl.err;
    const int total = BLK ? min(*a.n_items, a.items_cap) : a.ntiles * a.ngroups;
    const int per = (total + (int)gridDim.x - 1) / (int)gridDim.x;
    const int i0 = (int)blockIdx.x * per, n = max(0, min(total, i0 + per) - i0);

    if (warp == kEW) {
        // ---------------- copies
        if (lane == 0) {
            int nc = 0;   // items whose group copy is issued
            for (; nc < n; nc++) {
                const int s = nc % kPS;
                if (nc >= kPS && !prune_wait(&ctl.efree[s], (uint32_t)((nc / kPS - 1) & 1), err)) {
                    *err = 1;
                    break;
                }
                int tile, grp;
                uint32_t elig;
                prune_item<BLK>(a, i0 + nc, tile, grp, elig);
                mbar_arrive_expect_tx(&ctl.bfull[s], bstage);
                for (int p = 0; p < fs.nk; p++)
                    bulk_g2s(B + (size_t)s * bstage + (size_t)p * kPlane,
                             a.cop + (size_t)p * a.rows * 128u + (size_t)grp * kPlane, kPlane, &ctl.bfull[s]);
            }
            if (*err)   // the last copies still in flight land before the CTA leaves (bounded)
                for (int j = max(0, nc - kPS); j < nc; j++)
                    mbar_wait(&ctl.bfull[j % kPS], (uint32_t)((j / kPS) & 1), kFWait);
        }
        __syncwarp();
    } else if (warp == kEW + 1) {
        // ---------------- MMAs
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16_f32(kFT, kPN);
            const int ksteps = fs.kp / 16;
            int m_iss = -1;   // last item whose MMA pair is committed
            int a_tile = -1, a_iss = 0;
            bool a_pending = false;
            for (int j = 0; j < n && !*err; j++) {
                int tile, grp;
                uint32_t elig;
                prune_item<BLK>(a, i0 + j, tile, grp, elig);
                if (tile != a_tile) {
                    // every MMA reading the old tile's operand is done (the
                    // commit of the last one covers all before it)
                    if (m_iss >= 0 &&
                        !prune_wait(&ctl.mmad[m_iss % kPS], (uint32_t)((m_iss / kPS) & 1), err)) {
                        *err = 1;
                        break;
                    }
                    mbar_arrive_expect_tx(&ctl.afull, fs.arec_bytes);
                    bulk_g2s(base, a.arec + (size_t)tile * fs.arec_bytes, fs.arec_bytes, &ctl.afull);
                    a_iss++;
                    a_pending = true;
                    if (!prune_wait(&ctl.afull, (uint32_t)((a_iss - 1) & 1), err)) {
                        *err = 1;
                        break;
                    }
                    a_pending = false;
                    a_tile = tile;
                }
                const int s = j % kPS;
                if (!prune_wait(&ctl.bfull[s], (uint32_t)((j / kPS) & 1), err)) {
                    *err = 1;
                    break;
                }
                tc_fence_after();
                const uint64_t dah = smem_desc_sw128(smem_u32(base), 1024);
                const uint64_t dal = smem_desc_sw128(smem_u32(base + fs.atile_bytes), 1024);
                const uint64_t db = smem_desc_sw128(smem_u32(B + (size_t)s * bstage), 1024);
                const uint32_t dt = tmem + (uint32_t)s * kPAccCols;
                for (int kk = 0; kk < ksteps; kk++) {
                    const uint64_t ao = ((uint64_t)(kk >> 2) * (kFT * 128u) + (uint64_t)(kk & 3) * 32u) >> 4;
                    const uint64_t bo = ((uint64_t)(kk >> 2) * kPlane + (uint64_t)(kk & 3) * 32u) >> 4;
                    mma_bf16(dt, dah + ao, db + bo, idesc, kk > 0 ? 1u : 0u);
                }
                for (int kk = 0; kk < ksteps; kk++) {
                    const uint64_t ao = ((uint64_t)(kk >> 2) * (kFT * 128u) + (uint64_t)(kk & 3) * 32u) >> 4;
                    const uint64_t bo = ((uint64_t)(kk >> 2) * kPlane + (uint64_t)(kk & 3) * 32u) >> 4;
                    mma_bf16(dt, dal + ao, db + bo, idesc, 1u);
                }
                mma_commit(&ctl.mmad[s]);
                m_iss = j;
            }
            if (*err) {
                // a tile copy or MMAs still in flight finish before the CTA leaves (bounded)
                if (a_pending) mbar_wait(&ctl.afull, (uint32_t)((a_iss - 1) & 1), kFWait);
                if (m_iss >= 0) mbar_wait(&ctl.mmad[m_iss % kPS], (uint32_t)((m_iss / kPS) & 1), kFWait);
            }
        }
        __syncwarp();
    } else {
        // ---------------- epilogue
        const int quarter = warp & 3, slice = warp >> 2;   // TMEM lanes; balls kPBW * slice ..
        const int tl = 32 * quarter + lane;                // the thread's tile lane
        const float es = eps_scale(fs.kp);
        float4 *bd = ctl.bd[warp];
        int cur_tile = -1;
        float Qp = 0.f, Sp = 0.f, Eq = 0.f;
        uint32_t lane_ok = 0u;   // lanes holding a query with a seed
        for (int j = 0; j < n; j++) {
            const int s = j % kPS;
            int tile, grp;
            uint32_t elig;
            prune_item<BLK>(a, i0 + j, tile, grp, elig);
            if (lane < kPBW) {
                const int bi = kPBW * slice + lane;
                const int ball = grp * kPG + bi;
                const bool okb = ball < a.nball && ((elig >> bi) & 1u);
                const float c2 = okb ? a.c2[ball] : 0.f;
                const float rad = okb ? a.rad[ball] : -1.f;
                bd[lane] = make_float4(sqrtf(c2) * 1.000001f, c2 * (1.f - 5e-6f), rad,
                                       okb && rad >= 0.f ? 1.f : 0.f);
            }
            if (tile != cur_tile) {
                const int4 inf =
                    reinterpret_cast<const int4 *>(a.arec + (size_t)tile * fs.arec_bytes + 2 * fs.atile_bytes)[tl];
                const float q2 = __int_as_float(inf.y), qn = __int_as_float(inf.z);
                const float seed = inf.x >= 0 ? __int_as_float(a.r2_bits[inf.x]) : -1.f;
                lane_ok = __ballot_sync(0xffffffffu, inf.x >= 0 && seed >= 0.f);
                Qp = q2 * (1.f - 5e-6f);
                Sp = sqrtf(fmaxf(seed, 0.f)) * 1.000001f;
                Eq = 2.f * kEpsC * es * qn;
                cur_tile = tile;
            }
            const bool got = __all_sync(0xffffffffu, prune_wait(&ctl.mmad[s], (uint32_t)((j / kPS) & 1), err));
            if (!got && lane == 0) *err = 1;
            tc_fence_after();
            // columns 3 kPBW slice .. + 3 kPBW - 1 of the accumulator: 3 per ball
            const uint32_t taddr =
                tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)s * kPAccCols + (uint32_t)(3 * kPBW * slice);
            uint32_t r0[16], r1[16];
            __syncwarp();
            tmem_ld16_nowait(taddr, r0);
            tmem_ld16_nowait(taddr + 16, r1);
            tmem_wait_ld(r0);
            reg_fence(r1);
            // TMEM reads of this item done: the warp's share of the stage is free
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&ctl.efree[s]);
            uint32_t bits = 0u, mine = 0u;
#pragma unroll
            for (int i = 0; i < kPBW; i++) {
                auto col = [&](int c) -> float { return __uint_as_float(c < 16 ? r0[c] : r1[c - 16]); };
                const float4 b = bd[i];
                // q.c from the three centre columns, |q.c error| <= ec / 2
                const float qc = col(3 * i) + col(3 * i + 1) + col(3 * i + 2);
                const float ec = fmaf(Eq, b.x, 1e-6f);
                const float X = fmaf(-2.f, qc, Qp + b.y) - ec;
                const float rr = b.z + Sp;
                const bool skip = X * 0.999997f > rr * rr;
                const uint32_t m = (got && b.w != 0.f) ? (__ballot_sync(0xffffffffu, !skip) & lane_ok) : 0u;
                if (m) bits |= 1u << (kPBW * slice + i);
                if (lane == i) mine = m;
            }
            if (BLK) {
                if (a.plm && lane < kPBW)
                    a.plm[((size_t)(i0 + j) * kPG + kPBW * slice + lane) * 4 + quarter] = mine;
                if (lane == 0 && bits) atomicOr(&a.pword[i0 + j], bits);
            } else {
                if (lane == 0 && bits) atomicOr(&a.sb_mask[(size_t)tile * a.nsbw + grp], bits);
            }
            __syncwarp();   // bd is rewritten for the next item
        }
    }
    tc_fence_before();
    __syncthreads();
    if (t == 0 && ctl.err) atomicMax(a.status, 16 + 8);
    if (warp == 0) tmem_dealloc(tmem, 512);
}

// Needed-block lists from the block pass: one CTA per tile walks its items
// (group order) and appends the needed blocks of each in ascending order
// (blist[tile][..], bcnt[tile]); with plm also each block's lane masks
// (bmask) and pair counts (bq_cnt); stats[7]: the blocks tested.
__global__ void __launch_bounds__(256) k_prune_list(const int4 *__restrict__ items,
                                                    const uint32_t *__restrict__ pword,
                                                    const uint32_t *__restrict__ plm, const int *__restrict__ tfirst,
                                                    const int *__restrict__ tcnt, int *__restrict__ blist,
                                                    int *__restrict__ bcnt, int nbcap, uint4 *__restrict__ bmask,
                                                    int *__restrict__ bq_cnt, int item, int2 *__restrict__ fitems,
                                                    int *__restrict__ fn_items, int fitems_cap,
                                                    unsigned long long *stats)
{
    __shared__ int wsum[8];
    __shared__ int fbase;
    __shared__ unsigned long long tested_s;
    const int tile = blockIdx.x, t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int f = tfirst[tile], n = tcnt[tile];
    if (t == 0) tested_s = 0;
    int base = 0;
    unsigned long long tested = 0;
    for (int c0 = 0; c0 < n; c0 += 256) {
        const int i = c0 + t;
        const uint32_t w = i < n ? pword[f + i] : 0u;
        const int4 e = i < n ? items[f + i] : make_int4(0, 0, 0, 0);
        if (i < n) tested += __popc((uint32_t)e.z);
        // exclusive scan of the counts over the CTA
        const int cnt = __popc(w);
        int x = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        __syncthreads();   // wsum of the previous chunk consumed
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        int before = 0, total = 0;
#pragma unroll
        for (int v = 0; v < 8; v++) {
            const int sv = wsum[v];
            before += v < warp ? sv : 0;
            total += sv;
        }
        int pos = base + before + x - cnt;
        uint32_t m = w;
        while (m) {
            const int bit = __ffs(m) - 1;
            m &= m - 1;
            const int blk = e.y * kPG + bit;
            if (pos < nbcap) {
                blist[(size_t)tile * nbcap + pos] = blk;
                if (bmask) {
                    const uint32_t *l = plm + ((size_t)(f + i) * kPG + bit) * 4;
                    const uint4 lmk = make_uint4(l[0], l[1], l[2], l[3]);
                    bmask[(size_t)tile * nbcap + pos] = lmk;
                    atomicAdd(&bq_cnt[blk], __popc(lmk.x) + __popc(lmk.y) + __popc(lmk.z) + __popc(lmk.w));
                }
            }
            pos++;
        }
        base += total;
    }
    if (tested) atomicAdd(&tested_s, tested);
    __syncthreads();
    const int cnt = min(base, nbcap);
    // the tile filter's work items (as k_items makes them): the full ones
    // from the front, the partial one from the back
    const int full = fitems ? cnt / item : 0, rem = fitems ? cnt - full * item : 0;
    if (t == 0) {
        bcnt[tile] = cnt;
        if (stats && tested_s) atomicAdd(&stats[7], tested_s);
        if (full > 0) fbase = atomicAdd(&fn_items[0], full);
        if (rem > 0) fitems[fitems_cap - 1 - atomicAdd(&fn_items[1], 1)] = make_int2(tile, full * item);
    }
    __syncthreads();
    for (int i = t; i < full; i += blockDim.x) fitems[fbase + i] = make_int2(tile, i * item);
}

size_t prune_smem(const FastShape &fs)
{
    const size_t need = ((fs.arec_bytes + 1023u) & ~(size_t)1023u) + (size_t)kPS * fs.nk * kPlane + 1024;
    return std::max(need, kPMinSmem);
}

}  // namespace

size_t prune_cop_bytes(const FastShape &fs, int n)
{
    if (fs.kp > kFResKp || n <= 0) return 0;
    const size_t n32 = ((size_t)n + kPG - 1) / kPG * kPG;
    return (size_t)fs.nk * 3 * n32 * 128;
}

int prune_cop_build(const float *cen, int n, const FastShape &fs, unsigned char *cop, cudaStream_t st)
{
    if (!cop || n <= 0) return GTS_OK;
    const int rows = 3 * ((n + kPG - 1) / kPG * kPG);
    k_prune_cop<<<(n + 127) / 128, 128, 0, st>>>(cen, n, fs.kp, rows, cop);
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

size_t prune_items_cap(int ntiles, int nb) { return (size_t)ntiles * (((size_t)nb + kPG - 1) / kPG); }

// Persistent grid: one CTA per SM (each holds all 512 TMEM columns).
static int prune_grid(int total)
{
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, std::min(total, nsm));
}

int prune_superblocks(const unsigned char *arec, const FastShape &fs, const FastSummary &bs, int nsb, int ntiles,
                      const int *r2_bits, uint32_t *sb_mask, int nsbw, bool clear, int *status, cudaStream_t st)
{
    PruneArgs a{};
    a.arec = arec;
    a.cop = bs.scop;
    a.rows = 3 * ((nsb + kPG - 1) / kPG * kPG);
    a.c2 = bs.sb_c2;
    a.rad = bs.sb_rad;
    a.nball = nsb;
    a.fs = fs;
    a.r2_bits = r2_bits;
    a.ntiles = ntiles;
    a.ngroups = (nsb + kPG - 1) / kPG;
    a.sb_mask = sb_mask;
    a.nsbw = nsbw;
    a.status = status;
    // the epilogue warps OR their balls into the mask words
    if (clear) GTS_CUDA_TRY(cudaMemsetAsync(sb_mask, 0, sizeof(uint32_t) * (size_t)ntiles * nsbw, st));
    const size_t smem = prune_smem(fs);
    GTS_CUDA_TRY(cudaFuncSetAttribute(k_prune<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_prune<false><<<prune_grid(ntiles * a.ngroups), kPThreads, smem, st>>>(a);
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

size_t prune_block_bufs(int ntiles, int nb, bool lanes)
{
    const size_t cap = prune_items_cap(ntiles, nb);
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return al(sizeof(int4) * std::max(cap, (size_t)1)) + al(sizeof(uint32_t) * std::max(cap, (size_t)1)) +
           al(2 * sizeof(int) * (size_t)ntiles) + (lanes ? al(sizeof(uint32_t) * 4 * kPG * std::max(cap, (size_t)1)) : 0);
}

int prune_blocks(const unsigned char *arec, const FastShape &fs, const FastSummary &bs, int nb, int ntiles,
                 const int *r2_bits, const uint32_t *sb_mask, int nsbw, unsigned char *bufs, int *n_items, int *blist,
                 int *bcnt, uint4 *bmask, int *bq_cnt, int item, int2 *fitems, int *fn_items, int fitems_cap,
                 unsigned long long *stats, int *status, cudaStream_t st)
{
    const int ngroups = (nb + kPG - 1) / kPG;
    const int items_cap = (int)prune_items_cap(ntiles, nb);
    // the buffers prune_block_bufs counts, carved in its order
    size_t off = 0;
    auto take = [&](size_t b) { unsigned char *p = bufs + off; off += (b + 255) & ~(size_t)255; return p; };
    int4 *items = (int4 *)take(sizeof(int4) * std::max(items_cap, 1));
    uint32_t *pword = (uint32_t *)take(sizeof(uint32_t) * std::max(items_cap, 1));
    int *tfirst = (int *)take(2 * sizeof(int) * (size_t)ntiles);
    int *tcnt = tfirst + ntiles;
    uint32_t *plm = bmask ? (uint32_t *)take(sizeof(uint32_t) * 4 * kPG * (size_t)std::max(items_cap, 1)) : nullptr;
    const size_t gsmem = sizeof(uint32_t) * (size_t)ngroups;
    if (gsmem > 48 * 1024)
        GTS_CUDA_TRY(cudaFuncSetAttribute(k_prune_items, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsmem));
    k_prune_items<<<ntiles, 256, gsmem, st>>>(sb_mask, nsbw, bs.sb_b0, ngroups, items, pword, n_items, items_cap,
                                              tfirst, tcnt);
    GTS_CUDA_TRY(cudaGetLastError());
    PruneArgs a{};
    a.arec = arec;
    a.cop = bs.cop;
    a.rows = 3 * ngroups * kPG;
    a.c2 = bs.c2;
    a.rad = bs.rad;
    a.nball = nb;
    a.fs = fs;
    a.r2_bits = r2_bits;
    a.ntiles = ntiles;
    a.ngroups = ngroups;
    a.items = items;
    a.n_items = n_items;
    a.items_cap = items_cap;
    a.pword = pword;
    a.plm = plm;
    a.status = status;
    const size_t smem = prune_smem(fs);
    GTS_CUDA_TRY(cudaFuncSetAttribute(k_prune<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // the item count is known on the device only: a grid for the worst case
    // leaves CTAs without items at once
    k_prune<true><<<prune_grid(items_cap), kPThreads, smem, st>>>(a);
    GTS_CUDA_TRY(cudaGetLastError());
    k_prune_list<<<ntiles, 256, 0, st>>>(items, pword, plm, tfirst, tcnt, blist, bcnt, nb, bmask, bq_cnt, item,
                                         fitems, fn_items, fitems_cap, stats);
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

}  // namespace gts
