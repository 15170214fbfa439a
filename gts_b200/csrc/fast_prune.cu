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
// The epilogue sums the three columns of a ball and applies the filter's own
// certified ball test (the skip test of k_fast_tile), so the blocks kept are
// a superset of those the filter would not skip.  Up to a padded dimension
// of 128 (kFResKp); wider indexes use the FP32 pruning kernels in fast.cu.
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
constexpr int kPThreads = 128;          // four warps: TMEM lane quarters

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
// CTA per tile; items (tile, group, mask) appended at n_items.
__global__ void k_prune_items(const uint32_t *__restrict__ sb_mask, int nsbw, const int *__restrict__ sb_b0,
                              int ngroups, int4 *__restrict__ items, int *__restrict__ n_items, int items_cap)
{
    extern __shared__ uint32_t gm[];   // [ngroups]
    const int tile = blockIdx.x, t = threadIdx.x;
    for (int g = t; g < ngroups; g += blockDim.x) gm[g] = 0u;
    __syncthreads();
    int seen = 0;
    for (int w = 0; w < nsbw; w++) {
        uint32_t word = sb_mask[(size_t)tile * nsbw + w];
        while (word) {
            const int s = w * 32 + __ffs(word) - 1;
            word &= word - 1;
            if (seen++ % (int)blockDim.x != t) continue;
            const int b1 = sb_b0[s + 1];
            for (int b = sb_b0[s]; b < b1; b++) atomicOr(&gm[b >> 5], 1u << (b & 31));
        }
    }
    __syncthreads();
    for (int g = t; g < ngroups; g += blockDim.x) {
        const uint32_t m = gm[g];
        if (!m) continue;
        const int p = atomicAdd(n_items, 1);
        if (p < items_cap) items[p] = make_int4(tile, g, (int)m, 0);
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
    // block pass: items from k_prune_items; needed blocks appended to blist
    const int4 *items;
    const int *n_items;
    int items_cap;
    int *blist, *bcnt;
    int nbcap;
    uint4 *bmask;                // nullable: per needed block, the tile's lanes that reach it
    int *bq_cnt;                 // with bmask: pairs per block
    unsigned long long *stats;
    int *status;
};

// Persistent CTAs, each over a contiguous range of (tile, group) items (so
// consecutive items mostly share the tile and its operand stays in shared
// memory).  Thread 0 issues the copies and the MMA pair; the four warps read
// their TMEM lane quarter (32 queries x 96 columns) and ballot the ball
// tests; warp 0 turns the per-ball lane masks into the group's result.
template <bool BLK>
__global__ void __launch_bounds__(kPThreads) k_prune(PruneArgs a)
{
    extern __shared__ __align__(1024) unsigned char psm[];
    unsigned char *base = psm + ((1024u - (smem_u32(psm) & 1023u)) & 1023u);
    const FastShape fs = a.fs;
    const uint32_t arec_pad = (fs.arec_bytes + 1023u) & ~1023u;
    unsigned char *B = base + arec_pad;
    __shared__ __align__(8) uint64_t afull, bfull, mmad;
    __shared__ uint32_t tmem_s;
    __shared__ float pc2[kPG], pcn[kPG], prad[kPG];
    __shared__ uint32_t lm[kPG][4];
    __shared__ int err_s;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    if (t == 0) {
        mbar_init(&afull, 1);
        mbar_init(&bfull, 1);
        mbar_init(&mmad, 1);
        err_s = 0;
        fence_mbar_init();
    }
    if (warp == 0) {
        tmem_alloc(&tmem_s, 128);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_s;
    const uint32_t idesc = idesc_bf16_f32(kFT, kPN);
    const int total = BLK ? min(*a.n_items, a.items_cap) : a.ntiles * a.ngroups;
    const int per = (total + (int)gridDim.x - 1) / (int)gridDim.x;
    const int i0 = (int)blockIdx.x * per, i1 = min(total, i0 + per);
    int cur_tile = -1;
    uint32_t na = 0, nbp = 0, nm = 0;   // completed phases of afull, bfull, mmad
    const float es = eps_scale(fs.kp);
    for (int it = i0; it < i1; it++) {
        int tile, grp;
        uint32_t elig = 0xffffffffu;
        if (BLK) {
            const int4 e = a.items[it];
            tile = e.x;
            grp = e.y;
            elig = (uint32_t)e.z;
        } else {
            tile = it / a.ngroups;
            grp = it - tile * a.ngroups;
        }
        if (t < kPG) {
            const int ball = grp * kPG + t;
            const bool ok = ball < a.nball && ((elig >> t) & 1u);
            const float c2 = ok ? a.c2[ball] : 0.f;
            pc2[t] = c2;
            pcn[t] = sqrtf(c2) * 1.000001f;
            prad[t] = ok ? a.rad[ball] : -1.f;
        }
        __syncthreads();   // the previous item's TMEM reads and results are done; ball data visible
        if (t == 0) {
            const bool new_tile = tile != cur_tile;
            if (new_tile) {
                mbar_arrive_expect_tx(&afull, fs.arec_bytes);
                bulk_g2s(base, a.arec + (size_t)tile * fs.arec_bytes, fs.arec_bytes, &afull);
            }
            mbar_arrive_expect_tx(&bfull, (uint32_t)fs.nk * kPlane);
            for (int p = 0; p < fs.nk; p++)
                bulk_g2s(B + (size_t)p * kPlane, a.cop + (size_t)p * a.rows * 128u + (size_t)grp * kPlane, kPlane,
                         &bfull);
            bool ok = true;
            if (new_tile) ok = mbar_wait(&afull, na++ & 1u, kFWait);
            ok = mbar_wait(&bfull, nbp++ & 1u, kFWait) && ok;
            if (ok) {
                tc_fence_after();
                const uint64_t dah = smem_desc_sw128(smem_u32(base), 1024);
                const uint64_t dal = smem_desc_sw128(smem_u32(base + fs.atile_bytes), 1024);
                const uint64_t db = smem_desc_sw128(smem_u32(B), 1024);
                const int ksteps = fs.kp / 16;
                for (int kk = 0; kk < ksteps; kk++) {
                    const uint64_t ao = ((uint64_t)(kk >> 2) * (kFT * 128u) + (uint64_t)(kk & 3) * 32u) >> 4;
                    const uint64_t bo = ((uint64_t)(kk >> 2) * kPlane + (uint64_t)(kk & 3) * 32u) >> 4;
                    mma_bf16(tmem, dah + ao, db + bo, idesc, kk > 0 ? 1u : 0u);
                }
                for (int kk = 0; kk < ksteps; kk++) {
                    const uint64_t ao = ((uint64_t)(kk >> 2) * (kFT * 128u) + (uint64_t)(kk & 3) * 32u) >> 4;
                    const uint64_t bo = ((uint64_t)(kk >> 2) * kPlane + (uint64_t)(kk & 3) * 32u) >> 4;
                    mma_bf16(tmem, dal + ao, db + bo, idesc, 1u);
                }
                mma_commit(&mmad);
            } else {
                err_s = 1;
                mbar_arrive(&mmad);   // nothing to wait for: let the epilogue through
            }
        }
        cur_tile = tile;
        // ---- epilogue: warp w reads TMEM lanes 32w .. 32w + 31 (tile lanes)
        const bool got = __all_sync(0xffffffffu, mbar_wait(&mmad, nm & 1u, kFWait));
        nm++;
        if (!got && lane == 0) err_s = 1;
        tc_fence_after();
        const int4 inf = reinterpret_cast<const int4 *>(base + 2 * fs.atile_bytes)[32 * warp + lane];
        const int qi = inf.x;
        const float q2 = __int_as_float(inf.y), qn = __int_as_float(inf.z);
        const float seed = qi >= 0 ? __int_as_float(a.r2_bits[qi]) : -1.f;
        const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll
        for (int h = 0; h < 2; h++) {   // 16 balls (48 columns) at a time
            uint32_t r0[16], r1[16], r2[16];
            __syncwarp();
            tmem_ld16_nowait(trow + (uint32_t)(48 * h), r0);
            tmem_ld16_nowait(trow + (uint32_t)(48 * h + 16), r1);
            tmem_ld16_nowait(trow + (uint32_t)(48 * h + 32), r2);
            tmem_wait_ld(r0);
            reg_fence(r1);
            reg_fence(r2);
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const int g = 16 * h + i;
                auto col = [&](int c) -> float {
                    return __uint_as_float(c < 16 ? r0[c] : (c < 32 ? r1[c - 16] : r2[c - 32]));
                };
                // the filter's ball test (k_fast_tile): q.c from the three
                // centre columns, |q.c error| <= ec / 2
                const float qc = col(3 * i) + col(3 * i + 1) + col(3 * i + 2);
                const float cn = pcn[g], c2 = pc2[g], brad = prad[g];
                const float ec = 2.f * kEpsC * es * qn * cn + 1e-6f;
                const float qmc2 = q2 - 2.f * qc + c2;
                const float dlo = sqrtf(fmaxf(qmc2 - ec - 4e-6f * (q2 + c2), 0.f)) * 0.999999f - brad;
                const bool need = got && seed >= 0.f && brad >= 0.f && !(dlo > 0.f && dlo * dlo * 0.999999f > seed);
                const uint32_t m = __ballot_sync(0xffffffffu, need);
                if (lane == 0) lm[g][warp] = m;
            }
        }
        tc_fence_before();
        __syncthreads();   // masks complete; TMEM free for the next item's MMA
        tc_fence_after();
        if (warp == 0) {
            const uint4 lmk = make_uint4(lm[lane][0], lm[lane][1], lm[lane][2], lm[lane][3]);
            const bool any = (lmk.x | lmk.y | lmk.z | lmk.w) != 0u;
            const uint32_t word = __ballot_sync(0xffffffffu, any);
            if (!BLK) {
                if (lane == 0) a.sb_mask[(size_t)tile * a.nsbw + grp] = word;
            } else {
                if (lane == 0 && a.stats) atomicAdd(&a.stats[7], (unsigned long long)__popc(elig));
                int at = 0;
                if (lane == 0 && word) at = atomicAdd(&a.bcnt[tile], __popc(word));
                at = __shfl_sync(0xffffffffu, at, 0);
                if (any) {
                    const int pos = at + __popc(word & ((1u << lane) - 1u));
                    const int blk = grp * kPG + lane;
                    if (pos < a.nbcap) {
                        a.blist[(size_t)tile * a.nbcap + pos] = blk;
                        if (a.bmask) {
                            a.bmask[(size_t)tile * a.nbcap + pos] = lmk;
                            atomicAdd(&a.bq_cnt[blk], __popc(lmk.x) + __popc(lmk.y) + __popc(lmk.z) + __popc(lmk.w));
                        }
                    }
                }
            }
        }
        if (err_s) break;   // uniform: written by thread 0 before the barrier above
    }
    if (t == 0 && err_s) {
        // copies still in flight land before the CTA leaves (bounded)
        mbar_wait(&afull, (na - 1u) & 1u, kFWait);
        mbar_wait(&bfull, (nbp - 1u) & 1u, kFWait);
        atomicMax(a.status, 16 + 8);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 128);
}

size_t prune_smem(const FastShape &fs)
{
    return ((fs.arec_bytes + 1023u) & ~(size_t)1023u) + (size_t)fs.nk * kPlane + 1024;
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

static int prune_grid(int total)
{
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, std::min(total, 2 * nsm));
}

int prune_superblocks(const unsigned char *arec, const FastShape &fs, const FastSummary &bs, int nsb, int ntiles,
                      const int *r2_bits, uint32_t *sb_mask, int nsbw, int *status, cudaStream_t st)
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
    const size_t smem = prune_smem(fs);
    GTS_CUDA_TRY(cudaFuncSetAttribute(k_prune<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_prune<false><<<prune_grid(ntiles * a.ngroups), kPThreads, smem, st>>>(a);
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

int prune_blocks(const unsigned char *arec, const FastShape &fs, const FastSummary &bs, int nb, int nsb, int ntiles,
                 const int *r2_bits, const uint32_t *sb_mask, int nsbw, int4 *items, int *n_items, int *blist,
                 int *bcnt, uint4 *bmask, int *bq_cnt, unsigned long long *stats, int *status, cudaStream_t st)
{
    const int ngroups = (nb + kPG - 1) / kPG;
    const int items_cap = (int)prune_items_cap(ntiles, nb);
    const size_t gsmem = sizeof(uint32_t) * (size_t)ngroups;
    if (gsmem > 48 * 1024)
        GTS_CUDA_TRY(cudaFuncSetAttribute(k_prune_items, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsmem));
    GTS_CUDA_TRY(cudaMemsetAsync(n_items, 0, sizeof(int), st));
    k_prune_items<<<ntiles, 256, gsmem, st>>>(sb_mask, nsbw, bs.sb_b0, ngroups, items, n_items, items_cap);
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
    a.blist = blist;
    a.bcnt = bcnt;
    a.nbcap = nb;
    a.bmask = bmask;
    a.bq_cnt = bq_cnt;
    a.stats = stats;
    a.status = status;
    const size_t smem = prune_smem(fs);
    GTS_CUDA_TRY(cudaFuncSetAttribute(k_prune<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // the item count is known on the device only: a grid for the worst case
    // leaves CTAs without items at once
    k_prune<true><<<prune_grid(items_cap), kPThreads, smem, st>>>(a);
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

}  // namespace gts
