// fast.cuh -- layout shared by the tensor-core kNN filter (fast.cu) and the
// construction of its block order (fast_order.cu).
//
// The filter groups objects into blocks of at most 128 (padded to 128
// slots), and blocks into superblocks.  A slot is block * 128 + lane; slot_of
// maps an object id to its slot, id_of_slot the reverse (-1 for padding).
#pragma once
#include <stdint.h>
#include "index.cuh"

namespace gts {

constexpr int kFB = 128;              // slots per block
constexpr int kFN = 144;              // B rows per block: objects + centre rows + padding
constexpr int kFT = 128;              // queries per tile (A rows, TMEM lanes)
constexpr int kFMaxKp = 320;          // padded dimension limit of this path
constexpr int kFResKp = 128;          // up to this padded dimension a block record sits whole in one
                                      // filter stage; above it the filter streams K in 64-wide chunks
constexpr int kFChunkBytes = kFN * 128;   // one 64-wide K chunk of a block's operand rows
constexpr int kFMaxK = 64;

constexpr int kFCand = 1024;          // candidate slots per query
constexpr long long kFWait = 1ll << 22;   // bounded mbarrier polls (each at most 1 us)

// Error-bound constants.  Relative error of a q.x product out of the MMA:
// the hi/lo split of q (2^-16), FP32 accumulation over 2 x 128 products
// (taken as 2^-23 per add for margin), the FP32 rounding of r (2^-24).
constexpr float kEpsC = 5e-5f;        // q.c rows:  >= 2^-16 + 2 * 256 * 2^-24
constexpr float kEpsR = 8e-5f;        // q.r rows:  >= 2^-16 + 2 * 256 * 2^-23 + 2^-23

// The accumulation part grows with the products summed (2 kp of them), so
// above kp = 128 both constants scale by kp / 128: at kp = 320,
// 1.25e-4 >= 2^-16 + 2 * 640 * 2^-24 and 2e-4 >= 2^-16 + 2 * 640 * 2^-23 + 2^-23.
__host__ __device__ __forceinline__ float eps_scale(int kp) { return kp <= 128 ? 1.f : (float)kp / 128.f; }

// Record tail, after the BF16 operand rows (floats): w[128], dn[128], then
// |c|, the valid-object count (int), max |bf16(r)|, max |w|, the radius
// max |o - c| (rounded up).
constexpr int kTailW = 0, kTailDn = 128, kTailC = 256, kTailCnt = 257, kTailRb = 258, kTailWb = 259,
              kTailRad = 260;

// A candidate-list count at or above this marks a query the filter could not
// list in full (the recheck then sends it to the re-answer stages).
constexpr int kFListDropped = 1 << 30;

// Block order (hierarchical k-means, fast_order.cu):
constexpr int kOrdBranch = 16;        // k-means children per split at most
constexpr int kOrdHalve = 1024;       // segments up to this size are halved instead
constexpr int kOrdIters = 6;          // Lloyd iterations per level
constexpr int kOrdSbMax = 4096;       // a superblock: the first segment of at most this many objects
constexpr int kOrdMaxLevels = 64;

struct FastShape {
    int kp, nk;              // padded dim, number of 64-wide K chunks
    uint32_t btile_bytes;    // nk * kFN * 128
    uint32_t rec_bytes;      // btile_bytes + 1024 (w, dn) + 32 (block scalars)
    uint32_t atile_bytes;    // nk * kFT * 128
    uint32_t arec_bytes;     // query tile: hi + lo operands + 128 x int4 lane info
};

__host__ __device__ inline FastShape fast_shape(int dim)
{
    FastShape s;
    s.kp = (dim + 63) / 64 * 64;
    s.nk = s.kp / 64;
    s.btile_bytes = (uint32_t)s.nk * kFN * 128u;
    s.rec_bytes = s.btile_bytes + 1024u + 32u;
    s.atile_bytes = (uint32_t)s.nk * kFT * 128u;
    s.arec_bytes = 2u * s.atile_bytes + 16u * kFT;
    return s;
}

// Seeds per slot (fast.cu, k_fast_selfk): k = 2^j for j < kSelfKN
// (k = 1 .. 64) and one padding entry, 32 bytes per slot; made from the
// object's own block and the kSeedNbr blocks with the nearest centres,
// keeping the kSeedBest smallest distances per object.
constexpr int kSelfKN = 7;
constexpr int kSelfK = 8;
constexpr int kSeedNbr = 31;
constexpr int kSeedBest = 64;

// Per-block and per-superblock summaries, placed after the block records.
struct FastSummary {
    float *cen, *c2, *rad;          // [nb][kp] centre, [nb] |c|^2, [nb] max |o - c|
    int *ids;                       // [nb * kFB] slot -> object id (-1: padding)
    int *pos;                       // [num] object id -> slot
    float *sb_cen, *sb_c2, *sb_rad; // [nsb][kp], [nsb], [nsb]
    int *sb_b0;                     // [nsb + 1] first block of each superblock
    float *prow;                    // [nb * kFB][kp] FP32 rows in slot order (zero padding)
    int *selfk;                     // [nb * kFB][kSelfK] seeds (float bits), k = 1, 2, 4 .. 64
    int *nbr;                       // [nb][kSeedNbr] blocks with the nearest centres (-1: none)
    unsigned char *cop, *scop;      // centre operands of the blocks / superblocks for the tensor-core
                                    // pruning (fast_prune.cu; null above kFResKp)
};

// Tensor-core ball pruning (fast_prune.cu), padded dimension <= kFResKp:
// bytes of a centre operand of n balls (0 above kFResKp), and its build
// from FP32 centres ([n][kp]).
size_t prune_cop_bytes(const FastShape &fs, int n);
int prune_cop_build(const float *cen, int n, const FastShape &fs, unsigned char *cop, cudaStream_t st);
size_t prune_items_cap(int ntiles, int nb);

inline size_t fast_rec_region(const FastShape &fs, int nb)
{
    return ((size_t)nb * fs.rec_bytes + 255) & ~(size_t)255;
}

// Byte offsets of the summary arrays after the records, each 256-byte
// aligned (the pruning kernels read centres as float4).
struct FastSummaryOffsets {
    size_t cen, c2, rad, ids, pos, sb_cen, sb_c2, sb_rad, sb_b0, prow, selfk, nbr, cop, scop, end;
};

inline FastSummaryOffsets fast_summary_offsets(const FastShape &fs, int nb, int nsb, int n)
{
    FastSummaryOffsets o;
    size_t off = fast_rec_region(fs, nb);
    auto take = [&](size_t bytes) { size_t at = off; off += (bytes + 255) & ~(size_t)255; return at; };
    o.cen = take(sizeof(float) * (size_t)nb * fs.kp);
    o.c2 = take(sizeof(float) * (size_t)nb);
    o.rad = take(sizeof(float) * (size_t)nb);
    o.ids = take(sizeof(int) * (size_t)nb * kFB);
    o.pos = take(sizeof(int) * (size_t)n);
    o.sb_cen = take(sizeof(float) * (size_t)nsb * fs.kp);
    o.sb_c2 = take(sizeof(float) * (size_t)nsb);
    o.sb_rad = take(sizeof(float) * (size_t)nsb);
    o.sb_b0 = take(sizeof(int) * ((size_t)nsb + 1));
    o.prow = take(sizeof(float) * (size_t)nb * kFB * fs.kp);
    o.selfk = take(sizeof(int) * (size_t)nb * kFB * kSelfK);
    o.nbr = take(sizeof(int) * (size_t)nb * kSeedNbr);
    o.cop = take(prune_cop_bytes(fs, nb));
    o.scop = take(prune_cop_bytes(fs, nsb));
    o.end = off;
    return o;
}

inline size_t fast_bytes(const FastShape &fs, int nb, int nsb, int n)
{
    return fast_summary_offsets(fs, nb, nsb, n).end;
}

inline FastSummary fast_summary(unsigned char *recs, const FastShape &fs, int nb, int nsb, int n)
{
    const FastSummaryOffsets o = fast_summary_offsets(fs, nb, nsb, n);
    FastSummary s;
    s.cen = (float *)(recs + o.cen);
    s.c2 = (float *)(recs + o.c2);
    s.rad = (float *)(recs + o.rad);
    s.ids = (int *)(recs + o.ids);
    s.pos = (int *)(recs + o.pos);
    s.sb_cen = (float *)(recs + o.sb_cen);
    s.sb_c2 = (float *)(recs + o.sb_c2);
    s.sb_rad = (float *)(recs + o.sb_rad);
    s.sb_b0 = (int *)(recs + o.sb_b0);
    s.prow = (float *)(recs + o.prow);
    s.selfk = (int *)(recs + o.selfk);
    s.nbr = (int *)(recs + o.nbr);
    s.cop = prune_cop_bytes(fs, nb) ? recs + o.cop : nullptr;
    s.scop = prune_cop_bytes(fs, nsb) ? recs + o.scop : nullptr;
    return s;
}

// The tiles' needed superblocks (mask words sb_mask[tile][nsbw]; cleared
// first when `clear`) and then their needed blocks (blist[tile][..] in
// ascending order, counts in bcnt; with bmask, each block's lanes and pairs
// per block in bq_cnt), on the tensor cores (fast_prune.cu).  n_items: a
// zeroed counter of the block pass's items.  The block pass carves its items and result words from `bufs`,
// prune_block_bufs(ntiles, nb, bmask != nullptr) bytes.  With fitems the
// block lists also become the tile filter's work items of `item` blocks
// (full ones from the front at fn_items[0], each tile's partial one from
// the back of fitems_cap at fn_items[1]; both counters zeroed).
int prune_superblocks(const unsigned char *arec, const FastShape &fs, const FastSummary &bs, int nsb, int ntiles,
                      const int *r2_bits, uint32_t *sb_mask, int nsbw, bool clear, int *status, cudaStream_t st);
size_t prune_block_bufs(int ntiles, int nb, bool lanes);
int prune_blocks(const unsigned char *arec, const FastShape &fs, const FastSummary &bs, int nb, int ntiles,
                 const int *r2_bits, const uint32_t *sb_mask, int nsbw, unsigned char *bufs, int *n_items, int *blist,
                 int *bcnt, uint4 *bmask, int *bq_cnt, int item, int2 *fitems, int *fn_items, int fitems_cap,
                 unsigned long long *stats, int *status, cudaStream_t st);

// Result of the order construction, in the index's scratch: positions of
// the final order (perm: position -> object id), the blocks as position
// ranges, and the superblock starts (sb_start[pos] = 1 where a superblock
// begins).  Valid until the scratch is reused.
struct FastOrder {
    int nb = 0, nsb = 0;
    const int *perm = nullptr;
    const int *blk_l = nullptr, *blk_r = nullptr;   // [nb]
    const int *blk_sb = nullptr;                    // [nb] superblock of each block
    const int *sb_b0 = nullptr;                     // [nsb + 1]
};

// Build the filter's block order for the index's rows (L2).  Uses the
// index's growable scratch; one host read-back per level.
int fast_block_order(gts_index *idx, FastOrder *out, cudaStream_t st);

}  // namespace gts
