// fast_blk.cuh -- interface of the block-stationary filter (fast_blk.cu):
// every needed block read once per run and multiplied with the queries
// that need it.
#pragma once
#include <stddef.h>
#include "fast.cuh"

namespace gts {

constexpr int kBQ = 32;          // queries (MMA columns) per item at most
constexpr int kBHead = 1024;     // item header: kBQ columns of bound terms
constexpr int kBPairs = 64;      // (query, block) pairs per query a run stores, on average at most

struct FastBlkArgs {
    const unsigned char *recs;   // block records
    const unsigned char *irec;   // item headers (k_bq_build), kBHead bytes each
    const int4 *items;           // (block, first pair, queries, item index)
    const int *n_items;
    const int *bq;               // query slots of the pairs
    const unsigned char *arec;   // tile records: the queries' operand rows
    FastShape fs;
    int k;                       // kNN: neighbours per query (the running bound); range: unused
    int nst;                     // record stages
    int *cand_pos;               // [qnum][kFCand]
    float *cand_lb, *cand_ub;
    int *cand_cnt;
    int *r2_bits;                // per query: the bound its columns were built with
    int *status;
    unsigned long long *stats;
    float r2lo;                  // range: objects with ub below it are counted in rcnt
    int *rcnt;
};

// One run's inputs and scratch: the tile pruning's per-tile block lists
// with their query masks, and the pair and item buffers.
struct FastBlkRun {
    FastBlkArgs args;            // recs, irec, candidate lists, bounds, status, stats, r2lo, rcnt
    const float *cen;            // [nb][kp] block centres
    const unsigned char *arec;   // tile records (operand rows, lane info)
    const int *blist;            // [ntiles][nbcap] needed blocks of each tile
    const uint4 *bmask;          // [ntiles][nbcap] lanes of the tile that need the block
    const int *bcnt;             // [ntiles]
    const int *order;            // tile slot -> query index
    int *bq_cnt, *bq_off, *bq_fill;   // [nb] (bq_cnt counted by the pruning, bq_fill zeroed)
    int *bq;                     // [pairs_cap] query slots
    unsigned char *irec;         // [fast_blk_irec_bytes] item headers (the filter reads args.irec = irec)
    int4 *items;                 // [fast_blk_items_cap]
    int *n_items;
    int nb, nbcap, ntiles, qnum, pairs_cap, nsm;
    bool range;
    cudaEvent_t timed_begin, timed_end;   // recorded around the filter kernel when set
    bool capturing;                      // the events are recorded inside a graph capture
};

// Shared memory of the filter with nst stages; the most stages that fit
// (0: the form does not apply, kp above kFResKp).
size_t fast_blk_smem(const FastShape &fs, int nst);
int fast_blk_stages(const FastShape &fs);
// Items and item-header bytes a run with pairs_cap pairs may need.
size_t fast_blk_items_cap(int nb, int pairs_cap);
size_t fast_blk_irec_bytes(int nb, int pairs_cap);
// Items, pairs, item records and the filter, enqueued on st.
int fast_blk_enqueue(const FastBlkRun &r, cudaStream_t st, long long *launches);

}  // namespace gts
