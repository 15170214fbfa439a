// common.cuh -- device-side layout of a GTS index on one B200.
//
// HBM layout (all arrays device-resident, built once, read by every search):
//   rows      float[num * dim]     objects in id order (the caller's layout)
//   trows     float[num * dim]     the same rows permuted into tree order, so a
//                                  leaf's objects are one contiguous span
//   strs/tstrs char[num * 109]     strings (metric 6), id order / tree order
//   lens/tlens int[num]
//   tsig      uint4[num]           metric 6: the strings' character-class
//                                  signatures in tree order (edit lower bounds)
//   id_list   int[num]             tree position -> object id (tree.cuh:344)
//   pos_of_id int[num]             object id -> tree position
//   node_*    SoA over max_node_num nodes in the reference's implicit O-ary
//             numbering (child = nid*O + i + 1, parent = (nid-1)/O):
//             pid (parent's pivot), min_dis (ring lower bound), size, lid,
//             flags (bit0 exists, bit1 is_leaf), pivot (pivot chosen when the
//             node was split, -1 otherwise)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "metric.cuh"

namespace gts {

enum NodeFlag : uint8_t { kExists = 1, kLeaf = 2 };

struct DevData {
    int dim, num, metric;
    const float *rows;
    const char *strs;
    const int *lens;
};

struct DevTree {
    int num, dim, metric;
    int order, max_size, max_h, tree_h, max_node_num;
    int dis_code, infi_dis;
    const float *rows, *trows;
    const char *strs, *tstrs;
    const int *lens, *tlens;
    const uint4 *tsig;   // metric 6: character-class signature per tree position (metric.cuh)
    const int *id_list, *pos_of_id;
    const int *node_pid, *node_size, *node_lid, *node_pivot;
    const float *node_min_dis;
    const uint8_t *node_flags;
};

// Status codes written by kernels (never a trap: a kernel that cannot finish
// records why and returns).
enum KernelStatus : int {
    kKsOk = 0,
    kKsStackOverflow = 1,
    kKsBadNode = 2,
    kKsBadQuery = 3,
};

}  // namespace gts

#define GTS_CUDA_TRY(expr)                                                    \
    do {                                                                      \
        cudaError_t e__ = (expr);                                             \
        if (e__ != cudaSuccess) {                                             \
            gts_set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr,         \
                          cudaGetErrorString(e__));                           \
            return GTS_ERR_CUDA;                                              \
        }                                                                     \
    } while (0)

extern "C" void gts_set_error(const char *fmt, ...);
