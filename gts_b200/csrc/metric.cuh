// metric.cuh -- device distance library for the GTS path.
//
// The reference inlines ~14 copies of the same five metrics (metric codes
// 0 = L-inf, 1 = L1, 2 = L2, 5 = angle in degrees, 6 = edit distance) with a
// different accumulator type at different call sites:
//   F64 accumulator: build key    (tree.cuh:80-155)
//                    kNN pivot    (search_v2.cuh:664-745)
//                    kNN leaf     (search_v2.cuh:447-535)
//   F32 accumulator: child min_dis (tree.cuh:205-280)
//                    range node   (search_v2.cuh:63-129)
//                    range leaf   (search_v2.cuh:337-408)
//                    update leaf  (update.cuh:246-323)
//                    cache scan   (search_naive.cuh:31-68)
// The exact routines below evaluate the same expressions with the same types
// (same overloads of pow / abs / acos), so their results are bit-identical
// to the reference's.  The fast routines (warp-split FP32) are filters only:
// every value they produce is paired with a rounding bound and anything that
// can matter is recomputed exactly.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gts {

enum Metric { kLinf = 0, kL1 = 1, kL2 = 2, kAngle = 5, kEdit = 6 };
enum Acc { kAccF32 = 0, kAccF64 = 1 };

constexpr int kStrStride = 109;   // reference string row stride (file.cuh:15)

// ---------------------------------------------------------------------------
// exact, reference operation order (one thread, sequential over the row)
// ---------------------------------------------------------------------------

// Sequential F64-accumulated distance.  `pow(float_diff, 2)` in the
// reference resolves to a double-returning overload that is not always the
// exact square (measured on the device: ~6% of inputs differ in the last
// bit), and `pow(x, 0.5)` is not always `sqrt(x)`; both are called here
// literally so every value matches the reference bit for bit.
__device__ __forceinline__ double dist_row_f64(const float *__restrict__ a,
                                               const float *__restrict__ b,
                                               int dim, int metric)
{
    double r = 0.0;
    if (metric == kL2) {
        for (int j = 0; j < dim; j++) r += pow(a[j] - b[j], 2);
        return pow(r, 0.5);
    } else if (metric == kL1) {
        for (int j = 0; j < dim; j++) r += abs(a[j] - b[j]);
        return r;
    } else if (metric == kLinf) {
        for (int j = 0; j < dim; j++) {
            float t = abs(a[j] - b[j]);
            if (t > r) r = t;
        }
        return r;
    } else {   // angle
        float sa1 = 0.f, sa2 = 0.f, sa3 = 0.f;
        for (int j = 0; j < dim; j++) {
            sa1 = fmaf(a[j], a[j], sa1);
            sa2 = fmaf(b[j], b[j], sa2);
            sa3 = fmaf(a[j], b[j], sa3);
        }
        sa1 = pow(sa1, 0.5);
        sa2 = pow(sa2, 0.5);
        r = sa3 / (sa1 * sa2);
        if (r > 1) r = 0.99999999999999999;
        return abs(acos(r) * 180 / 3.1415926);
    }
}

// Sequential F32-accumulated distance (`float result += pow(..)` adds in
// double and rounds to float at every step), same literal calls.
__device__ __forceinline__ float dist_row_f32(const float *__restrict__ a,
                                              const float *__restrict__ b,
                                              int dim, int metric)
{
    float r = 0.f;
    if (metric == kL2) {
        for (int j = 0; j < dim; j++) r += pow(a[j] - b[j], 2);
        r = pow(r, 0.5);
        return r;
    } else if (metric == kL1) {
        for (int j = 0; j < dim; j++) r += abs(a[j] - b[j]);
        return r;
    } else if (metric == kLinf) {
        for (int j = 0; j < dim; j++) {
            float t = abs(a[j] - b[j]);
            if (t > r) r = t;
        }
        return r;
    } else {   // angle
        float sa1 = 0.f, sa2 = 0.f, sa3 = 0.f;
        for (int j = 0; j < dim; j++) {
            sa1 = fmaf(a[j], a[j], sa1);
            sa2 = fmaf(b[j], b[j], sa2);
            sa3 = fmaf(a[j], b[j], sa3);
        }
        sa1 = pow(sa1, 0.5);
        sa2 = pow(sa2, 0.5);
        r = sa3 / (sa1 * sa2);
        if (r > 1) r = 0.99999999999999999;
        r = abs(acos(r) * 180 / 3.1415926);
        return r;
    }
}

// Levenshtein distance.  Pattern (length m <= 64) as a bit-parallel column
// (Myers 1999, in Hyyro's formulation for global distance); peq[c] holds
// the positions of byte c in the pattern.  Exact, so equal to the
// reference's O(n*m) table (tree.cuh:128-153).
__device__ __forceinline__ int edit_myers64(const uint64_t *__restrict__ peq, int m,
                                            const char *__restrict__ t, int n)
{
    n = min(max(n, 0), kStrStride);
    if (m == 0) return n;
    if (n == 0) return m;
    uint64_t pv = (m == 64) ? ~0ull : ((1ull << m) - 1), mv = 0;
    const uint64_t hi = 1ull << (m - 1);
    int score = m;
    for (int j = 0; j < n; j++) {
        uint64_t eq = peq[(unsigned char)t[j]];
        uint64_t xv = eq | mv;
        uint64_t xh = (((eq & pv) + pv) ^ pv) | eq;
        uint64_t ph = mv | ~(xh | pv);
        uint64_t mh = pv & xh;
        if (ph & hi) score++;
        else if (mh & hi) score--;
        ph = (ph << 1) | 1ull;
        mh <<= 1;
        pv = mh | ~(xv | ph);
        mv = ph & xv;
    }
    return score;
}

// Plain dynamic programme (any lengths up to the row stride).
__device__ __forceinline__ int edit_dp(const char *__restrict__ a, int n,
                                       const char *__restrict__ b, int m)
{
    n = min(max(n, 0), kStrStride);
    m = min(max(m, 0), kStrStride);
    if (n == 0) return m;
    if (m == 0) return n;
    int row[kStrStride + 1];
    for (int k = 0; k <= m; k++) row[k] = k;
    for (int j = 1; j <= n; j++) {
        int diag = row[0];
        row[0] = j;
        char ca = a[j - 1];
        for (int k = 1; k <= m; k++) {
            int up = row[k];
            int v = 1 + min(up, row[k - 1]);
            v = min(diag + (ca == b[k - 1] ? 0 : 1), v);
            diag = up;
            row[k] = v;
        }
    }
    return row[m];
}

// ---------------------------------------------------------------------------
// fast filters (warp-cooperative, coalesced): FP32 with a rounding bound
// ---------------------------------------------------------------------------

// Character-class signature of a string: for each of 32 classes (a byte's
// low five bits; a..z are classes 1..26) the count of its characters,
// saturated at 15, four bits each.  One edit changes the counts' L1 distance
// by at most 2 (a substitution moves one count, an insertion or deletion
// changes one) and saturation only lowers it, so ceil(L1 / 2) of two
// signatures, like the length difference, is a lower bound on the edit
// distance of the strings.
__device__ __forceinline__ uint4 str_sig(const char *__restrict__ s, int n)
{
    n = min(max(n, 0), kStrStride);
    unsigned char cnt[32];
#pragma unroll
    for (int c = 0; c < 32; c++) cnt[c] = 0;
    for (int i = 0; i < n; i++) {
        const int c = (unsigned char)s[i] & 31;
        if (cnt[c] < 15) cnt[c]++;
    }
    uint32_t w[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        uint32_t v = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) v |= (uint32_t)cnt[8 * k + j] << (4 * j);
        w[k] = v;
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

// max(|la - lb|, ceil(L1(sig_a, sig_b) / 2)) <= edit distance.
__device__ __forceinline__ int edit_lower_bound(uint4 a, int la, uint4 b, int lb)
{
    const uint32_t x[4] = {a.x, a.y, a.z, a.w}, y[4] = {b.x, b.y, b.z, b.w};
    unsigned l1 = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        l1 += __vsadu4(x[k] & 0x0F0F0F0Fu, y[k] & 0x0F0F0F0Fu);
        l1 += __vsadu4((x[k] >> 4) & 0x0F0F0F0Fu, (y[k] >> 4) & 0x0F0F0F0Fu);
    }
    return max(abs(la - lb), (int)((l1 + 1) >> 1));
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_max(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Relative bound on |fp32 sum of n non-negative terms - exact sum| / sum,
// terms themselves rounded once: (n + 2) u / (1 - (n + 2) u), u = 2^-24.
__host__ __device__ __forceinline__ float f32_sum_rel_bound(int n)
{
    float nu = (float)(n + 2) * 5.9604645e-8f;
    return nu / (1.f - nu);
}

}  // namespace gts
