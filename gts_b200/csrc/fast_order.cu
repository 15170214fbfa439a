// fast_order.cu -- the block order of the tensor-core kNN filter.
//
// The filter streams objects in blocks of up to 128 and skips a block for a
// tile of queries when the triangle inequality puts it out of every query's
// reach (|q - c| - radius > bound).  That only works when blocks are tight
// balls that never straddle two groups of the data.  A pivot-tree position
// order or a projection ball tree cut at fixed 128-object boundaries mixes
// groups in most blocks; here the order comes from a hierarchical k-means,
// built level by level on the device:
//
//   * a segment of more than kOrdHalve objects is split by Lloyd's k-means
//     into up to kOrdBranch children (about kOrdHalve objects each), so
//     well-separated groups never share a child;
//   * a segment of 129..kOrdHalve objects (or one k-means could not split)
//     is halved at a balanced point of its projection on the axis of a
//     2-means, so blocks come out nearly full;
//   * a segment of at most 128 objects is a block (padded to 128 slots).
//
// Every split is stable, so a segment keeps its position range for the rest
// of the build and the order nests: the first segment of at most kOrdSbMax
// objects on every path is a superblock, a contiguous run of blocks whose
// ball lets the filter drop all of them with one test.
//
// Per level: plan (k-means or halving), centroid seeds at evenly spread
// positions of the segment, kOrdIters Lloyd passes (one warp per object,
// per-CTA shared-memory sums when a CTA's objects share a segment), a final
// pass that writes the sort key (segment, child) or (segment, projection),
// a stable radix sort, and the child segments.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cfloat>
#include <utility>
#include "fast.cuh"

namespace gts {

namespace {

constexpr int kOAsgPos = 256;   // positions per assignment CTA (8 warps)

__device__ __forceinline__ uint32_t order_bits(float f)
{
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void k_o_init(int n, int *perm, int *sid)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        perm[i] = i;
        sid[i] = 0;
    }
}

// kind: 0 leaf (<= 128 objects), 1 k-means split, 2 halving; kk: children.
__global__ void k_o_plan(int nseg, const int *__restrict__ sl, const int *__restrict__ sr,
                         const uint8_t *__restrict__ force, int *__restrict__ kind, int *__restrict__ kk,
                         int *__restrict__ active)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const int size = sr[s] - sl[s];
    int kd = 0, K = 0;
    if (size > kFB) {
        if (force[s] || size <= kOrdHalve) {
            kd = 2;
            K = 2;
        } else {
            kd = 1;
            K = min(kOrdBranch, (size + kOrdHalve - 1) / kOrdHalve);
        }
        atomicAdd(active, 1);
    }
    kind[s] = kd;
    kk[s] = K;
}

__global__ void k_o_total(int nseg, const int *__restrict__ cbase, const int *__restrict__ kk, int *__restrict__ out)
{
    out[0] = cbase[nseg - 1] + kk[nseg - 1];
}

// One CTA per segment: seed its K centroids with the rows at positions
// l + (2j + 1) size / (2K).
__global__ void k_o_seed(int nseg, int dim, const float *__restrict__ rows, const int *__restrict__ perm,
                         const int *__restrict__ sl, const int *__restrict__ sr, const int *__restrict__ kk,
                         const int *__restrict__ cbase, float *__restrict__ cent)
{
    const int s = blockIdx.x;
    const int K = kk[s];
    if (K == 0) return;
    const int l = sl[s], size = sr[s] - l;
    for (int j = 0; j < K; j++) {
        const int p = l + (int)(((long long)(2 * j + 1) * size) / (2 * K));
        const float *x = rows + (size_t)perm[p] * dim;
        for (int d = threadIdx.x; d < dim; d += blockDim.x) cent[(size_t)(cbase[s] + j) * dim + d] = x[d];
    }
}

// One warp per position.  Pass 0 (Lloyd): nearest centroid of the segment,
// its sum and count.  Pass 1 (final): the sort key (segment << 32 | child)
// for k-means segments, (segment << 32 | projection on c1 - c0) for halving
// segments, (segment << 32) for leaves; counts of the k-means children.
template <int NX>
__global__ void __launch_bounds__(256) k_o_assign(int n, int dim, const float *__restrict__ rows,
                                                  const int *__restrict__ perm, const int *__restrict__ sid,
                                                  const int *__restrict__ kind, const int *__restrict__ kk,
                                                  const int *__restrict__ cbase, const float *__restrict__ cent,
                                                  float *__restrict__ csum, int *__restrict__ ccnt, int final_pass,
                                                  unsigned long long *__restrict__ keys)
{
    __shared__ float ssum[kOrdBranch * NX * 32];
    __shared__ int scnt[kOrdBranch];
    const int p0 = blockIdx.x * kOAsgPos, p1 = min(n, p0 + kOAsgPos);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s0 = sid[p0];
    const bool uni = !final_pass && sid[p1 - 1] == s0 && kind[s0] != 0;
    const int K0 = uni ? kk[s0] : 0;
    if (uni) {
        for (int i = threadIdx.x; i < K0 * dim; i += blockDim.x) ssum[i] = 0.f;
        if (threadIdx.x < K0) scnt[threadIdx.x] = 0;
    }
    __syncthreads();
    for (int pos = p0 + warp; pos < p1; pos += 8) {
        const int s = sid[pos], kd = kind[s];
        if (kd == 0) {
            if (final_pass && lane == 0) keys[pos] = (unsigned long long)s << 32;
            continue;
        }
        const float *xr = rows + (size_t)perm[pos] * dim;
        float x[NX];
#pragma unroll
        for (int i = 0; i < NX; i++) {
            const int d = lane + 32 * i;
            x[i] = d < dim ? xr[d] : 0.f;
        }
        const int K = kk[s], cb = cbase[s];
        float best = FLT_MAX;
        int bj = 0;
        for (int j = 0; j < K; j++) {
            const float *c = cent + (size_t)(cb + j) * dim;
            float acc = 0.f;
#pragma unroll
            for (int i = 0; i < NX; i++) {
                const int d = lane + 32 * i;
                if (d < dim) {
                    const float e = x[i] - c[d];
                    acc = fmaf(e, e, acc);
                }
            }
            acc = warp_sum(acc);
            if (acc < best) {
                best = acc;
                bj = j;
            }
        }
        if (!final_pass) {
            if (uni) {
#pragma unroll
                for (int i = 0; i < NX; i++) {
                    const int d = lane + 32 * i;
                    if (d < dim) atomicAdd(&ssum[bj * dim + d], x[i]);
                }
                if (lane == 0) atomicAdd(&scnt[bj], 1);
            } else {
#pragma unroll
                for (int i = 0; i < NX; i++) {
                    const int d = lane + 32 * i;
                    if (d < dim) atomicAdd(&csum[(size_t)(cb + bj) * dim + d], x[i]);
                }
                if (lane == 0) atomicAdd(&ccnt[cb + bj], 1);
            }
        } else {
            uint32_t lo;
            if (kd == 1) {
                lo = (uint32_t)bj;
                if (lane == 0) atomicAdd(&ccnt[cb + bj], 1);
            } else {
                const float *c0 = cent + (size_t)cb * dim, *c1 = c0 + dim;
                float p = 0.f;
#pragma unroll
                for (int i = 0; i < NX; i++) {
                    const int d = lane + 32 * i;
                    if (d < dim) p = fmaf(x[i], c1[d] - c0[d], p);
                }
                lo = order_bits(warp_sum(p));
            }
            if (lane == 0) keys[pos] = ((unsigned long long)s << 32) | lo;
        }
    }
    __syncthreads();
    if (uni) {
        const int cb = cbase[s0];
        for (int i = threadIdx.x; i < K0 * dim; i += blockDim.x)
            if (scnt[i / dim]) atomicAdd(&csum[(size_t)cb * dim + i], ssum[i]);
        if (threadIdx.x < K0 && scnt[threadIdx.x]) atomicAdd(&ccnt[cb + threadIdx.x], scnt[threadIdx.x]);
    }
}

__global__ void k_o_update(int C, int dim, const float *__restrict__ csum, const int *__restrict__ ccnt,
                           float *__restrict__ cent)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)C * dim) return;
    const int c = (int)(i / dim);
    if (ccnt[c] > 0) cent[i] = csum[i] / (float)ccnt[c];
}

__global__ void k_o_nchild(int nseg, const int *__restrict__ kind, const int *__restrict__ kk,
                           const int *__restrict__ cbase, const int *__restrict__ ccnt, int *__restrict__ nchild)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    int c = 1;
    if (kind[s] == 2) c = 2;
    else if (kind[s] == 1) {
        c = 0;
        for (int j = 0; j < kk[s]; j++) c += ccnt[cbase[s] + j] > 0;
    }
    nchild[s] = c;
}

// Child segments of every segment, at newbase[s]; superblock starts where a
// segment of more than kOrdSbMax objects has a child of at most kOrdSbMax.
__global__ void k_o_children(int nseg, const int *__restrict__ sl, const int *__restrict__ sr,
                             const int *__restrict__ kind, const int *__restrict__ kk, const int *__restrict__ cbase,
                             const int *__restrict__ ccnt, const int *__restrict__ newbase, int *__restrict__ nsl,
                             int *__restrict__ nsr, uint8_t *__restrict__ nforce, uint8_t *__restrict__ sb_start)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const int l = sl[s], r = sr[s], size = r - l, b = newbase[s];
    const bool big = size > kOrdSbMax;
    if (kind[s] == 0) {
        nsl[b] = l;
        nsr[b] = r;
        nforce[b] = 0;
    } else if (kind[s] == 1) {
        const int cb = cbase[s], K = kk[s];
        int nz = 0;
        for (int j = 0; j < K; j++) nz += ccnt[cb + j] > 0;
        int run = l, c = 0;
        for (int j = 0; j < K; j++) {
            const int cnt = ccnt[cb + j];
            if (cnt == 0) continue;
            nsl[b + c] = run;
            nsr[b + c] = run + cnt;
            nforce[b + c] = nz == 1;   // k-means could not split it: halve next
            if (big && cnt <= kOrdSbMax) sb_start[run] = 1;
            run += cnt;
            c++;
        }
    } else {
        const int nbk = (size + kFB - 1) / kFB;
        const int m = l + (int)(((long long)size * ((nbk + 1) / 2)) / nbk);
        nsl[b] = l;
        nsr[b] = m;
        nsl[b + 1] = m;
        nsr[b + 1] = r;
        nforce[b] = nforce[b + 1] = 0;
        if (big && m - l <= kOrdSbMax) sb_start[l] = 1;
        if (big && r - m <= kOrdSbMax) sb_start[m] = 1;
    }
}

__global__ void k_o_relabel(int n, int *__restrict__ sid, const int *__restrict__ newbase,
                            const int *__restrict__ nchild, const int *__restrict__ nsl)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const int s = sid[pos], b = newbase[s], c = nchild[s];
    int j = 0;
    while (j + 1 < c && nsl[b + j + 1] <= pos) j++;
    sid[pos] = b + j;
}

// Superblock of every block: flags f[b] = sb_start[blk_l[b]].
__global__ void k_o_sbflag(int nb, const int *__restrict__ bl, const uint8_t *__restrict__ sb_start,
                           int *__restrict__ f)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb) f[b] = sb_start[bl[b]] ? 1 : 0;
}

__global__ void k_o_sbtable(int nb, const int *__restrict__ f, const int *__restrict__ incl, int *__restrict__ blk_sb,
                            int *__restrict__ sb_b0, int *__restrict__ nsb_out)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    blk_sb[b] = incl[b] - 1;
    if (f[b]) sb_b0[incl[b] - 1] = b;
    if (b == nb - 1) {
        sb_b0[incl[b]] = nb;
        *nsb_out = incl[b];
    }
}

}  // namespace

int fast_block_order(gts_index *idx, FastOrder *out, cudaStream_t st)
{
    const int n = idx->num, dim = idx->dim;
    if (n < 1 || dim > kFMaxKp) {
        gts_set_error("block order: %d objects of dimension %d (at most %d)", n, dim, kFMaxKp);
        return GTS_ERR_INVALID;
    }
    const int S = n + 1;                        // segments (each holds at least one object)
    const int Ccap = n / 32 + 4 * kOrdBranch;   // centroids: <= 16 per k-means segment (> kOrdHalve objects)
                                                // plus 2 per halving segment (> 128 objects)
    size_t cub_bytes = 0, tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, (unsigned long long *)nullptr, (unsigned long long *)nullptr,
                                    (int *)nullptr, (int *)nullptr, n, 0, 64, st);
    cub_bytes = tb;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, (int *)nullptr, (int *)nullptr, S, st);
    cub_bytes = std::max(cub_bytes, tb);
    cub::DeviceScan::InclusiveSum(nullptr, tb, (int *)nullptr, (int *)nullptr, S, st);
    cub_bytes = std::max(cub_bytes, tb);

    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~(size_t)255; return o; };
    const size_t o_perm = take(4 * (size_t)n), o_perm2 = take(4 * (size_t)n), o_sid = take(4 * (size_t)n);
    const size_t o_keys = take(8 * (size_t)n), o_keys2 = take(8 * (size_t)n);
    size_t o_seg[11];
    for (int i = 0; i < 11; i++) o_seg[i] = take(4 * (size_t)S);
    const size_t o_force = take(S), o_nforce = take(S), o_sbs = take((size_t)n);
    const size_t o_cent = take(4 * (size_t)Ccap * dim), o_csum = take(4 * (size_t)Ccap * dim);
    const size_t o_ccnt = take(4 * (size_t)Ccap), o_misc = take(64), o_cub = take(cub_bytes);
    int rc;
    if ((rc = ensure_scratch(idx, off))) return rc;
    unsigned char *B = (unsigned char *)idx->scratch;
    int *perm = (int *)(B + o_perm), *perm2 = (int *)(B + o_perm2), *sid = (int *)(B + o_sid);
    unsigned long long *keys = (unsigned long long *)(B + o_keys), *keys2 = (unsigned long long *)(B + o_keys2);
    int *sl = (int *)(B + o_seg[0]), *sr = (int *)(B + o_seg[1]), *nsl = (int *)(B + o_seg[2]);
    int *nsr = (int *)(B + o_seg[3]), *kind = (int *)(B + o_seg[4]), *kk = (int *)(B + o_seg[5]);
    int *cbase = (int *)(B + o_seg[6]), *nchild = (int *)(B + o_seg[7]), *newbase = (int *)(B + o_seg[8]);
    int *flag = (int *)(B + o_seg[9]), *incl = (int *)(B + o_seg[10]);
    uint8_t *force = B + o_force, *nforce = B + o_nforce, *sb_start = B + o_sbs;
    float *cent = (float *)(B + o_cent), *csum = (float *)(B + o_csum);
    int *ccnt = (int *)(B + o_ccnt), *misc = (int *)(B + o_misc);
    void *cub_tmp = B + o_cub;

    k_o_init<<<(n + 255) / 256, 256, 0, st>>>(n, perm, sid);
    const int h_seg[2] = {0, n};
    GTS_CUDA_TRY(cudaMemcpyAsync(sl, &h_seg[0], sizeof(int), cudaMemcpyHostToDevice, st));
    GTS_CUDA_TRY(cudaMemcpyAsync(sr, &h_seg[1], sizeof(int), cudaMemcpyHostToDevice, st));
    GTS_CUDA_TRY(cudaMemsetAsync(force, 0, 1, st));
    GTS_CUDA_TRY(cudaMemsetAsync(sb_start, 0, (size_t)n, st));
    if (n <= kOrdSbMax) GTS_CUDA_TRY(cudaMemsetAsync(sb_start, 1, 1, st));
    int nseg = 1, level = 0;
    const int agrid = (n + kOAsgPos - 1) / kOAsgPos;
    for (; level < kOrdMaxLevels; level++) {
        GTS_CUDA_TRY(cudaMemsetAsync(misc, 0, 2 * sizeof(int), st));
        k_o_plan<<<(nseg + 255) / 256, 256, 0, st>>>(nseg, sl, sr, force, kind, kk, misc);
        size_t tb2 = cub_bytes;
        GTS_CUDA_TRY(cub::DeviceScan::ExclusiveSum(cub_tmp, tb2, kk, cbase, nseg, st));
        k_o_total<<<1, 1, 0, st>>>(nseg, cbase, kk, misc + 1);
        int h[2];
        GTS_CUDA_TRY(cudaMemcpyAsync(h, misc, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
        GTS_CUDA_TRY(cudaStreamSynchronize(st));
        const int active = h[0], C = h[1];
        if (active == 0) break;
        if (C > Ccap) {
            gts_set_error("block order: %d centroids exceed the capacity %d", C, Ccap);
            return GTS_ERR_KERNEL;
        }
        k_o_seed<<<nseg, 128, 0, st>>>(nseg, dim, idx->rows, perm, sl, sr, kk, cbase, cent);
        const int ugrid = (int)(((size_t)C * dim + 255) / 256);
        for (int it = 0; it < kOrdIters; it++) {
            GTS_CUDA_TRY(cudaMemsetAsync(csum, 0, sizeof(float) * (size_t)C * dim, st));
            GTS_CUDA_TRY(cudaMemsetAsync(ccnt, 0, sizeof(int) * (size_t)C, st));
            if (dim <= kFResKp)
                k_o_assign<kFResKp / 32><<<agrid, 256, 0, st>>>(n, dim, idx->rows, perm, sid, kind, kk, cbase, cent,
                                                               csum, ccnt, 0, keys);
            else
                k_o_assign<kFMaxKp / 32><<<agrid, 256, 0, st>>>(n, dim, idx->rows, perm, sid, kind, kk, cbase, cent,
                                                               csum, ccnt, 0, keys);
            k_o_update<<<ugrid, 256, 0, st>>>(C, dim, csum, ccnt, cent);
        }
        GTS_CUDA_TRY(cudaMemsetAsync(ccnt, 0, sizeof(int) * (size_t)C, st));
        if (dim <= kFResKp)
            k_o_assign<kFResKp / 32><<<agrid, 256, 0, st>>>(n, dim, idx->rows, perm, sid, kind, kk, cbase, cent, csum,
                                                           ccnt, 1, keys);
        else
            k_o_assign<kFMaxKp / 32><<<agrid, 256, 0, st>>>(n, dim, idx->rows, perm, sid, kind, kk, cbase, cent, csum,
                                                           ccnt, 1, keys);
        int sbits = 1;
        while ((1 << sbits) < nseg) sbits++;
        size_t tb3 = cub_bytes;
        GTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(cub_tmp, tb3, keys, keys2, perm, perm2, n, 0, 32 + sbits, st));
        std::swap(perm, perm2);
        k_o_nchild<<<(nseg + 255) / 256, 256, 0, st>>>(nseg, kind, kk, cbase, ccnt, nchild);
        size_t tb4 = cub_bytes;
        GTS_CUDA_TRY(cub::DeviceScan::ExclusiveSum(cub_tmp, tb4, nchild, newbase, nseg, st));
        k_o_total<<<1, 1, 0, st>>>(nseg, newbase, nchild, misc);
        k_o_children<<<(nseg + 255) / 256, 256, 0, st>>>(nseg, sl, sr, kind, kk, cbase, ccnt, newbase, nsl, nsr,
                                                         nforce, sb_start);
        k_o_relabel<<<(n + 255) / 256, 256, 0, st>>>(n, sid, newbase, nchild, nsl);
        GTS_CUDA_TRY(cudaGetLastError());
        int total = 0;
        GTS_CUDA_TRY(cudaMemcpyAsync(&total, misc, sizeof(int), cudaMemcpyDeviceToHost, st));
        GTS_CUDA_TRY(cudaStreamSynchronize(st));
        if (total < nseg || total > S) {
            gts_set_error("block order: level %d produced %d segments from %d", level, total, nseg);
            return GTS_ERR_KERNEL;
        }
        nseg = total;
        std::swap(sl, nsl);
        std::swap(sr, nsr);
        std::swap(force, nforce);
    }
    if (level == kOrdMaxLevels) {
        gts_set_error("block order: no convergence after %d levels", kOrdMaxLevels);
        return GTS_ERR_KERNEL;
    }
    // blocks = the final segments; superblocks from the recorded starts
    const int nb = nseg;
    int *blk_sb = nchild, *sb_b0 = newbase;   // reuse (segment-sized arrays)
    k_o_sbflag<<<(nb + 255) / 256, 256, 0, st>>>(nb, sl, sb_start, flag);
    size_t tb5 = cub_bytes;
    GTS_CUDA_TRY(cub::DeviceScan::InclusiveSum(cub_tmp, tb5, flag, incl, nb, st));
    k_o_sbtable<<<(nb + 255) / 256, 256, 0, st>>>(nb, flag, incl, blk_sb, sb_b0, misc);
    GTS_CUDA_TRY(cudaGetLastError());
    int nsb = 0;
    GTS_CUDA_TRY(cudaMemcpyAsync(&nsb, misc, sizeof(int), cudaMemcpyDeviceToHost, st));
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    if (nsb < 1 || nsb > nb) {
        gts_set_error("block order: %d superblocks for %d blocks", nsb, nb);
        return GTS_ERR_KERNEL;
    }
    out->nb = nb;
    out->nsb = nsb;
    out->perm = perm;
    out->blk_l = sl;
    out->blk_r = sr;
    out->blk_sb = blk_sb;
    out->sb_b0 = sb_b0;
    return GTS_OK;
}

}  // namespace gts
