// mlp.cu -- learned kNN radius: a small MLP trained on the device.
//
// Features of a query (33): its FP32 distances to the pivots of the first 32
// internal nodes of the tree (root, level 1, the start of level 2 -- the
// "top-level pivots"), and log(k).  Output: the standardised log of the k-th
// neighbour distance.  Network 33 -> 128 -> 128 -> 1 with ReLU, FP32.
// Training data are exact radii produced by the index's own exact search.
// Kernels are plain SIMT code: the network is tiny (21k parameters) and the
// batches small, so the tensor cores have nothing to gain here.
//
// Parameter layout (flat, kMlpParams floats):
//   W1[128][33] b1[128] W2[128][128] b2[128] W3[128] b3[1]
#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <vector>
#include "index.cuh"

namespace gts {

constexpr int kMIn = 33, kMH = 128;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kMH * kMIn, kOffW2 = kOffB1 + kMH;
constexpr int kOffB2 = kOffW2 + kMH * kMH, kOffW3 = kOffB2 + kMH, kOffB3 = kOffW3 + kMH;
constexpr int kMlpParams = kOffB3 + 1;
constexpr int kMFeatPivots = 32;

// ---------------------------------------------------------------- features

// X[q][f] = FP32 distance from query q to feature pivot f; X[q][32] = log k.
__global__ void k_mlp_features(const float *__restrict__ rows, int dim, const int *__restrict__ qids,
                               int qnum, const int *__restrict__ piv, int npiv, const int *__restrict__ ks,
                               int kconst, float *__restrict__ X)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= qnum * kMIn) return;
    int q = t / kMIn, f = t % kMIn;
    float v = 0.f;
    if (f < kMFeatPivots) {
        if (f < npiv) {
            const float *a = rows + (size_t)qids[q] * dim, *b = rows + (size_t)piv[f] * dim;
            float s = 0.f;
            for (int j = 0; j < dim; j++) {
                float d = a[j] - b[j];
                s = fmaf(d, d, s);
            }
            v = sqrtf(s);
        }
    } else {
        v = logf((float)(ks ? ks[q] : kconst));
    }
    X[t] = v;
}

// ---------------------------------------------------------------- forward

// One CTA (128 threads = hidden units) per sample.  xs / ys standardise the
// inputs; H1, H2 (post-ReLU) are kept for the backward pass when non-null.
__global__ void __launch_bounds__(kMH) k_mlp_fwd(const float *__restrict__ X, const int *__restrict__ rowsel,
                                                 int B, const float *__restrict__ P, const float *__restrict__ xmu,
                                                 const float *__restrict__ xsig, float *__restrict__ H1,
                                                 float *__restrict__ H2, float *__restrict__ Y)
{
    __shared__ float x[kMIn], h1[kMH], red[kMH];
    const int b = blockIdx.x, j = threadIdx.x;
    if (b >= B) return;
    const int r = rowsel ? rowsel[b] : b;
    if (j < kMIn) x[j] = (X[(size_t)r * kMIn + j] - xmu[j]) / xsig[j];
    __syncthreads();
    float s = P[kOffB1 + j];
    for (int i = 0; i < kMIn; i++) s = fmaf(P[kOffW1 + j * kMIn + i], x[i], s);
    s = fmaxf(s, 0.f);
    h1[j] = s;
    if (H1) H1[(size_t)b * kMH + j] = s;
    __syncthreads();
    float s2 = P[kOffB2 + j];
    for (int i = 0; i < kMH; i++) s2 = fmaf(P[kOffW2 + j * kMH + i], h1[i], s2);
    s2 = fmaxf(s2, 0.f);
    if (H2) H2[(size_t)b * kMH + j] = s2;
    red[j] = s2 * P[kOffW3 + j];
    __syncthreads();
    for (int w = kMH / 2; w > 0; w >>= 1) {
        if (j < w) red[j] += red[j + w];
        __syncthreads();
    }
    if (j == 0) Y[b] = red[0] + P[kOffB3];
}

// ---------------------------------------------------------------- backward

// Per sample: dY = 2 (y - t) / B (mean squared error), then dH2, dH1
// (pre-activation gradients through the ReLUs).
__global__ void __launch_bounds__(kMH) k_mlp_bwd_act(const int *__restrict__ rowsel, int B,
                                                     const float *__restrict__ T, const float *__restrict__ P,
                                                     const float *__restrict__ H1, const float *__restrict__ H2,
                                                     const float *__restrict__ Y, float *__restrict__ dY,
                                                     float *__restrict__ dZ2, float *__restrict__ dZ1,
                                                     float *__restrict__ loss)
{
    __shared__ float dz2[kMH];
    const int b = blockIdx.x, j = threadIdx.x;
    if (b >= B) return;
    const int r = rowsel ? rowsel[b] : b;
    const float e = Y[b] - T[r];
    const float dy = 2.f * e / (float)B;
    if (j == 0) {
        dY[b] = dy;
        atomicAdd(loss, e * e / (float)B);
    }
    float g2 = H2[(size_t)b * kMH + j] > 0.f ? dy * P[kOffW3 + j] : 0.f;
    dz2[j] = g2;
    dZ2[(size_t)b * kMH + j] = g2;
    __syncthreads();
    float g1 = 0.f;
    if (H1[(size_t)b * kMH + j] > 0.f)
        for (int i = 0; i < kMH; i++) g1 = fmaf(dz2[i], P[kOffW2 + i * kMH + j], g1);
    dZ1[(size_t)b * kMH + j] = g1;
}

// Parameter gradients: one thread per parameter, summing over the batch
// (deterministic; no atomics).
__global__ void k_mlp_bwd_params(const float *__restrict__ X, const int *__restrict__ rowsel, int B,
                                 const float *__restrict__ xmu, const float *__restrict__ xsig,
                                 const float *__restrict__ H1, const float *__restrict__ H2,
                                 const float *__restrict__ dY, const float *__restrict__ dZ2,
                                 const float *__restrict__ dZ1, float *__restrict__ G)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams) return;
    float s = 0.f;
    if (p < kOffB1) {                       // W1[j][i]
        int j = p / kMIn, i = p % kMIn;
        for (int b = 0; b < B; b++) {
            int r = rowsel ? rowsel[b] : b;
            float x = (X[(size_t)r * kMIn + i] - xmu[i]) / xsig[i];
            s = fmaf(dZ1[(size_t)b * kMH + j], x, s);
        }
    } else if (p < kOffW2) {                // b1[j]
        int j = p - kOffB1;
        for (int b = 0; b < B; b++) s += dZ1[(size_t)b * kMH + j];
    } else if (p < kOffB2) {                // W2[j][i]
        int q = p - kOffW2, j = q / kMH, i = q % kMH;
        for (int b = 0; b < B; b++) s = fmaf(dZ2[(size_t)b * kMH + j], H1[(size_t)b * kMH + i], s);
    } else if (p < kOffW3) {                // b2[j]
        int j = p - kOffB2;
        for (int b = 0; b < B; b++) s += dZ2[(size_t)b * kMH + j];
    } else if (p < kOffB3) {                // W3[j]
        int j = p - kOffW3;
        for (int b = 0; b < B; b++) s = fmaf(dY[b], H2[(size_t)b * kMH + j], s);
    } else {                                // b3
        for (int b = 0; b < B; b++) s += dY[b];
    }
    G[p] = s;
}

// Adam (Kingma & Ba 2015) with bias correction.
__global__ void k_mlp_adam(float *__restrict__ P, const float *__restrict__ G, float *__restrict__ M,
                           float *__restrict__ V, float lr, float b1, float b2, float eps, float c1, float c2)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams) return;
    float g = G[p];
    float m = b1 * M[p] + (1.f - b1) * g;
    float v = b2 * V[p] + (1.f - b2) * g * g;
    M[p] = m;
    V[p] = v;
    P[p] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

// Inference for the filter's seed, kInferQ queries per CTA (128 threads =
// hidden units): features (the same FP32 expressions as k_mlp_features),
// both hidden layers (the same operation order as k_mlp_fwd) and the
// squared, widened radius.  W2 is read from L1/L2 once per CTA and reused
// by all its queries.
constexpr int kInferQ = 32;

__global__ void __launch_bounds__(kMH) k_mlp_infer(const float *__restrict__ rows, int dim,
                                                   const int *__restrict__ qids, int qnum,
                                                   const int *__restrict__ piv, int npiv, int k,
                                                   const float *__restrict__ P, const float *__restrict__ xmu,
                                                   const float *__restrict__ xsig, float ymu, float ysig,
                                                   float widen, int *__restrict__ r2_bits)
{
    __shared__ float xs[kInferQ][kMIn + 1];
    __shared__ float h1[kInferQ][kMH + 1];
    __shared__ float red[kInferQ][4];
    const int q0 = blockIdx.x * kInferQ, j = threadIdx.x, lane = j & 31, warp = j >> 5;
    const int nq = min(kInferQ, qnum - q0);
    // features: thread j -> query j / 4, pivots (j % 4) + 4 i
    {
        const int ql = j >> 2;
        if (ql < nq) {
            const float *a = rows + (size_t)qids[q0 + ql] * dim;
            for (int f = j & 3; f < kMFeatPivots; f += 4) {
                float v = 0.f;
                if (f < npiv) {
                    const float *b = rows + (size_t)piv[f] * dim;
                    float s = 0.f;
                    for (int d = 0; d < dim; d++) {
                        float e = a[d] - b[d];
                        s = fmaf(e, e, s);
                    }
                    v = sqrtf(s);
                }
                xs[ql][f] = (v - xmu[f]) / xsig[f];
            }
            if ((j & 3) == 0) xs[ql][kMFeatPivots] = (logf((float)k) - xmu[kMFeatPivots]) / xsig[kMFeatPivots];
        }
    }
    __syncthreads();
    // hidden layer 1: unit j for every query
    for (int q = 0; q < nq; q++) {
        float s = P[kOffB1 + j];
        for (int i = 0; i < kMIn; i++) s = fmaf(P[kOffW1 + j * kMIn + i], xs[q][i], s);
        h1[q][j] = fmaxf(s, 0.f);
    }
    __syncthreads();
    // hidden layer 2 and the output contribution of unit j
    float acc[kInferQ];
#pragma unroll
    for (int q = 0; q < kInferQ; q++) acc[q] = P[kOffB2 + j];
    for (int i = 0; i < kMH; i++) {
        const float w = P[kOffW2 + j * kMH + i];
#pragma unroll
        for (int q = 0; q < kInferQ; q++) acc[q] = fmaf(w, h1[q][i], acc[q]);
    }
    const float w3 = P[kOffW3 + j];
#pragma unroll
    for (int q = 0; q < kInferQ; q++) {
        float c = fmaxf(acc[q], 0.f) * w3;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) red[q][warp] = c;
    }
    __syncthreads();
    if (j < nq) {
        const float y = red[j][0] + red[j][1] + red[j][2] + red[j][3] + P[kOffB3];
        float r2 = 0.f;
        if (k > 1) {   // k = 1: the query object itself, at distance 0
            const float r = expf(y * ysig + ymu) * widen;
            r2 = r * r;
            if (!(r2 < 3.0e38f)) r2 = 3.0e38f;
        }
        r2_bits[q0 + j] = __float_as_int(r2);
    }
}

// ---------------------------------------------------------------- host

struct MlpBufs {
    DevVec v;
    float *X = nullptr, *H1 = nullptr, *H2 = nullptr, *Y = nullptr, *dY = nullptr, *dZ1 = nullptr,
          *dZ2 = nullptr, *G = nullptr, *loss = nullptr;
    int alloc(int n_rows, int batch)
    {
        int rc;
        if ((rc = v.alloc(&X, (size_t)n_rows * kMIn)) || (rc = v.alloc(&H1, (size_t)batch * kMH)) ||
            (rc = v.alloc(&H2, (size_t)batch * kMH)) || (rc = v.alloc(&Y, (size_t)std::max(batch, n_rows))) ||
            (rc = v.alloc(&dY, (size_t)batch)) || (rc = v.alloc(&dZ1, (size_t)batch * kMH)) ||
            (rc = v.alloc(&dZ2, (size_t)batch * kMH)) || (rc = v.alloc(&G, (size_t)kMlpParams + 1)))
            return rc;
        loss = G + kMlpParams;
        return GTS_OK;
    }
};

static int mlp_alloc_model(gts_index *idx)
{
    if (idx->mlp_P) return GTS_OK;
    int rc;
    if ((rc = dev_alloc(&idx->mlp_P, (size_t)kMlpParams, nullptr))) return rc;
    if ((rc = dev_alloc(&idx->mlp_norm, (size_t)2 * kMIn, nullptr))) return rc;
    if ((rc = dev_alloc(&idx->mlp_piv, (size_t)kMFeatPivots, nullptr))) return rc;
    return GTS_OK;
}

// Feature pivots: pivots of the first internal nodes in node order.
static int mlp_pick_pivots(gts_index *idx, cudaStream_t st)
{
    int n = std::min(idx->max_node_num, 4096);
    std::vector<int> piv(n);
    GTS_CUDA_TRY(cudaMemcpyAsync(piv.data(), idx->node_pivot, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<int> sel;
    for (int i = 0; i < n && (int)sel.size() < kMFeatPivots; i++)
        if (piv[i] >= 0) sel.push_back(piv[i]);
    idx->mlp_npiv = (int)sel.size();
    if (!sel.empty())
        GTS_CUDA_TRY(cudaMemcpyAsync(idx->mlp_piv, sel.data(), sizeof(int) * sel.size(), cudaMemcpyHostToDevice, st));
    return GTS_OK;
}

int mlp_features(gts_index *idx, const int *d_qids, int qnum, const int *d_ks, int k, float *d_X, cudaStream_t st)
{
    int n = qnum * kMIn;
    k_mlp_features<<<(n + 255) / 256, 256, 0, st>>>(idx->rows, idx->dim, d_qids, qnum, idx->mlp_piv,
                                                      idx->mlp_npiv, d_ks, k, d_X);
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

// Predicted squared radius bounds (as int bits) for the fast filter's seed:
// features, the forward pass and the seed in one kernel, no scratch.
// The widening for k: that of the smallest trained k >= k with enough
// held-out samples, else the global one.
static float widen_for(const gts_index *idx, int k)
{
    for (int kv = std::max(k, 0); kv <= 64; kv++)
        if (idx->mlp_widen_at[kv] > 0.f) return idx->mlp_widen_at[kv];
    return idx->mlp_widen;
}

int mlp_seed(gts_index *idx, const int *d_qids, int qnum, int k, int *d_r2_bits, cudaStream_t st)
{
    if (qnum <= 0) return GTS_OK;
    k_mlp_infer<<<(qnum + kInferQ - 1) / kInferQ, kMH, 0, st>>>(
        idx->rows, idx->dim, d_qids, qnum, idx->mlp_piv, idx->mlp_npiv, k, idx->mlp_P, idx->mlp_norm,
        idx->mlp_norm + kMIn, idx->mlp_ymu, idx->mlp_ysig, widen_for(idx, k), d_r2_bits);
    idx->kernel_launches++;
    GTS_CUDA_TRY(cudaGetLastError());
    return GTS_OK;
}

// One loss/gradient evaluation on a host batch with host parameters (used to
// check the device kernels against a CPU implementation).
int mlp_grad(const float *hX, const float *hT, int B, const float *hP, const float *hnorm, float *hG,
             float *hloss)
{
    MlpBufs b;
    int rc;
    if ((rc = b.alloc(B, B))) return rc;
    DevVec v2;
    float *P = nullptr, *T = nullptr, *norm = nullptr;
    if ((rc = v2.alloc(&P, kMlpParams)) || (rc = v2.alloc(&T, B)) || (rc = v2.alloc(&norm, 2 * kMIn))) return rc;
    GTS_CUDA_TRY(cudaMemcpy(b.X, hX, sizeof(float) * (size_t)B * kMIn, cudaMemcpyHostToDevice));
    GTS_CUDA_TRY(cudaMemcpy(T, hT, sizeof(float) * B, cudaMemcpyHostToDevice));
    GTS_CUDA_TRY(cudaMemcpy(P, hP, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
    GTS_CUDA_TRY(cudaMemcpy(norm, hnorm, sizeof(float) * 2 * kMIn, cudaMemcpyHostToDevice));
    GTS_CUDA_TRY(cudaMemset(b.loss, 0, sizeof(float)));
    k_mlp_fwd<<<B, kMH>>>(b.X, nullptr, B, P, norm, norm + kMIn, b.H1, b.H2, b.Y);
    k_mlp_bwd_act<<<B, kMH>>>(nullptr, B, T, P, b.H1, b.H2, b.Y, b.dY, b.dZ2, b.dZ1, b.loss);
    k_mlp_bwd_params<<<(kMlpParams + 255) / 256, 256>>>(b.X, nullptr, B, norm, norm + kMIn, b.H1, b.H2, b.dY, b.dZ2,
                                                         b.dZ1, b.G);
    GTS_CUDA_TRY(cudaGetLastError());
    GTS_CUDA_TRY(cudaMemcpy(hG, b.G, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
    GTS_CUDA_TRY(cudaMemcpy(hloss, b.loss, sizeof(float), cudaMemcpyDeviceToHost));
    return GTS_OK;
}

int mlp_train(gts_index *idx, int n_train, int k_max, int epochs, unsigned seed, float *val_rmse, float *widen_out)
{
    cudaStream_t st = idx->stream;
    if (n_train < 256 || k_max < 1 || k_max > 64 || epochs < 1) {
        gts_set_error("learn_radius: need n_train >= 256, 1 <= k_max <= 64, epochs >= 1");
        return GTS_ERR_INVALID;
    }
    if (idx->num < k_max) {
        gts_set_error("learn_radius: the data set has fewer than k_max objects");
        return GTS_ERR_INVALID;
    }
    int rc;
    if ((rc = mlp_alloc_model(idx))) return rc;
    if ((rc = mlp_pick_pivots(idx, st))) return rc;
    // ---- training set: random objects, random k, exact k-th distances
    std::mt19937 rng(seed);
    std::vector<int> qids(n_train), ks(n_train);
    std::uniform_int_distribution<int> pick(0, idx->num - 1);
    // k = 1 is not learned: the nearest object is the query itself (distance
    // 0), and the seed for k = 1 is 0
    const int kchoices[6] = {2, 4, 8, 16, 32, 64};
    std::vector<int> kc;
    for (int c : kchoices)
        if (c <= k_max) kc.push_back(c);
    if (k_max >= 2 && (kc.empty() || kc.back() != k_max)) kc.push_back(k_max);
    if (kc.empty()) {
        gts_set_error("learn_radius: k_max must be at least 2");
        return GTS_ERR_INVALID;
    }
    std::uniform_int_distribution<int> pickk(0, (int)kc.size() - 1);
    for (int i = 0; i < n_train; i++) {
        qids[i] = pick(rng);
        ks[i] = kc[pickk(rng)];
    }
    DevVec dv;
    int *d_q = nullptr, *d_k = nullptr, *d_sel = nullptr;
    float *d_kth = nullptr, *d_dis = nullptr, *d_T = nullptr, *M = nullptr, *V = nullptr;
    if ((rc = dv.alloc(&d_q, n_train)) || (rc = dv.alloc(&d_k, n_train)) || (rc = dv.alloc(&d_kth, n_train)) ||
        (rc = dv.alloc(&d_dis, (size_t)n_train * k_max)) || (rc = dv.alloc(&d_T, n_train)) ||
        (rc = dv.alloc(&d_sel, n_train)) || (rc = dv.alloc(&M, 2 * (size_t)kMlpParams)))
        return rc;
    V = M + kMlpParams;
    GTS_CUDA_TRY(cudaMemcpyAsync(d_q, qids.data(), sizeof(int) * n_train, cudaMemcpyHostToDevice, st));
    GTS_CUDA_TRY(cudaMemcpyAsync(d_k, ks.data(), sizeof(int) * n_train, cudaMemcpyHostToDevice, st));
    // exact radii from the index itself (unseeded exact search: the model is being trained)
    idx->mlp_ready = false;
    if ((rc = search_knn(idx, d_q, n_train, k_max, 1, d_kth, nullptr, d_dis, st))) return rc;
    std::vector<float> dis((size_t)n_train * k_max), T(n_train);
    GTS_CUDA_TRY(cudaMemcpyAsync(dis.data(), d_dis, sizeof(float) * dis.size(), cudaMemcpyDeviceToHost, st));
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < n_train; i++) {
        float r = dis[(size_t)i * k_max + ks[i] - 1];
        T[i] = logf(std::max(r, 1e-6f));
    }
    // ---- features and standardisation
    MlpBufs b;
    const int batch = 1024;
    if ((rc = b.alloc(n_train, batch))) return rc;
    if ((rc = mlp_features(idx, d_q, n_train, d_k, 0, b.X, st))) return rc;
    std::vector<float> X((size_t)n_train * kMIn);
    GTS_CUDA_TRY(cudaMemcpyAsync(X.data(), b.X, sizeof(float) * X.size(), cudaMemcpyDeviceToHost, st));
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    const int n_val = std::max(64, n_train / 10), n_fit = n_train - n_val;
    std::vector<float> norm(2 * kMIn);
    for (int f = 0; f < kMIn; f++) {
        double s = 0, s2 = 0;
        for (int i = 0; i < n_fit; i++) {
            double x = X[(size_t)i * kMIn + f];
            s += x;
            s2 += x * x;
        }
        double mu = s / n_fit, var = s2 / n_fit - mu * mu;
        norm[f] = (float)mu;
        norm[kMIn + f] = (float)std::max(1e-6, std::sqrt(std::max(var, 0.0)));
    }
    double ys = 0, ys2 = 0;
    for (int i = 0; i < n_fit; i++) {
        ys += T[i];
        ys2 += (double)T[i] * T[i];
    }
    const float ymu = (float)(ys / n_fit);
    const float ysig = (float)std::max(1e-6, std::sqrt(std::max(ys2 / n_fit - (ys / n_fit) * (ys / n_fit), 0.0)));
    for (int i = 0; i < n_train; i++) T[i] = (T[i] - ymu) / ysig;
    GTS_CUDA_TRY(cudaMemcpyAsync(d_T, T.data(), sizeof(float) * n_train, cudaMemcpyHostToDevice, st));
    GTS_CUDA_TRY(cudaMemcpyAsync(idx->mlp_norm, norm.data(), sizeof(float) * 2 * kMIn, cudaMemcpyHostToDevice, st));
    // ---- initial parameters (He-uniform), Adam state
    std::vector<float> P(kMlpParams, 0.f);
    auto init = [&](int off, int fan_in, int count) {
        std::uniform_real_distribution<float> u(-std::sqrt(6.f / fan_in), std::sqrt(6.f / fan_in));
        for (int i = 0; i < count; i++) P[off + i] = u(rng);
    };
    init(kOffW1, kMIn, kMH * kMIn);
    init(kOffW2, kMH, kMH * kMH);
    init(kOffW3, kMH, kMH);
    GTS_CUDA_TRY(cudaMemcpyAsync(idx->mlp_P, P.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, st));
    GTS_CUDA_TRY(cudaMemsetAsync(M, 0, sizeof(float) * 2 * kMlpParams, st));
    // ---- minibatch Adam
    std::vector<int> order(n_fit);
    std::iota(order.begin(), order.end(), 0);
    const float lr = 2e-3f, be1 = 0.9f, be2 = 0.999f;
    long step = 0;
    const int per_epoch = std::max(1, n_fit / batch);
    epochs = std::max(epochs, (3000 + per_epoch - 1) / per_epoch);   // at least ~3000 Adam steps
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(order.begin(), order.end(), rng);
        GTS_CUDA_TRY(cudaMemcpyAsync(d_sel, order.data(), sizeof(int) * n_fit, cudaMemcpyHostToDevice, st));
        for (int s0 = 0; s0 + batch <= n_fit; s0 += batch) {
            step++;
            const int *sel = d_sel + s0;
            k_mlp_fwd<<<batch, kMH, 0, st>>>(b.X, sel, batch, idx->mlp_P, idx->mlp_norm, idx->mlp_norm + kMIn, b.H1,
                                             b.H2, b.Y);
            k_mlp_bwd_act<<<batch, kMH, 0, st>>>(sel, batch, d_T, idx->mlp_P, b.H1, b.H2, b.Y, b.dY, b.dZ2, b.dZ1,
                                                 b.loss);
            k_mlp_bwd_params<<<(kMlpParams + 255) / 256, 256, 0, st>>>(b.X, sel, batch, idx->mlp_norm,
                                                                       idx->mlp_norm + kMIn, b.H1, b.H2, b.dY,
                                                                       b.dZ2, b.dZ1, b.G);
            float c1 = 1.f - std::pow(be1, (float)step), c2 = 1.f - std::pow(be2, (float)step);
            float lr_t = ep < epochs - 2 ? lr : lr * 0.2f;
            k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(idx->mlp_P, b.G, M, V, lr_t, be1, be2, 1e-8f, c1, c2);
        }
        GTS_CUDA_TRY(cudaGetLastError());
    }
    // ---- validation: residuals of the held-out samples set the widening
    std::vector<int> vsel(n_val);
    std::iota(vsel.begin(), vsel.end(), n_fit);
    GTS_CUDA_TRY(cudaMemcpyAsync(d_sel, vsel.data(), sizeof(int) * n_val, cudaMemcpyHostToDevice, st));
    float *Yv = nullptr;
    DevVec dv2;
    if ((rc = dv2.alloc(&Yv, n_val))) return rc;
    k_mlp_fwd<<<n_val, kMH, 0, st>>>(b.X, d_sel, n_val, idx->mlp_P, idx->mlp_norm, idx->mlp_norm + kMIn, nullptr,
                                     nullptr, Yv);
    std::vector<float> yv(n_val);
    GTS_CUDA_TRY(cudaMemcpyAsync(yv.data(), Yv, sizeof(float) * n_val, cudaMemcpyDeviceToHost, st));
    GTS_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<float> under(n_val);   // how much larger than predicted the true radius was (log)
    double se = 0;
    for (int i = 0; i < n_val; i++) {
        float d = (T[n_fit + i] - yv[i]) * ysig;
        under[i] = d;
        se += (double)d * d;
    }
    // per trained k, the 99.5th percentile of its own held-out
    // under-predictions (a class with fewer than 400 samples keeps the
    // global factor): a k whose radius the network predicts well is widened
    // less, so its seeds stay tighter for the same ~0.5% of re-answers
    {
        std::vector<std::vector<float>> byk(65);
        for (int i = 0; i < n_val; i++) byk[ks[n_fit + i]].push_back(under[i]);
        for (int kv = 0; kv <= 64; kv++) {
            idx->mlp_widen_at[kv] = 0.f;
            if (byk[kv].size() < 400) continue;
            std::sort(byk[kv].begin(), byk[kv].end());
            const float qk = byk[kv][(size_t)(0.995 * (byk[kv].size() - 1))];
            idx->mlp_widen_at[kv] = std::exp(std::max(qk, 0.f)) * 1.001f;
        }
    }
    std::sort(under.begin(), under.end());
    float q = under[(size_t)(0.995 * (n_val - 1))];   // 99.5th percentile: ~0.5% of queries rerun
    idx->mlp_ymu = ymu;
    idx->mlp_ysig = ysig;
    idx->mlp_widen = std::exp(std::max(q, 0.f)) * 1.001f;
    idx->mlp_ready = true;
    for (int &c : idx->fast_cfg) c = 0;   // tuned with the previous seeds
    graph_invalidate(idx);                 // captured the previous model's scalars
    if (val_rmse) *val_rmse = (float)std::sqrt(se / n_val);
    if (widen_out) *widen_out = idx->mlp_widen;
    return GTS_OK;
}

}  // namespace gts

extern "C" int gts_learn_radius(gts_index *idx, int n_train, int k_max, int epochs, unsigned seed,
                                float *val_rmse_log, float *widen)
{
    if (!idx) {
        gts_set_error("null index");
        return GTS_ERR_INVALID;
    }
    if (idx->metric != gts::kL2) {
        gts_set_error("the learned radius seeds the L2 tensor-core filter; metric %d has no use for it",
                      idx->metric);
        return GTS_ERR_INVALID;
    }
    return gts::mlp_train(idx, n_train, k_max, epochs, seed, val_rmse_log, widen);
}

extern "C" int gts_radius_model_params(const gts_index *idx, float *params, float *norm, float *ymu_ysig_widen)
{
    if (!idx || !idx->mlp_ready) {
        gts_set_error("no trained radius model on this index");
        return GTS_ERR_INVALID;
    }
    if (params) GTS_CUDA_TRY(cudaMemcpy(params, idx->mlp_P, sizeof(float) * gts::kMlpParams, cudaMemcpyDeviceToHost));
    if (norm) GTS_CUDA_TRY(cudaMemcpy(norm, idx->mlp_norm, sizeof(float) * 2 * gts::kMIn, cudaMemcpyDeviceToHost));
    if (ymu_ysig_widen) {
        ymu_ysig_widen[0] = idx->mlp_ymu;
        ymu_ysig_widen[1] = idx->mlp_ysig;
        ymu_ysig_widen[2] = idx->mlp_widen;
    }
    return GTS_OK;
}

extern "C" int gts_radius_model_grad(const float *X, const float *target, int batch, const float *params,
                                     const float *norm, float *grad, float *loss)
{
    if (!X || !target || !params || !norm || !grad || !loss || batch < 1) {
        gts_set_error("gts_radius_model_grad: invalid argument");
        return GTS_ERR_INVALID;
    }
    return gts::mlp_grad(X, target, batch, params, norm, grad, loss);
}
