// selector.cu -- schedule selection: per-batch statistics of the TB / PU
// records (k_features), the selector MLP (16 -> 64 -> 64 -> K, bf16 weights,
// fp32 accumulation) with its training kernels (forward, backward, Adam),
// and the device parts of exhaustive autotuning.  None of it touches pixels:
// it only chooses which schedule variant of k_residual / k_recon runs.
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "selector.cuh"

namespace hpvcd {

// ===========================================================================
// Features
// ===========================================================================

// Integer accumulators of k_features (exact, order-independent sums).
enum FeatAcc {
    FA_TB4 = 0, FA_TB8, FA_TB16, FA_TB32,  // luma TB area by size
    FA_CODED,        // coded luma TB area
    FA_INTRA,        // intra luma TB area
    FA_QP, FA_QP2,   // sum of QpY (+ 64) and its square over luma TBs
    FA_NTB,          // luma TB count
    FA_NX,           // sum of 64 * nx / n over coded luma TBs
    FA_NCODED,       // coded luma TB count
    FA_NPU,          // PU count
    FA_MV,           // sum of |mv_x| + |mv_y| over used lists (quarter-pel)
    FA_NMV,          // lists used
    FA_BI,           // bi-predicted PUs
    FA_COUNT
};

__global__ void k_features(const DevPic* __restrict__ pics, uint32_t n_pics,
                           unsigned long long* __restrict__ acc) {
    unsigned long long loc[FA_COUNT];
#pragma unroll
    for (int i = 0; i < FA_COUNT; ++i) loc[i] = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t p = 0; p < n_pics; ++p) {
        const DevPic& P = pics[p];
        for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < P.n_tus; r += stride) {
            const hpvcd_tu t = P.tus[r];
            if (t.comp != 0 || t.log2n < 2 || t.log2n > 5) continue;
            const bool coded = (t.flags & HPVCD_TU_CBF) != 0, intra = (t.flags & HPVCD_TU_INTRA) != 0;
            if (!coded && !intra) continue;  // "mark decoded" record of an inter CU
            const unsigned long long area = 1ull << (2 * t.log2n);
#pragma unroll
            for (int z = 0; z < 4; ++z) loc[FA_TB4 + z] += t.log2n == z + 2 ? area : 0ull;  // static indexes
            if (coded) {
                loc[FA_CODED] += area;
                const int n = 1 << t.log2n;
                const int nx = (t.nx == 0 || t.nx > n) ? n : t.nx;
                loc[FA_NX] += (unsigned long long)(64 * nx / n);
                loc[FA_NCODED] += 1;
            }
            if (intra) loc[FA_INTRA] += area;
            const int qp = t.qp_y + 64;
            loc[FA_QP] += (unsigned long long)qp;
            loc[FA_QP2] += (unsigned long long)(qp * qp);
            loc[FA_NTB] += 1;
        }
        for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < P.n_pus; u += stride) {
            const hpvcd_pu pu = P.pus[u];
            loc[FA_NPU] += 1;
            int lists = 0;
            for (int l = 0; l < 2; ++l)
                if (pu.flags & (1u << l)) {
                    loc[FA_MV] += (unsigned long long)(abs((int)pu.mv[l][0]) + abs((int)pu.mv[l][1]));
                    ++lists;
                }
            loc[FA_NMV] += (unsigned long long)lists;
            if (lists == 2) loc[FA_BI] += 1;
        }
    }
    // warp reduction, then one atomic per warp and accumulator
#pragma unroll
    for (int i = 0; i < FA_COUNT; ++i) {
        unsigned long long v = loc[i];
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(acc + i, v);
    }
}

// One thread: turn the sums (and the picture geometry) into the feature vector.
__global__ void k_features_finish(const DevPic* __restrict__ pics, uint32_t n_pics,
                                  const unsigned long long* __restrict__ acc, float* __restrict__ f) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double area = 0, bd = 0, a444 = 0;
    int wave = 0;
    for (uint32_t p = 0; p < n_pics; ++p) {
        const DevPic& P = pics[p];
        const double a = (double)P.w * P.h;
        area += a;
        bd += a * P.bd;
        if (P.idc == 3) a444 += a;
        wave = max(wave, P.ctb_cols + 2 * P.ctb_rows);
    }
    area = fmax(area, 1.0);
    const double tb = fmax((double)(acc[FA_TB4] + acc[FA_TB8] + acc[FA_TB16] + acc[FA_TB32]), 1.0);
    const double ntb = fmax((double)acc[FA_NTB], 1.0);
    const double qp_mean = (double)acc[FA_QP] / ntb;
    const double qp_var = fmax((double)acc[FA_QP2] / ntb - qp_mean * qp_mean, 0.0);
    const double nmv = fmax((double)acc[FA_NMV], 1.0);
    float v[kFeatures];
    v[0] = (float)(log2(area) / 24.0);
    v[1] = (float)(log2(1.0 + n_pics) / 8.0);
    v[2] = (float)(wave / 256.0);
    v[3] = (float)((bd / area - 8.0) / 4.0);
    v[4] = (float)(a444 / area);
    for (int k = 0; k < 4; ++k) v[5 + k] = (float)(acc[FA_TB4 + k] / tb);
    v[9] = (float)(acc[FA_CODED] / area);
    v[10] = (float)(acc[FA_INTRA] / area);
    v[11] = (float)((qp_mean - 64.0) / 51.0);
    v[12] = (float)(sqrt(qp_var) / 16.0);
    v[13] = (float)((double)acc[FA_NX] / fmax((double)acc[FA_NCODED], 1.0) / 64.0);
    v[14] = (float)(log2(1.0 + (double)acc[FA_MV] / nmv / 4.0) / 8.0);
    v[15] = (float)((double)acc[FA_BI] / fmax((double)acc[FA_NPU], 1.0));
    for (int k = 0; k < kFeatures; ++k) f[k] = v[k];
}

// ===========================================================================
// MLP: y = W3 relu(W2 relu(W1 x + b1) + b2) + b3
// ===========================================================================

__device__ __forceinline__ float bf(const __nv_bfloat16* p, int i) { return __bfloat162float(p[i]); }

// Forward for samples [blockIdx.x * kMlpTile, +kMlpTile): thread j owns
// hidden unit j.  Weights are read from global memory (a few KB, L1/L2
// resident); activations of the tile live in shared memory.  h1 / h2, when
// given, receive the post-ReLU activations for the backward pass.
__global__ void __launch_bounds__(kHidden)
k_mlp_forward(const __nv_bfloat16* __restrict__ w, const float* __restrict__ x, int B, int K,
              float* __restrict__ y, float* __restrict__ h1_out, float* __restrict__ h2_out) {
    __shared__ float xs[kMlpTile][kFeatures];
    __shared__ float h1[kMlpTile][kHidden + 1];
    __shared__ float h2[kMlpTile][kHidden + 1];
    const MlpLayout L(K);
    const int j = threadIdx.x;
    const int s0 = blockIdx.x * kMlpTile;
    const int ns = min(kMlpTile, B - s0);
    for (int i = j; i < ns * kFeatures; i += kHidden) xs[i / kFeatures][i % kFeatures] = x[(size_t)s0 * kFeatures + i];
    __syncthreads();
    {
        float wr[kFeatures];
#pragma unroll
        for (int i = 0; i < kFeatures; ++i) wr[i] = bf(w, L.w1 + j * kFeatures + i);
        const float b = bf(w, L.b1 + j);
        for (int s = 0; s < ns; ++s) {
            float a = b;
#pragma unroll
            for (int i = 0; i < kFeatures; ++i) a = fmaf(wr[i], xs[s][i], a);
            h1[s][j] = fmaxf(a, 0.f);
        }
    }
    __syncthreads();
    {
        const float b = bf(w, L.b2 + j);
        float a[kMlpTile];
#pragma unroll
        for (int s = 0; s < kMlpTile; ++s) a[s] = b;
        for (int i = 0; i < kHidden; ++i) {
            const float wv = bf(w, L.w2 + j * kHidden + i);
#pragma unroll
            for (int s = 0; s < kMlpTile; ++s) a[s] = fmaf(wv, h1[s][i], a[s]);
        }
#pragma unroll
        for (int s = 0; s < kMlpTile; ++s)
            if (s < ns) h2[s][j] = fmaxf(a[s], 0.f);
    }
    __syncthreads();
    for (int o = j; o < ns * K; o += kHidden) {
        const int s = o / K, k = o % K;
        float a = bf(w, L.b3 + k);
        for (int i = 0; i < kHidden; ++i) a = fmaf(bf(w, L.w3 + k * kHidden + i), h2[s][i], a);
        y[(size_t)(s0 + s) * K + k] = a;
    }
    if (h1_out)
        for (int i = j; i < ns * kHidden; i += kHidden) {
            h1_out[(size_t)s0 * kHidden + i] = h1[i / kHidden][i % kHidden];
            h2_out[(size_t)s0 * kHidden + i] = h2[i / kHidden][i % kHidden];
        }
}

// Per-sample error signals of the loss L = mean over B*K of (y - t)^2:
// dy = 2 (y - t) / (B K); dh2 = (W3^T dy) * [h2 > 0]; dh1 = (W2^T dh2) * [h1 > 0].
__global__ void __launch_bounds__(kHidden)
k_mlp_delta(const __nv_bfloat16* __restrict__ w, const float* __restrict__ y, const float* __restrict__ t,
            const float* __restrict__ h1, const float* __restrict__ h2, int B, int K, float* __restrict__ dy,
            float* __restrict__ dh2, float* __restrict__ dh1) {
    __shared__ float sdy[kMaxVariants];
    __shared__ float sdh2[kHidden];
    const MlpLayout L(K);
    const int j = threadIdx.x;
    const int s = blockIdx.x;
    if (s >= B) return;
    const float scale = 2.f / ((float)B * (float)K);
    if (j < K) {
        const float d = (y[(size_t)s * K + j] - t[(size_t)s * K + j]) * scale;
        sdy[j] = d;
        dy[(size_t)s * K + j] = d;
    }
    __syncthreads();
    float a = 0.f;
    for (int k = 0; k < K; ++k) a = fmaf(bf(w, L.w3 + k * kHidden + j), sdy[k], a);
    a = h2[(size_t)s * kHidden + j] > 0.f ? a : 0.f;
    sdh2[j] = a;
    dh2[(size_t)s * kHidden + j] = a;
    __syncthreads();
    float b = 0.f;
    for (int i = 0; i < kHidden; ++i) b = fmaf(bf(w, L.w2 + i * kHidden + j), sdh2[i], b);
    dh1[(size_t)s * kHidden + j] = h1[(size_t)s * kHidden + j] > 0.f ? b : 0.f;
}

// Parameter gradients, one thread per parameter, samples summed in order
// (deterministic): dW3 = dy^T h2, dW2 = dh2^T h1, dW1 = dh1^T x, biases the
// column sums of the error signals.
__global__ void k_mlp_wgrad(const float* __restrict__ x, const float* __restrict__ h1, const float* __restrict__ h2,
                            const float* __restrict__ dy, const float* __restrict__ dh2,
                            const float* __restrict__ dh1, int B, int K, float* __restrict__ grad) {
    const MlpLayout L(K);
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L.total) return;
    const float* e;  // error signal column
    const float* a;  // input activation column (nullptr: bias)
    int es, ec, as = 0, ac = 0;
    if (p < L.b1) {
        e = dh1; es = kHidden; ec = (p - L.w1) / kFeatures;
        a = x; as = kFeatures; ac = (p - L.w1) % kFeatures;
    } else if (p < L.w2) {
        e = dh1; es = kHidden; ec = p - L.b1; a = nullptr;
    } else if (p < L.b2) {
        e = dh2; es = kHidden; ec = (p - L.w2) / kHidden;
        a = h1; as = kHidden; ac = (p - L.w2) % kHidden;
    } else if (p < L.w3) {
        e = dh2; es = kHidden; ec = p - L.b2; a = nullptr;
    } else if (p < L.b3) {
        e = dy; es = K; ec = (p - L.w3) / kHidden;
        a = h2; as = kHidden; ac = (p - L.w3) % kHidden;
    } else {
        e = dy; es = K; ec = p - L.b3; a = nullptr;
    }
    float g = 0.f;
    if (a) {
        for (int s = 0; s < B; ++s) g = fmaf(e[(size_t)s * es + ec], a[(size_t)s * as + ac], g);
    } else {
        for (int s = 0; s < B; ++s) g += e[(size_t)s * es + ec];
    }
    grad[p] = g;
}

// Mean squared error of y against t (one CTA, fixed summation order).
__global__ void k_mlp_loss(const float* __restrict__ y, const float* __restrict__ t, int n, float* __restrict__ loss) {
    __shared__ float part[256];
    float a = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float d = y[i] - t[i];
        a = fmaf(d, d, a);
    }
    part[threadIdx.x] = a;
    __syncthreads();
    for (int o = blockDim.x / 2; o; o >>= 1) {
        if ((int)threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = part[0] / (float)max(n, 1);
}

// Adam on the fp32 master weights; the bf16 copy is what the forward pass reads.
__global__ void k_mlp_adam(float* __restrict__ master, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ grad, int n, float lr, float beta1, float beta2, float eps,
                           float c1, float c2, __nv_bfloat16* __restrict__ w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = grad[i];
    const float mi = beta1 * m[i] + (1.f - beta1) * g;
    const float vi = beta2 * v[i] + (1.f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float p = master[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    master[i] = p;
    w[i] = __float2bfloat16_rn(p);
}

__global__ void k_to_bf16(const float* __restrict__ src, int n, __nv_bfloat16* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = __float2bfloat16_rn(src[i]);
}

__global__ void k_from_bf16(const __nv_bfloat16* __restrict__ src, int n, float* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = __bfloat162float(src[i]);
}

// argmin over the K outputs of each sample; with a domain (lo[16], hi[16]),
// a sample with a feature outside it gets HPVCD_MLP_NO_PICK instead.
__global__ void k_mlp_argmin(const float* __restrict__ y, int B, int K, uint32_t* __restrict__ pick,
                             const float* __restrict__ x, const float* __restrict__ dom) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= B) return;
    int best = 0;
    for (int k = 1; k < K; ++k)
        if (y[(size_t)s * K + k] < y[(size_t)s * K + best]) best = k;
    if (dom)
        for (int i = 0; i < kFeatures; ++i) {
            const float v = x[(size_t)s * kFeatures + i];
            if (!(v >= dom[i] && v <= dom[kFeatures + i])) best = -1;
        }
    pick[s] = best < 0 ? (uint32_t)HPVCD_MLP_NO_PICK : (uint32_t)best;
}

}  // namespace hpvcd

// ---------------------------------------------------------------------------
// Launchers (used by the host runtime in runtime.cu)
// ---------------------------------------------------------------------------
using namespace hpvcd;

extern "C" void hpvcd_note_launches(uint32_t n);

extern "C" cudaError_t hpvcd_launch_features(const DevPic* pics, uint32_t n_pics, uint32_t max_records,
                                             unsigned long long* acc, float* out, int sms, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * FA_COUNT, st);
    if (e != cudaSuccess) return e;
    const int threads = 256;
    const int grid = std::max(1, std::min<int>((int)((max_records + threads - 1) / threads), sms * 4));
    k_features<<<grid, threads, 0, st>>>(pics, n_pics, acc);
    k_features_finish<<<1, 32, 0, st>>>(pics, n_pics, acc, out);
    hpvcd_note_launches(2);
    return cudaGetLastError();
}

extern "C" cudaError_t hpvcd_launch_mlp_forward(const void* w, const float* x, int B, int K, float* y, float* h1,
                                                float* h2, cudaStream_t st) {
    if (B <= 0) return cudaSuccess;
    k_mlp_forward<<<(B + kMlpTile - 1) / kMlpTile, kHidden, 0, st>>>((const __nv_bfloat16*)w, x, B, K, y, h1, h2);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

extern "C" cudaError_t hpvcd_launch_mlp_backward(const void* w, const float* x, const float* t, int B, int K,
                                                 const float* y, const float* h1, const float* h2, float* dy,
                                                 float* dh2, float* dh1, float* grad, float* loss, cudaStream_t st) {
    if (B <= 0) return cudaSuccess;
    k_mlp_delta<<<B, kHidden, 0, st>>>((const __nv_bfloat16*)w, y, t, h1, h2, B, K, dy, dh2, dh1);
    const MlpLayout L(K);
    k_mlp_wgrad<<<(L.total + 255) / 256, 256, 0, st>>>(x, h1, h2, dy, dh2, dh1, B, K, grad);
    k_mlp_loss<<<1, 256, 0, st>>>(y, t, B * K, loss);
    hpvcd_note_launches(3);
    return cudaGetLastError();
}

extern "C" cudaError_t hpvcd_launch_mlp_adam(float* master, float* m, float* v, const float* grad, int n, float lr,
                                             float beta1, float beta2, float eps, float c1, float c2, void* w,
                                             cudaStream_t st) {
    k_mlp_adam<<<(n + 255) / 256, 256, 0, st>>>(master, m, v, grad, n, lr, beta1, beta2, eps, c1, c2,
                                                (__nv_bfloat16*)w);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

extern "C" cudaError_t hpvcd_launch_bf16_convert(const float* src, int n, void* dst, int to_bf16, float* back,
                                                 cudaStream_t st) {
    if (to_bf16)
        k_to_bf16<<<(n + 255) / 256, 256, 0, st>>>(src, n, (__nv_bfloat16*)dst);
    else
        k_from_bf16<<<(n + 255) / 256, 256, 0, st>>>((const __nv_bfloat16*)dst, n, back);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

extern "C" cudaError_t hpvcd_launch_mlp_argmin(const float* y, int B, int K, uint32_t* pick, const float* x,
                                               const float* dom, cudaStream_t st) {
    k_mlp_argmin<<<(B + 127) / 128, 128, 0, st>>>(y, B, K, pick, x, dom);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

extern "C" cudaError_t hpvcd_launch_gather_rows(const float* src, const uint32_t* idx, int rows, int width,
                                                float* dst, cudaStream_t st);

namespace hpvcd {
__global__ void k_gather_rows(const float* __restrict__ src, const uint32_t* __restrict__ idx, int rows, int width,
                              float* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * width) return;
    dst[i] = src[(size_t)idx[i / width] * width + i % width];
}
}  // namespace hpvcd

extern "C" cudaError_t hpvcd_launch_gather_rows(const float* src, const uint32_t* idx, int rows, int width,
                                                float* dst, cudaStream_t st) {
    if (rows <= 0) return cudaSuccess;
    k_gather_rows<<<(rows * width + 255) / 256, 256, 0, st>>>(src, idx, rows, width, dst);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

// ===========================================================================
// Host side of the MLP (exported through include/hpvcd_gpu.h)
// ===========================================================================
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#define HPVCD_API extern "C" __attribute__((visibility("default")))

extern "C" hpvcd_status hpvcd_internal_status(cudaError_t e);

struct hpvcd_mlp {
    int K = 0, P = 0;
    __nv_bfloat16* w = nullptr;  // bf16 parameters read by the forward pass
    float* master = nullptr;     // fp32 master copy updated by Adam
    float* m = nullptr;
    float* v = nullptr;
    float* grad = nullptr;
    float* loss = nullptr;
    uint32_t* pick = nullptr;
    float* act = nullptr;  // per-sample scratch: y, h1, h2, dy, dh2, dh1, x, t
    int cap = 0;
    uint32_t* idx = nullptr;  // batch row indices
    int idx_cap = 0;
    long long step = 0;
    float* dom = nullptr;     // feature domain lo[16], hi[16] (device)
    bool has_domain = false;
    ~hpvcd_mlp() {
        cudaFree(w); cudaFree(master); cudaFree(m); cudaFree(v); cudaFree(grad); cudaFree(loss);
        cudaFree(pick); cudaFree(act); cudaFree(idx); cudaFree(dom);
    }
    size_t per_sample() const { return (size_t)2 * K + 4 * kHidden + kFeatures + K; }
    cudaError_t reserve(int B) {
        if (B <= cap) return cudaSuccess;
        cudaFree(act);
        act = nullptr;
        cap = 0;
        const cudaError_t e = cudaMalloc(&act, per_sample() * sizeof(float) * (size_t)B);
        if (e == cudaSuccess) cap = B;
        return e;
    }
    // scratch views for batch capacity `cap`
    float* y() const { return act; }
    float* h1() const { return act + (size_t)cap * K; }
    float* h2() const { return h1() + (size_t)cap * kHidden; }
    float* dy() const { return h2() + (size_t)cap * kHidden; }
    float* dh2() const { return dy() + (size_t)cap * K; }
    float* dh1() const { return dh2() + (size_t)cap * kHidden; }
    float* xb() const { return dh1() + (size_t)cap * kHidden; }
    float* tb() const { return xb() + (size_t)cap * kFeatures; }
};

namespace {

// splitmix64 -> uniform [0, 1)
struct SelRng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    double uni() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};

hpvcd_status upload_params(hpvcd_mlp* M, const float* host) {
    cudaError_t e = cudaMemcpy(M->master, host, sizeof(float) * M->P, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(M->m, 0, sizeof(float) * M->P);
    if (e == cudaSuccess) e = cudaMemset(M->v, 0, sizeof(float) * M->P);
    if (e == cudaSuccess) e = hpvcd_launch_bf16_convert(M->master, M->P, M->w, 1, nullptr, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    M->step = 0;
    return hpvcd_internal_status(e);
}

// Forward pass into y; keep = also store the activations for the backward
// pass in the scratch, which must already hold B samples (reserve).
hpvcd_status forward_into(hpvcd_mlp* M, const float* x, int B, float* y, bool keep, cudaStream_t st) {
    if (keep && B > M->cap) return HPVCD_ERR_INVALID_ARG;
    return hpvcd_internal_status(
        hpvcd_launch_mlp_forward(M->w, x, B, M->K, y, keep ? M->h1() : nullptr, keep ? M->h2() : nullptr, st));
}

}  // namespace

HPVCD_API hpvcd_status hpvcd_mlp_create(uint32_t n_variants, uint64_t seed, hpvcd_mlp** out) {
    if (!out || n_variants < 2 || n_variants > (uint32_t)kMaxVariants) return HPVCD_ERR_INVALID_ARG;
    hpvcd_mlp* M = new (std::nothrow) hpvcd_mlp();
    if (!M) return HPVCD_ERR_ALLOC;
    M->K = (int)n_variants;
    const MlpLayout L(M->K);
    M->P = L.total;
    cudaError_t e = cudaMalloc(&M->w, sizeof(__nv_bfloat16) * M->P);
    if (e == cudaSuccess) e = cudaMalloc(&M->master, sizeof(float) * M->P);
    if (e == cudaSuccess) e = cudaMalloc(&M->m, sizeof(float) * M->P);
    if (e == cudaSuccess) e = cudaMalloc(&M->v, sizeof(float) * M->P);
    if (e == cudaSuccess) e = cudaMalloc(&M->grad, sizeof(float) * M->P);
    if (e == cudaSuccess) e = cudaMalloc(&M->loss, sizeof(float) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&M->pick, sizeof(uint32_t) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&M->dom, sizeof(float) * 2 * kFeatures);
    if (e != cudaSuccess) {
        delete M;
        return hpvcd_internal_status(e);
    }
    // He-uniform weights (bound sqrt(6 / fan_in)), zero biases
    std::vector<float> p(M->P, 0.f);
    SelRng r{seed};
    auto fill = [&](int off, int rows, int cols) {
        const double bound = std::sqrt(6.0 / cols);
        for (int i = 0; i < rows * cols; ++i) p[off + i] = (float)((2.0 * r.uni() - 1.0) * bound);
    };
    fill(L.w1, kHidden, kFeatures);
    fill(L.w2, kHidden, kHidden);
    fill(L.w3, M->K, kHidden);
    const hpvcd_status s = upload_params(M, p.data());
    if (s != HPVCD_OK) {
        delete M;
        return s;
    }
    *out = M;
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_mlp_destroy(hpvcd_mlp* M) {
    if (!M) return HPVCD_ERR_INVALID_ARG;
    cudaDeviceSynchronize();
    delete M;
    return HPVCD_OK;
}

HPVCD_API uint32_t hpvcd_mlp_param_count(const hpvcd_mlp* M) { return M ? (uint32_t)M->P : 0; }
HPVCD_API uint32_t hpvcd_mlp_variants(const hpvcd_mlp* M) { return M ? (uint32_t)M->K : 0; }

// ---------------------------------------------------------------------------
// Host-side selection for batches whose records are in host memory (the
// hpvcd_gpu_submit path): the features from the host records and the
// network's forward pass on the host, so a submit picks its schedule without
// a device round trip.  The sums are the integer sums of k_features and the
// forward uses the bf16-rounded weights with fused multiply-adds in the
// kernel's order, so the outputs are those of k_mlp_forward.
// ---------------------------------------------------------------------------
HPVCD_API hpvcd_status hpvcd_batch_features(const hpvcd_picture* pics, uint32_t n, float* out) {
    if (!pics || !out) return HPVCD_ERR_INVALID_ARG;
    unsigned long long acc[FA_COUNT] = {};
    double area = 0, bdsum = 0, a444 = 0;
    int wave = 0;
    for (uint32_t p = 0; p < n; ++p) {
        const hpvcd_picture& P = pics[p];
        const double a = (double)P.width * P.height;
        area += a;
        bdsum += a * P.bit_depth_y;
        if (P.chroma_idc == 3) a444 += a;
        const int ctb = 1 << P.log2_ctb;
        wave = std::max(wave, (int)((P.width + ctb - 1) / ctb + 2 * ((P.height + ctb - 1) / ctb)));
        for (uint32_t r = 0; r < P.n_tus && P.tus; ++r) {
            const hpvcd_tu& t = P.tus[r];
            if (t.comp != 0 || t.log2n < 2 || t.log2n > 5) continue;
            const bool coded = (t.flags & HPVCD_TU_CBF) != 0, intra = (t.flags & HPVCD_TU_INTRA) != 0;
            if (!coded && !intra) continue;
            const unsigned long long ar = 1ull << (2 * t.log2n);
            acc[FA_TB4 + (t.log2n - 2)] += ar;
            if (coded) {
                acc[FA_CODED] += ar;
                const int nn = 1 << t.log2n;
                const int nx = (t.nx == 0 || t.nx > nn) ? nn : t.nx;
                acc[FA_NX] += (unsigned long long)(64 * nx / nn);
                acc[FA_NCODED] += 1;
            }
            if (intra) acc[FA_INTRA] += ar;
            const int qp = t.qp_y + 64;
            acc[FA_QP] += (unsigned long long)qp;
            acc[FA_QP2] += (unsigned long long)(qp * qp);
            acc[FA_NTB] += 1;
        }
        for (uint32_t u = 0; u < P.n_pus && P.pus; ++u) {
            const hpvcd_pu& pu = P.pus[u];
            acc[FA_NPU] += 1;
            int lists = 0;
            for (int l = 0; l < 2; ++l)
                if (pu.flags & (1u << l)) {
                    acc[FA_MV] += (unsigned long long)(std::abs((int)pu.mv[l][0]) + std::abs((int)pu.mv[l][1]));
                    ++lists;
                }
            acc[FA_NMV] += (unsigned long long)lists;
            if (lists == 2) acc[FA_BI] += 1;
        }
    }
    // k_features_finish
    area = std::max(area, 1.0);
    const double tb = std::max((double)(acc[FA_TB4] + acc[FA_TB8] + acc[FA_TB16] + acc[FA_TB32]), 1.0);
    const double ntb = std::max((double)acc[FA_NTB], 1.0);
    const double qp_mean = (double)acc[FA_QP] / ntb;
    const double qp_var = std::max((double)acc[FA_QP2] / ntb - qp_mean * qp_mean, 0.0);
    const double nmv = std::max((double)acc[FA_NMV], 1.0);
    out[0] = (float)(std::log2(area) / 24.0);
    out[1] = (float)(std::log2(1.0 + n) / 8.0);
    out[2] = (float)(wave / 256.0);
    out[3] = (float)((bdsum / area - 8.0) / 4.0);
    out[4] = (float)(a444 / area);
    for (int k = 0; k < 4; ++k) out[5 + k] = (float)(acc[FA_TB4 + k] / tb);
    out[9] = (float)(acc[FA_CODED] / area);
    out[10] = (float)(acc[FA_INTRA] / area);
    out[11] = (float)((qp_mean - 64.0) / 51.0);
    out[12] = (float)(std::sqrt(qp_var) / 16.0);
    out[13] = (float)((double)acc[FA_NX] / std::max((double)acc[FA_NCODED], 1.0) / 64.0);
    out[14] = (float)(std::log2(1.0 + (double)acc[FA_MV] / nmv / 4.0) / 8.0);
    out[15] = (float)((double)acc[FA_BI] / std::max((double)acc[FA_NPU], 1.0));
    return HPVCD_OK;
}

// Host copy of a network: its bf16-rounded parameters as fp32 and, when it
// has one, its feature domain (lo[16], hi[16]).
extern "C" hpvcd_status hpvcd_mlp_host_copy(hpvcd_mlp* M, float* params, float* lohi, int* has_domain);

// k_mlp_forward + k_mlp_argmin for one sample on the host.
extern "C" uint32_t hpvcd_mlp_pick_host(const float* w, uint32_t K, const float* x, const float* lohi,
                                        int has_domain) {
    const MlpLayout L((int)K);
    float h1[kHidden], h2[kHidden];
    for (int j = 0; j < kHidden; ++j) {
        float a = w[L.b1 + j];
        for (int i = 0; i < kFeatures; ++i) a = std::fma(w[L.w1 + j * kFeatures + i], x[i], a);
        h1[j] = std::max(a, 0.f);
    }
    for (int j = 0; j < kHidden; ++j) {
        float a = w[L.b2 + j];
        for (int i = 0; i < kHidden; ++i) a = std::fma(w[L.w2 + j * kHidden + i], h1[i], a);
        h2[j] = std::max(a, 0.f);
    }
    int best = 0;
    float best_y = 0.f;
    for (int k = 0; k < (int)K; ++k) {
        float a = w[L.b3 + k];
        for (int i = 0; i < kHidden; ++i) a = std::fma(w[L.w3 + k * kHidden + i], h2[i], a);
        if (k == 0 || a < best_y) {
            best = k;
            best_y = a;
        }
    }
    if (has_domain)
        for (int i = 0; i < kFeatures; ++i)
            if (!(x[i] >= lohi[i] && x[i] <= lohi[kFeatures + i])) return HPVCD_MLP_NO_PICK;
    return (uint32_t)best;
}

HPVCD_API hpvcd_status hpvcd_mlp_get_params(hpvcd_mlp* M, float* host, int master) {
    if (!M || !host) return HPVCD_ERR_INVALID_ARG;
    cudaError_t e;
    if (master) {
        e = cudaMemcpy(host, M->master, sizeof(float) * M->P, cudaMemcpyDeviceToHost);
    } else {
        // the bf16 values widened to fp32
        float* tmp = nullptr;
        e = cudaMalloc(&tmp, sizeof(float) * M->P);
        if (e == cudaSuccess) e = hpvcd_launch_bf16_convert(nullptr, M->P, M->w, 0, tmp, nullptr);
        if (e == cudaSuccess) e = cudaMemcpy(host, tmp, sizeof(float) * M->P, cudaMemcpyDeviceToHost);
        cudaFree(tmp);
    }
    return hpvcd_internal_status(e);
}

extern "C" hpvcd_status hpvcd_mlp_host_copy(hpvcd_mlp* M, float* params, float* lohi, int* has_domain) {
    if (!M || !params || !lohi || !has_domain) return HPVCD_ERR_INVALID_ARG;
    const hpvcd_status s = hpvcd_mlp_get_params(M, params, 0);
    if (s != HPVCD_OK) return s;
    *has_domain = M->has_domain ? 1 : 0;
    if (!M->has_domain) return HPVCD_OK;
    return hpvcd_internal_status(cudaMemcpy(lohi, M->dom, sizeof(float) * 2 * kFeatures, cudaMemcpyDeviceToHost));
}

// Feature domain of the training data: a pick for features outside
// [lo, hi] is HPVCD_MLP_NO_PICK (callers then keep the default schedule).
HPVCD_API hpvcd_status hpvcd_mlp_set_domain(hpvcd_mlp* M, const float* lo, const float* hi) {
    if (!M || (!lo) != (!hi)) return HPVCD_ERR_INVALID_ARG;
    if (!lo) {
        M->has_domain = false;
        return HPVCD_OK;
    }
    cudaError_t e = cudaMemcpy(M->dom, lo, sizeof(float) * kFeatures, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(M->dom + kFeatures, hi, sizeof(float) * kFeatures, cudaMemcpyHostToDevice);
    M->has_domain = e == cudaSuccess;
    return hpvcd_internal_status(e);
}

HPVCD_API hpvcd_status hpvcd_mlp_set_params(hpvcd_mlp* M, const float* host) {
    if (!M || !host) return HPVCD_ERR_INVALID_ARG;
    return upload_params(M, host);
}

HPVCD_API hpvcd_status hpvcd_mlp_forward(hpvcd_mlp* M, const float* dev_x, uint32_t B, float* dev_y, void* stream) {
    if (!M || !dev_x || !dev_y) return HPVCD_ERR_INVALID_ARG;
    return forward_into(M, dev_x, (int)B, dev_y, false, (cudaStream_t)stream);
}

HPVCD_API hpvcd_status hpvcd_mlp_grad(hpvcd_mlp* M, const float* dev_x, const float* dev_t, uint32_t B,
                                      float* dev_grad, float* dev_loss, void* stream) {
    if (!M || !dev_x || !dev_t || B == 0) return HPVCD_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    // the scratch views below are only valid once the scratch holds B samples
    cudaError_t e = M->reserve((int)B);
    if (e != cudaSuccess) return hpvcd_internal_status(e);
    hpvcd_status s = forward_into(M, dev_x, (int)B, M->y(), true, st);
    if (s != HPVCD_OK) return s;
    e = hpvcd_launch_mlp_backward(M->w, dev_x, dev_t, (int)B, M->K, M->y(), M->h1(), M->h2(), M->dy(),
                                              M->dh2(), M->dh1(), M->grad, M->loss, st);
    if (e == cudaSuccess && dev_grad)
        e = cudaMemcpyAsync(dev_grad, M->grad, sizeof(float) * M->P, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && dev_loss)
        e = cudaMemcpyAsync(dev_loss, M->loss, sizeof(float), cudaMemcpyDeviceToDevice, st);
    return hpvcd_internal_status(e);
}

HPVCD_API hpvcd_status hpvcd_mlp_adam_step(hpvcd_mlp* M, float lr, void* stream) {
    if (!M) return HPVCD_ERR_INVALID_ARG;
    const float b1 = 0.9f, b2 = 0.999f;
    ++M->step;
    const float c1 = 1.f - (float)std::pow(b1, (double)M->step);
    const float c2 = 1.f - (float)std::pow(b2, (double)M->step);
    return hpvcd_internal_status(hpvcd_launch_mlp_adam(M->master, M->m, M->v, M->grad, M->P, lr, b1, b2, 1e-8f, c1,
                                                       c2, M->w, (cudaStream_t)stream));
}

// Mini-batch Adam over n samples (rows of dev_x [n][16], dev_t [n][K]) for
// `epochs` passes in a seeded shuffled order; final_loss = loss of the last batch.
HPVCD_API hpvcd_status hpvcd_mlp_train(hpvcd_mlp* M, const float* dev_x, const float* dev_t, uint32_t n,
                                       uint32_t batch, uint32_t epochs, float lr, uint64_t seed, void* stream,
                                       float* final_loss) {
    if (!M || !dev_x || !dev_t || n == 0 || batch == 0) return HPVCD_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const int Bmax = (int)std::min<uint32_t>(batch, n);
    cudaError_t e = M->reserve(Bmax);
    if (e == cudaSuccess && M->idx_cap < (int)n) {
        cudaFree(M->idx);
        M->idx = nullptr;
        M->idx_cap = 0;
        e = cudaMalloc(&M->idx, sizeof(uint32_t) * n);
        if (e == cudaSuccess) M->idx_cap = (int)n;
    }
    if (e != cudaSuccess) return hpvcd_internal_status(e);
    std::vector<uint32_t> perm(n);
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    SelRng r{seed};
    for (uint32_t ep = 0; ep < epochs; ++ep) {
        for (uint32_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[r.next() % (i + 1)]);
        e = cudaMemcpyAsync(M->idx, perm.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // perm is reused next epoch
        if (e != cudaSuccess) return hpvcd_internal_status(e);
        for (uint32_t b0 = 0; b0 < n; b0 += (uint32_t)Bmax) {
            const int B = (int)std::min<uint32_t>((uint32_t)Bmax, n - b0);
            e = hpvcd_launch_gather_rows(dev_x, M->idx + b0, B, kFeatures, M->xb(), st);
            if (e == cudaSuccess) e = hpvcd_launch_gather_rows(dev_t, M->idx + b0, B, M->K, M->tb(), st);
            if (e != cudaSuccess) return hpvcd_internal_status(e);
            hpvcd_status s = hpvcd_mlp_grad(M, M->xb(), M->tb(), (uint32_t)B, nullptr, nullptr, st);
            if (s == HPVCD_OK) s = hpvcd_mlp_adam_step(M, lr, st);
            if (s != HPVCD_OK) return s;
        }
    }
    if (final_loss) {
        e = cudaMemcpyAsync(final_loss, M->loss, sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    return hpvcd_internal_status(e);
}

// Predicted-fastest variant for each of B feature rows (device), into a host array.
HPVCD_API hpvcd_status hpvcd_mlp_pick(hpvcd_mlp* M, const float* dev_x, uint32_t B, void* stream,
                                      uint32_t* host_variant) {
    if (!M || !dev_x || !host_variant || B == 0) return HPVCD_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = M->reserve((int)B);
    if (e != cudaSuccess) return hpvcd_internal_status(e);
    hpvcd_status s = forward_into(M, dev_x, (int)B, M->y(), false, st);
    if (s != HPVCD_OK) return s;
    uint32_t* dpick = M->pick;
    uint32_t* tmp = nullptr;
    if (B > 4) {
        e = cudaMalloc(&tmp, sizeof(uint32_t) * B);
        if (e != cudaSuccess) return hpvcd_internal_status(e);
        dpick = tmp;
    }
    e = hpvcd_launch_mlp_argmin(M->y(), (int)B, M->K, dpick, dev_x, M->has_domain ? M->dom : nullptr, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_variant, dpick, sizeof(uint32_t) * B, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(tmp);
    return hpvcd_internal_status(e);
}
