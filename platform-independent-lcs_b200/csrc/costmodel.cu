// costmodel.cu -- the learned part: a small FP32 MLP cost model, trained and
// evaluated on the GPU by hand-written kernels.  No counterpart in the
// reference.
//
// The model maps 4 shape features (log2 m, log2 n, log2 alphabet, log2 batch)
// through 64 -> 64 ReLU units to K outputs, the predicted log2 run time of K
// kernel variants.  The autotuner (slcs/autotune.py) times the variants; the
// planner picks the variant with the smallest prediction.  It never touches
// results: every variant produces identical strands.
//
// Parameter blob (floats): [feature mean 4][feature std 4][W1 64x4][b1 64]
// [W2 64x64][b2 64][W3 Kx64][b3 K]; Wn is row-major (output, input).
//
// One warp evaluates one sample: lanes own hidden units lane and lane+32, the
// weights sit in shared memory (W2 both row-major and transposed so that both
// the forward and the backward sweep read without bank conflicts), gradients
// are summed per block in shared memory and added to global memory once per
// block.  Training is full-batch Adam.
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "slcs_internal.cuh"

namespace slcs {
namespace {

constexpr int F = SLCS_MLP_FEATURES;
constexpr int H = SLCS_MLP_HIDDEN;
constexpr int MLP_WARPS = 8;

__host__ __device__ constexpr int off_mean() { return 0; }
__host__ __device__ constexpr int off_std() { return F; }
__host__ __device__ constexpr int off_w1() { return 2 * F; }
__host__ __device__ constexpr int off_b1() { return 2 * F + H * F; }
__host__ __device__ constexpr int off_w2() { return off_b1() + H; }
__host__ __device__ constexpr int off_b2() { return off_w2() + H * H; }
__host__ __device__ constexpr int off_w3() { return off_b2() + H; }
__host__ __device__ inline int off_b3(int k) { return off_w3() + k * H; }
__host__ __device__ inline int param_count(int k) { return off_b3(k) + k; }

__device__ __forceinline__ float warp_sum_f(float v)
{
    for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(FULL_MASK, v, off);
    return v;
}

// Shared-memory layout of one block, in floats.
struct MlpSmem {
    int w1, b1, w2, w2t, b2, w3, b3, g, act, total;
    __host__ __device__ MlpSmem(int k)
    {
        w1 = 0;
        b1 = w1 + H * F;
        w2 = b1 + H;
        w2t = w2 + H * H;
        b2 = w2t + H * H;
        w3 = b2 + H;
        b3 = w3 + k * H;
        g = b3 + k;                                  // gradient of params [w1 .. b3] (blob order, no mean/std)
        act = g + (param_count(k) - 2 * F);          // per warp: h1, h2, dh2 (3*H)
        total = act + MLP_WARPS * 3 * H;
    }
};

// Forward (and with BACKWARD, gradient and loss) for samples [0, n).
template <bool BACKWARD>
__global__ void __launch_bounds__(MLP_WARPS * 32) mlp_kernel(const float *__restrict__ P, int k,
                                                              const float *__restrict__ X, const float *__restrict__ T,
                                                              const uint8_t *__restrict__ M, int n, float *Y,
                                                              float *G, float *loss, float inv_count)
{
    extern __shared__ float sm[];
    const MlpSmem L(k);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int i = tid; i < H * F; i += blockDim.x) sm[L.w1 + i] = P[off_w1() + i];
    for (int i = tid; i < H; i += blockDim.x) {
        sm[L.b1 + i] = P[off_b1() + i];
        sm[L.b2 + i] = P[off_b2() + i];
    }
    for (int i = tid; i < H * H; i += blockDim.x) {
        const float v = P[off_w2() + i];
        sm[L.w2 + i] = v;
        sm[L.w2t + (i % H) * H + i / H] = v; // w2t[in][out]
    }
    for (int i = tid; i < k * H; i += blockDim.x) sm[L.w3 + i] = P[off_w3() + i];
    for (int i = tid; i < k; i += blockDim.x) sm[L.b3 + i] = P[off_b3(k) + i];
    if (BACKWARD)
        for (int i = tid; i < param_count(k) - 2 * F; i += blockDim.x) sm[L.g + i] = 0.f;
    __syncthreads();

    float *h1 = sm + L.act + w * 3 * H, *h2 = h1 + H, *dh2 = h2 + H;
    float lsum = 0.f;
    const int warps_total = gridDim.x * MLP_WARPS;
    for (int s = blockIdx.x * MLP_WARPS + w; s < n; s += warps_total) {
        float x[F];
#pragma unroll
        for (int f = 0; f < F; ++f) x[f] = (X[s * F + f] - P[off_mean() + f]) / P[off_std() + f];
        // layer 1: units lane, lane+32
        float z1[2], a1[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int u = lane + 32 * q;
            float z = sm[L.b1 + u];
#pragma unroll
            for (int f = 0; f < F; ++f) z += sm[L.w1 + u * F + f] * x[f];
            z1[q] = z;
            a1[q] = fmaxf(z, 0.f);
            h1[u] = a1[q];
        }
        __syncwarp();
        // layer 2
        float z2[2], a2[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int u = lane + 32 * q;
            float z = sm[L.b2 + u];
            for (int i = 0; i < H; ++i) z += sm[L.w2t + i * H + u] * h1[i];
            z2[q] = z;
            a2[q] = fmaxf(z, 0.f);
            h2[u] = a2[q];
        }
        __syncwarp();
        // output layer: warp-reduce each output
        for (int o = 0; o < k; ++o) {
            float part = sm[L.w3 + o * H + lane] * a2[0] + sm[L.w3 + o * H + lane + 32] * a2[1];
            const float y = warp_sum_f(part) + sm[L.b3 + o];
            if (!BACKWARD) {
                if (lane == 0) Y[size_t(s) * k + o] = y;
                continue;
            }
            const bool on = M[size_t(s) * k + o] != 0;
            const float diff = on ? y - T[size_t(s) * k + o] : 0.f;
            const float dy = 2.f * diff * inv_count;
            if (lane == 0) {
                lsum += diff * diff * inv_count;
                atomicAdd(&sm[L.g + (off_b3(k) - 2 * F) + o], dy);
            }
            // dW3[o][u] += dy * h2[u]
            atomicAdd(&sm[L.g + (off_w3() - 2 * F) + o * H + lane], dy * a2[0]);
            atomicAdd(&sm[L.g + (off_w3() - 2 * F) + o * H + lane + 32], dy * a2[1]);
            // keep dy per output in h2's partner buffer: dh2 accumulates below
            if (o == 0) {
                dh2[lane] = 0.f;
                dh2[lane + 32] = 0.f;
            }
            dh2[lane] += sm[L.w3 + o * H + lane] * dy;
            dh2[lane + 32] += sm[L.w3 + o * H + lane + 32] * dy;
        }
        if (BACKWARD) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int u = lane + 32 * q;
                const float d = z2[q] > 0.f ? dh2[u] : 0.f;
                dh2[u] = d;
                atomicAdd(&sm[L.g + (off_b2() - 2 * F) + u], d);
            }
            __syncwarp();
            // dW2[u][i] += dh2[u] * h1[i]: lanes own i = lane, lane+32
            for (int u = 0; u < H; ++u) {
                const float d = dh2[u];
                atomicAdd(&sm[L.g + (off_w2() - 2 * F) + u * H + lane], d * h1[lane]);
                atomicAdd(&sm[L.g + (off_w2() - 2 * F) + u * H + lane + 32], d * h1[lane + 32]);
            }
            // dh1[i] = relu'(z1[i]) * sum_u W2[u][i] dh2[u]
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int i = lane + 32 * q;
                float acc = 0.f;
                for (int u = 0; u < H; ++u) acc += sm[L.w2 + u * H + i] * dh2[u];
                const float d = z1[q] > 0.f ? acc : 0.f;
                atomicAdd(&sm[L.g + (off_b1() - 2 * F) + i], d);
#pragma unroll
                for (int f = 0; f < F; ++f) atomicAdd(&sm[L.g + (off_w1() - 2 * F) + i * F + f], d * x[f]);
            }
        }
        __syncwarp();
    }
    if (BACKWARD) {
        __syncthreads();
        for (int i = tid; i < param_count(k) - 2 * F; i += blockDim.x) atomicAdd(&G[i], sm[L.g + i]);
        if (lane == 0) atomicAdd(loss, lsum);
    }
}

// Adam on the weight part of the blob (everything after mean/std).
__global__ void adam_kernel(float *P, const float *G, float *m1, float *m2, int count, float lr, float b1, float b2,
                            float eps, float c1, float c2)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float g = G[i];
        const float a = b1 * m1[i] + (1.f - b1) * g;
        const float v = b2 * m2[i] + (1.f - b2) * g * g;
        m1[i] = a;
        m2[i] = v;
        P[2 * F + i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
    }
}

struct DeviceMlp {
    float *P = nullptr, *X = nullptr, *T = nullptr, *Y = nullptr, *G = nullptr, *loss = nullptr;
    float *m1 = nullptr, *m2 = nullptr;
    uint8_t *M = nullptr;
    ~DeviceMlp()
    {
        cudaFree(P);
        cudaFree(X);
        cudaFree(T);
        cudaFree(Y);
        cudaFree(G);
        cudaFree(loss);
        cudaFree(m1);
        cudaFree(m2);
        cudaFree(M);
    }
};

slcs_status mlp_launch_prep(int k, size_t &smem)
{
    smem = size_t(MlpSmem(k).total) * sizeof(float);
    SLCS_CUDA(cudaFuncSetAttribute(mlp_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    SLCS_CUDA(cudaFuncSetAttribute(mlp_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    return SLCS_OK;
}

int mlp_blocks(int n) { return std::max(1, std::min(4 * sm_count(), (n + MLP_WARPS - 1) / MLP_WARPS)); }

slcs_status check_k(int32_t k)
{
    if (k < 1 || k > SLCS_MLP_MAX_OUTPUTS) return fail(SLCS_ERR_RANGE, "cost model outputs must be 1..32");
    return SLCS_OK;
}

} // namespace
} // namespace slcs

using namespace slcs;

extern "C" {

int32_t slcs_costmodel_param_count(int32_t k) { return (k < 1 || k > SLCS_MLP_MAX_OUTPUTS) ? 0 : param_count(k); }

slcs_status slcs_costmodel_init(float *params, int32_t k, uint64_t seed, const float *feat_mean, const float *feat_std)
{
    slcs_status s = check_k(k);
    if (s != SLCS_OK) return s;
    if (!params || !feat_mean || !feat_std) return fail(SLCS_ERR_INVALID, "null pointer");
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    std::memset(params, 0, sizeof(float) * size_t(param_count(k)));
    for (int f = 0; f < F; ++f) {
        params[off_mean() + f] = feat_mean[f];
        params[off_std() + f] = feat_std[f] > 0.f ? feat_std[f] : 1.f;
    }
    // He initialisation for the ReLU layers, small output layer.
    for (int i = 0; i < H * F; ++i) params[off_w1() + i] = nd(rng) * std::sqrt(2.f / F);
    for (int i = 0; i < H * H; ++i) params[off_w2() + i] = nd(rng) * std::sqrt(2.f / H);
    for (int i = 0; i < k * H; ++i) params[off_w3() + i] = nd(rng) * std::sqrt(1.f / H);
    return SLCS_OK;
}

slcs_status slcs_costmodel_predict(const float *params, int32_t k, const float *X, int32_t n, float *Y)
{
    slcs_status s = check_k(k);
    if (s != SLCS_OK) return s;
    if (n < 0 || !params || (n > 0 && (!X || !Y))) return fail(SLCS_ERR_INVALID, "bad predict arguments");
    if (n == 0) return SLCS_OK;
    DeviceMlp D;
    const size_t pc = size_t(param_count(k));
    SLCS_CUDA(cudaMalloc(&D.P, pc * 4));
    SLCS_CUDA(cudaMalloc(&D.X, size_t(n) * F * 4));
    SLCS_CUDA(cudaMalloc(&D.Y, size_t(n) * k * 4));
    SLCS_CUDA(cudaMemcpy(D.P, params, pc * 4, cudaMemcpyHostToDevice));
    SLCS_CUDA(cudaMemcpy(D.X, X, size_t(n) * F * 4, cudaMemcpyHostToDevice));
    size_t smem = 0;
    s = mlp_launch_prep(k, smem);
    if (s != SLCS_OK) return s;
    mlp_kernel<false><<<mlp_blocks(n), MLP_WARPS * 32, smem>>>(D.P, k, D.X, nullptr, nullptr, n, D.Y, nullptr,
                                                                 nullptr, 0.f);
    SLCS_CUDA(cudaGetLastError());
    SLCS_CUDA(cudaMemcpy(Y, D.Y, size_t(n) * k * 4, cudaMemcpyDeviceToHost));
    return SLCS_OK;
}

static slcs_status upload_training(DeviceMlp &D, const float *params, int32_t k, const float *X, const float *T,
                                   const uint8_t *M, int32_t n, float &inv_count)
{
    const size_t pc = size_t(param_count(k));
    SLCS_CUDA(cudaMalloc(&D.P, pc * 4));
    SLCS_CUDA(cudaMalloc(&D.X, size_t(n) * F * 4));
    SLCS_CUDA(cudaMalloc(&D.T, size_t(n) * k * 4));
    SLCS_CUDA(cudaMalloc(&D.M, size_t(n) * k));
    SLCS_CUDA(cudaMalloc(&D.G, pc * 4));
    SLCS_CUDA(cudaMalloc(&D.loss, 4));
    SLCS_CUDA(cudaMemcpy(D.P, params, pc * 4, cudaMemcpyHostToDevice));
    SLCS_CUDA(cudaMemcpy(D.X, X, size_t(n) * F * 4, cudaMemcpyHostToDevice));
    SLCS_CUDA(cudaMemcpy(D.T, T, size_t(n) * k * 4, cudaMemcpyHostToDevice));
    SLCS_CUDA(cudaMemcpy(D.M, M, size_t(n) * k, cudaMemcpyHostToDevice));
    size_t cnt = 0;
    for (size_t i = 0; i < size_t(n) * k; ++i) cnt += M[i] != 0;
    inv_count = cnt ? 1.f / float(cnt) : 0.f;
    return SLCS_OK;
}

slcs_status slcs_costmodel_grad(const float *params, int32_t k, const float *X, const float *T, const uint8_t *M,
                                int32_t n, float *grad_out, float *loss_out)
{
    slcs_status s = check_k(k);
    if (s != SLCS_OK) return s;
    if (n <= 0 || !params || !X || !T || !M || !grad_out) return fail(SLCS_ERR_INVALID, "bad gradient arguments");
    DeviceMlp D;
    float inv = 0.f;
    s = upload_training(D, params, k, X, T, M, n, inv);
    if (s != SLCS_OK) return s;
    const int wc = param_count(k) - 2 * F;
    SLCS_CUDA(cudaMemset(D.G, 0, size_t(wc) * 4));
    SLCS_CUDA(cudaMemset(D.loss, 0, 4));
    size_t smem = 0;
    s = mlp_launch_prep(k, smem);
    if (s != SLCS_OK) return s;
    mlp_kernel<true><<<mlp_blocks(n), MLP_WARPS * 32, smem>>>(D.P, k, D.X, D.T, D.M, n, nullptr, D.G, D.loss, inv);
    SLCS_CUDA(cudaGetLastError());
    // gradient of the mean/std slots is zero: they are not trained
    std::memset(grad_out, 0, sizeof(float) * 2 * F);
    SLCS_CUDA(cudaMemcpy(grad_out + 2 * F, D.G, size_t(wc) * 4, cudaMemcpyDeviceToHost));
    if (loss_out) SLCS_CUDA(cudaMemcpy(loss_out, D.loss, 4, cudaMemcpyDeviceToHost));
    return SLCS_OK;
}

slcs_status slcs_costmodel_train(float *params, int32_t k, const float *X, const float *T, const uint8_t *M,
                                 int32_t n, int32_t epochs, float lr, float *loss_out)
{
    slcs_status s = check_k(k);
    if (s != SLCS_OK) return s;
    if (n <= 0 || epochs < 0 || !params || !X || !T || !M) return fail(SLCS_ERR_INVALID, "bad training arguments");
    DeviceMlp D;
    float inv = 0.f;
    s = upload_training(D, params, k, X, T, M, n, inv);
    if (s != SLCS_OK) return s;
    const int wc = param_count(k) - 2 * F;
    SLCS_CUDA(cudaMalloc(&D.m1, size_t(wc) * 4));
    SLCS_CUDA(cudaMalloc(&D.m2, size_t(wc) * 4));
    SLCS_CUDA(cudaMemset(D.m1, 0, size_t(wc) * 4));
    SLCS_CUDA(cudaMemset(D.m2, 0, size_t(wc) * 4));
    size_t smem = 0;
    s = mlp_launch_prep(k, smem);
    if (s != SLCS_OK) return s;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float c1 = 1.f, c2 = 1.f;
    const int blocks = mlp_blocks(n);
    for (int e = 0; e < epochs; ++e) {
        SLCS_CUDA(cudaMemsetAsync(D.G, 0, size_t(wc) * 4));
        SLCS_CUDA(cudaMemsetAsync(D.loss, 0, 4));
        mlp_kernel<true><<<blocks, MLP_WARPS * 32, smem>>>(D.P, k, D.X, D.T, D.M, n, nullptr, D.G, D.loss, inv);
        c1 *= b1;
        c2 *= b2;
        adam_kernel<<<(wc + 255) / 256, 256>>>(D.P, D.G, D.m1, D.m2, wc, lr, b1, b2, eps, 1.f - c1, 1.f - c2);
    }
    SLCS_CUDA(cudaGetLastError());
    SLCS_CUDA(cudaMemcpy(params, D.P, size_t(param_count(k)) * 4, cudaMemcpyDeviceToHost));
    if (loss_out) SLCS_CUDA(cudaMemcpy(loss_out, D.loss, 4, cudaMemcpyDeviceToHost));
    return SLCS_OK;
}

} // extern "C"
