// oz2_mlp.cu - the small MLP that picks the number of moduli per C tile: inference (one thread
// per tile, weights in shared memory) and training (one block, mini-batches of 256 samples,
// cross-entropy over s = 2..24 and "more than 24", Adam), both hand-written.
#include <cmath>

#include "oz2_adaptive.cuh"

namespace oz2 {
namespace {

constexpr int kW1 = 0;
constexpr int kB1 = kW1 + kHidden * kFeatures;
constexpr int kW2 = kB1 + kHidden;
constexpr int kB2 = kW2 + kHidden * kHidden;
constexpr int kW3 = kB2 + kHidden;
constexpr int kB3 = kW3 + kClasses * kHidden;
static_assert(kB3 + kClasses == kMlpParams, "parameter layout");

__device__ __forceinline__ void forward(const float* P, const float* f, float* h1, float* h2, float* logits) {
    for (int o = 0; o < kHidden; ++o) {
        float a = P[kB1 + o];
        for (int i = 0; i < kFeatures; ++i) a = fmaf(P[kW1 + o * kFeatures + i], f[i], a);
        h1[o] = fmaxf(a, 0.0f);
    }
    for (int o = 0; o < kHidden; ++o) {
        float a = P[kB2 + o];
        for (int i = 0; i < kHidden; ++i) a = fmaf(P[kW2 + o * kHidden + i], h1[i], a);
        h2[o] = fmaxf(a, 0.0f);
    }
    for (int o = 0; o < kClasses; ++o) {
        float a = P[kB3 + o];
        for (int i = 0; i < kHidden; ++i) a = fmaf(P[kW3 + o * kHidden + i], h2[i], a);
        logits[o] = a;
    }
}

__device__ __forceinline__ void softmax(float* z) {
    float mx = z[0];
    for (int c = 1; c < kClasses; ++c) mx = fmaxf(mx, z[c]);
    float sum = 0.0f;
    for (int c = 0; c < kClasses; ++c) {
        z[c] = __expf(z[c] - mx);
        sum += z[c];
    }
    const float inv = 1.0f / sum;
    for (int c = 0; c < kClasses; ++c) z[c] *= inv;
}

__global__ void mlp_infer_kernel(const float* __restrict__ params, int count, const float* __restrict__ feat,
                                 float threshold, int* __restrict__ s_out, float* __restrict__ probs_out) {
    __shared__ float P[kMlpParams];
    for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    float f[kFeatures], h1[kHidden], h2[kHidden], z[kClasses];
    for (int i = 0; i < kFeatures; ++i) f[i] = feat[static_cast<int64_t>(t) * kFeatures + i];
    forward(P, f, h1, h2, z);
    softmax(z);
    float cum = 0.0f;
    int cls = kClasses - 1;
    for (int c = 0; c < kClasses; ++c) {
        cum += z[c];
        if (cum >= threshold) {
            cls = c;
            break;
        }
    }
    s_out[t] = cls + 2;
    if (probs_out)
        for (int c = 0; c < kClasses; ++c) probs_out[static_cast<int64_t>(t) * kClasses + c] = z[c];
}

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return x;
}

constexpr int kBatch = 256;

__global__ void __launch_bounds__(kBatch) mlp_train_kernel(float* __restrict__ params, int count,
                                                           const float* __restrict__ feat,
                                                           const int* __restrict__ label, int epochs, float lr,
                                                           unsigned int seed, float* __restrict__ loss_out) {
    extern __shared__ float sm[];
    float* P = sm;                   // parameters
    float* G = P + kMlpParams;       // gradient of the batch
    float* Mo = G + kMlpParams;      // Adam first moment
    float* Vo = Mo + kMlpParams;     // Adam second moment
    __shared__ float loss_acc;
    for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) {
        P[i] = params[i];
        Mo[i] = 0.0f;
        Vo[i] = 0.0f;
    }
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float b1t = 1.0f, b2t = 1.0f;
    const int batches = (count + kBatch - 1) / kBatch;
    for (int ep = 0; ep < epochs; ++ep) {
        if (threadIdx.x == 0) loss_acc = 0.0f;
        const uint32_t rot = hash32(seed + 977u * static_cast<uint32_t>(ep)) % static_cast<uint32_t>(count);
        for (int b = 0; b < batches; ++b) {
            for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) G[i] = 0.0f;
            __syncthreads();
            const int slot = b * kBatch + threadIdx.x;
            const int in_batch = min(kBatch, count - b * kBatch);
            if (slot < count) {
                const int sidx = static_cast<int>((static_cast<uint32_t>(slot) + rot) % static_cast<uint32_t>(count));
                float f[kFeatures], h1[kHidden], h2[kHidden], z[kClasses];
                for (int i = 0; i < kFeatures; ++i) f[i] = feat[static_cast<int64_t>(sidx) * kFeatures + i];
                forward(P, f, h1, h2, z);
                softmax(z);
                const int y = min(max(label[sidx] - 2, 0), kClasses - 1);
                atomicAdd(&loss_acc, -__logf(fmaxf(z[y], 1e-12f)));
                const float scale = 1.0f / static_cast<float>(in_batch);
                float dz[kClasses];
                for (int c = 0; c < kClasses; ++c) dz[c] = (z[c] - (c == y ? 1.0f : 0.0f)) * scale;
                float dh2[kHidden];
                for (int i = 0; i < kHidden; ++i) dh2[i] = 0.0f;
                for (int c = 0; c < kClasses; ++c) {
                    atomicAdd(&G[kB3 + c], dz[c]);
                    for (int i = 0; i < kHidden; ++i) {
                        atomicAdd(&G[kW3 + c * kHidden + i], dz[c] * h2[i]);
                        dh2[i] = fmaf(P[kW3 + c * kHidden + i], dz[c], dh2[i]);
                    }
                }
                float dh1[kHidden];
                for (int i = 0; i < kHidden; ++i) dh1[i] = 0.0f;
                for (int o = 0; o < kHidden; ++o) {
                    const float g = h2[o] > 0.0f ? dh2[o] : 0.0f;
                    if (g == 0.0f) continue;
                    atomicAdd(&G[kB2 + o], g);
                    for (int i = 0; i < kHidden; ++i) {
                        atomicAdd(&G[kW2 + o * kHidden + i], g * h1[i]);
                        dh1[i] = fmaf(P[kW2 + o * kHidden + i], g, dh1[i]);
                    }
                }
                for (int o = 0; o < kHidden; ++o) {
                    const float g = h1[o] > 0.0f ? dh1[o] : 0.0f;
                    if (g == 0.0f) continue;
                    atomicAdd(&G[kB1 + o], g);
                    for (int i = 0; i < kFeatures; ++i) atomicAdd(&G[kW1 + o * kFeatures + i], g * f[i]);
                }
            }
            __syncthreads();
            b1t *= b1;
            b2t *= b2;
            for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) {
                const float g = G[i];
                Mo[i] = b1 * Mo[i] + (1.0f - b1) * g;
                Vo[i] = b2 * Vo[i] + (1.0f - b2) * g * g;
                const float mh = Mo[i] / (1.0f - b1t), vh = Vo[i] / (1.0f - b2t);
                P[i] -= lr * mh / (sqrtf(vh) + eps);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0 && loss_out) loss_out[ep] = loss_acc / static_cast<float>(count);
        __syncthreads();
    }
    for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) params[i] = P[i];
}

}  // namespace

void launch_mlp_infer(const float* params, int count, const float* feat, float threshold, int* s_out,
                      float* probs_out, cudaStream_t st) {
    if (count <= 0) return;
    mlp_infer_kernel<<<(count + 127) / 128, 128, 0, st>>>(params, count, feat, threshold, s_out, probs_out);
}

void launch_mlp_train(float* params, int count, const float* feat, const int* label, int epochs, float lr,
                      unsigned int seed, float* loss_out, cudaStream_t st) {
    if (count <= 0 || epochs <= 0) return;
    const size_t smem = 4 * kMlpParams * sizeof(float);
    cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    mlp_train_kernel<<<1, kBatch, smem, st>>>(params, count, feat, label, epochs, lr, seed, loss_out);
}

}  // namespace oz2
