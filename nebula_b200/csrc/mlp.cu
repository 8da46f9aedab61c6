// Training and evaluation kernels of the escape-probability network
// (mlp.cuh): forward, backward with binary cross-entropy on the sigmoid
// output, and Adam.  Every matrix product runs on the tensor cores as BF16
// mma.sync m16n8k16 with FP32 accumulation; operands are staged per warp in
// shared memory (row-major and transposed copies, so any product is a plain
// A[M][K] x Bt[N][K] fragment load).  One warp handles 32 samples.
#include <cuda_bf16.h>

#include "mlp.cuh"
#include "mlp_kernels.h"

namespace nbx {
namespace mlp {

namespace {

using bf16 = __nv_bfloat16;
constexpr int kWarps = 2;   // warps per training block

struct WarpBuf {
    bf16 x[32 * kIn];        // [sample][feature]
    bf16 xt[kIn * 32];       // [feature][sample]
    bf16 h1[32 * kHidden];
    bf16 h1t[kHidden * 32];
    bf16 h2[32 * kHidden];
    bf16 h2t[kHidden * 32];
    bf16 d3[32 * 16];        // dL/dz3, column 0 real
    bf16 d3t[16 * 32];
    bf16 d2[32 * kHidden];
    bf16 d2t[kHidden * 32];
    bf16 d1t[kHidden * 32];
    float z1[32 * kHidden];  // pre-activations for SiLU'
    float z2[32 * kHidden];
};

struct TrainSmem {
    Weights w;
    bf16 w2t[kHidden * kHidden];   // [in][out]
    bf16 w3t[kHidden * 16];        // [in][out padded to 16]
    float gacc[kParams];
    float loss;
    WarpBuf warp[kWarps];
};

// acc[MT][NT] += A[M][K] * Bt[N][K]^T for M = 16 MT, N = 8 NT, K = 16 KT.
template <int MT, int NT, int KT>
__device__ __forceinline__ void warp_gemm(const bf16* A, int lda, const bf16* Bt, int ldb, float (*acc)[NT][4]) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            const bf16* ar = A + (mt * 16) * lda + kt * 16;
            const uint32_t a[4] = {ld32(ar + g * lda + 2 * t), ld32(ar + (g + 8) * lda + 2 * t),
                                   ld32(ar + g * lda + 2 * t + 8), ld32(ar + (g + 8) * lda + 2 * t + 8)};
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const bf16* br = Bt + (nt * 8 + g) * ldb + kt * 16;
                const uint32_t b[2] = {ld32(br + 2 * t), ld32(br + 2 * t + 8)};
                mma_bf16(acc[mt][nt], a, b);
            }
        }
    }
}

template <int MT, int NT>
__device__ __forceinline__ void zero(float (*acc)[NT][4]) {
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = acc[mt][nt][2] = acc[mt][nt][3] = 0.f;
}

// Fragment element e of tile (mt, nt): row and column in the [16 MT][8 NT] result.
__device__ __forceinline__ int frag_row(int mt, int e) { return mt * 16 + ((threadIdx.x & 31) >> 2) + (e >= 2 ? 8 : 0); }
__device__ __forceinline__ int frag_col(int nt, int e) { return nt * 8 + 2 * (threadIdx.x & 3) + (e & 1); }

__device__ __forceinline__ float silu_grad(float z) {
    const float s = sigmoid(z);
    return s * (1.0f + z * (1.0f - s));
}

// Column sums of a [32][8 NT] fragment set over the warp's 32 rows.
template <int NT>
__device__ __forceinline__ void add_column_sums(float (*acc)[NT][4], float* dst, int n_valid_cols) {
    const int t = threadIdx.x & 3;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            float s = acc[0][nt][j] + acc[0][nt][j + 2] + acc[1][nt][j] + acc[1][nt][j + 2];
            s += __shfl_xor_sync(0xffffffffu, s, 4);
            s += __shfl_xor_sync(0xffffffffu, s, 8);
            s += __shfl_xor_sync(0xffffffffu, s, 16);
            const int col = nt * 8 + 2 * t + j;
            if ((threadIdx.x & 31) < 4 && col < n_valid_cols) atomicAdd(dst + col, s);
        }
    }
}

__device__ __forceinline__ void load_feature_tile(WarpBuf& wb, const float* features, const float* labels,
                                                  const uint32_t* index, uint64_t first, uint64_t n, float* y,
                                                  bool* valid) {
    const int lane = threadIdx.x & 31;
    const uint64_t s = first + lane;
    *valid = s < n;
    const uint64_t src = *valid ? (index ? index[s] : s) : 0;
    float f[kIn];
#pragma unroll
    for (int k = 0; k < kIn; ++k) f[k] = (*valid && k < kFeatures) ? features[src * kFeatures + k] : 0.0f;
    *y = *valid ? labels[src] : 0.0f;
#pragma unroll
    for (int k = 0; k < kIn; ++k) {
        const bf16 v = __float2bfloat16_rn(f[k]);
        wb.x[lane * kIn + k] = v;
        wb.xt[k * 32 + lane] = v;
    }
}

__device__ __forceinline__ void load_train_weights(TrainSmem& sm, const float* params) {
    load_weights(sm.w, params);
    for (int i = threadIdx.x; i < kHidden * kHidden; i += blockDim.x) {
        const int out = i / kHidden, in = i % kHidden;
        sm.w2t[in * kHidden + out] = __float2bfloat16_rn(params[kOffW2 + i]);
    }
    for (int i = threadIdx.x; i < kHidden * 16; i += blockDim.x) {
        const int in = i / 16, out = i % 16;
        sm.w3t[i] = __float2bfloat16_rn(out < kOut ? params[kOffW3 + out * kHidden + in] : 0.0f);
    }
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) sm.gacc[i] = 0.0f;
    if (threadIdx.x == 0) sm.loss = 0.0f;
}

// One block: kWarps x 32 samples of the batch [first, first + count).
__global__ void __launch_bounds__(kWarps * 32) train_kernel(const float* params, const float* features,
                                                            const float* labels, const uint32_t* index,
                                                            uint64_t first, uint64_t count, float inv_batch,
                                                            float* grad, float* loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem& sm = *reinterpret_cast<TrainSmem*>(smem_raw);
    load_train_weights(sm, params);
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    WarpBuf& wb = sm.warp[warp];
    const uint64_t tile = (uint64_t(blockIdx.x) * kWarps + warp) * 32;
    const uint64_t end = first + count;
    if (first + tile < end) {
        float y;
        bool valid;
        load_feature_tile(wb, features, labels, index, first + tile, end, &y, &valid);
        __syncwarp();

        // Layer 1
        float acc[2][8][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[mt][nt][e] = sm.w.b1[frag_col(nt, e)];
        warp_gemm<2, 8, 1>(wb.x, kIn, sm.w.w1, kIn, acc);
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int r = frag_row(mt, e), c = frag_col(nt, e);
                    const float z = acc[mt][nt][e];
                    const bf16 h = __float2bfloat16_rn(silu(z));
                    wb.z1[r * kHidden + c] = z;
                    wb.h1[r * kHidden + c] = h;
                    wb.h1t[c * 32 + r] = h;
                }
        __syncwarp();
        // Layer 2
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[mt][nt][e] = sm.w.b2[frag_col(nt, e)];
        warp_gemm<2, 8, 4>(wb.h1, kHidden, sm.w.w2, kHidden, acc);
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int r = frag_row(mt, e), c = frag_col(nt, e);
                    const float z = acc[mt][nt][e];
                    const bf16 h = __float2bfloat16_rn(silu(z));
                    wb.z2[r * kHidden + c] = z;
                    wb.h2[r * kHidden + c] = h;
                    wb.h2t[c * 32 + r] = h;
                }
        __syncwarp();
        // Layer 3 + loss
        float a3[2][1][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int e = 0; e < 4; ++e) a3[mt][0][e] = sm.w.b3[frag_col(0, e)];
        warp_gemm<2, 1, 4>(wb.h2, kHidden, sm.w.w3, kHidden, a3);
        for (int i = threadIdx.x & 31; i < 32 * 16; i += 32) {
            wb.d3[i] = __float2bfloat16_rn(0.0f);
            wb.d3t[i] = __float2bfloat16_rn(0.0f);
        }
        __syncwarp();
        // column 0 sits in lanes with t == 0
        const int src = 4 * (threadIdx.x & 7);
        const float l0 = __shfl_sync(0xffffffffu, a3[0][0][0], src), l1 = __shfl_sync(0xffffffffu, a3[0][0][2], src);
        const float l2 = __shfl_sync(0xffffffffu, a3[1][0][0], src), l3 = __shfl_sync(0xffffffffu, a3[1][0][2], src);
        const int lane = threadIdx.x & 31;
        const float logit = (lane >> 4) == 0 ? (((lane >> 3) & 1) ? l1 : l0) : (((lane >> 3) & 1) ? l3 : l2);
        const float p = sigmoid(logit);
        const float dz = valid ? (p - y) * inv_batch : 0.0f;
        // binary cross-entropy with logits: softplus(l) - y l
        const float lsp = logit > 0 ? logit + log1pf(__expf(-logit)) : log1pf(__expf(logit));
        float lsum = valid ? (lsp - y * logit) * inv_batch : 0.0f;
        float db3 = dz;
        for (int o = 16; o > 0; o >>= 1) {
            lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
            db3 += __shfl_xor_sync(0xffffffffu, db3, o);
        }
        if (lane == 0) {
            atomicAdd(&sm.loss, lsum);
            atomicAdd(&sm.gacc[kOffB3], db3);
        }
        wb.d3[lane * 16] = __float2bfloat16_rn(dz);
        wb.d3t[lane] = __float2bfloat16_rn(dz);
        __syncwarp();

        // dW3 (row 0) = dz3^T h2
        {
            float g3[1][8][4];
            zero<1, 8>(g3);
            warp_gemm<1, 8, 2>(wb.d3t, 32, wb.h2t, 32, g3);
#pragma unroll
            for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int r = frag_row(0, e), c = frag_col(nt, e);
                    if (r < kOut) atomicAdd(&sm.gacc[kOffW3 + r * kHidden + c], g3[0][nt][e]);
                }
        }
        // dh2 = dz3 W3 ; dz2 = dh2 * silu'(z2)
        zero<2, 8>(acc);
        warp_gemm<2, 8, 1>(wb.d3, 16, sm.w3t, 16, acc);
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int r = frag_row(mt, e), c = frag_col(nt, e);
                    const float d = acc[mt][nt][e] * silu_grad(wb.z2[r * kHidden + c]);
                    acc[mt][nt][e] = d;
                    const bf16 db = __float2bfloat16_rn(d);
                    wb.d2[r * kHidden + c] = db;
                    wb.d2t[c * 32 + r] = db;
                }
        add_column_sums<8>(acc, sm.gacc + kOffB2, kHidden);
        __syncwarp();
        // dW2 = dz2^T h1
        {
            float g2[4][8][4];
            zero<4, 8>(g2);
            warp_gemm<4, 8, 2>(wb.d2t, 32, wb.h1t, 32, g2);
#pragma unroll
            for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        atomicAdd(&sm.gacc[kOffW2 + frag_row(mt, e) * kHidden + frag_col(nt, e)], g2[mt][nt][e]);
        }
        // dh1 = dz2 W2 ; dz1 = dh1 * silu'(z1)
        zero<2, 8>(acc);
        warp_gemm<2, 8, 4>(wb.d2, kHidden, sm.w2t, kHidden, acc);
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int r = frag_row(mt, e), c = frag_col(nt, e);
                    const float d = acc[mt][nt][e] * silu_grad(wb.z1[r * kHidden + c]);
                    acc[mt][nt][e] = d;
                    wb.d1t[c * 32 + r] = __float2bfloat16_rn(d);
                }
        add_column_sums<8>(acc, sm.gacc + kOffB1, kHidden);
        __syncwarp();
        // dW1 = dz1^T x
        {
            float g1[4][2][4];
            zero<4, 2>(g1);
            warp_gemm<4, 2, 2>(wb.d1t, 32, wb.xt, 32, g1);
#pragma unroll
            for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                for (int nt = 0; nt < 2; ++nt)
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int c = frag_col(nt, e);
                        if (c < kFeatures) atomicAdd(&sm.gacc[kOffW1 + frag_row(mt, e) * kIn + c], g1[mt][nt][e]);
                    }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kParams; i += blockDim.x)
        if (sm.gacc[i] != 0.0f) atomicAdd(grad + i, sm.gacc[i]);
    if (threadIdx.x == 0 && loss) atomicAdd(loss, sm.loss);
}

__global__ void adam_kernel(float* params, const float* grad, float* m, float* v, float lr, float beta1, float beta2,
                            float eps, float bias1, float bias2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const float g = grad[i];
    const float mi = beta1 * m[i] + (1 - beta1) * g;
    const float vi = beta2 * v[i] + (1 - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    params[i] -= lr * (mi / bias1) / (sqrtf(vi / bias2) + eps);
}

// Probability for each of n feature rows.
__global__ void __launch_bounds__(128) predict_kernel(const float* params, const float* features, uint64_t n,
                                                      float* out) {
    __shared__ Weights w;
    __shared__ __align__(16) bf16 xs[4][32 * kIn];
    load_weights(w, params);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (uint64_t base = (uint64_t(blockIdx.x) * 4 + warp) * 32; base < n; base += uint64_t(gridDim.x) * 4 * 32) {
        const uint64_t s = base + lane;
#pragma unroll
        for (int k = 0; k < kIn; ++k)
            xs[warp][lane * kIn + k] = __float2bfloat16_rn((s < n && k < kFeatures) ? features[s * kFeatures + k] : 0.0f);
        __syncwarp();
        const float logit = warp_forward(w, xs[warp]);
        if (s < n) out[s] = sigmoid(logit);
        __syncwarp();
    }
}

}  // namespace

size_t train_smem_bytes() { return sizeof(TrainSmem); }

cudaError_t launch_train(const float* params, const float* features, const float* labels, const uint32_t* index,
                         uint64_t first, uint64_t count, float inv_batch, float* grad, float* loss, cudaStream_t s) {
    static bool configured = false;
    if (!configured) {
        const cudaError_t e = cudaFuncSetAttribute(train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   int(sizeof(TrainSmem)));
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const uint64_t blocks = (count + kWarps * 32 - 1) / (kWarps * 32);
    train_kernel<<<unsigned(blocks), kWarps * 32, sizeof(TrainSmem), s>>>(params, features, labels, index, first,
                                                                           count, inv_batch, grad, loss);
    return cudaGetLastError();
}

cudaError_t launch_adam(float* params, const float* grad, float* m, float* v, float lr, float beta1, float beta2,
                        float eps, int step, cudaStream_t s) {
    const float bias1 = 1.0f - powf(beta1, float(step));
    const float bias2 = 1.0f - powf(beta2, float(step));
    adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(params, grad, m, v, lr, beta1, beta2, eps, bias1, bias2);
    return cudaGetLastError();
}

cudaError_t launch_predict(const float* params, const float* features, uint64_t n, float* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    uint64_t blocks = (n + 127) / 128;
    if (blocks > 4096) blocks = 4096;
    predict_kernel<<<unsigned(blocks), 128, 0, s>>>(params, features, n, out);
    return cudaGetLastError();
}

}  // namespace mlp
}  // namespace nbx
