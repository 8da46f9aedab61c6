// Escape-probability network: MLP 6 -> 64 -> 64 -> 1, SiLU hidden
// activations, sigmoid output; BF16 weights and activations on the tensor
// cores (mma.sync m16n8k16, FP32 accumulation).  The network has no
// counterpart in the reference; it is only the importance function of the
// unbiased weighted roulette / splitting in the transport kernel.
//
// Parameters, row-major [out][in], inputs padded to 16 and the output to 8
// (padding entries stay zero: their gradients are zero by construction):
//   W1[64][16] b1[64]  W2[64][64] b2[64]  W3[8][64] b3[8]
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace nbx {
namespace mlp {

constexpr int kFeatures = 6;
constexpr int kIn = 16;
constexpr int kHidden = 64;
constexpr int kOut = 8;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kHidden * kIn;
constexpr int kOffW2 = kOffB1 + kHidden;
constexpr int kOffB2 = kOffW2 + kHidden * kHidden;
constexpr int kOffW3 = kOffB2 + kHidden;
constexpr int kOffB3 = kOffW3 + kOut * kHidden;
constexpr int kParams = kOffB3 + kOut;   // 5768

// Weights as the kernels read them (shared memory image).
struct Weights {
    __nv_bfloat16 w1[kHidden * kIn];
    __nv_bfloat16 w2[kHidden * kHidden];
    __nv_bfloat16 w3[kOut * kHidden];
    float b1[kHidden];
    float b2[kHidden];
    float b3[kOut];
};

#ifdef __CUDACC__
__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ float silu(float x) { return __fdividef(x, 1.0f + __expf(-x)); }
__device__ __forceinline__ float sigmoid(float x) { return __fdividef(1.0f, 1.0f + __expf(-x)); }

// Cooperative load of the FP32 master parameters into the shared BF16 image.
__device__ __forceinline__ void load_weights(Weights& w, const float* params) {
    for (int i = threadIdx.x; i < kHidden * kIn; i += blockDim.x) w.w1[i] = __float2bfloat16_rn(params[kOffW1 + i]);
    for (int i = threadIdx.x; i < kHidden * kHidden; i += blockDim.x) w.w2[i] = __float2bfloat16_rn(params[kOffW2 + i]);
    for (int i = threadIdx.x; i < kOut * kHidden; i += blockDim.x) w.w3[i] = __float2bfloat16_rn(params[kOffW3 + i]);
    for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
        w.b1[i] = params[kOffB1 + i];
        w.b2[i] = params[kOffB2 + i];
    }
    for (int i = threadIdx.x; i < kOut; i += blockDim.x) w.b3[i] = params[kOffB3 + i];
}

// Forward pass of one warp over 16 * NMT rows (NMT = 1 or 2 m-tiles): xs is
// the warp's [16 * NMT][16] BF16 feature tile in shared memory.  Returns the
// logit of row (lane mod 16 * NMT) to each lane, so with NMT = 2 lane r gets
// row r.  Processes the m-tiles one after the other and streams layer 2's
// output tiles straight into layer 3, so at most one m-tile of hidden
// activations is live (as packed BF16 A fragments).
template <int NMT>
__device__ __forceinline__ float warp_forward_rows(const Weights& w, const __nv_bfloat16* xs) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    float logit_lo[NMT], logit_hi[NMT];
#pragma unroll
    for (int mt = 0; mt < NMT; ++mt) {
        const __nv_bfloat16* xr = xs + (mt * 16) * kIn;
        uint32_t a[4];
        a[0] = ld32(xr + g * kIn + 2 * t);
        a[1] = ld32(xr + (g + 8) * kIn + 2 * t);
        a[2] = ld32(xr + g * kIn + 2 * t + 8);
        a[3] = ld32(xr + (g + 8) * kIn + 2 * t + 8);
        // Layer 1 -> packed BF16 A fragments of layer 2 (4 k-tiles).
        uint32_t h1[4][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float c[4] = {w.b1[nt * 8 + 2 * t], w.b1[nt * 8 + 2 * t + 1], w.b1[nt * 8 + 2 * t], w.b1[nt * 8 + 2 * t + 1]};
            const uint32_t b[2] = {ld32(w.w1 + (nt * 8 + g) * kIn + 2 * t), ld32(w.w1 + (nt * 8 + g) * kIn + 2 * t + 8)};
            mma_bf16(c, a, b);
            const int kt = nt >> 1, half = nt & 1;
            h1[kt][half * 2 + 0] = pack_bf16(silu(c[0]), silu(c[1]));
            h1[kt][half * 2 + 1] = pack_bf16(silu(c[2]), silu(c[3]));
        }
        // A fragment order is (row g | k 2t), (row g+8 | k 2t), (row g | k 2t+8), (row g+8 | k 2t+8).
        // Layer 2 n-tiles, two at a time, streamed into layer 3.
        float c3[4] = {w.b3[2 * t], w.b3[2 * t + 1], w.b3[2 * t], w.b3[2 * t + 1]};
#pragma unroll
        for (int kt3 = 0; kt3 < 4; ++kt3) {
            uint32_t a3[4];
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int nt = 2 * kt3 + half;
                float c[4] = {w.b2[nt * 8 + 2 * t], w.b2[nt * 8 + 2 * t + 1], w.b2[nt * 8 + 2 * t], w.b2[nt * 8 + 2 * t + 1]};
#pragma unroll
                for (int kt = 0; kt < 4; ++kt) {
                    const uint32_t af[4] = {h1[kt][0], h1[kt][1], h1[kt][2], h1[kt][3]};
                    const uint32_t b[2] = {ld32(w.w2 + (nt * 8 + g) * kHidden + kt * 16 + 2 * t),
                                           ld32(w.w2 + (nt * 8 + g) * kHidden + kt * 16 + 2 * t + 8)};
                    mma_bf16(c, af, b);
                }
                a3[half * 2 + 0] = pack_bf16(silu(c[0]), silu(c[1]));
                a3[half * 2 + 1] = pack_bf16(silu(c[2]), silu(c[3]));
            }
            const uint32_t af3[4] = {a3[0], a3[1], a3[2], a3[3]};
            const uint32_t b[2] = {ld32(w.w3 + g * kHidden + kt3 * 16 + 2 * t), ld32(w.w3 + g * kHidden + kt3 * 16 + 2 * t + 8)};
            mma_bf16(c3, af3, b);
        }
        // Output column 0 lives in lanes with t == 0: c3[0] row g, c3[2] row g+8.
        logit_lo[mt] = c3[0];
        logit_hi[mt] = c3[2];
    }
    // Deliver row r from lane 4 * (r % 8): rows g and g + 8 of m-tile mt sit
    // in lane 4 g (t == 0) as logit_lo[mt] and logit_hi[mt].
    const int src = 4 * (lane & 7);
    const int hi = (lane >> 3) & 1;
    const float v0 = __shfl_sync(0xffffffffu, logit_lo[0], src);
    const float v1 = __shfl_sync(0xffffffffu, logit_hi[0], src);
    if constexpr (NMT == 1) {
        return hi ? v1 : v0;
    } else {
        const float v2 = __shfl_sync(0xffffffffu, logit_lo[1], src);
        const float v3 = __shfl_sync(0xffffffffu, logit_hi[1], src);
        return (lane >> 4) == 0 ? (hi ? v1 : v0) : (hi ? v3 : v2);
    }
}

// All 32 rows of the warp's [32][16] tile; lane r gets row r's logit.
__device__ __forceinline__ float warp_forward(const Weights& w, const __nv_bfloat16* xs) {
    return warp_forward_rows<2>(w, xs);
}
#endif

}  // namespace mlp
}  // namespace nbx
