// The learned limiter's network: a 3-layer MLP of width 64 over 32 per-cell features, 16 outputs (5 used: one slope
// fraction per primitive variable). Weights and activations in BF16 on the tensor cores, FP32 accumulation, FP32 master
// weights. It has no counterpart in the reference.
//
// Layout of the FP32 parameter vector (kParams floats): W1 [64][32], b1 [64], W2 [64][64], b2 [64], W3 [16][64], b3 [16];
// W[n][k] maps input k to output n. Activation: ReLU after layers 1 and 2; the output o is a logit.
//
// Kernels (one warp = 16 rows, m16n8k16 BF16 MMA with FP32 accumulation; the activations of a warp stay in registers
// from layer to layer: the accumulator fragment of one layer is the A fragment of the next):
//   k_mlp_forward   logits [n][16] of feature rows [n][32] (BF16); inference runs forward_tc (tcgen05) instead
//   k_mlp_train     forward + backward of the loss sum_r sum_c w_rc (sigmoid(o_rc) - t_rc)^2 over 64 rows a block,
//                   the block's gradient written to its own slot (deterministic: no atomics)
//   k_mlp_reduce    the slots summed in order, scaled by 1 / sum(w)
//   k_mlp_adam      Adam on the FP32 master weights
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "luna_b200.h"

namespace luna {
namespace mlp {

// The forward pass on the 5th-generation tensor cores (mlp_tc.cuh; defined in learned.cu): logits [n][16] of feature
// rows [n][32] on `stream`; rows (device, may be null): only the first min(n, *rows) rows, a count written earlier on the
// stream; a wait that gives up sets bit 16 of *error.
luna_status forward_tc(const float* params, const __nv_bfloat16* x, int n, const unsigned int* rows, float* logits, unsigned long long* error,
                       cudaStream_t stream);

constexpr int kIn = 32, kHidden = 64, kOut = 16, kUsed = 5;
constexpr int kW1 = 0, kB1 = kW1 + kHidden * kIn, kW2 = kB1 + kHidden, kB2 = kW2 + kHidden * kHidden, kW3 = kB2 + kHidden,
              kB3 = kW3 + kOut * kHidden, kParams = kB3 + kOut;
constexpr int kRowsPerWarp = 16, kWarps = 4, kRowsPerBlock = kRowsPerWarp * kWarps;

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// D = A B + D, A 16x16 (row), B 16x8 (col), BF16 in, FP32 accumulate.
__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// The block's weights in shared memory as BF16, W[n][k] (B fragments of the forward) and W^T[k][n] (of the backward).
struct SmemWeights {
    __nv_bfloat16 w1[kHidden * kIn], w2[kHidden * kHidden], w3[kOut * kHidden];
    __nv_bfloat16 w2t[kHidden * kHidden], w3t[kHidden * kOut];
    float b1[kHidden], b2[kHidden], b3[kOut];
};

__device__ __forceinline__ void load_weights(const float* __restrict__ p, SmemWeights& s, bool transposed) {
    for (int x = threadIdx.x; x < kHidden * kIn; x += blockDim.x) s.w1[x] = __float2bfloat16_rn(p[kW1 + x]);
    for (int x = threadIdx.x; x < kHidden * kHidden; x += blockDim.x) {
        const __nv_bfloat16 v = __float2bfloat16_rn(p[kW2 + x]);
        s.w2[x] = v;
        if (transposed) s.w2t[(x % kHidden) * kHidden + x / kHidden] = v;
    }
    for (int x = threadIdx.x; x < kOut * kHidden; x += blockDim.x) {
        const __nv_bfloat16 v = __float2bfloat16_rn(p[kW3 + x]);
        s.w3[x] = v;
        if (transposed) s.w3t[(x % kHidden) * kOut + x / kHidden] = v;
    }
    for (int x = threadIdx.x; x < kHidden; x += blockDim.x) {
        s.b1[x] = p[kB1 + x];
        s.b2[x] = p[kB2 + x];
    }
    for (int x = threadIdx.x; x < kOut; x += blockDim.x) s.b3[x] = p[kB3 + x];
}

// B fragment (k0..k0+15, n0..n0+7) of a K-contiguous matrix M[n][k] with row length ld.
__device__ __forceinline__ void b_frag(const __nv_bfloat16* m, int ld, int n0, int k0, uint32_t* b) {
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    b[0] = *reinterpret_cast<const uint32_t*>(m + (n0 + gid) * ld + k0 + 2 * tig);
    b[1] = *reinterpret_cast<const uint32_t*>(m + (n0 + gid) * ld + k0 + 8 + 2 * tig);
}

// A fragments of the next layer from the accumulators of this one (16 rows x 8 columns per tile): k-step s takes tiles
// 2s and 2s+1.
template <int Tiles>
__device__ __forceinline__ void acc_to_a(const float (&acc)[Tiles][4], uint32_t (&a)[Tiles / 2][4]) {
#pragma unroll
    for (int s = 0; s < Tiles / 2; ++s) {
        a[s][0] = pack_bf16(acc[2 * s][0], acc[2 * s][1]);
        a[s][1] = pack_bf16(acc[2 * s][2], acc[2 * s][3]);
        a[s][2] = pack_bf16(acc[2 * s + 1][0], acc[2 * s + 1][1]);
        a[s][3] = pack_bf16(acc[2 * s + 1][2], acc[2 * s + 1][3]);
    }
}

// The forward pass of one warp's 16 rows [row0, row0 + 16) from BF16 feature rows. h1, h2: the post-ReLU activations
// (FP32 accumulators), kept for the backward; out: the logits.
__device__ __forceinline__ void forward_warp(const SmemWeights& s, const __nv_bfloat16* __restrict__ x, int n, int row0,
                                             float (&h1)[kHidden / 8][4], float (&h2)[kHidden / 8][4], float (&out)[kOut / 8][4]) {
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const int r0 = row0 + gid, r1 = row0 + gid + 8;
    uint32_t a[kIn / 16][4];
#pragma unroll
    for (int st = 0; st < kIn / 16; ++st) {
        const int k = 16 * st + 2 * tig;
        a[st][0] = r0 < n ? *reinterpret_cast<const uint32_t*>(x + static_cast<int64_t>(r0) * kIn + k) : 0u;
        a[st][1] = r1 < n ? *reinterpret_cast<const uint32_t*>(x + static_cast<int64_t>(r1) * kIn + k) : 0u;
        a[st][2] = r0 < n ? *reinterpret_cast<const uint32_t*>(x + static_cast<int64_t>(r0) * kIn + k + 8) : 0u;
        a[st][3] = r1 < n ? *reinterpret_cast<const uint32_t*>(x + static_cast<int64_t>(r1) * kIn + k + 8) : 0u;
    }
#pragma unroll
    for (int t = 0; t < kHidden / 8; ++t) {
        const float bl = s.b1[8 * t + 2 * tig], bh = s.b1[8 * t + 2 * tig + 1];
        h1[t][0] = bl;
        h1[t][1] = bh;
        h1[t][2] = bl;
        h1[t][3] = bh;
#pragma unroll
        for (int st = 0; st < kIn / 16; ++st) {
            uint32_t b[2];
            b_frag(s.w1, kIn, 8 * t, 16 * st, b);
            mma_bf16(h1[t], a[st], b);
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) h1[t][c] = fmaxf(h1[t][c], 0.0f);
    }
    uint32_t a2[kHidden / 16][4];
    acc_to_a<kHidden / 8>(h1, a2);
#pragma unroll
    for (int t = 0; t < kHidden / 8; ++t) {
        const float bl = s.b2[8 * t + 2 * tig], bh = s.b2[8 * t + 2 * tig + 1];
        h2[t][0] = bl;
        h2[t][1] = bh;
        h2[t][2] = bl;
        h2[t][3] = bh;
#pragma unroll
        for (int st = 0; st < kHidden / 16; ++st) {
            uint32_t b[2];
            b_frag(s.w2, kHidden, 8 * t, 16 * st, b);
            mma_bf16(h2[t], a2[st], b);
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) h2[t][c] = fmaxf(h2[t][c], 0.0f);
    }
    uint32_t a3[kHidden / 16][4];
    acc_to_a<kHidden / 8>(h2, a3);
#pragma unroll
    for (int t = 0; t < kOut / 8; ++t) {
        const float bl = s.b3[8 * t + 2 * tig], bh = s.b3[8 * t + 2 * tig + 1];
        out[t][0] = bl;
        out[t][1] = bh;
        out[t][2] = bl;
        out[t][3] = bh;
#pragma unroll
        for (int st = 0; st < kHidden / 16; ++st) {
            uint32_t b[2];
            b_frag(s.w3, kHidden, 8 * t, 16 * st, b);
            mma_bf16(out[t], a3[st], b);
        }
    }
}

static __global__ void __launch_bounds__(128) k_mlp_forward(const float* __restrict__ params, const __nv_bfloat16* __restrict__ x, int n,
                                                     float* __restrict__ logits) {
    __shared__ SmemWeights s;
    load_weights(params, s, false);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    for (int row0 = (blockIdx.x * kWarps + warp) * kRowsPerWarp; row0 < n; row0 += gridDim.x * kRowsPerBlock) {
        float h1[kHidden / 8][4], h2[kHidden / 8][4], out[kOut / 8][4];
        forward_warp(s, x, n, row0, h1, h2, out);
        const int r0 = row0 + gid, r1 = r0 + 8;
#pragma unroll
        for (int t = 0; t < kOut / 8; ++t) {
            const int c = 8 * t + 2 * tig;
            if (r0 < n) {
                logits[static_cast<int64_t>(r0) * kOut + c] = out[t][0];
                logits[static_cast<int64_t>(r0) * kOut + c + 1] = out[t][1];
            }
            if (r1 < n) {
                logits[static_cast<int64_t>(r1) * kOut + c] = out[t][2];
                logits[static_cast<int64_t>(r1) * kOut + c + 1] = out[t][3];
            }
        }
    }
}

// Per-warp staging for the backward's transposed fragments (row-major tiles of the warp's 16 rows).
struct SmemStage {
    __nv_bfloat16 x[kRowsPerWarp * kIn], h1[kRowsPerWarp * kHidden], h2[kRowsPerWarp * kHidden];
    __nv_bfloat16 dz1[kRowsPerWarp * kHidden], dz2[kRowsPerWarp * kHidden], dout[kRowsPerWarp * kOut];
};

// Stores a warp's accumulator tiles (16 rows x 8 Tiles columns) into a row-major BF16 tile of width Tiles * 8.
template <int Tiles>
__device__ __forceinline__ void stage_acc(const float (&acc)[Tiles][4], __nv_bfloat16* tile) {
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    constexpr int ld = Tiles * 8;
#pragma unroll
    for (int t = 0; t < Tiles; ++t) {
        const int c = 8 * t + 2 * tig;
        *reinterpret_cast<uint32_t*>(tile + gid * ld + c) = pack_bf16(acc[t][0], acc[t][1]);
        *reinterpret_cast<uint32_t*>(tile + (gid + 8) * ld + c) = pack_bf16(acc[t][2], acc[t][3]);
    }
}

// The weight gradient tile G[m0..m0+15][n0..n0+7] += sum over the warp's 16 rows of L[r][m] R[r][n]: one MMA with
// K = rows. L: row-major [16][ldl], R: row-major [16][ldr] (both staged).
__device__ __forceinline__ void grad_tile(const __nv_bfloat16* L, int ldl, int m0, const __nv_bfloat16* R, int ldr, int n0, float* acc) {
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    auto pair = [](const __nv_bfloat16* m, int ld, int r, int c) {
        const __nv_bfloat162 v = __halves2bfloat162(m[r * ld + c], m[(r + 1) * ld + c]);
        return *reinterpret_cast<const uint32_t*>(&v);
    };
    uint32_t a[4], b[2];
    // A(m, k = r) = L[r][m0 + m]: a0 rows gid, k 2tig..+1; a1 rows gid+8; a2 k+8; a3 both.
    a[0] = pair(L, ldl, 2 * tig, m0 + gid);
    a[1] = pair(L, ldl, 2 * tig, m0 + gid + 8);
    a[2] = pair(L, ldl, 2 * tig + 8, m0 + gid);
    a[3] = pair(L, ldl, 2 * tig + 8, m0 + gid + 8);
    // B(k = r, n) = R[r][n0 + n]: b0 k 2tig..+1, n gid; b1 k + 8.
    b[0] = pair(R, ldr, 2 * tig, n0 + gid);
    b[1] = pair(R, ldr, 2 * tig + 8, n0 + gid);
    mma_bf16(acc, a, b);
}

// Forward and backward of kRowsPerBlock rows; the block's gradient (FP32, kParams) goes to slot blockIdx.x.
// Rows beyond n or with zero weight add nothing.
struct SmemTrain {
    SmemWeights w;
    SmemStage stage[kWarps];
    float grad[kParams];
    float warp_loss[kWarps];
};

static __global__ void __launch_bounds__(128) k_mlp_train(const float* __restrict__ params, const __nv_bfloat16* __restrict__ x,
                                                   const float* __restrict__ target, const float* __restrict__ weight, int n,
                                                   float* __restrict__ slots, float* __restrict__ loss_slots) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmemTrain& sm = *reinterpret_cast<SmemTrain*>(smem_raw);
    SmemWeights& s = sm.w;
    SmemStage* stage = sm.stage;
    float* grad = sm.grad;
    float* warp_loss = sm.warp_loss;
    load_weights(params, s, true);
    for (int p = threadIdx.x; p < kParams; p += blockDim.x) grad[p] = 0.0f;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const int row0 = (blockIdx.x * kWarps + warp) * kRowsPerWarp;
    float h1[kHidden / 8][4], h2[kHidden / 8][4], out[kOut / 8][4];
    forward_warp(s, x, n, row0, h1, h2, out);
    SmemStage& st = stage[warp];
    // The loss and dL/do = 2 w (sigma - t) sigma (1 - sigma); unused outputs and padded rows have w = 0.
    float dout[kOut / 8][4];
    float loss = 0.0f;
#pragma unroll
    for (int t = 0; t < kOut / 8; ++t)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int col = 8 * t + 2 * tig + (c & 1), row = row0 + gid + (c >> 1) * 8;
            float g = 0.0f;
            if (row < n && col < kUsed) {
                const float w = weight[static_cast<int64_t>(row) * kUsed + col];
                const float sg = 1.0f / (1.0f + __expf(-out[t][c]));
                const float e = sg - target[static_cast<int64_t>(row) * kUsed + col];
                loss += w * e * e;
                g = 2.0f * w * e * sg * (1.0f - sg);
            }
            dout[t][c] = g;
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0) warp_loss[warp] = loss;
    // Input rows (for dW1), activations and output gradient, staged row-major.
    for (int e = lane; e < kRowsPerWarp * kIn; e += 32) {
        const int r = row0 + e / kIn;
        st.x[e] = r < n ? x[static_cast<int64_t>(r) * kIn + e % kIn] : __float2bfloat16_rn(0.0f);
    }
    stage_acc<kHidden / 8>(h1, st.h1);
    stage_acc<kHidden / 8>(h2, st.h2);
    stage_acc<kOut / 8>(dout, st.dout);
    // dH2 = dO W3 (B = W3 as [K = out][N = hidden]: its fragments from W3^T[hidden][out]), dZ2 = dH2 where h2 > 0.
    uint32_t ao[1][4];
    acc_to_a<kOut / 8>(dout, ao);
    float dz2[kHidden / 8][4];
#pragma unroll
    for (int t = 0; t < kHidden / 8; ++t) {
#pragma unroll
        for (int c = 0; c < 4; ++c) dz2[t][c] = 0.0f;
        uint32_t b[2];
        b_frag(s.w3t, kOut, 8 * t, 0, b);
        mma_bf16(dz2[t], ao[0], b);
#pragma unroll
        for (int c = 0; c < 4; ++c) dz2[t][c] = h2[t][c] > 0.0f ? dz2[t][c] : 0.0f;
    }
    stage_acc<kHidden / 8>(dz2, st.dz2);
    // dH1 = dZ2 W2 (fragments from W2^T), dZ1 = dH1 where h1 > 0.
    uint32_t az2[kHidden / 16][4];
    acc_to_a<kHidden / 8>(dz2, az2);
    float dz1[kHidden / 8][4];
#pragma unroll
    for (int t = 0; t < kHidden / 8; ++t) {
#pragma unroll
        for (int c = 0; c < 4; ++c) dz1[t][c] = 0.0f;
#pragma unroll
        for (int sk = 0; sk < kHidden / 16; ++sk) {
            uint32_t b[2];
            b_frag(s.w2t, kHidden, 8 * t, 16 * sk, b);
            mma_bf16(dz1[t], az2[sk], b);
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) dz1[t][c] = h1[t][c] > 0.0f ? dz1[t][c] : 0.0f;
    }
    stage_acc<kHidden / 8>(dz1, st.dz1);
    __syncwarp();
    // The block's weight gradients, one warp after another in a fixed order (the same bits every run).
    for (int w = 0; w < kWarps; ++w) {
        __syncthreads();
        if (warp != w) continue;
        // dW3[o][h] = sum_r dO[r][o] H2[r][h]; dW2[h2][h1] = sum_r dZ2[r][h2] H1[r][h1]; dW1[h1][x] = sum_r dZ1[r][h1] X[r][x].
        for (int t = 0; t < kHidden / 8; ++t) {
            float acc[4] = {0, 0, 0, 0};
            grad_tile(st.dout, kOut, 0, st.h2, kHidden, 8 * t, acc);
            const int col = 8 * t + 2 * tig;
            grad[kW3 + gid * kHidden + col] += acc[0];
            grad[kW3 + gid * kHidden + col + 1] += acc[1];
            grad[kW3 + (gid + 8) * kHidden + col] += acc[2];
            grad[kW3 + (gid + 8) * kHidden + col + 1] += acc[3];
        }
        for (int m = 0; m < kHidden / 16; ++m)
            for (int t = 0; t < kHidden / 8; ++t) {
                float acc[4] = {0, 0, 0, 0};
                grad_tile(st.dz2, kHidden, 16 * m, st.h1, kHidden, 8 * t, acc);
                const int row = 16 * m + gid, col = 8 * t + 2 * tig;
                grad[kW2 + row * kHidden + col] += acc[0];
                grad[kW2 + row * kHidden + col + 1] += acc[1];
                grad[kW2 + (row + 8) * kHidden + col] += acc[2];
                grad[kW2 + (row + 8) * kHidden + col + 1] += acc[3];
            }
        for (int m = 0; m < kHidden / 16; ++m)
            for (int t = 0; t < kIn / 8; ++t) {
                float acc[4] = {0, 0, 0, 0};
                grad_tile(st.dz1, kHidden, 16 * m, st.x, kIn, 8 * t, acc);
                const int row = 16 * m + gid, col = 8 * t + 2 * tig;
                grad[kW1 + row * kIn + col] += acc[0];
                grad[kW1 + row * kIn + col + 1] += acc[1];
                grad[kW1 + (row + 8) * kIn + col] += acc[2];
                grad[kW1 + (row + 8) * kIn + col + 1] += acc[3];
            }
        // Bias gradients: column sums of the staged gradients, in row order.
        for (int c = lane; c < kHidden; c += 32) {
            float a = 0, b = 0;
            for (int r = 0; r < kRowsPerWarp; ++r) {
                a += __bfloat162float(st.dz1[r * kHidden + c]);
                b += __bfloat162float(st.dz2[r * kHidden + c]);
            }
            grad[kB1 + c] += a;
            grad[kB2 + c] += b;
        }
        if (lane < kOut) {
            float a = 0;
            for (int r = 0; r < kRowsPerWarp; ++r) a += __bfloat162float(st.dout[r * kOut + lane]);
            grad[kB3 + lane] += a;
        }
    }
    __syncthreads();
    float* slot = slots + static_cast<int64_t>(blockIdx.x) * kParams;
    for (int p = threadIdx.x; p < kParams; p += blockDim.x) slot[p] = grad[p];
    if (threadIdx.x == 0) loss_slots[blockIdx.x] = warp_loss[0] + warp_loss[1] + warp_loss[2] + warp_loss[3];
}

// g[p] = scale * sum_b slots[b][p] in slot order; loss = scale * sum_b loss_slots[b].
static __global__ void k_mlp_reduce(const float* __restrict__ slots, const float* __restrict__ loss_slots, int blocks, float scale,
                             float* __restrict__ g, float* __restrict__ loss) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kParams) {
        float a = 0;
        for (int b = 0; b < blocks; ++b) a += slots[static_cast<int64_t>(b) * kParams + p];
        g[p] = scale * a;
    }
    if (p == 0) {
        float a = 0;
        for (int b = 0; b < blocks; ++b) a += loss_slots[b];
        *loss = scale * a;
    }
}

// Adam (Kingma and Ba) with bias correction; m, v: the moment estimates; step counts from 1.
static __global__ void k_mlp_adam(float* __restrict__ params, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, float lr,
                           float beta1, float beta2, float eps, int step) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    const float gp = g[p];
    const float mp = beta1 * m[p] + (1.0f - beta1) * gp;
    const float vp = beta2 * v[p] + (1.0f - beta2) * gp * gp;
    m[p] = mp;
    v[p] = vp;
    const float mh = mp / (1.0f - powf(beta1, static_cast<float>(step)));
    const float vh = vp / (1.0f - powf(beta2, static_cast<float>(step)));
    params[p] -= lr * mh / (sqrtf(vh) + eps);
}

}  // namespace mlp
}  // namespace luna
