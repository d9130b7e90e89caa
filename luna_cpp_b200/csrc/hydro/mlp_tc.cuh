// The learned limiter's forward pass on the 5th-generation tensor cores (tcgen05): one CTA of 4 warps takes tiles of
// 128 rows; each layer is D[128][N] = A[128][K] B[N][K]^T with BF16 operands in shared memory and FP32 accumulators in
// tensor memory (TMEM), issued by one thread; the 4 warps read their 32 TMEM lanes back, add the bias and apply ReLU,
// and write the next layer's BF16 operand. Same network and parameter layout as mlp.cuh.
//
// Shared-memory operands are K-major without swizzle: 8-row x 16-byte core matrices, row r and column k of an R x K
// matrix at byte ((r / 8) * (K / 8) + k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2. One MMA covers K = 16: its descriptor
// starts at the core matrix of column 16 s, the two core matrices along K are 128 B apart (leading byte offset) and the
// 8-row groups K / 8 * 128 B apart (stride byte offset).
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

#include "mlp.cuh"

namespace luna {
namespace mlp {

constexpr int kTcRows = 128;       // rows of a tile: the MMA's M
constexpr int kTcCols = 128;       // TMEM columns a CTA holds: D1 (and D3) at 0, D2 at 64
constexpr int kTcWaitLimit = 1 << 22;  // mbarrier polls before a wait gives up (an error bit, not a hang); the
                                       // default of the per-launch limit of the first waits (set_wait_limit), and
                                       // always the bound of the last wait before TMEM is freed
constexpr unsigned long long kTcTimeoutBit = 16ull;

struct __align__(128) SmemTc {
    __nv_bfloat16 x[kTcRows * kIn];        // layer 1's A
    __nv_bfloat16 h1[kTcRows * kHidden];   // layer 2's A
    __nv_bfloat16 h2[kTcRows * kHidden];   // layer 3's A
    __nv_bfloat16 w1[kHidden * kIn];       // layer 1's B: W1[n][k]
    __nv_bfloat16 w2[kHidden * kHidden];
    __nv_bfloat16 w3[kOut * kHidden];
    float b1[kHidden], b2[kHidden], b3[kOut];
    unsigned long long mbar;               // MMA completion
    uint32_t tmem;                         // the allocated TMEM address
    int failed;                            // a wait gave up
};

__host__ __device__ constexpr uint32_t core_offset(int r, int k, int K) {
    return static_cast<uint32_t>(((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// The instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B (bits 7-9, 10-12 = 1), both
// K-major (bits 15, 16 = 0), N / 8 at bit 17, M / 16 at bit 24.
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

// A shared-memory matrix descriptor (no swizzle): start, leading and stride byte offsets in 16-B units, version 1.
__host__ __device__ constexpr uint64_t tc_sdesc(uint32_t start_bytes, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    return static_cast<uint64_t>((start_bytes >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo_bytes >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// The descriptor of K-slice s (columns 16 s .. 16 s + 15) of an R x K core-matrix operand at shared address base.
__device__ __forceinline__ uint64_t tc_operand(uint32_t base, int s, int K) {
    return tc_sdesc(base + static_cast<uint32_t>(s) * 256u, 128u, static_cast<uint32_t>(K >> 3) * 128u);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate ? 1u : 0u)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t"
        "}"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    return done != 0;
}

// 16 consecutive FP32 columns of this warp's 32 TMEM lanes (one lane a thread).
__device__ __forceinline__ void tc_load16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]),
          "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = __uint_as_float(r[c]);
}

// Waits for the MMA completion of this phase, polling at most `limit` times; every thread sees the same outcome.
__device__ __forceinline__ bool tc_wait(SmemTc& s, uint32_t parity, int limit) {
    const uint32_t mbar = smem_addr(&s.mbar);
    bool ok = false;
    for (int it = 0; it < limit && !ok; ++it) ok = mbar_try_wait(mbar, parity);
    if (!ok) s.failed = 1;
    __syncthreads();
    return s.failed == 0;
}

// Bias, ReLU and BF16 of this thread's row of a 64-wide layer (columns col0 .. col0 + 63 of TMEM), written as the next
// layer's A operand.
__device__ __forceinline__ void tc_hidden_epilogue(uint32_t tbase, int col0, const float* bias, __nv_bfloat16* out, int row) {
    const int warp = static_cast<int>(threadIdx.x >> 5);
    const uint32_t taddr = tbase + (static_cast<uint32_t>(32 * warp) << 16) + static_cast<uint32_t>(col0);
    float v[kHidden];
#pragma unroll
    for (int c = 0; c < kHidden; c += 16) tc_load16(taddr + static_cast<uint32_t>(c), v + c);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int kc = 0; kc < kHidden / 8; ++kc) {
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int c = 8 * kc + 2 * q;
            w[q] = pack_bf16(fmaxf(v[c] + bias[c], 0.0f), fmaxf(v[c + 1] + bias[c + 1], 0.0f));
        }
        uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<char*>(out) + core_offset(row, 8 * kc, kHidden));
        *dst = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// logits [n][16] of feature rows [n][32] (BF16). A grid-stride loop over tiles of 128 rows; 128 threads; dynamic shared
// memory sizeof(SmemTc). rows (device, may be null): the rows are the first min(n, *rows), a count the previous launch on
// the stream wrote; a CTA with no tile returns before it stages weights or allocates TMEM. error: bit kTcTimeoutBit
// when a wait gave up after wait_limit polls (the CTA then stops, waits for the MMA it issued with the full bound
// kTcWaitLimit, and frees its TMEM: TMEM is never freed under an MMA in flight).
static __global__ void __launch_bounds__(128, 1) k_mlp_forward_tc(const float* __restrict__ params, const __nv_bfloat16* __restrict__ x, int n,
                                                                  const unsigned int* __restrict__ rows, float* __restrict__ logits,
                                                                  unsigned long long* __restrict__ error, int wait_limit) {
    extern __shared__ __align__(128) unsigned char tc_smem[];
    SmemTc& s = *reinterpret_cast<SmemTc*>(tc_smem);
    const int tid = static_cast<int>(threadIdx.x), warp = tid >> 5;
    if (rows) n = min(n, static_cast<int>(*rows));
    if (static_cast<int>(blockIdx.x) * kTcRows >= n) return;  // the same for every thread of the CTA
    // weights as BF16 operands, biases as FP32
    for (int i = tid; i < kHidden * kIn; i += blockDim.x)
        *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(s.w1) + core_offset(i / kIn, i % kIn, kIn)) = __float2bfloat16_rn(params[kW1 + i]);
    for (int i = tid; i < kHidden * kHidden; i += blockDim.x)
        *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(s.w2) + core_offset(i / kHidden, i % kHidden, kHidden)) =
            __float2bfloat16_rn(params[kW2 + i]);
    for (int i = tid; i < kOut * kHidden; i += blockDim.x)
        *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(s.w3) + core_offset(i / kHidden, i % kHidden, kHidden)) =
            __float2bfloat16_rn(params[kW3 + i]);
    for (int i = tid; i < kHidden; i += blockDim.x) {
        s.b1[i] = params[kB1 + i];
        s.b2[i] = params[kB2 + i];
    }
    for (int i = tid; i < kOut; i += blockDim.x) s.b3[i] = params[kB3 + i];
    if (tid == 0) {
        s.failed = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&s.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {  // TMEM for the three accumulators
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s.tmem)), "r"(kTcCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = s.tmem;
    const uint32_t ax = smem_addr(s.x), ah1 = smem_addr(s.h1), ah2 = smem_addr(s.h2);
    const uint32_t aw1 = smem_addr(s.w1), aw2 = smem_addr(s.w2), aw3 = smem_addr(s.w3);
    uint32_t parity = 0;
    bool ok = true;
    for (int row0 = static_cast<int>(blockIdx.x) * kTcRows; row0 < n && ok; row0 += static_cast<int>(gridDim.x) * kTcRows) {
        const int row = row0 + tid;  // this thread's row: TMEM lane tid (warp w reads lanes 32 w .. 32 w + 31)
        {  // layer 1's A: the row's 32 features (64 B) as four 16-B pieces
            uint4 piece[kIn / 8];
#pragma unroll
            for (int kc = 0; kc < kIn / 8; ++kc)
                piece[kc] = row < n ? *reinterpret_cast<const uint4*>(x + static_cast<int64_t>(row) * kIn + 8 * kc) : make_uint4(0, 0, 0, 0);
#pragma unroll
            for (int kc = 0; kc < kIn / 8; ++kc)
                *reinterpret_cast<uint4*>(reinterpret_cast<char*>(s.x) + core_offset(tid, 8 * kc, kIn)) = piece[kc];
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the operands, visible to the tensor cores
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {  // layer 1: D1 = X W1^T (K = 32: two MMAs)
#pragma unroll
            for (int k = 0; k < kIn / 16; ++k) tc_mma(tbase, tc_operand(ax, k, kIn), tc_operand(aw1, k, kIn), tc_idesc(kTcRows, kHidden), k > 0);
            tc_commit(smem_addr(&s.mbar));
        }
        if (!tc_wait(s, parity, wait_limit)) {
            ok = false;
            break;
        }
        parity ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        tc_hidden_epilogue(tbase, 0, s.b1, s.h1, tid);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {  // layer 2: D2 = H1 W2^T (K = 64)
#pragma unroll
            for (int k = 0; k < kHidden / 16; ++k)
                tc_mma(tbase + 64u, tc_operand(ah1, k, kHidden), tc_operand(aw2, k, kHidden), tc_idesc(kTcRows, kHidden), k > 0);
            tc_commit(smem_addr(&s.mbar));
        }
        if (!tc_wait(s, parity, wait_limit)) {
            ok = false;
            break;
        }
        parity ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        tc_hidden_epilogue(tbase, 64, s.b2, s.h2, tid);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {  // layer 3: D3 = H2 W3^T (N = 16), in D1's columns
#pragma unroll
            for (int k = 0; k < kHidden / 16; ++k)
                tc_mma(tbase, tc_operand(ah2, k, kHidden), tc_operand(aw3, k, kHidden), tc_idesc(kTcRows, kOut), k > 0);
            tc_commit(smem_addr(&s.mbar));
        }
        if (!tc_wait(s, parity, wait_limit)) {
            ok = false;
            break;
        }
        parity ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        {
            float v[kOut];
            tc_load16(tbase + (static_cast<uint32_t>(32 * warp) << 16), v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < n) {
                float4* out = reinterpret_cast<float4*>(logits + static_cast<int64_t>(row) * kOut);
#pragma unroll
                for (int c = 0; c < kOut; c += 4) out[c / 4] = make_float4(v[c] + s.b3[c], v[c + 1] + s.b3[c + 1], v[c + 2] + s.b3[c + 2], v[c + 3] + s.b3[c + 3]);
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();  // every lane read D3 before the next tile's layer 1 writes those columns
    }
    if (!ok) {  // a wait gave up: report it, give the MMA in flight one more bounded wait, then free TMEM
        if (tid == 0) atomicOr(error, kTcTimeoutBit);
        const uint32_t mbar = smem_addr(&s.mbar);
        for (int it = 0; it < kTcWaitLimit; ++it)
            if (mbar_try_wait(mbar, parity)) break;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kTcCols) : "memory");
}

}  // namespace mlp
}  // namespace luna
