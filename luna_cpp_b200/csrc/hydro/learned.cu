// The learned limiter's network entry points (mlp.cuh): inference, one training step's gradient, Adam.

#include <cuda_runtime.h>

#include <string>

#include "luna_b200.h"
#include "mlp.cuh"
#include "mlp_tc.cuh"

namespace luna {
luna_status report_error(luna_status s, const std::string& what);
}  // namespace luna

namespace {

luna_status fail(luna_status s, const std::string& what) { return luna::report_error(s, what); }

luna_status check_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(LUNA_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return LUNA_OK;
}

#ifndef LUNA_MLP_CTAS_PER_SM
#define LUNA_MLP_CTAS_PER_SM 4  // measured at 2.1M rows: 2 CTAs 0.218 ms, 4 CTAs 0.166 ms (mma.sync forward: 0.468)
#endif

// The standalone forward's error word (luna_mlp_forward).
__device__ unsigned long long g_forward_error;

// Polls of an MMA-completion wait before it gives up (luna_mlp_set_wait_limit).
int g_wait_limit = luna::mlp::kTcWaitLimit;

}  // namespace

namespace luna {
namespace mlp {

luna_status forward_tc(const float* params, const __nv_bfloat16* x, int n, const unsigned int* rows, float* logits, unsigned long long* error,
                       cudaStream_t stream) {
    if (n <= 0) return LUNA_OK;
    const int smem = static_cast<int>(sizeof(SmemTc));
    static bool configured = false;
    if (!configured) {
        const cudaError_t e = cudaFuncSetAttribute(k_mlp_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return fail(LUNA_ECUDA, std::string("k_mlp_forward_tc shared memory: ") + cudaGetErrorString(e));
        configured = true;
    }
    // a grid-stride loop over tiles of 128 rows; up to LUNA_MLP_CTAS_PER_SM CTAs an SM hold TMEM (128 of its 512 columns
    // each; 4 fill it)
    const int64_t tiles = (static_cast<int64_t>(n) + kTcRows - 1) / kTcRows;
    const int blocks = static_cast<int>(tiles < 148 * LUNA_MLP_CTAS_PER_SM ? tiles : 148 * LUNA_MLP_CTAS_PER_SM);
    k_mlp_forward_tc<<<blocks, 128, smem, stream>>>(params, x, n, rows, logits, error, g_wait_limit);
    return check_launch("k_mlp_forward_tc");
}

}  // namespace mlp
}  // namespace luna

extern "C" {

LUNA_API int64_t luna_mlp_param_count(void) { return luna::mlp::kParams; }

LUNA_API int luna_mlp_set_wait_limit(int polls) {
    const int previous = g_wait_limit;
    g_wait_limit = polls < 0 ? luna::mlp::kTcWaitLimit : polls;
    return previous;
}

LUNA_API int64_t luna_mlp_train_workspace_floats(int64_t n) {
    const int64_t blocks = (n + luna::mlp::kRowsPerBlock - 1) / luna::mlp::kRowsPerBlock;
    return blocks * (luna::mlp::kParams + 1);
}

LUNA_API luna_status luna_mlp_forward(const float* params, const void* features, int64_t n, float* logits, void* stream) {
    if (!params || !features || !logits || n < 0 || n >= (int64_t(1) << 31)) return fail(LUNA_EINVAL, "luna_mlp_forward: bad argument");
    if (n == 0) return LUNA_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    void* word = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&word, g_forward_error);
    if (e == cudaSuccess) e = cudaMemsetAsync(word, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return fail(LUNA_ECUDA, std::string("luna_mlp_forward error word: ") + cudaGetErrorString(e));
    const luna_status st = luna::mlp::forward_tc(params, static_cast<const __nv_bfloat16*>(features), static_cast<int>(n), nullptr, logits,
                                                 static_cast<unsigned long long*>(word), s);
    if (st != LUNA_OK) return st;
    unsigned long long bits = 0;
    e = cudaMemcpyAsync(&bits, word, sizeof(bits), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(LUNA_ECUDA, std::string("luna_mlp_forward: ") + cudaGetErrorString(e));
    if (bits & luna::mlp::kTcTimeoutBit) return fail(LUNA_ETIMEOUT, "luna_mlp_forward: a tensor-core completion wait gave up");
    return LUNA_OK;
}

LUNA_API luna_status luna_mlp_train_step(const float* params, const void* features, const float* target, const float* weight, int64_t n,
                                         float scale, float* grad, float* loss, float* workspace, int64_t workspace_floats, void* stream) {
    if (!params || !features || !target || !weight || !grad || !loss || !workspace || n <= 0 || n >= (int64_t(1) << 31))
        return fail(LUNA_EINVAL, "luna_mlp_train_step: bad argument");
    const int64_t blocks = (n + luna::mlp::kRowsPerBlock - 1) / luna::mlp::kRowsPerBlock;
    if (workspace_floats < blocks * (luna::mlp::kParams + 1)) return fail(LUNA_EINVAL, "luna_mlp_train_step: workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int smem = static_cast<int>(sizeof(luna::mlp::SmemTrain));
    static bool configured = false;
    if (!configured) {
        const cudaError_t e = cudaFuncSetAttribute(luna::mlp::k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return fail(LUNA_ECUDA, std::string("k_mlp_train shared memory: ") + cudaGetErrorString(e));
        configured = true;
    }
    float* slots = workspace;
    float* loss_slots = workspace + blocks * luna::mlp::kParams;
    luna::mlp::k_mlp_train<<<static_cast<int>(blocks), 128, smem, s>>>(params, static_cast<const __nv_bfloat16*>(features), target, weight,
                                                                      static_cast<int>(n), slots, loss_slots);
    luna_status st = check_launch("k_mlp_train");
    if (st != LUNA_OK) return st;
    luna::mlp::k_mlp_reduce<<<(luna::mlp::kParams + 255) / 256, 256, 0, s>>>(slots, loss_slots, static_cast<int>(blocks), scale, grad, loss);
    return check_launch("k_mlp_reduce");
}

LUNA_API luna_status luna_mlp_adam(float* params, const float* grad, float* m, float* v, float lr, float beta1, float beta2, float eps,
                                   int step, void* stream) {
    if (!params || !grad || !m || !v || step < 1) return fail(LUNA_EINVAL, "luna_mlp_adam: bad argument");
    luna::mlp::k_mlp_adam<<<(luna::mlp::kParams + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(params, grad, m, v, lr, beta1,
                                                                                                            beta2, eps, step);
    return check_launch("k_mlp_adam");
}

}  // extern "C"
