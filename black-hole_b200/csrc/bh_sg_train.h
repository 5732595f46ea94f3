// ---------------------------------------------------------------------------
// bh_sg_train.h -- state of the lensing surrogate and its training passes
// (bh_sg_train.cu), used by the C-ABI in bh_sg_api.cpp.
// ---------------------------------------------------------------------------
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include "bh_trace_params.h"

// Flat FP32 parameter vector: for each hidden layer l = 0..3 the 256 x 256
// weight (row = output unit) then its 256 biases; then the 16 x 256 head
// weight and its 16 biases.
struct SgLayout
{
    static constexpr int kHid = 256 * 256 + 256;
    static constexpr __host__ __device__ int w(int l) { return l * kHid; }
    static constexpr __host__ __device__ int b(int l) { return l < 4 ? l * kHid + 256 * 256 : 4 * kHid + 16 * 256; }
    static constexpr __host__ __device__ int count() { return 4 * kHid + 16 * 256 + 16; }
};

struct SgState
{
    int device = 0;
    float* params = nullptr;          // FP32 master copy (SgLayout)
    float* grads = nullptr;
    float* adamM = nullptr;
    float* adamV = nullptr;
    __nv_bfloat16* W = nullptr;       // BF16 W_l (out x in), hidden layers then the 16 x 256 head
    __nv_bfloat16* Wt = nullptr;      // BF16 W_l^T (in x out), hidden layers then the 256 x 64 padded head
    float* biasPacked = nullptr;      // all biases, contiguous (4 x 256 + 16), for the fused kernel
    float* loss = nullptr;            // 8 floats: loss sums of the last batch
    unsigned* err = nullptr;          // tensor-core kernels' error word
    int step = 0;                     // Adam steps taken
    float wEsc = 100.f, wDiskR = 1.f, wDiskG = 1.f, wConf = 0.1f, escTol = 1e-3f;

    // per-batch scratch (capacity `cap` rays)
    int cap = 0;
    void* X[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};   // BF16 n x 256 activations
    float* Z[4] = {nullptr, nullptr, nullptr, nullptr};           // FP32 n x 256 pre-activations
    float* Y = nullptr;               // FP32 n x 16
    void* dY = nullptr;               // BF16 n x 64
    void* dYt = nullptr;              // BF16 128 x n (rows >= 16 zero)
    float* dX = nullptr;              // FP32 n x 256
    void* dZ = nullptr;               // BF16 n x 256
    void* T0 = nullptr;               // BF16 256 x n transposes
    void* T1 = nullptr;
    float* headTmp = nullptr;         // FP32 128 x 256

    // the RK4-traced ray set: inputs (n x 8) and targets (n x 8)
    float* dsIn = nullptr;
    float* dsTgt = nullptr;
    long long dsN = 0;
};

cudaError_t sg_features(const float* in, void* X0, int n, cudaStream_t s);
cudaError_t sg_pack_weights(SgState& S, cudaStream_t s);
// grows the per-batch scratch to n rays; the zero fill is enqueued on s
cudaError_t sg_reserve(SgState& S, int n, cudaStream_t s);
void sg_free_batch(SgState& S);
cudaError_t sg_forward_train(SgState& S, const float* in, int n, cudaStream_t s);
cudaError_t sg_gradients(SgState& S, const float* in, const float* tgt, int n, cudaStream_t s);
cudaError_t sg_adam(SgState& S, float lr, cudaStream_t s);
cudaError_t sg_make_rays(const TraceParams& P, float aN, float qN, float rN, float iN, unsigned seed, float3* dirs,
                         float* in, int R, cudaStream_t s);
cudaError_t sg_make_targets(const void* rec, const TraceParams& P, float* tgt, int R, cudaStream_t s);
cudaError_t sg_gather(const SgState& S, unsigned seed, float* in, float* tgt, int n, cudaStream_t s);
