// ---------------------------------------------------------------------------
// bh_surrogate.h -- internal interfaces of the lensing surrogate (tensor-core
// GEMM, tensor maps, device error word).  The C-ABI is include/bh_surrogate_api.h.
// ---------------------------------------------------------------------------
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

// Tensor map of a row-major BF16 matrix (rows x cols, leading dimension ld
// elements) read in boxes of boxRows x 64 columns with the 128-byte swizzle.
// Requires a 16-byte-aligned base, ld % 8 == 0 and cols % 64 == 0.
cudaError_t bh_tensor_map_bf16(CUtensorMap* map, const void* base, int rows, int cols, int ld, int boxRows);

// C (=|+=) A . B^T (+ bias), A: M x K, B: N x K (BF16, K-major), C: M x N FP32.
// K % 64 == 0; `splits` must divide K / 64 (split-K accumulates with atomics).
// Timed-out waits inside the kernel set bit 0 of *err (device memory).
cudaError_t bh_gemm_bf16(const void* A, int lda, const void* B, int ldb, float* C, int ldc, int M, int N, int K,
                         int splits, bool accumulate, const float* bias, unsigned* err, cudaStream_t s);

// The library's device error word for tensor-core kernels (allocated on first use).
cudaError_t bh_tc_error_word(unsigned** out);
