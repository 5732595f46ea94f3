#pragma once
/*
 * bh_surrogate_api.h -- C-ABI of the learned lensing surrogate in libbh.so
 * (an extension: the reference renderer has no learned component).
 *
 * A small MLP predicts, per pixel, the outcome class of the ray (escaped
 * without touching the disk / captured without touching the disk / touched
 * the disk), its escape direction and its disk-hit radius and redshift.  Its
 * dense layers run on the B200 tensor cores (tcgen05, BF16 operands, FP32
 * accumulation in tensor memory); it is trained on the GPU, on rays the RK4
 * tracer of this library generates, by the library's own forward and backward
 * kernels.  Pixels the network is not sure of, pixels near the critical curve
 * and disk pixels are traced by the RK4 tracer.
 *
 * Conventions as in bh_launch.h: device buffers, asynchronous on `stream`
 * unless stated, the return value is the launch status.
 */
#include <cuda_runtime_api.h>
#include "bh_render_params.h"

#ifdef __cplusplus
extern "C" {
#endif

/* C (=|+=) A . B^T (+ bias): A is M x K, B is N x K, both row-major BF16
 * (leading dimensions lda / ldb elements, multiples of 8, 16-byte-aligned
 * bases); C is M x N row-major FP32 (ldc).  K must be a multiple of 64 and
 * `splits` must divide K / 64: with splits > 1 (split-K) or accumulate != 0
 * the tile results are added to C with atomics, otherwise stored; `bias`
 * (N floats, may be null) is added once.  One 128 x min(N, 256) tile per CTA,
 * TMA-fed, tcgen05.mma into tensor memory.  Internal waits are bounded: a
 * time-out sets a flag read by bhTcErrorFlags. */
cudaError_t bhTcGemm(const void* A, int lda, const void* B, int ldb, float* C, int ldc, int M, int N, int K,
                     int splits, int accumulate, const float* bias, cudaStream_t stream);

/* Reads and clears the tensor-core kernels' error flags (blocking): bit 0 =
 * a bounded wait inside a kernel timed out (its results are invalid). */
cudaError_t bhTcErrorFlags(unsigned* flags);

#ifdef __cplusplus
}
#endif
