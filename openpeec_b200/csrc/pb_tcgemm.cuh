// pb_tcgemm.cuh — batched complex FP32 trailing update C -= A * B on the sm_100a tensor
// cores (tcgen05.mma kind::f16 on BF16 terms, TMEM accumulators, operands staged by TMA).
#pragma once
#include "pb_common.cuh"

// True when the update (row-major, leading dimensions and batch stride in complex
// elements) meets the TMA alignment rules of the tensor-core kernel: 16-byte aligned base
// pointers, and row and batch strides that are multiples of 16 bytes.
bool pb_cgemm_tc_ok(const float2 *A, int lda, const float2 *B, int ldb, const float2 *C, int ldc,
                    long long stride, int nb);

// C[b] (m x nc) -= A[b] (m x k) * B[b] (k x nc) for b < nb, complex FP32, row-major, all
// three with batch stride `stride` (complex elements). Each FP32 operand is split into
// three BF16 terms carrying all its 24 bits; the six products of significance >= 2^-16
// are accumulated in FP32 (an FP32-accurate product). err: device int, set non-zero when
// a pipeline wait of the kernel times out (the update is then incomplete).
int pb_cgemm_tc(int m, int nc, int k, const float2 *A, int lda, const float2 *B, int ldb,
                float2 *C, int ldc, long long stride, int nb, int *err, cudaStream_t s, int lower = 0);
