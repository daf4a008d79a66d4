/*
 * sphg_learn.h — the learned particle stepper of libsphg (no counterpart in
 * the reference, whose step is the SPH solver alone): tensor-core (tcgen05)
 * BF16 GEMM used by the message-passing network's forward and backward
 * passes.  Device pointers throughout; errors are sphg_status codes.
 */
#ifndef SPHG_LEARN_H
#define SPHG_LEARN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* C[M x N] = A[M x K] * B[N x K]^T  (accumulate: C += ...).  A and B are
 * row-major bf16 with K contiguous, C row-major fp32; M % 128 == 0,
 * N % 16 == 0, K % 64 == 0, rows 16-byte aligned.  split_k > 1 splits K over
 * CTAs that add into C atomically (C must hold the value to add to).  A
 * device wait that gives up sets *err_dev to 1 (the call still returns). */
int sphg_gemm_bf16_tn(const void* A, const void* B, float* C, int M, int N, int K, int accumulate, int split_k,
                      int* err_dev, void* cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* SPHG_LEARN_H */
