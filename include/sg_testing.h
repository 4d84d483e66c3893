/*
 * sg_testing.h -- test hooks of libsuguru_b200.  Not part of the drop-in
 * boundary of sg_coupling.h and without a counterpart in the reference: they
 * exist so that tests can check single kernels against numpy.
 */
#ifndef SG_TESTING_H
#define SG_TESTING_H
#ifdef __cplusplus
extern "C" {
#endif

/* One batched Legendre contraction, as the coupling step runs it:
 *   D[m][q][j] = sum_k A[m][q][k] * B[m][j][k]   (k >= m only when tri != 0)
 * for m < M, q < Q, j < J, k < K, on the current device.  tensor_cores = 1
 * runs the tcgen05 BF16x3 kernel of the mixed path, 0 the FP32 CUDA-core
 * kernel.  A, D are host FP32 arrays, B host FP64 (split to bf16 hi/lo for
 * the tensor cores).  Returns 0, 5 (bad argument), 2 (CUDA error) or 3 (a
 * completion wait timed out). */
int sg_test_legendre(int tensor_cores, int M, int Q, int J, int K, int tri, const double* B,
                     const float* A, float* D);

#ifdef __cplusplus
}
#endif
#endif
