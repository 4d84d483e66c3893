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
 * or 3 runs the tcgen05 kernel of the mixed path in BF16x3, 6 in BF16x6, on
 * 128-row tiles; 103 and 106 the same on 64-row tiles; 0 the FP32 CUDA-core
 * kernel.  A, D are host FP32 arrays, B host FP64 (split
 * to bf16 parts for the tensor cores).  Returns 0, 5 (bad argument), 2 (CUDA
 * error) or 3 (the kernel raised its error flag). */
int sg_test_legendre(int tensor_cores, int M, int Q, int J, int K, int tri, const double* B,
                     const float* A, float* D);

/* One dense product of the surrogate network (sg_gemm.cu) on host data:
 *   C = alpha A B^T (+ bias[n]) (then GELU if gelu != 0), A [M][K], B [N][K],
 * K a multiple of 64.  split = 0: A, B are bf16 bit patterns (uint16);
 * split = 1: A, B are FP32 and run as BF16x3.  Optional outputs (may be
 * NULL): Cpre the FP32 value before GELU, Cb the bf16 result [M][N], CbT the
 * bf16 result transposed [N][M].  splitk != 0 gives the kernel a workspace
 * so that outputs of few tiles are computed in K slices and summed in order.
 * Returns 0, 5, 2 or 3 as above. */
int sg_test_gemm(int split, int M, int N, int K, const void* A, const void* B, const float* bias,
                 int gelu, float alpha, float* C, float* Cpre, unsigned short* Cb, unsigned short* CbT,
                 int splitk);

/* One forward and backward pass of the surrogate network's kernels with
 * given parameters (FP32, in the order W1 [dh][din], b1, W2 [dh][dh], b2,
 * W3 [dout][dh], b3), input rows X [B][din] (already normalised) and targets
 * T [B][dout]: loss = mean((yhat - T)^2) and its gradients (same layout as
 * params).  Dimensions and B are multiples of 64.  Returns 0, 5, 2 or 3. */
int sg_test_mlp_grad(int din, int dh, int dout, int B, const float* params, const float* X,
                     const float* T, float* loss, float* grads);

#ifdef __cplusplus
}
#endif
#endif
