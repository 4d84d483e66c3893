// sg_legendre.cu -- batched Legendre contractions (the theta half of the
// SPHEREPACK Gauss-grid analysis shagc.f:384-470 and synthesis shsgc.f:329-470)
// on CUDA cores, for the FP64 plain path and as the FP32 fallback.
//
// Each LegWork item is one (problem, m, 32-row tile): the m-th table slice
// B_m[J][K] is staged in shared memory (row stride K+1 to avoid bank
// conflicts), the tile's A rows next to it, and each thread forms dot
// products over K.  Synthesis problems start K at m (coefficients vanish for
// n < m).
#include "sg_common.cuh"
#include "sg_kernels.h"

namespace sg {

constexpr int LEG_QT = 32;

template <class T>
__global__ void __launch_bounds__(256) legendre_kernel(const LegProblem* __restrict__ probs,
                                                       const LegWork* __restrict__ work, int nwork) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if ((int)blockIdx.x >= nwork) return;
  const LegWork wk = work[blockIdx.x];
  const LegProblem P = probs[wk.prob];
  const int m = wk.m, q0 = wk.q0;
  const int nq = min(LEG_QT, P.Q - q0);
  const int K = P.K, J = P.J, Kp = K + 1;
  const int k0 = P.tri ? m : 0;
  T* sB = (T*)smem_raw;       // [J][Kp]
  T* sA = sB + J * Kp;        // [QT][Kp]
  const T* B = (const T*)P.B + (long long)m * P.sBm;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  // warp per row, lanes along K: no integer division by runtime values
  for (int j = warp; j < J; j += nwarp)
    for (int k = lane; k < K; k += 32) sB[j * Kp + k] = B[(long long)j * K + k];
  const T* A = (const T*)P.A;
  for (int q = warp; q < nq; q += nwarp) {
    const int qq = q0 + q, c = qq / P.rpc, r = qq - c * P.rpc;
    const T* arow = A + (long long)c * P.sAc + (long long)r * P.sAr + (long long)m * P.sAm;
    for (int k = lane; k < K; k += 32) sA[q * Kp + k] = arow[k];
  }
  __syncthreads();
  T* D = (T*)P.D;
  for (int q = warp; q < nq; q += nwarp) {
    const int qq = q0 + q, c = qq / P.rpc, r = qq - c * P.rpc;
    T* drow = D + (long long)c * P.sDc + (long long)r * P.sDr + (long long)m * P.sDm;
    const T* a = sA + q * Kp;
    for (int j = lane; j < J; j += 32) {
      const T* b = sB + j * Kp;
      T s = 0;
      for (int k = k0; k < K; ++k) s += a[k] * b[k];
      drow[j] = s;
    }
  }
}

template <class T>
cudaError_t launch_legendre(const LegProblem* d_probs, const LegWork* d_work, int nwork, int maxJ, int maxK,
                            cudaStream_t st) {
  if (nwork <= 0) return cudaSuccess;
  size_t smem = sizeof(T) * (size_t)(maxJ + LEG_QT) * (maxK + 1);
  // the table slice and the row tile must fit the device's opt-in limit
  // (SH degree 31 in FP64: (3*64 + 32) * 33 * 8 = 59 KB); refuse on the host
  // rather than launch with a request the device cannot grant
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  if (smem > (size_t)optin) return cudaErrorInvalidValue;
  e = smem_limit(legendre_kernel<T>, smem);
  if (e != cudaSuccess) return e;
  launch_pdl(legendre_kernel<T>, dim3(nwork), dim3(256), smem, st, d_probs, d_work, nwork);
  return cudaGetLastError();
}

template cudaError_t launch_legendre<double>(const LegProblem*, const LegWork*, int, int, int, cudaStream_t);
template cudaError_t launch_legendre<float>(const LegProblem*, const LegWork*, int, int, int, cudaStream_t);

}  // namespace sg
