// sg_gemm.cu -- the dense products of the membrane-force surrogate on the
// tcgen05 tensor cores: C = alpha * A B^T (+ bias, GELU) with A [M][K] and
// B [N][K] both K-major, FP32 accumulation in tensor memory.
//
// Two operand modes:
//  - bf16: A and B are bf16 (the network's weights and activations);
//  - split: A and B are FP32 and are split while staged into bf16 hi/lo, and
//    each K step issues hi.hi + hi.lo + lo.hi (BF16x3, ~16 significant bits),
//    used where the product must be accurate (the linear response layer).
//
// One CTA of 128 threads per 128 x 128 output tile; K advances in slabs of
// 64 through two shared-memory stages, so that the loads of slab k+1 overlap
// the MMAs of slab k (each stage has an mbarrier that the MMA commit arrives
// on; waits are bounded and set an error flag instead of trapping).  The
// epilogue reads the accumulator with tcgen05.ld (warp w owns rows
// 32w..32w+31) and fuses scale, bias, GELU and the stores: FP32, optionally
// the FP32 pre-activation, bf16, and a transposed bf16 copy for the
// weight-gradient products of the backward pass.
#include "sg_common.cuh"
#include "sg_kernels.h"
#include "sg_umma.cuh"

namespace sg {

using namespace umma;

namespace {
constexpr int BM = 128, BN = 128, BK = 64, KC = BK / 8;

// GELU with the exact erf form, 0.5 x (1 + erf(x / sqrt 2)).
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
}  // namespace

template <int SPLIT>
__global__ void __launch_bounds__(128) gemm_kernel(GemmArgs g, int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t s_bar[2];
  __shared__ uint32_t s_tmem;
  constexpr int TILE = BM * BK;                // bf16 elements of one operand tile
  constexpr int STAGE = (SPLIT ? 4 : 2) * TILE;  // A(hi,lo), B(hi,lo)
  uint16_t* smem = (uint16_t*)smem_raw;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  // K slice of this CTA (split-K: blockIdx.z of gridDim.z slices)
  const int nk_all = g.K / BK, nsl = gridDim.z, z = blockIdx.z;
  const int kt0 = (int)((long long)nk_all * z / nsl), kt1 = (int)((long long)nk_all * (z + 1) / nsl);
  const int nk = kt1 - kt0;

  if (warp == 0) tmem_alloc(&s_tmem, 128);
  if (tid == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = s_tmem;
  bool ok = true;

  for (int kt = 0; kt < nk; ++kt) {
    const int s = kt & 1;
    uint16_t* sA = smem + s * STAGE;
    uint16_t* sB = sA + (SPLIT ? 2 : 1) * TILE;
    if (kt >= 2) {  // the MMAs of slab kt-2 have finished reading this stage
      const int waited = mbar_wait(&s_bar[s], (uint32_t)(((kt >> 1) - 1) & 1)) ? 1 : 0;
      if (!__syncthreads_and(waited)) {
        ok = false;
        // give the last committed slab (kt-1) a bounded chance to finish
        // before its accumulator is freed below
        mbar_wait(&s_bar[(kt - 1) & 1], (uint32_t)(((kt - 1) >> 1) & 1));
        break;
      }
    }
    const int k0 = (kt0 + kt) * BK;
    // ---- stage A and B: consecutive threads take consecutive rows of one
    // 8-wide K chunk (conflict-free 16-byte shared stores)
#pragma unroll 2
    for (int idx = tid; idx < BM * KC; idx += 128) {
      const int kc = idx >> 7, r = idx & 127;
#pragma unroll
      for (int op = 0; op < 2; ++op) {
        const int row = (op == 0 ? m0 : n0) + r;
        const int lim = op == 0 ? g.M : g.N;
        uint16_t* dst = op == 0 ? sA : sB;
        const int o = cm_offset(r, kc, KC);
        if (SPLIT) {
          float x[8];
          if (row < lim) {
            const float* src = (const float*)(op == 0 ? g.A : g.B) + (long long)row * (op == 0 ? g.lda : g.ldb) + k0 + 8 * kc;
            const float4 a = *(const float4*)src, b = *(const float4*)(src + 4);
            x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w; x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
          } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) x[i] = 0.f;
          }
          uint4 hi, lo;
          split8(x, hi, lo);
          *(uint4*)(dst + o) = hi;
          *(uint4*)(dst + TILE + o) = lo;
        } else {
          uint4 v = make_uint4(0, 0, 0, 0);
          if (row < lim)
            v = *(const uint4*)((const uint16_t*)(op == 0 ? g.A : g.B) + (long long)row * (op == 0 ? g.lda : g.ldb) +
                                k0 + 8 * kc);
          *(uint4*)(dst + o) = v;
        }
      }
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    if (tid == 0) {
      const uint32_t id = idesc_bf16(BM, BN);
      const uint32_t lbo = 128, sbo = KC * 128;
      const uint32_t aH = smem_u32(sA), bH = smem_u32(sB);
#pragma unroll
      for (int j = 0; j < BK / 16; ++j) {
        const uint32_t o = (uint32_t)j * 256;
        const uint32_t acc = (kt > 0 || j > 0) ? 1u : 0u;
        mma_bf16(tmem, desc(aH + o, lbo, sbo), desc(bH + o, lbo, sbo), id, acc);
        if (SPLIT) {
          const uint32_t aL = aH + TILE * 2, bL = bH + TILE * 2;
          mma_bf16(tmem, desc(aH + o, lbo, sbo), desc(bL + o, lbo, sbo), id, 1);
          mma_bf16(tmem, desc(aL + o, lbo, sbo), desc(bH + o, lbo, sbo), id, 1);
        }
      }
      commit(&s_bar[s]);
    }
    __syncwarp();
  }
  if (ok && nk > 0) {  // the last commit covers every MMA issued before it
    const int waited = mbar_wait(&s_bar[(nk - 1) & 1], (uint32_t)(((nk - 1) >> 1) & 1)) ? 1 : 0;
    ok = __syncthreads_and(waited) != 0;
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
  } else {
    fence_after();
    const int r = m0 + warp * 32 + lane;
    for (int j0 = 0; j0 < BN && n0 + j0 < g.N; j0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)j0, v);
      if (r >= g.M) continue;
      if (nsl > 1) {  // partial product of this K slice
        float* w = g.ws + ((long long)z * g.M + r) * g.N + n0 + j0;
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (n0 + j0 + i < g.N) w[i] = nk > 0 ? v[i] : 0.f;
        continue;
      }
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int n = n0 + j0 + i;
        if (n >= g.N) break;
        float x = nk > 0 ? g.alpha * v[i] : 0.f;
        if (g.bias) x += g.bias[n];
        if (g.Cpre) g.Cpre[(long long)r * g.ldpre + n] = x;
        if (g.gelu) x = gelu(x);
        if (g.Cf) {
          float* c = g.Cf + (long long)r * g.ldc + n;
          *c = g.accumulate ? *c + x : x;
        }
        if (g.Cb) g.Cb[(long long)r * g.ldcb + n] = __float2bfloat16_rn(x);
        if (g.CbT) g.CbT[(long long)n * g.ldcbt + r] = __float2bfloat16_rn(x);
      }
    }
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_free(tmem, 128);
}

// split-K: sum the slices in order, then the epilogue of gemm_kernel
__global__ void gemm_splitk_reduce_kernel(GemmArgs g, int nsl) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)g.M * g.N) return;
  const int r = (int)(q / g.N), n = (int)(q - (long long)r * g.N);
  float acc = 0.f;
  for (int z = 0; z < nsl; ++z) acc += g.ws[(long long)z * g.M * g.N + q];
  float x = g.alpha * acc;
  if (g.bias) x += g.bias[n];
  if (g.Cpre) g.Cpre[(long long)r * g.ldpre + n] = x;
  if (g.gelu) x = gelu(x);
  if (g.Cf) {
    float* c = g.Cf + (long long)r * g.ldc + n;
    *c = g.accumulate ? *c + x : x;
  }
  if (g.Cb) g.Cb[(long long)r * g.ldcb + n] = __float2bfloat16_rn(x);
  if (g.CbT) g.CbT[(long long)n * g.ldcbt + r] = __float2bfloat16_rn(x);
}

size_t gemm_smem(int split) { return (size_t)2 * (split ? 4 : 2) * BM * BK * sizeof(uint16_t); }

cudaError_t launch_gemm(const GemmArgs& g, int* d_err, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0) return cudaSuccess;
  if (g.K < 0 || g.K % BK) return cudaErrorInvalidValue;
  // rows must start on 16-byte boundaries for the vector loads
  const int q = g.split ? 4 : 8;
  if (g.lda % q || g.ldb % q || ((uintptr_t)g.A & 15) || ((uintptr_t)g.B & 15)) return cudaErrorInvalidValue;
  const size_t smem = gemm_smem(g.split);
  dim3 grid((g.N + BN - 1) / BN, (g.M + BM - 1) / BM, 1);
  // split K when the output has too few tiles to fill the SMs (about 148)
  const int tiles = (int)(grid.x * grid.y), nk = g.K / BK;
  int ks = 1;
  if (g.ws && tiles < 96 && nk >= 4) {
    ks = 148 / tiles;
    if (ks > nk / 2) ks = nk / 2;
    while (ks > 1 && (long long)ks * g.M * g.N > g.ws_floats) --ks;
    if (ks < 1) ks = 1;
  }
  grid.z = ks;
  GemmArgs ga = g;
  ga.ksplit = ks;
  cudaError_t e;
  if (g.split) {
    e = smem_limit(gemm_kernel<1>, smem);
    if (e != cudaSuccess) return e;
    gemm_kernel<1><<<grid, 128, smem, st>>>(ga, d_err);
  } else {
    e = smem_limit(gemm_kernel<0>, smem);
    if (e != cudaSuccess) return e;
    gemm_kernel<0><<<grid, 128, smem, st>>>(ga, d_err);
  }
  if (ks > 1) {
    const long long nq = (long long)g.M * g.N;
    gemm_splitk_reduce_kernel<<<(unsigned)((nq + 255) / 256), 256, 0, st>>>(ga, ks);
  }
  return cudaGetLastError();
}

}  // namespace sg
