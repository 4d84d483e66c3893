// sg_legendre_mma.cu -- the Legendre contractions of the mixed-precision path
// on the 5th-generation tensor cores (tcgen05), in BF16x3 or BF16x6 split
// precision.
//
// Each Legendre stage of the coupling step (the theta half of SPHEREPACK's
// Gauss-grid analysis shagc.f:384-470 and synthesis shsgc.f:329-470, batched
// over capsules and fields) is, for every zonal wavenumber m, a product
//   D[q][j] = sum_k A[q][k] B_m[j][k]
// of FP32 data rows A (one per capsule and field) with a per-degree FP64
// table B_m (Legendre functions times Gauss weights).  Both operands are
// K-major, so one tile is a single "TN" UMMA: M = 128 data rows, N = J padded
// to a multiple of 16, K padded to a multiple of 16.
//
// Split precision: x = x0 + x1 + x2 with x0 = bf16(x), x1 = bf16(x - x0),
// x2 = bf16(x - x0 - x1).  A problem runs in one of two modes:
//   BF16x3 (terms = 3):  A B^T ~ A0 B0^T + A0 B1^T + A1 B0^T
//     (the dropped terms are ~2^-18 relative, about 16 significant bits);
//   BF16x6 (terms = 6):  + A0 B2^T + A2 B0^T + A1 B1^T
//     (dropped terms ~2^-27: FP32-level products for high degrees, whose
//     second derivatives amplify the BF16x3 error past 1e-4).
// Products accumulate in FP32 in tensor memory.  The tables are split once on
// the host into three bf16 images laid out as UMMA operands; the data rows are
// split while staged.
//
// Shared-memory operand layout (no swizzle, K-major canonical form): an
// R x Kp bf16 tile is stored as [R/8][Kp/8] core matrices of 8 rows x 16
// bytes, so the leading-dimension byte offset (next core matrix along K) is
// 128 B, the stride byte offset (next 8-row group) is Kp*16 B, and each K step
// of 16 advances the start address by 256 B.
//
// Persistent CTAs of 128 threads (one warp per 32-lane TMEM subpartition)
// loop over the (problem, m, 128-row tile) work list.  Thread 0 issues the
// MMAs and commits them to an mbarrier; all threads wait with a bounded spin
// (error flag, no trap, on timeout), read the accumulator with tcgen05.ld and
// store the rows.
#include "sg_common.cuh"
#include "sg_kernels.h"
#include "sg_umma.cuh"

namespace sg {

namespace {

using namespace umma;

}  // namespace

namespace {

// bf16 parts of the data operand (A) in shared memory, and the table (B)
// region of each chain level (its parts follow one another at the level's
// problem's own stride Jp Kp, as in the global image)
struct Operands {
  uint16_t* a[3];
  uint16_t* b[3];
};

__device__ __forceinline__ int parts_of(const LegProblem& P) { return P.terms == 6 ? 3 : 2; }

// The B_m image of problem P (the parts its mode reads, contiguous in the
// global image) into its level's region: one bulk copy on the TMA engine,
// completing on the level's mbarrier.  Issued by one thread.
__device__ __forceinline__ void fetch_table(const LegProblem& P, int m, uint16_t* dst, uint64_t* bar) {
  const uint16_t* src = (const uint16_t*)P.Bimg + (long long)m * P.sBimg;
  const uint32_t bytes = (uint32_t)(parts_of(P) * P.Jp * P.Kp) * 2u;
  bulk_g2s(dst, src, bytes, bar);
}

// Eight consecutive K values of one data row, split into the operand parts.
__device__ __forceinline__ void store_split(const float* x, int np, const Operands& op, int o) {
  uint4 p0, p1, p2;
  split8x3(x, p0, p1, p2);
  *(uint4*)(op.a[0] + o) = p0;
  *(uint4*)(op.a[1] + o) = p1;
  if (np == 3) *(uint4*)(op.a[2] + o) = p2;
}

// One thread issues the split products of every K step of 16 (largest terms
// first), then commits.  bt: the level's table region; tm: the tile's rows.
__device__ __forceinline__ void issue_mma(const LegProblem& P, int m, int tm, uint32_t tmem, const Operands& op,
                                          const uint16_t* bt, uint64_t* bar) {
  const uint32_t idesc = idesc_bf16(tm, P.Jp);
  const uint32_t lbo = 128, sbo = (uint32_t)P.Kp * 16;
  const uint32_t pb = (uint32_t)(P.Jp * P.Kp) * 2u;  // bytes per table part
  const uint32_t a0 = smem_u32(op.a[0]), a1 = smem_u32(op.a[1]), b0 = smem_u32(bt), b1 = b0 + pb;
  const bool six = P.terms == 6;
  const uint32_t a2 = six ? smem_u32(op.a[2]) : 0u, b2 = b0 + 2u * pb;
  const int s0 = P.tri ? (m >> 4) : 0;  // synthesis: coefficients below n = m vanish
  uint32_t acc = 0;
  for (int s = s0; s < (P.Kp >> 4); ++s) {
    const uint32_t o = (uint32_t)s * 256;
    mma_bf16(tmem, desc(a0 + o, lbo, sbo), desc(b0 + o, lbo, sbo), idesc, acc);
    acc = 1;
    mma_bf16(tmem, desc(a0 + o, lbo, sbo), desc(b1 + o, lbo, sbo), idesc, 1);
    mma_bf16(tmem, desc(a1 + o, lbo, sbo), desc(b0 + o, lbo, sbo), idesc, 1);
    if (six) {
      mma_bf16(tmem, desc(a0 + o, lbo, sbo), desc(b2 + o, lbo, sbo), idesc, 1);
      mma_bf16(tmem, desc(a2 + o, lbo, sbo), desc(b0 + o, lbo, sbo), idesc, 1);
      mma_bf16(tmem, desc(a1 + o, lbo, sbo), desc(b1 + o, lbo, sbo), idesc, 1);
    }
  }
  commit(bar);
}

}  // namespace

// Work items name root problems; a root's next[] problems take its output
// rows as their A operand for the same (m, tile) and run in the same CTA: the
// accumulator is read once from TMEM, written to global memory, and split into
// the next product's bf16 operand parts in shared memory, so the data
// never leaves the SM between the two contractions.
// A chain runs in its root's mode (one degree group: the same mode throughout).
// Tiles of TM = 128 data rows (M = 128: row r in TMEM lane r, so warp w
// holds rows 32w..32w+31) or TM = 64 (M = 64: row r in lane (r mod 16) +
// 32 floor(r / 16) -- the first half of every warp's 32-lane quadrant -- so
// warp w holds rows 16w..16w+15 in its lanes 0..15); 64-row tiles double the
// work items of a launch whose 128-row tiles would leave SMs idle.
// smem (bf16): nparts A parts of TM x lv.a_kp, then for each chain level l a
// table region of nparts x lv.jp[l] x lv.kp[l]; nparts = 3 when any problem of
// the launch is BF16x6, else 2.  At the start of a work item one thread issues
// the bulk copies of every level's table (each on its own mbarrier), so they
// overlap the staging of the data rows and the earlier products.
template <int TM>
__global__ void __launch_bounds__(128) legendre_mma_kernel(const LegProblem* __restrict__ probs,
                                                           const LegWork* __restrict__ work, int nwork, LegLevels lv,
                                                           int nparts, int tmem_cols, int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ __align__(8) uint64_t s_tbar[3];
  __shared__ uint32_t s_tmem;
  Operands op;
  {
    uint16_t* p = (uint16_t*)smem_raw;
    for (int i = 0; i < 3; ++i) {
      op.a[i] = p;
      if (i + 1 < nparts) p += TM * lv.a_kp;
    }
    p = (uint16_t*)smem_raw + nparts * TM * lv.a_kp;
    for (int l = 0; l < 3; ++l) {
      op.b[l] = p;
      p += nparts * lv.jp[l] * lv.kp[l];
    }
  }
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    tmem_alloc(&s_tmem, (uint32_t)tmem_cols);
  }
  if (tid == 0) {
    mbar_init(&s_bar, 1);
    for (int l = 0; l < 3; ++l) mbar_init(&s_tbar[l], 1);
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = s_tmem;
  uint32_t phase = 0;             // MMA commits
  uint32_t tphase[3] = {0, 0, 0};  // table copies, per level (a level completes one phase per item using it)
  int pending = 0;                 // levels whose copy was issued and not yet waited for (thread 0)
  bool ok = true;

  for (int it = blockIdx.x; it < nwork && ok; it += gridDim.x) {
    const LegWork wk = work[it];
    const int m = wk.m, q0 = wk.q0;
    int pid = wk.prob;
    const LegProblem& R = probs[pid];
    const int nq = min(TM, R.Q - q0);
    const int np = parts_of(R);
    // the chain: level 0 the root, 1 its next[0], 2 its next[1] (only after a level 1)
    const int chain[3] = {pid, R.next[0], R.next[0] >= 0 ? R.next[1] : -1};
    bool fits = np <= nparts;
    for (int l = 0; l < 3; ++l)
      if (chain[l] >= 0) {
        const LegProblem& P = probs[chain[l]];
        fits = fits && parts_of(P) == np && P.Jp <= lv.jp[l] && P.Kp <= lv.kp[l] && P.Kp <= lv.a_kp;
      }
    if (!fits) {  // the launch's shared memory was sized for other problems (uniform per CTA)
      if (tid == 0) atomicExch(err, 2);
      continue;
    }
    if (tid == 0) {
      fence_async_smem();  // earlier generic accesses of the regions before the async copies
      for (int l = 0; l < 3; ++l)
        if (chain[l] >= 0) {
          fetch_table(probs[chain[l]], m, op.b[l], &s_tbar[l]);
          pending |= 1 << l;
        }
    }
    // ---- data rows of the root: FP32 -> bf16 parts.  Thread tid stages
    // row tid % TM of the tile, every (128/TM)-th core-matrix row of 8 values
    // starting at tid / TM; all of its loads (up to 8 core-matrix rows) are
    // issued before any is split and stored, so their latencies overlap.
    {
      constexpr int NPH = 128 / TM;
      const int K = R.K, KC = R.Kp >> 3, q = tid % TM, ph = tid / TM;
      const float* row = nullptr;
      if (q < nq) {
        const int qq = q0 + q, c = qq / R.rpc, r = qq - c * R.rpc;
        row = (const float*)R.A + (long long)c * R.sAc + (long long)r * R.sAr + (long long)m * R.sAm;
      }
      for (int kc0 = ph; kc0 < KC; kc0 += 8 * NPH) {
        float x[8][8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int kc = kc0 + u * NPH, k0 = kc << 3;
          if (row && kc < KC && R.vecA && k0 + 8 <= K) {
            const float4 a = *(const float4*)(row + k0), b = *(const float4*)(row + k0 + 4);
            x[u][0] = a.x; x[u][1] = a.y; x[u][2] = a.z; x[u][3] = a.w;
            x[u][4] = b.x; x[u][5] = b.y; x[u][6] = b.z; x[u][7] = b.w;
          } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) x[u][i] = (row && kc < KC && k0 + i < K) ? row[k0 + i] : 0.f;
          }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (kc0 + u * NPH < KC) store_split(x[u], np, op, cm_offset(q, kc0 + u * NPH, KC));
      }
    }
    // ---- the root, then its chained products: one MMA group per problem
    for (int level = 0; level < 3 && ok; ++level) {
      const LegProblem& P = probs[pid];
      fence_async_smem();  // generic-proxy smem writes -> visible to the tensor core
      fence_before();
      __syncthreads();
      fence_after();
      if (tid == 0) {
        // the level's table has landed (bounded wait; on timeout the MMA wait
        // below runs out too and the CTA leaves with the error flag set)
        const bool landed = mbar_wait(&s_tbar[level], tphase[level]);
        pending &= ~(1 << level);
        tphase[level] ^= 1u;
        if (landed)
          issue_mma(P, m, TM, tmem, op, op.b[level], &s_bar);
        else
          atomicExch(err, 1);
      }
      __syncwarp();
      // every thread waits; the CTA then agrees on the outcome so that all of
      // its threads leave the loop together on a timeout
      const int waited = mbar_wait(&s_bar, phase) ? 1 : 0;
      if (!__syncthreads_and(waited)) {
        if (tid == 0) atomicExch(err, 1);
        ok = false;
        break;
      }
      phase ^= 1u;
      fence_after();
      // chained products of the root take its rows as their A operand
      const bool chain = level == 0 && P.next[0] >= 0;
      const int KC2 = P.Jp >> 3;  // next K padded = this J padded
      // ---- epilogue: warp w holds rows 32w..32w+31 of a 128-row tile, rows
      // 16w..16w+15 of a 64-row tile (its lanes 0..15)
      {
        const bool lane_row = TM == 128 || lane < 16;
        const int q = TM == 128 ? warp * 32 + lane : warp * 16 + lane;
        const int J = P.J;
        float* drow = nullptr;
        if (lane_row && q < nq) {
          const int qq = q0 + q, c = qq / P.rpc, r = qq - c * P.rpc;
          drow = (float*)P.D + (long long)c * P.sDc + (long long)r * P.sDr + (long long)m * P.sDm;
        }
        for (int j0 = 0; j0 < P.Jp; j0 += 16) {
          float v[16];
          tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)j0, v);
          if (drow) {
            if (P.vecD && j0 + 16 <= J) {
#pragma unroll
              for (int i = 0; i < 16; i += 4)
                *(float4*)(drow + j0 + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
            } else {
#pragma unroll
              for (int i = 0; i < 16; ++i)
                if (j0 + i < J) drow[j0 + i] = v[i];
            }
          }
          if (chain && lane_row) {  // root MMA is complete: its A tile is free for the next operand
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              float x[8];
#pragma unroll
              for (int i = 0; i < 8; ++i) x[i] = (j0 + 8 * h + i < J && q < nq) ? v[8 * h + i] : 0.f;
              store_split(x, np, op, cm_offset(q, (j0 >> 3) + h, KC2));
            }
          }
        }
      }
      if (level == 0) {
        if (!chain) break;
        pid = P.next[0];
      } else if (level == 1) {
        // the second chained product of the root (same A operand), if any
        const int n2 = probs[wk.prob].next[1];
        if (n2 < 0) break;
        pid = n2;
      } else {
        break;
      }
      // all TMEM reads and operand writes are done before the next MMA
      fence_before();
      __syncthreads();
      fence_after();
    }
    fence_before();
    __syncthreads();  // TMEM reads and smem operands done before the next tile
    fence_after();
  }
  if (!ok) {
    // a commit that never arrived: give the tensor core a bounded chance to
    // finish before freeing its accumulator, and the table copies still in
    // flight a bounded chance to land before the shared memory is released
    mbar_wait(&s_bar, phase);
    if (tid == 0)
      for (int l = 0; l < 3; ++l)
        if (pending & (1 << l)) mbar_wait(&s_tbar[l], tphase[l]);
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_free(tmem, (uint32_t)tmem_cols);
}

size_t legendre_mma_smem(const LegLevels& lv, int nparts, int tm) {
  size_t e = (size_t)tm * lv.a_kp;
  for (int l = 0; l < 3; ++l) e += (size_t)lv.jp[l] * lv.kp[l];
  return (size_t)nparts * sizeof(uint16_t) * e;
}

cudaError_t launch_legendre_mma(const LegProblem* d_probs, const LegWork* d_work, int nwork, const LegLevels& lv,
                                int nparts, int tm, int* d_err, int num_sms, cudaStream_t st) {
  if (nwork <= 0) return cudaSuccess;
  if (tm != 64 && tm != 128) return cudaErrorInvalidValue;
  int maxJp = 0;
  for (int l = 0; l < 3; ++l) {
    if (lv.jp[l] < 0 || lv.jp[l] > 256 || (lv.jp[l] & 15) || lv.kp[l] < 0 || (lv.kp[l] & 15))
      return cudaErrorInvalidValue;
    maxJp = lv.jp[l] > maxJp ? lv.jp[l] : maxJp;
  }
  if (lv.jp[0] < 16 || lv.kp[0] < 16 || lv.a_kp < 16 || (lv.a_kp & 15)) return cudaErrorInvalidValue;
  if (nparts != 2 && nparts != 3) return cudaErrorInvalidValue;
  // TMEM columns: a power of two >= 32 covering N = Jp; CTAs per SM limited
  // (through shared memory) so that their allocations always fit in 512 columns
  int cols = 32;
  while (cols < maxJp) cols <<= 1;
  const int per_sm = 512 / cols < 4 ? 512 / cols : 4;
  size_t smem = legendre_mma_smem(lv, nparts, tm);
  // (per_sm + 1) CTAs of this size exceed the SM's 228 KB of shared memory
  const size_t floor_smem = (size_t)(228 * 1024) / (size_t)(per_sm + 1);
  if (smem < floor_smem) smem = floor_smem;
  if (smem > (size_t)227 * 1024) return cudaErrorInvalidValue;
  const int grid = nwork < num_sms * per_sm ? nwork : num_sms * per_sm;
  if (tm == 64) {
    cudaError_t e = cudaFuncSetAttribute(legendre_mma_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    legendre_mma_kernel<64><<<grid, 128, smem, st>>>(d_probs, d_work, nwork, lv, nparts, cols, d_err);
  } else {
    cudaError_t e = cudaFuncSetAttribute(legendre_mma_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    legendre_mma_kernel<128><<<grid, 128, smem, st>>>(d_probs, d_work, nwork, lv, nparts, cols, d_err);
  }
  return cudaGetLastError();
}

}  // namespace sg
