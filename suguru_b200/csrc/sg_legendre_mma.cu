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
#include <algorithm>

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
// first) into the accumulator at tmem.  bt: the level's table region; tm: the
// tile's rows.  The caller commits.
__device__ __forceinline__ void issue_mma(const LegProblem& P, int m, int tm, uint32_t tmem, const Operands& op,
                                          const uint16_t* bt) {
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
}

}  // namespace

// Work items name root problems; a root's next[] problems take its output
// rows as their A operand for the same (m, tile) and run in the same CTA: the
// accumulator is read once from TMEM, written to global memory, and split into
// the next product's bf16 operand parts in shared memory, so the data never
// leaves the SM between the two contractions.  The two chained products share
// that operand, so they are issued together (level 1 at TMEM column 0, level 2
// at column off2) under one commit, and read back in one epilogue.
// A chain runs in its root's mode (one degree group: the same mode throughout).
// Tiles of TM = 128 data rows (M = 128: row r in TMEM lane r) or TM = 64
// (M = 64: row r in lane (r mod 16) + 32 floor(r / 16) -- the first half of
// every 32-lane quadrant).
//
// CTAs of kLegThreads = 256 threads (8 warps), up to three per SM, so that
// every work item of a launch is resident at once (the items are short
// chains of dependent phases; their latencies overlap across CTAs).  Warp w
// reads TMEM lane quadrant w % 4 (the hardware ties a warp to the quadrant of
// its index mod 4) and column group w / 4 of every 32-column slab, so the two
// warps of a quadrant read a row's columns in parallel; the slab goes through
// shared memory (s_slab, row stride 33 words) and every warp then writes
// whole rows of it to global memory as contiguous runs.  The data rows are
// staged by all threads in coalesced 32-byte pieces.
// smem (bf16, dynamic): nparts A parts of TM x lv.a_kp, then for each chain
// level l a table region of nparts x lv.jp[l] x lv.kp[l]; nparts = 3 when any
// problem of the launch is BF16x6, else 2.  At the start of a work item one
// thread issues the bulk copies of every level's table (each on its own
// mbarrier), so they overlap the staging of the data rows and the root product.
constexpr int kLegThreads = 256;
constexpr int kLegGroups = kLegThreads / 128;  // warps per TMEM lane quadrant
constexpr int kSlab = 16 * kLegGroups;         // columns per slab
constexpr int kLegPerSm = 3;                   // CTAs per SM (registers: launch bounds)

template <int TM>
__global__ void __launch_bounds__(kLegThreads, kLegPerSm) legendre_mma_kernel(const LegProblem* __restrict__ probs,
                                                                    const LegWork* __restrict__ work, int nwork,
                                                                    LegLevels lv, int nparts, int tmem_cols,
                                                                    int off2, int* __restrict__ err) {
  pdl_enter();
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ __align__(8) uint64_t s_tbar[3];
  __shared__ uint32_t s_tmem;
  // the work item's chain of problems, copied from global memory by the whole
  // CTA in one round of independent loads instead of field by field
  __shared__ __align__(16) LegProblem s_p[3];
  // element offsets of the tile's rows in the root's A (staging) and in a
  // level's D (epilogue), -1 past the problem's last row
  __shared__ long long s_roff[2][TM];
  __shared__ float s_slab[TM * (kSlab + 1)];
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
  const int quad = warp & 3, cgrp = warp >> 2;  // TMEM lane quadrant, column group

  if (warp == 0) tmem_alloc(&s_tmem, (uint32_t)tmem_cols);
  if (tid == 0) {
    mbar_init(&s_bar, 1);
    for (int l = 0; l < 3; ++l) mbar_init(&s_tbar[l], 1);
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = s_tmem;
  uint32_t phase = 0;              // MMA commits
  uint32_t tphase[3] = {0, 0, 0};  // table copies, per level (one phase per item that uses the level)
  int pending = 0;                 // levels whose copy was issued and not yet waited for (thread 0)
  bool ok = true;
  // this thread's TMEM row: quadrant quad, lane -> tile row (TM = 64: lanes 0-15 only)
  const bool lane_row = TM == 128 || lane < 16;
  const int q = TM == 128 ? quad * 32 + lane : quad * 16 + lane;

  constexpr int PW = (int)(sizeof(LegProblem) / sizeof(int));
  for (int it = blockIdx.x; it < nwork && ok; it += gridDim.x) {
    const LegWork wk = work[it];
    const int m = wk.m, q0 = wk.q0;
    // the chain: level 0 the root, 1 its next[0], 2 its next[1] (only after a level 1)
    const int lvl[3] = {wk.prob, wk.lvl1, wk.lvl1 >= 0 ? wk.lvl2 : -1};
    for (int l = 0; l < 3; ++l)
      if (lvl[l] >= 0)
        for (int i = tid; i < PW; i += kLegThreads) ((int*)&s_p[l])[i] = ((const int*)&probs[lvl[l]])[i];
    __syncthreads();
    const LegProblem& R = s_p[0];
    const int nq = min(TM, R.Q - q0);
    const int np = parts_of(R);
    bool fits = np <= nparts && (R.Kp >> 3) <= 8 && (lvl[2] < 0 || off2 >= lv.jp[1]);
    for (int l = 0; l < 3; ++l)
      if (lvl[l] >= 0) {
        const LegProblem& P = s_p[l];
        fits = fits && parts_of(P) == np && P.Jp <= lv.jp[l] && P.Kp <= lv.kp[l] && P.Kp <= lv.a_kp;
      }
    if (!fits) {  // the launch's shared memory was sized for other problems (uniform per CTA)
      if (tid == 0) atomicExch(err, 2);
      __syncthreads();  // every thread has read s_p before the next item overwrites it
      continue;
    }
    if (tid == 0) {
      fence_async_smem();  // earlier generic accesses of the regions before the async copies
      for (int l = 0; l < 3; ++l)
        if (lvl[l] >= 0) {
          fetch_table(s_p[l], m, op.b[l], &s_tbar[l]);
          pending |= 1 << l;
        }
    }
    // ---- data rows of the root: FP32 -> bf16 parts.  Row offsets first (one
    // division per row), then the rows are read in coalesced pieces: with KC =
    // Kp/8 chunks of 8 values per row, thread t takes chunk t % KC of rows
    // t / KC + u (kLegThreads / KC); all of a thread's loads are issued before
    // any is split.
    if (tid < TM) {
      long long o = -1;
      if (tid < nq) {
        const int qq = q0 + tid, c = qq / R.rpc, r = qq - c * R.rpc;
        o = (long long)c * R.sAc + (long long)r * R.sAr + (long long)m * R.sAm;
      }
      s_roff[0][tid] = o;
    }
    __syncthreads();
    {
      const float* Ab = (const float*)R.A;
      const int K = R.K, KC = R.Kp >> 3, rpp = kLegThreads / KC, kc = tid % KC, r0 = tid / KC, k0 = kc << 3;
      constexpr int NU = 128 * 8 / kLegThreads;  // passes: KC <= 8 and TM <= 128
      float x[NU][8];
#pragma unroll
      for (int u = 0; u < NU; ++u) {
        const int row = r0 + u * rpp;
        const long long o = (r0 < rpp && row < TM) ? s_roff[0][row] : -1;
        if (o >= 0 && R.vecA && k0 + 8 <= K) {
          const float4 a = *(const float4*)(Ab + o + k0), b = *(const float4*)(Ab + o + k0 + 4);
          x[u][0] = a.x; x[u][1] = a.y; x[u][2] = a.z; x[u][3] = a.w;
          x[u][4] = b.x; x[u][5] = b.y; x[u][6] = b.z; x[u][7] = b.w;
        } else {
#pragma unroll
          for (int i = 0; i < 8; ++i) x[u][i] = (o >= 0 && k0 + i < K) ? Ab[o + k0 + i] : 0.f;
        }
      }
#pragma unroll
      for (int u = 0; u < NU; ++u) {
        const int row = r0 + u * rpp;
        if (r0 < rpp && row < TM) store_split(x[u], np, op, cm_offset(row, kc, KC));
      }
    }
    // ---- stage 0: the root; stage 1: its chained products (levels 1 and 2,
    // one commit)
    const bool chained = lvl[1] >= 0;
    for (int stage = 0; stage < 2 && ok; ++stage) {
      if (stage == 1 && !chained) break;
      fence_async_smem();  // generic-proxy smem writes -> visible to the tensor core
      fence_before();
      __syncthreads();
      fence_after();
      if (tid == 0) {
        // each level's table has landed (bounded wait; on timeout the MMA wait
        // below runs out too and the CTA leaves with the error flag set)
        bool landed = true;
        for (int l = stage == 0 ? 0 : 1; l <= (stage == 0 ? 0 : 2); ++l) {
          if (lvl[l] < 0) continue;
          landed = mbar_wait(&s_tbar[l], tphase[l]) && landed;
          pending &= ~(1 << l);
          tphase[l] ^= 1u;
          if (landed) issue_mma(s_p[l], m, TM, tmem + (uint32_t)(l == 2 ? off2 : 0), op, op.b[l]);
        }
        if (landed)
          commit(&s_bar);
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
      // ---- epilogue of each level of this stage
      for (int l = stage == 0 ? 0 : 1; l <= (stage == 0 ? 0 : 2); ++l) {
        if (lvl[l] < 0) continue;
        const LegProblem& P = s_p[l];
        const bool split_next = stage == 0 && chained;  // root: its rows become the next A operand
        const int J = P.J, KC2 = P.Jp >> 3;
        const uint32_t cbase = l == 2 ? (uint32_t)off2 : 0u;
        if (cgrp == 0 && lane_row) {
          long long o = -1;
          if (q < nq) {
            const int qq = q0 + q, c = qq / P.rpc, r = qq - c * P.rpc;
            o = (long long)c * P.sDc + (long long)r * P.sDr + (long long)m * P.sDm;
          }
          s_roff[1][q] = o;
        }
        float* Db = (float*)P.D;
        for (int jc = 0; jc < P.Jp; jc += kSlab) {
          const int j0 = jc + 16 * cgrp;
          const bool mine = j0 < P.Jp;  // uniform per warp
          uint32_t raw[16];
          if (mine) {
            tmem_ld16_nowait(tmem + ((uint32_t)(quad * 32) << 16) + cbase + (uint32_t)j0, raw);
            tmem_wait_ld();
            if (lane_row) {
              float v[16];
#pragma unroll
              for (int i = 0; i < 16; ++i) {
                v[i] = __uint_as_float(raw[i]);
                s_slab[q * (kSlab + 1) + 16 * cgrp + i] = v[i];
              }
              if (split_next) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                  float xs[8];
#pragma unroll
                  for (int i = 0; i < 8; ++i) xs[i] = (j0 + 8 * h + i < J && q < nq) ? v[8 * h + i] : 0.f;
                  store_split(xs, np, op, cm_offset(q, (j0 >> 3) + h, KC2));
                }
              }
            }
          }
          __syncthreads();  // the slab and the row offsets are complete
          const int ncol = min(kSlab, J - jc);
          for (int rr = warp; rr < TM; rr += kLegThreads / 32) {
            const long long o = s_roff[1][rr];
            if (o >= 0)
#pragma unroll
              for (int c0 = 0; c0 < kSlab; c0 += 32)
                if (c0 + lane < ncol) Db[o + jc + c0 + lane] = s_slab[rr * (kSlab + 1) + c0 + lane];
          }
          __syncthreads();  // the slab is consumed before the next one is written
        }
      }
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
  for (int l = 0; l < 3; ++l)
    if (lv.jp[l] < 0 || lv.jp[l] > 256 || (lv.jp[l] & 15) || lv.kp[l] < 0 || (lv.kp[l] & 15))
      return cudaErrorInvalidValue;
  if (lv.jp[0] < 16 || lv.kp[0] < 16 || lv.a_kp < 16 || (lv.a_kp & 15) || lv.a_kp > 64) return cudaErrorInvalidValue;
  if (nparts != 2 && nparts != 3) return cudaErrorInvalidValue;
  // TMEM columns: the root's accumulator at column 0; the chained products at
  // columns 0 (level 1) and off2 (level 2, 32-column aligned) at the same
  // time; a power of two >= 32 covering both
  const int off2 = (lv.jp[1] + 31) / 32 * 32;
  const int need = std::max(lv.jp[0], off2 + lv.jp[2]);
  int cols = 32;
  while (cols < need) cols <<= 1;
  if (cols > 512) return cudaErrorInvalidValue;
  const size_t smem = legendre_mma_smem(lv, nparts, tm);
  cudaFuncAttributes fa{};
  cudaError_t e = tm == 64 ? cudaFuncGetAttributes(&fa, legendre_mma_kernel<64>)
                           : cudaFuncGetAttributes(&fa, legendre_mma_kernel<128>);
  if (e != cudaSuccess) return e;
  if (smem + fa.sharedSizeBytes > (size_t)227 * 1024) return cudaErrorInvalidValue;
  // up to kLegPerSm CTAs per SM, fewer when their TMEM allocations would not
  // all fit in the SM's 512 columns (a CTA that cannot allocate would wait)
  const int per_sm = std::min(kLegPerSm, 512 / cols);
  const int grid = nwork < num_sms * per_sm ? nwork : num_sms * per_sm;
  if (tm == 64) {
    e = smem_limit(legendre_mma_kernel<64>, smem);
    if (e != cudaSuccess) return e;
    launch_pdl(legendre_mma_kernel<64>, dim3(grid), dim3(kLegThreads), smem, st, d_probs, d_work, nwork, lv, nparts, cols, off2, d_err);
  } else {
    e = smem_limit(legendre_mma_kernel<128>, smem);
    if (e != cudaSuccess) return e;
    launch_pdl(legendre_mma_kernel<128>, dim3(grid), dim3(kLegThreads), smem, st, d_probs, d_work, nwork, lv, nparts, cols, off2,
                                                              d_err);
  }
  return cudaGetLastError();
}

}  // namespace sg
