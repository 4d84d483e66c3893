// sg_spread.cu -- deterministic spreading of Lagrangian forces onto the MAC grid.
//
// Replaces the scatter loop of lagr2eulr (interp_spread.f90:817-884):
//   forcex(i,j,k) += fxl * kernel(i-c_x) kernel(j-0.5-c_y) kernel(k-0.5-c_z) * area/dVeul
// (v and w likewise with their own face direction), after zeroing the whole
// field (:811-815) and followed by the periodic halo copy of updthalos
// (bound.f90:141-190).
//
// One CTA per output tile of TX x TY x TZ interior cells.  Its entries -- every
// point whose stencil reaches the tile, listed by the binning pass -- are
// processed one point per thread: the thread evaluates the point's 1-D kernel
// weights and adds its contributions to the cells of the stencil that lie in
// the tile.  Sums are kept in shared memory in fixed point with per-tile,
// per-component power-of-two scales and added with 32-bit integer atomics:
// integer addition is exact and associative, so the field is bitwise
// independent of the order in which threads add (no floating-point atomics,
// deterministic run to run).  Each component has its own scale, so that its
// relative precision does not depend on the other components' magnitudes.
//
//  - FP32: one signed 32-bit word per cell and component.  With m_c =
//    |f_c * area / dV| per entry, the scale of component c is the smaller of
//    two powers of two: one that puts 0.3 * sum over the tile's entries of m_c
//    below 2^30 (every 3-D kernel weight is at most (2/3)^3 < 0.3, so no cell
//    sum can reach 2^31), and one that puts 0.3 * the largest m_c below 2^22,
//    so that every contribution v satisfies |v| < 2^22.  The sum is needed
//    only above 2^8 entries (below, count * largest m_c bounds it tightly
//    enough) and is then an exact integer sum of m_c rounded up to 2^-12 of
//    the largest m_c's binade, so that the scales, like the cell sums, are
//    independent of the order of the entries.  Then one FMA, v + 1.5 * 2^23,
//    rounds v to the nearest integer (ties to even) in the low mantissa bits
//    of a float whose exponent is fixed, and the integer is its bit pattern
//    minus that of 1.5 * 2^23 -- no conversion instruction per contribution.
//    The fixed-point step is 2^-22 of 0.3 times the component's largest
//    contribution, below FP32 rounding of a typical cell value.
//  - FP64: 64-bit fixed point (|sum| < 2^56 from the component's largest
//    contribution in the tile times its entry count, or above 4096 entries
//    from 0.3 * the same exact integer sum of m_c as FP32 takes) kept as three limbs of 19 bits, the
//    lower two unsigned, so that the atomics stay native 32-bit adds; with at
//    most 4096 contributions per pass no limb can overflow, and between passes
//    the limbs are folded into 64-bit registers.
// Entries go to threads in blocks of 256: the lowest ceil(k/32) warps take the
// k entries of a block, interleaved, so that no warp idles on a short list and
// neighbouring points (adjacent entries) land in different warps, where they
// rarely hit the same shared-memory word in the same instruction.
#include "sg_common.cuh"
#include "sg_kernels.h"

namespace sg {

namespace {

constexpr float kMagic = 12582912.0f;          // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;          // its bit pattern
constexpr int LB = 19;      // FP64 limb width
constexpr int kOut = -(1 << 24);  // offset of a stencil node outside the tile
constexpr int MAXC = 4096;  // FP64 contributions per pass: 19 + 12 <= 31 bits per limb

template <class T>
struct Fixed;
template <>
struct Fixed<float> {
  static constexpr int NW = 1;
  static constexpr int QB = 30;
  static constexpr int PASS = 1 << 30;
};
template <>
struct Fixed<double> {
  static constexpr int NW = 3;
  static constexpr int QB = 3 * LB - 1;
  static constexpr int PASS = MAXC;
  __device__ static __forceinline__ void add(unsigned int* base, int stride, double v) {
    long long q = __double2ll_rn(v);  // q = sum_w limb_w 2^(LB w)
    atomicAdd(base, (unsigned int)(q & ((1ll << LB) - 1)));
    q >>= LB;
    atomicAdd(base + stride, (unsigned int)(q & ((1ll << LB) - 1)));
    q >>= LB;
    atomicAdd(base + 2 * stride, (unsigned int)(int)q);
  }
  __device__ static __forceinline__ long long fold(const unsigned int* base, int stride) {
    long long v = (long long)(int)base[2 * stride];
    v = (v << LB) + (long long)base[stride];
    return (v << LB) + (long long)base[0];
  }
};

// The smallest e with b < 2^e (0 for b <= 0), at least -60 so that the
// scales stay finite in float: the exponent field of b read directly (these
// run once per thread and tile, so no library frexp/ldexp calls).
__device__ __forceinline__ int exp_above(double b) {
  if (!(b > 0.0)) return 0;
  const int e = (int)((__double_as_longlong(b) >> 52) & 0x7ff) - 1022;
  return e < -60 ? -60 : e;
}

// exact 2^e, built from its exponent field inside the normal range
template <class T>
__device__ __forceinline__ T pow2(int e);
template <>
__device__ __forceinline__ float pow2<float>(int e) {
  return (e >= -126 && e <= 127) ? __int_as_float((e + 127) << 23) : (float)ldexp(1.0, e);
}
template <>
__device__ __forceinline__ double pow2<double>(int e) {
  return (e >= -1022 && e <= 1023) ? __longlong_as_double((long long)(e + 1023) << 52) : ldexp(1.0, e);
}

}  // namespace

// Fixed-point scales of one tile, one per component c, from m_c = |f_c *
// area / dV| over the tile's entries e0..e1 (blocks of 256 threads).  Only
// order-independent quantities enter them -- the largest m_c, the entry count
// and an integer sum -- so that the scales, like the sums, do not depend on
// the order of the entries.  A scale per component keeps each component's
// relative precision when another one is much larger (a wall force of
// collisions.f90 beside a membrane force).  scale[c] = 2^sh, iscale = 2^-sh.
template <class T>
__device__ __forceinline__ void tile_scales(int e0, int e1, const int* __restrict__ entries,
                                            const ForceRec<T>* __restrict__ frc, T (*s_red)[8],
                                            unsigned long long (*s_sum)[8], T* scale, T* iscale) {
  constexpr bool F32 = sizeof(T) == 4;
  constexpr int QB = Fixed<T>::QB;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  {
    T rmax[3] = {T(0), T(0), T(0)};
    for (int e = e0 + tid; e < e1; e += 256) {
      const ForceRec<T> fo = frc[entries[e]];
#pragma unroll
      for (int c = 0; c < 3; ++c) rmax[c] = fmax(rmax[c], fabs(fo.cf[c]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int c = 0; c < 3; ++c) rmax[c] = fmax(rmax[c], __shfl_xor_sync(0xffffffffu, rmax[c], o));
    if (lane == 0)
#pragma unroll
      for (int c = 0; c < 3; ++c) s_red[c][warp] = rmax[c];
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      rmax[c] = s_red[c][0];
#pragma unroll
      for (int q = 1; q < 8; ++q) rmax[c] = fmax(rmax[c], s_red[c][q]);
    }
    const int cnt = e1 - e0;
    // FP64: |sum| < 2^QB from the largest m_c times the entry count
    int sh[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) sh[c] = QB - exp_above((double)rmax[c] * (double)(F32 ? 0.3 * cnt : cnt));
    // FP32: every single contribution below 2^22 ...
    int sh1[3] = {QB, QB, QB};
    bool need[3] = {false, false, false}, dense = false;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if constexpr (F32) {
        sh1[c] = 22 - exp_above(0.3 * (double)rmax[c]);
        need[c] = sh[c] < sh1[c];
      } else {
        need[c] = cnt > MAXC;  // FP64: the count bound costs precision above one pass of entries
      }
      dense = dense || need[c];
    }
    {
      if (dense) {  // uniform across the CTA: computed from the block-wide maxima
        // ... and, where the count bound would cost precision (more than 2^8
        // entries), |sum| < 2^QB from 0.3 * sum of m_c, taken as an exact
        // integer sum of m_c rounded up to multiples of 2^-12 of the largest
        // m_c's binade (every 3-D weight is below 0.3)
        int exr[3];
        double u[3];
        unsigned long long sm[3] = {0ull, 0ull, 0ull};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          exr[c] = exp_above((double)rmax[c]);  // rmax_c < 2^exr
          u[c] = pow2<double>(12 - exr[c]);
        }
        for (int e = e0 + tid; e < e1; e += 256) {
          const ForceRec<T> fo = frc[entries[e]];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const double v = fabs((double)fo.cf[c]) * u[c];  // < 2^12, exact
            sm[c] += v > 0.0 ? (unsigned long long)ceil(v) : 0ull;
          }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
          for (int c = 0; c < 3; ++c) sm[c] += __shfl_xor_sync(0xffffffffu, sm[c], o);
        if (lane == 0)
#pragma unroll
          for (int c = 0; c < 3; ++c) s_sum[c][warp] = sm[c];
        __syncthreads();
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          unsigned long long t = 0;
#pragma unroll
          for (int q = 0; q < 8; ++q) t += s_sum[c][q];
          if (need[c]) sh[c] = QB - exp_above(0.3 * ((double)t * pow2<double>(exr[c] - 12)));
        }
      }
      if constexpr (F32)
#pragma unroll
        for (int c = 0; c < 3; ++c) sh[c] = min(sh[c], sh1[c]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      scale[c] = pow2<T>(sh[c]);
      iscale[c] = pow2<T>(-sh[c]);
    }
  }
}

// Force records cf = F * (A / dV) (interp_spread.f90:870-874 multiplies by
// area / dVeul in this order).
template <class T>
__global__ void pack_forces_kernel(long n, double dvi, const T* __restrict__ FX, const T* __restrict__ FY,
                                   const T* __restrict__ FZ, const T* __restrict__ A, ForceRec<T>* __restrict__ frc) {
  pdl_enter();
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const T s = A[p] * (T)dvi;
  ForceRec<T> r;
  r.cf[0] = FX[p] * s;
  r.cf[1] = FY[p] * s;
  r.cf[2] = FZ[p] * s;
  r.cf[3] = T(0);
  frc[p] = r;
}

// CTR: cell-centre weights in every direction for every component (the
// indicator's lagr2eulrind, interp_spread.f90:1319-1343) instead of the
// staggered ones.
template <class T, int TX, int TY, int TZ, bool CTR>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2) spread_kernel(IBGrid g, const int* __restrict__ entries,
                                                     const int* __restrict__ starts,
                                                     const PosRec<T>* __restrict__ pos,
                                                     const ForceRec<T>* __restrict__ frc, T* __restrict__ ox,
                                                     T* __restrict__ oy, T* __restrict__ oz) {
  pdl_enter();
  constexpr bool F32 = sizeof(T) == 4;
  constexpr int NC = TX * TY * TZ;
  constexpr int NW = Fixed<T>::NW;
  constexpr int CPT = (NC + 255) / 256;  // cells per thread in the fold / write loops
  constexpr int NT = F32 ? 1 : CPT;      // FP64 keeps running 64-bit totals
  // per (limb, component): the cells, rows padded by one word (row stride
  // RS = TX + 1, plane stride PS), so that lanes whose points sit at the same
  // x in different rows or planes add to different banks, and 32 per-lane
  // trash words that take the contributions falling outside the tile, so
  // that the walk has no branches
  constexpr int RS = TX + 1, PS = RS * TY, NCS = PS * TZ;
  constexpr int NCP = NCS + 32;
  __shared__ __align__(16) unsigned int acc[NW][3][NCP];
  __shared__ T s_red[3][8];
  __shared__ unsigned long long s_sum[3][8];
  long long tot[NT][3];
#pragma unroll
  for (int r = 0; r < NT; ++r) tot[r][0] = tot[r][1] = tot[r][2] = 0;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tile = blockIdx.x;
  const int tx = tile % g.ntx, ty = (tile / g.ntx) % g.nty, tz = tile / (g.ntx * g.nty);
  const int cw = min(TX, g.itot - TX * tx), ch = min(TY, g.jtot - TY * ty), cd = min(TZ, g.ktot - TZ * tz);
  const int i0 = 1 + TX * tx, j0 = 1 + TY * ty, k0 = 1 + TZ * tz;
  const int e0 = starts[tile], e1 = starts[tile + 1];
  T iscale[3] = {T(0), T(0), T(0)};

  if (e1 > e0) {
    for (int q = tid; q < NW * 3 * NCP / 4; q += 256) ((uint4*)&acc[0][0][0])[q] = make_uint4(0u, 0u, 0u, 0u);
    // ---- fixed-point scales, one per component (tile_scales)
    T scale[3];
    tile_scales<T>(e0, e1, entries, frc, s_red, s_sum, scale, iscale);

    // ---- one point per thread, in passes of at most PASS entries
    for (int c0 = e0; c0 < e1; c0 += Fixed<T>::PASS) {
      const int c1 = min(e1, c0 + Fixed<T>::PASS);
      for (int eb = c0; eb < c1; eb += 256) {
        // the nw = ceil(k/32) lowest warps take the k entries of this block,
        // interleaved: lane l of warp w takes entry l*nw + w
        const int k = min(256, c1 - eb), nw = (k + 31) >> 5;
        const int idx = lane * nw + warp;
        if (warp >= nw || idx >= k) continue;
        const int e = eb + idx;
        const int p = entries[e];
        const PosRec<T> rec = pos[p];
        const ForceRec<T> fo = frc[p];
        const int bb[3] = {rec.b[0], rec.b[1], rec.b[2]};
        const T fr[3] = {rec.f[0], rec.f[1], rec.f[2]};
        // scaled forces; each scale is a power of two, so these multiplies are exact
        const T cf[3] = {fo.cf[0] * scale[0], fo.cf[1] * scale[1], fo.cf[2] * scale[2]};
        // 1-D weights: the three nonzero values of the 3-point kernel around the
        // nearest node share one square root.  With r = (nearest node) - c,
        // |r| <= 1/2, s = sqrt(1 - 3 r^2):
        //   phi(r) = (1 + s)/3,  phi(r - 1) = (2 + 3r - s)/6,  phi(r + 1) = (2 - 3r - s)/6
        // (kernel.f90:7-25 evaluated at the three offsets).  Face nodes sit at
        // integer offsets o, cell centres at o - 1/2, o relative to the base cell.
        T wF[3][3], wC[3][3];
        bool hi[3];  // nearest face node is o = 1 (else o = 0)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          delta3_face<T>(fr[d], wF[d], hi[d]);
          delta3_centre<T>(fr[d], wC[d]);
        }
        // local offsets (x) or strides (y, z) of the cells at o = -1..2; -1 when
        // outside the tile.  Face weights cover o = hi-1 .. hi+1, centre weights o = 0..2.
        int lcF[3][3], lcC[3][3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          int lc[4];
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            if (d == 0) {
              const int a = wrap_near(bb[0] + t - 1, g.itot) - i0;
              lc[t] = (a >= 0 && a < cw) ? a : kOut;
            } else if (d == 1) {
              const int b = wrap_near(bb[1] + t - 1, g.jtot) - j0;
              lc[t] = (b >= 0 && b < ch) ? RS * b : kOut;
            } else {
              const int kk = bb[2] + t - 1;
              lc[t] = (kk - k0 >= 0 && kk - k0 < cd && kk >= 1 && kk <= g.ktot) ? PS * (kk - k0) : kOut;
            }
          }
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            lcF[d][q] = hi[d] ? lc[q + 1] : lc[q];
            lcC[d][q] = lc[q + 1];
          }
        }
        // component c has face weights along dimension c, centre weights along
        // the others.  A cell outside the tile has a negative offset sum (kOut
        // in at least one dimension) and goes to this lane's trash word.
        const int trash = NCS + lane;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
#pragma unroll
          for (int iz = 0; iz < 3; ++iz) {
            const int cz_ = (!CTR && c == 2) ? lcF[2][iz] : lcC[2][iz];
            const T wz = (!CTR && c == 2) ? wF[2][iz] : wC[2][iz];
#pragma unroll
            for (int iy = 0; iy < 3; ++iy) {
              const int cyz = cz_ + ((!CTR && c == 1) ? lcF[1][iy] : lcC[1][iy]);
              const T pyz = cf[c] * (((!CTR && c == 1) ? wF[1][iy] : wC[1][iy]) * wz);
#pragma unroll
              for (int ix = 0; ix < 3; ++ix) {
                const int cell = cyz + ((!CTR && c == 0) ? lcF[0][ix] : lcC[0][ix]);
                const T wx = (!CTR && c == 0) ? wF[0][ix] : wC[0][ix];
                // valid cells are below NCS, the negative ones wrap above it
                const unsigned slot = min((unsigned)cell, (unsigned)trash);
                if constexpr (F32) {
                  const float t = fmaf(pyz, wx, kMagic);  // round(pyz * wx) in the low mantissa bits
                  atomicAdd(&acc[0][c][slot], (unsigned int)(__float_as_int(t) - kMagicBits));
                } else {
                  Fixed<T>::add(&acc[0][c][slot], 3 * NCP, pyz * wx);
                }
              }
            }
          }
        }
      }
      __syncthreads();
      if constexpr (!F32) {
        // fold this pass's limbs into 64-bit totals and clear them
#pragma unroll
        for (int r = 0; r < NT; ++r) {
          const int q = tid + 256 * r;
          if (q < NC) {
            const int sq = q % TX + RS * ((q / TX) % TY) + PS * (q / (TX * TY));  // padded slot
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              tot[r][c] += Fixed<double>::fold(&acc[0][c][sq], 3 * NCP);
#pragma unroll
              for (int w = 0; w < NW; ++w) acc[w][c][sq] = 0u;
            }
          }
        }
        __syncthreads();
      }
    }
  }

  // ---- write the cells (32-bit offsets: make_ib_grid caps the field below
  // 2^31 elements); tiles at a domain face also write the periodic halo
  // copies and the zero z-halo planes (the test is uniform across the CTA)
  const bool face = i0 == 1 || i0 + cw - 1 == g.itot || j0 == 1 || j0 + ch - 1 == g.jtot || k0 == 1 ||
                    k0 + cd - 1 == g.ktot;
#pragma unroll
  for (int r = 0; r < CPT; ++r) {
    const int q = tid + 256 * r;
    if (q >= NC) continue;
    const int lx = q % TX, ly = (q / TX) % TY, lz = q / (TX * TY);
    if (lx >= cw || ly >= ch || lz >= cd) continue;
    T vu = T(0), vv = T(0), vw = T(0);
    if (e1 > e0) {
      if constexpr (F32) {
        // one rounding of the fixed-point value; each iscale is a power of two
        const int sq = lx + RS * ly + PS * lz;
        vu = (float)(int)acc[0][0][sq] * iscale[0];
        vv = (float)(int)acc[0][1][sq] * iscale[1];
        vw = (float)(int)acc[0][2][sq] * iscale[2];
      } else {
        vu = (double)tot[r][0] * iscale[0];
        vv = (double)tot[r][1] * iscale[1];
        vw = (double)tot[r][2] * iscale[2];
      }
    }
    const int i = i0 + lx, j = j0 + ly, k = k0 + lz;
    if (!face) {
      const int o = i + g.ldi * (j + g.ldj * k);
      ox[o] = vu;
      oy[o] = vv;
      oz[o] = vw;
      continue;
    }
    int is[2] = {i, -1}, js[2] = {j, -1};
    if (i == g.itot) is[1] = 0;
    if (i == 1) is[1] = g.itot + 1;
    if (j == g.jtot) js[1] = 0;
    if (j == 1) js[1] = g.jtot + 1;
    for (int a = 0; a < 2; ++a) {
      if (is[a] < 0) continue;
      for (int b = 0; b < 2; ++b) {
        if (js[b] < 0) continue;
        const long long o = fidx(is[a], js[b], k, g.ldi, g.ldj);
        ox[o] = vu;
        oy[o] = vv;
        oz[o] = vw;
        if (k == 1) {
          const long long o0 = fidx(is[a], js[b], 0, g.ldi, g.ldj);
          ox[o0] = T(0); oy[o0] = T(0); oz[o0] = T(0);
        }
        if (k == g.ktot) {
          const long long o1 = fidx(is[a], js[b], g.ktot + 1, g.ldi, g.ldj);
          ox[o1] = T(0); oy[o1] = T(0); oz[o1] = T(0);
        }
      }
    }
  }
}

// FP32 spreading on tiles of whole x rows: TY x TZ rows of itot cells (the x
// direction is periodic, so a row tile holds every x cell a stencil can reach
// and needs no x halo).  The fixed-point sums, scales and the walk are those
// of spread_kernel; what changes is the write: each warp writes whole rows of
// the Fortran field, i = 0 .. itot + 1 with both periodic x-halo copies, as
// runs of consecutive words, so that the misaligned 258-float rows of the
// reference layout split 32-byte sectors only at row ends.  Tiles at a y face
// also write the periodic y-halo rows, and tiles at a z wall the zero halo
// planes.  Shared memory (dynamic): 3 components x (itot TY TZ + 32) words.
template <int TY, int TZ>
__global__ void __launch_bounds__(256, 4) spread_rows_kernel(IBGrid g, const int* __restrict__ entries,
                                                             const int* __restrict__ starts,
                                                             const PosRec<float>* __restrict__ pos,
                                                             const ForceRec<float>* __restrict__ frc,
                                                             float* __restrict__ ox, float* __restrict__ oy,
                                                             float* __restrict__ oz) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned int racc[];  // [3][NCP]
  __shared__ float s_red[3][8];
  __shared__ unsigned long long s_sum[3][8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int NX = g.itot, NC = NX * TY * TZ, NCP = NC + 32;
  const int tile = blockIdx.x;
  const int ty = tile % g.nty, tz = tile / g.nty;
  const int ch = min(TY, g.jtot - TY * ty), cd = min(TZ, g.ktot - TZ * tz);
  const int j0 = 1 + TY * ty, k0 = 1 + TZ * tz;
  const int e0 = starts[tile], e1 = starts[tile + 1];
  float iscale[3] = {0.f, 0.f, 0.f};
  if (e1 > e0) {
    for (int q = tid; q < 3 * NCP / 4; q += 256) ((uint4*)racc)[q] = make_uint4(0u, 0u, 0u, 0u);
    float scale[3];
    tile_scales<float>(e0, e1, entries, frc, s_red, s_sum, scale, iscale);
    const int trash = NC + lane;
    for (int eb = e0; eb < e1; eb += 256) {
      const int k = min(256, e1 - eb), nw = (k + 31) >> 5;
      const int idx = lane * nw + warp;
      if (warp >= nw || idx >= k) continue;
      const int p = entries[eb + idx];
      const PosRec<float> rec = pos[p];
      const ForceRec<float> fo = frc[p];
      const float cf[3] = {fo.cf[0] * scale[0], fo.cf[1] * scale[1], fo.cf[2] * scale[2]};
      float wF[3][3], wC[3][3];
      bool hi[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        delta3_face<float>(rec.f[d], wF[d], hi[d]);
        delta3_centre<float>(rec.f[d], wC[d]);
      }
      // cell offsets at o = -1..2 per dimension (kOut outside the tile; x is
      // always inside: the row is whole and periodic)
      int lcF[3][3], lcC[3][3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        int lc[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          if (d == 0) {
            lc[t] = wrap_near(rec.b[0] + t - 1, NX) - 1;
          } else if (d == 1) {
            const int b = wrap_near(rec.b[1] + t - 1, g.jtot) - j0;
            lc[t] = (b >= 0 && b < ch) ? NX * b : kOut;
          } else {
            const int kk = rec.b[2] + t - 1;
            lc[t] = (kk - k0 >= 0 && kk - k0 < cd && kk >= 1 && kk <= g.ktot) ? NX * TY * (kk - k0) : kOut;
          }
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          lcF[d][q] = hi[d] ? lc[q + 1] : lc[q];
          lcC[d][q] = lc[q + 1];
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        unsigned int* a = racc + c * NCP;
#pragma unroll
        for (int iz = 0; iz < 3; ++iz) {
          const int cz_ = c == 2 ? lcF[2][iz] : lcC[2][iz];
          const float wz = c == 2 ? wF[2][iz] : wC[2][iz];
#pragma unroll
          for (int iy = 0; iy < 3; ++iy) {
            const int cyz = cz_ + (c == 1 ? lcF[1][iy] : lcC[1][iy]);
            const float pyz = cf[c] * ((c == 1 ? wF[1][iy] : wC[1][iy]) * wz);
#pragma unroll
            for (int ix = 0; ix < 3; ++ix) {
              const int cell = cyz + (c == 0 ? lcF[0][ix] : lcC[0][ix]);
              const float wx = c == 0 ? wF[0][ix] : wC[0][ix];
              const unsigned slot = min((unsigned)cell, (unsigned)trash);
              const float t = fmaf(pyz, wx, kMagic);
              atomicAdd(&a[slot], (unsigned int)(__float_as_int(t) - kMagicBits));
            }
          }
        }
      }
    }
    __syncthreads();
  }
  // ---- write: one warp per row of the tile, i = 0 .. itot + 1 in runs of 32
  const bool any = e1 > e0;
  const int ldi = g.ldi, ldj = g.ldj;
  for (int r = warp; r < ch * cd; r += 8) {
    const int ly = r % ch, lz = r / ch;
    const int j = j0 + ly, k = k0 + lz;
    // rows this one is copied to: itself and its periodic y-halo image
    const int jh = j == 1 ? g.jtot + 1 : (j == g.jtot ? 0 : -1);
    const int zp = k == 1 ? 0 : (k == g.ktot ? g.ktot + 1 : -1);  // zero wall-halo plane beside it
    const int base = NX * (ly + TY * lz);
    const long long o0 = (long long)ldi * (j + (long long)ldj * k);
    const long long oh = jh >= 0 ? (long long)ldi * (jh + (long long)ldj * k) : -1;
    for (int i = lane; i < ldi; i += 32) {
      const int xi = i == 0 ? NX - 1 : (i == NX + 1 ? 0 : i - 1);
      float vu = 0.f, vv = 0.f, vw = 0.f;
      if (any) {
        vu = (float)(int)racc[base + xi] * iscale[0];
        vv = (float)(int)racc[NCP + base + xi] * iscale[1];
        vw = (float)(int)racc[2 * NCP + base + xi] * iscale[2];
      }
      ox[o0 + i] = vu;
      oy[o0 + i] = vv;
      oz[o0 + i] = vw;
      if (oh >= 0) {
        ox[oh + i] = vu;
        oy[oh + i] = vv;
        oz[oh + i] = vw;
      }
      if (zp >= 0) {
        const long long z0 = (long long)ldi * (j + (long long)ldj * zp);
        ox[z0 + i] = 0.f;
        oy[z0 + i] = 0.f;
        oz[z0 + i] = 0.f;
        if (jh >= 0) {
          const long long z1 = (long long)ldi * (jh + (long long)ldj * zp);
          ox[z1 + i] = 0.f;
          oy[z1 + i] = 0.f;
          oz[z1 + i] = 0.f;
        }
      }
    }
  }
}

// Dynamic shared memory of a row tile (bytes), 0 when it exceeds what one CTA
// can hold.
static size_t rows_smem(int itot, int TY, int TZ) {
  const size_t b = sizeof(unsigned int) * 3 * ((size_t)itot * TY * TZ + 32);
  return b <= kRowTileSmemMax ? b : 0;
}

template <int TY, int TZ>
static cudaError_t spread_rows(const IBGrid& g, const IBWork& w, float* ox, float* oy, float* oz, cudaStream_t st) {
  const size_t smem = rows_smem(g.itot, TY, TZ);
  if (!smem || g.TX != g.itot || g.TY != TY || g.TZ != TZ) return cudaErrorInvalidValue;
  cudaError_t e = smem_limit(spread_rows_kernel<TY, TZ>, smem);
  if (e != cudaSuccess) return e;
  launch_pdl(spread_rows_kernel<TY, TZ>, dim3(g.ntiles), dim3(256), smem, st, g, w.entries, w.starts, (const PosRec<float>*)w.pos,
                                                         (const ForceRec<float>*)w.frc, ox, oy, oz);
  return cudaGetLastError();
}

template <class T, int TX, int TY, int TZ, bool CTR = false>
static void spread_one(const IBGrid& g, const IBWork& w, T* ox, T* oy, T* oz, cudaStream_t st) {
  launch_pdl(spread_kernel<T, TX, TY, TZ, CTR>, dim3(g.ntiles), dim3(256), 0, st, g, w.entries, w.starts, (const PosRec<T>*)w.pos,
                                                               (const ForceRec<T>*)w.frc, ox, oy, oz);
}

template <class T>
cudaError_t launch_pack_forces(const IBGrid& g, long n, const T* FX, const T* FY, const T* FZ, const T* A, IBWork& w,
                               cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  launch_pdl(pack_forces_kernel<T>, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, st, n, g.dvi, FX, FY, FZ, A, (ForceRec<T>*)w.frc);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_spread(const IBGrid& g, const IBWork& w, T* ox, T* oy, T* oz, cudaStream_t st) {
  switch (g.shape) {
    case 0: spread_one<T, 32, 8, 4>(g, w, ox, oy, oz, st); break;
    case 3: spread_one<T, 8, 8, 4>(g, w, ox, oy, oz, st); break;
    case 1:
      if constexpr (sizeof(T) == 4) { spread_one<T, 16, 16, 8>(g, w, ox, oy, oz, st); break; }
      return cudaErrorInvalidValue;
    case 2:
      if constexpr (sizeof(T) == 4) { spread_one<T, 32, 8, 8>(g, w, ox, oy, oz, st); break; }
      return cudaErrorInvalidValue;
    case 4:
      if constexpr (sizeof(T) == 4) return spread_rows<4, 4>(g, w, ox, oy, oz, st);
      return cudaErrorInvalidValue;
    case 5:
      if constexpr (sizeof(T) == 4) return spread_rows<8, 4>(g, w, ox, oy, oz, st);
      return cudaErrorInvalidValue;
    case 6:
      if constexpr (sizeof(T) == 4) { spread_one<T, 32, 16, 4>(g, w, ox, oy, oz, st); break; }
      return cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <>
cudaError_t launch_spread_centred<double>(const IBGrid& g, const IBWork& w, double* ox, double* oy, double* oz,
                                          cudaStream_t st) {
  switch (g.shape) {
    case 0: spread_one<double, 32, 8, 4, true>(g, w, ox, oy, oz, st); break;
    case 3: spread_one<double, 8, 8, 4, true>(g, w, ox, oy, oz, st); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template cudaError_t launch_pack_forces<double>(const IBGrid&, long, const double*, const double*, const double*,
                                                const double*, IBWork&, cudaStream_t);
template cudaError_t launch_pack_forces<float>(const IBGrid&, long, const float*, const float*, const float*,
                                               const float*, IBWork&, cudaStream_t);
template cudaError_t launch_spread<double>(const IBGrid&, const IBWork&, double*, double*, double*, cudaStream_t);
template cudaError_t launch_spread<float>(const IBGrid&, const IBWork&, float*, float*, float*, cudaStream_t);

}  // namespace sg
