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
// the tile.  Sums are kept in shared memory as 64-bit fixed point with a
// per-tile power-of-two scale (|sum| < 2^60 from the tile's largest
// contribution times its entry count) and added with integer atomics:
// integer addition is exact and associative, so the field is bitwise
// independent of the order in which threads add (no floating-point atomics,
// deterministic run to run).  Threads walk the stencil starting at a
// lane-dependent offset so that neighbouring points of one warp rarely hit
// the same cell in the same instruction.
#include "sg_common.cuh"
#include "sg_kernels.h"

namespace sg {

namespace {

SG_HD int wrap_near_s(int r, int n) { return r < 1 ? r + n : (r > n ? r - n : r); }

template <class T>
__device__ __forceinline__ long long quant(T v, T scale);
template <>
__device__ __forceinline__ long long quant<float>(float v, float scale) {
  return __float2ll_rn(v * scale);
}
template <>
__device__ __forceinline__ long long quant<double>(double v, double scale) {
  return __double2ll_rn(v * scale);
}

// Fixed-point sums are kept as NW 32-bit limbs of LB bits (the top limb
// signed) so that the shared-memory atomics are native 32-bit adds: with at
// most MAXC contributions per pass no limb sum can overflow
// (LB + log2(MAXC) <= 31).  Between passes the limbs are folded into 64-bit
// registers.  FP32 uses 2 limbs (38-bit fixed point), FP64 3 limbs (57 bits).
constexpr int LB = 19;
constexpr int MAXC = 4096;
template <class T>
struct Limbs {
  static constexpr int NW = sizeof(T) == 8 ? 3 : 2;
  static constexpr int QB = LB * NW - 1;  // |q| < 2^QB
};

template <int NW>
__device__ __forceinline__ void add_limbs(unsigned int* base, int stride, long long q) {
  // q = sum_w limb_w 2^(LB w), lower limbs unsigned, top limb signed
#pragma unroll
  for (int w = 0; w < NW - 1; ++w) {
    atomicAdd(base + w * stride, (unsigned int)(q & ((1ll << LB) - 1)));
    q >>= LB;
  }
  atomicAdd(base + (NW - 1) * stride, (unsigned int)(int)q);
}

template <int NW>
__device__ __forceinline__ long long fold_limbs(const unsigned int* base, int stride) {
  long long v = (long long)(int)base[(NW - 1) * stride];
#pragma unroll
  for (int w = NW - 2; w >= 0; --w) v = (v << LB) + (long long)base[w * stride];
  return v;
}

}  // namespace

template <class T, int TX, int TY, int TZ>
__global__ void __launch_bounds__(256) spread_kernel(IBGrid g, const int* __restrict__ entries,
                                                     const int* __restrict__ starts, const int* __restrict__ bx,
                                                     const int* __restrict__ by, const int* __restrict__ bz,
                                                     const T* __restrict__ fx, const T* __restrict__ fy,
                                                     const T* __restrict__ fz, const T* __restrict__ FX,
                                                     const T* __restrict__ FY, const T* __restrict__ FZ,
                                                     const T* __restrict__ AREA, T* __restrict__ ox,
                                                     T* __restrict__ oy, T* __restrict__ oz) {
  constexpr int NC = TX * TY * TZ;
  constexpr int NW = Limbs<T>::NW;
  constexpr int QB = Limbs<T>::QB < 62 ? Limbs<T>::QB : 62;
  constexpr int CPT = (NC + 255) / 256;  // cells per thread in the fold / write loops
  __shared__ unsigned int acc[NW][3][NC];
  __shared__ T s_red[8];
  long long tot[CPT][3];
#pragma unroll
  for (int r = 0; r < CPT; ++r) tot[r][0] = tot[r][1] = tot[r][2] = 0;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tile = blockIdx.x;
  const int tx = tile % g.ntx, ty = (tile / g.ntx) % g.nty, tz = tile / (g.ntx * g.nty);
  const int cw = min(TX, g.itot - TX * tx), ch = min(TY, g.jtot - TY * ty), cd = min(TZ, g.ktot - TZ * tz);
  const int i0 = 1 + TX * tx, j0 = 1 + TY * ty, k0 = 1 + TZ * tz;
  const int e0 = starts[tile], e1 = starts[tile + 1];
  double iscale = 0.0;

  if (e1 > e0) {
    for (int q = tid; q < NW * 3 * NC; q += 256) (&acc[0][0][0])[q] = 0u;
    // ---- fixed-point scale from the largest |f * area / dV| of the tile
    T mx = T(0);
    for (int e = e0 + tid; e < e1; e += 256) {
      const int p = entries[e];
      const T s = fabs(AREA[p] * (T)g.dvi);
      mx = fmax(mx, fmax(fabs(FX[p]) * s, fmax(fabs(FY[p]) * s, fabs(FZ[p]) * s)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) s_red[warp] = mx;
    __syncthreads();
    mx = s_red[0];
#pragma unroll
    for (int q = 1; q < 8; ++q) mx = fmax(mx, s_red[q]);
    int ex = 0;
    const double bound = (double)mx * (double)(e1 - e0);
    if (bound > 0.0) frexp(bound, &ex);  // bound < 2^ex
    if (ex < -60) ex = -60;              // keeps the scale finite in float
    const T scale = (T)ldexp(1.0, QB - ex);  // |sum| < 2^QB
    iscale = ldexp(1.0, ex - QB);

    // ---- one point per thread, in passes of at most MAXC entries
    for (int c0 = e0; c0 < e1; c0 += MAXC) {
    const int c1 = min(e1, c0 + MAXC);
    // thread t takes entries at offset (37 t) mod 256 of each block of 256,
    // so neighbouring points (adjacent entries) land in different warps
    for (int eb = c0; eb < c1; eb += 256) {
      const int e = eb + ((tid * 37) & 255);
      if (e >= c1) continue;
      const int p = entries[e];
      const int bb[3] = {bx[p], by[p], bz[p]};
      const T fr[3] = {fx[p], fy[p], fz[p]};
      const T s = AREA[p] * (T)g.dvi;  // interp_spread.f90:870-874
      const T cf[3] = {FX[p] * s, FY[p] * s, FZ[p] * s};
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
        const T f = fr[d];
        hi[d] = !(f < T(0.5));
        const T r = (hi[d] ? T(1) : T(0)) - f;
        const T sq = sqrt(T(1) - T(3) * r * r);
        wF[d][0] = (T(2) + T(3) * r - sq) / T(6);
        wF[d][1] = (T(1) + sq) / T(3);
        wF[d][2] = (T(2) - T(3) * r - sq) / T(6);
        const T rc = T(0.5) - f;
        const T sc = sqrt(T(1) - T(3) * rc * rc);
        wC[d][0] = (T(2) + T(3) * rc - sc) / T(6);
        wC[d][1] = (T(1) + sc) / T(3);
        wC[d][2] = (T(2) - T(3) * rc - sc) / T(6);
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
            const int a = wrap_near_s(bb[0] + t - 1, g.itot) - i0;
            lc[t] = (a >= 0 && a < cw) ? a : -1;
          } else if (d == 1) {
            const int b = wrap_near_s(bb[1] + t - 1, g.jtot) - j0;
            lc[t] = (b >= 0 && b < ch) ? TX * b : -1;
          } else {
            const int kk = bb[2] + t - 1;
            lc[t] = (kk - k0 >= 0 && kk - k0 < cd && kk >= 1 && kk <= g.ktot) ? TX * TY * (kk - k0) : -1;
          }
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          lcF[d][q] = hi[d] ? lc[q + 1] : lc[q];
          lcC[d][q] = lc[q + 1];
        }
      }
      // component c has face weights along dimension c, centre weights along the others
#pragma unroll
      for (int c = 0; c < 3; ++c) {
#pragma unroll
        for (int iz = 0; iz < 3; ++iz) {
          const int cz_ = (c == 2) ? lcF[2][iz] : lcC[2][iz];
          if (cz_ < 0) continue;
          const T wz = (c == 2) ? wF[2][iz] : wC[2][iz];
#pragma unroll
          for (int iy = 0; iy < 3; ++iy) {
            const int cy_ = (c == 1) ? lcF[1][iy] : lcC[1][iy];
            if (cy_ < 0) continue;
            const T pyz = cf[c] * (((c == 1) ? wF[1][iy] : wC[1][iy]) * wz);
#pragma unroll
            for (int ix = 0; ix < 3; ++ix) {
              const int cx_ = (c == 0) ? lcF[0][ix] : lcC[0][ix];
              if (cx_ < 0) continue;
              const T wx = (c == 0) ? wF[0][ix] : wC[0][ix];
              add_limbs<NW>(&acc[0][c][cx_ + cy_ + cz_], 3 * NC, quant<T>(pyz * wx, scale));
            }
          }
        }
      }
    }
    __syncthreads();
    // fold this pass's limbs into 64-bit totals and clear them
#pragma unroll
    for (int r = 0; r < CPT; ++r) {
      const int q = tid + 256 * r;
      if (q < NC) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          tot[r][c] += fold_limbs<NW>(&acc[0][c][q], 3 * NC);
#pragma unroll
          for (int w = 0; w < NW; ++w) acc[w][c][q] = 0u;
        }
      }
    }
    __syncthreads();
    }
  }

  // ---- write the cells, their periodic halo copies and the zero z-halo planes
#pragma unroll
  for (int r = 0; r < CPT; ++r) {
    const int q = tid + 256 * r;
    if (q >= NC) continue;
    const int lx = q % TX, ly = (q / TX) % TY, lz = q / (TX * TY);
    if (lx >= cw || ly >= ch || lz >= cd) continue;
    T vu = T(0), vv = T(0), vw = T(0);
    if (e1 > e0) {
      vu = (T)((double)tot[r][0] * iscale);
      vv = (T)((double)tot[r][1] * iscale);
      vw = (T)((double)tot[r][2] * iscale);
    }
    const int i = i0 + lx, j = j0 + ly, k = k0 + lz;
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

template <class T>
cudaError_t launch_spread(const IBGrid& g, const IBWork& w, const T* FX, const T* FY, const T* FZ, const T* A, T* ox,
                          T* oy, T* oz, cudaStream_t st) {
  if (g.TX == 32)
    spread_kernel<T, 32, 8, 4><<<g.ntiles, 256, 0, st>>>(g, w.entries, w.starts, w.bx, w.by, w.bz, (const T*)w.fx,
                                                          (const T*)w.fy, (const T*)w.fz, FX, FY, FZ, A, ox, oy, oz);
  else
    spread_kernel<T, 8, 8, 4><<<g.ntiles, 256, 0, st>>>(g, w.entries, w.starts, w.bx, w.by, w.bz, (const T*)w.fx,
                                                         (const T*)w.fy, (const T*)w.fz, FX, FY, FZ, A, ox, oy, oz);
  return cudaGetLastError();
}

template cudaError_t launch_spread<double>(const IBGrid&, const IBWork&, const double*, const double*, const double*,
                                           const double*, double*, double*, double*, cudaStream_t);
template cudaError_t launch_spread<float>(const IBGrid&, const IBWork&, const float*, const float*, const float*,
                                          const float*, float*, float*, float*, cudaStream_t);

}  // namespace sg
