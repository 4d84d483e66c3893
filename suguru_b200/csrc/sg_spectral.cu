// sg_spectral.cu -- spherical-harmonic transforms and the Skalak membrane force.
//
// Replaces complagrforces (forcing.f90:11-114) -> cal_spectral_force
// (sph.f90:1523-1755) with its SPHEREPACK TRSSPH/shagc/shsgc transforms, for
// all capsules at once.  The reference's chain per capsule is
//   TRSSPH force grid -> SH grid, analysis (degree < N), synthesis of the
//   tangent basis and its derivatives on the dealias grid, pointwise geometry
//   and mechanics, analysis of force and normals on the dealias grid,
//   truncated synthesis on the SH grid, renormalised normals, surface metric,
//   TRSSPH SH grid -> force grid, area = surfmet * w/sin(theta) * dphi.
// Here the transforms are split into longitude DFTs (CUDA cores, one capsule
// row per warp/block) and batched Legendre contractions over all capsules of
// a degree group (sg_legendre.cu).  TRSSPH-in followed by the SH-grid
// analysis is exact for band-limited data, so it is fused into one analysis
// of the force grid truncated to degree < N; the force filter followed by
// TRSSPH-out is likewise one truncated analysis followed by synthesis.
//
// The reference sphere x = R (sin t sin p, sin t cos p, cos t) (sph.f90:84-86)
// is subtracted from the positions before the transforms and its geometry
// added back analytically, so the transforms only carry the displacement.
#include <algorithm>

#include "sg_common.cuh"
#include "sg_kernels.h"
#include "sg_mechanics.cuh"
#include "sg_umma.cuh"

namespace sg {

template <class T>
constexpr int pidx() {
  return sizeof(T) == 8 ? 0 : 1;
}

// Thread mapping of the staging loops: thread t takes row r = t % RP of every
// (t / RP + k blockDim / RP)-th staged element, so that no loop iteration
// divides by a runtime value; the threads past the last whole group of RP
// stay idle.  Element offsets come from per-item tables in shared memory.
struct StageMap {
  int r, e0, es;
  bool on;
};
__device__ __forceinline__ StageMap stage_map(int RP) {
  StageMap m;
  m.es = (int)blockDim.x / RP;
  m.r = (int)threadIdx.x % RP;
  m.e0 = (int)threadIdx.x / RP;
  m.on = (int)threadIdx.x < m.es * RP;
  return m;
}

// The trig table rows hm < nrow, columns j < H, of a [nrow][ld] global table
// into [nrow][ts] shared rows.
template <class T>
__device__ __forceinline__ void stage_trig(T* dst, int ts, const T* src, int ld, int nrow, int H) {
  const StageMap sm = stage_map(H);
  if (sm.on)
    for (int hm = sm.e0; hm < nrow; hm += sm.es) dst[hm * ts + sm.r] = src[hm * ld + sm.r];
}

// ------------------------------------------------- positions -> Fourier ---
// Persistent CTAs over capsule row ranges; per item the half-turn trig table
// (j < mD/2) is staged once, then rows are taken in chunks of blockDim/(mD/2):
// the displacement d = X - cen - R s(t_i, p_j) in FP64, one thread per pair of
// points j and j + mD/2 (half a turn apart), stored as their sum and
// difference; then the real DFT of shagc (shagc.f:364-380: 2/nlon scaling,
// forward transform carries -sin) for m < N, one warp per (row, component)
// line with lane = m: cos and sin of m (phi + pi) are (-1)^m those of m phi,
// so an even m sums the pair sums and an odd m the pair differences over
// j < mD/2.
// The capsule's centroid (the mean of its points, subtracted before the
// analysis) comes from centroid_kernel, launched just before.
//
// Centroids: one CTA per capsule, 256 strided FP64 sums (the thread's points
// in batches of 8: the 24 loads of a batch are all issued before any is
// summed; these are the step's first reads of the positions, from HBM), then
// added in the same order as one at a time and reduced by a fixed tree, so
// the result does not depend on the launch.
__device__ __forceinline__ void centroid_block(int cap, const CapInfo* __restrict__ caps,
                                               const double* __restrict__ X, const double* __restrict__ Y,
                                               const double* __restrict__ Z, double* __restrict__ cen) {
  __shared__ double s_cen[3][256];
  const int tid = threadIdx.x;
  const CapInfo ci = caps[cap];
  const long long n = 8LL * ci.N * ci.N;
  double sx = 0, sy = 0, sz = 0;
  const double* Xc = X + ci.pt_off;
  const double* Yc = Y + ci.pt_off;
  const double* Zc = Z + ci.pt_off;
  for (long long p0 = tid; p0 < n; p0 += 8LL * blockDim.x) {
    double bx[8], by[8], bz[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const long long p = p0 + (long long)u * blockDim.x;
      const bool in = p < n;
      bx[u] = in ? Xc[p] : 0.0;
      by[u] = in ? Yc[p] : 0.0;
      bz[u] = in ? Zc[p] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      sx += bx[u];
      sy += by[u];
      sz += bz[u];
    }
  }
  __syncthreads();  // the previous capsule's reads of s_cen are done
  s_cen[0][tid] = sx;
  s_cen[1][tid] = sy;
  s_cen[2][tid] = sz;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (tid < o) {
      s_cen[0][tid] += s_cen[0][tid + o];
      s_cen[1][tid] += s_cen[1][tid + o];
      s_cen[2][tid] += s_cen[2][tid + o];
    }
    __syncthreads();
  }
  if (tid < 3) cen[3 * cap + tid] = s_cen[tid][0] / (double)n;
}

__global__ void __launch_bounds__(256) centroid_kernel(int ncap, const CapInfo* __restrict__ caps,
                                                       const double* __restrict__ X, const double* __restrict__ Y,
                                                       const double* __restrict__ Z, double* __restrict__ cen) {
  pdl_enter();
  if ((int)blockIdx.x < ncap) centroid_block(blockIdx.x, caps, X, Y, Z, cen);
}

template <class T>
__device__ __forceinline__ void posfwd_item(const RowWork it,
                                                     const CapInfo* __restrict__ caps,
                                                     const GroupDev* __restrict__ groups, const double* __restrict__ X,
                                                     const double* __restrict__ Y, const double* __restrict__ Z,
                                                     const double* __restrict__ cen) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  {
    const CapInfo ci = caps[it.cap];
    const GroupDev gd = groups[it.group];
    const int N = gd.N, nD = gd.nD, mD = gd.mD, H = mD >> 1, hP = H + 1, lP = 2 * H + 2;
    const int RP = (int)blockDim.x / H > 0 ? (int)blockDim.x / H : 1;
    T* sTrig = (T*)smem_raw;       // [2N][H+1]
    T* sd = sTrig + 2 * N * hP;    // [RP][3][2H+2]: pair sums at [j], differences at [H+1+j]
    const double* lat64 = (const double*)gd.latD[0];
    const double* trig64 = (const double*)gd.trigD[0];
    const T* trig = (const T*)gd.trigD[pidx<T>()];
    const double R = ci.R;
    const double c0 = cen[3 * it.cap], c1 = cen[3 * it.cap + 1], c2 = cen[3 * it.cap + 2];
    T* Fpos = (T*)gd.buf.Fpos + (long long)ci.gidx * 6 * N * nD;
    __syncthreads();  // the previous item's reads of shared memory are done
    stage_trig<T>(sTrig, hP, trig, mD, 2 * N, H);
    for (int rb = it.row0; rb < it.row0 + it.nrows; rb += RP) {
      const int rows = min(RP, it.row0 + it.nrows - rb);
      __syncthreads();
      {
        const int r = tid / H, j = tid - (tid / H) * H;
        if (r < rows) {
          const int i = rb + r;
          const double st = lat64[4 * i], ct = lat64[4 * i + 1];
          const long long p = ci.pt_off + (long long)i * mD + j;
          // the point half a turn on has cos p, sin p of opposite sign
          const double cp = trig64[1 * mD + j], sp = trig64[N * mD + 1 * mD + j];
          const T ax = (T)(X[p] - c0 - R * (st * sp)), bx = (T)(X[p + H] - c0 + R * (st * sp));
          const T ay = (T)(Y[p] - c1 - R * (st * cp)), by = (T)(Y[p + H] - c1 + R * (st * cp));
          const T az = (T)(Z[p] - c2 - R * ct), bz = (T)(Z[p + H] - c2 - R * ct);
          T* o = sd + r * 3 * lP;
          o[0 * lP + j] = ax + bx;
          o[0 * lP + hP + j] = ax - bx;
          o[1 * lP + j] = ay + by;
          o[1 * lP + hP + j] = ay - by;
          o[2 * lP + j] = az + bz;
          o[2 * lP + hP + j] = az - bz;
        }
      }
      __syncthreads();
      const T sfn = T(2) / T(mD);
      // lane p < 2N: trig row p (cos m = p, then sin m = p - N); rows of
      // Fpos are (comp, cos/sin, m), so the output row is c 2N + p
      // one warp per row: one load of the lane's trig value serves the three
      // components
      for (int r = warp; r < rows; r += nwarp) {
        const T* o = sd + r * 3 * lP;
        for (int p = lane; p < 2 * N; p += 32) {
          const int m = p < N ? p : p - N;
          const T* oo = o + ((m & 1) ? hP : 0);
          const T* t = sTrig + p * hP;
          T a[3] = {T(0), T(0), T(0)};
          for (int j = 0; j < H; ++j) {
            const T tt = t[j];
#pragma unroll
            for (int c = 0; c < 3; ++c) a[c] += oo[c * lP + j] * tt;
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) Fpos[(long long)(c * 2 * N + p) * nD + rb + r] = (p < N ? sfn : -sfn) * a[c];
        }
      }
    }
  }
}

template <class T>
__global__ void __launch_bounds__(256) posfwd_kernel(const RowWork* __restrict__ work, int nwork,
                                                     const CapInfo* __restrict__ caps,
                                                     const GroupDev* __restrict__ groups, const double* __restrict__ X,
                                                     const double* __restrict__ Y, const double* __restrict__ Z,
                                                     const double* __restrict__ cen) {
  pdl_enter();
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) posfwd_item<T>(work[w], caps, groups, X, Y, Z, cen);
}

// ------------------------------------------------- membrane pointwise -----
// Staged Legendre output of one dealias row: for each m, the 18 values
// (ccs = 2c + cos/sin, kind = P, dP, d2P) at k = 3 ccs + kind, padded to 20 so
// that a thread reads them with 16-byte loads.
constexpr int kGK = 20;

// The 15 basis sums of one point's longitude synthesis (per component c:
// v1, v2, v11, v12, v22 of cal_co_tang_basis2) for one m, accumulated into acc.
template <class T>
__device__ __forceinline__ void synth_m(const T* g, T cm, T sm, T fm, T (&acc)[5][3]) {
  T v[18];
  if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 x = ((const float4*)g)[q];
      v[4 * q] = x.x; v[4 * q + 1] = x.y; v[4 * q + 2] = x.z; v[4 * q + 3] = x.w;
    }
    const float2 x = ((const float2*)g)[8];
    v[16] = x.x; v[17] = x.y;
  } else {
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const double2 x = ((const double2*)g)[q];
      v[2 * q] = x.x; v[2 * q + 1] = x.y;
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const T P_a = v[6 * c + 0], D_a = v[6 * c + 1], E_a = v[6 * c + 2];  // cos rows
    const T P_b = v[6 * c + 3], D_b = v[6 * c + 4], E_b = v[6 * c + 5];  // sin rows
    const T t0P = P_a * cm - P_b * sm;
    const T t1P = fm * (P_a * (-sm) - P_b * cm);
    acc[0][c] += D_a * cm - D_b * sm;             // vat1 = sum dP * parthe0
    acc[1][c] += t1P;                             // vat2 = sum P * parthe1
    acc[2][c] += E_a * cm - E_b * sm;             // deFvat1(:,1) = sum d2P * parthe0
    acc[3][c] += fm * (D_a * (-sm) - D_b * cm);   // deFvat1(:,2) = sum dP * parthe1
    acc[4][c] += -fm * fm * t0P;                  // deFvat2(:,2) = sum P * parthe2
  }
}

// Geometry and Skalak force of one point from its synthesised sums v (the
// perturbation part) and the reference sphere at (st, ct, cp, sp).
template <class T>
__device__ __forceinline__ void point_force(const T (&v)[5][3], T st, T ct, T cp, T sp, T R, T hf, T csk,
                                            int law, bool normals_only, T* f, T* nrm) {
  Geo<T> Gm;
  // reference sphere: a1 = x_t, a2 = x_p and second derivatives (sph.f90:84-86)
  Gm.a1[0] = R * (ct * sp); Gm.a1[1] = R * (ct * cp); Gm.a1[2] = -R * st;
  Gm.a2[0] = R * (st * cp); Gm.a2[1] = -R * (st * sp); Gm.a2[2] = T(0);
  Gm.d11[0] = -R * (st * sp); Gm.d11[1] = -R * (st * cp); Gm.d11[2] = -R * ct;
  Gm.d12[0] = R * (ct * cp); Gm.d12[1] = -R * (ct * sp); Gm.d12[2] = T(0);
  Gm.d22[0] = -R * (st * sp); Gm.d22[1] = -R * (st * cp); Gm.d22[2] = T(0);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Gm.a1[c] += v[0][c];
    Gm.a2[c] += v[1][c];
    Gm.d11[c] += v[2][c];
    Gm.d12[c] += v[3][c];
    Gm.d22[c] += v[4][c];
  }
  f[0] = f[1] = f[2] = T(0);
  if (normals_only) {
    T cc[3];
    cross3(Gm.a1, Gm.a2, cc);  // sph1.f90:611-651
    const T sm = sqrt(cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2]);
    for (int c = 0; c < 3; ++c) Gm.n[c] = fdiv(cc[c], sm);
  } else {
    geometry<T>(Gm);
    // reference contravariant metric of the sphere: A^11 = 1/R^2,
    // A^22 = 1/(R^2 sin^2 t), d/dt A^22 = -2 cos t / (R^2 sin^3 t)
    const T iR2 = fdiv(T(1), R * R);
    T A[3] = {iR2, fdiv(iR2, st * st), T(0)};
    T Ad[2][3] = {{T(0), fdiv(-T(2) * ct * iR2, st * st * st), T(0)}, {T(0), T(0), T(0)}};
    mechanics<T>(Gm, A, Ad, hf, csk, law, f);
  }
  nrm[0] = Gm.n[0];
  nrm[1] = Gm.n[1];
  nrm[2] = Gm.n[2];
}

// One block per item of `nrows` dealias rows of one capsule.  Synthesises the
// 15 basis fields of cal_co_tang_basis2 (sph3.f90:111-134) from the Legendre
// output G, adds the reference sphere's analytic part, evaluates geometry and
// mechanics, and takes the forward DFT of force and normal.
//
// Half-turn symmetry of the longitude grid (mD = 4N points, phi_{j+mD/2} =
// phi_j + pi): cos and sin of m (phi + pi) are (-1)^m times those of m phi, so
// a thread sums the even-m and odd-m terms of every series separately and gets
// the point j from their sum and the point j + mD/2 from their difference --
// two points for the loads and multiplies of one.  The forward DFT folds the
// same way: the coefficient of an even (odd) m is the sum over j < mD/2 of
// the sum (difference) of the outputs at j and j + mD/2.
//
// Capsules whose force comes from the surrogate (sur_flag[cap] != 0) need only
// the normal here: their force rows are written as zeros and replaced after
// the force analysis.
template <class T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2) membrane_kernel(const RowWork* __restrict__ work, int nwork,
                                                       const CapInfo* __restrict__ caps,
                                                       const GroupDev* __restrict__ groups,
                                                       const int* __restrict__ sur_flag, int* __restrict__ err) {
  pdl_enter();
  (void)err;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const RowWork it = work[w];
    const CapInfo ci = caps[it.cap];
    const T hf = (T)(0.5 * ci.gs), csk = (T)ci.csk;  // hf_gscell = 0.5 gscell (sph.f90:35)
    const bool normals_only = sur_flag && sur_flag[it.cap];
    const GroupDev gd = groups[it.group];
    const int N = gd.N, nD = gd.nD, mD = gd.mD, H = mD >> 1;
    const int RP = (int)blockDim.x / H > 0 ? (int)blockDim.x / H : 1;  // rows per chunk, H threads each
    const int SR = N * kGK + 16 / (int)sizeof(T);  // staged row stride (one 16-byte pad: fewer bank conflicts)
    T* sG = (T*)smem_raw;                  // [RP][SR]
    T* sTrig = sG + RP * SR;               // [2N][H+1]: cos m phi_j (rows m), sin m phi_j (rows N+m), j < H
    T* sOut = sTrig + 2 * N * (H + 1);     // [RP][6][2H+2]: sum over the half turn at [j], difference at [H+1+j]
    int* sOff = (int*)(sOut + RP * 6 * (2 * H + 2));  // [18N] staged offset of element e
    const T* G = (const T*)gd.buf.G + (long long)ci.gidx * (18 * N * nD);  // [ccs][m][kind][lat]
    const T* trig = (const T*)gd.trigD[pidx<T>()];
    const T* lat = (const T*)gd.latD[pidx<T>()];
    T* Fout = (T*)gd.buf.Fout + (long long)ci.gidx * 12 * N * nD;
    const T sfn = T(2) / T(mD);
    const T R = (T)ci.R;
    __syncthreads();  // the previous item's reads of shared memory are done
    stage_trig<T>(sTrig, H + 1, trig, mD, 2 * N, H);
    for (int e = tid; e < 18 * N; e += blockDim.x) {  // e = (ccs N + m) 3 + kind
      const int kind = e % 3, cm_ = e / 3, m = cm_ % N, ccs = cm_ / N;
      sOff[e] = m * kGK + 3 * ccs + kind;
    }
    const StageMap sm = stage_map(RP);
    for (int rb = it.row0; rb < it.row0 + it.nrows; rb += RP) {
      const int rows = min(RP, it.row0 + it.nrows - rb);
      __syncthreads();  // the previous chunk's staged rows and outputs are consumed
      // stage the chunk's rows, transposed to [row][m][3 ccs + kind]; a warp
      // reads runs of RP consecutive latitudes of one (ccs, m, kind)
      if (sm.on && sm.r < rows)
        for (int e = sm.e0; e < 18 * N; e += sm.es) stage_async(&sG[sm.r * SR + sOff[e]], &G[(long long)e * nD + rb + sm.r]);
      stage_wait();
      __syncthreads();
      {
        const int r = tid / H, j = tid - (tid / H) * H;
        if (r < rows) {
          const int i = rb + r;
          T ev[5][3], od[5][3];
#pragma unroll
          for (int a = 0; a < 5; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c) ev[a][c] = od[a][c] = T(0);
          const T* g = sG + r * SR;
          for (int m = 0; m < N; m += 2) {
            synth_m<T>(g + m * kGK, sTrig[m * (H + 1) + j], sTrig[(N + m) * (H + 1) + j], (T)m, ev);
            if (m + 1 < N)
              synth_m<T>(g + (m + 1) * kGK, sTrig[(m + 1) * (H + 1) + j], sTrig[(N + m + 1) * (H + 1) + j],
                         (T)(m + 1), od);
          }
          // point j = even + odd, point j + mD/2 = even - odd
#pragma unroll
          for (int a = 0; a < 5; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const T e = ev[a][c];
              ev[a][c] = e + od[a][c];
              od[a][c] = e - od[a][c];
            }
          const T st = lat[4 * i], ct = lat[4 * i + 1];
          const T cp = sTrig[1 * (H + 1) + j], sp = sTrig[(N + 1) * (H + 1) + j];
          T fa[3], na[3], fb[3], nb[3];
          point_force<T>(ev, st, ct, cp, sp, R, hf, csk, ci.law, normals_only, fa, na);
          point_force<T>(od, st, ct, -cp, -sp, R, hf, csk, ci.law, normals_only, fb, nb);
          T* o = sOut + r * 6 * (2 * H + 2);
          const T va[6] = {fa[0], fa[1], fa[2], na[0], na[1], na[2]};
          const T vb[6] = {fb[0], fb[1], fb[2], nb[0], nb[1], nb[2]};
#pragma unroll
          for (int f = 0; f < 6; ++f) {
            o[f * (2 * H + 2) + j] = va[f] + vb[f];
            o[f * (2 * H + 2) + H + 1 + j] = va[f] - vb[f];
          }
        }
      }
      __syncthreads();
      // forward DFT of the six outputs (force, normal) per row: warp =
      // (row, field) line, lane p < 2N = trig row p (cos m = p, sin m = p - N)
      for (int line = warp; line < rows * 6; line += nwarp) {
        const int f = line % 6, rr = line / 6;
        const T* o = sOut + line * (2 * H + 2);
        for (int p = lane; p < 2 * N; p += 32) {
          const int m = p < N ? p : p - N;
          const T* oo = o + ((m & 1) ? H + 1 : 0);
          const T* t = sTrig + p * (H + 1);
          T a = 0;
          for (int jj = 0; jj < H; ++jj) a += oo[jj] * t[jj];
          Fout[((long long)f * 2 * N + p) * nD + rb + rr] = (p < N ? sfn : -sfn) * a;
        }
      }
    }
  }
}

// ------------------------------------------------- membrane, FP32 pairs ---
// The FP32 membrane kernel with the longitude synthesis and the forward DFT
// on packed pairs (sm_100 f32x2 arithmetic: __ffma2_rn and friends compute
// each lane as an IEEE FP32 operation).  In the synthesis the pair is
// (even m, odd m): the two half-turn sums of membrane_kernel take one
// instruction per operation.  In the forward DFT it is (even j, odd j): two
// partial sums, added at the end.  Staging keeps a pair's 18 values
// interleaved, [m pair][k][m parity], and the trig table of the synthesis
// holds (cos m, cos m+1, sin m, sin m+1) per point, so that a thread reads
// its operands with 16-byte loads; an odd N pads the last pair with zeros.
constexpr int kGP = 36;  // staged floats per m pair: 18 values x (even m, odd m)

__device__ __forceinline__ float2 p2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 p2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 p2add(float2 a, float2 b) { return __fadd2_rn(a, b); }

// synth_m for the m pair (2 mp, 2 mp + 1) at one point: g = the pair's staged
// block, t = (cos, cos, sin, sin) of the two m at the point, fm = (m, m + 1)
__device__ __forceinline__ void synth_pair(const float* g, float4 t, float2 fm, float2 (&acc)[5][3]) {
  const float2 cm = make_float2(t.x, t.y), nsm = make_float2(-t.z, -t.w), ncm = make_float2(-t.x, -t.y);
  const float2 nfm2 = make_float2(-fm.x * fm.x, -fm.y * fm.y);
  const float4* gq = (const float4*)g;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    // k = 6c .. 6c+5: P, dP, d2P of the cos row, then of the sin row
    const float4 x0 = gq[3 * c], x1 = gq[3 * c + 1], x2 = gq[3 * c + 2];
    const float2 P_a = make_float2(x0.x, x0.y), D_a = make_float2(x0.z, x0.w), E_a = make_float2(x1.x, x1.y);
    const float2 P_b = make_float2(x1.z, x1.w), D_b = make_float2(x2.x, x2.y), E_b = make_float2(x2.z, x2.w);
    const float2 t0P = p2fma(P_a, cm, p2mul(P_b, nsm));                      // P_a cm - P_b sm
    const float2 t1P = p2mul(fm, p2fma(P_a, nsm, p2mul(P_b, ncm)));          // m (-P_a sm - P_b cm)
    acc[0][c] = p2fma(D_a, cm, p2fma(D_b, nsm, acc[0][c]));                  // vat1
    acc[1][c] = p2add(acc[1][c], t1P);                                       // vat2
    acc[2][c] = p2fma(E_a, cm, p2fma(E_b, nsm, acc[2][c]));                  // deFvat1(:,1)
    acc[3][c] = p2fma(fm, p2fma(D_a, nsm, p2mul(D_b, ncm)), acc[3][c]);      // deFvat1(:,2)
    acc[4][c] = p2fma(nfm2, t0P, acc[4][c]);                                 // deFvat2(:,2)
  }
}

__device__ __forceinline__ void membrane_item_f2(const RowWork it,
                                                             const CapInfo* __restrict__ caps,
                                                             const GroupDev* __restrict__ groups,
                                                             const int* __restrict__ sur_flag, int* __restrict__ err) {
  (void)err;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  {
    const CapInfo ci = caps[it.cap];
    const float hf = (float)(0.5 * ci.gs), csk = (float)ci.csk;  // hf_gscell = 0.5 gscell (sph.f90:35)
    const bool normals_only = sur_flag && sur_flag[it.cap];
    const GroupDev gd = groups[it.group];
    const int N = gd.N, nD = gd.nD, mD = gd.mD, H = mD >> 1, NP = (N + 1) >> 1;
    const int RP = (int)blockDim.x / H > 0 ? (int)blockDim.x / H : 1;  // rows per chunk, H threads each
    const int SR = NP * kGP + 4;      // staged row stride (one 16-byte pad)
    const int TS = H + 2;             // row stride of the DFT trig table (8-byte aligned rows)
    const int OS = 2 * H + 4;         // output line: half-turn sums at [j], differences at [H + 2 + j]
    float* sG = (float*)smem_raw;                       // [RP][SR]
    float4* sTP = (float4*)(sG + RP * SR);              // [NP][H]
    float* sTrig = (float*)(sTP + NP * H);              // [2N][TS]: cos m phi_j (rows m), sin (rows N + m)
    float* sOut = sTrig + 2 * N * TS;                   // [RP][6][OS]
    int* sOff = (int*)(sOut + RP * 6 * OS);              // [18N] staged offset of element e
    const float* G = (const float*)gd.buf.G + (long long)ci.gidx * (18 * N * nD);  // [ccs][m][kind][lat]
    const float* trig = (const float*)gd.trigD[1];
    const float* lat = (const float*)gd.latD[1];
    float* Fout = (float*)gd.buf.Fout + (long long)ci.gidx * 12 * N * nD;
    const float sfn = 2.0f / (float)mD;
    const float R = (float)ci.R;
    __syncthreads();  // the previous item's reads of shared memory are done
    {
      const StageMap tm = stage_map(H);
      if (tm.on)
        for (int mp = tm.e0; mp < NP; mp += tm.es) {
          const int j = tm.r, m = 2 * mp;
          const bool odd = m + 1 < N;
          sTP[mp * H + j] = make_float4(trig[m * mD + j], odd ? trig[(m + 1) * mD + j] : 0.0f,
                                        trig[(N + m) * mD + j], odd ? trig[(N + m + 1) * mD + j] : 0.0f);
        }
    }
    stage_trig<float>(sTrig, TS, trig, mD, 2 * N, H);
    for (int e = tid; e < 18 * N; e += blockDim.x) {  // e = (ccs N + m) 3 + kind
      const int kind = e % 3, cm_ = e / 3, m = cm_ % N, ccs = cm_ / N;
      sOff[e] = (m >> 1) * kGP + 2 * (3 * ccs + kind) + (m & 1);
    }
    const StageMap sm = stage_map(RP);
    for (int rb = it.row0; rb < it.row0 + it.nrows; rb += RP) {
      const int rows = min(RP, it.row0 + it.nrows - rb);
      __syncthreads();  // the previous chunk's staged rows and outputs are consumed
      // stage the chunk's rows to [row][m pair][k][m parity], k = 3 ccs + kind;
      // a warp reads runs of RP consecutive latitudes of one (ccs, m, kind)
      if (sm.on && sm.r < rows)
        for (int e = sm.e0; e < 18 * N; e += sm.es) stage_async(&sG[sm.r * SR + sOff[e]], &G[(long long)e * nD + rb + sm.r]);
      if (N & 1)
        for (int q = tid; q < 18 * rows; q += blockDim.x) {
          const int r = q / 18, k = q - r * 18;
          sG[r * SR + (N >> 1) * kGP + 2 * k + 1] = 0.0f;
        }
      stage_wait();
      __syncthreads();
      {
        const int r = tid / H, j = tid - (tid / H) * H;
        if (r < rows) {
          const int i = rb + r;
          float2 acc[5][3];
#pragma unroll
          for (int a = 0; a < 5; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[a][c] = make_float2(0.0f, 0.0f);
          const float* g = sG + r * SR;
          for (int mp = 0; mp < NP; ++mp)
            synth_pair(g + mp * kGP, sTP[mp * H + j], make_float2((float)(2 * mp), (float)(2 * mp + 1)), acc);
          // point j = even + odd, point j + mD/2 = even - odd
          float ev[5][3], od[5][3];
#pragma unroll
          for (int a = 0; a < 5; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              ev[a][c] = acc[a][c].x + acc[a][c].y;
              od[a][c] = acc[a][c].x - acc[a][c].y;
            }
          const float st = lat[4 * i], ct = lat[4 * i + 1];
          const float cp = sTrig[1 * TS + j], sp = sTrig[(N + 1) * TS + j];
          float fa[3], na[3], fb[3], nb[3];
          point_force<float>(ev, st, ct, cp, sp, R, hf, csk, ci.law, normals_only, fa, na);
          point_force<float>(od, st, ct, -cp, -sp, R, hf, csk, ci.law, normals_only, fb, nb);
          float* o = sOut + r * 6 * OS;
          const float va[6] = {fa[0], fa[1], fa[2], na[0], na[1], na[2]};
          const float vb[6] = {fb[0], fb[1], fb[2], nb[0], nb[1], nb[2]};
#pragma unroll
          for (int f = 0; f < 6; ++f) {
            o[f * OS + j] = va[f] + vb[f];
            o[f * OS + H + 2 + j] = va[f] - vb[f];
          }
        }
      }
      __syncthreads();
      // forward DFT of the six outputs per row: warp = (row, field triple)
      // line, lane p < 2N = trig row p (cos m = p, sin m = p - N); even and
      // odd j summed as a pair; one load of the lane's trig pair serves the
      // triple's three fields (force or normal)
      for (int line = warp; line < rows * 2; line += nwarp) {
        const int f0 = 3 * (line & 1), rr = line >> 1;
        const float* o = sOut + (rr * 6 + f0) * OS;
        for (int p = lane; p < 2 * N; p += 32) {
          const int m = p < N ? p : p - N;
          const float2* oo = (const float2*)(o + ((m & 1) ? H + 2 : 0));
          const float2* t = (const float2*)(sTrig + p * TS);
          float2 a2[3] = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};
          for (int jj = 0; jj < (H >> 1); ++jj) {
            const float2 tt = t[jj];
#pragma unroll
            for (int f = 0; f < 3; ++f) a2[f] = p2fma(oo[f * (OS >> 1) + jj], tt, a2[f]);
          }
#pragma unroll
          for (int f = 0; f < 3; ++f)
            Fout[((long long)(f0 + f) * 2 * N + p) * nD + rb + rr] = (p < N ? sfn : -sfn) * (a2[f].x + a2[f].y);
        }
      }
    }
  }
}

__global__ void __launch_bounds__(256, 3) membrane_kernel_f2(const RowWork* __restrict__ work, int nwork,
                                                             const CapInfo* __restrict__ caps,
                                                             const GroupDev* __restrict__ groups,
                                                             const int* __restrict__ sur_flag, int* __restrict__ err) {
  pdl_enter();
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) membrane_item_f2(work[w], caps, groups, sur_flag, err);
}

// Shared memory (bytes) of membrane_kernel_f2 for degrees up to nmax: the
// largest over n <= nmax of staged rows RP (NP kGP + 4), the staging offsets
// 18n, the pair trig table
// NP H float4, the DFT trig table 2n (H + 2) and outputs RP 6 (2H + 4), with
// H = 2n, NP = ceil(n / 2) and RP = max(1, 256 / H).
static size_t membrane_f2_smem(int nmax) {
  size_t e = 0;
  for (size_t n = 1; n <= (size_t)nmax; ++n) {
    const size_t H = 2 * n, NP = (n + 1) / 2, RP = 256 / H > 0 ? 256 / H : 1;
    const size_t en = RP * (NP * kGP + 4) + NP * H * 4 + 2 * n * (H + 2) + RP * 6 * (2 * H + 4) + 18 * n + 64;
    if (en > e) e = en;
  }
  return sizeof(float) * e;
}

// ------------------------------------------------- SH-grid stage ----------
// cal_unitO_filter (sph1.f90:1378-1402): truncated normals on the SH grid,
// renormalised; cal_surface_metric_sph__OPT (sph3.f90:186-277): |a1 x a2| on
// the SH grid from the shape coefficients.  Then their forward DFT.
// The SH grid has mO = 2N longitudes, so points j and j + N are half a turn
// apart: one thread per pair, even-m and odd-m sums kept apart (as in the
// membrane kernel), and the forward DFT folded over j < N.
// Staged per (row, m): normal P cos/sin, shape P cos/sin, shape dP cos/sin of
// component c at 6c + 0..5.
constexpr int kSK = 20;

template <class T>
__device__ __forceinline__ void load18(const T* g, T (&v)[18]) {
  if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 x = ((const float4*)g)[q];
      v[4 * q] = x.x; v[4 * q + 1] = x.y; v[4 * q + 2] = x.z; v[4 * q + 3] = x.w;
    }
    const float2 x = ((const float2*)g)[8];
    v[16] = x.x; v[17] = x.y;
  } else {
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const double2 x = ((const double2*)g)[q];
      v[2 * q] = x.x; v[2 * q + 1] = x.y;
    }
  }
}

template <class T>
__device__ __forceinline__ void shgrid_item(const RowWork it,
                                                     const CapInfo* __restrict__ caps,
                                                     const GroupDev* __restrict__ groups, int* __restrict__ err) {
  (void)err;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  {
    const CapInfo ci = caps[it.cap];
    const GroupDev gd = groups[it.group];
    const int N = gd.N, nO = gd.nO, mO = gd.mO, H = mO >> 1, hP = H + 1, lP = 2 * H + 2;
    const int RP = (int)blockDim.x / H > 0 ? (int)blockDim.x / H : 1;
    const int SR = N * kSK + 16 / (int)sizeof(T);
    T* sG = (T*)smem_raw;                 // [RP][SR]
    T* sTrig = sG + RP * SR;              // [2N][H+1]
    T* sOut = sTrig + 2 * N * hP;         // [RP][4][2H+2]
    int* sOff = (int*)(sOut + RP * 4 * lP);  // [18N][2]: staged offset and source row of element e
    const T* GO = (const T*)gd.buf.GO + (long long)ci.gidx * (24 * N * nO);  // [rr][m][kind][lat]
    const T* trig = (const T*)gd.trigO[pidx<T>()];
    const T* lat = (const T*)gd.latO[pidx<T>()];
    T* Fsh = (T*)gd.buf.Fsh + (long long)ci.gidx * 8 * N * nO;
    const T sfn = T(2) / T(mO);
    const T R = (T)ci.R;
    __syncthreads();  // the previous item's reads of shared memory are done
    stage_trig<T>(sTrig, hP, trig, mO, 2 * N, H);
    // staged elements e = (s, c, cs, m) with s = 0 normal P (rr = 2c+cs,
    // kind 0), s = 1 shape P (rr = 2(3+c)+cs, kind 0), s = 2 shape dP (kind 1)
    for (int e = tid; e < 18 * N; e += blockDim.x) {
      const int m = e % N, t = e / N, cs = t & 1, c = (t >> 1) % 3, sk = t / 6;
      const int rr = sk == 0 ? 2 * c + cs : 2 * (3 + c) + cs, kind = sk == 2 ? 1 : 0;
      sOff[2 * e] = m * kSK + 6 * c + 2 * sk + cs;
      sOff[2 * e + 1] = (rr * N + m) * 2 + kind;
    }
    const StageMap sm = stage_map(RP);
    for (int rb = it.row0; rb < it.row0 + it.nrows; rb += RP) {
      const int rows = min(RP, it.row0 + it.nrows - rb);
      __syncthreads();
      if (sm.on && sm.r < rows)
        for (int e = sm.e0; e < 18 * N; e += sm.es)
          stage_async(&sG[sm.r * SR + sOff[2 * e]], &GO[(long long)sOff[2 * e + 1] * nO + rb + sm.r]);
      stage_wait();
      __syncthreads();
      const int r = tid / H, j = tid - (tid / H) * H;
      if (r < rows) {
        const int i = rb + r;
        const T st = lat[4 * i], ct = lat[4 * i + 1];
        T ev[3][3], od[3][3];  // [normal, a1 part, a2 part][c]
#pragma unroll
        for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
          for (int c = 0; c < 3; ++c) ev[a2][c] = od[a2][c] = T(0);
        const T* g = sG + r * SR;
        auto term = [&](int m, T(&acc)[3][3]) {
          const T cm = sTrig[m * hP + j], sm = sTrig[(N + m) * hP + j];
          T v[18];
          load18<T>(g + m * kSK, v);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            acc[0][c] += v[6 * c + 0] * cm - v[6 * c + 1] * sm;
            acc[1][c] += v[6 * c + 4] * cm - v[6 * c + 5] * sm;
            acc[2][c] += (T)m * (v[6 * c + 2] * (-sm) - v[6 * c + 3] * cm);
          }
        };
        for (int m = 0; m < N; m += 2) {
          term(m, ev);
          if (m + 1 < N) term(m + 1, od);
        }
        const T cp = sTrig[1 * hP + j], sp = sTrig[(N + 1) * hP + j];
        T out[2][4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {  // h = 1: half a turn on (cos p, sin p change sign)
          const T sg = h ? T(-1) : T(1);
          T nv[3], a1[3] = {R * (ct * (sg * sp)), R * (ct * (sg * cp)), -R * st},
                   a2[3] = {R * (st * (sg * cp)), -R * (st * (sg * sp)), T(0)};
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            nv[c] = h ? ev[0][c] - od[0][c] : ev[0][c] + od[0][c];
            a1[c] += h ? ev[1][c] - od[1][c] : ev[1][c] + od[1][c];
            a2[c] += h ? ev[2][c] - od[2][c] : ev[2][c] + od[2][c];
          }
          const T rn = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
          T cc[3];
          cross3(a1, a2, cc);
          out[h][0] = fdiv(nv[0], rn);
          out[h][1] = fdiv(nv[1], rn);
          out[h][2] = fdiv(nv[2], rn);
          out[h][3] = sqrt(cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2]);
        }
        T* o = sOut + r * 4 * lP;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          o[f * lP + j] = out[0][f] + out[1][f];
          o[f * lP + hP + j] = out[0][f] - out[1][f];
        }
      }
      __syncthreads();
      // (row, field pair) line per warp: one load of the lane's trig value
      // serves two fields
      for (int line = warp; line < rows * 2; line += nwarp) {
        const int f0 = 2 * (line & 1), rr = line >> 1;
        const T* o = sOut + (rr * 4 + f0) * lP;
        for (int p = lane; p < 2 * N; p += 32) {
          const int m = p < N ? p : p - N;
          const T* oo = o + ((m & 1) ? hP : 0);
          const T* t = sTrig + p * hP;
          T a[2] = {T(0), T(0)};
          for (int jj = 0; jj < H; ++jj) {
            const T tt = t[jj];
            a[0] += oo[jj] * tt;
            a[1] += oo[lP + jj] * tt;
          }
#pragma unroll
          for (int f = 0; f < 2; ++f) Fsh[((long long)(f0 + f) * 2 * N + p) * nO + rb + rr] = (p < N ? sfn : -sfn) * a[f];
        }
      }
    }
  }
}

template <class T>
__global__ void __launch_bounds__(256) shgrid_kernel(const RowWork* __restrict__ work, int nwork,
                                                     const CapInfo* __restrict__ caps,
                                                     const GroupDev* __restrict__ groups, int* __restrict__ err) {
  pdl_enter();
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) shgrid_item<T>(work[w], caps, groups, err);
}

// ------------------------------------------------- final synthesis --------
// TRSSPH SH grid -> force grid of force, normals and surface metric
// (forcing.f90:67-88), area = surfmetDf * wgtdsinf (forcing.f90:91).
// One thread per pair of points half a turn apart (j, j + mD/2), even-m and
// odd-m sums kept apart; the chunk's rows of the Legendre output are staged
// transposed to [row][m][2f + cos/sin] (14 values, padded to 16).
constexpr int kFK = 16;

template <class T>
__device__ __forceinline__ void final_item(const RowWork it,
                                                    const CapInfo* __restrict__ caps,
                                                    const GroupDev* __restrict__ groups, T* __restrict__ FX,
                                                    T* __restrict__ FY, T* __restrict__ FZ, T* __restrict__ NX,
                                                    T* __restrict__ NY, T* __restrict__ NZ, T* __restrict__ AREA,
                                                    ForceRec<T>* __restrict__ frc, double dvi,
                                                    int* __restrict__ err) {
  (void)err;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x;
  {
    const CapInfo ci = caps[it.cap];
    const GroupDev gd = groups[it.group];
    const int N = gd.N, nD = gd.nD, mD = gd.mD, H = mD >> 1, hP = H + 1;
    const int RP = (int)blockDim.x / H > 0 ? (int)blockDim.x / H : 1;
    const int SR = N * kFK + 16 / (int)sizeof(T);
    T* sG = (T*)smem_raw;         // [RP][SR]
    T* sTrig = sG + RP * SR;      // [2N][H+1]
    int* sOff = (int*)(sTrig + 2 * N * hP);  // [14N] staged offset of element e = rr N + m
    const T* GF = (const T*)gd.buf.GF + (long long)ci.gidx * (14 * N * nD);  // [rr][m][lat]
    const T* trig = (const T*)gd.trigD[pidx<T>()];
    const T* lat = (const T*)gd.latD[pidx<T>()];
    __syncthreads();  // the previous item's reads of shared memory are done
    stage_trig<T>(sTrig, hP, trig, mD, 2 * N, H);
    for (int e = tid; e < 14 * N; e += blockDim.x) sOff[e] = (e % N) * kFK + e / N;
    const StageMap sm = stage_map(RP);
    for (int rb = it.row0; rb < it.row0 + it.nrows; rb += RP) {
      const int rows = min(RP, it.row0 + it.nrows - rb);
      __syncthreads();
      if (sm.on && sm.r < rows)
        for (int e = sm.e0; e < 14 * N; e += sm.es) stage_async(&sG[sm.r * SR + sOff[e]], &GF[(long long)e * nD + rb + sm.r]);
      stage_wait();
      __syncthreads();
      const int r = tid / H, j = tid - (tid / H) * H;
      if (r < rows) {
        const int i = rb + r;
        T ev[7], od[7];
#pragma unroll
        for (int f = 0; f < 7; ++f) ev[f] = od[f] = T(0);
        const T* g = sG + r * SR;
        auto term = [&](int m, T(&acc)[7]) {
          const T cm = sTrig[m * hP + j], sm = sTrig[(N + m) * hP + j];
          T v[16];
          if constexpr (sizeof(T) == 4) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const float4 x = ((const float4*)(g + m * kFK))[q];
              v[4 * q] = x.x; v[4 * q + 1] = x.y; v[4 * q + 2] = x.z; v[4 * q + 3] = x.w;
            }
          } else {
#pragma unroll
            for (int q = 0; q < 7; ++q) {
              const double2 x = ((const double2*)(g + m * kFK))[q];
              v[2 * q] = x.x; v[2 * q + 1] = x.y;
            }
          }
#pragma unroll
          for (int f = 0; f < 7; ++f) acc[f] += v[2 * f] * cm - v[2 * f + 1] * sm;
        };
        for (int m = 0; m < N; m += 2) {
          term(m, ev);
          if (m + 1 < N) term(m + 1, od);
        }
        const long long p = ci.pt_off + (long long)i * mD + j;
        const T wa = lat[4 * i + 2];
        FX[p] = ev[0] + od[0];
        FY[p] = ev[1] + od[1];
        FZ[p] = ev[2] + od[2];
        NX[p] = ev[3] + od[3];
        NY[p] = ev[4] + od[4];
        NZ[p] = ev[5] + od[5];
        AREA[p] = (ev[6] + od[6]) * wa;
        FX[p + H] = ev[0] - od[0];
        FY[p + H] = ev[1] - od[1];
        FZ[p + H] = ev[2] - od[2];
        NX[p + H] = ev[3] - od[3];
        NY[p + H] = ev[4] - od[4];
        NZ[p + H] = ev[5] - od[5];
        AREA[p + H] = (ev[6] - od[6]) * wa;
        if (frc) {  // the spread's force records: F * (area / dV), as pack_forces computes them
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const T s = (h ? ev[6] - od[6] : ev[6] + od[6]) * wa * (T)dvi;
            ForceRec<T> rc;
            rc.cf[0] = (h ? ev[0] - od[0] : ev[0] + od[0]) * s;
            rc.cf[1] = (h ? ev[1] - od[1] : ev[1] + od[1]) * s;
            rc.cf[2] = (h ? ev[2] - od[2] : ev[2] + od[2]) * s;
            rc.cf[3] = T(0);
            frc[p + h * H] = rc;
          }
        }
      }
    }
  }
}

template <class T>
__global__ void __launch_bounds__(256) final_kernel(const RowWork* __restrict__ work, int nwork,
                                                    const CapInfo* __restrict__ caps,
                                                    const GroupDev* __restrict__ groups, T* __restrict__ FX,
                                                    T* __restrict__ FY, T* __restrict__ FZ, T* __restrict__ NX,
                                                    T* __restrict__ NY, T* __restrict__ NZ, T* __restrict__ AREA,
                                                    ForceRec<T>* __restrict__ frc, double dvi,
                                                    int* __restrict__ err) {
  pdl_enter();
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) final_item<T>(work[w], caps, groups, FX, FY, FZ, NX, NY, NZ, AREA, frc, dvi, err);
}

// ------------------------------------------------- fused force stage ------
// The whole force stage of one capsule in one CTA (mixed path): centroid,
// longitude DFT of the displacement, the eight Legendre contractions of its
// degree group on CUDA cores in FP32, the membrane, SH-grid and final
// pointwise stages.  Persistent CTAs take whole capsules, largest degree
// first, and run the stages back to back with block barriers between them:
// no launch boundary separates the stages, and on an SM the CTAs of other
// capsules fill one capsule's waits.  The intermediates stay in the same
// per-capsule global buffers as in the staged pipeline (in L2), and every
// pointwise stage is the same device code, so the fused step gives the bits
// of the staged step with FP32 contractions (sg_set_tensor_cores(0)).
//
// One capsule's rows of a problem, all m: D_m[r][j] = sum_{k >= k0}
// A_m[r][k] B_m[j][k] with k0 = m for a synthesis (tri), in the same order
// of k as legendre_kernel.  The capsule's A rows for every m are staged as
// [m][k][r] (its R rows side by side), then thread task (m, j) forms the R
// sums, reading B_m[j][k] from the (L2-resident) FP32 table.
template <int R>
__device__ __forceinline__ void contract_rows(const LegProblem& P, long long gidx, float* sA) {
  const int M = P.M, J = P.J, K = P.K;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const float* A = (const float*)P.A + gidx * P.sAc;
  float* D = (float*)P.D + gidx * P.sDc;
  const float* B = (const float*)P.B;
  __syncthreads();  // the previous stage's reads of shared memory are done
  for (int rm = warp; rm < R * M; rm += nwarp) {
    const int r = rm / M, m = rm - r * M;
    const float* a = A + (long long)r * P.sAr + (long long)m * P.sAm;
    for (int k = lane; k < K; k += 32) sA[(m * K + k) * R + r] = a[k];
  }
  __syncthreads();
  for (int t = tid; t < M * J; t += blockDim.x) {
    const int m = t / J, j = t - m * J;
    const int k0 = P.tri ? m : 0;
    const float* b = B + (long long)m * P.sBm + (long long)j * K;
    const float* a = sA + m * K * R;
    float acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0.0f;
    for (int k = k0; k < K; ++k) {
      const float bk = __ldg(b + k);
#pragma unroll
      for (int r = 0; r < R; ++r) acc[r] += a[k * R + r] * bk;
    }
    float* d = D + (long long)m * P.sDm + j;
#pragma unroll
    for (int r = 0; r < R; ++r) d[(long long)r * P.sDr] = acc[r];
  }
}

__device__ __forceinline__ void contract_capsule(const LegProblem& P, long long gidx, float* sA) {
  switch (P.rpc) {
    case 6: contract_rows<6>(P, gidx, sA); break;
    case 8: contract_rows<8>(P, gidx, sA); break;
    default: contract_rows<12>(P, gidx, sA); break;
  }
}

// Per degree group the problems are, in order, S0 S1 S2 S3a S3b S4 S5a S5b
// (8 g .. 8 g + 7 of probs).
__global__ void __launch_bounds__(256, 2) force_fused_kernel(
    const int* __restrict__ order, int ncap, const CapInfo* __restrict__ caps, const GroupDev* __restrict__ groups,
    const LegProblem* __restrict__ probs, const double* __restrict__ X, const double* __restrict__ Y,
    const double* __restrict__ Z, double* __restrict__ cen, float* __restrict__ FX, float* __restrict__ FY,
    float* __restrict__ FZ, float* __restrict__ NX, float* __restrict__ NY, float* __restrict__ NZ,
    float* __restrict__ AREA, ForceRec<float>* __restrict__ frc, double dvi) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* sA = (float*)smem_raw;
  for (int w = blockIdx.x; w < ncap; w += gridDim.x) {
    const int cap = order[w];
    const CapInfo ci = caps[cap];
    const GroupDev gd = groups[ci.group];
    const LegProblem* pg = probs + 8 * ci.group;
    const RowWork dealias{cap, 0, gd.nD, ci.group}, shgrid{cap, 0, gd.nO, ci.group};
    centroid_block(cap, caps, X, Y, Z, cen);
    __syncthreads();  // the centroid is written
    posfwd_item<float>(dealias, caps, groups, X, Y, Z, cen);
    contract_capsule(pg[0], ci.gidx, sA);  // S0: analysis of the displacement
    contract_capsule(pg[1], ci.gidx, sA);  // S1: P, dP, d2P series on the dealias grid
    contract_capsule(pg[4], ci.gidx, sA);  // S3b: the shape on the SH grid
    membrane_item_f2(dealias, caps, groups, nullptr, nullptr);
    contract_capsule(pg[2], ci.gidx, sA);  // S2: analysis of force and normals
    contract_capsule(pg[3], ci.gidx, sA);  // S3a: the normals on the SH grid
    contract_capsule(pg[6], ci.gidx, sA);  // S5a: the force on the force grid
    shgrid_item<float>(shgrid, caps, groups, nullptr);
    contract_capsule(pg[5], ci.gidx, sA);  // S4: analysis of renormalised normals and surface metric
    contract_capsule(pg[7], ci.gidx, sA);  // S5b: them on the force grid
    final_item<float>(dealias, caps, groups, FX, FY, FZ, NX, NY, NZ, AREA, frc, dvi, nullptr);
  }
}

// ------------------------------------------------- launchers --------------

// Persistent launches: CTAs of 256 threads loop over the capsule work items
// (whole capsules, largest first); the grid is what the SMs hold at once.
constexpr int kPointThreads = 256;

template <class K>
static int persistent_grid(K kernel, size_t smem, int nwork) {
  int dev = 0, sms = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kPointThreads, smem) != cudaSuccess || per < 1)
    per = 1;
  const int g = sms * per;
  return nwork < g ? nwork : g;
}

// Shared memory of the pointwise kernels for degrees up to nmax: the
// capsule's staged input block, the trig table, and per-chunk outputs of at
// most kPointThreads points.
enum PointKernel { kPosfwd, kMembrane, kShgrid, kFinal };
template <class T>
size_t pointwise_smem(int kind, int nmax) {
  const size_t N = nmax;
  size_t e = 0;
  switch (kind) {
    case kPosfwd:
      // half-turn trig table 2n (2n + 1) and RP = max(1, 256 / 2n) rows of
      // 3 (4n + 2) pair sums and differences, largest over n <= N
      for (size_t n = 1; n <= N; ++n) {
        const size_t RP = kPointThreads / (2 * n) > 0 ? kPointThreads / (2 * n) : 1;
        const size_t en = 2 * n * (2 * n + 1) + RP * 3 * (4 * n + 2) + 64;
        if (en > e) e = en;
      }
      break;
    case kMembrane:
      // staged rows RP (n kGK + pad) with RP = max(1, 256 / 2n), 18n staging offsets, the half-turn
      // trig table 2n (2n + 1), outputs RP 6 (4n + 2): the largest over the
      // degrees n <= N (smaller degrees stage more rows per chunk)
      for (size_t n = 1; n <= N; ++n) {
        const size_t RP = kPointThreads / (2 * n) > 0 ? kPointThreads / (2 * n) : 1;
        const size_t en = RP * (n * kGK + 16 / sizeof(T)) + 2 * n * (2 * n + 1) + RP * 6 * (4 * n + 2) +
                          (18 * n * sizeof(int) + sizeof(T) - 1) / sizeof(T) + 64;
        if (en > e) e = en;
      }
      break;
    case kShgrid:
      // staged rows RP (n kSK + pad) with RP = max(1, 256 / n), 36n staging offsets, trig 2n (n + 1),
      // outputs RP 4 (2n + 2)
      for (size_t n = 1; n <= N; ++n) {
        const size_t RP = kPointThreads / n > 0 ? kPointThreads / n : 1;
        const size_t en = RP * (n * kSK + 16 / sizeof(T)) + 2 * n * (n + 1) + RP * 4 * (2 * n + 2) +
                          (36 * n * sizeof(int) + sizeof(T) - 1) / sizeof(T) + 64;
        if (en > e) e = en;
      }
      break;
    default:
      // staged rows RP (n kFK + pad) with RP = max(1, 256 / 2n), 14n staging offsets, trig 2n (2n + 1)
      for (size_t n = 1; n <= N; ++n) {
        const size_t RP = kPointThreads / (2 * n) > 0 ? kPointThreads / (2 * n) : 1;
        const size_t en = RP * (n * kFK + 16 / sizeof(T)) + 2 * n * (2 * n + 1) +
                          (14 * n * sizeof(int) + sizeof(T) - 1) / sizeof(T) + 64;
        if (en > e) e = en;
      }
      break;
  }
  return sizeof(T) * e;
}

template <class T>
cudaError_t launch_posfwd(const RowWork* work, int nwork, const CapInfo* caps, const GroupDev* groups, const double* X,
                          const double* Y, const double* Z, int ncap, double* cen, int nmax, cudaStream_t st) {
  if (nwork <= 0 || ncap <= 0) return cudaSuccess;
  launch_pdl(centroid_kernel, dim3(ncap), dim3(256), 0, st, ncap, caps, X, Y, Z, cen);
  const size_t smem = pointwise_smem<T>(kPosfwd, nmax);
  cudaError_t e = smem_limit(posfwd_kernel<T>, smem);
  if (e != cudaSuccess) return e;
  launch_pdl(posfwd_kernel<T>, dim3(persistent_grid(posfwd_kernel<T>, smem, nwork)), dim3(kPointThreads), smem, st, 
      work, nwork, caps, groups, X, Y, Z, cen);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_membrane(const RowWork* work, int nwork, const CapInfo* caps, const GroupDev* groups,
                            const int* sur_flag, int nmax, int* err, cudaStream_t st) {
  if (nwork <= 0) return cudaSuccess;
  if constexpr (sizeof(T) == 4) {
    const size_t smem = membrane_f2_smem(nmax);
    cudaError_t e = smem_limit(membrane_kernel_f2, smem);
    if (e != cudaSuccess) return e;
    launch_pdl(membrane_kernel_f2, dim3(persistent_grid(membrane_kernel_f2, smem, nwork)), dim3(kPointThreads), smem, st, 
        work, nwork, caps, groups, sur_flag, err);
  } else {
    const size_t smem = pointwise_smem<T>(kMembrane, nmax);
    cudaError_t e = smem_limit(membrane_kernel<T>, smem);
    if (e != cudaSuccess) return e;
    launch_pdl(membrane_kernel<T>, dim3(persistent_grid(membrane_kernel<T>, smem, nwork)), dim3(kPointThreads), smem, st, 
        work, nwork, caps, groups, sur_flag, err);
  }
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_shgrid(const RowWork* work, int nwork, const CapInfo* caps, const GroupDev* groups, int nmax,
                          int* err, cudaStream_t st) {
  if (nwork <= 0) return cudaSuccess;
  const size_t smem = pointwise_smem<T>(kShgrid, nmax);
  cudaError_t e = smem_limit(shgrid_kernel<T>, smem);
  if (e != cudaSuccess) return e;
  launch_pdl(shgrid_kernel<T>, dim3(persistent_grid(shgrid_kernel<T>, smem, nwork)), dim3(kPointThreads), smem, st, work, nwork, caps,
                                                                                                  groups, err);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_final(const RowWork* work, int nwork, const CapInfo* caps, const GroupDev* groups, T* FX, T* FY,
                         T* FZ, T* NX, T* NY, T* NZ, T* AREA, void* frc, double dvi, int nmax, int* err,
                         cudaStream_t st) {
  if (nwork <= 0) return cudaSuccess;
  const size_t smem = pointwise_smem<T>(kFinal, nmax);
  cudaError_t e = smem_limit(final_kernel<T>, smem);
  if (e != cudaSuccess) return e;
  launch_pdl(final_kernel<T>, dim3(persistent_grid(final_kernel<T>, smem, nwork)), dim3(kPointThreads), smem, st, 
      work, nwork, caps, groups, FX, FY, FZ, NX, NY, NZ, AREA, (ForceRec<T>*)frc, dvi, err);
  return cudaGetLastError();
}

// Shared memory of the fused force stage: the largest of its pointwise
// stages' and of the staged A rows (rpc M K floats) of its contractions.
size_t fused_force_smem(int nmax, size_t max_contract_floats);

cudaError_t launch_force_fused(const int* order, int ncap, const CapInfo* caps, const GroupDev* groups,
                               const LegProblem* probs, const double* X, const double* Y, const double* Z, double* cen,
                               float* FX, float* FY, float* FZ, float* NX, float* NY, float* NZ, float* AREA, void* frc,
                               double dvi, int nmax, size_t max_contract_floats, cudaStream_t st) {
  if (ncap <= 0) return cudaSuccess;
  const size_t smem = fused_force_smem(nmax, max_contract_floats);
  cudaError_t e = smem_limit(force_fused_kernel, smem);
  if (e != cudaSuccess) return e;
  force_fused_kernel<<<persistent_grid(force_fused_kernel, smem, ncap), kPointThreads, smem, st>>>(
      order, ncap, caps, groups, probs, X, Y, Z, cen, FX, FY, FZ, NX, NY, NZ, AREA, (ForceRec<float>*)frc, dvi);
  return cudaGetLastError();
}

size_t fused_force_smem(int nmax, size_t max_contract_floats) {
  size_t b = std::max(pointwise_smem<float>(kPosfwd, nmax), membrane_f2_smem(nmax));
  b = std::max(b, pointwise_smem<float>(kShgrid, nmax));
  b = std::max(b, pointwise_smem<float>(kFinal, nmax));
  return std::max(b, sizeof(float) * max_contract_floats);
}

#define SG_INST(T)                                                                                                    \
  template cudaError_t launch_posfwd<T>(const RowWork*, int, const CapInfo*, const GroupDev*, const double*,         \
                                        const double*, const double*, int, double*, int, cudaStream_t);             \
  template cudaError_t launch_membrane<T>(const RowWork*, int, const CapInfo*, const GroupDev*, const int*, int,     \
                                          int*, cudaStream_t);                                                      \
  template cudaError_t launch_shgrid<T>(const RowWork*, int, const CapInfo*, const GroupDev*, int, int*,             \
                                        cudaStream_t);                                                              \
  template cudaError_t launch_final<T>(const RowWork*, int, const CapInfo*, const GroupDev*, T*, T*, T*, T*, T*, T*,  \
                                       T*, void*, double, int, int*, cudaStream_t);
SG_INST(double)
SG_INST(float)

}  // namespace sg
