// sg_ib.cu -- binning, interpolation and deterministic spreading kernels.
// See sg_ib.cuh for the reference routines these replace.
#include "sg_ib.cuh"
#include "sg_kernels.h"

namespace sg {

// ------------------------------------------------------------------ binning
// Storage index of a base-relative stencil cell, periodic in [1, n]: the
// stencil of a point with base b covers b-1 .. b+2 (kernel support |r|<1.5
// for both face and cell-centre locations).
SG_HD int wrap_near(int r, int n) { return r < 1 ? r + n : (r > n ? r - n : r); }

// Tiles touched by the stencil of a point in one periodic dimension: the
// tiles of its first and last cell (the stencil is narrower than a tile).
SG_HD int tiles_1d(int b, int n, int TW, int* t) {
  const int t0 = (wrap_near(b - 1, n) - 1) / TW, t1 = (wrap_near(b + 2, n) - 1) / TW;
  t[0] = t0;
  t[1] = t1;
  return t0 == t1 ? 1 : 2;
}
// Non-periodic z: cells clipped to [1, ktot] (interp_spread.f90:346-351).
SG_HD int tiles_z(int b, int ktot, int TW, int* t) {
  const int lo = max(b - 1, 1), hi = min(b + 2, ktot);
  if (lo > hi) return 0;
  t[0] = (lo - 1) / TW;
  t[1] = (hi - 1) / TW;
  return t[0] == t[1] ? 1 : 2;
}

// One thread per point: base indices, fractional offsets, and one entry per
// tile that its stencil reaches.
template <class T>
__global__ void bin_points_kernel(IBGrid g, long n, const double* __restrict__ X, const double* __restrict__ Y,
                                  const double* __restrict__ Z, int* __restrict__ bx, int* __restrict__ by,
                                  int* __restrict__ bz, T* __restrict__ fx, T* __restrict__ fy, T* __restrict__ fz,
                                  int* __restrict__ counts) {
  long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  // interp_spread.f90:337-339: coorxfp = x * dxi (boundleftmyid = 0 on one domain)
  const double cx = X[p] * g.dxi, cy = Y[p] * g.dyi, cz = Z[p] * g.dzi;
  const double ffx = floor(cx), ffy = floor(cy), ffz = floor(cz);
  const long long ix = (long long)ffx, iy = (long long)ffy, iz = (long long)ffz;
  const int wx = (int)(((ix % g.itot) + g.itot) % g.itot);
  const int wy = (int)(((iy % g.jtot) + g.jtot) % g.jtot);
  const int zc = (int)(iz < -4 ? -4 : (iz > g.ktot + 4 ? g.ktot + 4 : iz));
  bx[p] = wx;
  by[p] = wy;
  bz[p] = zc;
  fx[p] = (T)(cx - ffx);
  fy[p] = (T)(cy - ffy);
  fz[p] = (T)(cz - ffz);
  int tx[2], ty[2], tz[2];
  const int nx = tiles_1d(wx, g.itot, g.TX, tx), ny = tiles_1d(wy, g.jtot, g.TY, ty), nz = tiles_z(zc, g.ktot, g.TZ, tz);
  for (int c = 0; c < nz; ++c)
    for (int b = 0; b < ny; ++b)
      for (int a = 0; a < nx; ++a) atomicAdd(&counts[tx[a] + g.ntx * (ty[b] + g.nty * tz[c])], 1);
}

// Exclusive scan of tile counts by one block; starts has ntiles+1 entries.
__global__ void scan_counts_kernel(int ntiles, const int* __restrict__ counts, int* __restrict__ starts,
                                   int* __restrict__ fill) {
  __shared__ int s_part[1024];
  const int T = blockDim.x, t = threadIdx.x;
  const int per = (ntiles + T - 1) / T;
  const int lo = t * per, hi = min(ntiles, lo + per);
  int sum = 0;
  for (int i = lo; i < hi; ++i) sum += counts[i];
  s_part[t] = sum;
  __syncthreads();
  for (int off = 1; off < T; off <<= 1) {
    int v = (t >= off) ? s_part[t - off] : 0;
    __syncthreads();
    s_part[t] += v;
    __syncthreads();
  }
  int run = s_part[t] - sum;
  for (int i = lo; i < hi; ++i) {
    starts[i] = run;
    fill[i] = 0;
    run += counts[i];
  }
  if (t == T - 1) starts[ntiles] = s_part[T - 1];
}

__global__ void bin_scatter_kernel(IBGrid g, long n, const int* __restrict__ bx, const int* __restrict__ by,
                                   const int* __restrict__ bz, const int* __restrict__ starts, int* __restrict__ fill,
                                   int* __restrict__ entries) {
  long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int tx[2], ty[2], tz[2];
  const int nx = tiles_1d(bx[p], g.itot, g.TX, tx), ny = tiles_1d(by[p], g.jtot, g.TY, ty);
  const int nz = tiles_z(bz[p], g.ktot, g.TZ, tz);
  for (int c = 0; c < nz; ++c)
    for (int b = 0; b < ny; ++b)
      for (int a = 0; a < nx; ++a) {
        const int t = tx[a] + g.ntx * (ty[b] + g.nty * tz[c]);
        entries[starts[t] + atomicAdd(&fill[t], 1)] = (int)p;
      }
}

// ------------------------------------------------------------------ interp
// eulr2lagr hot loop (interp_spread.f90:335-378) as a per-point gather in the
// reference's point order (consecutive points share cache lines):
// u at faces i*dx (kernel(i-c)), cell centres at (i-0.5)dx (kernel(i-0.5-c)).
template <class T>
__global__ void __launch_bounds__(256) interp_kernel(IBGrid g, long n, const int* __restrict__ bx,
                                                     const int* __restrict__ by, const int* __restrict__ bz,
                                                     const T* __restrict__ fx, const T* __restrict__ fy,
                                                     const T* __restrict__ fz, const T* __restrict__ u,
                                                     const T* __restrict__ v, const T* __restrict__ w,
                                                     T* __restrict__ U, T* __restrict__ V, T* __restrict__ W) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int b0 = bx[p], b1 = by[p], b2 = bz[p];
  const T f0 = fx[p], f1 = fy[p], f2 = fz[p];
  T wfx[4], wcx[4], wfy[4], wcy[4], wfz[4], wcz[4];
  int ii[4], jj[4], kk[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    wfx[t] = delta3<T>(T(t - 1) - f0);
    wcx[t] = delta3<T>(T(t - 1) - T(0.5) - f0);
    wfy[t] = delta3<T>(T(t - 1) - f1);
    wcy[t] = delta3<T>(T(t - 1) - T(0.5) - f1);
    wfz[t] = delta3<T>(T(t - 1) - f2);
    wcz[t] = delta3<T>(T(t - 1) - T(0.5) - f2);
    ii[t] = wrap_near(b0 + t - 1, g.itot);
    jj[t] = wrap_near(b1 + t - 1, g.jtot);
    const int k = b2 + t - 1;
    kk[t] = (k >= 1 && k <= g.ktot) ? k : -1;  // window clipped to [1,kmax]
  }
  T su = 0, sv = 0, sw = 0;
#pragma unroll
  for (int tk = 0; tk < 4; ++tk) {
    if (kk[tk] < 0) continue;
#pragma unroll
    for (int tj = 0; tj < 4; ++tj) {
      const long long row = (long long)g.ldi * ((long long)jj[tj] + (long long)g.ldj * kk[tk]);
#pragma unroll
      for (int ti = 0; ti < 4; ++ti) {
        const long long o = row + ii[ti];
        const T wu = wfx[ti] * wcy[tj] * wcz[tk];
        const T wv = wcx[ti] * wfy[tj] * wcz[tk];
        const T ww = wcx[ti] * wcy[tj] * wfz[tk];
        if (wu != T(0)) su += u[o] * wu;
        if (wv != T(0)) sv += v[o] * wv;
        if (ww != T(0)) sw += w[o] * ww;
      }
    }
  }
  U[p] = su;
  V[p] = sv;
  W[p] = sw;
}

// ------------------------------------------------------------------ launchers
template <class T>
cudaError_t launch_bin(const IBGrid& g, long n, const double* X, const double* Y, const double* Z, IBWork& w,
                       cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(w.counts, 0, sizeof(int) * g.ntiles, st);
  if (e != cudaSuccess) return e;
  if (n > 0)
    bin_points_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, n, X, Y, Z, w.bx, w.by, w.bz, (T*)w.fx,
                                                                       (T*)w.fy, (T*)w.fz, w.counts);
  scan_counts_kernel<<<1, 1024, 0, st>>>(g.ntiles, w.counts, w.starts, w.fill);
  if (n > 0)
    bin_scatter_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, n, w.bx, w.by, w.bz, w.starts, w.fill,
                                                                     w.entries);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_interp(const IBGrid& g, long n, const IBWork& w, const T* u, const T* v, const T* ww, T* U, T* V,
                          T* W, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  interp_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, n, w.bx, w.by, w.bz, (const T*)w.fx,
                                                                 (const T*)w.fy, (const T*)w.fz, u, v, ww, U, V, W);
  return cudaGetLastError();
}

template cudaError_t launch_bin<double>(const IBGrid&, long, const double*, const double*, const double*, IBWork&,
                                        cudaStream_t);
template cudaError_t launch_bin<float>(const IBGrid&, long, const double*, const double*, const double*, IBWork&,
                                       cudaStream_t);
template cudaError_t launch_interp<double>(const IBGrid&, long, const IBWork&, const double*, const double*,
                                           const double*, double*, double*, double*, cudaStream_t);
template cudaError_t launch_interp<float>(const IBGrid&, long, const IBWork&, const float*, const float*, const float*,
                                          float*, float*, float*, cudaStream_t);

bool make_ib_grid(int itot, int jtot, int ktot, double lx, double ly, double lz, IBGrid& g) {
  if (itot < 8 || jtot < 8 || ktot < 1) return false;
  g.itot = itot;
  g.jtot = jtot;
  g.ktot = ktot;
  g.ldi = itot + 2;
  g.ldj = jtot + 2;
  g.ldk = ktot + 2;
  double dx = lx / itot, dy = ly / jtot, dz = lz / ktot;
  g.dxi = 1.0 / dx;
  g.dyi = 1.0 / dy;
  g.dzi = 1.0 / dz;
  g.dvi = 1.0 / (dx * dy * dz);
  // tile shape: 32 x 8 x 4 (128-byte rows in x) or 8 x 8 x 4 on narrow grids
  if (itot >= 32) {
    g.TX = 32; g.TY = 8; g.TZ = 4;
  } else {
    g.TX = 8; g.TY = 8; g.TZ = 4;
  }
  g.ntx = (itot + g.TX - 1) / g.TX;
  g.nty = (jtot + g.TY - 1) / g.TY;
  g.ntz = (ktot + g.TZ - 1) / g.TZ;
  g.ntiles = g.ntx * g.nty * g.ntz;
  return true;
}

}  // namespace sg
