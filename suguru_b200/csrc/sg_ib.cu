// sg_ib.cu -- binning, interpolation and deterministic spreading kernels.
// See sg_ib.cuh for the reference routines these replace.
#include "sg_ib.cuh"
#include "sg_kernels.h"

namespace sg {

// ------------------------------------------------------------------ binning
// The stencil of a point with base b covers b-1 .. b+2 (kernel support
// |r| < 1.5 for both face and cell-centre locations); wrap_near gives the
// periodic storage index in [1, n].

// Tiles touched by the stencil of a point in one periodic dimension: the
// tiles of its first and last cell (the stencil is narrower than a tile, and
// make_ib_grid keeps the last tile at 3 cells or more, so that a stencil
// that wraps around the periodic end still meets two tiles at most).
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

// Tile of stencil slot s (0..7: z, y, x halves) of a point, or -1.
SG_HD int slot_tile(const IBGrid& g, int s, int nx, int ny, int nz, const int* tx, const int* ty, const int* tz) {
  const int a = s & 1, b = (s >> 1) & 1, c = s >> 2;
  if (a >= nx || b >= ny || c >= nz) return -1;
  return tx[a] + g.ntx * (ty[b] + g.nty * tz[c]);
}

// Periodic wrap of an integer-valued double into [0, n) without 64-bit
// integer division (exact for |v| < 2^52).
__device__ __forceinline__ int wrap_cell(double v, int n) {
  int w = (int)(v - floor(v / (double)n) * (double)n);
  return w < 0 ? w + n : (w >= n ? w - n : w);
}

// One thread per point: base indices, fractional offsets, and one entry per
// tile that its stencil reaches.  Lanes of a warp that hit the same tile
// (neighbouring points usually do) are counted by one atomic.
template <class T>
__global__ void bin_points_kernel(IBGrid g, long n, const double* __restrict__ X, const double* __restrict__ Y,
                                  const double* __restrict__ Z, PosRec<T>* __restrict__ pos,
                                  int* __restrict__ counts) {
  pdl_enter();
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = p < n;
  int tx[2] = {0, 0}, ty[2] = {0, 0}, tz[2] = {0, 0}, nx = 0, ny = 0, nz = 0;
  if (valid) {
    // interp_spread.f90:337-339: coorxfp = x * dxi (boundleftmyid = 0 on one domain)
    const double cx = X[p] * g.dxi, cy = Y[p] * g.dyi, cz = Z[p] * g.dzi;
    const double ffx = floor(cx), ffy = floor(cy), ffz = floor(cz);
    const int wx = wrap_cell(ffx, g.itot), wy = wrap_cell(ffy, g.jtot);
    const int zc = (int)(ffz < -4.0 ? -4.0 : (ffz > g.ktot + 4.0 ? g.ktot + 4.0 : ffz));
    PosRec<T> r;
    r.b[0] = wx;
    r.b[1] = wy;
    r.b[2] = zc;
    r.b[3] = 0;
    r.f[0] = (T)(cx - ffx);
    r.f[1] = (T)(cy - ffy);
    r.f[2] = (T)(cz - ffz);
    r.f[3] = T(0);
    pos[p] = r;
    nx = tiles_1d(wx, g.itot, g.TX, tx);
    ny = tiles_1d(wy, g.jtot, g.TY, ty);
    nz = tiles_z(zc, g.ktot, g.TZ, tz);
  }
  const unsigned lane = threadIdx.x & 31;
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const int t = slot_tile(g, s, nx, ny, nz, tx, ty, tz);
    const unsigned same = __match_any_sync(0xffffffffu, t);
    if (t >= 0 && lane == (unsigned)(__ffs(same) - 1)) atomicAdd(&counts[t], __popc(same));
  }
}

// Exclusive scan of tile counts by one block of 1024 threads; starts has
// ntiles+1 entries.  The tiles go in chunks of 1024 x 8: thread t owns the 8
// consecutive tiles from chunk + 8t (two 16-byte loads and stores, a warp's
// accesses contiguous), the block scans the 1024 run totals (warp shuffles,
// then one warp over the 32 warp totals) and each thread writes its run's
// starts from its offset plus the running total of the earlier chunks.
__global__ void __launch_bounds__(1024) scan_counts_kernel(int ntiles, const int* __restrict__ counts,
                                                           int* __restrict__ starts, int* __restrict__ fill) {
  pdl_enter();
  constexpr int V = 8;
  __shared__ int warp_sum[32];
  __shared__ int s_carry;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t == 0) s_carry = 0;
  for (int c0 = 0; c0 < ntiles; c0 += 1024 * V) {
    const int b0 = c0 + t * V;
    int v[V];
    if (b0 + V <= ntiles) {
      const int4 lo = *(const int4*)(counts + b0), hi = *(const int4*)(counts + b0 + 4);
      v[0] = lo.x; v[1] = lo.y; v[2] = lo.z; v[3] = lo.w; v[4] = hi.x; v[5] = hi.y; v[6] = hi.z; v[7] = hi.w;
    } else {
#pragma unroll
      for (int q = 0; q < V; ++q) v[q] = b0 + q < ntiles ? counts[b0 + q] : 0;
    }
    int run = 0;
#pragma unroll
    for (int q = 0; q < V; ++q) run += v[q];
    int x = run;  // inclusive scan of the run totals within the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[warp] = x;
    __syncthreads();  // the warp totals, and s_carry from the previous chunk
    if (warp == 0) {
      int w = warp_sum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      warp_sum[lane] = w;
    }
    __syncthreads();
    const int carry = s_carry, chunk_total = warp_sum[31];
    int excl = carry + (warp > 0 ? warp_sum[warp - 1] : 0) + x - run;
    int st[V];
#pragma unroll
    for (int q = 0; q < V; ++q) {
      st[q] = excl;
      excl += v[q];
    }
    if (b0 + V <= ntiles) {
      *(int4*)(starts + b0) = make_int4(st[0], st[1], st[2], st[3]);
      *(int4*)(starts + b0 + 4) = make_int4(st[4], st[5], st[6], st[7]);
      *(int4*)(fill + b0) = make_int4(0, 0, 0, 0);
      *(int4*)(fill + b0 + 4) = make_int4(0, 0, 0, 0);
    } else {
#pragma unroll
      for (int q = 0; q < V; ++q)
        if (b0 + q < ntiles) {
          starts[b0 + q] = st[q];
          fill[b0 + q] = 0;
        }
    }
    __syncthreads();  // every thread has read s_carry and warp_sum
    if (t == 0) s_carry = carry + chunk_total;
  }
  __syncthreads();
  if (t == 0) starts[ntiles] = s_carry;
}

template <class T>
__global__ void bin_scatter_kernel(IBGrid g, long n, const PosRec<T>* __restrict__ pos,
                                   const int* __restrict__ starts, int* __restrict__ fill, int* __restrict__ entries) {
  pdl_enter();
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int tx[2] = {0, 0}, ty[2] = {0, 0}, tz[2] = {0, 0}, nx = 0, ny = 0, nz = 0;
  if (p < n) {
    const int4 b = *(const int4*)pos[p].b;
    nx = tiles_1d(b.x, g.itot, g.TX, tx);
    ny = tiles_1d(b.y, g.jtot, g.TY, ty);
    nz = tiles_z(b.z, g.ktot, g.TZ, tz);
  }
  const unsigned lane = threadIdx.x & 31, lt = (1u << lane) - 1u;
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const int t = slot_tile(g, s, nx, ny, nz, tx, ty, tz);
    // lanes with the same tile take consecutive slots reserved by their leader
    const unsigned same = __match_any_sync(0xffffffffu, t);
    const int leader = __ffs(same) - 1;
    int base = 0;
    if (t >= 0 && (int)lane == leader) base = atomicAdd(&fill[t], __popc(same));
    base = __shfl_sync(same, base, leader);
    if (t >= 0) {
      const int slot = starts[t] + base + __popc(same & lt);
      if (slot < starts[t + 1]) entries[slot] = (int)p;  // counts and entries agree by construction
    }
  }
}

// ------------------------------------------------------------------ interp
// eulr2lagr hot loop (interp_spread.f90:335-378) as a gather: one thread per
// (component, point), component-major, so that a warp takes 32 consecutive
// points (consecutive points share cache lines) of one component and each
// thread keeps only its component's 27 loads in flight.  u sits at faces i*dx
// (kernel(i-c)), cell centres at (i-0.5)dx (kernel(i-0.5-c)); each component
// has 3 x 3 x 3 nonzero weights, face weights along its own direction and
// centre weights along the other two (delta3_face/_centre).  z-levels outside
// [1,kmax] are skipped (interp_spread.f90:346-351).
template <class T>
__global__ void __launch_bounds__(256) interp_kernel(IBGrid g, long n, const PosRec<T>* __restrict__ pos,
                                                     const T* __restrict__ u, const T* __restrict__ v,
                                                     const T* __restrict__ w, T* __restrict__ U, T* __restrict__ V,
                                                     T* __restrict__ W) {
  pdl_enter();
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * n) return;
  const int c = (int)(t / n);
  const long p = t - (long)c * n;
  const PosRec<T> rec = pos[p];
  // weights along each dimension: face weights along c (nearest face node
  // o = hi, nodes o = hi-1 .. hi+1), centre weights otherwise (o = 0..2)
  T wt[3][3];
  int o0[3];  // first node offset (o) per dimension
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d == c) {
      bool hi;
      delta3_face<T>(rec.f[d], wt[d], hi);
      o0[d] = hi ? 0 : -1;
    } else {
      delta3_centre<T>(rec.f[d], wt[d]);
      o0[d] = 0;
    }
  }
  // storage offsets of the three nodes per dimension (periodic x, y; z read
  // at the nearest level inside [1, kmax] and weighted by zero outside, so
  // that the 27 loads are independent; 32-bit: make_ib_grid caps the field
  // at 2^31 - 1 elements)
  int ox[3], oy[3], oz[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    ox[q] = wrap_near(rec.b[0] + o0[0] + q, g.itot);
    oy[q] = g.ldi * wrap_near(rec.b[1] + o0[1] + q, g.jtot);
    const int k = rec.b[2] + o0[2] + q;
    if (k < 1 || k > g.ktot) wt[2][q] = T(0);
    oz[q] = g.ldi * g.ldj * (k < 1 ? 1 : (k > g.ktot ? g.ktot : k));
  }
  const T* src = c == 0 ? u : (c == 1 ? v : w);
  T sum = T(0);
#pragma unroll
  for (int tz = 0; tz < 3; ++tz)
#pragma unroll
    for (int ty = 0; ty < 3; ++ty) {
      const T wyz = wt[1][ty] * wt[2][tz];
      const T* row = src + oz[tz] + oy[ty];
#pragma unroll
      for (int tx = 0; tx < 3; ++tx) sum += row[ox[tx]] * (wt[0][tx] * wyz);
    }
  (c == 0 ? U : (c == 1 ? V : W))[p] = sum;
}

// ------------------------------------------------------------------ launchers
template <class T>
cudaError_t launch_bin(const IBGrid& g, long n, const double* X, const double* Y, const double* Z, IBWork& w,
                       cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(w.counts, 0, sizeof(int) * g.ntiles, st);
  if (e != cudaSuccess) return e;
  if (n > 0)
    launch_pdl(bin_points_kernel<T>, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, st, g, n, X, Y, Z, (PosRec<T>*)w.pos, w.counts);
  launch_pdl(scan_counts_kernel, dim3(1), dim3(1024), 0, st, g.ntiles, w.counts, w.starts, w.fill);
  if (n > 0)
    launch_pdl(bin_scatter_kernel<T>, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, st, g, n, (const PosRec<T>*)w.pos, w.starts,
                                                                        w.fill, w.entries);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_interp(const IBGrid& g, long n, const IBWork& w, const T* u, const T* v, const T* ww, T* U, T* V,
                          T* W, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  launch_pdl(interp_kernel<T>, dim3((unsigned)((3 * n + 255) / 256)), dim3(256), 0, st, g, n, (const PosRec<T>*)w.pos, u, v, ww, U, V,
                                                                     W);
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

bool make_ib_grid(int itot, int jtot, int ktot, double lx, double ly, double lz, IBGrid& g, int shape,
                  unsigned allowed) {
  if (itot < 8 || jtot < 8 || ktot < 1) return false;
  if (shape >= kNumTileShapes) return false;
  if (shape >= 0 && !((allowed >> shape) & 1u)) return false;
  // a last tile of 1 or 2 cells in a periodic dimension would let a
  // stencil wrap across three tiles
  auto fits = [&](int s) {
    const TileShape& t = kTileShapes[s];
    if (t.TX == 0 && 4ull * 3 * ((unsigned long long)itot * t.TY * t.TZ + 32) > kRowTileSmemMax) return false;
    const int rx = t.TX ? itot % t.TX : 0, ry = jtot % t.TY;
    return ((allowed >> s) & 1u) && rx != 1 && rx != 2 && ry != 1 && ry != 2;
  };
  if (shape < 0) {
    // default tile shape: 32 x 8 x 4 (128-byte rows in x), 8 x 8 x 4 on
    // narrow grids, else the first shape that fits
    const int order[4] = {itot >= 32 ? 0 : 3, 2, 1, 3};
    for (int s : order)
      if (fits(s)) {
        shape = s;
        break;
      }
    if (shape < 0) return false;
  }
  if (!fits(shape)) return false;
  if ((long long)(itot + 2) * (jtot + 2) * (ktot + 2) > 2147483647LL) return false;  // 32-bit offsets
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
  g.shape = shape;
  g.TX = kTileShapes[shape].TX ? kTileShapes[shape].TX : itot;
  g.TY = kTileShapes[shape].TY;
  g.TZ = kTileShapes[shape].TZ;
  g.ntx = (itot + g.TX - 1) / g.TX;
  g.nty = (jtot + g.TY - 1) / g.TY;
  g.ntz = (ktot + g.TZ - 1) / g.TZ;
  g.ntiles = g.ntx * g.nty * g.ntz;
  return true;
}

}  // namespace sg
