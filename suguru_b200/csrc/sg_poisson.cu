// sg_poisson.cu -- solver1d (solver.f90:43-157) after initsolver(e)
// (initsolver.f90:11-130) on the GPU: periodic x and y by a real 2-D FFT of
// every z plane, then for every (x, y) mode the reference's tridiagonal
// elimination in z, one thread per mode in FP64, then the inverse FFT.
//
// The FFTs are the library's own (the reference's fft.f / 2DECOMP transforms
// are FFTPACK-style mixed-radix FFTs): self-sorting (Stockham) mixed-radix
// passes in shared memory, FP64, with twiddle factors tabulated once on the
// host.  Per plane, forward: a real-to-complex transform of every x row (a
// complex FFT of half length on x_even + i x_odd, then the usual split into the
// itot/2 + 1 modes), then a complex FFT of every y column of those modes;
// inverse: the y columns, then complex-to-real rows.  Both directions are
// unnormalised, so that the pair multiplies by itot * jtot (the convention of
// the callers).  Any itot/2 and jtot whose prime factors are at most
// kMaxRadix are accepted.
//
// The rows of initsolver(e), built in the kernel in the reference's order:
//   a = c = dzi^2, b = -(a + c);
//   e = 0, 1: b(1) += a(1), b(kmax) += c(kmax), a(1) = c(kmax) = 0 (Neumann);
//   e = 2:    b(1) -= a(1), b(kmax) -= c(kmax), a(1) = c(kmax) = 0 (the
//             no-slip ghost rows of u and v), then b -= Rep/dt;
//   e = 3:    b(kmax) = 1, a(1) = a(kmax) = c(kmax) = 0 (w = 0 at the top
//             face), then b -= Rep/dt and b(kmax) = 1 again;
// the eigenvalues xrt + yrt of the mode join b except in the last row of
// e = 3.  The elimination keeps the reference's operations and roundings
// (no fused multiply-add): for e = 0, 1 the mean mode's last pivot is then
// exactly zero whenever it is in exact arithmetic, and that mode's top value
// is set to zero, as the reference does.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "sg_common.cuh"
#include "sg_ctx.h"

namespace sg {
namespace {

constexpr double kPi = 3.14159265358979323846264338327950288;

struct Rows {
  double a, b, c;
};

__device__ __forceinline__ Rows solver_row(int k, int kmax, int e, double dzi, double shift) {
  Rows r;
  r.a = __dmul_rn(dzi, dzi);
  r.c = __dmul_rn(dzi, dzi);
  r.b = -__dadd_rn(r.a, r.c);
  const bool first = k == 0, last = k == kmax - 1;
  if (e <= 1) {
    if (first) r.b = __dadd_rn(r.b, r.a);
    if (last) r.b = __dadd_rn(r.b, r.c);
    if (first) r.a = 0.;
    if (last) r.c = 0.;
  } else {
    if (e == 2) {
      if (first) r.b = __dsub_rn(r.b, r.a);
      if (last) r.b = __dsub_rn(r.b, r.c);
      if (first) r.a = 0.;
      if (last) r.c = 0.;
    } else {
      if (last) {
        r.b = 1.;
        r.a = 0.;
        r.c = 0.;
      }
      if (first) r.a = 0.;
    }
    r.b = __dsub_rn(r.b, shift);
    if (e == 3 && last) r.b = 1.;
  }
  return r;
}

// The elimination split in two.  Its pivots and multipliers depend only on
// the mode's eigenvalue, the row type e and the shift, not on the right-hand
// side, so tri_coeff_kernel runs the reference's forward recurrence for them
// once per (e, shift) and tabulates, per plane k and mode slot,
//   z_k = 1 / (b_k + lam - a_k d_{k-1})  (k < kmax-1; d_{-1} = 0),
//   d_k = c_k z_k                        (k < kmax-1),
//   z_{kmax-1} = bb - a d_{kmax-2}        (the last pivot itself, bb = b + lam
//                                          except for e = 3),
// with the same operations in the same order (no fused multiply-add), so a
// solve with the tables gives the bits of the one-pass elimination.  The
// solve (tri_apply_kernel) is then two first-order sweeps per mode:
//   q_0 = r_0 z_0, q_k = (r_k - a_k q_{k-1}) z_k, the last row divided by its
//   pivot (or set to zero when the pivot is exactly zero: the mean mode of
//   the Neumann rows, as the reference does), then x_k = q_k - d_k x_{k+1}.
// A thread per mode; the columns of neighbouring threads are adjacent in
// memory, and the loads of the next kPre planes are issued ahead of the
// dependent arithmetic (a ring of registers).  Modes are laid out [k][j][m]
// with nmp >= nxm slots per y row; slots m >= nxm are padding and skipped.
constexpr int kPre = 32;

__global__ void __launch_bounds__(128) tri_coeff_kernel(int kmax, int jtot, int nmp, int nxm, int e, double dzi,
                                                        double shift, const double* __restrict__ xrt,
                                                        const double* __restrict__ yrt, double* __restrict__ zt,
                                                        double* __restrict__ dt) {
  const long nm = (long)jtot * nmp;
  const long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nm || m % nmp >= nxm) return;
  const double lam = __dadd_rn(xrt[m % nmp], yrt[m / nmp]);
  Rows r = solver_row(0, kmax, e, dzi, shift);
  double z = __drcp_rn(__dadd_rn(r.b, lam));
  double dk = __dmul_rn(r.c, z);
  zt[m] = z;
  dt[m] = dk;
  for (int k = 1; k < kmax - 1; ++k) {
    r = solver_row(k, kmax, e, dzi, shift);
    z = __drcp_rn(__dsub_rn(__dadd_rn(r.b, lam), __dmul_rn(r.a, dk)));
    dk = __dmul_rn(r.c, z);
    zt[k * nm + m] = z;
    dt[k * nm + m] = dk;
  }
  r = solver_row(kmax - 1, kmax, e, dzi, shift);
  const double bb = e == 3 ? r.b : __dadd_rn(r.b, lam);
  zt[(kmax - 1) * nm + m] = __dsub_rn(bb, __dmul_rn(r.a, dk));
}

__global__ void __launch_bounds__(128) tri_apply_kernel(int kmax, int jtot, int nmp, int nxm, int e, double dzi,
                                                        const double* __restrict__ zt, const double* __restrict__ dt,
                                                        double2* __restrict__ c) {
  const long nm = (long)jtot * nmp;
  const long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nm || m % nmp >= nxm) return;
  // a_k of solver_row: 0 in row 0, dzi^2 in rows 1 .. kmax-2, and in row
  // kmax-1 dzi^2 except for e = 3 (the identity row of w at the top)
  const double a = __dmul_rn(dzi, dzi), a_last = e == 3 ? 0.0 : a;
  double2 ring[kPre];
  double zring[kPre];
#pragma unroll
  for (int t = 0; t < kPre; ++t)
    if (1 + t < kmax) {
      ring[t] = c[(1 + t) * nm + m];
      zring[t] = zt[(1 + t) * nm + m];
    }
  double2 p = c[m];
  {
    const double z = zt[m];
    p.x = __dmul_rn(p.x, z);
    p.y = __dmul_rn(p.y, z);
    c[m] = p;
  }
  // forward sweep, rows 1 .. kmax-2
  for (int k0 = 1; k0 < kmax - 1; k0 += kPre) {
#pragma unroll
    for (int t = 0; t < kPre; ++t) {
      const int k = k0 + t;
      if (k < kmax - 1) {
        double2 q = ring[t];
        const double z = zring[t];
        if (k + kPre < kmax) {
          ring[t] = c[(k + kPre) * nm + m];
          zring[t] = zt[(k + kPre) * nm + m];
        }
        q.x = __dmul_rn(__dsub_rn(q.x, __dmul_rn(a, p.x)), z);
        q.y = __dmul_rn(__dsub_rn(q.y, __dmul_rn(a, p.y)), z);
        c[k * nm + m] = q;
        p = q;
      }
    }
  }
  {
    const int k = kmax - 1;
    const double z = zt[k * nm + m];
    double2 q = c[k * nm + m];
    if (z != 0.0) {
      q.x = __ddiv_rn(__dsub_rn(q.x, __dmul_rn(a_last, p.x)), z);
      q.y = __ddiv_rn(__dsub_rn(q.y, __dmul_rn(a_last, p.y)), z);
    } else {
      q.x = q.y = 0.0;
    }
    c[k * nm + m] = q;
    p = q;
  }
  // back substitution, rows kmax-2 .. 0
#pragma unroll
  for (int t = 0; t < kPre; ++t) {
    const int k = kmax - 2 - t;
    if (k >= 0) {
      ring[t] = c[k * nm + m];
      zring[t] = dt[k * nm + m];
    }
  }
  for (int k0 = kmax - 2; k0 >= 0; k0 -= kPre) {
#pragma unroll
    for (int t = 0; t < kPre; ++t) {
      const int k = k0 - t;
      if (k >= 0) {
        double2 q = ring[t];
        const double dd = zring[t];
        if (k - kPre >= 0) {
          ring[t] = c[(k - kPre) * nm + m];
          zring[t] = dt[(k - kPre) * nm + m];
        }
        q.x = __dsub_rn(q.x, __dmul_rn(dd, p.x));
        q.y = __dsub_rn(q.y, __dmul_rn(dd, p.y));
        c[k * nm + m] = q;
        p = q;
      }
    }
  }
}

// ---------------------------------------------------------------- FFT ---
constexpr int kMaxRadix = 61;
constexpr int kMaxFactors = 16;
constexpr int kFftThreads = 256;
constexpr int kFftSmemComplex = 2048;  // complex values per buffer (two buffers: 64 KB)

// Factorisation of a transform length (radices applied in this order) and its
// twiddle table w[t] = exp(-2 pi i t / n), t < n.
struct FftPlan {
  int n, nf;
  int radix[kMaxFactors];
  const double2* w;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// One radix-P butterfly of a self-sorting pass: v[r] = in[j + r n/P] times
// exp(sign 2 pi i r k / (ns P)) (k = j mod ns), then the P-point DFT, V[q]
// written to out[q ns] (out already offset to (j / ns) ns P + k).  The pass
// twiddle index r k stride is below n (k < ns, r < P, stride = n / (ns P)).
// Radices 2 and 4 apply their DFT with sign changes and swaps only; 3 and 5
// take its roots from the table; all keep their values in registers.
template <int P>
__device__ __forceinline__ void butterfly(const double2* __restrict__ src, double2* __restrict__ dst, int j, int k,
                                          int np, int ns, int stride, int wstep,
                                          const double2* __restrict__ w, int sign) {
  double2 v[P];
#pragma unroll
  for (int r = 0; r < P; ++r) {
    double2 x = src[j + r * np];
    if (r && k) {
      double2 t = w[r * k * stride];
      if (sign > 0) t = cconj(t);
      x = cmul(x, t);
    }
    v[r] = x;
  }
  if constexpr (P == 2) {
    dst[0] = make_double2(v[0].x + v[1].x, v[0].y + v[1].y);
    dst[ns] = make_double2(v[0].x - v[1].x, v[0].y - v[1].y);
  } else if constexpr (P == 4) {
    // V_q = sum_r v_r exp(sign 2 pi i q r / 4): exp(sign i pi/2) = sign * i
    const double2 s02 = make_double2(v[0].x + v[2].x, v[0].y + v[2].y);
    const double2 d02 = make_double2(v[0].x - v[2].x, v[0].y - v[2].y);
    const double2 s13 = make_double2(v[1].x + v[3].x, v[1].y + v[3].y);
    const double2 d13 = make_double2(v[1].x - v[3].x, v[1].y - v[3].y);
    // i * d13 = (-d13.y, d13.x)
    const double sx = sign > 0 ? -d13.y : d13.y, sy = sign > 0 ? d13.x : -d13.x;  // sign * i * d13
    dst[0] = make_double2(s02.x + s13.x, s02.y + s13.y);
    dst[ns] = make_double2(d02.x + sx, d02.y + sy);
    dst[2 * ns] = make_double2(s02.x - s13.x, s02.y - s13.y);
    dst[3 * ns] = make_double2(d02.x - sx, d02.y - sy);
  } else {
#pragma unroll
    for (int q = 0; q < P; ++q) {
      double2 acc = v[0];
#pragma unroll
      for (int r = 1; r < P; ++r) {
        double2 t = w[((q * r) % P) * wstep];
        if (sign > 0) t = cconj(t);
        const double2 m = cmul(v[r], t);
        acc.x += m.x;
        acc.y += m.y;
      }
      dst[q * ns] = acc;
    }
  }
}

// The same for any radix p <= kMaxRadix: each output reads the p twiddled
// inputs again from shared memory (no per-thread array).
__device__ __forceinline__ void butterfly_any(const double2* __restrict__ src, double2* __restrict__ dst, int p,
                                              int j, int k, int np, int ns, int stride, int wstep,
                                              const double2* __restrict__ w, int sign) {
#pragma unroll 1
  for (int q = 0; q < p; ++q) {
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll 1
    for (int r = 0; r < p; ++r) {
      double2 x = src[j + r * np];
      if (r && k) {
        double2 t = w[r * k * stride];
        if (sign > 0) t = cconj(t);
        x = cmul(x, t);
      }
      double2 t = w[((q * r) % p) * wstep];
      if (sign > 0) t = cconj(t);
      const double2 m = cmul(x, t);
      acc.x += m.x;
      acc.y += m.y;
    }
    dst[q * ns] = acc;
  }
}

// nb sequences of length P.n in shared memory, sequence s at buf0 + s ld: self-sorting
// mixed-radix passes (Stockham), ping-ponging between buf0 and buf1; returns
// the buffer that holds the result.  sign = -1: forward (exp(-i..)), +1:
// inverse, unnormalised.  For a pass of radix p after sub-transforms of
// length ns: butterfly j < n/p takes v[r] = in[j + r n/p], twiddles it by
// exp(sign 2 pi i r k / (ns p)) with k = j mod ns, forms the p-point DFT and
// writes V[q] to out[(j / ns) ns p + k + q ns].
__device__ double2* fft_smem(double2* buf0, double2* buf1, int nb, int ld, const FftPlan& P, int sign) {
  const int n = P.n;
  double2* in = buf0;
  double2* out = buf1;
  int ns = 1;
  for (int f = 0; f < P.nf; ++f) {
    const int p = P.radix[f], np = n / p, stride = n / (ns * p), wstep = n / p;
    __syncthreads();
    for (int idx = threadIdx.x; idx < nb * np; idx += blockDim.x) {
      const int sq = idx / np, j = idx - sq * np, k = j % ns;
      const double2* src = in + sq * ld;
      double2* dst = out + sq * ld + (j / ns) * ns * p + k;
      switch (p) {
        case 2: butterfly<2>(src, dst, j, k, np, ns, stride, wstep, P.w, sign); break;
        case 3: butterfly<3>(src, dst, j, k, np, ns, stride, wstep, P.w, sign); break;
        case 4: butterfly<4>(src, dst, j, k, np, ns, stride, wstep, P.w, sign); break;
        case 5: butterfly<5>(src, dst, j, k, np, ns, stride, wstep, P.w, sign); break;
        default: butterfly_any(src, dst, p, j, k, np, ns, stride, wstep, P.w, sign); break;
      }
    }
    ns *= p;
    double2* t = in;
    in = out;
    out = t;
  }
  __syncthreads();
  return in;
}

// Forward real-to-complex transform of rows of nx = 2 n reals (row r of the
// block at src + r nx): z_m = x_2m + i x_2m+1, Z = FFT_n(z), then for
// k = 0 .. n: X_k = (Z_k + conj Z_{n-k}) / 2 - (i/2) W^k (Z_k - conj Z_{n-k}),
// W = exp(-2 pi i / nx), Z_n = Z_0; rows of n + 1 modes at dst + r ld.
__global__ void __launch_bounds__(kFftThreads) fft_rows_r2c(long nrows, int rows_per_cta, int ld, FftPlan P,
                                                            const double2* __restrict__ wpost,
                                                            const double* __restrict__ src, double2* __restrict__ dst) {
  extern __shared__ __align__(16) double2 fsm[];
  const int n = P.n, nm = n + 1;
  const long r0 = (long)blockIdx.x * rows_per_cta;
  const int nb = (int)min((long)rows_per_cta, nrows - r0);
  double2* b0 = fsm;
  double2* b1 = fsm + rows_per_cta * n;
  const double2* s2 = (const double2*)(src + r0 * 2 * n);
  for (int t = threadIdx.x; t < nb * n; t += blockDim.x) b0[t] = s2[t];
  const double2* Z = fft_smem(b0, b1, nb, n, P, -1);
  for (int t = threadIdx.x; t < nb * nm; t += blockDim.x) {
    const int r = t / nm, k = t - r * nm;
    const double2 zk = Z[r * n + (k == n ? 0 : k)], zc = cconj(Z[r * n + (k == 0 ? 0 : n - k)]);
    const double2 e = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y + zc.y));
    const double2 o = make_double2(0.5 * (zk.x - zc.x), 0.5 * (zk.y - zc.y));
    const double2 wo = cmul(wpost[k], o);  // W^k o; times -i: (wo.y, -wo.x)
    dst[(r0 + r) * ld + k] = make_double2(e.x + wo.y, e.y - wo.x);
  }
}

// Inverse complex-to-real rows: from the n + 1 modes X_k of a row,
// Z_k = (X_k + conj X_{n-k}) + i conj(W^k) (X_k - conj X_{n-k}), k < n,
// z = unnormalised inverse FFT_n(Z), x_2m = Re z_m, x_2m+1 = Im z_m (nx x).
__global__ void __launch_bounds__(kFftThreads) fft_rows_c2r(long nrows, int rows_per_cta, int ld, FftPlan P,
                                                            const double2* __restrict__ wpost,
                                                            const double2* __restrict__ src, double* __restrict__ dst) {
  extern __shared__ __align__(16) double2 fsm[];
  const int n = P.n, nm = n + 1;
  const long r0 = (long)blockIdx.x * rows_per_cta;
  const int nb = (int)min((long)rows_per_cta, nrows - r0);
  double2* b0 = fsm;
  double2* b1 = fsm + rows_per_cta * n;
  double2* b2 = fsm + 2 * rows_per_cta * n;  // the modes, [nb][n + 1]
  for (int t = threadIdx.x; t < nb * nm; t += blockDim.x) {
    const int r = t / nm, k = t - r * nm;
    b2[t] = src[(r0 + r) * ld + k];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nb * n; t += blockDim.x) {
    const int r = t / n, k = t - r * n;
    const double2 xk = b2[r * nm + k], xc = cconj(b2[r * nm + n - k]);
    const double2 sum = make_double2(xk.x + xc.x, xk.y + xc.y), dif = make_double2(xk.x - xc.x, xk.y - xc.y);
    const double2 t2 = cmul(cconj(wpost[k]), dif);  // times i: (-t2.y, t2.x)
    b0[t] = make_double2(sum.x - t2.y, sum.y + t2.x);
  }
  const double2* z = fft_smem(b0, b1, nb, n, P, +1);
  double2* d2 = (double2*)(dst + r0 * 2 * n);
  for (int t = threadIdx.x; t < nb * n; t += blockDim.x) d2[t] = z[t];
}

// Complex transforms of the columns of planes [nplanes][ny][ld] (ncols of
// them valid): the CTA takes plane blockIdx.y and columns c0 .. c0 + cb - 1;
// each warp loads runs of cb consecutive modes of a row.
__global__ void __launch_bounds__(kFftThreads) fft_cols(int ncols, int ld, int cols_per_cta, FftPlan P, int sign,
                                                        double2* __restrict__ data) {
  extern __shared__ __align__(16) double2 fsm[];
  const int ny = P.n, lds = ny + 1, c0 = blockIdx.x * cols_per_cta, cb = min(cols_per_cta, ncols - c0);
  double2* plane = data + (long)blockIdx.y * ny * ld;
  double2* b0 = fsm;
  double2* b1 = fsm + cols_per_cta * lds;
  // sequences at stride ny + 1: the transposing stores of neighbouring
  // columns fall in different banks
  for (int t = threadIdx.x; t < cb * ny; t += blockDim.x) {
    const int j = t / cb, c = t - j * cb;
    b0[c * lds + j] = plane[(long)j * ld + c0 + c];
  }
  const double2* Y = fft_smem(b0, b1, cb, lds, P, sign);
  for (int t = threadIdx.x; t < cb * ny; t += blockDim.x) {
    const int j = t / cb, c = t - j * cb;
    plane[(long)j * ld + c0 + c] = Y[c * lds + j];
  }
}

// ------------------------------------------------- power-of-two FFTs ---
// Lengths N = 32, 64, 128, 256: a sequence belongs to TPS = N/8 consecutive
// lanes of one warp, each holding 8 values in registers.  A Stockham pass of
// radix R after sub-transforms of length NS gives thread tau the butterflies
// j = tau + b TPS (b < 8/R); butterfly j reads x[j + r N/R], twiddles it by
// W_{NS R}^{r (j mod NS)}, forms the R-point DFT and writes V[q] to
// (j / NS) NS R + j mod NS + q NS.  Between passes the values go through the
// sequence's slot in shared memory, element e at e ^ ((e >> 3) & 7): every
// read and write pattern of the passes then puts the 8 lanes of a quarter
// warp on 8 different 16-byte bank groups.  Radices: 32 = 8.4, 64 = 8.8,
// 128 = 8.4.4, 256 = 8.8.4.  Twiddles come from per-pass tables in shared
// memory (TwTab); the 8-point DFT uses sqrt(1/2) as a constant.
__device__ __forceinline__ int swz(int e) { return e ^ ((e >> 3) & 7); }

template <int R>
__device__ __forceinline__ void dft_reg(double2* v, int sign) {
  if constexpr (R == 2) {
    const double2 a = v[0], b = v[1];
    v[0] = make_double2(a.x + b.x, a.y + b.y);
    v[1] = make_double2(a.x - b.x, a.y - b.y);
  } else if constexpr (R == 4) {
    const double2 s02 = make_double2(v[0].x + v[2].x, v[0].y + v[2].y);
    const double2 d02 = make_double2(v[0].x - v[2].x, v[0].y - v[2].y);
    const double2 s13 = make_double2(v[1].x + v[3].x, v[1].y + v[3].y);
    const double2 d13 = make_double2(v[1].x - v[3].x, v[1].y - v[3].y);
    const double sx = sign > 0 ? -d13.y : d13.y, sy = sign > 0 ? d13.x : -d13.x;  // sign * i * d13
    v[0] = make_double2(s02.x + s13.x, s02.y + s13.y);
    v[1] = make_double2(d02.x + sx, d02.y + sy);
    v[2] = make_double2(s02.x - s13.x, s02.y - s13.y);
    v[3] = make_double2(d02.x - sx, d02.y - sy);
  } else {
    static_assert(R == 8, "radix");
    // V_q = E_q + W^q O_q, V_{q+4} = E_q - W^q O_q, W = exp(sign 2 pi i / 8)
    double2 E[4] = {v[0], v[2], v[4], v[6]}, O[4] = {v[1], v[3], v[5], v[7]};
    dft_reg<4>(E, sign);
    dft_reg<4>(O, sign);
    constexpr double h = 0.70710678118654752440;
    double2 t1, t2, t3;
    if (sign < 0) {
      t1 = make_double2(h * (O[1].x + O[1].y), h * (O[1].y - O[1].x));
      t2 = make_double2(O[2].y, -O[2].x);
      t3 = make_double2(h * (O[3].y - O[3].x), -h * (O[3].x + O[3].y));
    } else {
      t1 = make_double2(h * (O[1].x - O[1].y), h * (O[1].x + O[1].y));
      t2 = make_double2(-O[2].y, O[2].x);
      t3 = make_double2(-h * (O[3].x + O[3].y), h * (O[3].x - O[3].y));
    }
    v[0] = make_double2(E[0].x + O[0].x, E[0].y + O[0].y);
    v[4] = make_double2(E[0].x - O[0].x, E[0].y - O[0].y);
    v[1] = make_double2(E[1].x + t1.x, E[1].y + t1.y);
    v[5] = make_double2(E[1].x - t1.x, E[1].y - t1.y);
    v[2] = make_double2(E[2].x + t2.x, E[2].y + t2.y);
    v[6] = make_double2(E[2].x - t2.x, E[2].y - t2.y);
    v[3] = make_double2(E[3].x + t3.x, E[3].y + t3.y);
    v[7] = make_double2(E[3].x - t3.x, E[3].y - t3.y);
  }
}

// Twiddles of a pass (NS > 1) as their own table, tp[(r-1) NS + k] =
// W_{NS R}^{r k}: the lanes of a quarter warp (consecutive k) read
// consecutive 16-byte values.  Tables of a length's passes lie one after the
// other: 32: 24 values; 64: 56; 128: 24 + 96; 256: 56 + 192.
template <int N> struct TwTab;
template <> struct TwTab<32> { static constexpr int size = 24; };
template <> struct TwTab<64> { static constexpr int size = 56; };
template <> struct TwTab<128> { static constexpr int size = 120, off2 = 0, off3 = 24; };
template <> struct TwTab<256> { static constexpr int size = 248, off2 = 0, off3 = 56; };

template <int N, int R, int NS>
__device__ __forceinline__ void fill_pass_tw(double2* tp, const double2* __restrict__ tw_g, int tid, int nthr) {
  for (int i = tid; i < (R - 1) * NS; i += nthr) {
    const int r = i / NS + 1, k = i % NS;
    tp[i] = tw_g[r * k * (N / (NS * R))];
  }
}

// the pass tables of length N from the table W_N^t (t < N) in global memory
template <int N>
__device__ __forceinline__ void fill_tw(double2* tp, const double2* __restrict__ tw_g, int tid, int nthr) {
  if constexpr (N == 32) {
    fill_pass_tw<32, 4, 8>(tp, tw_g, tid, nthr);
  } else if constexpr (N == 64) {
    fill_pass_tw<64, 8, 8>(tp, tw_g, tid, nthr);
  } else if constexpr (N == 128) {
    fill_pass_tw<128, 4, 8>(tp + TwTab<128>::off2, tw_g, tid, nthr);
    fill_pass_tw<128, 4, 32>(tp + TwTab<128>::off3, tw_g, tid, nthr);
  } else {
    fill_pass_tw<256, 8, 8>(tp + TwTab<256>::off2, tw_g, tid, nthr);
    fill_pass_tw<256, 4, 64>(tp + TwTab<256>::off3, tw_g, tid, nthr);
  }
}

// v[b R + r] = x[j_b + r N/R] on entry; V[q] of butterfly b in v[b R + q] on
// exit; tp: this pass's twiddle table (unused when NS = 1)
template <int N, int R, int NS>
__device__ __forceinline__ void pass_reg(double2 (&v)[8], int tau, const double2* __restrict__ tp, int sign) {
  constexpr int TPS = N / 8, NB = 8 / R;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int j = tau + b * TPS, k = j & (NS - 1);
    if constexpr (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        double2 t = tp[(r - 1) * NS + k];
        if (sign > 0) t = cconj(t);
        v[b * R + r] = cmul(v[b * R + r], t);
      }
    }
    dft_reg<R>(&v[b * R], sign);
  }
}

template <int N, int R>
__device__ __forceinline__ void load_pass(double2 (&v)[8], const double2* seq, int tau) {
  constexpr int TPS = N / 8, NB = 8 / R;
#pragma unroll
  for (int b = 0; b < NB; ++b)
#pragma unroll
    for (int r = 0; r < R; ++r) v[b * R + r] = seq[swz(tau + b * TPS + r * (N / R))];
}

template <int N, int R, int NS>
__device__ __forceinline__ int out_pos(int tau, int b, int q) {
  const int j = tau + b * (N / 8);
  return (j / NS) * NS * R + (j & (NS - 1)) + q * NS;
}

template <int N, int R, int NS>
__device__ __forceinline__ void store_pass(const double2 (&v)[8], double2* seq, int tau) {
  constexpr int NB = 8 / R;
#pragma unroll
  for (int b = 0; b < NB; ++b)
#pragma unroll
    for (int q = 0; q < R; ++q) seq[swz(out_pos<N, R, NS>(tau, b, q))] = v[b * R + q];
}

// The last pass of each length, for the callers' output positions.
template <int N> struct LastPass;
template <> struct LastPass<32> { static constexpr int R = 4, NS = 8; };
template <> struct LastPass<64> { static constexpr int R = 8, NS = 8; };
template <> struct LastPass<128> { static constexpr int R = 4, NS = 32; };
template <> struct LastPass<256> { static constexpr int R = 4, NS = 64; };

// v holds x[tau + r TPS] (the first pass's inputs); on exit v[b R + q] holds
// the transform at out_pos<N, LastPass R, LastPass NS>(tau, b, q).  Every lane
// of the warp calls it (the passes synchronise the warp); seq is the
// sequence's shared-memory slot (N values, swizzled), tw the pass tables
// (fill_tw).
template <int N>
__device__ __forceinline__ void fft_reg(double2 (&v)[8], double2* seq, int tau, const double2* __restrict__ tw,
                                        int sign) {
  pass_reg<N, 8, 1>(v, tau, tw, sign);
  __syncwarp();  // every lane has read its inputs (the caller's, if from seq)
  store_pass<N, 8, 1>(v, seq, tau);
  __syncwarp();
  if constexpr (N == 32) {
    load_pass<N, 4>(v, seq, tau);
    pass_reg<N, 4, 8>(v, tau, tw, sign);
  } else if constexpr (N == 64) {
    load_pass<N, 8>(v, seq, tau);
    pass_reg<N, 8, 8>(v, tau, tw, sign);
  } else if constexpr (N == 128) {
    load_pass<N, 4>(v, seq, tau);
    pass_reg<N, 4, 8>(v, tau, tw + TwTab<N>::off2, sign);
    __syncwarp();
    store_pass<N, 4, 8>(v, seq, tau);
    __syncwarp();
    load_pass<N, 4>(v, seq, tau);
    pass_reg<N, 4, 32>(v, tau, tw + TwTab<N>::off3, sign);
  } else {
    static_assert(N == 256, "length");
    load_pass<N, 8>(v, seq, tau);
    pass_reg<N, 8, 8>(v, tau, tw + TwTab<N>::off2, sign);
    __syncwarp();
    store_pass<N, 8, 8>(v, seq, tau);
    __syncwarp();
    load_pass<N, 4>(v, seq, tau);
    pass_reg<N, 4, 64>(v, tau, tw + TwTab<N>::off3, sign);
  }
}

template <int N>
__device__ __forceinline__ void store_last(const double2 (&v)[8], double2* seq, int tau) {
  store_pass<N, LastPass<N>::R, LastPass<N>::NS>(v, seq, tau);
}

constexpr int kRegThreads = 256;

// Real-to-complex rows (complex length N = nx / 2), 256 / (N / 8) rows per
// CTA, the post-processing split of fft_rows_r2c.  Loads go straight from
// global memory into the first pass's registers (a half-row run of 16-byte
// values per group of lanes); the modes are written with stride ld.
template <int N>
__global__ void __launch_bounds__(kRegThreads) rows_r2c_reg(long nrows, int ld, const double2* __restrict__ tw_g,
                                                           const double2* __restrict__ wp_g,
                                                           const double* __restrict__ src, double2* __restrict__ dst) {
  constexpr int TPS = N / 8, SPC = kRegThreads / TPS, LD = N + 1;
  __shared__ double2 tw[TwTab<N>::size], wp[N + 1];
  __shared__ double2 buf[SPC * LD];
  fill_tw<N>(tw, tw_g, threadIdx.x, kRegThreads);
  for (int t = threadIdx.x; t <= N; t += kRegThreads) wp[t] = wp_g[t];
  const int sq = threadIdx.x / TPS, tau = threadIdx.x % TPS;
  const long row = (long)blockIdx.x * SPC + sq;
  const bool ok = row < nrows;
  const double2* s = (const double2*)src + row * N;
  double2 v[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) v[r] = ok ? s[tau + r * TPS] : make_double2(0.0, 0.0);
  __syncthreads();  // the tables
  double2* seq = buf + sq * LD;
  fft_reg<N>(v, seq, tau, tw, -1);
  __syncwarp();
  store_last<N>(v, seq, tau);
  __syncwarp();
  if (!ok) return;
  double2* o = dst + row * ld;
#pragma unroll
  for (int i = 0; i <= 8; ++i) {
    const int k = tau + i * TPS;
    if (k <= N) {
      const double2 zk = seq[swz(k & (N - 1))], zc = cconj(seq[swz((N - k) & (N - 1))]);
      const double2 e = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y + zc.y));
      const double2 od = make_double2(0.5 * (zk.x - zc.x), 0.5 * (zk.y - zc.y));
      const double2 wo = cmul(wp[k], od);
      o[k] = make_double2(e.x + wo.y, e.y - wo.x);
    }
  }
}

// Where the inverse rows put the solution: dense (f == nullptr: into the
// transform's own real array), or scaled into the interior of a field with a
// one-cell halo, value (i, j, k) (0-based) at f[(k+1) plane + (j+1) ldi + i+1].
struct RowsOut {
  double* f;
  long ldi, plane;
  double scale;
  int jtot;
};

// Complex-to-real rows, the pre-processing of fft_rows_c2r: the modes of the
// CTA's rows go through shared memory (row pairs X_k, X_{n-k}), the first
// pass's inputs are formed in registers, the last pass writes the reals
// straight to global memory (16-byte runs, or pairs of 8-byte values into a
// halo field).
template <int N>
__global__ void __launch_bounds__(kRegThreads) rows_c2r_reg(long nrows, int ld, const double2* __restrict__ tw_g,
                                                           const double2* __restrict__ wp_g,
                                                           const double2* __restrict__ src, double* __restrict__ dst,
                                                           RowsOut out) {
  constexpr int TPS = N / 8, SPC = kRegThreads / TPS, LD = N + 1;
  __shared__ double2 tw[TwTab<N>::size], wp[N + 1];
  __shared__ double2 buf[SPC * LD];
  fill_tw<N>(tw, tw_g, threadIdx.x, kRegThreads);
  for (int t = threadIdx.x; t <= N; t += kRegThreads) wp[t] = wp_g[t];
  const int sq = threadIdx.x / TPS, tau = threadIdx.x % TPS;
  const long row = (long)blockIdx.x * SPC + sq;
  const bool ok = row < nrows;
  double2* seq = buf + sq * LD;  // first the row's N + 1 modes (linear), then the FFT slot
  const double2* s = src + row * ld;
#pragma unroll
  for (int i = 0; i <= 8; ++i) {
    const int k = tau + i * TPS;
    if (k <= N) seq[k] = ok ? s[k] : make_double2(0.0, 0.0);
  }
  __syncthreads();  // the tables and the modes
  double2 v[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int k = tau + r * TPS;
    const double2 xk = seq[k], xc = cconj(seq[N - k]);
    const double2 sum = make_double2(xk.x + xc.x, xk.y + xc.y), dif = make_double2(xk.x - xc.x, xk.y - xc.y);
    const double2 t2 = cmul(cconj(wp[k]), dif);
    v[r] = make_double2(sum.x - t2.y, sum.y + t2.x);
  }
  fft_reg<N>(v, seq, tau, tw, +1);
  if (!ok) return;
  constexpr int R = LastPass<N>::R, NS = LastPass<N>::NS;
  if (!out.f) {
    double2* d2 = (double2*)dst + row * N;
#pragma unroll
    for (int b = 0; b < 8 / R; ++b)
#pragma unroll
      for (int q = 0; q < R; ++q) d2[out_pos<N, R, NS>(tau, b, q)] = v[b * R + q];
  } else {
    const long j = row % out.jtot, k = row / out.jtot;
    double* f = out.f + (k + 1) * out.plane + (j + 1) * out.ldi + 1;
#pragma unroll
    for (int b = 0; b < 8 / R; ++b)
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int m = out_pos<N, R, NS>(tau, b, q);
        f[2 * m] = v[b * R + q].x * out.scale;
        f[2 * m + 1] = v[b * R + q].y * out.scale;
      }
  }
}

// Column transforms (length N = ny) of planes [nplanes][N][ld], ncols valid
// columns: 256 / (N / 8) columns per CTA, loaded row by row (runs of
// consecutive modes) into per-column slots of shared memory, transformed by
// a lane group each, and written back the same way.
template <int N>
__global__ void __launch_bounds__(kRegThreads) cols_reg(int ncols, int ld, const double2* __restrict__ tw_g, int sign,
                                                       double2* __restrict__ data) {
  constexpr int TPS = N / 8, CB = kRegThreads / TPS, LD = N + 1, YS = kRegThreads / CB;
  __shared__ double2 tw[TwTab<N>::size];
  __shared__ double2 buf[CB * LD];
  fill_tw<N>(tw, tw_g, threadIdx.x, kRegThreads);
  double2* plane = data + (long)blockIdx.y * N * ld;
  const int c0 = blockIdx.x * CB;
  {
    const int c = threadIdx.x % CB, y0 = threadIdx.x / CB;
    const bool in = c0 + c < ncols;
#pragma unroll 4
    for (int y = y0; y < N; y += YS) buf[c * LD + swz(y)] = in ? plane[(long)y * ld + c0 + c] : make_double2(0., 0.);
  }
  __syncthreads();
  const int sq = threadIdx.x / TPS, tau = threadIdx.x % TPS;
  double2* seq = buf + sq * LD;
  double2 v[8];
  load_pass<N, 8>(v, seq, tau);
  fft_reg<N>(v, seq, tau, tw, sign);
  __syncwarp();
  store_last<N>(v, seq, tau);
  __syncthreads();
  {
    const int c = threadIdx.x % CB, y0 = threadIdx.x / CB;
    if (c0 + c < ncols)
#pragma unroll 4
      for (int y = y0; y < N; y += YS) plane[(long)y * ld + c0 + c] = buf[c * LD + swz(y)];
  }
}

// dense solution -> scaled halo field (the generic inverse rows' epilogue)
__global__ void scatter_out_kernel(long n, int itot, const double* __restrict__ r, RowsOut out) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const long i = q % itot, row = q / itot, j = row % out.jtot, k = row / out.jtot;
  out.f[(k + 1) * out.plane + (j + 1) * out.ldi + i + 1] = r[q] * out.scale;
}

}  // namespace

namespace {

// radices of n (4s first, then the other primes up to kMaxRadix); false when
// a prime factor is larger or there are too many factors
bool factor(int n, FftPlan& P) {
  P.n = n;
  P.nf = 0;
  int m = n;
  while (m % 4 == 0 && P.nf < kMaxFactors) { P.radix[P.nf++] = 4; m /= 4; }
  for (int p = 2; p <= kMaxRadix && m > 1; ++p)
    while (m % p == 0 && P.nf < kMaxFactors) { P.radix[P.nf++] = p; m /= p; }
  return m == 1 && n >= 1;
}

std::vector<double> twiddles(int n) {  // exp(-2 pi i t / n) as (re, im) pairs
  std::vector<double> w(2 * (size_t)n);
  for (int t = 0; t < n; ++t) {
    w[2 * t] = std::cos(2.0 * kPi * t / n);
    w[2 * t + 1] = -std::sin(2.0 * kPi * t / n);
  }
  return w;
}

}  // namespace

namespace {
bool pow2_fast(int n) { return n == 32 || n == 64 || n == 128 || n == 256; }
int mode_stride(int itot) { return (itot / 2 + 1 + 7) / 8 * 8; }  // nxm rounded up to 8 slots (128 B)
}  // namespace

int poisson_setup(sg_ctx* c, unsigned types) {
  auto& s = c->pois;
  const sg_config& f = c->cfg;
  const long nslots = (long)mode_stride(f.itot) * f.jtot;
  void* p = nullptr;
  if (s.ready) {
    for (int e = 0; e < 4; ++e)
      if ((types >> e & 1u) && !s.zt[e]) {
        SG_TRY(dalloc(c, p, sizeof(double) * nslots * f.ktot), "alloc");
        s.zt[e] = (double*)p;
        SG_TRY(dalloc(c, p, sizeof(double) * nslots * f.ktot), "alloc");
        s.dt[e] = (double*)p;
      }
    return SG_OK;
  }
  if (f.itot % 2 != 0 || f.ktot < 4) return fail(c, SG_ERR_CONFIG, "solver1d here needs an even itot and ktot >= 4");
  const long nreal = (long)f.itot * f.jtot * f.ktot, nxm = f.itot / 2 + 1;
  SG_TRY(dalloc(c, p, sizeof(double) * nreal), "alloc");
  s.r = (double*)p;
  SG_TRY(dalloc(c, p, sizeof(double2) * nslots * f.ktot), "alloc");
  s.c = p;
  for (int e = 0; e < 4; ++e)
    if (types >> e & 1u) {
      SG_TRY(dalloc(c, p, sizeof(double) * nslots * f.ktot), "alloc");
      s.zt[e] = (double*)p;
      SG_TRY(dalloc(c, p, sizeof(double) * nslots * f.ktot), "alloc");
      s.dt[e] = (double*)p;
    }
  // initsolver.f90:111-130: xrt(2m) = xrt(2m+1) = -4 dxi^2 sin(2m pi / (2 itot))^2, the
  // modes of a real transform in x; in y the complex modes j and jtot - j share yrt
  std::vector<double> tab(nxm + f.jtot);
  const double dxi = 1.0 / (f.lx / f.itot), dyi = 1.0 / (f.ly / f.jtot);
  for (long m = 0; m < nxm; ++m) tab[m] = -4. * dxi * dxi * std::pow(std::sin((double)(2 * m) * kPi / (2. * f.itot)), 2.);
  for (int j = 0; j < f.jtot; ++j) {
    const int jm = std::min(j, f.jtot - j);
    tab[nxm + j] = -4. * dyi * dyi * std::pow(std::sin((double)(2 * jm) * kPi / (2. * f.jtot)), 2.);
  }
  SG_TRY(dalloc(c, p, sizeof(double) * tab.size()), "alloc");
  s.tab = (double*)p;
  SG_TRY(cudaMemcpy(s.tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice), "upload");
  // FFT plans: complex length itot/2 for the rows (real length itot), jtot
  // for the columns; twiddle tables exp(-2 pi i t / n) and the row split's
  // W^k = exp(-2 pi i k / itot), k <= itot/2
  FftPlan px{}, py{};
  if (!factor(f.itot / 2, px) || !factor(f.jtot, py) || f.itot / 2 > kFftSmemComplex || f.jtot > kFftSmemComplex)
    return fail(c, SG_ERR_CONFIG, "solver1d here needs itot/2 and jtot of at most 2048 whose prime factors are "
                                  "at most 61");
  std::vector<double> w = twiddles(f.itot / 2), wy = twiddles(f.jtot), wp(2 * (size_t)nxm);
  for (long k = 0; k < nxm; ++k) {
    wp[2 * k] = std::cos(2.0 * kPi * k / f.itot);
    wp[2 * k + 1] = -std::sin(2.0 * kPi * k / f.itot);
  }
  w.insert(w.end(), wy.begin(), wy.end());
  w.insert(w.end(), wp.begin(), wp.end());
  SG_TRY(dalloc(c, p, sizeof(double) * w.size()), "alloc");
  SG_TRY(cudaMemcpy(p, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice), "upload");
  s.w = (double2*)p;
  px.w = s.w;
  py.w = s.w + f.itot / 2;
  s.wpost = s.w + f.itot / 2 + f.jtot;
  static_assert(sizeof(FftPlan) <= sizeof(s.plan_x), "plan storage");
  std::memcpy(s.plan_x, &px, sizeof(px));
  std::memcpy(s.plan_y, &py, sizeof(py));
  s.ready = true;
  return SG_OK;
}

void poisson_free(sg_ctx* c) { (void)c; }

namespace {

template <int N>
void launch_r2c(long nrows, int ld, const double2* tw, const double2* wp, const double* r, double2* m,
                cudaStream_t st) {
  constexpr int SPC = kRegThreads / (N / 8);
  rows_r2c_reg<N><<<(unsigned)((nrows + SPC - 1) / SPC), kRegThreads, 0, st>>>(nrows, ld, tw, wp, r, m);
}
template <int N>
void launch_c2r(long nrows, int ld, const double2* tw, const double2* wp, const double2* m, double* r,
                const RowsOut& o, cudaStream_t st) {
  constexpr int SPC = kRegThreads / (N / 8);
  rows_c2r_reg<N><<<(unsigned)((nrows + SPC - 1) / SPC), kRegThreads, 0, st>>>(nrows, ld, tw, wp, m, r, o);
}
template <int N>
void launch_cols(int ncols, int ld, int planes, const double2* tw, int sign, double2* m, cudaStream_t st) {
  constexpr int CB = kRegThreads / (N / 8);
  cols_reg<N><<<dim3((unsigned)((ncols + CB - 1) / CB), (unsigned)planes), kRegThreads, 0, st>>>(ncols, ld, tw, sign,
                                                                                                 m);
}
#define SG_POW2_DISPATCH(n, call) \
  switch (n) {                    \
    case 32: call(32); break;     \
    case 64: call(64); break;     \
    case 128: call(128); break;   \
    default: call(256); break;    \
  }

}  // namespace

int poisson_solve(sg_ctx* c, double* r, int e, double shift, cudaStream_t st, const PoisOut* out) {
  auto& s = c->pois;
  const sg_config& f = c->cfg;
  FftPlan px, py;
  std::memcpy(&px, s.plan_x, sizeof(px));
  std::memcpy(&py, s.plan_y, sizeof(py));
  const int n = f.itot / 2, nxm = n + 1, ld = mode_stride(f.itot);
  const long nrows = (long)f.jtot * f.ktot, nslots = (long)ld * f.jtot;
  const bool rows_fast = pow2_fast(n), cols_fast = pow2_fast(f.jtot);
  const RowsOut ro{out ? out->f : nullptr, out ? out->ldi : 0, out ? out->plane : 0, out ? out->scale : 0.0, f.jtot};
  // generic passes: rows per CTA in two (forward) or three (inverse) buffers
  // of at most kFftSmemComplex values; columns per CTA likewise
  const int rpc = std::max(1, kFftSmemComplex / n), cpc = std::max(1, kFftSmemComplex / f.jtot);
  const size_t sm_f = sizeof(double2) * 2 * rpc * n, sm_i = sizeof(double2) * rpc * (2 * n + nxm);
  const size_t sm_c = sizeof(double2) * 2 * cpc * (f.jtot + 1);
  if (!rows_fast) {
    SG_TRY(smem_limit(fft_rows_r2c, sm_f), "fft");
    SG_TRY(smem_limit(fft_rows_c2r, sm_i), "fft");
  }
  if (!cols_fast) SG_TRY(smem_limit(fft_cols, sm_c), "fft");
  const unsigned gr = (unsigned)((nrows + rpc - 1) / rpc);
  const dim3 gc((unsigned)((nxm + cpc - 1) / cpc), (unsigned)f.ktot);
  double2* modes = (double2*)s.c;
  const double2* twx = s.w;
  const double2* twy = s.w + n;
#define SG_R2C(N) launch_r2c<N>(nrows, ld, twx, s.wpost, r, modes, st)
#define SG_COLS_F(N) launch_cols<N>(nxm, ld, f.ktot, twy, -1, modes, st)
#define SG_COLS_I(N) launch_cols<N>(nxm, ld, f.ktot, twy, +1, modes, st)
#define SG_C2R(N) launch_c2r<N>(nrows, ld, twx, s.wpost, modes, r, ro, st)
  if (rows_fast) {
    SG_POW2_DISPATCH(n, SG_R2C)
  } else {
    fft_rows_r2c<<<gr, kFftThreads, sm_f, st>>>(nrows, rpc, ld, px, s.wpost, r, modes);
  }
  if (cols_fast) {
    SG_POW2_DISPATCH(f.jtot, SG_COLS_F)
  } else {
    fft_cols<<<gc, kFftThreads, sm_c, st>>>(nxm, ld, cpc, py, -1, modes);
  }
  const double dzi = 1.0 / (f.lz / f.ktot);
  const unsigned gt = (unsigned)((nslots + 127) / 128);
  int launches = 5;
  if (e < 0 || e > 3 || !s.zt[e]) return fail(c, SG_ERR_STATE, "solver1d: tables of this row type were not set up");
  if (!s.tvalid[e] || s.tshift[e] != shift) {
    // (re)build the tables for this shift; inside a stream capture the build
    // is recorded but has not run, so they are not marked valid for the
    // direct calls that may come before the graph's first launch
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    SG_TRY(cudaStreamIsCapturing(st, &cap), "solver1d");
    tri_coeff_kernel<<<gt, 128, 0, st>>>(f.ktot, f.jtot, ld, nxm, e, dzi, shift, s.tab, s.tab + nxm, s.zt[e], s.dt[e]);
    s.tvalid[e] = cap == cudaStreamCaptureStatusNone;
    s.tshift[e] = shift;
    launches += 1;
  }
  tri_apply_kernel<<<gt, 128, 0, st>>>(f.ktot, f.jtot, ld, nxm, e, dzi, s.zt[e], s.dt[e], modes);
  if (cols_fast) {
    SG_POW2_DISPATCH(f.jtot, SG_COLS_I)
  } else {
    fft_cols<<<gc, kFftThreads, sm_c, st>>>(nxm, ld, cpc, py, +1, modes);
  }
  if (rows_fast) {
    SG_POW2_DISPATCH(n, SG_C2R)
  } else {
    fft_rows_c2r<<<gr, kFftThreads, sm_i, st>>>(nrows, rpc, ld, px, s.wpost, modes, r);
    if (out) {
      const long nreal = nrows * f.itot;
      scatter_out_kernel<<<(unsigned)((nreal + 255) / 256), 256, 0, st>>>(nreal, f.itot, r, ro);
      launches += 1;
    }
  }
#undef SG_R2C
#undef SG_COLS_F
#undef SG_COLS_I
#undef SG_C2R
  SG_TRY(cudaGetLastError(), "solver1d");
  c->launches += launches;
  return SG_OK;
}

}  // namespace sg
