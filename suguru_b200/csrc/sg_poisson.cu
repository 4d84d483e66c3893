// sg_poisson.cu -- solver1d (solver.f90:43-157) after initsolver(e)
// (initsolver.f90:11-130) on the GPU: periodic x and y by a real 2-D FFT of
// every z plane (cuFFT D2Z / Z2D, batched over the planes), then for every
// (x, y) mode the reference's tridiagonal elimination in z, one thread per
// mode in FP64, then the inverse FFT.
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
#include <cufft.h>

#include <cmath>
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

// A thread per mode walks its column of kmax planes twice; the columns of
// neighbouring threads are adjacent in memory, and the loads of the next
// kPre planes are issued ahead of the dependent arithmetic (a ring of
// registers), since one column per thread leaves few warps to hide latency.
constexpr int kPre = 8;

__global__ void __launch_bounds__(128) tridiag_kernel(int kmax, int nmodes, int nxm, int e, double dzi, double shift,
                                                      const double* __restrict__ xrt, const double* __restrict__ yrt,
                                                      double2* __restrict__ c, double* __restrict__ d) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nmodes) return;
  const long nm = nmodes;
  const double lam = __dadd_rn(xrt[m % nxm], yrt[m / nxm]);
  double2 ring[kPre];
#pragma unroll
  for (int t = 0; t < kPre; ++t)
    if (1 + t < kmax) ring[t] = c[(1 + t) * nm + m];
  Rows r = solver_row(0, kmax, e, dzi, shift);
  double z = __drcp_rn(__dadd_rn(r.b, lam));
  double dk = __dmul_rn(r.c, z);
  double2 p = c[m];
  p.x = __dmul_rn(p.x, z);
  p.y = __dmul_rn(p.y, z);
  c[m] = p;
  d[m] = dk;
  // forward elimination, rows 1 .. kmax-2
  for (int k0 = 1; k0 < kmax - 1; k0 += kPre) {
#pragma unroll
    for (int t = 0; t < kPre; ++t) {
      const int k = k0 + t;
      if (k < kmax - 1) {
        double2 q = ring[t];
        if (k + kPre < kmax) ring[t] = c[(k + kPre) * nm + m];
        r = solver_row(k, kmax, e, dzi, shift);
        z = __drcp_rn(__dsub_rn(__dadd_rn(r.b, lam), __dmul_rn(r.a, dk)));
        dk = __dmul_rn(r.c, z);
        q.x = __dmul_rn(__dsub_rn(q.x, __dmul_rn(r.a, p.x)), z);
        q.y = __dmul_rn(__dsub_rn(q.y, __dmul_rn(r.a, p.y)), z);
        c[k * nm + m] = q;
        d[k * nm + m] = dk;
        p = q;
      }
    }
  }
  {
    const int k = kmax - 1;
    r = solver_row(k, kmax, e, dzi, shift);
    const double bb = e == 3 ? r.b : __dadd_rn(r.b, lam);
    z = __dsub_rn(bb, __dmul_rn(r.a, dk));
    double2 q = c[k * nm + m];
    if (z != 0.0) {
      q.x = __ddiv_rn(__dsub_rn(q.x, __dmul_rn(r.a, p.x)), z);
      q.y = __ddiv_rn(__dsub_rn(q.y, __dmul_rn(r.a, p.y)), z);
    } else {
      q.x = q.y = 0.0;
    }
    c[k * nm + m] = q;
    p = q;
  }
  // back substitution, rows kmax-2 .. 0
  double dring[kPre];
#pragma unroll
  for (int t = 0; t < kPre; ++t) {
    const int k = kmax - 2 - t;
    if (k >= 0) {
      ring[t] = c[k * nm + m];
      dring[t] = d[k * nm + m];
    }
  }
  for (int k0 = kmax - 2; k0 >= 0; k0 -= kPre) {
#pragma unroll
    for (int t = 0; t < kPre; ++t) {
      const int k = k0 - t;
      if (k >= 0) {
        double2 q = ring[t];
        const double dd = dring[t];
        if (k - kPre >= 0) {
          ring[t] = c[(k - kPre) * nm + m];
          dring[t] = d[(k - kPre) * nm + m];
        }
        q.x = __dsub_rn(q.x, __dmul_rn(dd, p.x));
        q.y = __dsub_rn(q.y, __dmul_rn(dd, p.y));
        c[k * nm + m] = q;
        p = q;
      }
    }
  }
}

}  // namespace

int poisson_setup(sg_ctx* c) {
  auto& s = c->pois;
  if (s.ready) return SG_OK;
  const sg_config& f = c->cfg;
  if (f.itot % 2 != 0 || f.ktot < 4) return fail(c, SG_ERR_CONFIG, "solver1d here needs an even itot and ktot >= 4");
  const long nreal = (long)f.itot * f.jtot * f.ktot, nxm = f.itot / 2 + 1, nmodes = nxm * f.jtot;
  void* p = nullptr;
  SG_TRY(dalloc(c, p, sizeof(double) * nreal), "alloc");
  s.r = (double*)p;
  SG_TRY(dalloc(c, p, sizeof(double2) * nmodes * f.ktot), "alloc");
  s.c = p;
  SG_TRY(dalloc(c, p, sizeof(double) * nmodes * f.ktot), "alloc");
  s.d = (double*)p;
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
  int n2[2] = {f.jtot, f.itot};
  if (cufftPlanMany(&s.plan_f, 2, n2, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, f.ktot) != CUFFT_SUCCESS)
    return fail(c, SG_ERR_CUDA, "cuFFT plan");
  if (cufftPlanMany(&s.plan_b, 2, n2, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2D, f.ktot) != CUFFT_SUCCESS) {
    cufftDestroy(s.plan_f);
    return fail(c, SG_ERR_CUDA, "cuFFT plan");
  }
  s.have_plans = true;
  s.ready = true;
  return SG_OK;
}

void poisson_free(sg_ctx* c) {
  if (c->pois.have_plans) {
    cufftDestroy(c->pois.plan_f);
    cufftDestroy(c->pois.plan_b);
    c->pois.have_plans = false;
  }
}

int poisson_solve(sg_ctx* c, double* r, int e, double shift, cudaStream_t st) {
  auto& s = c->pois;
  const sg_config& f = c->cfg;
  if (cufftSetStream(s.plan_f, st) != CUFFT_SUCCESS || cufftSetStream(s.plan_b, st) != CUFFT_SUCCESS ||
      cufftExecD2Z(s.plan_f, r, (cufftDoubleComplex*)s.c) != CUFFT_SUCCESS)
    return fail(c, SG_ERR_CUDA, "cuFFT forward");
  const int nxm = f.itot / 2 + 1, nmodes = nxm * f.jtot;
  tridiag_kernel<<<(unsigned)((nmodes + 127) / 128), 128, 0, st>>>(f.ktot, nmodes, nxm, e, 1.0 / (f.lz / f.ktot), shift,
                                                                     s.tab, s.tab + nxm, (double2*)s.c, s.d);
  SG_TRY(cudaGetLastError(), "solver1d");
  if (cufftExecZ2D(s.plan_b, (cufftDoubleComplex*)s.c, r) != CUFFT_SUCCESS) return fail(c, SG_ERR_CUDA, "cuFFT inverse");
  c->launches += 1;
  return SG_OK;
}

}  // namespace sg
