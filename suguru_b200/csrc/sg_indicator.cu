// sg_indicator.cu -- the indicator function of indicator.f90:19-182 on the
// main mesh (the overlap mesh, ifoverlap = 1, is off by default).
//
//  1. The capsules are raised by ktot/4 dz (:24-31) and their normals times
//     area spread with cell-centre weights in every direction, the z window
//     reaching the wall halo planes (lagr2eulrind, interp_spread.f90:
//     978-1387).  The deterministic tile spread runs on a grid two planes
//     taller, shifted down by one plane, so that its interior covers k = 0 ..
//     kmax + 1 of the real grid.
//  2. The central-difference divergence of g (:49-66) is the right-hand side
//     of the Poisson equation that solver1d solves after initsolver(0)
//     (sg_poisson.cu).
//  3. indic = the solution lowered back by ktot/4 planes (zero above), its
//     halos from boundind (bound.f90:113-139: Neumann z, periodic x, y) taken
//     before the 0.01 / 0.9 thresholds, which apply to the interior only
//     (:94-111); visc = visc0 (1 + (lambda - 1) indic) with boundp
//     (:137-154); and the centrifugal terms added to forcey, forcez on the
//     interior (:156-180).
// Everything runs in FP64; the mixed path converts its FP32 inputs and
// rounds its FP32 outputs once.
#include <cmath>

#include "sg_common.cuh"
#include "sg_ctx.h"

namespace sg {
namespace {

__global__ void raise_z_kernel(long n, double off, const double* __restrict__ Z, double* __restrict__ Zr) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) Zr[p] = Z[p] + off;
}

// normals * area / dV as the spread's force records
template <class T>
__global__ void pack_normals_kernel(long n, double dvi, const T* __restrict__ NX, const T* __restrict__ NY,
                                    const T* __restrict__ NZ, const T* __restrict__ A,
                                    ForceRec<double>* __restrict__ frc) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double s = (double)A[p] * dvi;
  ForceRec<double> r;
  r.cf[0] = (double)NX[p] * s;
  r.cf[1] = (double)NY[p] * s;
  r.cf[2] = (double)NZ[p] * s;
  r.cf[3] = 0.0;
  frc[p] = r;
}

struct IndGrid {
  int itot, jtot, ktot, ldi, ldj;
  double dxi, dyi, dzi;
};

// dg at the interior cell (i, j, k) from g on the taller grid (plane k + 1 of
// g holds level k), written to the FFT input [k-1][j-1][i-1]
__global__ void divergence_kernel(IndGrid g, const double* __restrict__ gx, const double* __restrict__ gy,
                                  const double* __restrict__ gz, double* __restrict__ rhs) {
  const long n = (long)g.itot * g.jtot * g.ktot;
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int i = (int)(q % g.itot) + 1, j = (int)((q / g.itot) % g.jtot) + 1, k = (int)(q / ((long)g.itot * g.jtot)) + 1;
  const long plane = (long)g.ldi * g.ldj;
  const long o = (long)(k + 1) * plane + (long)j * g.ldi + i;
  const double dgx = __dmul_rn((gx[o + 1] - gx[o - 1]) * .5, g.dxi);
  const double dgy = __dmul_rn((gy[o + g.ldi] - gy[o - g.ldi]) * .5, g.dyi);
  const double dgz = __dmul_rn((gz[o + plane] - gz[o - plane]) * .5, g.dzi);
  rhs[q] = __dadd_rn(__dadd_rn(dgx, dgy), dgz);
}

struct IndPost {
  IndGrid g;
  int q;         // ktot / 4
  double inv_n;  // 1 / (itot jtot): the unnormalised FFT pair
  double visc0, lam_m1;
};

// the indicator at cell (i, j, k) of (0:i1, 0:j1, 0:k1) before the
// thresholds: the solution at the interior cell that (i, j, k) copies
// (periodic x, y; Neumann z), lowered by q planes, zero above kmax - q
__device__ __forceinline__ double ind_value(const IndPost& P, const double* __restrict__ sol, int i, int j, int k) {
  const IndGrid& g = P.g;
  const int is = i == 0 ? g.itot : (i == g.itot + 1 ? 1 : i);
  const int js = j == 0 ? g.jtot : (j == g.jtot + 1 ? 1 : j);
  const int ks = k == 0 ? 1 : (k == g.ktot + 1 ? g.ktot : k);
  double v = 0.0;
  if (ks <= g.ktot - P.q)
    v = sol[((long)(ks + P.q - 1) * g.jtot + (js - 1)) * g.itot + (is - 1)] * P.inv_n;
  return v;
}
__device__ __forceinline__ double thresholds(double v) {
  if (v < .01) v = 0.;
  if (v >= .9) v = 1.;
  return v;
}

template <class T>
__global__ void indic_kernel(IndPost P, const double* __restrict__ sol, T* __restrict__ indic, T* __restrict__ visc) {
  const IndGrid& g = P.g;
  const long n = (long)g.ldi * g.ldj * (g.ktot + 2);
  const long o = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  const int i = (int)(o % g.ldi), j = (int)((o / g.ldi) % g.ldj), k = (int)(o / ((long)g.ldi * g.ldj));
  const double v = ind_value(P, sol, i, j, k);
  const double t = thresholds(v);
  const bool interior = i >= 1 && i <= g.itot && j >= 1 && j <= g.jtot && k >= 1 && k <= g.ktot;
  indic[o] = (T)(interior ? t : v);
  if (visc) visc[o] = (T)__dmul_rn(P.visc0, __dadd_rn(1., __dmul_rn(P.lam_m1, t)));
}

// forcey += .5 (I(i,j,k) + I(i,j+1,k)) sin(thetainc) (ta/Rep^2)^(1/4), forcez
// likewise with I(i,j,k+1) and -cos(thetainc), in the reference's order
template <class T>
__global__ void centrifugal_kernel(IndPost P, const double* __restrict__ sol, double sin_t, double mcos_t,
                                   double amp, T* __restrict__ fy, T* __restrict__ fz) {
  const IndGrid& g = P.g;
  const long n = (long)g.itot * g.jtot * g.ktot;
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int i = (int)(q % g.itot) + 1, j = (int)((q / g.itot) % g.jtot) + 1, k = (int)(q / ((long)g.itot * g.jtot)) + 1;
  auto I = [&](int a, int b, int c) {
    const double v = ind_value(P, sol, a, b, c);
    const bool interior = b <= g.jtot && c <= g.ktot;  // a, b, c >= 1 here
    return interior ? thresholds(v) : v;
  };
  const long o = ((long)k * g.ldj + j) * g.ldi + i;
  const double c0 = I(i, j, k);
  if (fy) fy[o] = (T)__dadd_rn((double)fy[o], __dmul_rn(__dmul_rn(.5 * (c0 + I(i, j + 1, k)), sin_t), amp));
  if (fz) fz[o] = (T)__dadd_rn((double)fz[o], __dmul_rn(__dmul_rn(.5 * (c0 + I(i, j, k + 1)), mcos_t), amp));
}

unsigned blocks(long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

int indicator_setup(sg_ctx* c, double visc0, double lambda, double thetainc, double ta, double rep) {
  const sg_config& f = c->cfg;
  if (!std::isfinite(visc0) || !std::isfinite(lambda) || !std::isfinite(thetainc) || !(ta >= 0.0) ||
      !std::isfinite(ta) || !(rep > 0.0) || !std::isfinite(rep))
    return fail(c, SG_ERR_ARG, "indicator parameters must be finite, ta >= 0 and rep > 0");
  SG_RET(poisson_setup(c, 1u << 0));
  auto& s = c->ind;
  s.visc0 = visc0;
  s.lambda = lambda;
  s.sin_t = std::sin(thetainc);
  s.mcos_t = -std::cos(thetainc);
  s.amp = std::pow(ta / std::pow(rep, 2.), .25);
  if (s.ready) return SG_OK;
  const double dz = f.lz / f.ktot;
  // the taller grid: ktot + 2 planes, so that its interior is k = 0 .. kmax + 1
  if (!make_ib_grid(f.itot, f.jtot, f.ktot + 2, f.lx, f.ly, f.lz + 2 * dz, s.grid, 0) &&
      !make_ib_grid(f.itot, f.jtot, f.ktot + 2, f.lx, f.ly, f.lz + 2 * dz, s.grid, 3))
    return fail(c, SG_ERR_CONFIG, "no FP64 tile shape fits the indicator grid");
  const IBGrid& g = s.grid;
  const long np = c->npts;
  SG_TRY(dalloc(c, s.w.pos, sizeof(PosRec<double>) * std::max(np, 1L)), "alloc");
  SG_TRY(dalloc(c, s.w.frc, sizeof(ForceRec<double>) * std::max(np, 1L)), "alloc");
  SG_TRY(dalloc(c, s.w.entries, sizeof(int) * 8 * std::max(np, 1L)), "alloc");
  SG_TRY(dalloc(c, s.w.counts, sizeof(int) * g.ntiles), "alloc");
  SG_TRY(dalloc(c, s.w.starts, sizeof(int) * (g.ntiles + 1)), "alloc");
  SG_TRY(dalloc(c, s.w.fill, sizeof(int) * g.ntiles), "alloc");
  SG_TRY(dalloc(c, s.zr, sizeof(double) * std::max(np, 1L)), "alloc");
  SG_TRY(dalloc(c, s.g, sizeof(double) * 3 * (size_t)g.ldi * g.ldj * g.ldk), "alloc");
  s.ready = true;
  return SG_OK;
}

template <class T>
int indicator_run(sg_ctx* c, const double* X, const double* Y, const double* Z, const T* NX, const T* NY, const T* NZ,
                  const T* A, T* indic, T* visc, T* fy, T* fz) {
  const sg_config& f = c->cfg;
  auto& s = c->ind;
  const IBGrid& g = s.grid;
  cudaStream_t st = c->st;
  const long np = c->npts;
  const double dz = f.lz / f.ktot;
  const int q = f.ktot / 4;
  // 1. raised positions (+ q dz, and one more plane for the taller grid), binning, records, spread
  if (np > 0) {
    raise_z_kernel<<<blocks(np), 256, 0, st>>>(np, (q + 1) * dz, Z, s.zr);
    pack_normals_kernel<T><<<blocks(np), 256, 0, st>>>(np, g.dvi, NX, NY, NZ, A, (ForceRec<double>*)s.w.frc);
  }
  SG_TRY(launch_bin<double>(g, np, X, Y, s.zr, s.w, st), "indicator binning");
  const long gsz = (long)g.ldi * g.ldj * g.ldk;
  SG_TRY(launch_spread_centred<double>(g, s.w, s.g, s.g + gsz, s.g + 2 * gsz, st), "indicator spread");
  // 2. divergence, then solver1d after initsolver(0)
  IndGrid ig{f.itot, f.jtot, f.ktot, g.ldi, g.ldj, g.dxi, g.dyi, g.dzi};
  const long nreal = (long)f.itot * f.jtot * f.ktot;
  double* r = c->pois.r;
  divergence_kernel<<<blocks(nreal), 256, 0, st>>>(ig, s.g, s.g + gsz, s.g + 2 * gsz, r);
  SG_RET(poisson_solve(c, r, 0, 0.0, st));
  // 3. indicator, viscosity, centrifugal terms
  IndPost P{ig, q, 1.0 / ((double)f.itot * f.jtot), s.visc0, s.lambda - 1.};
  const long nf = (long)g.ldi * g.ldj * (f.ktot + 2);
  indic_kernel<T><<<blocks(nf), 256, 0, st>>>(P, r, indic, visc);
  if (fy || fz) centrifugal_kernel<T><<<blocks(nreal), 256, 0, st>>>(P, r, s.sin_t, s.mcos_t, s.amp, fy, fz);
  SG_TRY(cudaGetLastError(), "indicator");
  c->launches += 5 + (np > 0 ? 2 : 0) + ((fy || fz) ? 1 : 0);
  return SG_OK;
}

template int indicator_run<double>(sg_ctx*, const double*, const double*, const double*, const double*,
                                   const double*, const double*, const double*, double*, double*, double*,
                                   double*);
template int indicator_run<float>(sg_ctx*, const double*, const double*, const double*, const float*, const float*,
                                  const float*, const float*, float*, float*, float*, float*);

}  // namespace sg
