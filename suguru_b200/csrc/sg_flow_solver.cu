// sg_flow_solver.cu -- one step of the reference's FFT flow solver
// (fsolver = 'f', main.f90:333-347) on the GPU, FP64:
//
//  fftuvw (fftuvw.f90:13-127): per interior cell the right-hand sides
//      Rep (-(momxp) - (momxad) - uo / dt), and likewise for v and w:
//      momxp = -dxi (p(i+1) - p(i)) + forcex (mom.f90:113-134), momxad the
//      Adams-Bashforth convection 1.5 (level n) - 0.5 (level n-1) of the
//      face fluxes (mom.f90:9-54, 136-181, 266-311); the w right-hand side
//      is zero in the top row; then the Helmholtz solves of solver1d after
//      initsolver(3) for w and initsolver(2) for u and v (sg_poisson.cu);
//  bounduvw (bound.f90:7-86): wall rows and periodic x, y halos;
//  fillps (fillps.f90): the divergence over dt, solver1d after
//      initsolver(1), boundp;
//  correc (correc.f90): the velocity minus dt times the pressure gradient,
//      bounduvw; pnew += p, boundp.
//
// One thread per cell; every field is (0:i1,0:j1,0:k1) with x fastest.  A
// halo kernel computes each halo cell from the interior cell it copies, so
// that it reads nothing another thread writes.
#include <cmath>

#include "sg_common.cuh"
#include "sg_ctx.h"

namespace sg {
namespace {

struct FGrid {
  int itot, jtot, ktot, ldi, ldj;
  long plane;
  double dxi, dyi, dzi;
};

__device__ __forceinline__ long at(const FGrid& g, int i, int j, int k) {
  return (long)k * g.plane + (long)j * g.ldi + i;
}

// interior cell q (x fastest) -> (i, j, k), 1-based
__device__ __forceinline__ void cell_of(const FGrid& g, long q, int& i, int& j, int& k) {
  i = (int)(q % g.itot) + 1;
  j = (int)((q / g.itot) % g.jtot) + 1;
  k = (int)(q / ((long)g.itot * g.jtot)) + 1;
}

struct Flux {
  double x, y, z;  // -p + m of each direction
};

// the face fluxes of momxad / momyad / momzad for component C at one level
template <int C>
__device__ __forceinline__ Flux fluxes(const FGrid& g, const double* __restrict__ U, const double* __restrict__ V,
                                       const double* __restrict__ W, int i, int j, int k) {
  const long o = at(g, i, j, k), ox = 1, oy = g.ldi, oz = g.plane;
  double xp, xm, yp, ym, zp, zm;
  if (C == 0) {
    xp = 0.25 * (U[o + ox] + U[o]) * (U[o + ox] + U[o]);
    xm = 0.25 * (U[o - ox] + U[o]) * (U[o - ox] + U[o]);
    yp = 0.25 * (U[o + oy] + U[o]) * (V[o + ox] + V[o]);
    ym = 0.25 * (U[o - oy] + U[o]) * (V[o + ox - oy] + V[o - oy]);
    zp = 0.25 * (U[o + oz] + U[o]) * (W[o + ox] + W[o]);
    zm = 0.25 * (U[o - oz] + U[o]) * (W[o + ox - oz] + W[o - oz]);
  } else if (C == 1) {
    xp = 0.25 * (U[o] + U[o + oy]) * (V[o] + V[o + ox]);
    xm = 0.25 * (U[o - ox] + U[o - ox + oy]) * (V[o] + V[o - ox]);
    yp = 0.25 * (V[o] + V[o + oy]) * (V[o] + V[o + oy]);
    ym = 0.25 * (V[o] + V[o - oy]) * (V[o] + V[o - oy]);
    zp = 0.25 * (W[o] + W[o + oy]) * (V[o + oz] + V[o]);
    zm = 0.25 * (W[o - oz] + W[o - oz + oy]) * (V[o - oz] + V[o]);
  } else {
    xp = 0.25 * (W[o] + W[o + ox]) * (U[o] + U[o + oz]);
    xm = 0.25 * (W[o] + W[o - ox]) * (U[o - ox] + U[o - ox + oz]);
    yp = 0.25 * (W[o] + W[o + oy]) * (V[o] + V[o + oz]);
    ym = 0.25 * (W[o] + W[o - oy]) * (V[o - oy] + V[o - oy + oz]);
    zp = 0.25 * (W[o] + W[o + oz]) * (W[o] + W[o + oz]);
    zm = 0.25 * (W[o] + W[o - oz]) * (W[o] + W[o - oz]);
  }
  return Flux{-xp + xm, -yp + ym, -zp + zm};
}

struct Fields {
  const double *uo, *vo, *wo, *uoo, *voo, *woo, *p, *fx, *fy, *fz;
};

// fftuvw's right-hand sides of u, v and w into the solver's layout
// [k-1][j-1][i-1], one thread per interior cell for all three (the stencils
// share most of their loads)
template <int C>
__device__ __forceinline__ double momentum_rhs(const FGrid& g, const Fields& F, double dt, double rep, int i, int j,
                                               int k) {
  const long o = at(g, i, j, k);
  const long step = C == 0 ? 1 : (C == 1 ? g.ldi : g.plane);
  const double dd = C == 0 ? g.dxi : (C == 1 ? g.dyi : g.dzi);
  const double* f = C == 0 ? F.fx : (C == 1 ? F.fy : F.fz);
  const double* vo = C == 0 ? F.uo : (C == 1 ? F.vo : F.wo);
  const double durk = (-dd * ((F.p[o + step] - F.p[o]))) + f[o];
  const Flux a = fluxes<C>(g, F.uo, F.vo, F.wo, i, j, k);
  const Flux b = fluxes<C>(g, F.uoo, F.voo, F.woo, i, j, k);
  const double ad = g.dxi * ((1.5 * a.x) - (.5 * b.x)) + g.dyi * ((1.5 * a.y) - (.5 * b.y)) +
                    g.dzi * ((1.5 * a.z) - (.5 * b.z));
  double d = -durk;
  d = d - ad;
  d = d - (vo[o] / dt);
  return d * rep;
}

// Blocks of 32 x 8 cells in (x, y) that march up kMomZ consecutive z levels,
// so that the stencil's y neighbours of a warp are mostly the block's own
// loads and its z neighbours the block's loads of the levels just before
// and after (L1), not L2's.
constexpr int kMomZ = 8;

__global__ void __launch_bounds__(256) momentum_rhs_kernel(FGrid g, Fields F, double dt, double rep,
                                                           double* __restrict__ ru, double* __restrict__ rv,
                                                           double* __restrict__ rw) {
  const int nbx = (g.itot + 31) / 32;
  const int i = (int)(blockIdx.x % nbx) * 32 + (int)(threadIdx.x & 31) + 1;
  const int j = (int)(blockIdx.x / nbx) * 8 + (int)(threadIdx.x >> 5) + 1;
  if (i > g.itot || j > g.jtot) return;
  const int k0 = (int)blockIdx.y * kMomZ + 1, k1 = min(k0 + kMomZ, g.ktot + 1);
  for (int k = k0; k < k1; ++k) {
    const long q = ((long)(k - 1) * g.jtot + (j - 1)) * g.itot + (i - 1);
    ru[q] = momentum_rhs<0>(g, F, dt, rep, i, j, k);
    rv[q] = momentum_rhs<1>(g, F, dt, rep, i, j, k);
    rw[q] = k == g.ktot ? 0.0 : momentum_rhs<2>(g, F, dt, rep, i, j, k);  // dwdt(i,j,kmax) = 0 (fftuvw.f90:86-92)
  }
}

// bounduvw (mode 0: u; 1: v with wall values vb2, vt2; 2: w) or boundp (mode
// 3) on the cells outside the interior, from the rule of bound.f90:7-139 at
// the interior column each copies.  One thread per halo cell: the two z
// planes (all i, j), then the two y rows (k = 1..kmax, all i), then the two
// x columns (k = 1..kmax, j = 1..jmax).  The w row kmax of the interior is
// already zero: its right-hand side is zero and its row the identity.
__global__ void halo_kernel(FGrid g, int mode, double vb2, double vt2, double* __restrict__ f) {
  const long nz = 2L * g.ldi * g.ldj, ny = 2L * g.ldi * g.ktot, nx = 2L * g.jtot * g.ktot;
  long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (q < nz) {
    k = q < g.plane ? 0 : g.ktot + 1;
    q %= g.plane;
    j = (int)(q / g.ldi);
    i = (int)(q % g.ldi);
  } else if ((q -= nz) < ny) {
    const long side = (long)g.ldi * g.ktot;
    j = q < side ? 0 : g.jtot + 1;
    q %= side;
    k = 1 + (int)(q / g.ldi);
    i = (int)(q % g.ldi);
  } else if ((q -= ny) < nx) {
    const long side = (long)g.jtot * g.ktot;
    i = q < side ? 0 : g.itot + 1;
    q %= side;
    k = 1 + (int)(q / g.jtot);
    j = 1 + (int)(q % g.jtot);
  } else {
    return;
  }
  const long o = at(g, i, j, k);
  const int is = i == 0 ? g.itot : (i == g.itot + 1 ? 1 : i);
  const int js = j == 0 ? g.jtot : (j == g.jtot + 1 ? 1 : j);
  double v;
  if (mode == 2 && k == g.ktot) {  // w(i,j,kmax) = 0 in the halos too
    v = 0.0;
  } else if (k >= 1 && k <= g.ktot) {
    v = f[at(g, is, js, k)];
  } else if (k == 0) {
    const double f1 = f[at(g, is, js, 1)];
    v = mode == 0 ? -f1 : (mode == 1 ? vb2 - f1 : (mode == 2 ? 0.0 : f1));
  } else {
    const double fk = f[at(g, is, js, g.ktot)];
    v = mode == 0 ? -fk : (mode == 1 ? vt2 - fk : (mode == 2 ? f[at(g, is, js, g.ktot - 1)] : fk));
  }
  f[o] = v;
}

// fillps: the divergence of the predicted velocity over dt
__global__ void fillps_kernel(FGrid g, double dti, const double* __restrict__ u, const double* __restrict__ v,
                              const double* __restrict__ w, double* __restrict__ rhs) {
  const long n = (long)g.itot * g.jtot * g.ktot;
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  int i, j, k;
  cell_of(g, q, i, j, k);
  const long o = at(g, i, j, k);
  rhs[q] = ((w[o] - w[o - g.plane]) * (dti * g.dzi) + (v[o] - v[o - g.ldi]) * (dti * g.dyi)) +
           (u[o] - u[o - 1]) * (dti * g.dxi);
}

// correc
__global__ void correc_kernel(FGrid g, double dt, const double* __restrict__ p, double* __restrict__ u,
                              double* __restrict__ v, double* __restrict__ w) {
  const long n = (long)g.itot * g.jtot * g.ktot;
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  int i, j, k;
  cell_of(g, q, i, j, k);
  const long o = at(g, i, j, k);
  u[o] = u[o] - (dt * g.dxi) * (p[o + 1] - p[o]);
  v[o] = v[o] - (dt * g.dyi) * (p[o + g.ldi] - p[o]);
  w[o] = w[o] - (dt * g.dzi) * (p[o + g.plane] - p[o]);
}

__global__ void add_interior_kernel(FGrid g, const double* __restrict__ p, double* __restrict__ pn) {
  const long n = (long)g.itot * g.jtot * g.ktot;
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  int i, j, k;
  cell_of(g, q, i, j, k);
  const long o = at(g, i, j, k);
  pn[o] = pn[o] + p[o];
}

unsigned blocks(long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

int flow_setup(sg_ctx* c, double rep, double vb2, double vt2) {
  if (c->mixed) return fail(c, SG_ERR_CONFIG, "the flow solver runs on FP64 contexts");
  if (!(rep > 0.0) || !std::isfinite(rep) || !std::isfinite(vb2) || !std::isfinite(vt2))
    return fail(c, SG_ERR_ARG, "rep must be positive and finite, the wall values finite");
  SG_RET(poisson_setup(c, (1u << 1) | (1u << 2) | (1u << 3)));
  auto& s = c->flow;
  s.rep = rep;
  s.vb2 = vb2;
  s.vt2 = vt2;
  if (s.ready) return SG_OK;
  const sg_config& f = c->cfg;
  const long nreal = (long)f.itot * f.jtot * f.ktot;
  SG_TRY(dalloc(c, s.ru, sizeof(double) * nreal), "alloc");
  SG_TRY(dalloc(c, s.rv, sizeof(double) * nreal), "alloc");
  SG_TRY(dalloc(c, s.p, sizeof(double) * c->nfield), "alloc");
  if (f.mem == SG_MEM_HOST)
    for (int q = 0; q < 13; ++q) SG_TRY(dalloc(c, s.stage[q], sizeof(double) * c->nfield), "alloc");
  s.ready = true;
  return SG_OK;
}

int flow_run(sg_ctx* c, double dt, const double* uo, const double* vo, const double* wo, const double* uoo,
             const double* voo, const double* woo, double* p, const double* fx, const double* fy, const double* fz,
             double* u, double* v, double* w) {
  const sg_config& f = c->cfg;
  auto& s = c->flow;
  cudaStream_t st = c->st;
  const IBGrid& ib = c->grid;
  FGrid g{f.itot, f.jtot, f.ktot, ib.ldi, ib.ldj, (long)ib.ldi * ib.ldj, 1.0 / (f.lx / f.itot),
          1.0 / (f.ly / f.jtot), 1.0 / (f.lz / f.ktot)};
  const long nreal = (long)f.itot * f.jtot * f.ktot, nf = c->nfield - nreal;  // halo cells
  const double inv_n = 1.0 / ((double)f.itot * f.jtot), shift = s.rep / dt;
  double* rw = c->pois.r;
  Fields F{uo, vo, wo, uoo, voo, woo, p, fx, fy, fz};
  // fftuvw: right-hand sides, then w (initsolver(3)) and u, v (initsolver(2))
  const dim3 mgrid((unsigned)(((f.itot + 31) / 32) * ((f.jtot + 7) / 8)), (unsigned)((f.ktot + kMomZ - 1) / kMomZ));
  momentum_rhs_kernel<<<mgrid, 256, 0, st>>>(g, F, dt, s.rep, s.ru, s.rv, rw);
  SG_TRY(cudaGetLastError(), "momentum");
  // each solution goes, times 1 / (itot jtot), straight into its field
  const PoisOut ow{w, g.ldi, g.plane, inv_n}, ou{u, g.ldi, g.plane, inv_n}, ov{v, g.ldi, g.plane, inv_n},
      op{s.p, g.ldi, g.plane, inv_n};
  SG_RET(poisson_solve(c, rw, 3, shift, st, &ow));
  SG_RET(poisson_solve(c, s.ru, 2, shift, st, &ou));
  SG_RET(poisson_solve(c, s.rv, 2, shift, st, &ov));
  halo_kernel<<<blocks(nf), 256, 0, st>>>(g, 0, s.vb2, s.vt2, u);
  halo_kernel<<<blocks(nf), 256, 0, st>>>(g, 1, s.vb2, s.vt2, v);
  halo_kernel<<<blocks(nf), 256, 0, st>>>(g, 2, s.vb2, s.vt2, w);
  // projection: fillps, solver1d after initsolver(1), boundp, correc, bounduvw
  fillps_kernel<<<blocks(nreal), 256, 0, st>>>(g, 1.0 / dt, u, v, w, rw);
  SG_RET(poisson_solve(c, rw, 1, 0.0, st, &op));
  halo_kernel<<<blocks(nf), 256, 0, st>>>(g, 3, 0.0, 0.0, s.p);
  correc_kernel<<<blocks(nreal), 256, 0, st>>>(g, dt, s.p, u, v, w);
  halo_kernel<<<blocks(nf), 256, 0, st>>>(g, 0, s.vb2, s.vt2, u);
  halo_kernel<<<blocks(nf), 256, 0, st>>>(g, 1, s.vb2, s.vt2, v);
  halo_kernel<<<blocks(nf), 256, 0, st>>>(g, 2, s.vb2, s.vt2, w);
  // pnew += p, boundp
  add_interior_kernel<<<blocks(nreal), 256, 0, st>>>(g, s.p, p);
  halo_kernel<<<blocks(nf), 256, 0, st>>>(g, 3, 0.0, 0.0, p);
  SG_TRY(cudaGetLastError(), "flow step");
  c->launches += 12;
  return SG_OK;
}

}  // namespace sg
