/*
 * sg_oracle.h -- CPU FP64 restatement of the reference coupling step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle and the timed
 * CPU baseline.  Only tests/, __graft_entry__.smoke() and the cpu_baseline leg
 * of bench.py may load it; the product path (suguru_b200/) never does.
 *
 * Every routine restates an algorithm of the reference (WhiteTshirtXI/Suguru,
 * Fortran 90 + SPHEREPACK 3.2 + GSL 1.16); the file:line it follows is given
 * beside each declaration.  Grid arrays are row-major [lat][lon] (longitude
 * fastest), which is the reference's flat point order cap=(i-1)*m_capf+j
 * (forcing.f90:39).  SH coefficients are a[m*ld+n], b[m*ld+n].
 * Eulerian arrays are Fortran column-major (0:i1,0:j1,0:k1), x fastest
 * (common.f90:6).
 */
#ifndef SG_ORACLE_H
#define SG_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* gaqd.f:45 -- Gauss-Legendre colatitudes (0,pi) north->south and weights (sum 2). */
int or_gaqd(int nlat, double* theta, double* wts);

/* sphharm.c:38-108 (GSL sphPlm * sqrt(2pi) * (-1)^m), converted to theta
 * derivatives as sph3.f90:57-65 does.  Tables are [m*nn+n] for m<mm, n<nn
 * (zero for n<m) at one colatitude.  dP, d2P may be NULL. */
void or_legendre(double theta, int mm, int nn, double* P, double* dP, double* d2P);

/* shagc.f:306-526 -- Gaussian-grid analysis of nf fields g[f][lat][lon];
 * a,b are [f][m*nlat+n] with m<l=min(nlat,(nlon+2)/2), n<nlat. */
int or_shagc(int nlat, int nlon, int nf, const double* g, double* a, double* b);
/* shsgc.f:289-500 -- synthesis (inverse of or_shagc). */
int or_shsgc(int nlat, int nlon, int nf, const double* a, const double* b, double* g);
/* trssph.f:480-690 with igrida=igridb=(-2,1) -- Gauss grid A -> Gauss grid B. */
int or_trssph(int nlata, int nlona, int nf, const double* da, int nlatb, int nlonb, double* db);

/* kernel.f90:7-25 -- Roma-Peskin 3-point delta (times the grid spacing). */
double or_kernel(double r);
/* kernel.f90:43-63 */
double or_kerneltest(void);

/* One capsule of SH degree L (force grid 2(L+1) x 4(L+1), SH grid (L+1) x 2(L+1)).
 * Reference state: sphere of radius `radius` (sph.f90:60-88, scaled).
 * complagrforces (forcing.f90:11-114) for that capsule: positions xfp,yfp,zfp
 * (flat, cap=i*m_capf+j) -> force fx,fy,fz, normals nx,ny,nz, area.
 * faithful=1 re-initialises Gauss nodes and Legendre tables on every analysis
 * as the reference does (sph1.f90:54-76, trssph intl=0); faithful=0 caches them.
 * gs, csk: Skalak modulus and area-dilation constant (membmodel.c:81-99). */
int or_complagrforces(int L, double radius, double gs, double csk, int faithful,
                      const double* xfp, const double* yfp, const double* zfp,
                      double* fx, double* fy, double* fz,
                      double* nx, double* ny, double* nz, double* area);
/* Same with the membrane law chosen: law 0 Skalak (membmodel.c:81-99), 1
 * neo-Hookean (membmodel.c:60-79, the reference's -DNONHOOK build). */
int or_complagrforces_law(int L, double radius, double gs, double csk, int law, int faithful,
                          const double* xfp, const double* yfp, const double* zfp,
                          double* fx, double* fy, double* fz,
                          double* nx, double* ny, double* nz, double* area);

/* Same with the bending terms of ibend = 1 (param.f90:90-91): eb is the
 * bending modulus (ebend = cbend gscell); the third and fourth derivatives of
 * the shape (sph3.f90:137-180), the curvature and metric derivatives
 * (sph.f90:479-731, 802-890, 962-1111, sph1.f90:299-542), the moment, the
 * transverse shear and their terms in the equilibrium (sph.f90:1236-1454,
 * 1705-1709), with the reference sphere's tensors as the reference state.
 * eb = 0 gives or_complagrforces_law. */
int or_complagrforces_bend(int L, double radius, double gs, double csk, int law, double eb, int faithful,
                           const double* xfp, const double* yfp, const double* zfp,
                           double* fx, double* fy, double* fz,
                           double* nx, double* ny, double* nz, double* area);

/* Same, but also returns the dealias-grid pointwise force before filtering
 * (fxN..) and the shape coefficients; used by the surrogate data path tests.
 * coef: [3][m*N+n] a then b (each 3*N*N); fcoef: force coefficients (degree<N)
 * of the filtered force, same layout.  Any output pointer may be NULL. */
int or_capsule_spectra(int L, double radius, double gs, double csk,
                       const double* xfp, const double* yfp, const double* zfp,
                       double* shape_a, double* shape_b, double* force_a, double* force_b);

/* Eulerian grid: itot x jtot x ktot interior cells, spacing dx,dy,dz; arrays
 * carry a one-cell halo, Fortran order, so ld_i=itot+2, ld_j=jtot+2, ld_k=ktot+2. */
/* eulr2lagr (interp_spread.f90:12-475) for npts points, periodic x,y, walls z. */
int or_interp(int itot, int jtot, int ktot, double dx, double dy, double dz, int faithful,
              const double* u, const double* v, const double* w,
              long npts, const double* xp, const double* yp, const double* zp,
              double* ul, double* vl, double* wl);
/* lagr2eulr (interp_spread.f90:510-922): zero, scatter f*area/dV, halo copy (bound.f90:141-190). */
int or_spread(int itot, int jtot, int ktot, double dx, double dy, double dz, int faithful,
              long npts, const double* xp, const double* yp, const double* zp,
              const double* fxl, const double* fyl, const double* fzl, const double* area,
              double* fx, double* fy, double* fz);

/* lagr2eulrind (interp_spread.f90:978-1387): normals * area spread with
 * cell-centre weights in every direction, z window [0, kmax+1], periodic
 * x, y halo copies.  Fields (0:i1,0:j1,0:k1), x fastest. */
int or_spread_ind(int itot, int jtot, int ktot, double dx, double dy, double dz, int faithful, long npts,
                  const double* xp, const double* yp, const double* zp, const double* nxl, const double* nyl,
                  const double* nzl, const double* area, double* gx, double* gy, double* gz);

/* Update_Pos.f90:95-126: forward Euler + wall clamp to [0,lz]. */
void or_update_pos(long npts, double dt, double lz, double* xp, double* yp, double* zp,
                   const double* ul, const double* vl, const double* wl);
/* Update_Pos.f90:95-180 for ncap capsules (points off[p] .. off[p+1]-1):
 * or_update_pos, then each capsule's sequential centroid and its shift by
 * one period in x or y when the centroid has left [0, lx] x [0, ly]. */
void or_update_pos_capsules(int ncap, const long* off, double dt, double lx, double ly, double lz, double* xp,
                            double* yp, double* zp, const double* ul, const double* vl, const double* wl);

/* surf_vol.f90:12-131 for one capsule of nl points.  out[0]=volume,
 * out[1]=total area, out[2]=exy1, out[3]=exy2, out[4..6]=centroid.
 * exy1_prev is returned in out[2] when no principal axis matches (the
 * reference leaves the global exy1 unchanged then). */
void or_surf_vol(long nl, const double* xp, const double* yp, const double* zp,
                 const double* nx, const double* ny, const double* nz, const double* area,
                 double exy1_prev, double* out);

/* collisions.f90:10-32: Morse wall force added to fzl (bottom wall). */
void or_collisions(long nl, const double* zp, const double* area, double dx, double dy,
                   double col, double betacol, double rep, double rad0, double* fzl);

/* membmodel.c:81-99 (Skalak) restated: out = W1, W2, dW1/dxi[2], dW2/dxi[2]. */
void or_skalak(double I1, double I2, const double* I1de, const double* I2de, double gs, double csk, double* out);
/* membmodel.c:60-99 restated for law 0 (Skalak) or 1 (neo-Hookean). */
void or_membrane_law(int law, double I1, double I2, const double* I1de, const double* I2de, double gs, double csk,
                     double* out);

/* Whole step over ncap capsules (interp, forces, spread) with OpenMP over
 * capsules when nthreads>1; returns seconds spent per stage in t[3]. */
int or_coupling_step(int itot, int jtot, int ktot, double dx, double dy, double dz,
                     int ncap, const int* degree, const double* radius, double gs, double csk,
                     int faithful, int nthreads,
                     const double* u, const double* v, const double* w,
                     const double* xp, const double* yp, const double* zp,
                     double* ul, double* vl, double* wl,
                     double* fxl, double* fyl, double* fzl,
                     double* nx, double* ny, double* nz, double* area,
                     double* fx, double* fy, double* fz, double* t);

#ifdef __cplusplus
}
#endif
#endif
