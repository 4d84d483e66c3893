/*
 * sg_coupling.h -- C ABI of the B200 fluid-structure coupling step.
 *
 * Drop-in boundary for the reference's coupling step (WhiteTshirtXI/Suguru,
 * Fortran 90).  The reference calls, once per time step (main.f90:225-241):
 *
 *   call eulr2lagr        ! interp_spread.f90:12   Eulerian velocity -> ul,vl,wl
 *   call complagrforces   ! forcing.f90:11         membrane force fxl.., normals xn.., area
 *   call collisions       ! collisions.f90:10      (wall Morse term, optional)
 *   call lagr2eulr        ! interp_spread.f90:510  fxl.. * area -> forcex,forcey,forcez
 *   call Update_Pos       ! Update_Pos.f90:12      xfp += ul*dt, wall clamp
 *   call surf_vol         ! surf_vol.f90:12        volume / deformation diagnostics
 *
 * None of those subroutines takes arguments; they act on module globals
 * (common.f90:6-9,67-90).  The functions below take the same arrays as plain
 * pointers, so a thin iso_c_binding shim keeps the Fortran names and packs
 * ap(p)%xfp... into contiguous buffers.
 *
 * Conventions
 *  - Eulerian arrays: Fortran (0:i1,0:j1,0:k1), x fastest, i1=itot+1 etc.
 *    (common.f90:6); u at faces i*dx, v at j*dy, w at k*dz (MAC grid).
 *  - Lagrangian arrays: capsules concatenated; capsule c of SH degree L owns
 *    8(L+1)^2 points in the reference flat order cap=(i-1)*m_capf+j on the
 *    2(L+1) x 4(L+1) Gauss force grid (forcing.f90:37-44).
 *  - Precision SG_PREC_FP64: every array is double.  SG_PREC_MIXED: positions
 *    X,Y,Z stay double; Eulerian fields and Lagrangian outputs are float.
 *  - mem = SG_MEM_HOST: arrays are host memory, copied in and out per call;
 *    SG_MEM_DEVICE: arrays are device pointers on cfg->device.
 *  - Every function returns 0 on success or an SG_ERR_* code; sg_last_error
 *    gives the text.  Errors are integer status codes in the spirit of
 *    SPHEREPACK's ierror (shagc.f:221-231), never aborts.
 *  - One host thread per context; calls are synchronous at return unless
 *    cfg->async is set.
 */
#ifndef SG_COUPLING_H
#define SG_COUPLING_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

#define SG_OK 0
#define SG_ERR_CONFIG 1   /* invalid configuration */
#define SG_ERR_CUDA 2     /* CUDA runtime error */
#define SG_ERR_TIMEOUT 3  /* a bounded device wait expired */
#define SG_ERR_FALLBACK 4 /* surrogate fallback count above the allowed maximum */
#define SG_ERR_ARG 5      /* bad argument (null pointer, size) */
#define SG_ERR_STATE 6    /* call not valid in the current state */
#define SG_ERR_TOO_LARGE 7 /* problem larger than sg_spread_noalloc's fixed scratch */

#define SG_PREC_FP64 0
#define SG_PREC_MIXED 1
#define SG_MEM_HOST 0
#define SG_MEM_DEVICE 1

typedef struct sg_ctx sg_ctx;

typedef struct sg_config {
  int itot, jtot, ktot;   /* interior cells imax, jmax, kmax (param.f90:18-21) */
  double lx, ly, lz;      /* domain lengths (param.f90:23); periodic x,y, walls z */
  int ncap;               /* number of capsules (np, param.f90:43) */
  const int* degree;      /* [ncap] SH degree L per capsule, 2 <= L <= 31 */
  const double* radius;   /* [ncap] reference-sphere radius (sph.f90:60-88) */
  double gs;              /* surface shear modulus Gs (gscell, param.f90:88) */
  double csk;             /* Skalak area-dilation constant C (CSK, param.f90:88) */
  int precision;          /* SG_PREC_FP64 or SG_PREC_MIXED */
  int surrogate;          /* 1: learned membrane force with plain fallback (mixed only) */
  int mem;                /* SG_MEM_HOST or SG_MEM_DEVICE */
  int device;             /* CUDA device ordinal */
  int async;              /* 1: return without synchronising the context stream */
  void* stream;           /* cudaStream_t to run on, or NULL for a private stream */
} sg_config;

/* Create / destroy a context.  All device memory is allocated here; the step
 * calls below allocate nothing. */
int sg_create(const sg_config* cfg, sg_ctx** out);
void sg_destroy(sg_ctx* ctx);
const char* sg_last_error(const sg_ctx* ctx);
int sg_synchronize(sg_ctx* ctx);

/* eulr2lagr (interp_spread.f90:12-475): U,V,W = J(X) [u,v,w]. */
int sg_interp(sg_ctx* ctx, const void* u, const void* v, const void* w,
              const double* X, const double* Y, const double* Z,
              void* U, void* V, void* W);

/* complagrforces (forcing.f90:11-114): membrane force, unit normals and
 * area of every force point. */
int sg_membrane_force(sg_ctx* ctx, const double* X, const double* Y, const double* Z,
                      void* FX, void* FY, void* FZ, void* NX, void* NY, void* NZ, void* AREA);

/* lagr2eulr (interp_spread.f90:510-922): fx,fy,fz = S(X)[F * AREA / dV],
 * whole field written, periodic halos copied as updthalos does (bound.f90:141-190). */
int sg_spread(sg_ctx* ctx, const double* X, const double* Y, const double* Z,
              const void* FX, const void* FY, const void* FZ, const void* AREA,
              void* fx, void* fy, void* fz);

/* One coupling step in the reference order (main.f90:225-233): interpolation,
 * membrane force, spreading; the points are binned once. */
int sg_step(sg_ctx* ctx, const void* u, const void* v, const void* w,
            const double* X, const double* Y, const double* Z,
            void* U, void* V, void* W,
            void* FX, void* FY, void* FZ, void* NX, void* NY, void* NZ, void* AREA,
            void* fx, void* fy, void* fz);

/* Update_Pos.f90:95-180: X += U*dt, clamp z into [0, lz], then shift every
 * point of a capsule by -lx (+lx) when the capsule's centroid is beyond lx
 * (below 0), and likewise in y. */
int sg_update_pos(sg_ctx* ctx, double dt, double* X, double* Y, double* Z,
                  const void* U, const void* V, const void* W);

/* surf_vol.f90:12-131 per capsule, FP64: out[7*c + {0..6}] = volume, area,
 * exy1, exy2, centroid x, y, z.  exy1_prev[c] is kept when no principal axis
 * matches (as the reference keeps the global exy1); may be NULL. */
int sg_surf_vol(sg_ctx* ctx, const double* X, const double* Y, const double* Z,
                const void* NX, const void* NY, const void* NZ, const void* AREA,
                const double* exy1_prev, double* out);

/* collisions (collisions.f90:10-32): FZ += the Morse-potential force of the
 * wall z = 0 on every point closer than rad0, summed over the wall's lattice
 * images (j dy, k dx) within the cutoff:
 *   fc = sum 2 col/rep^2 (e^{2 betacol (rad0-ss)} - e^{betacol (rad0-ss)})
 *        |z/ss| min(area, dx^2)/max(area, dx^2),  ss < rad0,
 * in FP64, added to FZ with one rounding.  A point exactly on the wall gives
 * 0/0 in |z/ss|, as in the reference.  The constants are those of the
 * reference's param.f90:57,64 (col = 5.68533e-2, betacol = 15.36,
 * rad0 = 2.5 dz, rep = Rep = 0.0016), set once with sg_set_wall_collisions.
 * in_step = 1 makes sg_step (and a graph captured from it) apply the force
 * between the membrane force and the spreading, as main.f90:229-233 calls
 * complagrforces, collisions, lagr2eulr; then FZ returned by sg_step includes
 * it.  sg_membrane_force never includes it (complagrforces does not).
 * Returns SG_ERR_STATE from sg_collisions before any parameters are set, and
 * from sg_set_wall_collisions while a captured graph exists. */
int sg_set_wall_collisions(sg_ctx* ctx, int in_step, double col, double betacol, double rad0, double rep);
int sg_collisions(sg_ctx* ctx, const double* Z, const void* AREA, void* FZ);

/* indicator (indicator.f90:19-182) on the main mesh (the overlap mesh,
 * ifoverlap = 1, is off by default): the capsules raised by ktot/4 dz,
 * G = normals * area spread with cell-centre weights (lagr2eulrind,
 * interp_spread.f90:978-1387), its central-difference divergence, the
 * Poisson solve of solver1d after initsolver(0) (periodic x, y by FFT,
 * Neumann z by the reference's elimination), the shift back, boundind, the
 * 0.01 / 0.9 thresholds on the interior; visc = visc0 (1 + (lambda - 1) I)
 * with boundp; and, when fy / fz are not NULL, forcey += .5 (I_j + I_j+1)
 * sin(thetainc) (ta/rep^2)^(1/4), forcez += .5 (I_k + I_k+1) (-cos(thetainc))
 * (ta/rep^2)^(1/4) on the interior.  indic, visc, fy, fz are fields in the
 * Eulerian layout above (visc, fy, fz may be NULL); NX.. AREA are the
 * normals and areas of sg_membrane_force.  The constants are those of
 * param.f90:52,57 (visc0 = 1/Rep, lambda, thetainc in radians, ta, Rep).
 * sg_set_indicator_params allocates the indicator's workspace and FFT plans
 * (itot even, ktot >= 4); sg_indicator allocates nothing and returns
 * SG_ERR_STATE before the parameters are set.  Computed in FP64 in both
 * precisions (the mixed path rounds its FP32 outputs once). */
int sg_set_indicator_params(sg_ctx* ctx, double visc0, double lambda, double thetainc, double ta, double rep);
int sg_indicator(sg_ctx* ctx, const double* X, const double* Y, const double* Z,
                 const void* NX, const void* NY, const void* NZ, const void* AREA,
                 void* indic, void* visc, void* fy, void* fz);

/* One step of the reference's FFT flow solver (fsolver = 'f',
 * main.f90:333-347), FP64 contexts only: fftuvw (fftuvw.f90:13-127: pressure
 * gradient plus the IB force, momxp..momzp; Adams-Bashforth convection from
 * the velocities uo (level n) and uoo (level n-1), momxad..momzad; implicit
 * Helmholtz solves of solver1d after initsolver(3) for w and initsolver(2)
 * for u, v), bounduvw, fillps, solver1d after initsolver(1), boundp, correc,
 * bounduvw, p += the pressure correction and boundp.  All arrays are fields
 * in the Eulerian layout above with their halos set as bounduvw / boundp
 * leave them; p (the reference's pnew) is updated in place; u, v, w receive
 * the new velocity.  fx, fy, fz are the IB force (sg_spread, plus the
 * centrifugal terms of sg_indicator when used).  sg_set_flow_params takes
 * Rep (param.f90:57) and the wall values of v, vb2 = v(0) + v(1) and
 * vt2 = v(k1) + v(kmax) (0, 0 for no-slip walls, iniu 'zer'; lz shear and
 * -lz shear for 'cou'; 2 bulk_v_sup for free slip), and allocates the
 * solver's workspace (itot even, ktot >= 4; in host memory mode also device
 * copies of the 13 fields).  The flow solver of the Crank-Nicolson path
 * (fsolver = 'c', crnk.f90) is not provided. */
int sg_set_flow_params(sg_ctx* ctx, double rep, double vb2, double vt2);
int sg_flow_step(sg_ctx* ctx, double dt, const double* uo, const double* vo, const double* wo,
                 const double* uoo, const double* voo, const double* woo, double* p,
                 const double* fx, const double* fy, const double* fz,
                 double* u, double* v, double* w);

/* The overlap mesh's lid (interpolation.f90:10-69, ifoverlap = 1): the main
 * mesh's u, v, w, p and indicator (FP64, Eulerian layout above) bilinearly
 * interpolated at the plane between z cells nf and nf + 1 onto the nodes
 * (i, j), 0 <= i <= itot nr + 1, 0 <= j <= jtot nr + 1, of the finer mesh
 * (nr = main cell / fine cell, param.f90:33-41): node (i, j) at
 * x = i dx/nr + (1 - 1/nr) dx / 2, y likewise.  u, v, p and the indicator are
 * the mean of planes nf and nf + 1, w its value at nf + 1.  Outputs
 * ub, vb, wb, pb, indb: (itot nr + 2) x (jtot nr + 2) doubles, i fastest, the
 * reference's (0:i1c, 0:j1c) arrays.  Bitwise the oracle's.  SG_ERR_ARG for
 * nr < 2 or nf outside 0 <= nf <= kmax.  In host memory mode the first call
 * allocates its device staging (two planes per field and the lid). */
int sg_overlap_lid(sg_ctx* ctx, int nf, int nr, const double* u, const double* v, const double* w,
                   const double* p, const double* indic, double* ub, double* vb, double* wb, double* pb,
                   double* indb);

/* Spreading for callers that cannot allocate device memory.  It has no
 * counterpart in the reference; it is sg_spread (lagr2eulr) without a
 * context.  It is for host codes whose device memory is all owned by their
 * own pool, and for code that must not call cudaMalloc or create an sg_ctx
 * (sg_create allocates).
 * The caller passes device arrays: the points X,Y,Z, force FX,FY,FZ and AREA
 * (npts each, FP64), and the fields fx,fy,fz in the Eulerian layout above.
 * The binning scratch is one fixed array of SG_NOALLOC_SCRATCH_BYTES compiled
 * into the library; every GPU that loads the library holds it until exit.
 * Output tiles: 32x8x4 cells when itot >= 32 and neither itot mod 32 nor
 * jtot mod 8 is 1 or 2, else 8x8x4 when neither itot mod 8 nor jtot mod 8 is
 * 1 or 2; a grid that neither fits returns SG_ERR_ARG.  The tile count is
 * ceil(itot/TX) ceil(jtot/TY) ceil(ktot/TZ) of the shape chosen.
 * Limits: npts <= SG_NOALLOC_MAX_POINTS and at most SG_NOALLOC_MAX_TILES
 * output tiles; a larger problem returns SG_ERR_TOO_LARGE before doing
 * anything.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress), so make that
 * first call before any stream capture.  Work is queued on `stream` (NULL:
 * the default stream) and the call returns without waiting.  All calls share
 * the one array, so calls that overlap on the GPU race; each call clears the
 * counters it needs, and otherwise the previous call's contents stay there.
 * Returns SG_OK, SG_ERR_ARG, SG_ERR_TOO_LARGE or SG_ERR_CUDA. */
#define SG_NOALLOC_MAX_POINTS 65536
#define SG_NOALLOC_MAX_TILES 16384
#define SG_NOALLOC_SCRATCH_BYTES (7424u * 1024u)
int sg_spread_noalloc(int itot, int jtot, int ktot, double lx, double ly, double lz, long npts,
                      const double* X, const double* Y, const double* Z,
                      const double* FX, const double* FY, const double* FZ, const double* AREA,
                      double* fx, double* fy, double* fz, void* stream);

/* Per-capsule Skalak constants (both NULL-able; default cfg->gs, cfg->csk).
 * The reference has one pair per run (gscell, CSK, param.f90:88); per-capsule
 * values serve training-data generation over a range of C. */
int sg_set_capsule_membrane(sg_ctx* ctx, const double* gs, const double* csk);

/* Membrane law per capsule (host array of ncap): SG_LAW_SKALAK (the default;
 * membmodel.c:81-99) or SG_LAW_NEO_HOOKEAN (membmodel.c:60-79, which the
 * reference selects at compile time with -DNONHOOK; C plays no part in it).
 * The surrogate, trained on the Skalak law, never takes neo-Hookean capsules.
 * Returns SG_ERR_ARG for another value, SG_ERR_STATE while a graph is
 * captured. */
#define SG_LAW_SKALAK 0
#define SG_LAW_NEO_HOOKEAN 1
int sg_set_capsule_law(sg_ctx* ctx, const int* law);

/* Force stage of the mixed path: fused (on = 1) runs the whole
 * stage -- centroid, longitude DFTs, the eight Legendre contractions in FP32
 * on CUDA cores, the pointwise geometry and mechanics, the SH-grid filter and
 * the final synthesis -- in one kernel, one CTA per capsule; staged (on = 0)
 * runs it as separate launches (the default), with the contractions on the
 * tensor cores (sg_set_tensor_cores).  Fused gives the bits of the staged
 * stage with FP32 contractions (sg_set_tensor_cores(0)), in one launch, at
 * about the staged stage's time.  Capsules that bend, and steps with the surrogate
 * on, always take the staged stage.  SG_ERR_CONFIG on an FP64 context,
 * SG_ERR_STATE while a graph is captured.  sg_get_fused_force: 1 or 0. */
int sg_set_fused_force(sg_ctx* ctx, int on);
int sg_get_fused_force(sg_ctx* ctx);

/* Bending modulus per capsule (host array of ncap, NULL = all 0): a nonzero
 * eb adds the bending terms of ibend = 1 (param.f90:90-91, eb = cbend gscell)
 * to the membrane force: the moment tensor from the curvature change
 * (cal_moment_deri, sph.f90:1236-1372), its transverse shear (cal_Q,
 * sph.f90:1375-1424) and the curvature-membrane products (cal_bcurmix,
 * sph.f90:1427-1454) in the equilibrium sums (sph.f90:1705-1709).  The
 * first nonzero modulus sets up the third and fourth theta-derivative
 * tables (sphharm.c:110-145) and one more contraction per step; with every
 * modulus 0 the step is the plain (ibend = 0) one.  Capsules with bending
 * never take the surrogate.  SG_ERR_ARG for a non-finite value,
 * SG_ERR_STATE while a graph is captured. */
int sg_set_capsule_bending(sg_ctx* ctx, const double* eb);

/* Spectral coefficients of the plain membrane model, per capsule: the
 * displacement from the reference sphere after the centroid is removed
 * (the analysis of cal_3dcrd_spectral_coeff, sph1.f90:29-79) and the force
 * after its filter (filter_modes4__OPT, sph1.f90:919-932).  Capsule k of
 * degree L writes 3 (L+1)^2 doubles to each array at offset
 * 3 * sum_{j<k} (L_j+1)^2: per component x, y, z, the SPHEREPACK a(m,n) for
 * 0 <= m <= n <= L in m-major order, then b(m,n) for 1 <= m <= n <= L.
 * Arrays follow cfg->mem.  Allocates its scratch on the first call. */
int sg_capsule_spectra(sg_ctx* ctx, const double* X, const double* Y, const double* Z,
                       double* disp, double* force);

/* Learned membrane-force surrogate (mixed precision, capsules of degree 15;
 * no counterpart in the reference, whose force is always the plain model).
 * Per capsule, with x the 768 displacement coefficients above divided by R
 * (slot 0, the x translation, carrying C; slots 256 and 512 zero), the force
 * coefficients times R/Gs are predicted as
 *   y = (L0 + C L1) x + a^2 MLP(x / a, C, log a),  a = |x|,
 * MLP 768 -> 1024 -> 1024 -> 768, GELU, bf16 weights, FP32 accumulation,
 * trained by the library's own kernels on the O(a^2) remainder.
 * When cfg->surrogate is set and a trained network and trust limits are
 * present, sg_step and sg_membrane_force use it for every degree-15 capsule
 * that passes the residual check (|x| <= amp_max, |MLP(x)| <= ratio_max
 * |(L0 + C L1) x|, c_min <= C <= c_max); the others, and all capsules of
 * other degrees, take the plain model. */
long sg_surrogate_param_count(void);
/* set != 0: load parameters from buf (marks the network trained); set == 0:
 * copy them out.  Order: W1, b1, W2, b2, W3, b3, L0, L1, mu_x, sd_x, mu_y, sd_y. */
int sg_surrogate_params(sg_ctx* ctx, int set, float* buf, long n);
/* The linear response about the sphere, [768][768] each, row = output slot. */
int sg_surrogate_set_linear(sg_ctx* ctx, const float* L0, const float* L1);
/* Train on n host rows X [n][768], Y [n][768] (dimensionless as above):
 * residual targets (Y - (L0 + C L1) X) / a^2, normalisation from the data, Adam with
 * cosine decay, minibatches of `batch` (a multiple of 64, <= 1024) in seeded
 * random order; loss_hist[epochs] receives the mean training loss per epoch. */
int sg_surrogate_train(sg_ctx* ctx, const float* X, const float* Y, long n, int epochs, int batch,
                       float lr, unsigned long long seed, float* loss_hist);
/* Predict Y [n][768] for host rows X; parts: 1 linear only, 2 MLP only, 3 both. */
int sg_surrogate_predict(sg_ctx* ctx, const float* X, long n, int parts, float* Y);
/* Residual-check limits; amp_max = 0 turns the surrogate off. */
int sg_surrogate_set_trust(sg_ctx* ctx, float amp_max, float ratio_max, float c_min, float c_max);
/* Capsules that used the surrogate and that fell back, in the last step. */
int sg_surrogate_last_counts(sg_ctx* ctx, int* n_surrogate, int* n_fallback);

/* Host-side tables (tests): Gauss colatitudes and SPHEREPACK-normalised
 * Legendre functions with theta derivatives, [m*nn+n] layout. */
int sg_gauss(int nlat, double* theta, double* weights);
int sg_legendre(double theta, int mm, int nn, double* P, double* dP, double* d2P);

/* Number of this library's kernels launched by the last step call. */
int sg_last_launch_count(const sg_ctx* ctx);

/* Spreading tile shape (no counterpart in the reference, whose spreading loops
 * over points, interp_spread.f90:817-884).  shape indexes the cell tiles
 * 0: 32x8x4, 1: 16x16x8, 2: 32x8x8, 3: 8x8x4, 4: whole x rows x 4 x 4,
 * 5: whole x rows x 8 x 4, 6: 32x16x4, or -1 for the grid's default; FP64 contexts take
 * shapes 0 and 3 only, and the row tiles need 12 (itot TY TZ + 32) bytes of
 * shared memory, at most 200 KiB.  Results do not depend on the shape beyond
 * rounding of the per-tile fixed-point scale.  Not allowed while a graph is
 * captured.  sg_get_tile_shape reports a row tile's TX as itot. */
int sg_set_tile_shape(sg_ctx* ctx, int shape);
int sg_get_tile_shape(const sg_ctx* ctx, int* shape, int* tx, int* ty, int* tz);

/* Mixed precision only: split mode of the tensor-core Legendre contractions.
 * terms = 3 (BF16x3: A0B0 + A0B1 + A1B0, about 16 significant bits per
 * product), 6 (BF16x6: + A0B2 + A2B0 + A1B1, FP32-level products) or 0
 * (automatic, the default: BF16x6 for capsules of SH degree >= 16, whose
 * force error under BF16x3 approaches 1e-4, BF16x3 below).  Returns
 * SG_ERR_STATE while a graph is captured. */
int sg_set_legendre_terms(sg_ctx* ctx, int terms);
/* The split products (3 or 6) a capsule of this SH degree runs with. */
int sg_get_legendre_terms(sg_ctx* ctx, int degree);

/* Mixed precision only: data rows per tile of the tensor-core Legendre
 * contractions, 128 (the default; M = 128 products) or 64 (M = 64: twice the
 * work items, for launches with few tiles).  sg_autotune times both.
 * Results do not depend on it.  SG_ERR_STATE while a graph is captured. */
int sg_set_legendre_tile_rows(sg_ctx* ctx, int rows);
int sg_get_legendre_tile_rows(sg_ctx* ctx);

/* Mixed precision only: run the Legendre contractions on the tensor cores in
 * BF16x3 (on = 1, the default) or on the CUDA cores in FP32 (on = 0), for
 * comparisons of the two. */
int sg_set_tensor_cores(sg_ctx* ctx, int on);

/* Schedule of the persistent per-capsule kernels (no counterpart in the
 * reference): every capsule is cut into `split` row ranges, 1 <= split <= 8,
 * so that few capsules still fill every SM.  Results do not depend on it. */
int sg_set_point_split(sg_ctx* ctx, int split);
int sg_get_point_split(const sg_ctx* ctx);

/* Autotuner: times `reps` sg_step calls with the same arguments for every
 * tile shape valid for the context, then for every point split (1, 2, 4, 8)
 * with the best shape, then (mixed precision) for both tensor-core Legendre
 * tile heights; keeps the fastest choices and returns the shape with the
 * best milliseconds per step.  The outputs hold the last step's results. */
int sg_autotune(sg_ctx* ctx, const void* u, const void* v, const void* w,
                const double* X, const double* Y, const double* Z,
                void* U, void* V, void* W,
                void* FX, void* FY, void* FZ, void* NX, void* NY, void* NZ, void* AREA,
                void* fx, void* fy, void* fz, int reps, int* best_shape, float* best_ms);

/* CUDA graph of one sg_step on fixed device arrays (SG_MEM_DEVICE only): the
 * capture records every launch of the step on the context stream; each
 * sg_graph_launch replays it (same pointers, current array contents).
 * sg_graph_release drops the graph.  The stream must not be the legacy
 * default stream. */
int sg_graph_capture(sg_ctx* ctx, const void* u, const void* v, const void* w,
                     const double* X, const double* Y, const double* Z,
                     void* U, void* V, void* W,
                     void* FX, void* FY, void* FZ, void* NX, void* NY, void* NZ, void* AREA,
                     void* fx, void* fy, void* fz);
int sg_graph_launch(sg_ctx* ctx);
int sg_graph_release(sg_ctx* ctx);

/* Stage timing with CUDA events on the context stream.  When enabled, each
 * step call records events around its stages (and runs them on one stream);
 * sg_stage_times returns the last step's milliseconds for SG_STAGE_* (bin,
 * interp, membrane, spread) and, as SG_STAGE_CONTRACT, the summed time of the
 * Legendre contraction launches inside the membrane stage (tensor-core
 * launches in mixed precision, CUDA-core launches in FP64). */
#define SG_STAGE_BIN 0
#define SG_STAGE_INTERP 1
#define SG_STAGE_MEMBRANE 2
#define SG_STAGE_SPREAD 3
#define SG_STAGE_CONTRACT 4
#define SG_NSTAGE 5
int sg_set_profiling(sg_ctx* ctx, int on);
int sg_stage_times(sg_ctx* ctx, float* ms, int n);

/* Work of one step's Legendre contractions (no counterpart in the reference):
 * out[0] = algorithmic flops (2 x the multiply-adds of the transforms, with
 * the products the triangular structure makes zero left out: synthesis terms
 * of degree n < m and analysis outputs of degree n < m), out[1] = flops the
 * tensor cores issue (padded tiles times the split products; 0 on the CUDA-core
 * path), out[2] = contraction launches per step. */
int sg_contraction_work(const sg_ctx* ctx, double* out);

#ifdef __cplusplus
}
#endif
#endif
