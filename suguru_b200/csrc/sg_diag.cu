// sg_diag.cu -- position update and capsule diagnostics.
//
// Update_Pos.f90:95-180: forward-Euler advection of the force points with the
// interpolated velocity, the wall clamp z in [0, lz], and the periodic shift
// of a capsule whose centroid has left the box.  The master/slave migration
// of Update_Pos.f90:58-72 has no counterpart on one GPU.
// surf_vol.f90:12-131: centroid, volume by the 1000-layer radial quadrature,
// inertia tensor -> Taylor deformation exy1, exy2; all in FP64.
#include "sg_common.cuh"
#include "sg_kernels.h"

namespace sg {

// One block per capsule: advection and wall clamp of every point
// (Update_Pos.f90:95-99, 118-126), then the capsule's centroid and, when it
// has left the periodic box in x or y, the shift of all its points by one
// period (Update_Pos.f90:131-180; the reference's centroid is a sequential
// sum, this one a fixed tree in FP64, so the two agree unless the centroid
// lies within rounding of a box face).
template <class T>
__global__ void __launch_bounds__(256) update_pos_kernel(const CapInfo* __restrict__ caps, double dt, double lx,
                                                         double ly, double lz, double* __restrict__ X,
                                                         double* __restrict__ Y, double* __restrict__ Z,
                                                         const T* __restrict__ U, const T* __restrict__ V,
                                                         const T* __restrict__ W) {
  __shared__ double s_sum[2][8];
  const CapInfo ci = caps[blockIdx.x];
  const long long p0 = ci.pt_off, nl = 8LL * (ci.L + 1) * (ci.L + 1);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double sx = 0.0, sy = 0.0;
  for (long long l = tid; l < nl; l += 256) {
    const long long p = p0 + l;
    // x + (u dt) with two roundings, as the reference's expression (no fused multiply-add)
    const double x = __dadd_rn(X[p], __dmul_rn((double)U[p], dt));
    const double y = __dadd_rn(Y[p], __dmul_rn((double)V[p], dt));
    double z = __dadd_rn(Z[p], __dmul_rn((double)W[p], dt));
    if (z < 0.) z = 0.;
    else if (z > lz) z = lz;
    X[p] = x;
    Y[p] = y;
    Z[p] = z;
    sx += x;
    sy += y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
  }
  if (lane == 0) {
    s_sum[0][warp] = sx;
    s_sum[1][warp] = sy;
  }
  __syncthreads();
  sx = sy = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    sx += s_sum[0][q];
    sy += s_sum[1][q];
  }
  const double xm = sx / (double)nl, ym = sy / (double)nl;
  const double shx = xm > lx ? -lx : (xm < 0. ? lx : 0.);
  const double shy = ym > ly ? -ly : (ym < 0. ? ly : 0.);
  if (shx == 0. && shy == 0.) return;  // uniform across the block
  for (long long l = tid; l < nl; l += 256) {
    const long long p = p0 + l;
    if (shx != 0.) X[p] = X[p] + shx;
    if (shy != 0.) Y[p] = Y[p] + shy;
  }
}

// collisions.f90:10-32: the Morse-potential force of the wall z = 0 on every
// point closer than rad0, summed over the wall's lattice images
// (j dy, k dx) within the cutoff, added to fz.  Evaluated in FP64 in the
// reference's operation order (including its k dx spacing under a bound taken
// from dy, and |z / ss|, which is 0/0 for a point exactly on the wall); the
// sum is added to FZ with one rounding.
template <class T>
__global__ void collisions_kernel(long n, WallParams wp, const double* __restrict__ Z, const T* __restrict__ A,
                                  T* __restrict__ FZ, ForceRec<T>* __restrict__ frc, double dvi) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double z = Z[p], a = (double)A[p], dx2 = wp.dx * wp.dx;
  const long jm = lround(sqrt(fmax(wp.rad0 * wp.rad0 - z * z, 0.)) * (1.0 / wp.dy));
  if (jm == 0 && !(fabs(z) < wp.rad0)) return;  // no lattice image within the cutoff: fc = 0
  const double amp = 2. * (wp.col / (wp.rep * wp.rep));
  const double ratio = fmin(a, dx2) / fmax(a, dx2);
  double fc = 0.;
  for (long j = -jm; j <= jm; ++j)
    for (long k = -jm; k <= jm; ++k) {
      const double ss = sqrt(z * z + (j * wp.dy) * (j * wp.dy) + (k * wp.dx) * (k * wp.dx));
      if (ss < wp.rad0)
        fc += amp * (exp(2. * wp.betacol * (wp.rad0 - ss)) - exp(wp.betacol * (wp.rad0 - ss))) * fabs(z / ss) * ratio;
    }
  const T fz = (T)((double)FZ[p] + fc);
  FZ[p] = fz;
  if (frc) frc[p].cf[2] = fz * (A[p] * (T)dvi);
}

// One block per capsule; deterministic tree reductions in FP64.
template <class T>
__global__ void __launch_bounds__(256) surf_vol_kernel(const CapInfo* __restrict__ caps, const double* __restrict__ X,
                                                       const double* __restrict__ Y, const double* __restrict__ Z,
                                                       const T* __restrict__ NX, const T* __restrict__ NY,
                                                       const T* __restrict__ NZ, const T* __restrict__ AREA,
                                                       const double* __restrict__ exy1_prev, double S2, double S22,
                                                       double* __restrict__ out) {
  __shared__ double s[11][256];
  const int c = blockIdx.x, t = threadIdx.x;
  const CapInfo ci = caps[c];
  const long long n = 8LL * ci.N * ci.N, o = ci.pt_off;
  double sx = 0, sy = 0, sz = 0;
  for (long long p = t; p < n; p += 256) {
    sx += X[o + p];
    sy += Y[o + p];
    sz += Z[o + p];
  }
  s[0][t] = sx;
  s[1][t] = sy;
  s[2][t] = sz;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (t < h)
      for (int q = 0; q < 3; ++q) s[q][t] += s[q][t + h];
    __syncthreads();
  }
  const double xm = s[0][0] / n, ym = s[1][0] / n, zm = s[2][0] / n;
  __syncthreads();
  double vol = 0, ixx = 0, ixy = 0, ixz = 0, iyy = 0, iyz = 0, izz = 0, at = 0, rmax = -1.0, rmin = 1e300;
  for (long long p = t; p < n; p += 256) {
    const double dx = X[o + p] - xm, dy = Y[o + p] - ym, dz = Z[o + p] - zm;
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    const double cs = (dx * (double)NX[o + p] + dy * (double)NY[o + p] + dz * (double)NZ[o + p]) / r;
    const double base = (double)AREA[o + p] * (r / 1000.) * fabs(cs);
    vol += base * S2;
    ixx += base * S22 * (dy * dy + dz * dz);
    ixy -= base * S22 * (dx * dy);
    ixz -= base * S22 * (dx * dz);
    iyy += base * S22 * (dx * dx + dz * dz);
    iyz -= base * S22 * (dy * dz);
    izz += base * S22 * (dx * dx + dy * dy);
    at += (double)AREA[o + p];
    rmax = fmax(rmax, r);
    rmin = fmin(rmin, r);
  }
  s[0][t] = vol; s[1][t] = ixx; s[2][t] = ixy; s[3][t] = ixz; s[4][t] = iyy; s[5][t] = iyz;
  s[6][t] = izz; s[7][t] = at; s[8][t] = rmax; s[9][t] = rmin;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (t < h) {
      for (int q = 0; q < 8; ++q) s[q][t] += s[q][t + h];
      s[8][t] = fmax(s[8][t], s[8][t + h]);
      s[9][t] = fmin(s[9][t], s[9][t + h]);
    }
    __syncthreads();
  }
  if (t != 0) return;
  vol = s[0][0]; ixx = s[1][0]; ixy = s[2][0]; ixz = s[3][0]; iyy = s[4][0]; iyz = s[5][0]; izz = s[6][0];
  at = s[7][0]; rmax = s[8][0]; rmin = s[9][0];
  const double pi = 3.14159265358979323846;
  const double i1 = ixx + iyy + izz;
  const double i2 = ixx * iyy + iyy * izz + ixx * izz - ixy * ixy - iyz * iyz - ixz * ixz;
  const double i3 = ixx * iyy * izz - ixx * iyz * iyz - iyy * ixz * ixz - izz * ixy * ixy + 2. * ixy * ixz * iyz;
  const double r = (2. * i1 * i1 * i1 - 9. * i1 * i2 + 27. * i3) / 54.;
  const double q = (3. * i2 - i1 * i1) / 9.;
  const double teta = acos(r / sqrt(-(q * q * q)));
  const double ip1 = i1 / 3. + 2. * sqrt(-q) * cos(teta / 3.);
  const double ip2 = i1 / 3. + 2. * sqrt(-q) * cos((teta + 2. * pi) / 3.);
  const double ip3 = i1 / 3. + 2. * sqrt(-q) * cos((teta + 4. * pi) / 3.);
  const double mass = (4. / 3.) * pi;
  const double ic1 = ip1 / (mass / 5.), ic2 = ip2 / (mass / 5.), ic3 = ip3 / (mass / 5.);
  const double lp2 = sqrt(.5 * (ic1 + ic3 - ic2));
  const double lp1 = sqrt(ic3 - lp2 * lp2);
  const double lp3 = sqrt(ic1 - lp2 * lp2);
  double exy1 = exy1_prev ? exy1_prev[c] : 0.0;
  if (fabs(ip1 - ixx) < 0.0001) exy1 = fabs(lp2 - lp3) / (lp2 + lp3);
  else if (fabs(ip2 - ixx) < 0.0001) exy1 = fabs(lp1 - lp3) / (lp1 + lp3);
  else if (fabs(ip3 - ixx) < 0.0001) exy1 = fabs(lp1 - lp2) / (lp1 + lp2);
  double* oc = out + 7 * c;
  oc[0] = vol;
  oc[1] = at;
  oc[2] = exy1;
  oc[3] = fabs(rmax - rmin) / (rmax + rmin);
  oc[4] = xm;
  oc[5] = ym;
  oc[6] = zm;
}

template <class T>
cudaError_t launch_update_pos(int ncap, const CapInfo* caps, double dt, double lx, double ly, double lz, double* X,
                              double* Y, double* Z, const T* U, const T* V, const T* W, cudaStream_t st) {
  if (ncap <= 0) return cudaSuccess;
  update_pos_kernel<T><<<ncap, 256, 0, st>>>(caps, dt, lx, ly, lz, X, Y, Z, U, V, W);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_collisions(long n, const WallParams& wp, const double* Z, const T* A, T* FZ, void* frc, double dvi,
                              cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  collisions_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, wp, Z, A, FZ, (ForceRec<T>*)frc, dvi);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_surf_vol(int ncap, const CapInfo* caps, const double* X, const double* Y, const double* Z,
                            const T* NX, const T* NY, const T* NZ, const T* AREA, const double* exy1_prev,
                            double* out, cudaStream_t st) {
  if (ncap <= 0) return cudaSuccess;
  // radial layer sums of surf_vol.f90:77-96: sum ma^2 and sum ma^2 na^2
  double S2 = 0, S22 = 0;
  for (int l = 1; l <= 1000; ++l) {
    double ma = (l - 1) / 1000., na = (l - .5) / 1000.;
    S2 += ma * ma;
    S22 += ma * ma * na * na;
  }
  surf_vol_kernel<T><<<ncap, 256, 0, st>>>(caps, X, Y, Z, NX, NY, NZ, AREA, exy1_prev, S2, S22, out);
  return cudaGetLastError();
}

template cudaError_t launch_update_pos<double>(int, const CapInfo*, double, double, double, double, double*,
                                               double*, double*, const double*, const double*, const double*,
                                               cudaStream_t);
template cudaError_t launch_update_pos<float>(int, const CapInfo*, double, double, double, double, double*, double*,
                                              double*, const float*, const float*, const float*, cudaStream_t);
template cudaError_t launch_collisions<double>(long, const WallParams&, const double*, const double*, double*, void*,
                                                double, cudaStream_t);
template cudaError_t launch_collisions<float>(long, const WallParams&, const double*, const float*, float*, void*,
                                               double, cudaStream_t);
template cudaError_t launch_surf_vol<double>(int, const CapInfo*, const double*, const double*, const double*,
                                             const double*, const double*, const double*, const double*,
                                             const double*, double*, cudaStream_t);
template cudaError_t launch_surf_vol<float>(int, const CapInfo*, const double*, const double*, const double*,
                                            const float*, const float*, const float*, const float*, const double*,
                                            double*, cudaStream_t);

}  // namespace sg
