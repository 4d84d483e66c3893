// sg_overlap.cu -- the overlap mesh's lid values: interpolation
// (interpolation.f90:10-69), the bilinear interpolation of the main mesh's
// u, v, w, p and indicator at the plane between z cells nf and nf + 1 onto
// the nodes (i, j), 0 <= i <= itot nr + 1, 0 <= j <= jtot nr + 1, of the
// finer mesh near the bottom wall (ifoverlap = 1, param.f90:32-41; one GPU,
// so the reference's per-rank extents i1c, j1c are the whole mesh's).
//
// Node (i, j) sits at xp = i dxc + (1/2)(1 - 1/nr) dx, yp likewise; its main
// mesh cell is (im, jm) = (floor(xp/dx), floor(yp/dy)) and its weights are the
// reference's four area fractions.  u, v, p and the indicator are the mean of
// planes nf and nf + 1, w the value at nf + 1 (its face).  The arithmetic is
// the reference's, operation for operation and without fused multiply-adds,
// so the lid is bitwise the oracle's.
#include <cmath>

#include "sg_kernels.h"

namespace sg {
namespace {

__global__ void overlap_lid_kernel(LidArgs a) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long)a.ni * a.nj) return;
  const int i = (int)(q % a.ni), j = (int)(q / a.ni);
  const double xp = __dadd_rn(__dmul_rn((double)i, a.dxc), a.offx);
  const double yp = __dadd_rn(__dmul_rn((double)j, a.dyc), a.offy);
  const double fx = floor(__ddiv_rn(xp, a.dx)), fy = floor(__ddiv_rn(yp, a.dy));
  const double x1 = __dmul_rn(fx, a.dx), x2 = __dmul_rn(__dadd_rn(fx, 1.0), a.dx);
  const double y1 = __dmul_rn(fy, a.dy), y2 = __dmul_rn(__dadd_rn(fy, 1.0), a.dy);
  const double den = __dmul_rn(__dsub_rn(x2, x1), __dsub_rn(y2, y1));
  const double c11 = __ddiv_rn(__dmul_rn(__dsub_rn(x2, xp), __dsub_rn(y2, yp)), den);
  const double c12 = __ddiv_rn(__dmul_rn(__dsub_rn(x2, xp), __dsub_rn(yp, y1)), den);
  const double c21 = __ddiv_rn(__dmul_rn(__dsub_rn(xp, x1), __dsub_rn(y2, yp)), den);
  const double c22 = __ddiv_rn(__dmul_rn(__dsub_rn(xp, x1), __dsub_rn(yp, y1)), den);
  const long im = (long)fx, jm = (long)fy;
  const long s11 = jm * a.ldi + im, s12 = (jm + 1) * a.ldi + im, s21 = jm * a.ldi + im + 1,
             s22 = (jm + 1) * a.ldi + im + 1;
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    const double* lo = a.f[f];
    const double* hi = a.f[f] + a.plane;
    double q11, q12, q21, q22;
    if (f == 2) {  // w: its value at the face nf + 1
      q11 = hi[s11];
      q12 = hi[s12];
      q21 = hi[s21];
      q22 = hi[s22];
    } else {
      q11 = __dmul_rn(0.5, __dadd_rn(lo[s11], hi[s11]));
      q12 = __dmul_rn(0.5, __dadd_rn(lo[s12], hi[s12]));
      q21 = __dmul_rn(0.5, __dadd_rn(lo[s21], hi[s21]));
      q22 = __dmul_rn(0.5, __dadd_rn(lo[s22], hi[s22]));
    }
    a.o[f][q] = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(c11, q11), __dmul_rn(c12, q12)), __dmul_rn(c21, q21)),
                          __dmul_rn(c22, q22));
  }
}

}  // namespace

cudaError_t launch_overlap_lid(const LidArgs& a, cudaStream_t st) {
  const long n = (long)a.ni * a.nj;
  if (n <= 0) return cudaSuccess;
  overlap_lid_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace sg
