// sg_flow.cu -- the prescribed velocity of the time-stepped benchmark
// (include/sg_workload.h): a synthetic input, not part of the coupling step.
//
// Two kernels.  The first evaluates the horizontal factor of each component,
//   F_c[j][i] = sum_q amp[q][c] cos(kx_q x_c(i) + ky_q y_c(j) + phase_q + omega_q t),
// once per (c, j, i) in FP64 (3 (jtot+2)(itot+2) values, a few MB that stay in
// L2).  The second writes the three fields: a block owns one j row and a run
// of k planes, keeps that row of F in registers and streams
//   u_c[k][j][i] = sin(pi z_c(k) / Lz) F_c[j][i] (+ shear z_c(k) for u)
// to memory, coalesced along i and rounded once to the output type, so the
// fields cost one write pass.
#include <cmath>

#include "sg_coupling.h"
#include "sg_workload.h"

namespace {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr int kThreads = 256;
constexpr int kPlanes = 32;    // k planes per block of the write kernel
constexpr int kPerThread = 4;  // i values per thread (rows of up to 1024 cells in registers)

struct FlowModes {
  int n;
  double kx[SG_FLOW_MAX_MODES], ky[SG_FLOW_MAX_MODES], phase[SG_FLOW_MAX_MODES], omega[SG_FLOW_MAX_MODES];
  double amp[SG_FLOW_MAX_MODES][3];
};

struct FlowGrid {
  int ldi, ldj, ldk;
  double dx, dy, dz, Lz, shear;
};

// face location i * d along the component's own direction, centre (i - 1/2) d otherwise
__device__ __forceinline__ double loc(int i, double d, bool face) { return face ? i * d : (i - 0.5) * d; }

__global__ void flow_factor_kernel(FlowGrid g, FlowModes m, const double* __restrict__ t, double* __restrict__ F) {
  const long n = (long)g.ldi * g.ldj;
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (p >= n) return;
  const int i = (int)(p % g.ldi), j = (int)(p / g.ldi);
  const double x = loc(i, g.dx, c == 0), y = loc(j, g.dy, c == 1), tt = *t;
  double s = 0.0;
  for (int q = 0; q < m.n; ++q) s += m.amp[q][c] * cos(m.kx[q] * x + m.ky[q] * y + (m.phase[q] + m.omega[q] * tt));
  F[(long)c * n + p] = s;
}

template <class T>
__global__ void __launch_bounds__(kThreads) flow_write_kernel(FlowGrid g, const double* __restrict__ F,
                                                              T* __restrict__ u, T* __restrict__ v,
                                                              T* __restrict__ w) {
  const int j = blockIdx.x, k0 = blockIdx.y * kPlanes;
  const long plane = (long)g.ldi * g.ldj;
  double f[3][kPerThread];
#pragma unroll
  for (int r = 0; r < kPerThread; ++r) {
    const int i = threadIdx.x + kThreads * r;
#pragma unroll
    for (int c = 0; c < 3; ++c) f[c][r] = i < g.ldi ? F[c * plane + (long)j * g.ldi + i] : 0.0;
  }
  const int k1 = min(k0 + kPlanes, g.ldk);
  for (int k = k0; k < k1; ++k) {
    // z of the centres (u, v) and of the faces (w)
    const double zc = (k - 0.5) * g.dz, zf = k * g.dz;
    const double sc = sin(kPi * zc / g.Lz), sf = sin(kPi * zf / g.Lz), sh = g.shear * zc;
    const long row = k * plane + (long)j * g.ldi;
#pragma unroll
    for (int r = 0; r < kPerThread; ++r) {
      const int i = threadIdx.x + kThreads * r;
      if (i < g.ldi) {
        u[row + i] = (T)(sc * f[0][r] + sh);
        v[row + i] = (T)(sc * f[1][r]);
        w[row + i] = (T)(sf * f[2][r]);
      }
    }
  }
}

}  // namespace

extern "C" int sg_prescribed_flow(int itot, int jtot, int ktot, double dx, double dy, double dz, int nmodes,
                                  const double* nx, const double* ny, const double* phase, const double* amp,
                                  const double* omega, double shear, const double* t, int fp32, void* u, void* v,
                                  void* w, void* work, void* stream) {
  if (itot < 1 || jtot < 1 || ktot < 1 || !(dx > 0 && dy > 0 && dz > 0)) return SG_ERR_ARG;
  if (itot + 2 > kThreads * kPerThread) return SG_ERR_ARG;
  if (nmodes < 0 || nmodes > SG_FLOW_MAX_MODES) return SG_ERR_ARG;
  if (nmodes > 0 && (!nx || !ny || !phase || !amp || !omega)) return SG_ERR_ARG;
  if (!t || !u || !v || !w || !work) return SG_ERR_ARG;
  FlowGrid g{itot + 2, jtot + 2, ktot + 2, dx, dy, dz, ktot * dz, shear};
  const double Lx = itot * dx, Ly = jtot * dy;
  FlowModes m{};
  m.n = nmodes;
  for (int q = 0; q < nmodes; ++q) {
    m.kx[q] = 2.0 * kPi * nx[q] / Lx;
    m.ky[q] = 2.0 * kPi * ny[q] / Ly;
    m.phase[q] = phase[q];
    m.omega[q] = omega[q];
    for (int c = 0; c < 3; ++c) m.amp[q][c] = amp[3 * q + c];
  }
  cudaStream_t st = (cudaStream_t)stream;
  double* F = (double*)work;
  const long n = (long)g.ldi * g.ldj;
  flow_factor_kernel<<<dim3((unsigned)((n + kThreads - 1) / kThreads), 3), kThreads, 0, st>>>(g, m, t, F);
  const dim3 grid((unsigned)g.ldj, (unsigned)((g.ldk + kPlanes - 1) / kPlanes));
  if (fp32)
    flow_write_kernel<float><<<grid, kThreads, 0, st>>>(g, F, (float*)u, (float*)v, (float*)w);
  else
    flow_write_kernel<double><<<grid, kThreads, 0, st>>>(g, F, (double*)u, (double*)v, (double*)w);
  return cudaGetLastError() == cudaSuccess ? SG_OK : SG_ERR_CUDA;
}
