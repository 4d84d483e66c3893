// sg_common.cuh -- shared device helpers for the B200 coupling-step library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define SG_HD __host__ __device__ __forceinline__

namespace sg {

// Roma-Peskin 3-point regularised delta, multiplied by the grid spacing
// (kernel.f90:7-25).  Same expression shape as the reference.
template <class T>
SG_HD T delta3(T r) {
  T ar = r < T(0) ? -r : r;
  if (ar > T(1.5)) return T(0);
  if (ar > T(0.5))
    return (T(1) / T(6)) * (T(5) - T(3) * ar - sqrt(-T(3) * ((T(1) - ar) * (T(1) - ar)) + T(1)));
  return (T(1) / T(3)) * (T(1) + sqrt(-T(3) * (r * r) + T(1)));
}

// The three nonzero values of delta3 around the nearest node, with one square
// root.  For a node at offset o from the base index and a point at fraction f
// in [0,1): faces sit at o, cell centres at o - 1/2.  With r = (nearest node)
// - f, |r| <= 1/2 and s = sqrt(1 - 3 r^2), kernel.f90:7-25 gives
//   phi(r) = (1 + s)/3,  phi(r - 1) = (2 + 3r - s)/6,  phi(r + 1) = (2 - 3r - s)/6.
// face: w[t] is the weight of node o = hi - 1 + t, hi = (f >= 1/2);
// centre: w[t] is the weight of the centre at o = t.
template <class T>
SG_HD void delta3_face(T f, T* w, bool& hi) {
  hi = !(f < T(0.5));
  const T r = (hi ? T(1) : T(0)) - f;
  const T s = sqrt(T(1) - T(3) * r * r);
  w[0] = (T(2) + T(3) * r - s) * (T(1) / T(6));
  w[1] = (T(1) + s) * (T(1) / T(3));
  w[2] = (T(2) - T(3) * r - s) * (T(1) / T(6));
}
template <class T>
SG_HD void delta3_centre(T f, T* w) {
  const T r = T(0.5) - f;
  const T s = sqrt(T(1) - T(3) * r * r);
  w[0] = (T(2) + T(3) * r - s) * (T(1) / T(6));
  w[1] = (T(1) + s) * (T(1) / T(3));
  w[2] = (T(2) - T(3) * r - s) * (T(1) / T(6));
}

SG_HD int wrap_near(int r, int n) { return r < 1 ? r + n : (r > n ? r - n : r); }

SG_HD int wrap1(int i, int n) {  // periodic storage index in [1, n]
  int r = (i - 1) % n;
  if (r < 0) r += n;
  return r + 1;
}

SG_HD long long fidx(int i, int j, int k, int ldi, int ldj) {
  return (long long)i + (long long)ldi * ((long long)j + (long long)ldj * (long long)k);
}

template <class T>
struct V3 {
  T x, y, z;
};

template <class T>
SG_HD void cross3(const T* u, const T* v, T* w) {
  w[0] = u[1] * v[2] - u[2] * v[1];
  w[1] = u[2] * v[0] - u[0] * v[2];
  w[2] = u[0] * v[1] - u[1] * v[0];
}
template <class T>
SG_HD T dot3(const T* u, const T* v) {
  return u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
}

#if defined(__CUDACC__)
// Lets a kernel take up to the device's opt-in limit of dynamic shared memory
// (less its static shared memory).  Every launcher sets this one value
// instead of its own request: a kernel launched with different requests
// (the Legendre stages, contexts of different degrees) would otherwise carry
// whatever its last launcher set, and a launch outside that launcher's
// sequence -- a CUDA graph node replayed on its own, as a profiler does --
// could ask for more than that limit and fail to launch.  The launch's own
// request still sets its occupancy.
template <class K>
inline cudaError_t smem_limit_max(K kernel) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa{};
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kernel);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
  return e;
}

// Programmatic dependent launch.  The step's kernels follow one another on
// a stream; launched with launch_pdl, a kernel's grid may be set up while its
// predecessor is still running.  Each such kernel calls pdl_wait() before it
// reads anything an earlier kernel wrote (it returns once the predecessor has
// completed and its writes are visible), and pdl_launch_dependents() to let
// its own successor be set up: called by every CTA at its start, so the
// successor's CTAs come only after all of this grid's CTAs are resident or
// done.  In a kernel launched without the attribute both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_enter() {
  pdl_wait();
  pdl_launch_dependents();
}

template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Asynchronous copy of one 4- or 8-byte element from global to shared memory
// (cp.async, no register round trip): a staging loop issues all of its
// copies before any completes; stage_wait() waits for this thread's copies,
// and a barrier after it publishes them to the block.
template <class T>
__device__ __forceinline__ void stage_async(T* dst, const T* src) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "element size");
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void stage_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Bounded spin on a global flag; returns false on timeout (never traps).
__device__ __forceinline__ bool spin_until_ge(volatile int* flag, int target, long long max_iter) {
  for (long long it = 0; it < max_iter; ++it) {
    if (*flag >= target) return true;
    __nanosleep(64);
  }
  return false;
}
#endif

}  // namespace sg
