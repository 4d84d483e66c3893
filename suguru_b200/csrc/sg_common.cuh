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
// Raises a kernel's dynamic shared-memory limit to at least `bytes`, and
// never lowers it.  A kernel launched with different requests (the Legendre
// stages, contexts of different degrees) would otherwise keep whatever its
// last launcher set, and a launch outside that launcher's sequence -- a CUDA
// graph node replayed on its own, as a profiler does -- could ask for more
// than that and fail to launch.  The limit stays at the largest request
// made, not the device maximum, which could otherwise steer the shared
// memory / L1 split of the SMs that other kernels share.
template <class K>
inline cudaError_t smem_limit(K kernel, size_t bytes) {
  cudaFuncAttributes fa{};
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess || (size_t)fa.maxDynamicSharedSizeBytes >= bytes) return e;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Programmatic dependent launch.  The step's kernels follow one another on
// a stream; launched with launch_pdl, a kernel's grid is set up while its
// predecessor is still running and starts as the predecessor's last CTAs
// retire.  Each such kernel calls pdl_enter() first: it returns once the
// predecessor has completed and its writes are visible.  The successor is
// released implicitly as each CTA exits -- not earlier, since CTAs of a
// successor that wait for their predecessor would hold SM slots that the
// kernels of the step's other stream need.  Without the launch attribute the
// wait is a no-op.
__device__ __forceinline__ void pdl_enter() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

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
