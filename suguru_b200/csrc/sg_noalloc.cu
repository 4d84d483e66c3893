// sg_noalloc.cu -- the spreading step (lagr2eulr) for callers that cannot
// allocate device memory.
//
// Who needs this: a host code that hands every byte of device memory to its
// own pool or budget (the Fortran solver that owns forcex/y/z and the point
// arrays), code running where cudaMalloc is forbidden or would stall (inside
// an allocator callback, a real-time loop with no allocation allowed, a
// library that may not create a context-wide heap), or a caller that simply
// must not create the sg_ctx of sg_create, which allocates its workspace.
// Such a caller passes its own input and output arrays; the binning scratch
// this step needs instead lives in one fixed array compiled into the library.
//
// The scratch array is a file-scope __device__ variable: every GPU that loads
// the library holds it (SG_NOALLOC_SCRATCH_BYTES, about 7.3 MB) until the
// process exits.  All calls share it, so calls that overlap on the GPU (two
// streams, two host threads, or a call still running when the next one is
// queued on another stream) race on it; the previous call's contents remain
// in it, and this file clears what must start at zero (the tile counters) on
// every call.
#include <mutex>

#include "sg_coupling.h"
#include "sg_kernels.h"

using namespace sg;

namespace {

constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// scratch layout: per point position and force records, per tile counters,
// entry lists
constexpr size_t kPos = align256(sizeof(PosRec<double>) * SG_NOALLOC_MAX_POINTS);
constexpr size_t kFrc = align256(sizeof(ForceRec<double>) * SG_NOALLOC_MAX_POINTS);
constexpr size_t kTile = align256(sizeof(int) * (SG_NOALLOC_MAX_TILES + 1));
constexpr size_t kEntr = align256(sizeof(int) * 8 * SG_NOALLOC_MAX_POINTS);
constexpr size_t kScratch = kPos + kFrc + 3 * kTile + kEntr;
static_assert(kScratch <= SG_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the stated size");

}  // namespace

// Host code may not use this name as a device address: outside device code it
// is a host-side stand-in.  The device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_spread_scratch[SG_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_dev_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device (the first call on a device does this; make that first call
// outside any stream capture).
cudaError_t scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_dev_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_spread_scratch);
    if (e != cudaSuccess) return e;
    g_dev_ptr[dev] = p;
  }
  *out = g_dev_ptr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int sg_spread_noalloc(int itot, int jtot, int ktot, double lx, double ly, double lz, long npts,
                                 const double* X, const double* Y, const double* Z, const double* FX,
                                 const double* FY, const double* FZ, const double* AREA, double* fx, double* fy,
                                 double* fz, void* stream) {
  if (npts < 0 || !fx || !fy || !fz) return SG_ERR_ARG;
  if (npts > 0 && (!X || !Y || !Z || !FX || !FY || !FZ || !AREA)) return SG_ERR_ARG;
  if (!(lx > 0 && ly > 0 && lz > 0)) return SG_ERR_ARG;
  IBGrid g{};
  if (!make_ib_grid(itot, jtot, ktot, lx, ly, lz, g, -1, kFp64TileShapes)) return SG_ERR_ARG;
  if (npts > SG_NOALLOC_MAX_POINTS || g.ntiles > SG_NOALLOC_MAX_TILES) return SG_ERR_TOO_LARGE;
  void* base = nullptr;
  if (scratch_address(&base) != cudaSuccess) return SG_ERR_CUDA;
  unsigned char* s = (unsigned char*)base;
  IBWork w{};
  w.pos = s; s += kPos;
  w.frc = s; s += kFrc;
  w.counts = (int*)s; s += kTile;  // zeroed by launch_bin on every call
  w.starts = (int*)s; s += kTile;
  w.fill = (int*)s; s += kTile;    // zeroed by the scan on every call
  w.entries = (int*)s;
  cudaStream_t st = (cudaStream_t)stream;
  if (launch_bin<double>(g, npts, X, Y, Z, w, st) != cudaSuccess) return SG_ERR_CUDA;
  if (launch_pack_forces<double>(g, npts, FX, FY, FZ, AREA, w, st) != cudaSuccess) return SG_ERR_CUDA;
  if (launch_spread<double>(g, w, fx, fy, fz, st) != cudaSuccess) return SG_ERR_CUDA;
  return SG_OK;
}
