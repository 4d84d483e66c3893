// sg_kernels.h -- internal declarations shared by the .cu files of the library.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <vector>

#include "sg_ib.cuh"

namespace sg {

// ------------------------------------------------------------ IB transfer --
// Per point, written by the binning: base cell b[0..2] (b[3] unused) and the
// fractional offsets f[0..2] in cell units (f[3] unused).  A record is 16-byte
// aligned, so that the spread's gather of a point takes whole 16-byte loads
// from one or two sectors instead of six scattered words.
template <class T>
struct alignas(16) PosRec {
  int b[4];
  T f[4];
};
// Per point, for the spread: cf[c] = F_c * area / dV (c = 0..2); cf[3] pads
// the record to 16 (FP32) or 32 (FP64) bytes and is written as zero.
template <class T>
struct alignas(16) ForceRec {
  T cf[4];
};

struct IBWork {
  void* pos = nullptr;    // PosRec<T>[npts]
  void* frc = nullptr;    // ForceRec<T>[npts]
  int* counts = nullptr;  // [ntiles]
  int* starts = nullptr;  // [ntiles+1]
  int* fill = nullptr;    // [ntiles]
  int* entries = nullptr; // [8*npts] point index per (tile, point) pair
};

// shape: index into kTileShapes, or -1 for the default of the grid size.
// A shape whose last tile in x or y would have 1 or 2 cells is rejected (a
// stencil could then reach three tiles in that periodic dimension); shape -1
// takes the first shape that fits.  `allowed` is a bit mask of the shapes the
// caller's spread kernel has (kFp64TileShapes for FP64 spreading, whose
// shared accumulators hold at most 1024 cells); shapes outside it are never
// chosen, so a grid that no allowed shape fits is refused here, before any
// launch.
constexpr unsigned kAllTileShapes = 0x7Fu;
constexpr unsigned kFp64TileShapes = (1u << 0) | (1u << 3);
bool make_ib_grid(int itot, int jtot, int ktot, double lx, double ly, double lz, IBGrid& g, int shape = -1,
                  unsigned allowed = kAllTileShapes);
template <class T>
cudaError_t launch_bin(const IBGrid& g, long n, const double* X, const double* Y, const double* Z, IBWork& w,
                       cudaStream_t st);
template <class T>
cudaError_t launch_interp(const IBGrid& g, long n, const IBWork& w, const T* u, const T* v, const T* ww, T* U, T* V,
                          T* W, cudaStream_t st);
// Force records from caller arrays (the coupling step's final synthesis
// writes them itself): cf = F * (A / dV).
template <class T>
cudaError_t launch_pack_forces(const IBGrid& g, long n, const T* FX, const T* FY, const T* FZ, const T* A, IBWork& w,
                               cudaStream_t st);
// Spreads the force records of w.frc (points binned in w).
template <class T>
cudaError_t launch_spread(const IBGrid& g, const IBWork& w, T* ox, T* oy, T* oz, cudaStream_t st);
// The same with cell-centre weights in every direction for every component
// (lagr2eulrind); FP64 only, tile shapes 0 and 3.
template <class T>
cudaError_t launch_spread_centred(const IBGrid& g, const IBWork& w, T* ox, T* oy, T* oz, cudaStream_t st);

// ------------------------------------------------------------ host tables --
// Gauss-Legendre colatitudes north->south and weights (gaqd.f:45 semantics).
void host_gauss(int n, double* th, double* w);
// SPHEREPACK-normalised P, dP/dtheta, d2P/dtheta2 at one colatitude as
// [m*nn+n] for m<mm, n<nn (zero for n<m).
void host_legendre(double th, int mm, int nn, double* P, double* dP, double* d2P);
// The third and fourth theta derivatives, same layout.
void host_legendre_d34(double th, int mm, int nn, double* d3P, double* d4P);

// ---------------------------------------------------------- spectral stage --
// Per-degree constant data on the device (built from FP64 host tables).
struct DegreeTables {
  int L = 0, N = 0, nD = 0, mD = 0, nO = 0, mO = 0;
  // Legendre GEMM operands, K fastest: B[m][j][k]
  //  syn_D : j = kind*nD + i (kind 0:P 1:dP 2:d2P, m=0 row halved), k = n < N   (J=3nD, K=N)
  //  ana_D : j = n,  k = i  (w_i P)                                            (J=N,   K=nD)
  //  syn_O : j = kind*nO + i (kind 0:P 1:dP), k = n                             (J=2nO, K=N)
  //  ana_O : j = n,  k = i  (w_i P on the SH grid)                              (J=N,   K=nO)
  void* syn_D[2] = {nullptr, nullptr};  // [0] double, [1] float
  void* ana_D[2] = {nullptr, nullptr};
  void* syn_O[2] = {nullptr, nullptr};
  void* ana_O[2] = {nullptr, nullptr};
  //  syn_B : j = kind*nD + i (kind 0: d3P, 1: d4P, m=0 row halved), k = n   (J=2nD, K=N; bending)
  void* syn_B[2] = {nullptr, nullptr};
  // per-latitude data: sin, cos of theta on both grids, area weight w/sin*dphi
  void* latD[2] = {nullptr, nullptr};  // [nD][4]: sin, cos, wgtdsinf, theta
  void* latO[2] = {nullptr, nullptr};  // [nO][4]
  // cos/sin(m phi_j), [m][j], on both longitude grids
  void* trigD[2] = {nullptr, nullptr};  // [2][N][mD]
  void* trigO[2] = {nullptr, nullptr};  // [2][N][mO]
};

// One batched Legendre contraction over the capsules of one degree group.
// Row q = (c, r) with c = q / rpc, r = q % rpc; for m < M, j < J:
//   D[c*sDc + r*sDr + m*sDm + j] = sum_{k<K} A[c*sAc + r*sAr + m*sAm + k] * B[m*sBm + j*K + k]
struct LegProblem {
  const void* A;
  long long sAc, sAr, sAm;
  const void* B;
  long long sBm;
  void* D;
  long long sDc, sDr, sDm;
  int rpc;
  int Q, M, J, K;
  int tri;       // 1: k starts at m (synthesis: coefficients vanish for n<m)
  int group;     // degree group
  int kind;      // 0 syn_D, 1 ana_D, 2 syn_O, 3 ana_O
  // tensor-core operands (mixed path): per m, the three bf16 parts of B_m
  // (B = B0 + B1 + B2), each Jp x Kp in UMMA core-matrix order; sBimg = 3 Jp Kp
  const void* Bimg;
  long long sBimg;
  int Jp, Kp;    // J, K rounded up to multiples of 16
  int terms;     // split products: 3 (BF16x3) or 6 (BF16x6)
  int vecA;      // A rows 16-byte aligned with K % 8 == 0: float4 loads
  int vecD;      // D rows 16-byte aligned with J % 4 == 0: float4 stores
  int next[2];   // tensor-core path: problems whose A operand is this problem's output (-1: none)
};

struct LegWork {  // one tile of a problem
  int prob, m, q0;
  // tensor-core path: the root's chained problems (its next[0], then next[1]
  // after a next[0]), -1 for none -- carried here so that a CTA can fetch the
  // whole chain at once
  int lvl1 = -1, lvl2 = -1;
};

template <class T>
cudaError_t launch_legendre(const LegProblem* d_probs, const LegWork* d_work, int nwork, int maxJ, int maxK,
                            cudaStream_t st);
// Shared-memory sizes of one tensor-core launch: for each chain level (0 the
// root problems, 1 their next[0], 2 their next[1]) the largest padded J and K
// of its problems (0 for a level no chain reaches), and the largest padded K
// of any data operand.
struct LegLevels {
  int jp[3], kp[3];
  int a_kp;
};
// Tensor-core (tcgen05, BF16x3 / BF16x6) contraction of FP32 problems; work
// items are tiles of tm (64 or 128) rows of root problems and their chains
// (q0 a multiple of tm).  nparts = 3 if any problem reached is BF16x6, else 2.
// d_err is set to 1 if an MMA or a table copy wait times out, 2 if a problem
// does not fit the sizes of lv and nparts or its mode differs along a chain.
cudaError_t launch_legendre_mma(const LegProblem* d_probs, const LegWork* d_work, int nwork, const LegLevels& lv,
                                int nparts, int tm, int* d_err, int num_sms, cudaStream_t st);
// Dense product on the tensor cores (sg_gemm.cu):
//   C = alpha A B^T (+ bias[n]) (then GELU), A [M][K], B [N][K], K % 64 == 0.
// split = 0: A, B bf16; split = 1: A, B FP32, split into bf16 hi/lo (BF16x3).
// Outputs that are null are skipped; CbT is [N][M] (transposed).
struct GemmArgs {
  int M = 0, N = 0, K = 0;
  int split = 0;
  const void* A = nullptr;
  long long lda = 0;
  const void* B = nullptr;
  long long ldb = 0;
  float alpha = 1.f;
  const float* bias = nullptr;
  int gelu = 0;
  int accumulate = 0;  // Cf += result
  float* Cf = nullptr;
  long long ldc = 0;
  float* Cpre = nullptr;  // FP32 value after bias, before GELU
  long long ldpre = 0;
  __nv_bfloat16* Cb = nullptr;
  long long ldcb = 0;
  __nv_bfloat16* CbT = nullptr;
  long long ldcbt = 0;
  // optional FP32 workspace for split-K when the output has few tiles: each
  // K slice writes its partial product there and a second kernel sums the
  // slices in fixed order and applies the epilogue
  float* ws = nullptr;
  long long ws_floats = 0;
  int ksplit = 0;  // set by launch_gemm
};
cudaError_t launch_gemm(const GemmArgs& g, int* d_err, cudaStream_t st);

// The three bf16 parts (B = B0 + B1 + B2, Bi = bf16 of what the earlier parts
// leave) of a table B[m][j][k] (row stride K, m stride sBm) in UMMA
// core-matrix order: out[m][3][Jp/8][Kp/8][8][8]
void host_umma_image(const double* B, long long sBm, int M, int J, int K, int Jp, int Kp, uint16_t* out);

// Capsule-row work items for the pointwise kernels.
struct RowWork {
  int cap;    // capsule index (global)
  int row0;   // first latitude row
  int nrows;  // rows in this item
  int group;  // degree group
};

struct CapInfo {  // per capsule, device
  int L, N, group;
  int law;            // membrane law: 0 Skalak (membmodel.c:81-99), 1 neo-Hookean (:60-79)
  long long pt_off;   // first point (global flat index)
  long long gidx;     // index within its degree group
  double R;
  double gs, csk;     // shear modulus and (Skalak) area-dilation constant
  double eb;          // bending modulus (ebend, param.f90:91); 0: no bending terms
};

struct SpecBuffers {  // per degree group base pointers (T)
  void* Fpos;   // [ncap_g][3][2][N][nD]
  void* Cpos;   // [ncap_g][3][2][N][N]
  void* G;      // [ncap_g][3][2][N][3*nD]
  void* Fout;   // [ncap_g][6][2][N][nD]
  void* Cout;   // [ncap_g][6][2][N][N]   fields: f0 f1 f2 n0 n1 n2
  void* GO;     // [ncap_g][6][2][N][2*nO]  (normals: rows 0-2 from Cout n; shape: rows 3-5 from Cpos)
  void* Fsh;    // [ncap_g][4][2][N][nO]
  void* Csh;    // [ncap_g][4][2][N][N]    n0 n1 n2 surfmet
  void* GF;     // [ncap_g][7][2][N][nD]   f0 f1 f2 n0 n1 n2 surfmet (P only)
  void* GB;     // [ncap_g][3][2][N][2*nD] third and fourth theta-derivative series (bending only)
};

struct GroupDev {  // device copy of per-group constants; [0] double, [1] float
  int L, N, nD, mD, nO, mO;
  const void* latD[2];
  const void* latO[2];
  const void* trigD[2];
  const void* trigO[2];
  SpecBuffers buf;
};

template <class T>
cudaError_t launch_posfwd(const RowWork* work, int nwork, const CapInfo* caps, const GroupDev* groups,
                          const double* X, const double* Y, const double* Z, int ncap, double* cen, int nmax,
                          cudaStream_t st);  // cen: 3 ncap doubles of scratch (the centroids)
// The whole force stage, one CTA per capsule (sg_spectral.cu, mixed path):
// order = the capsules, largest degree first; probs = the per-group problems
// S0 S1 S2 S3a S3b S4 S5a S5b (FP32 tables); max_contract_floats = the
// largest rpc M K over them.
cudaError_t launch_force_fused(const int* order, int ncap, const CapInfo* caps, const GroupDev* groups,
                               const LegProblem* probs, const double* X, const double* Y, const double* Z, double* cen,
                               float* FX, float* FY, float* FZ, float* NX, float* NY, float* NZ, float* AREA, void* frc,
                               double dvi, int nmax, size_t max_contract_floats, cudaStream_t st);
template <class T>
cudaError_t launch_membrane(const RowWork* work, int nwork, const CapInfo* caps, const GroupDev* groups,
                            const int* sur_flag, int nmax, int* err, cudaStream_t st);
template <class T>
cudaError_t launch_shgrid(const RowWork* work, int nwork, const CapInfo* caps, const GroupDev* groups, int nmax,
                          int* err, cudaStream_t st);
template <class T>
// Also writes the spread's force records frc (ForceRec<T>[npts], cf = F * AREA
// * dvi) when frc is not null.
cudaError_t launch_final(const RowWork* work, int nwork, const CapInfo* caps, const GroupDev* groups, T* FX, T* FY,
                         T* FZ, T* NX, T* NY, T* NZ, T* AREA, void* frc, double dvi, int nmax, int* err,
                         cudaStream_t st);

// The membrane kernel with the bending terms (sg_bending.cu): every capsule
// of the work list, reading the group buffers G and GB.
template <class T>
cudaError_t launch_membrane_bend(const RowWork* work, int nwork, const CapInfo* caps, const GroupDev* groups,
                                 const int* sur_flag, int nmax, cudaStream_t st);

template <class T>
cudaError_t launch_update_pos(int ncap, const CapInfo* caps, double dt, double lx, double ly, double lz, double* X,
                              double* Y, double* Z, const T* U, const T* V, const T* W, cudaStream_t st);
// Wall collision force of collisions.f90:10-32 (constants of param.f90:57,64)
struct WallParams {
  double col, betacol, rad0, rep, dx, dy;
};
// FZ += the wall force of each point (in place).  With frc, the spread's force
// records are brought up to date as well (cf[2] = FZ * (A * dvi)), as
// pack_forces would compute them.
template <class T>
cudaError_t launch_collisions(long n, const WallParams& wp, const double* Z, const T* A, T* FZ, void* frc, double dvi,
                              cudaStream_t st);
template <class T>
cudaError_t launch_surf_vol(int ncap, const CapInfo* caps, const double* X, const double* Y, const double* Z,
                            const T* NX, const T* NY, const T* NZ, const T* AREA, const double* exy1_prev,
                            double* out, cudaStream_t st);

// Overlap mesh lid (sg_overlap.cu, interpolation.f90:10-69)
struct LidArgs {
  const double* f[5];  // u, v, w, p, indic, each at plane nf (plane nf + 1 one plane further)
  long ldi, plane;     // row and plane strides of the fields
  double* o[5];        // ub, vb, wb, pb, indb: [nj][ni]
  int ni, nj;          // itot nr + 2, jtot nr + 2
  double dx, dy, dxc, dyc, offx, offy;
};
cudaError_t launch_overlap_lid(const LidArgs& a, cudaStream_t st);

}  // namespace sg
