// sg_ctx.h -- the context behind the opaque sg_ctx handle of the C ABI
// (internal to the library): configuration, degree groups with their tables
// and spectral buffers, binning work, work lists, staging buffers, the
// surrogate network, and the helpers shared by the files that implement the
// ABI functions.
#pragma once
#include <string>
#include <vector>

#include "sg_coupling.h"
#include "sg_kernels.h"
#include "sg_surrogate.h"

namespace sg {

struct Group {
  int L = 0, N = 0, nD = 0, mD = 0, nO = 0, mO = 0;
  std::vector<int> caps;
  DegreeTables tab;
  SpecBuffers buf{};
  std::vector<double> h_tab[5];  // host FP64 syn_D, ana_D, syn_O, ana_O, syn_B (by LegProblem::kind)
};

}  // namespace sg

struct sg_ctx {
  using Group = sg::Group;
  using IBGrid = sg::IBGrid;
  using IBWork = sg::IBWork;
  using CapInfo = sg::CapInfo;
  using GroupDev = sg::GroupDev;
  using RowWork = sg::RowWork;
  using LegProblem = sg::LegProblem;
  using LegWork = sg::LegWork;
  using LegLevels = sg::LegLevels;
  sg_config cfg{};
  std::vector<int> degree;
  std::vector<double> radius;
  int mixed = 0;
  size_t esz = 8;
  IBGrid grid{};
  IBWork ibw{};
  long npts = 0;
  long long nfield = 0;
  std::vector<long long> off;
  std::vector<Group> groups;
  CapInfo* d_caps = nullptr;
  std::vector<CapInfo> h_caps;
  GroupDev* d_groups = nullptr;
  RowWork* d_wpos = nullptr;
  RowWork* d_wmem = nullptr;
  RowWork* d_wsh = nullptr;
  RowWork* d_wfin = nullptr;
  int nwpos = 0, nwmem = 0, nwsh = 0, nwfin = 0;
  int point_split = 1;  // work items per capsule of the pointwise kernels
  // wall collision force (collisions.f90): parameters set, and applied inside sg_step
  bool wall_set = false, wall_in_step = false;
  sg::WallParams wall{};
  LegProblem* d_probs = nullptr;
  LegWork* d_lw[6] = {};
  int nlw[6] = {};
  int maxJ[6] = {}, maxK[6] = {};
  // tensor-core Legendre path (mixed precision): 128-row work lists
  bool leg_tc = false;
  // fused force stage (mixed path): one CTA per capsule runs every stage
  // (sg_set_fused_force); used when no capsule bends and the surrogate is off
  bool fused = false;
  int* d_order = nullptr;      // the capsules, largest degree first
  size_t fused_cf = 0;         // largest rpc M K over the contractions (staged floats)
  // split mode of the tensor-core contractions: 0 automatic (BF16x6 from
  // degree kSixTermDegree up, BF16x3 below), 3 or 6 for every group
  int leg_terms = 0;
  int leg_parts = 2;                  // bf16 parts staged per operand (3 if any group is BF16x6)
  std::vector<LegProblem> h_probs;    // host copy of d_probs (the split mode is rewritten in place)
  LegWork* d_lwF[3] = {};  // root work items of the three chained launches (tiles of tmF rows)
  int nlwF[3] = {};
  LegWork* d_lwT[2][3] = {};  // the work items on 128-row [0] and 64-row [1] tiles
  int nlwT[2][3] = {};
  LegLevels lvF[3] = {};    // shared-memory sizes of the three chained launches
  int tmF[3] = {128, 128, 128};  // their tile rows (sg_set_legendre_tile_rows, the autotuner)
  int num_sms = 148;
  int* d_err = nullptr;   // device error flag (bounded waits that expired)
  double* d_cen = nullptr;  // capsule centroids of the step (posfwd scratch)
  double* ovl_in = nullptr;   // sg_overlap_lid in host memory mode: planes nf, nf + 1 of 5 fields
  double* ovl_out = nullptr;  // and the 5 lid arrays
  size_t ovl_out_n = 0;
  int* h_err = nullptr;   // pinned copy, refreshed at the end of every step
  int nmax = 0;
  // host-mode staging
  void* s_u = nullptr;
  void* s_v = nullptr;
  void* s_w = nullptr;
  double* s_X = nullptr;
  double* s_Y = nullptr;
  double* s_Z = nullptr;
  void* s_lag[10] = {};
  void* s_f[3] = {};
  double* s_out = nullptr;
  double* s_exy = nullptr;
  cudaStream_t st = nullptr;
  bool own_stream = false;
  // host-memory contexts: a second stream for the interpolation branch of a
  // full step (velocity upload, interp, velocity download), so that its copies
  // overlap the force branch's in the other direction; events join the two
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_bin = nullptr, ev_join = nullptr;
  // host memory: the force downloads on a third stream, beside the spread
  cudaStream_t st3 = nullptr;
  cudaEvent_t ev_frc = nullptr, ev_join3 = nullptr;
  bool join3 = false;
  std::vector<void*> allocs;
  std::string err;
  int launches = 0;
  bool profiling = false;
  // stage marks: ev[k] .. ev[k+1] bound stage k of SG_STAGE_BIN..SPREAD
  static constexpr int kMarkStages = 4;
  cudaEvent_t ev[kMarkStages + 1] = {};
  bool ev_used[kMarkStages] = {};
  // the Legendre contraction launches of the last profiled step (start, end)
  static constexpr int kMaxContract = 8;
  cudaEvent_t ev_con[2][kMaxContract] = {};
  int ncon = 0;
  std::vector<int> leg_roots[3];  // root problems of the three tensor-core launches
  // bending (sg_set_capsule_bending): the synthesis of the third and fourth
  // theta derivatives, one problem per group, as its own contraction launch
  bool bend = false;        // some capsule has a nonzero bending modulus
  bool bend_ready = false;  // tables, buffers and problems set up
  LegWork* d_lwB = nullptr;   // CUDA-core work list (32-row tiles)
  int nlwB = 0, maxJB = 0, maxKB = 0;
  LegWork* d_lwBT = nullptr;  // tensor-core work list (128-row tiles)
  int nlwBT = 0;
  LegLevels lvB{};
  int max_tiles = 0;            // binning arrays are sized for the largest tile count
  bool capturing = false;       // inside sg_graph_capture: no synchronisation, no events
  cudaGraph_t graph = nullptr;  // captured step (device memory mode)
  cudaGraphExec_t graph_exec = nullptr;
  int graph_launches = 0;
  // surrogate of the membrane force (mixed path, capsules of SH degree 15)
  sg::SurrogateNet sur;
  bool sur_ready = false;       // network allocated (cfg.surrogate)
  int sur_group = -1;           // degree group with L = 15, or -1
  int sur_n = 0;                // capsules in that group
  int* d_sur_caps = nullptr;    // [sur_n] capsule ids in group order
  int* d_sur_flag = nullptr;    // [ncap] 1: this step's force comes from the surrogate
  float* d_sur_x = nullptr;     // [sur_n][768] inputs
  float* d_sur_ylin = nullptr;  // [sur_n][768] linear response
  float* d_sur_y = nullptr;     // [sur_n][768] predicted force coefficients
  int* d_sur_count = nullptr;   // [2] capsules on the surrogate, on the fallback
  int* h_sur_count = nullptr;   // pinned copy of the last step's counts
  float sur_trust[5] = {0.f, 0.f, 0.f, 0.f, 0.f};  // amp_max, ratio_max, c_min, c_max, enabled
  // Lagrangian scratch for sg_capsule_spectra in device mode (allocated on first use)
  void* spec_scratch[7] = {};
  // solver1d on the GPU (sg_poisson.cu), shared by the indicator and the flow solver
  struct PoissonState {
    bool ready = false;
    double* r = nullptr;     // real FFT input / output [ktot][jtot][itot]
    void* c = nullptr;       // modes [ktot][jtot][nmp] (double2), nmp = itot/2 + 1 rounded up to 8
    // elimination tables per row type e = 0..3 (sg_poisson.cu): pivots z and
    // multipliers d, [ktot][jtot][nmp] each, for the shift they were made with
    double* zt[4] = {nullptr, nullptr, nullptr, nullptr};
    double* dt[4] = {nullptr, nullptr, nullptr, nullptr};
    double tshift[4] = {0, 0, 0, 0};
    bool tvalid[4] = {false, false, false, false};
    double* tab = nullptr;   // xrt [itot/2 + 1], yrt [jtot]
    double2* w = nullptr;    // twiddles of the row and column FFTs, then the row split's W^k
    double2* wpost = nullptr;
    alignas(8) unsigned char plan_x[128], plan_y[128];  // FFT plans (factorisations), see sg_poisson.cu
  } pois;
  // indicator function (sg_indicator.cu), set up by sg_set_indicator_params
  struct IndState {
    bool ready = false;
    double visc0 = 0, lambda = 1, sin_t = 0, mcos_t = 0, amp = 0;
    sg::IBGrid grid{};       // ktot + 2 planes: interior k = 0 .. kmax + 1 of the real grid
    sg::IBWork w{};          // FP64 records of the normals
    double* zr = nullptr;    // raised z of the points
    double* g = nullptr;     // gx, gy, gz on the taller grid
  } ind;
  // flow solver (sg_flow_solver.cu), set up by sg_set_flow_params
  struct FlowState {
    bool ready = false;
    double rep = 1, vb2 = 0, vt2 = 0;
    double* ru = nullptr;    // right-hand sides of u and v, [ktot][jtot][itot]
    double* rv = nullptr;
    double* p = nullptr;     // pressure correction with halos
    void* stage[13] = {};    // device copies of the fields in host memory mode
  } flow;
};

namespace sg {

inline int fail(sg_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

inline int cuda_fail(sg_ctx* c, cudaError_t e, const char* where) {
  return fail(c, SG_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define SG_TRY(expr, where)                       \
  do {                                            \
    cudaError_t _e = (expr);                      \
    if (_e != cudaSuccess) return cuda_fail(c, _e, where); \
  } while (0)

#define SG_RET(x)             \
  do {                        \
    int _r = (x);             \
    if (_r != SG_OK) return _r; \
  } while (0)

constexpr int kMaxPointSplit = 8;

// surrogate hooks (sg_surrogate_abi.cu)
int sur_setup(sg_ctx* c);
int sur_step_pre(sg_ctx* c);   // after Legendre stage 0
int sur_step_post(sg_ctx* c);  // after Legendre stage 2
const int* sur_flags(sg_ctx* c);
// force pipeline only, outputs into device arrays lag[0..6] (sg_context.cu)
int run_forces_only(sg_ctx* c, const double* X, const double* Y, const double* Z, void* const* lag);

// solver1d (sg_poisson.cu): FFT buffers and plans made once per context;
// poisson_solve replaces r ([ktot][jtot][itot], interior values) with
// itot * jtot times the solution of the rows of initsolver(e) (shift = Rep/dt
// for e = 2, 3): the FFT pair is left unnormalised.  With out, the solution
// times out->scale goes to the interior of a field with a one-cell halo
// instead (value (i, j, k), 0-based, at f[(k+1) plane + (j+1) ldi + i+1]),
// and r is left holding intermediate values.
struct PoisOut {
  double* f;
  long ldi, plane;
  double scale;
};
int poisson_setup(sg_ctx* c, unsigned types);  // types: bit e for each row type e the caller solves
void poisson_free(sg_ctx* c);
int poisson_solve(sg_ctx* c, double* r, int e, double shift, cudaStream_t st, const PoisOut* out = nullptr);
// indicator function (sg_indicator.cu)
int indicator_setup(sg_ctx* c, double visc0, double lambda, double thetainc, double ta, double rep);
template <class T>
int indicator_run(sg_ctx* c, const double* X, const double* Y, const double* Z, const T* NX, const T* NY, const T* NZ,
                  const T* A, T* indic, T* visc, T* fy, T* fz);
// flow solver (sg_flow_solver.cu), FP64 fields
int flow_setup(sg_ctx* c, double rep, double vb2, double vt2);
int flow_run(sg_ctx* c, double dt, const double* uo, const double* vo, const double* wo, const double* uoo,
             const double* voo, const double* woo, double* p, const double* fx, const double* fy, const double* fz,
             double* u, double* v, double* w);

template <class P>
cudaError_t dalloc(sg_ctx* c, P*& p, size_t bytes) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, bytes ? bytes : 16);
  if (e == cudaSuccess) {
    c->allocs.push_back(q);
    p = (P*)q;
  }
  return e;
}


}  // namespace sg
