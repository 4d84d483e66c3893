// sg_surrogate_abi.cu -- C ABI of the membrane-force surrogate and of the
// spectral coefficient export (include/sg_coupling.h), the training driver,
// and the two hooks by which the mixed-precision step uses the network.
//
// Coefficient slots.  Per capsule of degree L (N = L + 1) and per component
// c = x, y, z there are N^2 real SH coefficients in SPHEREPACK's (a, b)
// convention (shagc.f:189-220): a(m, n) for 0 <= m <= n < N in m-major order,
// then b(m, n) for 1 <= m <= n < N; component c occupies slots
// [c N^2, (c + 1) N^2).  These are the coefficients of the displacement from
// the reference sphere (after the centroid is removed) and of the force after
// the reference's force filter (filter_modes4__OPT, sph1.f90:919-932).
#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <vector>

#include "sg_ctx.h"

using namespace sg;

namespace {

// slot -> offset in a capsule's [6][N][N] block (rows (comp, a/b), m, n)
__device__ __forceinline__ int slot_offset(int s, int N) {
  const int NN = N * N, c = s / NN;
  int t = s - c * NN, m = 0, ab = 0;
  const int na = N * (N + 1) / 2;
  if (t >= na) {
    t -= na;
    ab = 1;
    m = 1;
  }
  while (t >= N - m) {
    t -= N - m;
    ++m;
  }
  const int n = m + t;
  return (2 * c + ab) * NN + m * N + n;
}

// out[k][s] for the capsules of one degree group: src is Cpos (rows 0..5 of
// 6) or Cout (rows 0..5 of 12, the force)
template <class T>
__global__ void export_spectra_kernel(const CapInfo* __restrict__ caps, const GroupDev* __restrict__ groups,
                                      const int* __restrict__ capids, int ncap, int which, double* __restrict__ out,
                                      const long long* __restrict__ out_off) {
  const int k = blockIdx.x;
  if (k >= ncap) return;
  const CapInfo ci = caps[capids[k]];
  const GroupDev gd = groups[ci.group];
  const int N = gd.N, NN = N * N;
  const T* src = which == 0 ? (const T*)gd.buf.Cpos + ci.gidx * 6 * NN : (const T*)gd.buf.Cout + ci.gidx * 12 * NN;
  double* o = out + out_off[capids[k]];
  for (int s = threadIdx.x; s < 3 * NN; s += blockDim.x) o[s] = (double)src[slot_offset(s, N)];
}

// Surrogate inputs of the degree-15 group: x = Cpos / R, slot 0 = C, slots
// N^2 and 2 N^2 (the y and z translations) = 0.
__global__ void sur_pack_kernel(const CapInfo* __restrict__ caps, const GroupDev* __restrict__ groups,
                                const int* __restrict__ capids, int n, float* __restrict__ x) {
  const int b = blockIdx.x;
  if (b >= n) return;
  const CapInfo ci = caps[capids[b]];
  const GroupDev gd = groups[ci.group];
  const int N = gd.N, NN = N * N;
  const float* src = (const float*)gd.buf.Cpos + ci.gidx * 6 * NN;
  const float iR = (float)(1.0 / ci.R);
  float* xo = x + (long long)b * 3 * NN;
  for (int s = threadIdx.x; s < 3 * NN; s += blockDim.x) {
    float v = src[slot_offset(s, N)] * iR;
    if (s == 0) v = (float)ci.csk;
    if (s == NN || s == 2 * NN) v = 0.f;
    xo[s] = v;
  }
}

// Residual check per capsule: the surrogate is used when the capsule follows
// the Skalak law it was trained on, and the displacement amplitude |x|, the
// size of the learned nonlinear residual relative to the linear response
// |y_mlp| / |y_lin|, and C lie in the validated ranges.
__global__ void sur_trust_kernel(const CapInfo* __restrict__ caps, const int* __restrict__ capids, int n, int din,
                                 const float* __restrict__ x,
                                 const float* __restrict__ ylin, const float* __restrict__ y,
                                 const float* __restrict__ ampv, float amp_max, float ratio_max, float c_min,
                                 float c_max, int* __restrict__ flag, int* __restrict__ count) {
  __shared__ float red[2][128];
  const int b = blockIdx.x, t = threadIdx.x;
  if (b >= n) return;
  const float* xb = x + (long long)b * din;
  const float* lb = ylin + (long long)b * din;
  const float* yb = y + (long long)b * din;
  float l = 0.f, r = 0.f;
  for (int s = t; s < din; s += 128) {
    l += lb[s] * lb[s];
    const float q = yb[s] - lb[s];
    r += q * q;
  }
  red[0][t] = l;
  red[1][t] = r;
  __syncthreads();
  for (int o = 64; o > 0; o >>= 1) {
    if (t < o)
      for (int q = 0; q < 2; ++q) red[q][t] += red[q][t + o];
    __syncthreads();
  }
  if (t == 0) {
    const float amp = ampv[b], lin = sqrtf(red[0][0]), res = sqrtf(red[1][0]);
    const float C = xb[0];
    const bool ok = caps[capids[b]].law == SG_LAW_SKALAK && caps[capids[b]].eb == 0.0 && amp <= amp_max &&
                    res <= ratio_max * lin &&
                    C >= c_min && C <= c_max;
    flag[capids[b]] = ok ? 1 : 0;
    atomicAdd(&count[ok ? 0 : 1], 1);
  }
}

// Force coefficients of the surrogate capsules into Cout rows 0..5 (after the
// force analysis, which left zeros there): y * Gs / R.
__global__ void sur_unpack_kernel(const CapInfo* __restrict__ caps, const GroupDev* __restrict__ groups,
                                  const int* __restrict__ capids, int n, const int* __restrict__ flag,
                                  const float* __restrict__ y) {
  const int b = blockIdx.x;
  if (b >= n) return;
  const int cap = capids[b];
  if (!flag[cap]) return;
  const CapInfo ci = caps[cap];
  const GroupDev gd = groups[ci.group];
  const int N = gd.N, NN = N * N;
  float* dst = (float*)gd.buf.Cout + ci.gidx * 12 * NN;
  const float sc = (float)(ci.gs / ci.R);
  const float* yb = y + (long long)b * 3 * NN;
  for (int s = threadIdx.x; s < 3 * NN; s += blockDim.x) dst[slot_offset(s, N)] = yb[s] * sc;
}

// residual targets t = (Y - ylin - mu_y) / sd_y for gathered rows
__global__ void sur_target_kernel(const float* __restrict__ R, const int* __restrict__ rows, int B, int dout,
                                  const float* __restrict__ mu, const float* __restrict__ sd, float* __restrict__ t) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)B * dout) return;
  const int b = (int)(q / dout), o = (int)(q - (long long)b * dout);
  t[q] = (R[(long long)rows[b] * dout + o] - mu[o]) / sd[o];
}

// R[b][o] /= amp[b]^2
__global__ void scale_rows_kernel(float* __restrict__ R, const float* __restrict__ amp, int B, int dout) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)B * dout) return;
  const float a = amp[q / dout];
  R[q] /= a * a;
}

__global__ void sub_kernel(float* __restrict__ a, const float* __restrict__ b, long long n) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) a[q] -= b[q];
}

// per-column mean and standard deviation in two passes with a fixed
// summation order: partial sums of 64 row chunks, then their total
constexpr int kStatChunks = 64;
__global__ void col_partial_kernel(const float* __restrict__ A, long long n, int C, double* __restrict__ part) {
  __shared__ double s1[8][33], s2[8][33];
  const int tx = threadIdx.x, ty = threadIdx.y, c = blockIdx.x * 32 + tx, chunk = blockIdx.y;
  const long long r0 = n * chunk / kStatChunks, r1 = n * (chunk + 1) / kStatChunks;
  double a = 0.0, b = 0.0;
  if (c < C)
    for (long long r = r0 + ty; r < r1; r += 8) {
      const double v = A[r * C + c];
      a += v;
      b += v * v;
    }
  s1[ty][tx] = a;
  s2[ty][tx] = b;
  __syncthreads();
  if (ty == 0 && c < C) {
    for (int q = 1; q < 8; ++q) {
      a += s1[q][tx];
      b += s2[q][tx];
    }
    part[(long long)chunk * 2 * C + c] = a;
    part[(long long)chunk * 2 * C + C + c] = b;
  }
}
__global__ void col_finish_kernel(const double* __restrict__ part, long long n, int C, float* __restrict__ mu,
                                  float* __restrict__ sd) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  double s = 0.0, s2 = 0.0;
  for (int k = 0; k < kStatChunks; ++k) {
    s += part[(long long)k * 2 * C + c];
    s2 += part[(long long)k * 2 * C + C + c];
  }
  const double m = s / (double)n;
  const double var = s2 / (double)n - m * m;
  mu[c] = (float)m;
  sd[c] = (float)(var > 0 ? sqrt(var) : 0.0);
}
cudaError_t col_stats(const float* A, long long n, int C, float* mu, float* sd, double* part, cudaStream_t st) {
  col_partial_kernel<<<dim3((C + 31) / 32, kStatChunks), dim3(32, 8), 0, st>>>(A, n, C, part);
  col_finish_kernel<<<(C + 255) / 256, 256, 0, st>>>(part, n, C, mu, sd);
  return cudaGetLastError();
}
__global__ void sd_floor_kernel(float* __restrict__ sd, int C) {
  __shared__ float mx;
  if (threadIdx.x == 0) {
    float m = 0.f;
    for (int c = 0; c < C; ++c) m = fmaxf(m, sd[c]);
    mx = m;
  }
  __syncthreads();
  for (int c = threadIdx.x; c < C; c += blockDim.x)
    if (!(sd[c] > 1e-6f * mx)) sd[c] = 1.f;
}

inline unsigned nblk(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

int sur_check(sg_ctx* c) {
  if (!c) return SG_ERR_ARG;
  if (!c->sur_ready) return fail(c, SG_ERR_STATE, "the context was created without the surrogate");
  return SG_OK;
}

}  // namespace

namespace sg {

// Called from sg_create: the network and its step buffers.
int sur_setup(sg_ctx* c) {
  if (!c->cfg.surrogate) return SG_OK;
  for (size_t g = 0; g < c->groups.size(); ++g)
    if (c->groups[g].L == SUR_N - 1) c->sur_group = (int)g;
  std::vector<int> ids;
  if (c->sur_group >= 0) ids = c->groups[c->sur_group].caps;
  c->sur_n = (int)ids.size();
  const int cap = std::max(1024, (c->sur_n + 63) / 64 * 64);
  SG_TRY(sur_alloc(c->sur, cap), "surrogate alloc");
  for (void* p : c->sur.allocs) c->allocs.push_back(p);  // freed with the context
  c->sur.allocs.clear();
  const size_t nx = (size_t)std::max(c->sur_n, 1) * SUR_DIN;
  SG_TRY(dalloc(c, c->d_sur_x, 4 * nx), "alloc");
  SG_TRY(dalloc(c, c->d_sur_ylin, 4 * nx), "alloc");
  SG_TRY(dalloc(c, c->d_sur_y, 4 * nx), "alloc");
  SG_TRY(dalloc(c, c->d_sur_flag, sizeof(int) * std::max(c->cfg.ncap, 1)), "alloc");
  SG_TRY(cudaMemset(c->d_sur_flag, 0, sizeof(int) * std::max(c->cfg.ncap, 1)), "memset");
  SG_TRY(dalloc(c, c->d_sur_count, 2 * sizeof(int)), "alloc");
  SG_TRY(cudaMallocHost(&c->h_sur_count, 2 * sizeof(int)), "cudaMallocHost");
  c->h_sur_count[0] = c->h_sur_count[1] = 0;
  void* tmp = nullptr;
  if (ids.empty()) ids.push_back(0);
  SG_TRY(dalloc(c, tmp, sizeof(int) * ids.size()), "alloc");
  SG_TRY(cudaMemcpy(tmp, ids.data(), sizeof(int) * ids.size(), cudaMemcpyHostToDevice), "upload");
  c->d_sur_caps = (int*)tmp;
  SG_TRY(sur_init_params(c->sur, 1, c->st), "surrogate init");
  c->sur_ready = true;
  return SG_OK;
}

// After Legendre stage 0 (displacement coefficients in Cpos): predict, check.
int sur_step_pre(sg_ctx* c) {
  if (!c->sur_ready) return SG_OK;
  c->h_sur_count[0] = c->h_sur_count[1] = 0;
  if (c->sur_n == 0 || !c->sur.trained || c->sur_trust[4] == 0.f) return SG_OK;
  SurrogateNet& s = c->sur;
  const int n = c->sur_n;
  SG_TRY(cudaMemsetAsync(c->d_sur_count, 0, 2 * sizeof(int), c->st), "memset");
  sur_pack_kernel<<<n, 256, 0, c->st>>>(c->d_caps, c->d_groups, c->d_sur_caps, n, c->d_sur_x);
  SG_TRY(cudaGetLastError(), "surrogate pack");
  SG_TRY(sur_features(c->d_sur_x, n, s.din, s.feat, s.amp, c->st), "surrogate features");
  SG_TRY(sur_normalise(s, s.feat, nullptr, n, c->st), "surrogate normalise");
  SG_TRY(sur_forward(s, n, c->d_err, c->st), "surrogate forward");
  SG_TRY(sur_linear(s, c->d_sur_x, n, c->d_sur_ylin, c->d_err, c->st), "surrogate linear");
  SG_TRY(sur_combine(s, c->d_sur_ylin, s.yhat, s.amp, n, 1, 1, c->d_sur_y, c->st), "surrogate combine");
  sur_trust_kernel<<<n, 128, 0, c->st>>>(c->d_caps, c->d_sur_caps, n, s.din, c->d_sur_x, c->d_sur_ylin, c->d_sur_y, s.amp,
                                         c->sur_trust[0], c->sur_trust[1], c->sur_trust[2], c->sur_trust[3],
                                         c->d_sur_flag, c->d_sur_count);
  SG_TRY(cudaGetLastError(), "surrogate check");
  c->launches += 13;
  return SG_OK;
}

// After Legendre stage 2 (force analysis): surrogate force into Cout.
int sur_step_post(sg_ctx* c) {
  if (!c->sur_ready || c->sur_n == 0 || !c->sur.trained || c->sur_trust[4] == 0.f) return SG_OK;
  sur_unpack_kernel<<<c->sur_n, 256, 0, c->st>>>(c->d_caps, c->d_groups, c->d_sur_caps, c->sur_n, c->d_sur_flag,
                                                 c->d_sur_y);
  SG_TRY(cudaGetLastError(), "surrogate unpack");
  SG_TRY(cudaMemcpyAsync(c->h_sur_count, c->d_sur_count, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->st), "counts");
  c->launches += 1;
  return SG_OK;
}

const int* sur_flags(sg_ctx* c) {
  if (!c->sur_ready || c->sur_n == 0 || !c->sur.trained || c->sur_trust[4] == 0.f) return nullptr;
  return c->d_sur_flag;
}

}  // namespace sg

extern "C" {

int sg_capsule_spectra(sg_ctx* c, const double* X, const double* Y, const double* Z, double* disp, double* force) {
  if (!c) return SG_ERR_ARG;
  if (!X || !Y || !Z || !disp || !force) return fail(c, SG_ERR_ARG, "null array argument");
  const int nc = c->cfg.ncap;
  if (nc == 0) return SG_OK;
  // Lagrangian outputs of the force pipeline are not returned: scratch
  if (!c->spec_scratch[0])
    for (int q = 0; q < 7; ++q) SG_TRY(dalloc(c, c->spec_scratch[q], c->esz * std::max(c->npts, 1L)), "alloc");
  // the plain model: no surrogate while exporting
  const float en = c->sur_trust[4];
  c->sur_trust[4] = 0.f;
  const int rc = run_forces_only(c, X, Y, Z, c->spec_scratch);
  c->sur_trust[4] = en;
  SG_RET(rc);
  std::vector<long long> off(nc + 1, 0);
  for (int k = 0; k < nc; ++k) off[k + 1] = off[k] + 3LL * (c->degree[k] + 1) * (c->degree[k] + 1);
  std::vector<int> ids(nc);
  std::iota(ids.begin(), ids.end(), 0);
  int* d_ids = nullptr;
  long long* d_off = nullptr;
  double *d_disp = nullptr, *d_force = nullptr;
  const bool host = c->cfg.mem == SG_MEM_HOST;
  int rc2 = SG_OK;
  auto ck = [&](cudaError_t e, const char* w) {
    if (e != cudaSuccess && rc2 == SG_OK) rc2 = cuda_fail(c, e, w);
    return rc2 == SG_OK;
  };
  if (ck(cudaMalloc(&d_ids, sizeof(int) * nc), "alloc") && ck(cudaMalloc(&d_off, sizeof(long long) * (nc + 1)), "alloc") &&
      ck(cudaMemcpy(d_ids, ids.data(), sizeof(int) * nc, cudaMemcpyHostToDevice), "upload") &&
      ck(cudaMemcpy(d_off, off.data(), sizeof(long long) * (nc + 1), cudaMemcpyHostToDevice), "upload")) {
    if (host) {
      ck(cudaMalloc(&d_disp, sizeof(double) * off[nc]), "alloc");
      ck(cudaMalloc(&d_force, sizeof(double) * off[nc]), "alloc");
    } else {
      d_disp = disp;
      d_force = force;
    }
    if (rc2 == SG_OK) {
      for (int w = 0; w < 2; ++w) {
        double* o = w == 0 ? d_disp : d_force;
        if (c->mixed)
          export_spectra_kernel<float><<<nc, 256, 0, c->st>>>(c->d_caps, c->d_groups, d_ids, nc, w, o, d_off);
        else
          export_spectra_kernel<double><<<nc, 256, 0, c->st>>>(c->d_caps, c->d_groups, d_ids, nc, w, o, d_off);
      }
      ck(cudaGetLastError(), "export");
      ck(cudaStreamSynchronize(c->st), "synchronize");
      if (host && rc2 == SG_OK) {
        ck(cudaMemcpy(disp, d_disp, sizeof(double) * off[nc], cudaMemcpyDeviceToHost), "download");
        ck(cudaMemcpy(force, d_force, sizeof(double) * off[nc], cudaMemcpyDeviceToHost), "download");
      }
    }
  }
  if (d_ids) cudaFree(d_ids);
  if (d_off) cudaFree(d_off);
  if (host) {
    if (d_disp) cudaFree(d_disp);
    if (d_force) cudaFree(d_force);
  }
  return rc2;
}

int sg_set_capsule_membrane(sg_ctx* c, const double* gs, const double* csk) {
  if (!c) return SG_ERR_ARG;
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph first");
  for (int k = 0; k < c->cfg.ncap; ++k) {
    if (gs) {
      if (!(gs[k] > 0)) return fail(c, SG_ERR_ARG, "Gs must be positive");
      c->h_caps[k].gs = gs[k];
    }
    if (csk) c->h_caps[k].csk = csk[k];
  }
  SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
  SG_TRY(cudaMemcpy(c->d_caps, c->h_caps.data(), sizeof(CapInfo) * c->h_caps.size(), cudaMemcpyHostToDevice),
         "upload");
  return SG_OK;
}

int sg_set_capsule_law(sg_ctx* c, const int* law) {
  if (!c || !law) return SG_ERR_ARG;
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph first");
  for (int k = 0; k < c->cfg.ncap; ++k)
    if (law[k] != SG_LAW_SKALAK && law[k] != SG_LAW_NEO_HOOKEAN) return fail(c, SG_ERR_ARG, "unknown membrane law");
  for (int k = 0; k < c->cfg.ncap; ++k) c->h_caps[k].law = law[k];
  SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
  SG_TRY(cudaMemcpy(c->d_caps, c->h_caps.data(), sizeof(CapInfo) * c->h_caps.size(), cudaMemcpyHostToDevice),
         "upload");
  return SG_OK;
}

long sg_surrogate_param_count(void) {
  const long din = SUR_DIN, dh = SUR_DH, dout = SUR_DOUT;
  return dh * din + dh + dh * dh + dh + dout * dh + dout  // network
         + 2 * dout * din                                // L0, L1
         + 2 * din + 2 * dout;                           // mu_x, sd_x, mu_y, sd_y
}

int sg_surrogate_params(sg_ctx* c, int set, float* buf, long n) {
  SG_RET(sur_check(c));
  if (!buf || n != sg_surrogate_param_count()) return fail(c, SG_ERR_ARG, "buffer size must be sg_surrogate_param_count()");
  SurrogateNet& s = c->sur;
  struct Piece {
    float* p;
    size_t n;
  };
  const Piece pieces[6] = {{s.P, s.np},
                           {s.Lcat, (size_t)2 * s.dout * s.din},
                           {s.mu_x, (size_t)s.din},
                           {s.sd_x, (size_t)s.din},
                           {s.mu_y, (size_t)s.dout},
                           {s.sd_y, (size_t)s.dout}};
  SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
  size_t o = 0;
  for (const Piece& p : pieces) {
    if (set)
      SG_TRY(cudaMemcpy(p.p, buf + o, 4 * p.n, cudaMemcpyHostToDevice), "upload");
    else
      SG_TRY(cudaMemcpy(buf + o, p.p, 4 * p.n, cudaMemcpyDeviceToHost), "download");
    o += p.n;
  }
  if (set) {
    SG_TRY(sur_refresh_bf16(s, c->st), "refresh");
    SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
    s.trained = true;
  }
  return SG_OK;
}

int sg_surrogate_set_linear(sg_ctx* c, const float* L0, const float* L1) {
  SG_RET(sur_check(c));
  if (!L0 || !L1) return fail(c, SG_ERR_ARG, "null array argument");
  const size_t nn = (size_t)c->sur.dout * c->sur.din;
  SG_TRY(cudaMemcpy(c->sur.Lcat, L0, 4 * nn, cudaMemcpyHostToDevice), "upload");
  SG_TRY(cudaMemcpy(c->sur.Lcat + nn, L1, 4 * nn, cudaMemcpyHostToDevice), "upload");
  return SG_OK;
}

int sg_surrogate_set_trust(sg_ctx* c, float amp_max, float ratio_max, float c_min, float c_max) {
  SG_RET(sur_check(c));
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph first");
  c->sur_trust[0] = amp_max;
  c->sur_trust[1] = ratio_max;
  c->sur_trust[2] = c_min;
  c->sur_trust[3] = c_max;
  c->sur_trust[4] = (amp_max > 0 && ratio_max > 0) ? 1.f : 0.f;  // zero limits turn the surrogate off
  return SG_OK;
}

int sg_surrogate_last_counts(sg_ctx* c, int* n_surrogate, int* n_fallback) {
  SG_RET(sur_check(c));
  SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
  if (n_surrogate) *n_surrogate = c->h_sur_count[0];
  if (n_fallback) *n_fallback = c->h_sur_count[1];
  return SG_OK;
}

int sg_surrogate_train(sg_ctx* c, const float* X, const float* Y, long n, int epochs, int batch, float lr,
                       unsigned long long seed, float* loss_hist) {
  SG_RET(sur_check(c));
  SurrogateNet& s = c->sur;
  if (!X || !Y || n < 1 || epochs < 1) return fail(c, SG_ERR_ARG, "bad training arguments");
  if (batch < 64 || batch % 64 || batch > s.cap || batch > n)
    return fail(c, SG_ERR_ARG, "batch must be a multiple of 64, at most 1024 and at most n");
  const size_t din = s.din, dout = s.dout;
  float *dX = nullptr, *dR = nullptr;
  int* dperm = nullptr;
  SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
  int rc = SG_OK;
  auto ck = [&](cudaError_t e, const char* w) {
    if (e != cudaSuccess && rc == SG_OK) rc = cuda_fail(c, e, w);
    return rc == SG_OK;
  };
  if (ck(cudaMalloc(&dX, 4 * din * n), "alloc") && ck(cudaMalloc(&dR, 4 * dout * n), "alloc") &&
      ck(cudaMalloc(&dperm, sizeof(int) * n), "alloc") &&
      ck(cudaMemcpy(dX, X, 4 * din * n, cudaMemcpyHostToDevice), "upload") &&
      ck(cudaMemcpy(dR, Y, 4 * dout * n, cudaMemcpyHostToDevice), "upload")) {
    // residual targets R = (Y - (L0 + C L1) x) / a^2 and features phi(x)
    // (in place), in chunks of the batch capacity
    for (long r0 = 0; r0 < n && rc == SG_OK; r0 += s.cap) {
      const int B = (int)std::min<long>(s.cap, n - r0);
      ck(sur_linear(s, dX + r0 * din, B, s.yhat, c->d_err, c->st), "linear");
      sub_kernel<<<nblk((long long)B * dout), 256, 0, c->st>>>(dR + r0 * dout, s.yhat, (long long)B * dout);
      ck(cudaGetLastError(), "residual");
      ck(sur_features(dX + r0 * din, B, (int)din, dX + r0 * din, s.amp, c->st), "features");
      scale_rows_kernel<<<nblk((long long)B * dout), 256, 0, c->st>>>(dR + r0 * dout, s.amp, B, (int)dout);
      ck(cudaGetLastError(), "scale");
    }
    double* part = nullptr;
    if (ck(cudaMalloc(&part, sizeof(double) * kStatChunks * 2 * std::max(din, dout)), "alloc")) {
      ck(col_stats(dX, n, (int)din, s.mu_x, s.sd_x, part, c->st), "stats");
      ck(col_stats(dR, n, (int)dout, s.mu_y, s.sd_y, part, c->st), "stats");
      ck(cudaStreamSynchronize(c->st), "synchronize");
      cudaFree(part);
    }
    sd_floor_kernel<<<1, 256, 0, c->st>>>(s.sd_x, (int)din);
    sd_floor_kernel<<<1, 256, 0, c->st>>>(s.sd_y, (int)dout);
    ck(cudaGetLastError(), "stats");
    ck(sur_init_params(s, seed, c->st), "init");
    std::mt19937_64 rng(seed ^ 0x5a5a5a5aull);
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    const long nb = n / batch;
    const long total = nb * epochs;
    long step = 0;
    for (int ep = 0; ep < epochs && rc == SG_OK; ++ep) {
      std::shuffle(perm.begin(), perm.end(), rng);
      ck(cudaMemcpyAsync(dperm, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->st), "upload");
      ck(cudaMemsetAsync(s.loss, 0, sizeof(float), c->st), "memset");
      for (long b = 0; b < nb && rc == SG_OK; ++b, ++step) {
        const int* rows = dperm + b * batch;
        ck(sur_normalise(s, dX, rows, batch, c->st), "normalise");
        sur_target_kernel<<<nblk((long long)batch * dout), 256, 0, c->st>>>(dR, rows, batch, (int)dout, s.mu_y,
                                                                             s.sd_y, s.tgt);
        ck(cudaGetLastError(), "targets");
        ck(sur_forward(s, batch, c->d_err, c->st), "forward");
        ck(sur_backward(s, batch, c->d_err, c->st), "backward");
        // cosine decay to 1% of lr
        const float f = 0.01f + 0.99f * 0.5f * (1.f + std::cos(3.14159265f * (float)step / (float)total));
        ck(sur_adam(s, lr * f, c->st), "adam");
      }
      float l = 0.f;
      if (ck(cudaMemcpyAsync(&l, s.loss, sizeof(float), cudaMemcpyDeviceToHost, c->st), "loss") &&
          ck(cudaStreamSynchronize(c->st), "synchronize") && loss_hist)
        loss_hist[ep] = l / (float)nb;
    }
    int err = 0;
    ck(cudaMemcpy(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost), "error flag");
    if (rc == SG_OK && err) {
      cudaMemset(c->d_err, 0, sizeof(int));
      rc = fail(c, SG_ERR_TIMEOUT, "a tensor-core completion wait timed out during training");
    }
  }
  if (dX) cudaFree(dX);
  if (dR) cudaFree(dR);
  if (dperm) cudaFree(dperm);
  if (rc == SG_OK) s.trained = true;
  return rc;
}

int sg_surrogate_predict(sg_ctx* c, const float* X, long n, int parts, float* Y) {
  SG_RET(sur_check(c));
  SurrogateNet& s = c->sur;
  if (!X || !Y || n < 0 || parts < 1 || parts > 3) return fail(c, SG_ERR_ARG, "bad arguments");
  const size_t din = s.din, dout = s.dout;
  float *dX = nullptr, *dY = nullptr;
  int rc = SG_OK;
  auto ck = [&](cudaError_t e, const char* w) {
    if (e != cudaSuccess && rc == SG_OK) rc = cuda_fail(c, e, w);
    return rc == SG_OK;
  };
  SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
  if (ck(cudaMalloc(&dX, 4 * din * std::max(n, 1L)), "alloc") && ck(cudaMalloc(&dY, 4 * dout * std::max(n, 1L)), "alloc") &&
      ck(cudaMemcpy(dX, X, 4 * din * n, cudaMemcpyHostToDevice), "upload")) {
    for (long r0 = 0; r0 < n && rc == SG_OK; r0 += s.cap) {
      const int B = (int)std::min<long>(s.cap, n - r0);
      ck(sur_features(dX + r0 * din, B, (int)din, s.feat, s.amp, c->st), "features");
      ck(sur_normalise(s, s.feat, nullptr, B, c->st), "normalise");
      ck(sur_forward(s, B, c->d_err, c->st), "forward");
      ck(sur_linear(s, dX + r0 * din, B, s.tgt, c->d_err, c->st), "linear");
      ck(sur_combine(s, s.tgt, s.yhat, s.amp, B, parts & 1, (parts >> 1) & 1, dY + r0 * dout, c->st), "combine");
    }
    ck(cudaStreamSynchronize(c->st), "synchronize") &&
        ck(cudaMemcpy(Y, dY, 4 * dout * n, cudaMemcpyDeviceToHost), "download");
  }
  if (dX) cudaFree(dX);
  if (dY) cudaFree(dY);
  return rc;
}

}  // extern "C"
