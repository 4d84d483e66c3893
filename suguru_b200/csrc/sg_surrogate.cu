// sg_surrogate.cu -- forward, backward and Adam kernels of the membrane-force
// surrogate network (sg_surrogate.h), on the tcgen05 dense-product kernel of
// sg_gemm.cu plus small element-wise kernels written here.
//
// Layer l: pre_l = h_{l-1} W_l^T + b_l, h_l = GELU(pre_l) (l = 1, 2), and
// yhat = h_2 W_3^T + b_3.  Activations are kept in bf16 twice, row-major for
// the next forward product and transposed for the weight-gradient product
// (dW_l = dpre_l^T h_{l-1} with the batch as the contraction dimension).
// Backward: dyhat = 2 (yhat - t) / (B dout); dh = dpre_{l+1} W_{l+1};
// dpre = dh * GELU'(pre); db = column sums of dpre (fixed order).
#include <cmath>
#include <random>

#include "sg_kernels.h"
#include "sg_surrogate.h"

namespace sg {

namespace {

// d/dx GELU = Phi(x) + x phi(x)
__device__ __forceinline__ float gelu_grad(float x) {
  const float Phi = 0.5f * (1.f + erff(x * 0.70710678118654752f));
  const float phi = 0.39894228040143268f * expf(-0.5f * x * x);
  return Phi + x * phi;
}

// in [R][C] FP32 -> out [R][C] bf16 and outT [C][R] bf16 (either may be null);
// 32 x 32 tiles through shared memory so that both stores are coalesced.
__global__ void cvt_pair_kernel(const float* __restrict__ in, int R, int C, __nv_bfloat16* __restrict__ out,
                                __nv_bfloat16* __restrict__ outT) {
  __shared__ float t[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int k = ty; k < 32; k += 8) {
    const int r = r0 + k, c = c0 + tx;
    float v = 0.f;
    if (r < R && c < C) {
      v = in[(long long)r * C + c];
      if (out) out[(long long)r * C + c] = __float2bfloat16_rn(v);
    }
    t[k][tx] = v;
  }
  if (!outT) return;
  __syncthreads();
  for (int k = ty; k < 32; k += 8) {
    const int c = c0 + k, r = r0 + tx;
    if (r < R && c < C) outT[(long long)c * R + r] = __float2bfloat16_rn(t[tx][k]);
  }
}

cudaError_t cvt_pair(const float* in, int R, int C, __nv_bfloat16* out, __nv_bfloat16* outT, cudaStream_t st) {
  dim3 grid((C + 31) / 32, (R + 31) / 32), block(32, 8);
  cvt_pair_kernel<<<grid, block, 0, st>>>(in, R, C, out, outT);
  return cudaGetLastError();
}

// xf[b][i] = (X[row_b][i] - mu[i]) / sd[i]
__global__ void normalise_kernel(const float* __restrict__ X, const int* __restrict__ rows, int B, int din,
                                 const float* __restrict__ mu, const float* __restrict__ sd, float* __restrict__ xf) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)B * din) return;
  const int b = (int)(q / din), i = (int)(q - (long long)b * din);
  const long long r = rows ? rows[b] : b;
  xf[q] = (X[r * din + i] - mu[i]) / sd[i];
}

// dy = 2 (yhat - t) / (B dout); loss += sum (yhat - t)^2 / (B dout)
__global__ void loss_grad_kernel(const float* __restrict__ yhat, const float* __restrict__ t, long long n, float scale,
                                 float* __restrict__ dy, float* __restrict__ loss) {
  __shared__ float red[256];
  float acc = 0.f;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const float e = yhat[q] - t[q];
    dy[q] = 2.f * e * scale;
    acc += e * e;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] * scale);
}

// dpre = dh * GELU'(pre), in place on dh
__global__ void gelu_back_kernel(float* __restrict__ dh, const float* __restrict__ pre, long long n) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) dh[q] *= gelu_grad(pre[q]);
}

// out[c] = sum_r in[r][c], rows in fixed order
__global__ void colsum_kernel(const float* __restrict__ in, int R, int C, float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  float s = 0.f;
  for (int r = 0; r < R; ++r) s += in[(long long)r * C + c];
  out[c] = s;
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr, float b1, float b2, float c1, float c2,
                            float eps) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float gq = g[q];
  const float mq = b1 * m[q] + (1.f - b1) * gq;
  const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
  m[q] = mq;
  v[q] = vq;
  p[q] -= lr * (mq * c1) / (sqrtf(vq * c2) + eps);
}

// ylin[b][o] = Y01[b][o] + C_b Y01[b][dout + o], C_b = X[b][0]
__global__ void linear_combine_kernel(const float* __restrict__ y01, const float* __restrict__ X, int B, int din,
                                      int dout, float* __restrict__ ylin) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)B * dout) return;
  const int b = (int)(q / dout), o = (int)(q - (long long)b * dout);
  const float C = X[(long long)b * din];
  ylin[q] = y01[(long long)b * 2 * dout + o] + C * y01[(long long)b * 2 * dout + dout + o];
}

__global__ void combine_kernel(const float* __restrict__ ylin, const float* __restrict__ yhat,
                               const float* __restrict__ amp, long long n, int dout, const float* __restrict__ mu,
                               const float* __restrict__ sd, int use_linear, int use_mlp, float* __restrict__ y) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int o = (int)(q % dout);
  const float a = amp[q / dout];
  float v = use_linear ? ylin[q] : 0.f;
  if (use_mlp) v += a * a * (yhat[q] * sd[o] + mu[o]);
  y[q] = v;
}

// phi(x): direction of the displacement slots, C in slot 0, log a in slot
// N^2 (din / 3), zero in slot 2 N^2; one block per row, in place allowed
__global__ void features_kernel(const float* __restrict__ X, int din, float* __restrict__ F,
                                float* __restrict__ amp) {
  __shared__ float red[128];
  const int b = blockIdx.x, t = threadIdx.x, nn = din / 3;
  const float* x = X + (long long)b * din;
  float acc = 0.f;
  for (int i = t; i < din; i += 128)
    if (i != 0 && i != nn && i != 2 * nn) acc += x[i] * x[i];
  red[t] = acc;
  __syncthreads();
  for (int o = 64; o > 0; o >>= 1) {
    if (t < o) red[t] += red[t + o];
    __syncthreads();
  }
  const float a = fmaxf(sqrtf(red[0]), 1e-12f);
  const float C = x[0];
  __syncthreads();  // every read of the row precedes the writes below (F may alias X)
  float* f = F + (long long)b * din;
  for (int i = t; i < din; i += 128) {
    float v;
    if (i == 0) v = C;
    else if (i == nn) v = logf(a);
    else if (i == 2 * nn) v = 0.f;
    else v = x[i] / a;
    f[i] = v;
  }
  if (t == 0) amp[b] = a;
}

inline unsigned blocks(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace

#define SG_CK(x)                            \
  do {                                      \
    cudaError_t _e = (x);                   \
    if (_e != cudaSuccess) return _e;       \
  } while (0)

cudaError_t sur_alloc(SurrogateNet& s, int cap) {
  auto al = [&](void** p, size_t bytes) -> cudaError_t {
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e == cudaSuccess) s.allocs.push_back(*p);
    return e;
  };
  const size_t din = s.din, dh = s.dh, dout = s.dout;
  s.off[0] = 0;
  s.off[1] = s.off[0] + dh * din;
  s.off[2] = s.off[1] + dh;
  s.off[3] = s.off[2] + dh * dh;
  s.off[4] = s.off[3] + dh;
  s.off[5] = s.off[4] + dout * dh;
  s.np = s.off[5] + dout;
  SG_CK(al((void**)&s.P, 4 * s.np));
  SG_CK(al((void**)&s.G, 4 * s.np));
  SG_CK(al((void**)&s.M, 4 * s.np));
  SG_CK(al((void**)&s.V, 4 * s.np));
  const size_t wn[3] = {dh * din, dh * dh, dout * dh};
  for (int l = 0; l < 3; ++l) {
    SG_CK(al((void**)&s.Wb[l], 2 * wn[l]));
    SG_CK(al((void**)&s.WbT[l], 2 * wn[l]));
  }
  SG_CK(al((void**)&s.Lcat, 4 * 2 * dout * din));
  SG_CK(al((void**)&s.mu_x, 4 * din));
  SG_CK(al((void**)&s.sd_x, 4 * din));
  SG_CK(al((void**)&s.mu_y, 4 * dout));
  SG_CK(al((void**)&s.sd_y, 4 * dout));
  s.cap = cap;
  const size_t B = cap;
  SG_CK(al((void**)&s.xf, 4 * B * din));
  SG_CK(al((void**)&s.xb, 2 * B * din));
  SG_CK(al((void**)&s.xbT, 2 * B * din));
  for (int l = 0; l < 2; ++l) {
    SG_CK(al((void**)&s.hpre[l], 4 * B * dh));
    SG_CK(al((void**)&s.hb[l], 2 * B * dh));
    SG_CK(al((void**)&s.hbT[l], 2 * B * dh));
  }
  SG_CK(al((void**)&s.yhat, 4 * B * dout));
  SG_CK(al((void**)&s.tgt, 4 * B * dout));
  SG_CK(al((void**)&s.dy, 4 * B * (dout > dh ? dout : dh)));
  SG_CK(al((void**)&s.dyb, 2 * B * dout));
  SG_CK(al((void**)&s.dybT, 2 * B * dout));
  SG_CK(al((void**)&s.dhid, 4 * B * dh));
  SG_CK(al((void**)&s.dhb, 2 * B * dh));
  SG_CK(al((void**)&s.dhbT, 2 * B * dh));
  SG_CK(al((void**)&s.ylin, 4 * B * 2 * dout));
  SG_CK(al((void**)&s.feat, 4 * B * din));
  SG_CK(al((void**)&s.amp, 4 * B));
  SG_CK(al((void**)&s.loss, 4));
  s.ws_floats = 4ll << 20;
  SG_CK(al((void**)&s.ws, 4 * (size_t)s.ws_floats));
  // identity normalisation and zero linear part until set
  std::vector<float> one(din > dout ? din : dout, 1.f), zero(din > dout ? din : dout, 0.f);
  SG_CK(cudaMemcpy(s.mu_x, zero.data(), 4 * din, cudaMemcpyHostToDevice));
  SG_CK(cudaMemcpy(s.sd_x, one.data(), 4 * din, cudaMemcpyHostToDevice));
  SG_CK(cudaMemcpy(s.mu_y, zero.data(), 4 * dout, cudaMemcpyHostToDevice));
  SG_CK(cudaMemcpy(s.sd_y, one.data(), 4 * dout, cudaMemcpyHostToDevice));
  SG_CK(cudaMemset(s.Lcat, 0, 4 * 2 * dout * din));
  SG_CK(cudaMemset(s.M, 0, 4 * s.np));
  SG_CK(cudaMemset(s.V, 0, 4 * s.np));
  return cudaSuccess;
}

void sur_free(SurrogateNet& s) {
  for (void* p : s.allocs) cudaFree(p);
  s.allocs.clear();
}

cudaError_t sur_init_params(SurrogateNet& s, unsigned long long seed, cudaStream_t st) {
  // W ~ N(0, 1/fan_in) (last layer scaled by 0.1), biases zero
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  std::vector<float> h(s.np, 0.f);
  const int fin[3] = {s.din, s.dh, s.dh};
  const size_t wn[3] = {(size_t)s.dh * s.din, (size_t)s.dh * s.dh, (size_t)s.dout * s.dh};
  for (int l = 0; l < 3; ++l) {
    const float sc = (l == 2 ? 0.1f : 1.f) / std::sqrt((float)fin[l]);
    for (size_t q = 0; q < wn[l]; ++q) h[s.off[2 * l] + q] = sc * nd(rng);
  }
  SG_CK(cudaMemcpyAsync(s.P, h.data(), 4 * s.np, cudaMemcpyHostToDevice, st));
  SG_CK(cudaStreamSynchronize(st));
  SG_CK(cudaMemsetAsync(s.M, 0, 4 * s.np, st));
  SG_CK(cudaMemsetAsync(s.V, 0, 4 * s.np, st));
  s.adam_t = 0;
  return sur_refresh_bf16(s, st);
}

cudaError_t sur_refresh_bf16(SurrogateNet& s, cudaStream_t st) {
  const int rows[3] = {s.dh, s.dh, s.dout}, cols[3] = {s.din, s.dh, s.dh};
  for (int l = 0; l < 3; ++l) SG_CK(cvt_pair(s.P + s.off[2 * l], rows[l], cols[l], s.Wb[l], s.WbT[l], st));
  return cudaSuccess;
}

cudaError_t sur_normalise(SurrogateNet& s, const float* F, const int* rows, int B, cudaStream_t st) {
  const long long n = (long long)B * s.din;
  normalise_kernel<<<blocks(n), 256, 0, st>>>(F, rows, B, s.din, s.mu_x, s.sd_x, s.xf);
  SG_CK(cudaGetLastError());
  return cvt_pair(s.xf, B, s.din, s.xb, s.xbT, st);
}

cudaError_t sur_forward(SurrogateNet& s, int B, int* d_err, cudaStream_t st) {
  const __nv_bfloat16* in = s.xb;
  int k = s.din;
  for (int l = 0; l < 2; ++l) {
    GemmArgs g;
    g.ws = s.ws; g.ws_floats = s.ws_floats;
    g.M = B; g.N = s.dh; g.K = k;
    g.A = in; g.lda = k; g.B = s.Wb[l]; g.ldb = k;
    g.bias = s.P + s.off[2 * l + 1]; g.gelu = 1;
    g.Cpre = s.hpre[l]; g.ldpre = s.dh;
    g.Cb = s.hb[l]; g.ldcb = s.dh;
    g.CbT = s.hbT[l]; g.ldcbt = B;
    SG_CK(launch_gemm(g, d_err, st));
    in = s.hb[l];
    k = s.dh;
  }
  GemmArgs g;
  g.ws = s.ws; g.ws_floats = s.ws_floats;
  g.M = B; g.N = s.dout; g.K = s.dh;
  g.A = s.hb[1]; g.lda = s.dh; g.B = s.Wb[2]; g.ldb = s.dh;
  g.bias = s.P + s.off[5];
  g.Cf = s.yhat; g.ldc = s.dout;
  return launch_gemm(g, d_err, st);
}

cudaError_t sur_backward(SurrogateNet& s, int B, int* d_err, cudaStream_t st) {
  if (B % 64) return cudaErrorInvalidValue;  // the batch is the contraction dimension of dW
  const long long ny = (long long)B * s.dout, nh = (long long)B * s.dh;
  loss_grad_kernel<<<256, 256, 0, st>>>(s.yhat, s.tgt, ny, 1.f / (float)ny, s.dy, s.loss);
  SG_CK(cudaGetLastError());
  SG_CK(cvt_pair(s.dy, B, s.dout, s.dyb, s.dybT, st));
  // layer 3: dW3 = dy^T h2, db3 = colsum(dy), dh2 = dy W3
  {
    GemmArgs g;
    g.ws = s.ws; g.ws_floats = s.ws_floats;
    g.M = s.dout; g.N = s.dh; g.K = B;
    g.A = s.dybT; g.lda = B; g.B = s.hbT[1]; g.ldb = B;
    g.Cf = s.G + s.off[4]; g.ldc = s.dh;
    SG_CK(launch_gemm(g, d_err, st));
    colsum_kernel<<<blocks(s.dout), 256, 0, st>>>(s.dy, B, s.dout, s.G + s.off[5]);
    SG_CK(cudaGetLastError());
    GemmArgs d;
    d.ws = s.ws; d.ws_floats = s.ws_floats;
    d.M = B; d.N = s.dh; d.K = s.dout;
    d.A = s.dyb; d.lda = s.dout; d.B = s.WbT[2]; d.ldb = s.dout;
    d.Cf = s.dhid; d.ldc = s.dh;
    SG_CK(launch_gemm(d, d_err, st));
  }
  // layers 2 and 1
  for (int l = 1; l >= 0; --l) {
    gelu_back_kernel<<<blocks(nh), 256, 0, st>>>(s.dhid, s.hpre[l], nh);
    SG_CK(cudaGetLastError());
    SG_CK(cvt_pair(s.dhid, B, s.dh, s.dhb, s.dhbT, st));
    const int kin = l == 0 ? s.din : s.dh;
    const __nv_bfloat16* inT = l == 0 ? s.xbT : s.hbT[0];
    GemmArgs g;
    g.ws = s.ws; g.ws_floats = s.ws_floats;
    g.M = s.dh; g.N = kin; g.K = B;
    g.A = s.dhbT; g.lda = B; g.B = inT; g.ldb = B;
    g.Cf = s.G + s.off[2 * l]; g.ldc = kin;
    SG_CK(launch_gemm(g, d_err, st));
    colsum_kernel<<<blocks(s.dh), 256, 0, st>>>(s.dhid, B, s.dh, s.G + s.off[2 * l + 1]);
    SG_CK(cudaGetLastError());
    if (l == 1) {  // dh1 = dpre2 W2 (the input gradient of layer 1 is not needed)
      GemmArgs d;
      d.ws = s.ws; d.ws_floats = s.ws_floats;
      d.M = B; d.N = s.dh; d.K = s.dh;
      d.A = s.dhb; d.lda = s.dh; d.B = s.WbT[1]; d.ldb = s.dh;
      d.Cf = s.dhid; d.ldc = s.dh;  // A is the bf16 copy, so dhid can be overwritten
      SG_CK(launch_gemm(d, d_err, st));
    }
  }
  return cudaSuccess;
}

cudaError_t sur_adam(SurrogateNet& s, float lr, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  s.adam_t += 1;
  const float c1 = 1.f / (1.f - std::pow(b1, (float)s.adam_t)), c2 = 1.f / (1.f - std::pow(b2, (float)s.adam_t));
  adam_kernel<<<blocks((long long)s.np), 256, 0, st>>>(s.P, s.G, s.M, s.V, (long long)s.np, lr, b1, b2, c1, c2, eps);
  SG_CK(cudaGetLastError());
  return sur_refresh_bf16(s, st);
}

cudaError_t sur_linear(SurrogateNet& s, const float* X, int B, float* ylin_out, int* d_err, cudaStream_t st) {
  GemmArgs g;
  g.ws = s.ws; g.ws_floats = s.ws_floats;
  g.M = B; g.N = 2 * s.dout; g.K = s.din; g.split = 1;
  g.A = X; g.lda = s.din; g.B = s.Lcat; g.ldb = s.din;
  g.Cf = s.ylin; g.ldc = 2 * s.dout;
  SG_CK(launch_gemm(g, d_err, st));
  linear_combine_kernel<<<blocks((long long)B * s.dout), 256, 0, st>>>(s.ylin, X, B, s.din, s.dout, ylin_out);
  return cudaGetLastError();
}

cudaError_t sur_combine(SurrogateNet& s, const float* ylin, const float* yhat, const float* amp, int B,
                        int use_linear, int use_mlp, float* y, cudaStream_t st) {
  const long long n = (long long)B * s.dout;
  combine_kernel<<<blocks(n), 256, 0, st>>>(ylin, yhat, amp, n, s.dout, s.mu_y, s.sd_y, use_linear, use_mlp, y);
  return cudaGetLastError();
}

cudaError_t sur_features(const float* X, int B, int din, float* F, float* amp, cudaStream_t st) {
  if (B <= 0) return cudaSuccess;
  features_kernel<<<B, 128, 0, st>>>(X, din, F, amp);
  return cudaGetLastError();
}

}  // namespace sg
