// sg_surrogate.h -- the learned membrane-force surrogate (internal).
//
// Per capsule of SH degree 15 the surrogate maps the displacement
// coefficients (3 x 256 SPHEREPACK coefficients of X - centroid - sphere,
// divided by R) to the force coefficients that the plain model's force filter
// produces (3 x 256, times R / Gs):
//   y = (L0 + C L1) x + a^2 (S_y MLP((phi(x) - mu_x) / S_x) + mu_y)
// L0 + C L1 is the exact linear response of the Skalak membrane about the
// sphere (the force is affine in C: W2 = Gs/2 (C I2 - 1), membmodel.c:81-99)
// applied in BF16x3 on the tensor cores; the MLP 768 -> 1024 -> 1024 -> 768
// (GELU, bf16 weights, FP32 accumulation) learns the nonlinear remainder,
// which is O(a^2) in the displacement amplitude a = |x| (the norm over the
// displacement slots).  Its input phi(x) is scale free: the direction x / a
// in the displacement slots, C in slot 0 and log a in slot 256.
// The three l = 0 slots (0, 256, 512: translations, which the force ignores)
// carry C, log a and 0 in the network input; in x, slot 0 carries C and the
// other two are zero.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <vector>

namespace sg {

constexpr int SUR_N = 16;                   // SH degree 15: N = L + 1
constexpr int SUR_DIN = 3 * SUR_N * SUR_N;  // 768
constexpr int SUR_DH = 1024;
constexpr int SUR_DOUT = 3 * SUR_N * SUR_N;  // 768

struct SurrogateNet {
  int din = SUR_DIN, dh = SUR_DH, dout = SUR_DOUT;
  // FP32 parameters, gradients and Adam moments, one block each, in the
  // order W1 [dh][din], b1, W2 [dh][dh], b2, W3 [dout][dh], b3
  float* P = nullptr;
  float* G = nullptr;
  float* M = nullptr;
  float* V = nullptr;
  size_t np = 0;
  size_t off[6] = {};
  // bf16 weights [out][in] (forward) and transposed [in][out] (backward)
  __nv_bfloat16* Wb[3] = {};
  __nv_bfloat16* WbT[3] = {};
  // exact linear response [2 dout][din] (rows 0..dout-1: L0, then L1)
  float* Lcat = nullptr;
  // normalisation of inputs and of the residual targets
  float* mu_x = nullptr;
  float* sd_x = nullptr;
  float* mu_y = nullptr;
  float* sd_y = nullptr;
  long long adam_t = 0;
  bool trained = false;
  // batch work buffers (capacity cap rows)
  int cap = 0;
  float* xf = nullptr;         // [B][din] normalised input, FP32
  __nv_bfloat16* xb = nullptr;  // [B][din]
  __nv_bfloat16* xbT = nullptr; // [din][B]
  float* hpre[2] = {};         // [B][dh]
  __nv_bfloat16* hb[2] = {};
  __nv_bfloat16* hbT[2] = {};
  float* yhat = nullptr;       // [B][dout]
  float* tgt = nullptr;        // [B][dout]
  float* dy = nullptr;         // [B][dout]   (reused as [B][dh] scratch)
  __nv_bfloat16* dyb = nullptr;
  __nv_bfloat16* dybT = nullptr;
  float* dhid = nullptr;       // [B][dh] gradient of a hidden layer
  __nv_bfloat16* dhb = nullptr;
  __nv_bfloat16* dhbT = nullptr;
  float* ylin = nullptr;       // [B][2 dout]
  float* feat = nullptr;       // [B][din] scale-free features phi(x)
  float* amp = nullptr;        // [B] displacement amplitude a
  float* loss = nullptr;       // [1]
  float* ws = nullptr;         // split-K workspace of the dense products
  long long ws_floats = 0;
  std::vector<void*> allocs;
};

// Allocation, initialisation, and release (host side, stream-ordered work on st).
cudaError_t sur_alloc(SurrogateNet& s, int batch_cap);
void sur_free(SurrogateNet& s);
cudaError_t sur_init_params(SurrogateNet& s, unsigned long long seed, cudaStream_t st);
cudaError_t sur_refresh_bf16(SurrogateNet& s, cudaStream_t st);

// One forward pass on B rows already normalised in s.xf (B <= cap):
// yhat = MLP(x) (no output de-normalisation).
cudaError_t sur_forward(SurrogateNet& s, int B, int* d_err, cudaStream_t st);
// Backward pass for the loss mean((yhat - tgt)^2) and gradients into s.G;
// the loss (sum of squares / (B dout)) is added to *s.loss.
cudaError_t sur_backward(SurrogateNet& s, int B, int* d_err, cudaStream_t st);
cudaError_t sur_adam(SurrogateNet& s, float lr, cudaStream_t st);

// Kernels on raw coefficient rows (X [n][din] with C in slot 0).
// features: F[b] = phi(X[b]) and amp[b] = a (F may alias X)
cudaError_t sur_features(const float* X, int B, int din, float* F, float* amp, cudaStream_t st);
// gathered rows of features, normalised into s.xf / s.xb / s.xbT
cudaError_t sur_normalise(SurrogateNet& s, const float* F, const int* rows, int B, cudaStream_t st);
// ylin[b][o] = (L0 x_b)[o] + C_b (L1 x_b)[o] for B rows of X (rows may be null)
cudaError_t sur_linear(SurrogateNet& s, const float* X, int B, float* ylin_out, int* d_err, cudaStream_t st);
// y = ylin + amp^2 (yhat * sd_y + mu_y) (linear part optional, MLP part optional)
cudaError_t sur_combine(SurrogateNet& s, const float* ylin, const float* yhat, const float* amp, int B,
                        int use_linear, int use_mlp, float* y, cudaStream_t st);

}  // namespace sg
