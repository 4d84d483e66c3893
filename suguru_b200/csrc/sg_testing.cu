// sg_testing.cu -- test hooks (include/sg_testing.h): run one batched
// Legendre contraction through the tensor-core or the CUDA-core kernel on
// caller data, so that the tests can check the UMMA operand layout, the
// BF16x3 and BF16x6 splits, the 64- and 128-row tiles and the epilogue element
// by element against numpy.
#include <cstring>
#include <vector>

#include "sg_kernels.h"
#include "sg_testing.h"

using namespace sg;

extern "C" int sg_test_legendre(int tensor_cores, int M, int Q, int J, int K, int tri, const double* B,
                                const float* A, float* D) {
  if (M < 1 || Q < 1 || J < 1 || K < 1 || J > 256 || K > 256 || !B || !A || !D) return 5;
  // tensor_cores: 0 CUDA cores; 1 or 3 BF16x3, 6 BF16x6 on 128-row tiles; +100 for 64-row tiles
  const int tm = tensor_cores >= 100 ? 64 : 128, mode = tensor_cores % 100;
  if (mode != 0 && mode != 1 && mode != 3 && mode != 6) return 5;
  if (tensor_cores >= 100 && mode == 0) return 5;
  const int terms = mode == 6 ? 6 : 3;
  const int Jp = (J + 15) / 16 * 16, Kp = (K + 15) / 16 * 16;
  // problem: A[m][q][k] rows, B[m][j][k], D[m][q][j]
  LegProblem p{};
  p.sAc = (long long)K;  // capsule index = q (one row per capsule)
  p.sAr = 0;
  p.sAm = (long long)Q * K;
  p.sBm = (long long)J * K;
  p.sDc = J;
  p.sDr = 0;
  p.sDm = (long long)Q * J;
  p.rpc = 1;
  p.Q = Q;
  p.M = M;
  p.J = J;
  p.K = K;
  p.tri = tri;
  p.Jp = Jp;
  p.Kp = Kp;
  p.next[0] = p.next[1] = -1;
  p.terms = terms;
  p.sBimg = 3LL * Jp * Kp;
  std::vector<uint16_t> img((size_t)M * p.sBimg);
  host_umma_image(B, p.sBm, M, J, K, Jp, Kp, img.data());
  std::vector<float> Bf((size_t)M * J * K);
  for (size_t i = 0; i < Bf.size(); ++i) Bf[i] = (float)B[i];
  std::vector<LegWork> work;
  const int qt = tensor_cores ? tm : 32;
  for (int m = 0; m < M; ++m)
    for (int q0 = 0; q0 < Q; q0 += qt) work.push_back(LegWork{0, m, q0});
  void *dA = nullptr, *dB = nullptr, *dD = nullptr, *dI = nullptr, *dP = nullptr, *dW = nullptr, *dE = nullptr;
  const size_t na = (size_t)M * Q * K, nd = (size_t)M * Q * J;
  int rc = 0;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == 0) rc = 2;
    return rc == 0;
  };
  if (ok(cudaMalloc(&dA, 4 * na)) && ok(cudaMalloc(&dB, 4 * Bf.size())) && ok(cudaMalloc(&dD, 4 * nd)) &&
      ok(cudaMalloc(&dI, 2 * img.size())) && ok(cudaMalloc(&dP, sizeof(LegProblem))) &&
      ok(cudaMalloc(&dW, sizeof(LegWork) * work.size())) && ok(cudaMalloc(&dE, sizeof(int)))) {
    p.A = dA;
    p.B = dB;
    p.D = dD;
    p.Bimg = dI;
    p.vecA = (K % 8 == 0) ? 1 : 0;
    p.vecD = (J % 4 == 0) ? 1 : 0;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (ok(cudaMemcpy(dA, A, 4 * na, cudaMemcpyHostToDevice)) &&
        ok(cudaMemcpy(dB, Bf.data(), 4 * Bf.size(), cudaMemcpyHostToDevice)) &&
        ok(cudaMemcpy(dI, img.data(), 2 * img.size(), cudaMemcpyHostToDevice)) &&
        ok(cudaMemcpy(dP, &p, sizeof(p), cudaMemcpyHostToDevice)) &&
        ok(cudaMemcpy(dW, work.data(), sizeof(LegWork) * work.size(), cudaMemcpyHostToDevice)) &&
        ok(cudaMemset(dE, 0, sizeof(int))) && ok(cudaMemset(dD, 0xff, 4 * nd))) {
      if (tensor_cores) {
        LegLevels lv{};
        lv.jp[0] = Jp;
        lv.kp[0] = Kp;
        lv.a_kp = Kp;
        ok(launch_legendre_mma((const LegProblem*)dP, (const LegWork*)dW, (int)work.size(), lv, terms == 6 ? 3 : 2,
                               tm, (int*)dE, sms, 0));
      } else {
        ok(launch_legendre<float>((const LegProblem*)dP, (const LegWork*)dW, (int)work.size(), J, K, 0));
      }
      int err = 0;
      if (ok(cudaDeviceSynchronize()) && ok(cudaMemcpy(&err, dE, sizeof(int), cudaMemcpyDeviceToHost)) &&
          ok(cudaMemcpy(D, dD, 4 * nd, cudaMemcpyDeviceToHost)))
        if (err) rc = 3;
    }
  }
  for (void* q : {dA, dB, dD, dI, dP, dW, dE})
    if (q) cudaFree(q);
  return rc;
}

extern "C" int sg_test_gemm(int split, int M, int N, int K, const void* A, const void* B, const float* bias,
                            int gelu, float alpha, float* C, float* Cpre, unsigned short* Cb, unsigned short* CbT,
                            int splitk) {
  if (M < 1 || N < 1 || K < 0 || K % 64 || !A || !B || !C) return 5;
  const size_t es = split ? 4 : 2;
  void *dA = nullptr, *dB = nullptr, *dC = nullptr, *dP = nullptr, *dCb = nullptr, *dCbT = nullptr, *dbias = nullptr,
       *dE = nullptr;
  int rc = 0;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == 0) rc = 2;
    return rc == 0;
  };
  const size_t nc = (size_t)M * N;
  if (ok(cudaMalloc(&dA, es * M * (size_t)K + 16)) && ok(cudaMalloc(&dB, es * N * (size_t)K + 16)) &&
      ok(cudaMalloc(&dC, 4 * nc)) && ok(cudaMalloc(&dP, 4 * nc)) && ok(cudaMalloc(&dCb, 2 * nc)) &&
      ok(cudaMalloc(&dCbT, 2 * nc)) && ok(cudaMalloc(&dbias, 4 * (size_t)N)) && ok(cudaMalloc(&dE, sizeof(int))) &&
      ok(cudaMemcpy(dA, A, es * M * (size_t)K, cudaMemcpyHostToDevice)) &&
      ok(cudaMemcpy(dB, B, es * N * (size_t)K, cudaMemcpyHostToDevice)) && ok(cudaMemset(dE, 0, sizeof(int))) &&
      ok(cudaMemset(dC, 0xff, 4 * nc)) && (!bias || ok(cudaMemcpy(dbias, bias, 4 * (size_t)N, cudaMemcpyHostToDevice)))) {
    GemmArgs g;
    g.M = M; g.N = N; g.K = K; g.split = split;
    g.A = dA; g.lda = K; g.B = dB; g.ldb = K;
    g.alpha = alpha; g.bias = bias ? (const float*)dbias : nullptr; g.gelu = gelu;
    g.Cf = (float*)dC; g.ldc = N;
    g.Cpre = Cpre ? (float*)dP : nullptr; g.ldpre = N;
    g.Cb = Cb ? (__nv_bfloat16*)dCb : nullptr; g.ldcb = N;
    g.CbT = CbT ? (__nv_bfloat16*)dCbT : nullptr; g.ldcbt = M;
    float* ws = nullptr;
    if (splitk) {
      g.ws_floats = 16ll * M * N;
      ok(cudaMalloc(&ws, 4 * (size_t)g.ws_floats));
      g.ws = ws;
    }
    int err = 0;
    if (ok(launch_gemm(g, (int*)dE, 0)) && ok(cudaDeviceSynchronize()) &&
        ok(cudaMemcpy(&err, dE, sizeof(int), cudaMemcpyDeviceToHost)) &&
        ok(cudaMemcpy(C, dC, 4 * nc, cudaMemcpyDeviceToHost)) &&
        (!Cpre || ok(cudaMemcpy(Cpre, dP, 4 * nc, cudaMemcpyDeviceToHost))) &&
        (!Cb || ok(cudaMemcpy(Cb, dCb, 2 * nc, cudaMemcpyDeviceToHost))) &&
        (!CbT || ok(cudaMemcpy(CbT, dCbT, 2 * nc, cudaMemcpyDeviceToHost))))
      if (err) rc = 3;
    if (ws) cudaFree(ws);
  }
  for (void* q : {dA, dB, dC, dP, dCb, dCbT, dbias, dE})
    if (q) cudaFree(q);
  return rc;
}

#include "sg_surrogate.h"

extern "C" int sg_test_mlp_grad(int din, int dh, int dout, int B, const float* params, const float* X,
                                const float* T, float* loss, float* grads) {
  if (din < 64 || dh < 64 || dout < 64 || din % 64 || dh % 64 || dout % 64 || B < 64 || B % 64 || !params || !X ||
      !T || !loss || !grads)
    return 5;
  SurrogateNet s;
  s.din = din;
  s.dh = dh;
  s.dout = dout;
  int rc = 0;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == 0) rc = 2;
    return rc == 0;
  };
  int* dE = nullptr;
  float* dX = nullptr;
  if (ok(sur_alloc(s, B)) && ok(cudaMalloc(&dE, sizeof(int))) && ok(cudaMemset(dE, 0, sizeof(int))) &&
      ok(cudaMalloc(&dX, 4 * (size_t)B * din)) &&
      ok(cudaMemcpy(dX, X, 4 * (size_t)B * din, cudaMemcpyHostToDevice)) &&
      ok(cudaMemcpy(s.P, params, 4 * s.np, cudaMemcpyHostToDevice)) &&
      ok(cudaMemcpy(s.tgt, T, 4 * (size_t)B * dout, cudaMemcpyHostToDevice)) && ok(cudaMemset(s.loss, 0, 4)) &&
      ok(sur_refresh_bf16(s, 0)) && ok(sur_normalise(s, dX, nullptr, B, 0)) && ok(sur_forward(s, B, dE, 0)) &&
      ok(sur_backward(s, B, dE, 0)) && ok(cudaDeviceSynchronize()) &&
      ok(cudaMemcpy(grads, s.G, 4 * s.np, cudaMemcpyDeviceToHost)) &&
      ok(cudaMemcpy(loss, s.loss, 4, cudaMemcpyDeviceToHost))) {
    int err = 0;
    if (ok(cudaMemcpy(&err, dE, sizeof(int), cudaMemcpyDeviceToHost)) && err) rc = 3;
  }
  if (dE) cudaFree(dE);
  if (dX) cudaFree(dX);
  sur_free(s);
  return rc;
}
