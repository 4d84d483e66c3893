// sg_mechanics.cuh -- pointwise geometry and membrane mechanics of one
// surface point (device code shared by the spectral force kernels).
//
// sph1.f90:581-651 (unit normal and its derivatives), sph.f90:442-476
// (curvature), sph1.f90:197-297 with co2contra (capsulesolid.f90:106-146:
// contravariant basis and derivatives), sph.f90:735-893 (Christoffel
// symbols), sph.f90:896-961 (metric tensors and derivatives);
// cal_spectral_force's equilibrium (sph.f90:1668-1715) with
// cal_Js_I1_I2_deri (sph.f90:1115-1156), the membrane laws of membmodel.c
// and calculate_cauchy_tensor_deri (sph.f90:1179-1234).  Same operation
// order as the reference.
#pragma once
#include "sg_common.cuh"

namespace sg {

// Division in the pointwise geometry and mechanics: the FP32 path uses the
// fast reciprocal-based division (2 ulp), the FP64 path the IEEE division.
template <class T>
__device__ __forceinline__ T fdiv(T a, T b);
template <>
__device__ __forceinline__ float fdiv<float>(float a, float b) {
  return __fdividef(a, b);
}
template <>
__device__ __forceinline__ double fdiv<double>(double a, double b) {
  return a / b;
}

// ------------------------------------------------- geometry + mechanics ---
template <class T>
struct Geo {
  T a1[3], a2[3], d11[3], d12[3], d22[3];
  T n[3];
  T c1[3], c2[3];
  T cat[3], catd1[2][3], conat[3], conatd1[2][3], bcur[3], chf[8];
  // derivatives of the unit normal and of the contravariant basis along
  // xi^al (cderi3, conderi1, conderi2 of the reference; the bending terms read
  // them, the plain force leaves them unused)
  T nde[2][3], cdc1[2][3], cdc2[2][3];
};

// sph1.f90:581-651 (normal), sph.f90:442-476 (curvature), sph1.f90:197-297
// with co2contra (capsulesolid.f90:106-146), sph.f90:735-893 (christof),
// sph.f90:896-961 (metrics).  Same operation order as the reference.
template <class T>
__device__ __forceinline__ void geometry(Geo<T>& G) {
  const T* cd1[2] = {G.d11, G.d12};
  const T* cd2[2] = {G.d12, G.d22};
  T cc[3];
  cross3(G.a1, G.a2, cc);
  const T sm = sqrt(cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2]);
  for (int c = 0; c < 3; ++c) G.n[c] = fdiv(cc[c], sm);
  T (&nde)[2][3] = G.nde;
#pragma unroll
  for (int al = 0; al < 2; ++al) {
    T x1[3], x2[3], dc[3];
    cross3(cd1[al], G.a2, x1);
    cross3(G.a1, cd2[al], x2);
    for (int c = 0; c < 3; ++c) dc[c] = x1[c] + x2[c];
    const T tmp = fdiv(dot3(cc, dc), sqrt(cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2]));
    for (int c = 0; c < 3; ++c) nde[al][c] = fdiv(T(1), sm) * (x1[c] + x2[c] - tmp * G.n[c]);
  }
  G.bcur[0] = dot3(G.n, G.d11);
  G.bcur[1] = dot3(G.n, G.d22);
  G.bcur[2] = dot3(G.n, G.d12);
  T a2n[3], na1[3];
  cross3(G.a2, G.n, a2n);
  cross3(G.n, G.a1, na1);
  const T hyb1 = dot3(G.a1, a2n), hyb2 = dot3(G.a2, na1);
  for (int c = 0; c < 3; ++c) {
    G.c1[c] = fdiv(a2n[c], hyb1);
    G.c2[c] = fdiv(na1[c], hyb2);
  }
  const T g = hyb1;
  T (&cdc1)[2][3] = G.cdc1;
  T (&cdc2)[2][3] = G.cdc2;
#pragma unroll
  for (int al = 0; al < 2; ++al) {
    T a2de_n3[3], a2_n3de[3], n3de_a1[3], n3_a1de[3], vt[3];
    cross3(cd2[al], G.n, a2de_n3);
    cross3(G.a2, nde[al], a2_n3de);
    cross3(nde[al], G.a1, n3de_a1);
    cross3(G.n, cd1[al], n3_a1de);
    for (int c = 0; c < 3; ++c) vt[c] = a2de_n3[c] + a2_n3de[c];
    const T gde = dot3(cd1[al], a2n) + dot3(G.a1, vt);
    for (int c = 0; c < 3; ++c) {
      cdc1[al][c] = fdiv(T(1), g) * (-gde * G.c1[c] + a2de_n3[c] + a2_n3de[c]);
      cdc2[al][c] = fdiv(T(1), g) * (-gde * G.c2[c] + n3de_a1[c] + n3_a1de[c]);
    }
  }
  // christof(gamma,beta,alpha) at [(gamma-1) + 2(beta-1) + 4(alpha-1)]
  G.chf[0 + 0 + 0] = dot3(G.d11, G.c1);  // (1,1,1)
  G.chf[1 + 0 + 0] = dot3(G.d12, G.c1);  // (2,1,1)
  G.chf[0 + 2 + 0] = dot3(G.d11, G.c2);  // (1,2,1)
  G.chf[1 + 2 + 0] = dot3(G.d12, G.c2);  // (2,2,1)
  G.chf[1 + 0 + 4] = dot3(G.d22, G.c1);  // (2,1,2)
  G.chf[1 + 2 + 4] = dot3(G.d22, G.c2);  // (2,2,2)
  G.chf[0 + 0 + 4] = G.chf[1];           // (1,1,2) = (2,1,1)
  G.chf[0 + 2 + 4] = G.chf[3];           // (1,2,2) = (2,2,1)
  G.cat[0] = G.a1[0] * G.a1[0] + G.a1[1] * G.a1[1] + G.a1[2] * G.a1[2];
  G.cat[1] = G.a2[0] * G.a2[0] + G.a2[1] * G.a2[1] + G.a2[2] * G.a2[2];
  G.cat[2] = dot3(G.a1, G.a2);
  G.conat[0] = G.c1[0] * G.c1[0] + G.c1[1] * G.c1[1] + G.c1[2] * G.c1[2];
  G.conat[1] = G.c2[0] * G.c2[0] + G.c2[1] * G.c2[1] + G.c2[2] * G.c2[2];
  G.conat[2] = dot3(G.c1, G.c2);
#pragma unroll
  for (int al = 0; al < 2; ++al) {
    G.catd1[al][0] = T(2) * dot3(G.a1, cd1[al]);
    G.catd1[al][1] = T(2) * dot3(G.a2, cd2[al]);
    G.catd1[al][2] = dot3(G.a1, cd2[al]) + dot3(G.a2, cd1[al]);
    G.conatd1[al][0] = T(2) * dot3(G.c1, cdc1[al]);
    G.conatd1[al][1] = T(2) * dot3(G.c2, cdc2[al]);
    G.conatd1[al][2] = dot3(G.c1, cdc2[al]) + dot3(G.c2, cdc1[al]);
  }
}

// sph.f90:1668-1715 with cal_Js_I1_I2_deri (sph.f90:1115-1156), the Skalak
// law of membmodel.c:81-99 and calculate_cauchy_tensor_deri (sph.f90:1179-1234).
// A: reference contravariant metric (11,22,12); Ad[al]: its derivatives.
// bq: the bending terms of ibend = 1 (sph.f90:1705-1709) or nullptr:
// bq[0..3] = bcurmix(1,1), (2,1), (1,2), (2,2); bq[4..5] = Q(1), Q(2);
// bq[6] = Qcode.
template <class T>
__device__ __forceinline__ void mechanics(const Geo<T>& G, const T* A, const T (*Ad)[3], T hf, T csk, int law,
                                          T* f, const T* bq = nullptr) {
  const T A11 = A[0], A22 = A[1], A12 = A[2];
  const T c11 = G.cat[0], c22 = G.cat[1], c12 = G.cat[2];
  const T abs_conA = A11 * A22 - A12 * A12;
  const T abs_ca = c11 * c22 - c12 * c12;
  const T I1 = A11 * c11 + A22 * c22 + T(2) * A12 * c12 - T(2);
  const T I2 = abs_conA * abs_ca - T(1);
  const T Js = sqrt(T(1) + I2);
  T I1de[2], I2de[2], Jsde[2];
#pragma unroll
  for (int al = 0; al < 2; ++al) {
    const T Ad11 = Ad[al][0], Ad22 = Ad[al][1], Ad12 = Ad[al][2];
    const T cd11 = G.catd1[al][0], cd22 = G.catd1[al][1], cd12 = G.catd1[al][2];
    I1de[al] = Ad11 * c11 + A11 * cd11 + Ad22 * c22 + A22 * cd22 + T(2) * (Ad12 * c12 + A12 * cd12);
    const T abs_conAd = Ad11 * A22 + A11 * Ad22 - T(2) * A12 * Ad12;
    const T abs_cad = cd11 * c22 + c11 * cd22 - T(2) * c12 * cd12;
    I2de[al] = abs_conAd * abs_ca + abs_cad * abs_conA;
    Jsde[al] = fdiv(T(0.5), Js) * I2de[al];
  }
  // strain-energy derivatives: Skalak W1 = hf (1 + I1), W2 = hf (C I2 - 1)
  // (membmodel.c:81-99); neo-Hookean W1 = hf, W2 = -hf (I2 + 1)^-2
  // (membmodel.c:60-79, the reference's -DNONHOOK build)
  const bool nh = law == 1;
  const T iJ2 = fdiv(T(1), T(1) + I2);  // neo-Hookean: (I2 + 1)^-1
  const T W1 = nh ? hf : hf * (T(1) + I1);
  const T W2 = nh ? -hf * iJ2 * iJ2 : hf * (csk * I2 - T(1));
  const T coef1 = fdiv(T(2), Js) * W1, coef2 = T(2) * Js * W2;
  const T a11 = G.conat[0], a22 = G.conat[1], a12 = G.conat[2];
  const T T11 = coef1 * A11 + coef2 * a11;
  const T T22 = coef1 * A22 + coef2 * a22;
  const T T12 = coef1 * A12 + coef2 * a12;
  T Td11[2], Td22[2], Td12[2];
#pragma unroll
  for (int al = 0; al < 2; ++al) {
    const T W1de = nh ? T(0) : hf * I1de[al];
    const T W2de = nh ? (T(2) * hf) * (iJ2 * iJ2 * iJ2) * I2de[al] : csk * hf * I2de[al];
    const T v1 = fdiv(-T(2), Js * Js) * Jsde[al] * W1;
    const T v2 = fdiv(T(2), Js) * W1de;
    const T v3 = fdiv(T(2), Js) * W1;
    const T v4 = T(2) * Jsde[al] * W2;
    const T v5 = T(2) * Js * W2de;
    const T v6 = T(2) * Js * W2;
    Td11[al] = v1 * A11 + v2 * A11 + v3 * Ad[al][0] + v4 * a11 + v5 * a11 + v6 * G.conatd1[al][0];
    Td22[al] = v1 * A22 + v2 * A22 + v3 * Ad[al][1] + v4 * a22 + v5 * a22 + v6 * G.conatd1[al][1];
    Td12[al] = v1 * A12 + v2 * A12 + v3 * Ad[al][2] + v4 * a12 + v5 * a12 + v6 * G.conatd1[al][2];
  }
  const T* ch = G.chf;
  // ch index: (g,b,a) -> (g-1) + 2(b-1) + 4(a-1)
  const T c111 = ch[0], c211 = ch[1], c121 = ch[2], c221 = ch[3], c112 = ch[4], c212 = ch[5], c122 = ch[6],
          c222 = ch[7];
  const T q1 = Td11[0] + Td12[1] + c111 * T11 + c211 * T12 + c122 * T11 + c222 * T12 + c111 * T11 + c211 * T12 +
               c112 * T12 + c212 * T22;
  const T q2 = Td12[0] + Td22[1] + c111 * T12 + c211 * T22 + c122 * T12 + c222 * T22 + c121 * T11 + c221 * T12 +
               c122 * T12 + c222 * T22;
  T q3 = T11 * G.bcur[0] + T22 * G.bcur[1] + T(2) * T12 * G.bcur[2];
  T p1 = q1, p2 = q2;
  if (bq) {
    p1 = q1 - bq[0] * bq[4] - bq[1] * bq[5];
    p2 = q2 - bq[2] * bq[4] - bq[3] * bq[5];
    q3 = q3 + bq[6];
  }
  for (int c = 0; c < 3; ++c) f[c] = p1 * G.a1[c] + p2 * G.a2[c] + q3 * G.n[c];
}

}  // namespace sg
