// sg_bending.cu -- the bending terms of the membrane force (ibend = 1,
// param.f90:90-91) on the GPU.
//
// With bending, cal_spectral_force (sph.f90:1523-1755) also synthesises the
// third and fourth derivatives of the shape (cal_co_tang_basis2 with
// ibend = 1, sph3.f90:137-180), differentiates the curvature tensor twice
// (cal_curvature_derivative, sph.f90:479-731), the contravariant basis twice
// (cal_contra_second_derivative, sph1.f90:299-542), the Christoffel symbols
// once (cal_christof, sph.f90:802-890) and the contravariant metric twice
// (cal_contra_metric_second_deri, sph.f90:962-1111), forms the bending moment
// and its derivatives (cal_moment_deri, sph.f90:1236-1372), the transverse
// shear Q and its divergence (cal_Q, :1375-1424) and the mixed curvature
// (cal_bcurmix, :1427-1454), and adds them to the equilibrium
// (sph.f90:1705-1709).
//
// Here: a fourth Legendre synthesis problem per degree group (the third and
// fourth theta derivatives of the shape's series, one extra contraction launch
// after the analysis), and a membrane kernel that evaluates the whole chain per
// point.  The reference sphere's tensors (conAR .. BRd2 of sph.f90:153-161)
// enter analytically, as the plain force's reference metric does.  The
// kernel computes every capsule of the context (capsules with a zero bending
// modulus skip the bending terms), one point per thread.
#include <algorithm>
#include <vector>

#include "sg_ctx.h"
#include "sg_mechanics.cuh"

namespace sg {

namespace {

// The bending tensors of one point in the reference's index order (0-based):
// bd1[c][b][a] = d b_ab / d xi^c, bd2[d][c][b][a], cad2[l][lm][b][a] =
// d^2 a^ab / d xi^lm d xi^l, chd[l][lm][b][a] = d christof(lm,b,a) / d xi^l.
template <class T>
struct BendT {
  T bd1[2][2][2], bd2[2][2][2][2], cad2[2][2][2][2], chd[2][2][2][2];
};

template <class T>
__device__ __forceinline__ T d3(const T* u, const T* v) {
  return u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
}

// S[k] = x_ttt, x_ttp, x_tpp, x_ppp; Q4[k] = x_tttt, x_tttp, x_ttpp, x_tppp, x_pppp.
template <class T>
__device__ void bend_tensors(const Geo<T>& G, const T (*S)[3], const T (*Q4)[3], BendT<T>& B) {
  const T* x1[2] = {G.d11, G.d12};  // cderi1(:,al): d a1 / d xi^al
  const T* x2[2] = {G.d12, G.d22};  // cderi2(:,al)
  const T* nd[2] = {G.nde[0], G.nde[1]};
  const T* n = G.n;
  const T *c1 = G.c1, *c2 = G.c2;
  const T b11 = G.bcur[0], b22 = G.bcur[1], b12 = G.bcur[2];
  // ---- first derivatives of b_ab: (d/dxi^c)(x_ab . n) = x_abc . n + x_ab . n_c
  T(&D1)[2][2][2] = B.bd1;
  D1[0][0][0] = d3(S[0], n) + d3(x1[0], nd[0]);
  D1[1][0][0] = d3(S[1], n) + d3(x1[0], nd[1]);
  D1[0][1][1] = d3(S[2], n) + d3(x2[1], nd[0]);
  D1[1][1][1] = d3(S[3], n) + d3(x2[1], nd[1]);
  D1[0][0][1] = D1[0][1][0] = d3(S[1], n) + d3(x2[0], nd[0]);
  D1[1][0][1] = D1[1][1][0] = d3(S[2], n) + d3(x2[0], nd[1]);
  // second derivatives of the normal (Weingarten differentiated): n_tt, n_pp, n_tp
  T ns[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    ns[0][c] = -(D1[0][0][0] * c1[c] + D1[0][1][0] * c2[c] + b11 * G.cdc1[0][c] + b12 * G.cdc2[0][c]);
    ns[1][c] = -(D1[1][0][1] * c1[c] + D1[1][1][1] * c2[c] + b12 * G.cdc1[1][c] + b22 * G.cdc2[1][c]);
    ns[2][c] = -(D1[1][0][0] * c1[c] + D1[1][1][0] * c2[c] + b11 * G.cdc1[1][c] + b12 * G.cdc2[1][c]);
  }
  // ---- second derivatives of b_ab (product rule on x_ab . n)
  auto e2 = [&](const T* q, const T* s1, const T* m1, const T* s2, const T* m2, const T* x, const T* nn) {
    return d3(q, n) + d3(s1, m1) + d3(s2, m2) + d3(x, nn);
  };
  T(&D2)[2][2][2][2] = B.bd2;
  D2[0][0][0][0] = e2(Q4[0], S[0], nd[0], S[0], nd[0], x1[0], ns[0]);
  D2[1][0][0][0] = D2[0][1][0][0] = e2(Q4[1], S[0], nd[1], S[1], nd[0], x1[0], ns[2]);
  D2[1][1][0][0] = e2(Q4[2], S[1], nd[1], S[1], nd[1], x1[0], ns[1]);
  D2[0][0][1][1] = e2(Q4[2], S[2], nd[0], S[2], nd[0], x2[1], ns[0]);
  D2[1][0][1][1] = D2[0][1][1][1] = e2(Q4[3], S[2], nd[1], S[3], nd[0], x2[1], ns[2]);
  D2[1][1][1][1] = e2(Q4[4], S[3], nd[1], S[3], nd[1], x2[1], ns[1]);
  D2[0][0][1][0] = D2[0][0][0][1] = e2(Q4[1], S[1], nd[0], S[1], nd[0], x1[1], ns[0]);
  D2[1][0][1][0] = D2[0][1][1][0] = D2[1][0][0][1] = D2[0][1][0][1] =
      e2(Q4[2], S[1], nd[1], S[2], nd[0], x1[1], ns[2]);
  D2[1][1][1][0] = D2[1][1][0][1] = e2(Q4[3], S[2], nd[1], S[2], nd[1], x1[1], ns[1]);
  // ---- second derivatives of the contravariant basis a^1 = (a2 x n)/g,
  // a^2 = (n x a1)/g, g = a1 . (a2 x n), for the index pairs tt, pp, tp
  T cS[2][3][3];  // [vector][pair][c]
  {
    const T* a1 = G.a1;
    const T* a2 = G.a2;
    T a2n[3], na1[3], a2dn[2][3], a2nd[2][3], ndA1[2][3], nA1d[2][3];
    cross3(a2, n, a2n);
    cross3(n, a1, na1);
#pragma unroll
    for (int al = 0; al < 2; ++al) {
      cross3(x2[al], n, a2dn[al]);
      cross3(a2, nd[al], a2nd[al]);
      cross3(nd[al], a1, ndA1[al]);
      cross3(n, x1[al], nA1d[al]);
    }
    const T g = d3(a1, a2n);
    T gde[2];
#pragma unroll
    for (int al = 0; al < 2; ++al) {
      T vt[3];
      for (int c = 0; c < 3; ++c) vt[c] = a2dn[al][c] + a2nd[al][c];
      gde[al] = d3(x1[al], a2n) + d3(a1, vt);
    }
    // second derivatives of a1 and a2 for the pairs (tt, pp, tp)
    const T* a1S[3] = {S[0], S[2], S[1]};
    const T* a2S[3] = {S[1], S[3], S[2]};
    const int I[3] = {0, 1, 0}, J[3] = {0, 1, 1};
    const T gi1 = T(1) / g, gi2 = gi1 * gi1, gi3 = gi1 * gi2;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int i = I[k], j = J[k];
      T a2Sn[3], a2ns[3], a2dndij[3], a2dndji[3], nsA1[3], nA1S[3], ndA1dij[3], ndA1dji[3];
      cross3(a2S[k], n, a2Sn);
      cross3(a2, ns[k], a2ns);
      cross3(x2[i], nd[j], a2dndij);  // a2de_n3de(:,j,i) = a2_,i x n_,j
      cross3(x2[j], nd[i], a2dndji);
      cross3(ns[k], a1, nsA1);
      cross3(n, a1S[k], nA1S);
      cross3(nd[i], x1[j], ndA1dij);  // n3de_a1de(:,j,i) = n_,i x a1_,j
      cross3(nd[j], x1[i], ndA1dji);
      T w1[3], w2[3], v1[3], v2[3];
      for (int c = 0; c < 3; ++c) {
        w1[c] = a2Sn[c] + a2dndij[c] + a2dndji[c] + a2ns[c];
        w2[c] = nsA1[c] + ndA1dij[c] + ndA1dji[c] + nA1S[c];
        v1[c] = a2dn[i][c] + a2nd[i][c];
        v2[c] = a2dn[j][c] + a2nd[j][c];
      }
      // gdeS: d^2 g for the pair (the reference's tmp1 + tmp2 + tmp3 + tmp4)
      const T gS = d3(a1S[k], a2n) + d3(x1[i], v2) + d3(x1[j], v1) + d3(a1, w1);
      const T gg = k == 2 ? gde[1] * gde[0] : gde[i] * gde[i];
      for (int c = 0; c < 3; ++c) {
        cS[0][k][c] = T(2) * gi3 * gg * a2n[c] - gi2 * gS * a2n[c] - gi2 * gde[i] * (a2dn[j][c] + a2nd[j][c]) -
                      gi2 * gde[j] * (a2dn[i][c] + a2nd[i][c]) + gi1 * w1[c];
        cS[1][k][c] = T(2) * gi3 * gg * na1[c] - gi2 * gS * na1[c] - gi2 * gde[i] * (ndA1[j][c] + nA1d[j][c]) -
                      gi2 * gde[j] * (ndA1[i][c] + nA1d[i][c]) + gi1 * w2[c];
      }
    }
  }
  // ---- derivatives of the Christoffel symbols christof(lm,b,a) = a_a,lm . a^b:
  // d/dxi^l = a_a,lm,l . a^b + a_a,lm . a^b_,l; the entry (l,lm,b,a) =
  // (2,2,1,2) keeps the reference's second product cderi1(:,2) . conderi2(:,2)
  T(&CD)[2][2][2][2] = B.chd;
  const T* cv[2] = {c1, c2};
  const T* cvd[2][2] = {{G.cdc1[0], G.cdc1[1]}, {G.cdc2[0], G.cdc2[1]}};  // [vector][l]
  // third derivative a_a,lm,l: S index of (a, lm, l), a_1 = x_t, a_2 = x_p
  auto s3 = [&](int a, int lm, int l) { return S[a + lm + l]; };  // x with (a+lm+l) phi-derivatives
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      CD[l][0][b][0] = d3(s3(0, 0, l), cv[b]) + d3(x1[0], cvd[b][l]);
      CD[l][1][b][0] = d3(s3(0, 1, l), cv[b]) + d3(x1[1], cvd[b][l]);
      CD[l][1][b][1] = d3(s3(1, 1, l), cv[b]) + d3(x2[1], cvd[b][l]);
    }
  CD[1][1][0][1] = d3(S[3], c1) + d3(x1[1], G.cdc2[1]);  // as the reference writes it
#pragma unroll
  for (int l = 0; l < 2; ++l)
#pragma unroll
    for (int b = 0; b < 2; ++b) CD[l][0][b][1] = CD[l][1][b][0];
  // ---- second derivatives of a^ab = a^a . a^b: (a^a_,lm,l . a^b + a^a_,lm . a^b_,l
  // + a^a_,l . a^b_,lm + a^a . a^b_,lm,l), the pair index of (lm, l)
  T(&M2)[2][2][2][2] = B.cad2;
#pragma unroll
  for (int l = 0; l < 2; ++l)
#pragma unroll
    for (int lm = 0; lm < 2; ++lm) {
      const int k = l == lm ? l : 2;
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int a = 0; a < 2; ++a)
          M2[l][lm][b][a] = d3(cS[a][k], cv[b]) + d3(cvd[a][lm], cvd[b][l]) + d3(cvd[a][l], cvd[b][lm]) +
                            d3(cv[a], cS[b][k]);
    }
}

// cal_moment_deri, cal_Q, cal_bcurmix at one point with the reference sphere
// of radius R (st = sin t, ct = cos t) analytic: A^11 = 1/R^2, A^22 =
// 1/(R st)^2, d_t A^22 = -2 ct / (R^2 st^3), d_tt A^22 = (2/st^2 +
// 6 ct^2/st^4) / R^2; B_11 = R, B_22 = R st^2, d_t B_22 = 2 R st ct,
// d_tt B_22 = 2 R (ct^2 - st^2); every other entry zero.
// bq: bcurmix(1,1), (2,1), (1,2), (2,2), Q(1), Q(2), Qcode.
template <class T>
__device__ void bend_q(const Geo<T>& G, const BendT<T>& B, T R, T st, T ct, T eb, T* bq) {
  T a[2][2], ad1[2][2][2], b[2][2], ch[2][2][2];
  a[0][0] = G.conat[0];
  a[1][1] = G.conat[1];
  a[0][1] = a[1][0] = G.conat[2];
#pragma unroll
  for (int l = 0; l < 2; ++l) {
    ad1[l][0][0] = G.conatd1[l][0];
    ad1[l][1][1] = G.conatd1[l][1];
    ad1[l][0][1] = ad1[l][1][0] = G.conatd1[l][2];
  }
  b[0][0] = G.bcur[0];
  b[1][1] = G.bcur[1];
  b[0][1] = b[1][0] = G.bcur[2];
#pragma unroll
  for (int g = 0; g < 2; ++g)
#pragma unroll
    for (int bb = 0; bb < 2; ++bb)
#pragma unroll
      for (int aa = 0; aa < 2; ++aa) ch[g][bb][aa] = G.chf[g + 2 * bb + 4 * aa];
  const T iR2 = T(1) / (R * R), s2 = st * st;
  T AR[2][2] = {{iR2, T(0)}, {T(0), iR2 / s2}};
  T ARd1[2][2][2] = {};
  ARd1[0][1][1] = -T(2) * ct * iR2 / (s2 * st);
  T ARd2[2][2][2][2] = {};
  ARd2[0][0][1][1] = (T(2) / s2 + T(6) * ct * ct / (s2 * s2)) * iR2;
  T BR[2][2] = {{R, T(0)}, {T(0), R * s2}};
  T BRd1[2][2][2] = {};
  BRd1[0][1][1] = T(2) * R * st * ct;
  T BRd2[2][2][2][2] = {};
  BRd2[0][0][1][1] = T(2) * R * (ct * ct - s2);
  // cal_moment_deri (indices: a(i,j) -> a[i-1][j-1], as the reference)
  T mom[2][2] = {}, momdF[2][2][2] = {}, momdS = T(0);
#pragma unroll
  for (int al = 0; al < 2; ++al)
#pragma unroll
    for (int be = 0; be < 2; ++be) {
#pragma unroll
      for (int ga = 0; ga < 2; ++ga)
#pragma unroll
        for (int gp = 0; gp < 2; ++gp) {
          const T X0 = AR[gp][al] * BR[ga][gp] - a[gp][al] * b[ga][gp];
          momdS = momdS + B.cad2[be][al][be][ga] * X0 +
                  ad1[al][be][ga] * (ARd1[be][gp][al] * BR[ga][gp] + AR[gp][al] * BRd1[be][ga][gp] -
                                     ad1[be][gp][al] * b[ga][gp] - a[gp][al] * B.bd1[be][ga][gp]) +
                  ad1[be][be][ga] * (ARd1[al][gp][al] * BR[ga][gp] + AR[gp][al] * BRd1[al][ga][gp] -
                                     ad1[al][gp][al] * b[ga][gp] - a[gp][al] * B.bd1[al][ga][gp]) +
                  a[be][ga] * (ARd2[be][al][gp][al] * BR[ga][gp] + ARd1[al][gp][al] * BRd1[be][ga][gp] +
                               ARd1[be][gp][al] * BRd1[al][ga][gp] + AR[gp][al] * BRd2[be][al][ga][gp] -
                               B.cad2[be][al][gp][al] * b[ga][gp] - ad1[al][gp][al] * B.bd1[be][ga][gp] -
                               ad1[be][gp][al] * B.bd1[al][ga][gp] - a[gp][al] * B.bd2[be][al][ga][gp]);
        }
      if (al == 1 && be == 0) continue;
#pragma unroll
      for (int ga = 0; ga < 2; ++ga)
#pragma unroll
        for (int gp = 0; gp < 2; ++gp) mom[be][al] = mom[be][al] + a[be][ga] * (AR[gp][al] * BR[ga][gp] - a[gp][al] * b[ga][gp]);
#pragma unroll
      for (int l = 0; l < 2; ++l)
#pragma unroll
        for (int ga = 0; ga < 2; ++ga)
#pragma unroll
          for (int gp = 0; gp < 2; ++gp)
            momdF[l][be][al] = momdF[l][be][al] + ad1[l][be][ga] * (AR[gp][al] * BR[ga][gp] - a[gp][al] * b[ga][gp]) +
                               a[be][ga] * (ARd1[l][gp][al] * BR[ga][gp] + AR[gp][al] * BRd1[l][ga][gp] -
                                            ad1[l][gp][al] * b[ga][gp] - a[gp][al] * B.bd1[l][ga][gp]);
    }
  mom[0][1] = mom[1][0];
  momdF[0][0][1] = momdF[0][1][0];
  momdF[1][0][1] = momdF[1][1][0];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      mom[i][j] = mom[i][j] * eb;
      momdF[0][i][j] = momdF[0][i][j] * eb;
      momdF[1][i][j] = momdF[1][i][j] * eb;
    }
  momdS = momdS * eb;
  // cal_Q
  T Q[2] = {T(0), T(0)}, Qc = momdS;
#pragma unroll
  for (int be = 0; be < 2; ++be)
#pragma unroll
    for (int al = 0; al < 2; ++al) {
      Q[be] = Q[be] + momdF[al][be][al];
#pragma unroll
      for (int lm = 0; lm < 2; ++lm) {
        Q[be] = Q[be] + ch[lm][al][al] * mom[be][lm] + ch[lm][be][al] * mom[lm][al];
        Qc = Qc + B.chd[be][lm][al][al] * mom[be][lm] + ch[lm][al][al] * momdF[be][be][lm] +
             B.chd[be][lm][be][al] * mom[lm][al] + ch[lm][be][al] * momdF[be][lm][al];
      }
    }
#pragma unroll
  for (int be = 0; be < 2; ++be)
#pragma unroll
    for (int lm = 0; lm < 2; ++lm) Qc = Qc + Q[lm] * ch[lm][be][be];
  // cal_bcurmix: bcurmix(be,al) = sum_lm conat(lm,al) bcur(be,lm)
#pragma unroll
  for (int al = 0; al < 2; ++al)
#pragma unroll
    for (int be = 0; be < 2; ++be) bq[be + 2 * al] = a[0][al] * b[be][0] + a[1][al] * b[be][1];
  bq[4] = Q[0];
  bq[5] = Q[1];
  bq[6] = Qc;
}

// Staged values per (row, m): G's 18 (ccs = 2c + cos/sin, kind P, dP, d2P at
// 3 ccs + kind) then GB's 12 (kind d3P, d4P at 18 + 2 ccs + kind).
constexpr int kBK = 30;

template <class T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1) membrane_bend_kernel(const RowWork* __restrict__ work, int nwork,
                                                            const CapInfo* __restrict__ caps,
                                                            const GroupDev* __restrict__ groups,
                                                            const int* __restrict__ sur_flag) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const RowWork it = work[w];
    const CapInfo ci = caps[it.cap];
    const T hf = (T)(0.5 * ci.gs), csk = (T)ci.csk, eb = (T)ci.eb;
    const bool normals_only = sur_flag && sur_flag[it.cap];
    const GroupDev gd = groups[it.group];
    const int N = gd.N, nD = gd.nD, mD = gd.mD;
    const int RP = (int)blockDim.x / mD > 0 ? (int)blockDim.x / mD : 1;  // rows per chunk, one point per thread
    const int SR = N * kBK + 2;
    T* sG = (T*)smem_raw;               // [RP][SR]
    T* sTrig = sG + RP * SR;            // [2N][mD]: cos m phi_j (rows m), sin (rows N + m)
    T* sTrigT = sTrig + 2 * N * mD;     // [mD][2N]: the same, transposed for the forward DFT
    T* sOut = sTrigT + 2 * N * mD;      // [RP][6][mD]
    int* sOff = (int*)(sOut + RP * 6 * mD);  // [30N]: staged offsets of G's then GB's elements
    const T* Gs = (const T*)gd.buf.G + (long long)ci.gidx * (18 * N * nD);   // [ccs][m][kind][lat]
    const T* Gb = (const T*)gd.buf.GB + (long long)ci.gidx * (12 * N * nD);  // [ccs][m][kind][lat]
    const T* trig = (const T*)gd.trigD[sizeof(T) == 8 ? 0 : 1];
    const T* lat = (const T*)gd.latD[sizeof(T) == 8 ? 0 : 1];
    T* Fout = (T*)gd.buf.Fout + (long long)ci.gidx * 12 * N * nD;
    const T sfn = T(2) / T(mD);
    const T R = (T)ci.R;
    __syncthreads();  // the previous item's reads of shared memory are done
    for (int q = tid; q < 2 * N * mD; q += blockDim.x) sTrig[q] = trig[q];
    for (int q = tid; q < 2 * N * mD; q += blockDim.x) sTrigT[q] = trig[(q % (2 * N)) * mD + q / (2 * N)];
    for (int e = tid; e < 18 * N; e += blockDim.x) {  // e = (ccs N + m) 3 + kind
      const int kind = e % 3, cm_ = e / 3, m = cm_ % N, ccs = cm_ / N;
      sOff[e] = m * kBK + 3 * ccs + kind;
    }
    for (int e = tid; e < 12 * N; e += blockDim.x) {  // e = (ccs N + m) 2 + kind
      const int kind = e & 1, cm_ = e >> 1, m = cm_ % N, ccs = cm_ / N;
      sOff[18 * N + e] = m * kBK + 18 + 2 * ccs + kind;
    }
    const int sr = tid % RP, se0 = tid / RP, ses = (int)blockDim.x / RP;
    const bool son = tid < ses * RP;
    for (int rb = it.row0; rb < it.row0 + it.nrows; rb += RP) {
      const int rows = min(RP, it.row0 + it.nrows - rb);
      __syncthreads();  // the previous chunk's staged rows and outputs are consumed
      if (son && sr < rows) {
        for (int e = se0; e < 18 * N; e += ses) stage_async(&sG[sr * SR + sOff[e]], &Gs[(long long)e * nD + rb + sr]);
        for (int e = se0; e < 12 * N; e += ses)
          stage_async(&sG[sr * SR + sOff[18 * N + e]], &Gb[(long long)e * nD + rb + sr]);
      }
      stage_wait();
      __syncthreads();
      {
        const int r = tid / mD, j = tid - (tid / mD) * mD;
        if (r < rows) {
          const int i = rb + r;
          // a1, a2, d11, d12, d22, S1..S4, Q1..Q5 per component
          T acc[14][3];
#pragma unroll
          for (int q = 0; q < 14; ++q) acc[q][0] = acc[q][1] = acc[q][2] = T(0);
          const T* g = sG + r * SR;
          for (int m = 0; m < N; ++m) {
            const T cm = sTrig[m * mD + j], sm = sTrig[(N + m) * mD + j], fm = (T)m, fm2 = fm * fm;
            const T* gm = g + m * kBK;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              T ga[5], gb[5];  // P^(k) series of the cos and sin rows, k = 0..4
#pragma unroll
              for (int k = 0; k < 3; ++k) {
                ga[k] = gm[3 * (2 * c) + k];
                gb[k] = gm[3 * (2 * c + 1) + k];
              }
#pragma unroll
              for (int k = 0; k < 2; ++k) {
                ga[3 + k] = gm[18 + 2 * (2 * c) + k];
                gb[3 + k] = gm[18 + 2 * (2 * c + 1) + k];
              }
              T t0[5], t1[5];  // parthe0 and parthe1 forms of the P^(k) series
#pragma unroll
              for (int k = 0; k < 5; ++k) {
                t0[k] = ga[k] * cm - gb[k] * sm;
                t1[k] = fm * (ga[k] * (-sm) - gb[k] * cm);
              }
              acc[0][c] += t0[1];               // x_t
              acc[1][c] += t1[0];               // x_p
              acc[2][c] += t0[2];               // x_tt
              acc[3][c] += t1[1];               // x_tp
              acc[4][c] += -fm2 * t0[0];        // x_pp
              acc[5][c] += t0[3];               // x_ttt
              acc[6][c] += t1[2];               // x_ttp
              acc[7][c] += -fm2 * t0[1];        // x_tpp
              acc[8][c] += -fm2 * t1[0];        // x_ppp (m^3 (a sin + b cos))
              acc[9][c] += t0[4];               // x_tttt
              acc[10][c] += t1[3];              // x_tttp
              acc[11][c] += -fm2 * t0[2];       // x_ttpp
              acc[12][c] += -fm2 * t1[1];       // x_tppp
              acc[13][c] += fm2 * fm2 * t0[0];  // x_pppp
            }
          }
          // the reference sphere: x = R u, u = (st sp, st cp, ct)
          const T st = lat[4 * i], ct = lat[4 * i + 1];
          const T cp = sTrig[1 * mD + j], sp = sTrig[(N + 1) * mD + j];
          const T u[3] = {st * sp, st * cp, ct};
          const T ut[3] = {ct * sp, ct * cp, -st};
          const T up[3] = {st * cp, -st * sp, T(0)};
          const T utp[3] = {ct * cp, -ct * sp, T(0)};
          const T upp[3] = {-st * sp, -st * cp, T(0)};
          const T utpp[3] = {-ct * sp, -ct * cp, T(0)};
          // derivatives of u in the order of acc: u_t, u_p, u_tt = -u, u_tp, u_pp,
          // u_ttt = -u_t, u_ttp = -u_p, u_tpp, u_ppp = -u_p, u_tttt = u,
          // u_tttp = -u_tp, u_ttpp = -u_pp, u_tppp = -u_tp, u_pppp = -u_pp
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const T sph[14] = {ut[c], up[c], -u[c], utp[c], upp[c], -ut[c], -up[c], utpp[c], -up[c],
                               u[c], -utp[c], -upp[c], -utp[c], -upp[c]};
#pragma unroll
            for (int q = 0; q < 14; ++q) acc[q][c] += R * sph[q];
          }
          Geo<T> Gm;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            Gm.a1[c] = acc[0][c];
            Gm.a2[c] = acc[1][c];
            Gm.d11[c] = acc[2][c];
            Gm.d12[c] = acc[3][c];
            Gm.d22[c] = acc[4][c];
          }
          T f[3] = {T(0), T(0), T(0)};
          geometry<T>(Gm);
          if (!normals_only) {
            const T iR2 = fdiv(T(1), R * R);
            T A[3] = {iR2, fdiv(iR2, st * st), T(0)};
            T Ad[2][3] = {{T(0), fdiv(-T(2) * ct * iR2, st * st * st), T(0)}, {T(0), T(0), T(0)}};
            if (eb != T(0)) {
              BendT<T> B;
              bend_tensors<T>(Gm, (const T(*)[3]) & acc[5][0], (const T(*)[3]) & acc[9][0], B);
              T bq[7];
              bend_q<T>(Gm, B, R, st, ct, eb, bq);
              mechanics<T>(Gm, A, Ad, hf, csk, ci.law, f, bq);
            } else {
              mechanics<T>(Gm, A, Ad, hf, csk, ci.law, f);
            }
          }
          T* o = sOut + r * 6 * mD;
          o[0 * mD + j] = f[0];
          o[1 * mD + j] = f[1];
          o[2 * mD + j] = f[2];
          o[3 * mD + j] = Gm.n[0];
          o[4 * mD + j] = Gm.n[1];
          o[5 * mD + j] = Gm.n[2];
        }
      }
      __syncthreads();
      // forward DFT (shagc.f:364-380) of the six outputs per row: warp = (row,
      // field) line, lane p < 2N = cos m = p, sin m = p - N; the lanes read
      // consecutive words of the transposed table (no bank conflicts) and the
      // row's value as a broadcast
      // (row, field triple) line per warp: one load of the trig value serves
      // the triple's three fields (force or normal)
      for (int line = warp; line < rows * 2; line += nwarp) {
        const int f0 = 3 * (line & 1), rr = line >> 1;
        const T* o = sOut + (rr * 6 + f0) * mD;
        for (int p = lane; p < 2 * N; p += 32) {
          const T* t = sTrigT + p;
          T a[3] = {T(0), T(0), T(0)};
          for (int jj = 0; jj < mD; ++jj) {
            const T tt = t[jj * 2 * N];
#pragma unroll
            for (int f = 0; f < 3; ++f) a[f] += o[f * mD + jj] * tt;
          }
#pragma unroll
          for (int f = 0; f < 3; ++f) Fout[((long long)(f0 + f) * 2 * N + p) * nD + rb + rr] = (p < N ? sfn : -sfn) * a[f];
        }
      }
    }
  }
}

}  // namespace

template <class T>
cudaError_t launch_membrane_bend(const RowWork* work, int nwork, const CapInfo* caps, const GroupDev* groups,
                                 const int* sur_flag, int nmax, cudaStream_t st) {
  if (nwork <= 0) return cudaSuccess;
  size_t e = 0;  // shared memory (elements of T) over the degrees up to nmax
  for (size_t n = 1; n <= (size_t)nmax; ++n) {
    const size_t mD = 4 * n, RP = 256 / mD > 0 ? 256 / mD : 1;
    const size_t en = RP * (n * kBK + 2) + 4 * n * mD + RP * 6 * mD + (30 * n * sizeof(int) + sizeof(T) - 1) / sizeof(T) + 8;
    e = std::max(e, en);
  }
  const size_t smem = sizeof(T) * e;
  cudaError_t err = smem_limit(membrane_bend_kernel<T>, smem);
  if (err != cudaSuccess) return err;
  int dev = 0, sms = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, membrane_bend_kernel<T>, 256, smem) != cudaSuccess || per < 1)
    per = 1;
  const int grid = std::min(nwork, sms * per);
  launch_pdl(membrane_bend_kernel<T>, dim3(grid), dim3(256), smem, st, work, nwork, caps, groups, sur_flag);
  return cudaGetLastError();
}

template cudaError_t launch_membrane_bend<double>(const RowWork*, int, const CapInfo*, const GroupDev*, const int*, int,
                                                  cudaStream_t);
template cudaError_t launch_membrane_bend<float>(const RowWork*, int, const CapInfo*, const GroupDev*, const int*, int,
                                                 cudaStream_t);

}  // namespace sg
