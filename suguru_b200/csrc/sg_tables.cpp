// sg_tables.cpp -- FP64 host tables: Gauss-Legendre nodes and weights and
// SPHEREPACK-normalised associated Legendre functions with theta derivatives.
//
// gaqd.f:45-180 computes the Gauss colatitudes north to south in (0, pi) with
// weights summing to 2; sphharm.c:38-108 evaluates P^m_n through GSL's
// sphPlm times sqrt(2 pi)(-1)^m (int_{-1}^{1} P^2 dx = 1, no Condon-Shortley
// phase) and its x-derivatives, which sph3.f90:63-65 turns into theta
// derivatives.  Restated here: Newton iteration in t on the Fourier form of P_n(cos t) for the nodes,
// the standard normalised three-term recurrence for P^m_n, and the m+-1
// ladder identity for d/dtheta (applied twice for the second derivative).
#include <cmath>
#include <cstring>
#include <vector>

#include "sg_kernels.h"

namespace sg {

namespace {
const double kPi = 3.14159265358979323846264338327950288;

}  // namespace

// P_n(cos t) = sum_k a_k a_{n-k} cos((n-2k) t), a_k = binom(2k,k)/4^k, and its
// t-derivative, evaluated in t so the nodes near the poles keep full accuracy.
static void pn_theta(int n, double t, double* p, double* dp) {
  std::vector<double> a(n + 1);
  a[0] = 1.0;
  for (int k = 1; k <= n; ++k) a[k] = a[k - 1] * (2.0 * k - 1.0) / (2.0 * k);
  double s = 0.0, d = 0.0;
  for (int k = 0; k <= n; ++k) {
    const double c = a[k] * a[n - k], q = (double)(n - 2 * k);
    s += c * std::cos(q * t);
    d -= c * q * std::sin(q * t);
  }
  *p = s;
  *dp = d;
}

void host_gauss(int n, double* th, double* w) {
  const int half = (n + 1) / 2;
  for (int k = 1; k <= half; ++k) {
    double t = kPi * (k - 0.25) / (n + 0.5);
    const bool equator = (n % 2 == 1) && k == half;
    if (equator) {
      t = 0.5 * kPi;
    } else {
      for (int it = 0; it < 100; ++it) {
        double pn, dp;
        pn_theta(n, t, &pn, &dp);
        const double dt = -pn / dp;
        t += dt;
        if (std::fabs(dt) < 1e-17) break;
      }
    }
    double pn, dp;
    pn_theta(n, t, &pn, &dp);
    const double ww = 2.0 / (dp * dp);  // 2 / ((1-x^2) P_n'(x)^2)
    th[k - 1] = t;
    w[k - 1] = ww;
    th[n - k] = kPi - t;
    w[n - k] = ww;
  }
  if (n % 2 == 1) th[half - 1] = 0.5 * kPi;
}

void host_legendre(double th, int mm, int nn, double* P, double* dP, double* d2P) {
  const int nt = nn + 2;
  std::vector<double> T((size_t)nt * nt, 0.0), D((size_t)nt * nt, 0.0), D2((size_t)nt * nt, 0.0);
  const double x = std::cos(th), s = std::sin(th);
  double pmm = std::sqrt(0.5);
  for (int m = 0; m < nt; ++m) {
    if (m > 0) pmm *= std::sqrt((2.0 * m + 1.0) / (2.0 * m)) * s;
    T[(size_t)m * nt + m] = pmm;
    if (m + 1 < nt) T[(size_t)m * nt + m + 1] = std::sqrt(2.0 * m + 3.0) * x * pmm;
    for (int n = m + 2; n < nt; ++n) {
      double a = std::sqrt((4.0 * n * n - 1.0) / ((double)n * n - (double)m * m));
      double b = std::sqrt(((n - 1.0) * (n - 1.0) - (double)m * m) / (4.0 * (n - 1.0) * (n - 1.0) - 1.0));
      T[(size_t)m * nt + n] = a * (x * T[(size_t)m * nt + n - 1] - b * T[(size_t)m * nt + n - 2]);
    }
  }
  auto at = [&](const std::vector<double>& A, int m, int n) -> double {
    return (m < 0 || m > n || n >= nt) ? 0.0 : A[(size_t)m * nt + n];
  };
  auto ladder = [&](const std::vector<double>& A, std::vector<double>& B) {
    for (int m = 0; m < nt; ++m)
      for (int n = m; n < nt; ++n)
        B[(size_t)m * nt + n] = (m == 0) ? -std::sqrt((double)n * (n + 1.0)) * at(A, 1, n)
                                         : 0.5 * (std::sqrt((n + m) * (n - m + 1.0)) * at(A, m - 1, n) -
                                                  std::sqrt((n + m + 1.0) * (n - m)) * at(A, m + 1, n));
  };
  ladder(T, D);
  ladder(D, D2);
  for (int m = 0; m < mm; ++m)
    for (int n = 0; n < nn; ++n) {
      const size_t o = (size_t)m * nn + n, q = (size_t)m * nt + n;
      const bool ok = n >= m && m < nt;
      if (P) P[o] = ok ? T[q] : 0.0;
      if (dP) dP[o] = ok ? D[q] : 0.0;
      if (d2P) d2P[o] = ok ? D2[q] : 0.0;
    }
}

void host_legendre_d34(double th, int mm, int nn, double* d3P, double* d4P) {
  // d/dtheta of P^m_n is a combination of P^{m-1}_n and P^{m+1}_n (the ladder
  // of host_legendre), so the third and fourth derivatives come from applying
  // it to the second and third
  const int nt = nn + 2;
  std::vector<double> D2f((size_t)nt * nt), T3((size_t)nt * nt, 0.0), T4((size_t)nt * nt, 0.0);
  host_legendre(th, nt, nt, nullptr, nullptr, D2f.data());
  auto at = [&](const std::vector<double>& A, int m, int n) -> double {
    return (m < 0 || m > n || n >= nt) ? 0.0 : A[(size_t)m * nt + n];
  };
  auto ladder = [&](const std::vector<double>& A, std::vector<double>& B) {
    for (int m = 0; m < nt; ++m)
      for (int n = m; n < nt; ++n)
        B[(size_t)m * nt + n] = (m == 0) ? -std::sqrt((double)n * (n + 1.0)) * at(A, 1, n)
                                         : 0.5 * (std::sqrt((n + m) * (n - m + 1.0)) * at(A, m - 1, n) -
                                                  std::sqrt((n + m + 1.0) * (n - m)) * at(A, m + 1, n));
  };
  ladder(D2f, T3);
  ladder(T3, T4);
  for (int m = 0; m < mm; ++m)
    for (int n = 0; n < nn; ++n) {
      const size_t o = (size_t)m * nn + n, q = (size_t)m * nt + n;
      const bool ok = n >= m && m < nt;
      if (d3P) d3P[o] = ok ? T3[q] : 0.0;
      if (d4P) d4P[o] = ok ? T4[q] : 0.0;
    }
}

// ---------------------------------------------------------------- bf16 split
// Round-to-nearest-even FP32 -> bf16 (bit pattern), and back.
static uint16_t f32_to_bf16(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);  // NaN stays NaN
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
static double bf16_to_double(uint16_t h) {
  const uint32_t u = (uint32_t)h << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return (double)f;
}

void host_umma_image(const double* B, long long sBm, int M, int J, int K, int Jp, int Kp, uint16_t* out) {
  const int KC = Kp / 8;
  const size_t img = (size_t)Jp * Kp;
  for (int m = 0; m < M; ++m) {
    uint16_t* part = out + (size_t)m * 3 * img;
    for (int j = 0; j < Jp; ++j)
      for (int k = 0; k < Kp; ++k) {
        double x = (j < J && k < K) ? B[(size_t)m * sBm + (size_t)j * K + k] : 0.0;
        const size_t o = ((size_t)(j / 8) * KC + k / 8) * 64 + (j % 8) * 8 + (k % 8);
        for (int t = 0; t < 3; ++t) {  // each part rounds what the earlier ones leave
          const uint16_t h = f32_to_bf16((float)x);
          part[t * img + o] = h;
          x -= bf16_to_double(h);
        }
      }
  }
}

}  // namespace sg
