// sg_oracle.cpp -- CPU FP64 restatement of the reference IB coupling step.
//
// TEST INFRASTRUCTURE ONLY: the parity oracle and the timed CPU baseline.
// Loaded only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
// leg.  See sg_oracle.h for the layouts; each routine cites the reference
// (WhiteTshirtXI/Suguru) file:line it restates.
//
// Third-party arithmetic restated here (not vendored as source in the
// reference): GSL 1.16 gsl_sf_legendre_sphPlm(_deriv)_array, called from
// sphharm.c:45,62,79.  We use the standard normalised three-term recurrence
// for P^m_n and the m+-1 ladder identities for the theta derivatives, which are
// exact in exact arithmetic.
#include "sg_oracle.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>
#include <chrono>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double kPi = 3.14159265358979323846264338327950288;

// ---------------------------------------------------------------- gaqd ------
// gaqd.f:45-180: Gauss points in colatitude, north to south, and weights.
// Restated with Newton iterations on P_n(cos theta) in theta.
[[maybe_unused]] void pn_eval(int n, double x, double* pn, double* pnm1) {
  double p0 = 1.0, p1 = x;
  if (n == 0) { *pn = 1.0; *pnm1 = 0.0; return; }
  for (int k = 2; k <= n; ++k) {
    double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
    p0 = p1;
    p1 = pk;
  }
  *pn = p1;
  *pnm1 = p0;
}

// P_n(cos t) = sum_k a_k a_{n-k} cos((n-2k) t), a_k = binom(2k,k)/4^k, and its
// t-derivative: evaluated in t, this keeps full relative accuracy near the
// poles where x = cos t has lost digits (gaqd.f works in theta for the same reason).
void pn_theta(int n, double t, double* p, double* dp) {
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

void gauss(int n, double* th, double* w) {
  int half = (n + 1) / 2;
  for (int k = 1; k <= half; ++k) {
    double t = kPi * (k - 0.25) / (n + 0.5);
    if ((n % 2 == 1) && k == half) {
      t = 0.5 * kPi;
    } else {
      for (int it = 0; it < 100; ++it) {
        double pn, dp;
        pn_theta(n, t, &pn, &dp);
        double dt = -pn / dp;
        t += dt;
        if (std::fabs(dt) < 1e-17) break;
      }
    }
    double pn, dp;
    pn_theta(n, t, &pn, &dp);
    double ww = 2.0 / (dp * dp);  // w = 2 / ((1-x^2) P_n'(x)^2) = 2 / (dP_n/dt)^2
    th[k - 1] = t;
    w[k - 1] = ww;
    th[n - k] = kPi - t;
    w[n - k] = ww;
  }
  if (n % 2 == 1) th[half - 1] = 0.5 * kPi;
}

// --------------------------------------------------------- Legendre ---------
// Full triangle T[m*nn+n] (n<nn, m<=n) of SPHEREPACK-normalised P^m_n(cos th)
// (sphharm.c:38-50: int_{-1}^{1} P^2 dx = 1, no Condon-Shortley phase), and
// the theta derivatives (sph3.f90:63-65 converts d/dx to d/dtheta).
void legendre_full(double th, int nn, std::vector<double>& T, std::vector<double>& D,
                   std::vector<double>& D2) {
  T.assign((size_t)nn * nn, 0.0);
  D.assign((size_t)nn * nn, 0.0);
  D2.assign((size_t)nn * nn, 0.0);
  double x = std::cos(th), s = std::sin(th);
  double pmm = std::sqrt(0.5);
  for (int m = 0; m < nn; ++m) {
    if (m > 0) pmm *= std::sqrt((2.0 * m + 1.0) / (2.0 * m)) * s;
    T[(size_t)m * nn + m] = pmm;
    if (m + 1 < nn) T[(size_t)m * nn + m + 1] = std::sqrt(2.0 * m + 3.0) * x * pmm;
    for (int n = m + 2; n < nn; ++n) {
      double a = std::sqrt((4.0 * n * n - 1.0) / ((double)n * n - (double)m * m));
      double b = std::sqrt(((n - 1.0) * (n - 1.0) - (double)m * m) / (4.0 * (n - 1.0) * (n - 1.0) - 1.0));
      T[(size_t)m * nn + n] = a * (x * T[(size_t)m * nn + n - 1] - b * T[(size_t)m * nn + n - 2]);
    }
  }
  auto at = [&](const std::vector<double>& A, int m, int n) -> double {
    return (m < 0 || m > n || n >= nn) ? 0.0 : A[(size_t)m * nn + n];
  };
  // dP^m_n/dtheta = 1/2 [ sqrt((n+m)(n-m+1)) P^{m-1}_n - sqrt((n+m+1)(n-m)) P^{m+1}_n ],
  // m=0: -sqrt(n(n+1)) P^1_n.  Applied twice for the second derivative.
  auto ladder = [&](const std::vector<double>& A, std::vector<double>& B) {
    for (int m = 0; m < nn; ++m)
      for (int n = m; n < nn; ++n) {
        double v;
        if (m == 0)
          v = -std::sqrt((double)n * (n + 1.0)) * at(A, 1, n);
        else
          v = 0.5 * (std::sqrt((n + m) * (n - m + 1.0)) * at(A, m - 1, n) -
                     std::sqrt((n + m + 1.0) * (n - m)) * at(A, m + 1, n));
        B[(size_t)m * nn + n] = v;
      }
  };
  ladder(T, D);
  ladder(D, D2);
}

// The same with the third and fourth theta derivatives (cal_legendre_deri4_array,
// sphharm.c:110-145, converted to theta as sph3.f90:72-95 does): the ladder
// applied twice more (d/dtheta of P^m_n involves P^{m-1}_n and P^{m+1}_n of the
// same degree only, so every order stays exact).
void legendre_full4(double th, int nn, std::vector<double>& T, std::vector<double>& D, std::vector<double>& D2,
                    std::vector<double>& D3, std::vector<double>& D4) {
  legendre_full(th, nn, T, D, D2);
  auto at = [&](const std::vector<double>& A, int m, int n) -> double {
    return (m < 0 || m > n || n >= nn) ? 0.0 : A[(size_t)m * nn + n];
  };
  auto ladder = [&](const std::vector<double>& A, std::vector<double>& B) {
    B.assign((size_t)nn * nn, 0.0);
    for (int m = 0; m < nn; ++m)
      for (int n = m; n < nn; ++n)
        B[(size_t)m * nn + n] = m == 0 ? -std::sqrt((double)n * (n + 1.0)) * at(A, 1, n)
                                       : 0.5 * (std::sqrt((n + m) * (n - m + 1.0)) * at(A, m - 1, n) -
                                                std::sqrt((n + m + 1.0) * (n - m)) * at(A, m + 1, n));
  };
  ladder(D2, D3);
  ladder(D3, D4);
}

// Analysis/synthesis plan for a Gauss grid nlat x nlon (shagci/shsgci work).
struct Plan {
  int nlat, nlon, l, lm1;
  bool nyq;
  std::vector<double> th, w, P;  // P[(i*l+m)*nlat+n]
  std::vector<double> ct, st;    // cos/sin(2 pi k / nlon)
};

int trunc_l(int nlat, int nlon) {
  int l = (nlon % 2 == 0) ? (nlon + 2) / 2 : (nlon + 1) / 2;
  return l < nlat ? l : nlat;
}

std::shared_ptr<Plan> build_plan(int nlat, int nlon) {
  auto p = std::make_shared<Plan>();
  p->nlat = nlat;
  p->nlon = nlon;
  p->l = trunc_l(nlat, nlon);
  p->nyq = (nlon == 2 * p->l - 2);  // shagc.f:385-386
  p->lm1 = p->nyq ? p->l - 1 : p->l;
  p->th.resize(nlat);
  p->w.resize(nlat);
  gauss(nlat, p->th.data(), p->w.data());
  p->P.assign((size_t)nlat * p->l * nlat, 0.0);
  std::vector<double> T, D, D2;
  for (int i = 0; i < nlat; ++i) {
    legendre_full(p->th[i], nlat, T, D, D2);
    for (int m = 0; m < p->l; ++m)
      for (int n = m; n < nlat; ++n) p->P[((size_t)i * p->l + m) * nlat + n] = T[(size_t)m * nlat + n];
  }
  p->ct.resize(nlon);
  p->st.resize(nlon);
  for (int k = 0; k < nlon; ++k) {
    p->ct[k] = std::cos(2.0 * kPi * k / nlon);
    p->st[k] = std::sin(2.0 * kPi * k / nlon);
  }
  return p;
}

std::mutex g_plan_mu;
std::map<std::pair<int, int>, std::shared_ptr<Plan>> g_plans;

// faithful: rebuild on every call as shagci/trssph(intl=0) do (sph1.f90:54-76).
std::shared_ptr<Plan> get_plan(int nlat, int nlon, bool faithful) {
  if (faithful) return build_plan(nlat, nlon);
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto key = std::make_pair(nlat, nlon);
  auto it = g_plans.find(key);
  if (it != g_plans.end()) return it->second;
  auto p = build_plan(nlat, nlon);
  g_plans[key] = p;
  return p;
}

// shagc.f:364-470 (mode 0), restated without the even/odd folding.
// a,b: [m*nlat+n], m<l.
void analysis(const Plan& p, const double* g, double* a, double* b) {
  const int nlat = p.nlat, nlon = p.nlon, l = p.l;
  std::memset(a, 0, sizeof(double) * (size_t)l * nlat);
  std::memset(b, 0, sizeof(double) * (size_t)l * nlat);
  std::vector<double> c(l), s(l);
  const double sfn = 2.0 / nlon;
  for (int i = 0; i < nlat; ++i) {
    const double* row = g + (size_t)i * nlon;
    for (int m = 0; m < l; ++m) {
      double cs = 0.0, ss = 0.0;
      for (int j = 0; j < nlon; ++j) {
        int k = (int)(((long)m * j) % nlon);
        cs += row[j] * p.ct[k];
        ss += row[j] * p.st[k];
      }
      c[m] = sfn * cs;
      s[m] = -sfn * ss;  // hrfft.f:114 forward transform carries -sin
    }
    const double wi = p.w[i];
    for (int m = 0; m < l; ++m) {
      const double* P = &p.P[((size_t)i * l + m) * nlat];
      bool isnyq = p.nyq && m == l - 1;
      double cm = wi * c[m] * (isnyq ? 0.5 : 1.0);
      double sm = (m == 0 || isnyq) ? 0.0 : wi * s[m];
      for (int n = m; n < nlat; ++n) {
        a[(size_t)m * nlat + n] += cm * P[n];
        b[(size_t)m * nlat + n] += sm * P[n];
      }
    }
  }
}

// shsgc.f:329-500 (mode 0) + hrfftb and the final 0.5 scaling.
void synthesis(const Plan& p, const double* a, const double* b, double* g) {
  const int nlat = p.nlat, nlon = p.nlon, l = p.l;
  std::vector<double> A(l), B(l);
  for (int i = 0; i < nlat; ++i) {
    for (int m = 0; m < l; ++m) {
      const double* P = &p.P[((size_t)i * l + m) * nlat];
      double sa = 0.0, sb = 0.0;
      for (int n = m; n < nlat; ++n) {
        sa += a[(size_t)m * nlat + n] * P[n];
        sb += b[(size_t)m * nlat + n] * P[n];
      }
      bool isnyq = p.nyq && m == l - 1;
      A[m] = (m == 0) ? 0.5 * sa : sa;   // 0.5*(G_0) ; Nyquist 0.5*2*sum
      B[m] = (m == 0 || isnyq) ? 0.0 : sb;
    }
    double* row = g + (size_t)i * nlon;
    for (int j = 0; j < nlon; ++j) {
      double v = 0.0;
      for (int m = 0; m < l; ++m) {
        int k = (int)(((long)m * j) % nlon);
        v += A[m] * p.ct[k] - B[m] * p.st[k];
      }
      row[j] = v;
    }
  }
}

// trssph.f:652-765 trab: copy the common triangle, zero the rest.
void trab(int ma, int na, const double* aa, const double* ba, int mb, int nb, double* ab, double* bb) {
  std::memset(ab, 0, sizeof(double) * (size_t)mb * nb);
  std::memset(bb, 0, sizeof(double) * (size_t)mb * nb);
  int m = ma < mb ? ma : mb, n = na < nb ? na : nb;
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) {
      ab[(size_t)i * nb + j] = aa[(size_t)i * na + j];
      bb[(size_t)i * nb + j] = ba[(size_t)i * na + j];
    }
}

void trssph1(int nlata, int nlona, const double* da, int nlatb, int nlonb, double* db, bool faithful) {
  auto pa = get_plan(nlata, nlona, faithful);
  auto pb = get_plan(nlatb, nlonb, faithful);
  std::vector<double> aa((size_t)pa->l * nlata), ba((size_t)pa->l * nlata);
  std::vector<double> ab((size_t)pb->l * nlatb), bb((size_t)pb->l * nlatb);
  analysis(*pa, da, aa.data(), ba.data());
  trab(pa->l, nlata, aa.data(), ba.data(), pb->l, nlatb, ab.data(), bb.data());
  synthesis(*pb, ab.data(), bb.data(), db);
}

inline double kern(double r) {
  // kernel.f90:7-25
  double ar = std::fabs(r);
  if (ar > 1.5) return 0.0;
  if (ar > 0.5) return (1.0 / 6.0) * (5.0 - 3.0 * ar - std::sqrt(-3.0 * ((1.0 - ar) * (1.0 - ar)) + 1.0));
  return (1.0 / 3.0) * (1.0 + std::sqrt(-3.0 * (r * r) + 1.0));
}

inline void cross(const double* u, const double* v, double* w) {
  // math.f90:361-375 vcross
  w[0] = u[1] * v[2] - u[2] * v[1];
  w[1] = u[2] * v[0] - u[0] * v[2];
  w[2] = u[0] * v[1] - u[1] * v[0];
}
inline double dot(const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; }

// The tensors of the bending terms at one point, in the reference's Fortran
// index order through 1-based accessors: bcur(b,a) = b_ab, bcurde1(c,b,a) =
// d b_ab / d xi^c, bcurde2(d,c,b,a), conat(b,a) = a^ab, conatd1(l,b,a),
// conatd2(l,lm,b,a), christof(g,b,a), chrisderi(l,lm,b,a) = d christof(lm,b,a)
// / d xi^l.
struct BendTensors {
  double bc[2][2], bd1[2][2][2], bd2[2][2][2][2];
  double ca[2][2], cad1[2][2][2], cad2[2][2][2][2];
  double ch[2][2][2], chd[2][2][2][2];
  double& bcur(int b, int a) { return bc[b - 1][a - 1]; }
  double& bcurde1(int c, int b, int a) { return bd1[c - 1][b - 1][a - 1]; }
  double& bcurde2(int d, int c, int b, int a) { return bd2[d - 1][c - 1][b - 1][a - 1]; }
  double& conat(int b, int a) { return ca[b - 1][a - 1]; }
  double& conatd1(int l, int b, int a) { return cad1[l - 1][b - 1][a - 1]; }
  double& conatd2(int l, int m, int b, int a) { return cad2[l - 1][m - 1][b - 1][a - 1]; }
  double& christof(int g, int b, int a) { return ch[g - 1][b - 1][a - 1]; }
  double& chrisderi(int l, int m, int b, int a) { return chd[l - 1][m - 1][b - 1][a - 1]; }
};

// ----------------------------------------------------- capsule geometry -----
// Per-degree state: grids, cached synthesis tables (sph3.f90:46-105 saved
// tables), and the reference-sphere contravariant metric conAR/conARd1
// (sph.f90:16-191 -> cal_contra_metric_deri sph.f90:193-299).
struct Capsule {
  int L, N, nO, mO, nD, mD;
  double R;
  std::vector<double> thO, wO, thD, wD;
  std::vector<double> PD, dPD, d2PD;  // dealias-grid tables [(i*N+m)*N+n]
  std::vector<double> PO, dPO;        // SH-grid tables
  std::vector<double> cosD, sinD;     // cos/sin(m phi_j) on dealias grid [m*mD+j]
  std::vector<double> cosO, sinO;     // on SH grid [m*mO+j]
  std::vector<double> conAR, conARd1; // [pt*4 + (a*2+b)], [pt*8 + al*4 + (a*2+b)]
  std::vector<double> wgtdsinf;       // [i] (independent of j)
  // bending (ibend = 1): third and fourth theta derivatives on the dealias
  // grid, and the reference sphere's tensors conAR, conARd1, conARd2, BR,
  // BRd1, BRd2 (sph.f90:153-161), built on first use
  std::vector<double> d3PD, d4PD;
  std::vector<BendTensors> refB;
};

// Geometry fields on the dealias grid, one point.
struct Geo {
  double a1[3], a2[3], d11[3], d12[3], d22[3];
  double n[3], sm, nde[2][3];
  double c1[3], c2[3], cd1[2][3], cd2[2][3];
  double cat[3], catd1[2][3];   // (11,22,12)
  double conat[3], conatd1[2][3];
  double bcur[3];               // (11,22,12)
  double chf[8];                // christof(g,b,a) at [(g-1)+2*(b-1)+4*(a-1)]
};

// cal_co_tang_basis2 (sph3.f90:111-134, ibend=0) for all dealias points.
void synth_basis(const Capsule& C, const double* a, const double* b, std::vector<double>& out15) {
  const int N = C.N, nD = C.nD, mD = C.mD;
  out15.assign((size_t)nD * mD * 15, 0.0);
  for (int i = 0; i < nD; ++i)
    for (int j = 0; j < mD; ++j) {
      double* o = &out15[((size_t)i * mD + j) * 15];
      for (int m = 0; m < N; ++m) {
        double cm = C.cosD[(size_t)m * mD + j], sm = C.sinD[(size_t)m * mD + j];
        const double* P = &C.PD[((size_t)i * N + m) * N];
        const double* P1 = &C.dPD[((size_t)i * N + m) * N];
        const double* P2 = &C.d2PD[((size_t)i * N + m) * N];
        double h = (m == 0) ? 0.5 : 1.0;   // sph3.f90:69-71
        for (int n = m; n < N; ++n) {
          for (int c = 0; c < 3; ++c) {
            double am = a[(size_t)c * N * N + (size_t)m * N + n];
            double bm = b[(size_t)c * N * N + (size_t)m * N + n];
            double t0 = am * cm - bm * sm;
            double t1 = m * (am * (-sm) - bm * cm);
            double t2 = -(double)m * m * t0;
            o[0 + c] += h * P1[n] * t0;   // vat1
            o[3 + c] += h * P[n] * t1;    // vat2
            o[6 + c] += h * P2[n] * t0;   // deFvat1(:,1)
            o[9 + c] += h * P1[n] * t1;   // deFvat1(:,2)
            o[12 + c] += h * P[n] * t2;   // deFvat2(:,2)
          }
        }
      }
    }
}

// cal_co_tang_basis2 with ibend = 1 (sph3.f90:137-180): the 15 values of
// synth_basis, then cdeSvat(:,1..4) (12) and cdeTvat(:,1..5) (15) per point.
void synth_basis_bend(const Capsule& C, const double* a, const double* b, std::vector<double>& out42) {
  const int N = C.N, nD = C.nD, mD = C.mD;
  out42.assign((size_t)nD * mD * 42, 0.0);
  for (int i = 0; i < nD; ++i)
    for (int j = 0; j < mD; ++j) {
      double* o = &out42[((size_t)i * mD + j) * 42];
      for (int m = 0; m < N; ++m) {
        double cm = C.cosD[(size_t)m * mD + j], sm = C.sinD[(size_t)m * mD + j];
        const size_t t = ((size_t)i * N + m) * N;
        const double *P = &C.PD[t], *P1 = &C.dPD[t], *P2 = &C.d2PD[t], *P3 = &C.d3PD[t], *P4 = &C.d4PD[t];
        double h = (m == 0) ? 0.5 : 1.0;  // sph3.f90:98-102
        for (int n = m; n < N; ++n) {
          for (int c = 0; c < 3; ++c) {
            double am = a[(size_t)c * N * N + (size_t)m * N + n];
            double bm = b[(size_t)c * N * N + (size_t)m * N + n];
            double t0 = am * cm - bm * sm;
            double t1 = m * (am * (-sm) - bm * cm);
            double t2 = -(double)m * m * t0;
            double t3 = (double)m * m * m * (am * sm + bm * cm);
            double t4 = (double)m * m * m * m * t0;
            o[0 + c] += h * P1[n] * t0;   // vat1
            o[3 + c] += h * P[n] * t1;    // vat2
            o[6 + c] += h * P2[n] * t0;   // deFvat1(:,1)
            o[9 + c] += h * P1[n] * t1;   // deFvat1(:,2)
            o[12 + c] += h * P[n] * t2;   // deFvat2(:,2)
            o[15 + c] += h * P3[n] * t0;  // deSvat(:,1)
            o[18 + c] += h * P2[n] * t1;  // deSvat(:,2)
            o[21 + c] += h * P1[n] * t2;  // deSvat(:,3)
            o[24 + c] += h * P[n] * t3;   // deSvat(:,4)
            o[27 + c] += h * P4[n] * t0;  // deTvat(:,1)
            o[30 + c] += h * P3[n] * t1;  // deTvat(:,2)
            o[33 + c] += h * P2[n] * t2;  // deTvat(:,3)
            o[36 + c] += h * P1[n] * t3;  // deTvat(:,4)
            o[39 + c] += h * P[n] * t4;   // deTvat(:,5)
          }
        }
      }
    }
}

// Pointwise geometry: sph1.f90:581-651 (normal), sph.f90:442-476 (curvature),
// sph1.f90:197-297 (contravariant, co2contra capsulesolid.f90:106-146),
// sph.f90:735-893 (christof), sph.f90:896-961 (metrics).
void geometry(const double* f15, Geo& G) {
  for (int c = 0; c < 3; ++c) {
    G.a1[c] = f15[c];
    G.a2[c] = f15[3 + c];
    G.d11[c] = f15[6 + c];
    G.d12[c] = f15[9 + c];
    G.d22[c] = f15[12 + c];
  }
  const double* cd1[2] = {G.d11, G.d12};  // cderi1(:,al)
  const double* cd2[2] = {G.d12, G.d22};  // cderi2(:,al)
  double cc[3];
  cross(G.a1, G.a2, cc);
  G.sm = std::sqrt(cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2]);
  for (int c = 0; c < 3; ++c) G.n[c] = cc[c] / G.sm;
  for (int al = 0; al < 2; ++al) {
    double x1[3], x2[3], dc[3];
    cross(cd1[al], G.a2, x1);
    cross(G.a1, cd2[al], x2);
    for (int c = 0; c < 3; ++c) dc[c] = x1[c] + x2[c];
    double tmp = dot(cc, dc) / std::sqrt(cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2]);
    for (int c = 0; c < 3; ++c) G.nde[al][c] = 1.0 / G.sm * (x1[c] + x2[c] - tmp * G.n[c]);
  }
  G.bcur[0] = dot(G.n, G.d11);
  G.bcur[1] = dot(G.n, G.d22);
  G.bcur[2] = dot(G.n, G.d12);
  // co2contra
  double a2n[3], na1[3];
  cross(G.a2, G.n, a2n);
  cross(G.n, G.a1, na1);
  double hyb1 = dot(G.a1, a2n);
  double hyb2 = dot(G.a2, na1);
  for (int c = 0; c < 3; ++c) {
    G.c1[c] = a2n[c] / hyb1;
    G.c2[c] = na1[c] / hyb2;
  }
  double g = dot(G.a1, a2n);
  for (int al = 0; al < 2; ++al) {
    double a2de_n3[3], a2_n3de[3], n3de_a1[3], n3_a1de[3], vt[3];
    cross(cd2[al], G.n, a2de_n3);
    cross(G.a2, G.nde[al], a2_n3de);
    cross(G.nde[al], G.a1, n3de_a1);
    cross(G.n, cd1[al], n3_a1de);
    for (int c = 0; c < 3; ++c) vt[c] = a2de_n3[c] + a2_n3de[c];
    double gde = dot(cd1[al], a2n) + dot(G.a1, vt);
    for (int c = 0; c < 3; ++c) {
      G.cd1[al][c] = 1.0 / g * (-gde * G.c1[c] + a2de_n3[c] + a2_n3de[c]);
      G.cd2[al][c] = 1.0 / g * (-gde * G.c2[c] + n3de_a1[c] + n3_a1de[c]);
    }
  }
  // christof(gamma,beta,alpha) = a_{alpha,gamma} . a^beta
  auto CH = [&](int gg, int bb, int aa) -> double& { return G.chf[(gg - 1) + 2 * (bb - 1) + 4 * (aa - 1)]; };
  CH(1, 1, 1) = dot(G.d11, G.c1);
  CH(2, 1, 1) = dot(G.d12, G.c1);
  CH(1, 2, 1) = dot(G.d11, G.c2);
  CH(2, 2, 1) = dot(G.d12, G.c2);
  CH(2, 1, 2) = dot(G.d22, G.c1);
  CH(2, 2, 2) = dot(G.d22, G.c2);
  CH(1, 1, 2) = CH(2, 1, 1);
  CH(1, 2, 2) = CH(2, 2, 1);
  // cal_metric_deri (covariant)
  G.cat[0] = G.a1[0] * G.a1[0] + G.a1[1] * G.a1[1] + G.a1[2] * G.a1[2];
  G.cat[1] = G.a2[0] * G.a2[0] + G.a2[1] * G.a2[1] + G.a2[2] * G.a2[2];
  G.cat[2] = dot(G.a1, G.a2);
  for (int al = 0; al < 2; ++al) {
    G.catd1[al][0] = 2 * dot(G.a1, cd1[al]);
    G.catd1[al][1] = 2 * dot(G.a2, cd2[al]);
    G.catd1[al][2] = dot(G.a1, cd2[al]) + dot(G.a2, cd1[al]);
  }
  // cal_metric_deri (contravariant)
  G.conat[0] = G.c1[0] * G.c1[0] + G.c1[1] * G.c1[1] + G.c1[2] * G.c1[2];
  G.conat[1] = G.c2[0] * G.c2[0] + G.c2[1] * G.c2[1] + G.c2[2] * G.c2[2];
  G.conat[2] = dot(G.c1, G.c2);
  for (int al = 0; al < 2; ++al) {
    G.conatd1[al][0] = 2 * dot(G.c1, G.cd1[al]);
    G.conatd1[al][1] = 2 * dot(G.c2, G.cd2[al]);
    G.conatd1[al][2] = dot(G.c1, G.cd2[al]) + dot(G.c2, G.cd1[al]);
  }
}

// Strain-energy derivatives of the membrane law (membmodel.c, selected there
// at compile time: -DSKALAK or -DNONHOOK): W1 = dW/dI1, W2 = dW/dI2 and their
// derivatives along xi_1, xi_2.  law 0: Skalak, calpwspi_deri_sk
// (membmodel.c:81-99); law 1: neo-Hookean, calpwspi_deri_nh (:60-79).
void membrane_law(int law, double hf, double csk, double I1, double I2, const double* I1de, const double* I2de,
                  double& W1, double& W2, double* W1de, double* W2de) {
  if (law == 1) {
    const double gs = 2.0 * hf;
    W1 = hf;
    W2 = -hf * std::pow(I2 + 1, -2);
    const double coeff = gs * std::pow(I2 + 1, -3);
    for (int al = 0; al < 2; ++al) {
      W1de[al] = 0;
      W2de[al] = coeff * I2de[al];
    }
    return;
  }
  W1 = hf * (1 + I1);
  W2 = hf * (csk * I2 - 1);
  for (int al = 0; al < 2; ++al) {
    W1de[al] = hf * I1de[al];
    W2de[al] = csk * hf * I2de[al];
  }
}

// Mechanics at one point: sph.f90:1668-1715 with cal_Js_I1_I2_deri
// (sph.f90:1115-1156), the membrane law (membrane_law) and
// calculate_cauchy_tensor_deri (sph.f90:1179-1234).  A* = reference (conAR).
struct BendQ {  // bending terms of the equilibrium (sph.f90:1705-1709)
  double bm[2][2];  // bcurmix(be,al) at [be-1][al-1]
  double Q[2], Qcode;
};
void mechanics(const Geo& G, const double* A, const double* Ad, double hf, double csk, int law, double* f,
               const BendQ* bq = nullptr) {
  const double A11 = A[0], A22 = A[3], A12 = A[1];
  const double c11 = G.cat[0], c22 = G.cat[1], c12 = G.cat[2];
  double abs_conA = A11 * A22 - A12 * A12;
  double abs_ca = c11 * c22 - c12 * c12;
  double I1 = A11 * c11 + A22 * c22 + 2 * A12 * c12 - 2;
  double I2 = abs_conA * abs_ca - 1;
  double Js = std::sqrt(1 + I2);
  double I1de[2], I2de[2], Jsde[2];
  for (int al = 0; al < 2; ++al) {
    double Ad11 = Ad[al * 4 + 0], Ad22 = Ad[al * 4 + 3], Ad12 = Ad[al * 4 + 1];
    double cd11 = G.catd1[al][0], cd22 = G.catd1[al][1], cd12 = G.catd1[al][2];
    I1de[al] = Ad11 * c11 + A11 * cd11 + Ad22 * c22 + A22 * cd22 + 2 * (Ad12 * c12 + A12 * cd12);
    double abs_conAd = Ad11 * A22 + A11 * Ad22 - 2 * A12 * Ad12;
    double abs_cad = cd11 * c22 + c11 * cd22 - 2 * c12 * cd12;
    I2de[al] = abs_conAd * abs_ca + abs_cad * abs_conA;
  }
  for (int al = 0; al < 2; ++al) Jsde[al] = 0.5 / Js * I2de[al];
  double W1, W2, W1de[2], W2de[2];
  membrane_law(law, hf, csk, I1, I2, I1de, I2de, W1, W2, W1de, W2de);
  // Cauchy tension and derivatives
  double coef1 = 2. / Js * W1, coef2 = 2. * Js * W2;
  double a11 = G.conat[0], a22 = G.conat[1], a12 = G.conat[2];
  double T11 = coef1 * A11 + coef2 * a11;
  double T22 = coef1 * A22 + coef2 * a22;
  double T12 = coef1 * A12 + coef2 * a12;
  double Td11[2], Td22[2], Td12[2];
  for (int al = 0; al < 2; ++al) {
    double v1 = -2.0 / (Js * Js) * Jsde[al] * W1;
    double v2 = 2.0 / Js * W1de[al];
    double v3 = 2.0 / Js * W1;
    double v4 = 2.0 * Jsde[al] * W2;
    double v5 = 2.0 * Js * W2de[al];
    double v6 = 2.0 * Js * W2;
    double Ad11 = Ad[al * 4 + 0], Ad22 = Ad[al * 4 + 3], Ad12 = Ad[al * 4 + 1];
    Td11[al] = v1 * A11 + v2 * A11 + v3 * Ad11 + v4 * a11 + v5 * a11 + v6 * G.conatd1[al][0];
    Td22[al] = v1 * A22 + v2 * A22 + v3 * Ad22 + v4 * a22 + v5 * a22 + v6 * G.conatd1[al][1];
    Td12[al] = v1 * A12 + v2 * A12 + v3 * Ad12 + v4 * a12 + v5 * a12 + v6 * G.conatd1[al][2];
  }
  auto ch = [&](int gg, int bb, int aa) -> double { return G.chf[(gg - 1) + 2 * (bb - 1) + 4 * (aa - 1)]; };
  double q1 = Td11[0] + Td12[1] + ch(1, 1, 1) * T11 + ch(2, 1, 1) * T12 + ch(1, 2, 2) * T11 + ch(2, 2, 2) * T12 +
              ch(1, 1, 1) * T11 + ch(2, 1, 1) * T12 + ch(1, 1, 2) * T12 + ch(2, 1, 2) * T22;
  double q2 = Td12[0] + Td22[1] + ch(1, 1, 1) * T12 + ch(2, 1, 1) * T22 + ch(1, 2, 2) * T12 + ch(2, 2, 2) * T22 +
              ch(1, 2, 1) * T11 + ch(2, 2, 1) * T12 + ch(1, 2, 2) * T12 + ch(2, 2, 2) * T22;
  double q3 = T11 * G.bcur[0] + T22 * G.bcur[1] + 2 * T12 * G.bcur[2];
  if (bq) {  // ibend = 1 (sph.f90:1705-1709)
    q1 = q1 - bq->bm[0][0] * bq->Q[0] - bq->bm[1][0] * bq->Q[1];
    q2 = q2 - bq->bm[0][1] * bq->Q[0] - bq->bm[1][1] * bq->Q[1];
    q3 = q3 + bq->Qcode;
  }
  for (int c = 0; c < 3; ++c) f[c] = q1 * G.a1[c] + q2 * G.a2[c] + q3 * G.n[c];
}

// ---------------------------------------------------- bending (ibend = 1) ---
// cal_curvature_derivative (sph.f90:479-731), cal_contra_second_derivative
// (sph1.f90:299-542), the ibend part of cal_christof (sph.f90:802-890) and
// cal_contra_metric_second_deri (sph.f90:962-1111) at one point, from the
// geometry G and the synthesised third (S: x_ttt, x_ttp, x_tpp, x_ppp) and
// fourth (T: x_tttt, x_tttp, x_ttpp, x_tppp, x_pppp) derivatives, with the
// reference's expressions term for term (including its chrisderi(2,2,1,2),
// whose second product is cderi1(:,2) . conderi2(:,2)).
void bend_tensors(const Geo& G, const double (*S)[3], const double (*T)[3], BendTensors& B) {
  const double* cderi1[2] = {G.d11, G.d12};
  const double* cderi2[2] = {G.d12, G.d22};
  const double* cderi3[2] = {G.nde[0], G.nde[1]};
  const double* conderi1[2] = {G.cd1[0], G.cd1[1]};
  const double* conderi2[2] = {G.cd2[0], G.cd2[1]};
  const double* n = G.n;
  const double *c1 = G.c1, *c2 = G.c2;
  B.bcur(1, 1) = G.bcur[0];
  B.bcur(2, 2) = G.bcur[1];
  B.bcur(1, 2) = B.bcur(2, 1) = G.bcur[2];
  B.conat(1, 1) = G.conat[0];
  B.conat(2, 2) = G.conat[1];
  B.conat(1, 2) = B.conat(2, 1) = G.conat[2];
  for (int al = 1; al <= 2; ++al) {
    B.conatd1(al, 1, 1) = G.conatd1[al - 1][0];
    B.conatd1(al, 2, 2) = G.conatd1[al - 1][1];
    B.conatd1(al, 1, 2) = B.conatd1(al, 2, 1) = G.conatd1[al - 1][2];
  }
  for (int g = 1; g <= 2; ++g)
    for (int b = 1; b <= 2; ++b)
      for (int a = 1; a <= 2; ++a) B.christof(g, b, a) = G.chf[(g - 1) + 2 * (b - 1) + 4 * (a - 1)];
  // ---- cal_curvature_derivative
  B.bcurde1(1, 1, 1) = dot(S[0], n) + dot(cderi1[0], cderi3[0]);
  B.bcurde1(2, 1, 1) = dot(S[1], n) + dot(cderi1[0], cderi3[1]);
  B.bcurde1(1, 2, 2) = dot(S[2], n) + dot(cderi2[1], cderi3[0]);
  B.bcurde1(2, 2, 2) = dot(S[3], n) + dot(cderi2[1], cderi3[1]);
  B.bcurde1(1, 1, 2) = dot(S[1], n) + dot(cderi2[0], cderi3[0]);
  B.bcurde1(1, 2, 1) = B.bcurde1(1, 1, 2);
  B.bcurde1(2, 1, 2) = dot(S[2], n) + dot(cderi2[0], cderi3[1]);
  B.bcurde1(2, 2, 1) = B.bcurde1(2, 1, 2);
  double nS[3][3];  // cderiS3(:,1..3): n_tt, n_pp, n_tp
  for (int c = 0; c < 3; ++c) {
    nS[0][c] = -(B.bcurde1(1, 1, 1) * c1[c] + B.bcurde1(1, 2, 1) * c2[c] + B.bcur(1, 1) * conderi1[0][c] +
                 B.bcur(1, 2) * conderi2[0][c]);
    nS[1][c] = -(B.bcurde1(2, 1, 2) * c1[c] + B.bcurde1(2, 2, 2) * c2[c] + B.bcur(2, 1) * conderi1[1][c] +
                 B.bcur(2, 2) * conderi2[1][c]);
    nS[2][c] = -(B.bcurde1(2, 1, 1) * c1[c] + B.bcurde1(2, 2, 1) * c2[c] + B.bcur(1, 1) * conderi1[1][c] +
                 B.bcur(1, 2) * conderi2[1][c]);
  }
  auto bd2 = [&](const double* t, const double* s1, const double* n1, const double* s2, const double* n2,
                 const double* x, const double* ns) { return dot(t, n) + dot(s1, n1) + dot(s2, n2) + dot(x, ns); };
  B.bcurde2(1, 1, 1, 1) = bd2(T[0], S[0], cderi3[0], S[0], cderi3[0], cderi1[0], nS[0]);
  B.bcurde2(2, 1, 1, 1) = bd2(T[1], S[0], cderi3[1], S[1], cderi3[0], cderi1[0], nS[2]);
  B.bcurde2(1, 2, 1, 1) = B.bcurde2(2, 1, 1, 1);
  B.bcurde2(2, 2, 1, 1) = bd2(T[2], S[1], cderi3[1], S[1], cderi3[1], cderi1[0], nS[1]);
  B.bcurde2(1, 1, 2, 2) = bd2(T[2], S[2], cderi3[0], S[2], cderi3[0], cderi2[1], nS[0]);
  B.bcurde2(2, 1, 2, 2) = bd2(T[3], S[2], cderi3[1], S[3], cderi3[0], cderi2[1], nS[2]);
  B.bcurde2(1, 2, 2, 2) = B.bcurde2(2, 1, 2, 2);
  B.bcurde2(2, 2, 2, 2) = bd2(T[4], S[3], cderi3[1], S[3], cderi3[1], cderi2[1], nS[1]);
  B.bcurde2(1, 1, 2, 1) = bd2(T[1], S[1], cderi3[0], S[1], cderi3[0], cderi1[1], nS[0]);
  B.bcurde2(1, 1, 1, 2) = B.bcurde2(1, 1, 2, 1);
  B.bcurde2(2, 1, 2, 1) = bd2(T[2], S[1], cderi3[1], S[2], cderi3[0], cderi1[1], nS[2]);
  B.bcurde2(1, 2, 2, 1) = B.bcurde2(2, 1, 2, 1);
  B.bcurde2(2, 1, 1, 2) = B.bcurde2(2, 1, 2, 1);
  B.bcurde2(1, 2, 1, 2) = B.bcurde2(2, 1, 2, 1);
  B.bcurde2(2, 2, 2, 1) = bd2(T[3], S[2], cderi3[1], S[2], cderi3[1], cderi1[1], nS[1]);
  B.bcurde2(2, 2, 1, 2) = B.bcurde2(2, 2, 2, 1);
  // ---- cal_contra_second_derivative: condeS1(:,1..3), condeS2(:,1..3)
  double cS1[3][3], cS2[3][3];
  {
    const double* a1 = G.a1;
    const double* a2 = G.a2;
    const double* a1de[2] = {cderi1[0], cderi1[1]};
    const double* a2de[2] = {cderi2[0], cderi2[1]};
    const double* n3de[2] = {cderi3[0], cderi3[1]};
    // adeS = cdeSvat: adeS(:,1) = S[0] (a1_tt), (:,2) = S[1], (:,3) = S[2], (:,4) = S[3]
    double a2_n3[3], n3_a1[3], a2de_n3[2][3], a2_n3de[2][3], n3de_a1[2][3], n3_a1de[2][3];
    cross(a2, n, a2_n3);
    cross(n, a1, n3_a1);
    for (int al = 0; al < 2; ++al) {
      cross(a2de[al], n, a2de_n3[al]);
      cross(a2, n3de[al], a2_n3de[al]);
      cross(n3de[al], a1, n3de_a1[al]);
      cross(n, a1de[al], n3_a1de[al]);
    }
    const double g = dot(a1, a2_n3);
    double gde[2], gdeS[3];
    for (int al = 0; al < 2; ++al) {
      double vt[3];
      for (int c = 0; c < 3; ++c) vt[c] = a2de_n3[al][c] + a2_n3de[al][c];
      gde[al] = dot(a1de[al], a2_n3) + dot(a1, vt);
    }
    double a2_n3deS[3][3], a2de_n3de[2][2][3], a2deS_n3[3][3], n3_a1deS[3][3], n3de_a1de[2][2][3], n3deS_a1[3][3];
    for (int al = 0; al < 3; ++al) cross(a2, nS[al], a2_n3deS[al]);
    for (int al = 0; al < 2; ++al)
      for (int al2 = 0; al2 < 2; ++al2) cross(a2de[al], n3de[al2], a2de_n3de[al][al2]);  // (:,al2,al)
    cross(S[1], n, a2deS_n3[0]);
    cross(S[3], n, a2deS_n3[1]);
    cross(S[2], n, a2deS_n3[2]);
    cross(n, S[0], n3_a1deS[0]);
    cross(n, S[2], n3_a1deS[1]);
    cross(n, S[1], n3_a1deS[2]);
    for (int al = 0; al < 2; ++al)
      for (int al2 = 0; al2 < 2; ++al2) cross(n3de[al], a1de[al2], n3de_a1de[al][al2]);  // (:,al2,al)
    for (int al = 0; al < 3; ++al) cross(nS[al], a1, n3deS_a1[al]);
    // gdeS(1..3): tt, pp, tp.  X(:,al2,al) is stored X[al][al2].
    auto gdes = [&](const double* adeS_, int i1, int i2, int ia, int ib, const double* v3) {
      double v1[3], v2[3];
      for (int c = 0; c < 3; ++c) {
        v1[c] = a2de_n3[ia][c] + a2_n3de[ia][c];
        v2[c] = a2de_n3[ib][c] + a2_n3de[ib][c];
      }
      return dot(adeS_, a2_n3) + dot(a1de[i1], v1) + dot(a1de[i2], v2) + dot(a1, v3);
    };
    double v3[3][3];
    for (int c = 0; c < 3; ++c) {
      v3[0][c] = a2deS_n3[0][c] + a2de_n3de[0][0][c] + a2de_n3de[0][0][c] + a2_n3deS[0][c];
      v3[1][c] = a2deS_n3[1][c] + a2de_n3de[1][1][c] + a2de_n3de[1][1][c] + a2_n3deS[1][c];
      v3[2][c] = a2deS_n3[2][c] + a2de_n3de[0][1][c] + a2de_n3de[1][0][c] + a2_n3deS[2][c];
    }
    gdeS[0] = gdes(S[0], 0, 0, 0, 0, v3[0]);
    gdeS[1] = gdes(S[2], 1, 1, 1, 1, v3[1]);
    gdeS[2] = gdes(S[1], 0, 1, 1, 0, v3[2]);
    const double ginv1 = 1. / g, ginv2 = ginv1 * ginv1, ginv3 = ginv1 * ginv2;
    // (index pairs of the three second derivatives: tt -> (1,1), pp -> (2,2), tp -> (1,2))
    const int I[3] = {0, 1, 0}, J[3] = {0, 1, 1};
    for (int k = 0; k < 3; ++k) {
      const int i = I[k], j = J[k];
      double w1[3], w2[3];
      for (int c = 0; c < 3; ++c) {
        w1[c] = a2deS_n3[k][c] + a2de_n3de[i][j][c] + a2de_n3de[j][i][c] + a2_n3deS[k][c];
        w2[c] = n3deS_a1[k][c] + n3de_a1de[i][j][c] + n3de_a1de[j][i][c] + n3_a1deS[k][c];
      }
      // condeS1(:,1) = 2 ginv3 gde(1) gde(1) a2_n3 - ginv2 gdeS(1) a2_n3 - ginv2 gde(1)(..)(:,1)
      //               - ginv2 gde(1)(..)(:,1) + ginv1 (...); the tp entry pairs gde(2)gde(1),
      //               gde(1) with (:,2) and gde(2) with (:,1)
      const double gg = k == 2 ? gde[1] * gde[0] : gde[i] * gde[i];
      for (int c = 0; c < 3; ++c) {
        cS1[k][c] = 2 * ginv3 * gg * a2_n3[c] - ginv2 * gdeS[k] * a2_n3[c] -
                    ginv2 * gde[i] * (a2de_n3[j][c] + a2_n3de[j][c]) -
                    ginv2 * gde[j] * (a2de_n3[i][c] + a2_n3de[i][c]) + ginv1 * w1[c];
        cS2[k][c] = 2 * ginv3 * gg * n3_a1[c] - ginv2 * gdeS[k] * n3_a1[c] -
                    ginv2 * gde[i] * (n3de_a1[j][c] + n3_a1de[j][c]) -
                    ginv2 * gde[j] * (n3de_a1[i][c] + n3_a1de[i][c]) + ginv1 * w2[c];
      }
    }
  }
  // ---- cal_christof, ibend part
  auto CD = [&](const double* sv, const double* cv, const double* xd, const double* cd) {
    return dot(sv, cv) + dot(xd, cd);
  };
  B.chrisderi(1, 1, 1, 1) = CD(S[0], c1, cderi1[0], conderi1[0]);
  B.chrisderi(2, 1, 1, 1) = CD(S[1], c1, cderi1[0], conderi1[1]);
  B.chrisderi(1, 2, 1, 1) = CD(S[1], c1, cderi1[1], conderi1[0]);
  B.chrisderi(2, 2, 1, 1) = CD(S[2], c1, cderi1[1], conderi1[1]);
  B.chrisderi(1, 1, 2, 1) = CD(S[0], c2, cderi1[0], conderi2[0]);
  B.chrisderi(2, 1, 2, 1) = CD(S[1], c2, cderi1[0], conderi2[1]);
  B.chrisderi(1, 2, 2, 1) = CD(S[1], c2, cderi1[1], conderi2[0]);
  B.chrisderi(2, 2, 2, 1) = CD(S[2], c2, cderi1[1], conderi2[1]);
  B.chrisderi(1, 2, 1, 2) = CD(S[2], c1, cderi2[1], conderi1[0]);
  B.chrisderi(2, 2, 1, 2) = CD(S[3], c1, cderi1[1], conderi2[1]);  // as the reference writes it
  B.chrisderi(1, 2, 2, 2) = CD(S[2], c2, cderi2[1], conderi2[0]);
  B.chrisderi(2, 2, 2, 2) = CD(S[3], c2, cderi2[1], conderi2[1]);
  for (int l = 1; l <= 2; ++l)
    for (int b = 1; b <= 2; ++b) B.chrisderi(l, 1, b, 2) = B.chrisderi(l, 2, b, 1);
  // ---- cal_contra_metric_second_deri: conatd2(l,lm,b,a), a^a_{lm l} . a^b + ...
  const double* cv[2] = {c1, c2};
  const double* cdv[2][2] = {{conderi1[0], conderi1[1]}, {conderi2[0], conderi2[1]}};  // [vec][al]
  const double* cSv[2][3] = {{cS1[0], cS1[1], cS1[2]}, {cS2[0], cS2[1], cS2[2]}};   // [vec][tt,pp,tp]
  auto CM = [&](int va, int vb, int s, int l1, int l2) {
    return dot(cSv[va][s], cv[vb]) + dot(cdv[va][l1], cdv[vb][l2]) + dot(cdv[va][l2], cdv[vb][l1]) +
           dot(cv[va], cSv[vb][s]);
  };
  B.conatd2(1, 1, 1, 1) = CM(0, 0, 0, 0, 0);
  B.conatd2(2, 2, 1, 1) = CM(0, 0, 1, 1, 1);
  B.conatd2(2, 1, 1, 1) = CM(0, 0, 2, 0, 1);
  B.conatd2(1, 2, 1, 1) = B.conatd2(2, 1, 1, 1);
  B.conatd2(1, 1, 2, 2) = CM(1, 1, 0, 0, 0);
  B.conatd2(2, 2, 2, 2) = CM(1, 1, 1, 1, 1);
  B.conatd2(2, 1, 2, 2) = CM(1, 1, 2, 0, 1);
  B.conatd2(1, 2, 2, 2) = B.conatd2(2, 1, 2, 2);
  B.conatd2(2, 1, 2, 1) = CM(0, 1, 2, 0, 1);
  B.conatd2(1, 2, 2, 1) = B.conatd2(2, 1, 2, 1);
  B.conatd2(2, 1, 1, 2) = B.conatd2(2, 1, 2, 1);
  B.conatd2(1, 2, 1, 2) = B.conatd2(2, 1, 2, 1);
  B.conatd2(1, 1, 2, 1) = CM(0, 1, 0, 0, 0);
  B.conatd2(1, 1, 1, 2) = B.conatd2(1, 1, 2, 1);
  B.conatd2(2, 2, 2, 1) = CM(0, 1, 1, 1, 1);
  B.conatd2(2, 2, 1, 2) = B.conatd2(2, 2, 2, 1);
}

// cal_moment_deri (sph.f90:1236-1372), cal_Q (:1375-1424) and cal_bcurmix
// (:1427-1454) at one point: X the deformed surface, R the reference
// sphere (conAR.., BR.. of sph.f90:153-161), EB the bending modulus.
void bend_q(BendTensors& X, BendTensors& R, double EB, BendQ& out) {
  double mom[2][2] = {{0, 0}, {0, 0}}, momdF[2][2][2] = {}, momdS = 0;
  auto a = [&](int i, int j) { return X.conat(i, j); };
  auto ad1 = [&](int i, int j, int k) { return X.conatd1(i, j, k); };
  auto ad2 = [&](int i, int j, int k, int l) { return X.conatd2(i, j, k, l); };
  auto b = [&](int i, int j) { return X.bcur(i, j); };
  auto bd1 = [&](int i, int j, int k) { return X.bcurde1(i, j, k); };
  auto bd2 = [&](int i, int j, int k, int l) { return X.bcurde2(i, j, k, l); };
  auto AR = [&](int i, int j) { return R.conat(i, j); };
  auto ARd1 = [&](int i, int j, int k) { return R.conatd1(i, j, k); };
  auto ARd2 = [&](int i, int j, int k, int l) { return R.conatd2(i, j, k, l); };
  auto BRI = [&](int i, int j) { return R.bcur(i, j); };
  auto BRId1 = [&](int i, int j, int k) { return R.bcurde1(i, j, k); };
  auto BRId2 = [&](int i, int j, int k, int l) { return R.bcurde2(i, j, k, l); };
  for (int al = 1; al <= 2; ++al)
    for (int be = 1; be <= 2; ++be) {
      for (int gam = 1; gam <= 2; ++gam)
        for (int gamp = 1; gamp <= 2; ++gamp)
          momdS = momdS + ad2(be, al, be, gam) * (AR(gamp, al) * BRI(gam, gamp) - a(gamp, al) * b(gam, gamp)) +
                  ad1(al, be, gam) * (ARd1(be, gamp, al) * BRI(gam, gamp) + AR(gamp, al) * BRId1(be, gam, gamp) -
                                      ad1(be, gamp, al) * b(gam, gamp) - a(gamp, al) * bd1(be, gam, gamp)) +
                  ad1(be, be, gam) * (ARd1(al, gamp, al) * BRI(gam, gamp) + AR(gamp, al) * BRId1(al, gam, gamp) -
                                      ad1(al, gamp, al) * b(gam, gamp) - a(gamp, al) * bd1(al, gam, gamp)) +
                  a(be, gam) * (ARd2(be, al, gamp, al) * BRI(gam, gamp) + ARd1(al, gamp, al) * BRId1(be, gam, gamp) +
                                ARd1(be, gamp, al) * BRId1(al, gam, gamp) + AR(gamp, al) * BRId2(be, al, gam, gamp) -
                                ad2(be, al, gamp, al) * b(gam, gamp) - ad1(al, gamp, al) * bd1(be, gam, gamp) -
                                ad1(be, gamp, al) * bd1(al, gam, gamp) - a(gamp, al) * bd2(be, al, gam, gamp));
      if (al == 2 && be == 1) continue;
      for (int gam = 1; gam <= 2; ++gam)
        for (int gamp = 1; gamp <= 2; ++gamp)
          mom[be - 1][al - 1] = mom[be - 1][al - 1] + a(be, gam) * (AR(gamp, al) * BRI(gam, gamp) -
                                                                  a(gamp, al) * b(gam, gamp));
      for (int l = 1; l <= 2; ++l)
        for (int gam = 1; gam <= 2; ++gam)
          for (int gamp = 1; gamp <= 2; ++gamp)
            momdF[l - 1][be - 1][al - 1] =
                momdF[l - 1][be - 1][al - 1] +
                ad1(l, be, gam) * (AR(gamp, al) * BRI(gam, gamp) - a(gamp, al) * b(gam, gamp)) +
                a(be, gam) * (ARd1(l, gamp, al) * BRI(gam, gamp) + AR(gamp, al) * BRId1(l, gam, gamp) -
                              ad1(l, gamp, al) * b(gam, gamp) - a(gamp, al) * bd1(l, gam, gamp));
    }
  mom[0][1] = mom[1][0];
  for (int l = 0; l < 2; ++l) momdF[l][0][1] = momdF[l][1][0];
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) {
      mom[i][j] = mom[i][j] * EB;
      for (int l = 0; l < 2; ++l) momdF[l][i][j] = momdF[l][i][j] * EB;
    }
  momdS = momdS * EB;
  // cal_Q: Q(be), Qcode = Q^be|be
  auto M = [&](int i, int j) { return mom[i - 1][j - 1]; };
  auto MF = [&](int l, int i, int j) { return momdF[l - 1][i - 1][j - 1]; };
  auto CH = [&](int g, int bb, int aa) { return X.christof(g, bb, aa); };
  auto CHD = [&](int l, int g, int bb, int aa) { return X.chrisderi(l, g, bb, aa); };
  double Q[2] = {0, 0}, Qcode = momdS;
  for (int be = 1; be <= 2; ++be)
    for (int al = 1; al <= 2; ++al) {
      Q[be - 1] = Q[be - 1] + MF(al, be, al);
      for (int lm = 1; lm <= 2; ++lm) {
        Q[be - 1] = Q[be - 1] + CH(lm, al, al) * M(be, lm) + CH(lm, be, al) * M(lm, al);
        Qcode = Qcode + CHD(be, lm, al, al) * M(be, lm) + CH(lm, al, al) * MF(be, be, lm) +
                CHD(be, lm, be, al) * M(lm, al) + CH(lm, be, al) * MF(be, lm, al);
      }
    }
  for (int be = 1; be <= 2; ++be)
    for (int lm = 1; lm <= 2; ++lm) Qcode = Qcode + Q[lm - 1] * CH(lm, be, be);
  // cal_bcurmix: bcurmix(be,al) = sum_lm conat(lm,al) bcur(be,lm)
  for (int al = 1; al <= 2; ++al)
    for (int be = 1; be <= 2; ++be) {
      double v = 0;
      for (int lm = 1; lm <= 2; ++lm) v = v + a(lm, al) * b(be, lm);
      out.bm[be - 1][al - 1] = v;
    }
  out.Q[0] = Q[0];
  out.Q[1] = Q[1];
  out.Qcode = Qcode;
}

// Reference-sphere setup (capsule_init_cal_coeff, sph.f90:16-191).
std::shared_ptr<Capsule> build_capsule(int L, double R) {
  auto C = std::make_shared<Capsule>();
  C->L = L;
  C->N = L + 1;
  C->R = R;
  const int N = C->N;
  C->nO = N;
  C->mO = 2 * N;
  C->nD = 2 * N;
  C->mD = 4 * N;
  C->thO.resize(C->nO);
  C->wO.resize(C->nO);
  C->thD.resize(C->nD);
  C->wD.resize(C->nD);
  gauss(C->nO, C->thO.data(), C->wO.data());
  gauss(C->nD, C->thD.data(), C->wD.data());
  std::vector<double> T, D, D2, D3, D4;
  C->PD.assign((size_t)C->nD * N * N, 0.0);
  C->dPD = C->PD;
  C->d2PD = C->PD;
  C->d3PD = C->PD;
  C->d4PD = C->PD;
  for (int i = 0; i < C->nD; ++i) {
    legendre_full4(C->thD[i], N + 2, T, D, D2, D3, D4);
    for (int m = 0; m < N; ++m)
      for (int n = m; n < N; ++n) {
        size_t o = ((size_t)i * N + m) * N + n;
        C->PD[o] = T[(size_t)m * (N + 2) + n];
        C->dPD[o] = D[(size_t)m * (N + 2) + n];
        C->d2PD[o] = D2[(size_t)m * (N + 2) + n];
        C->d3PD[o] = D3[(size_t)m * (N + 2) + n];
        C->d4PD[o] = D4[(size_t)m * (N + 2) + n];
      }
  }
  C->PO.assign((size_t)C->nO * N * N, 0.0);
  C->dPO = C->PO;
  for (int i = 0; i < C->nO; ++i) {
    legendre_full(C->thO[i], N + 2, T, D, D2);
    for (int m = 0; m < N; ++m)
      for (int n = m; n < N; ++n) {
        size_t o = ((size_t)i * N + m) * N + n;
        C->PO[o] = T[(size_t)m * (N + 2) + n];
        C->dPO[o] = D[(size_t)m * (N + 2) + n];
      }
  }
  C->cosD.resize((size_t)N * C->mD);
  C->sinD.resize((size_t)N * C->mD);
  for (int m = 0; m < N; ++m)
    for (int j = 0; j < C->mD; ++j) {
      double phi = j * (2.0 * kPi / C->mD);
      C->cosD[(size_t)m * C->mD + j] = std::cos(m * phi);
      C->sinD[(size_t)m * C->mD + j] = std::sin(m * phi);
    }
  C->cosO.resize((size_t)N * C->mO);
  C->sinO.resize((size_t)N * C->mO);
  for (int m = 0; m < N; ++m)
    for (int j = 0; j < C->mO; ++j) {
      double phi = j * (2.0 * kPi / C->mO);
      C->cosO[(size_t)m * C->mO + j] = std::cos(m * phi);
      C->sinO[(size_t)m * C->mO + j] = std::sin(m * phi);
    }
  // wgtdsinf = w_i / sin(theta_i) * dphi  (sph.f90:129-130)
  C->wgtdsinf.resize(C->nD);
  for (int i = 0; i < C->nD; ++i) C->wgtdsinf[i] = C->wD[i] / std::sin(C->thD[i]) * (2.0 * kPi / C->mD);
  // reference sphere on the SH grid, x=sin t sin p, y=sin t cos p, z=cos t
  std::vector<double> crd((size_t)3 * C->nO * C->mO);
  for (int i = 0; i < C->nO; ++i)
    for (int j = 0; j < C->mO; ++j) {
      double t = C->thO[i], p = j * (2.0 * kPi / C->mO);
      size_t o = (size_t)i * C->mO + j;
      crd[o] = R * std::sin(t) * std::sin(p);
      crd[(size_t)C->nO * C->mO + o] = R * std::sin(t) * std::cos(p);
      crd[(size_t)2 * C->nO * C->mO + o] = R * std::cos(t);
    }
  auto plan = get_plan(C->nO, C->mO, false);
  std::vector<double> a((size_t)3 * N * N), b((size_t)3 * N * N);
  for (int c = 0; c < 3; ++c)
    analysis(*plan, &crd[(size_t)c * C->nO * C->mO], &a[(size_t)c * N * N], &b[(size_t)c * N * N]);
  std::vector<double> f15;
  synth_basis(*C, a.data(), b.data(), f15);
  size_t np = (size_t)C->nD * C->mD;
  C->conAR.resize(np * 4);
  C->conARd1.resize(np * 8);
  Geo G;
  for (size_t p = 0; p < np; ++p) {
    geometry(&f15[p * 15], G);
    C->conAR[p * 4 + 0] = G.conat[0];
    C->conAR[p * 4 + 3] = G.conat[1];
    C->conAR[p * 4 + 1] = G.conat[2];
    C->conAR[p * 4 + 2] = G.conat[2];
    for (int al = 0; al < 2; ++al) {
      C->conARd1[p * 8 + al * 4 + 0] = G.conatd1[al][0];
      C->conARd1[p * 8 + al * 4 + 3] = G.conatd1[al][1];
      C->conARd1[p * 8 + al * 4 + 1] = G.conatd1[al][2];
      C->conARd1[p * 8 + al * 4 + 2] = G.conatd1[al][2];
    }
  }
  // the reference sphere's bending tensors (cal_contra_metric_deri with
  // ibend = 1, sph.f90:153-161, 193-299)
  {
    std::vector<double> f42;
    synth_basis_bend(*C, a.data(), b.data(), f42);
    C->refB.resize(np);
    for (size_t p = 0; p < np; ++p) {
      geometry(&f42[p * 42], G);
      bend_tensors(G, (const double(*)[3]) & f42[p * 42 + 15], (const double(*)[3]) & f42[p * 42 + 27], C->refB[p]);
    }
  }
  return C;
}

std::mutex g_cap_mu;
std::map<std::pair<int, double>, std::shared_ptr<Capsule>> g_caps;
std::shared_ptr<Capsule> get_capsule(int L, double R) {
  std::lock_guard<std::mutex> lk(g_cap_mu);
  auto key = std::make_pair(L, R);
  auto it = g_caps.find(key);
  if (it != g_caps.end()) return it->second;
  auto C = build_capsule(L, R);
  g_caps[key] = C;
  return C;
}

// SH-grid synthesis of degree<N coefficients with the filter tables
// (filter_modes_unitout sph1.f90:688-719, filter_modes4__OPT :919-932):
// identical in form to shsgc on the N x 2N grid.
void filter_synth(const Capsule& C, const double* a, const double* b, int lda, double* out) {
  const int N = C.N, nO = C.nO, mO = C.mO;
  for (int i = 0; i < nO; ++i)
    for (int j = 0; j < mO; ++j) {
      double v = 0.0;
      for (int m = 0; m < N; ++m) {
        const double* P = &C.PO[((size_t)i * N + m) * N];
        double h = (m == 0) ? 0.5 : 1.0;
        double cm = C.cosO[(size_t)m * mO + j], sm = C.sinO[(size_t)m * mO + j];
        for (int n = m; n < N; ++n)
          v += h * P[n] * (a[(size_t)m * lda + n] * cm - b[(size_t)m * lda + n] * sm);
      }
      out[(size_t)i * mO + j] = v;
    }
}

// cal_surface_metric_sph__OPT (sph3.f90:186-277) on the SH grid.
void surface_metric(const Capsule& C, const double* a, const double* b, double* sm) {
  const int N = C.N, nO = C.nO, mO = C.mO;
  for (int i = 0; i < nO; ++i)
    for (int j = 0; j < mO; ++j) {
      double v1[3] = {0, 0, 0}, v2[3] = {0, 0, 0};
      for (int m = 0; m < N; ++m) {
        const double* P = &C.PO[((size_t)i * N + m) * N];
        const double* P1 = &C.dPO[((size_t)i * N + m) * N];
        double h = (m == 0) ? 0.5 : 1.0;
        double cm = C.cosO[(size_t)m * mO + j], smm = C.sinO[(size_t)m * mO + j];
        for (int n = m; n < N; ++n)
          for (int c = 0; c < 3; ++c) {
            double am = a[(size_t)c * N * N + (size_t)m * N + n], bm = b[(size_t)c * N * N + (size_t)m * N + n];
            double t0 = am * cm - bm * smm;
            double t1 = m * (am * (-smm) - bm * cm);
            v1[c] += h * P1[n] * t0;
            v2[c] += h * P[n] * t1;
          }
      }
      double cc[3];
      cross(v1, v2, cc);
      sm[(size_t)i * mO + j] = std::sqrt(cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2]);
    }
}

// complagrforces for one capsule (forcing.f90:11-114 -> cal_spectral_force
// sph.f90:1523-1755).  Optionally returns the shape and filtered-force
// coefficients (degree < N) for the surrogate data path.
int capsule_force(int L, double R, double gs, double csk, int law, bool faithful,
                  const double* xfp, const double* yfp, const double* zfp,
                  double* fxl, double* fyl, double* fzl, double* xn, double* yn, double* zn, double* area,
                  double* shape_a, double* shape_b, double* force_a, double* force_b, double eb = 0.0) {
  if (L < 2 || L > 63 || !(R > 0)) return 1;
  auto Cp = get_capsule(L, R);
  const Capsule& C = *Cp;
  const int N = C.N, nO = C.nO, mO = C.mO, nD = C.nD, mD = C.mD;
  const size_t nF = (size_t)nD * mD, nS = (size_t)nO * mO;
  // The geometry is translation invariant.  Unless `faithful`, the capsule's
  // mean position is subtracted first: a constant offset (e.g. a capsule at
  // (2,1,1) of radius 0.25) otherwise leaks roundoff of order eps*|offset|
  // into every coefficient, which the second-derivative and 1/sin^3 terms
  // amplify to ~2e-9 absolute force on an undeformed sphere.
  std::vector<double> xc(3 * nF);
  {
    double mx = 0, my = 0, mz = 0;
    for (size_t p = 0; p < nF; ++p) { mx += xfp[p]; my += yfp[p]; mz += zfp[p]; }
    mx /= (double)nF; my /= (double)nF; mz /= (double)nF;
    if (faithful) mx = my = mz = 0.0;
    for (size_t p = 0; p < nF; ++p) {
      xc[p] = xfp[p] - mx;
      xc[nF + p] = yfp[p] - my;
      xc[2 * nF + p] = zfp[p] - mz;
    }
  }
  // (1) TRSSPH force grid -> SH grid (forcing.f90:48-55)
  std::vector<double> xs(3 * nS);
  trssph1(nD, mD, &xc[0], nO, mO, &xs[0], faithful);
  trssph1(nD, mD, &xc[nF], nO, mO, &xs[nS], faithful);
  trssph1(nD, mD, &xc[2 * nF], nO, mO, &xs[2 * nS], faithful);
  // (2) cal_3dcrd_spectral_coeff (sph1.f90:29-79, re-initialised per call)
  auto pO = get_plan(nO, mO, faithful);
  std::vector<double> a((size_t)3 * N * N), b((size_t)3 * N * N);
  for (int c = 0; c < 3; ++c) analysis(*pO, &xs[c * nS], &a[(size_t)c * N * N], &b[(size_t)c * N * N]);
  if (shape_a) std::memcpy(shape_a, a.data(), sizeof(double) * a.size());
  if (shape_b) std::memcpy(shape_b, b.data(), sizeof(double) * b.size());
  // (3) geometry + mechanics on the dealias grid; with bending (eb != 0,
  // ibend = 1) the third and fourth derivatives, the moment and transverse
  // shear terms of cal_spectral_force (sph.f90:1636-1709)
  std::vector<double> fN(3 * nF), unitN(3 * nF);
  const double hf = 0.5 * gs;  // sph.f90:35 hf_gscell
  Geo G;
  const int nv = eb != 0.0 ? 42 : 15;
  std::vector<double> fv;
  if (eb != 0.0)
    synth_basis_bend(C, a.data(), b.data(), fv);
  else
    synth_basis(C, a.data(), b.data(), fv);
  for (size_t p = 0; p < nF; ++p) {
    geometry(&fv[p * nv], G);
    double f[3];
    if (eb != 0.0) {
      BendTensors X;
      BendQ bq;
      bend_tensors(G, (const double(*)[3]) & fv[p * nv + 15], (const double(*)[3]) & fv[p * nv + 27], X);
      bend_q(X, const_cast<BendTensors&>(C.refB[p]), eb, bq);
      mechanics(G, &C.conAR[p * 4], &C.conARd1[p * 8], hf, csk, law, f, &bq);
    } else {
      mechanics(G, &C.conAR[p * 4], &C.conARd1[p * 8], hf, csk, law, f);
    }
    for (int c = 0; c < 3; ++c) {
      fN[c * nF + p] = f[c];
      unitN[c * nF + p] = G.n[c];
    }
  }
  auto pD = get_plan(nD, mD, faithful);
  const int lD = pD->l;  // = 2N
  std::vector<double> aD((size_t)lD * nD), bD((size_t)lD * nD);
  // (4) cal_unitO_filter (sph1.f90:1378-1402)
  std::vector<double> unitO(3 * nS);
  for (int c = 0; c < 3; ++c) {
    analysis(*pD, &unitN[c * nF], aD.data(), bD.data());
    filter_synth(C, aD.data(), bD.data(), nD, &unitO[c * nS]);
  }
  for (size_t q = 0; q < nS; ++q) {
    double r = std::sqrt(unitO[q] * unitO[q] + unitO[nS + q] * unitO[nS + q] + unitO[2 * nS + q] * unitO[2 * nS + q]);
    for (int c = 0; c < 3; ++c) unitO[c * nS + q] /= r;
  }
  // (5) surfmetD (sph3.f90:186-277)
  std::vector<double> smD(nS);
  surface_metric(C, a.data(), b.data(), smD.data());
  // (6) filter_modes4__OPT (sph1.f90:919-932)
  std::vector<double> fS(3 * nS);
  for (int c = 0; c < 3; ++c) {
    analysis(*pD, &fN[c * nF], aD.data(), bD.data());
    if (force_a && force_b)
      for (int m = 0; m < N; ++m)
        for (int n = 0; n < N; ++n) {
          force_a[(size_t)c * N * N + (size_t)m * N + n] = (n >= m) ? aD[(size_t)m * nD + n] : 0.0;
          force_b[(size_t)c * N * N + (size_t)m * N + n] = (n >= m) ? bD[(size_t)m * nD + n] : 0.0;
        }
    filter_synth(C, aD.data(), bD.data(), nD, &fS[c * nS]);
  }
  if (!fxl) return 0;
  // (7) TRSSPH SH grid -> force grid (forcing.f90:67-88)
  trssph1(nO, mO, &fS[0], nD, mD, fxl, faithful);
  trssph1(nO, mO, &fS[nS], nD, mD, fyl, faithful);
  trssph1(nO, mO, &fS[2 * nS], nD, mD, fzl, faithful);
  trssph1(nO, mO, &unitO[0], nD, mD, xn, faithful);
  trssph1(nO, mO, &unitO[nS], nD, mD, yn, faithful);
  trssph1(nO, mO, &unitO[2 * nS], nD, mD, zn, faithful);
  std::vector<double> smF(nF);
  trssph1(nO, mO, smD.data(), nD, mD, smF.data(), faithful);
  // (8) area = surfmetDf * wgtdsinf (forcing.f90:91)
  for (int i = 0; i < nD; ++i)
    for (int j = 0; j < mD; ++j) area[(size_t)i * mD + j] = smF[(size_t)i * mD + j] * C.wgtdsinf[i];
  return 0;
}

// ----------------------------------------------------- interp / spread ------
inline long fidx(int i, int j, int k, int ldi, int ldj) { return (long)i + (long)ldi * ((long)j + (long)ldj * k); }
inline long nint_(double x) { return std::lround(x); }  // Fortran nint: half away from zero

struct Grid {
  int itot, jtot, ktot;
  double dxi, dyi, dzi;
};

// Cells touched by one point, per image, in the reference's clipped window.
// Calls fn(i,j,k, kxs,kx, kys,ky, kzs,kz) for every window cell.
template <class F>
void window_faithful(const Grid& g, double xc, double yc, double zc, F&& fn, int kc0 = 1, int kc1 = -1) {
  // interp_spread.f90:340-378: window nint(c-2)..nint(c+2), clipped to
  // [1,imax]x[1,jmax]x[1,kmax]; periodic x,y via image copies (:72-145).
  // lagr2eulrind (:1311-1316) clips z to [0,kmax+1] instead: kc0, kc1.
  if (kc1 < 0) kc1 = g.ktot;
  double cz = zc;
  for (int sx = -1; sx <= 1; ++sx)
    for (int sy = -1; sy <= 1; ++sy) {
      double cx = xc + sx * g.itot, cy = yc + sy * g.jtot;
      long il = nint_(cx - 2.), ih = nint_(cx + 2.), jl = nint_(cy - 2.), jh = nint_(cy + 2.);
      long kl = nint_(cz - 2.), kh = nint_(cz + 2.);
      if (il < 1) il = 1;
      if (jl < 1) jl = 1;
      if (kl < kc0) kl = kc0;
      if (ih > g.itot) ih = g.itot;
      if (jh > g.jtot) jh = g.jtot;
      if (kh > kc1) kh = kc1;
      if (il > ih || jl > jh) continue;
      for (long k = kl; k <= kh; ++k) {
        double czs = (1. * k) - cz, czz = czs - 0.5;
        double kzs = kern(czs), kz = kern(czz);
        for (long j = jl; j <= jh; ++j) {
          double cys = (1. * j) - cy, cyy = cys - 0.5;
          double kys = kern(cys), ky = kern(cyy);
          for (long i = il; i <= ih; ++i) {
            double cxs = (1. * i) - cx, cxx = cxs - 0.5;
            double kxs = kern(cxs), kx = kern(cxx);
            fn((int)i, (int)j, (int)k, kxs, kx, kys, ky, kzs, kz);
          }
        }
      }
    }
}

// Same cells via modular wrap over the 4-wide candidate window (exact
// equivalent: the 5-wide window covers the kernel support |r|<1.5).
template <class F>
void window_fast(const Grid& g, double xc, double yc, double zc, F&& fn, int kc0 = 1, int kc1 = -1) {
  if (kc1 < 0) kc1 = g.ktot;
  long fx = (long)std::floor(xc), fy = (long)std::floor(yc), fz = (long)std::floor(zc);
  double kxs[4], kx[4], kys[4], ky[4], kzs[4], kz[4];
  for (int t = 0; t < 4; ++t) {
    double cxs = (double)(fx - 1 + t) - xc, cys = (double)(fy - 1 + t) - yc, czs = (double)(fz - 1 + t) - zc;
    kxs[t] = kern(cxs); kx[t] = kern(cxs - 0.5);
    kys[t] = kern(cys); ky[t] = kern(cys - 0.5);
    kzs[t] = kern(czs); kz[t] = kern(czs - 0.5);
  }
  for (int tk = 0; tk < 4; ++tk) {
    long k = fz - 1 + tk;
    if (k < kc0 || k > kc1) continue;
    for (int tj = 0; tj < 4; ++tj) {
      long j = fy - 1 + tj;
      long jw = ((j - 1) % g.jtot + g.jtot) % g.jtot + 1;
      for (int ti = 0; ti < 4; ++ti) {
        long i = fx - 1 + ti;
        long iw = ((i - 1) % g.itot + g.itot) % g.itot + 1;
        fn((int)iw, (int)jw, (int)k, kxs[ti], kx[ti], kys[tj], ky[tj], kzs[tk], kz[tk]);
      }
    }
  }
}

void interp_points(const Grid& g, bool faithful, const double* u, const double* v, const double* w,
                   long p0, long p1, const double* xp, const double* yp, const double* zp,
                   double* ul, double* vl, double* wl) {
  const int ldi = g.itot + 2, ldj = g.jtot + 2;
  for (long p = p0; p < p1; ++p) {
    double cx = xp[p] * g.dxi, cy = yp[p] * g.dyi, cz = zp[p] * g.dzi;
    double su = 0, sv = 0, sw = 0;
    auto acc = [&](int i, int j, int k, double kxs, double kx, double kys, double ky, double kzs, double kz) {
      long o = fidx(i, j, k, ldi, ldj);
      su += u[o] * kxs * ky * kz;
      sv += v[o] * kx * kys * kz;
      sw += w[o] * kx * ky * kzs;
    };
    if (faithful) window_faithful(g, cx, cy, cz, acc);
    else window_fast(g, cx, cy, cz, acc);
    ul[p] = su;
    vl[p] = sv;
    wl[p] = sw;
  }
}

// Scatter of points [p0,p1) restricted to cells with k in [klo,khi].
void spread_points(const Grid& g, bool faithful, long p0, long p1, const double* xp, const double* yp,
                   const double* zp, const double* fxl, const double* fyl, const double* fzl,
                   const double* area, double dVi, int klo, int khi, double* fx, double* fy, double* fz) {
  const int ldi = g.itot + 2, ldj = g.jtot + 2;
  for (long p = p0; p < p1; ++p) {
    double cx = xp[p] * g.dxi, cy = yp[p] * g.dyi, cz = zp[p] * g.dzi;
    double s = area[p] * dVi;
    double ax = fxl[p] * s, ay = fyl[p] * s, az = fzl[p] * s;
    (void)ax;
    auto acc = [&](int i, int j, int k, double kxs, double kx, double kys, double ky, double kzs, double kz) {
      if (k < klo || k > khi) return;
      long o = fidx(i, j, k, ldi, ldj);
      // interp_spread.f90:870-874 (f * phi*phi*phi * (area/dVeul))
      fx[o] += fxl[p] * kxs * ky * kz * (area[p] * dVi);
      fy[o] += fyl[p] * kx * kys * kz * (area[p] * dVi);
      fz[o] += fzl[p] * kx * ky * kzs * (area[p] * dVi);
    };
    (void)ay; (void)az;
    if (faithful) window_faithful(g, cx, cy, cz, acc);
    else window_fast(g, cx, cy, cz, acc);
  }
}

// updthalos (bound.f90:141-190): x then y halo copies, periodic.
void halo_copy(const Grid& g, double* f) {
  const int ldi = g.itot + 2, ldj = g.jtot + 2, ldk = g.ktot + 2;
  for (int k = 0; k < ldk; ++k)
    for (int j = 0; j < ldj; ++j) {
      f[fidx(g.itot + 1, j, k, ldi, ldj)] = f[fidx(1, j, k, ldi, ldj)];
      f[fidx(0, j, k, ldi, ldj)] = f[fidx(g.itot, j, k, ldi, ldj)];
    }
  for (int k = 0; k < ldk; ++k)
    for (int i = 0; i < ldi; ++i) {
      f[fidx(i, g.jtot + 1, k, ldi, ldj)] = f[fidx(i, 1, k, ldi, ldj)];
      f[fidx(i, 0, k, ldi, ldj)] = f[fidx(i, g.jtot, k, ldi, ldj)];
    }
}

// lagr2eulrind (interp_spread.f90:978-1387): g = sum_l n_l phi(x) phi(y)
// phi(z) area_l / dV with cell-centre weights in all three directions for
// all three components (:1319-1343), z window clipped to [0, kmax+1] (the
// wall halo planes keep their contributions), then the periodic x and y halo
// copies (:1371-1382).
void spread_ind_all(const Grid& g, bool faithful, long npts, const double* xp, const double* yp, const double* zp,
                    const double* nxl, const double* nyl, const double* nzl, const double* area, double dVi,
                    double* gx, double* gy, double* gz) {
  const int ldi = g.itot + 2, ldj = g.jtot + 2;
  const long ntot = (long)ldi * ldj * (g.ktot + 2);
  std::memset(gx, 0, sizeof(double) * ntot);
  std::memset(gy, 0, sizeof(double) * ntot);
  std::memset(gz, 0, sizeof(double) * ntot);
  for (long p = 0; p < npts; ++p) {
    double cx = xp[p] * g.dxi, cy = yp[p] * g.dyi, cz = zp[p] * g.dzi;
    auto acc = [&](int i, int j, int k, double, double kx, double, double ky, double, double kz) {
      long o = fidx(i, j, k, ldi, ldj);
      gx[o] += nxl[p] * kx * ky * kz * (area[p] * dVi);
      gy[o] += nyl[p] * kx * ky * kz * (area[p] * dVi);
      gz[o] += nzl[p] * kx * ky * kz * (area[p] * dVi);
    };
    if (faithful) window_faithful(g, cx, cy, cz, acc, 0, g.ktot + 1);
    else window_fast(g, cx, cy, cz, acc, 0, g.ktot + 1);
  }
  halo_copy(g, gx);
  halo_copy(g, gy);
  halo_copy(g, gz);
}

int nthreads_of(int req) {
#ifdef _OPENMP
  return req > 0 ? req : omp_get_max_threads();
#else
  (void)req;
  return 1;
#endif
}

void spread_all(const Grid& g, bool faithful, int nth, long npts, const double* xp, const double* yp,
                const double* zp, const double* fxl, const double* fyl, const double* fzl, const double* area,
                double dVi, double* fx, double* fy, double* fz) {
  const long ntot = (long)(g.itot + 2) * (g.jtot + 2) * (g.ktot + 2);
  // interp_spread.f90:811-815 zero everything
  std::memset(fx, 0, sizeof(double) * ntot);
  std::memset(fy, 0, sizeof(double) * ntot);
  std::memset(fz, 0, sizeof(double) * ntot);
  if (nth <= 1) {
    spread_points(g, faithful, 0, npts, xp, yp, zp, fxl, fyl, fzl, area, dVi, 1, g.ktot, fx, fy, fz);
  } else {
#ifdef _OPENMP
#pragma omp parallel num_threads(nth)
    {
      int t = omp_get_thread_num(), T = omp_get_num_threads();
      int klo = 1 + (int)((long)g.ktot * t / T), khi = (int)((long)g.ktot * (t + 1) / T);
      // each thread owns a z-slab of cells; points outside it are skipped cheaply
      double zlo = (klo - 3) / g.dzi, zhi = (khi + 2) / g.dzi;
      for (long p = 0; p < npts; ++p) {
        if (zp[p] < zlo || zp[p] > zhi) continue;
        spread_points(g, faithful, p, p + 1, xp, yp, zp, fxl, fyl, fzl, area, dVi, klo, khi, fx, fy, fz);
      }
    }
#endif
  }
  halo_copy(g, fx);
  halo_copy(g, fy);
  halo_copy(g, fz);
}

}  // namespace

// ============================================================== C ABI =====
extern "C" {

int or_gaqd(int nlat, double* theta, double* wts) {
  if (nlat < 1) return 1;
  gauss(nlat, theta, wts);
  return 0;
}

void or_legendre(double theta, int mm, int nn, double* P, double* dP, double* d2P) {
  std::vector<double> T, D, D2;
  int nt = nn + 2;
  legendre_full(theta, nt, T, D, D2);
  for (int m = 0; m < mm; ++m)
    for (int n = 0; n < nn; ++n) {
      size_t o = (size_t)m * nn + n, s = (size_t)m * nt + n;
      bool ok = (n >= m);
      if (P) P[o] = ok ? T[s] : 0.0;
      if (dP) dP[o] = ok ? D[s] : 0.0;
      if (d2P) d2P[o] = ok ? D2[s] : 0.0;
    }
}

int or_shagc(int nlat, int nlon, int nf, const double* g, double* a, double* b) {
  if (nlat < 3) return 1;
  if (nlon < 4) return 2;
  auto p = get_plan(nlat, nlon, false);
  for (int f = 0; f < nf; ++f)
    analysis(*p, g + (size_t)f * nlat * nlon, a + (size_t)f * p->l * nlat, b + (size_t)f * p->l * nlat);
  return 0;
}

int or_shsgc(int nlat, int nlon, int nf, const double* a, const double* b, double* g) {
  if (nlat < 3) return 1;
  if (nlon < 4) return 2;
  auto p = get_plan(nlat, nlon, false);
  for (int f = 0; f < nf; ++f)
    synthesis(*p, a + (size_t)f * p->l * nlat, b + (size_t)f * p->l * nlat, g + (size_t)f * nlat * nlon);
  return 0;
}

int or_trssph(int nlata, int nlona, int nf, const double* da, int nlatb, int nlonb, double* db) {
  // trssph.f:497-518 argument checks
  if (nlona < 4) return 4;
  if (nlata < 3) return 5;
  if (nlonb < 4) return 8;
  if (nlatb < 3) return 9;
  for (int f = 0; f < nf; ++f)
    trssph1(nlata, nlona, da + (size_t)f * nlata * nlona, nlatb, nlonb, db + (size_t)f * nlatb * nlonb, false);
  return 0;
}

double or_kernel(double r) { return kern(r); }

double or_kerneltest(void) {
  double sum = 0.;
  for (int k = -25; k <= 25; ++k) {
    double cz = k / 12.;
    for (int j = -25; j <= 25; ++j) {
      double cy = j / 12.;
      for (int i = -25; i <= 25; ++i) {
        double cx = i / 12.;
        sum = sum + (1. / 12.) * (1. / 12.) * (1. / 12.) * kern(cx) * kern(cy) * kern(cz);
      }
    }
  }
  return sum;
}

int or_complagrforces(int L, double radius, double gs, double csk, int faithful, const double* xfp,
                      const double* yfp, const double* zfp, double* fx, double* fy, double* fz, double* nx,
                      double* ny, double* nz, double* area) {
  return capsule_force(L, radius, gs, csk, 0, faithful != 0, xfp, yfp, zfp, fx, fy, fz, nx, ny, nz, area, nullptr,
                       nullptr, nullptr, nullptr);
}

// complagrforces with a chosen membrane law (0 Skalak, 1 neo-Hookean)
int or_complagrforces_bend(int L, double radius, double gs, double csk, int law, double eb, int faithful,
                           const double* xfp, const double* yfp, const double* zfp, double* fx, double* fy,
                           double* fz, double* nx, double* ny, double* nz, double* area) {
  return capsule_force(L, radius, gs, csk, law, faithful != 0, xfp, yfp, zfp, fx, fy, fz, nx, ny, nz, area, nullptr,
                       nullptr, nullptr, nullptr, eb);
}

int or_complagrforces_law(int L, double radius, double gs, double csk, int law, int faithful, const double* xfp,
                          const double* yfp, const double* zfp, double* fx, double* fy, double* fz, double* nx,
                          double* ny, double* nz, double* area) {
  if (law != 0 && law != 1) return 1;
  return capsule_force(L, radius, gs, csk, law, faithful != 0, xfp, yfp, zfp, fx, fy, fz, nx, ny, nz, area, nullptr,
                       nullptr, nullptr, nullptr);
}

int or_capsule_spectra(int L, double radius, double gs, double csk, const double* xfp, const double* yfp,
                       const double* zfp, double* shape_a, double* shape_b, double* force_a, double* force_b) {
  return capsule_force(L, radius, gs, csk, 0, false, xfp, yfp, zfp, nullptr, nullptr, nullptr, nullptr, nullptr,
                       nullptr, nullptr, shape_a, shape_b, force_a, force_b);
}

int or_interp(int itot, int jtot, int ktot, double dx, double dy, double dz, int faithful, const double* u,
              const double* v, const double* w, long npts, const double* xp, const double* yp, const double* zp,
              double* ul, double* vl, double* wl) {
  Grid g{itot, jtot, ktot, 1.0 / dx, 1.0 / dy, 1.0 / dz};
  interp_points(g, faithful != 0, u, v, w, 0, npts, xp, yp, zp, ul, vl, wl);
  return 0;
}

int or_spread_ind(int itot, int jtot, int ktot, double dx, double dy, double dz, int faithful, long npts,
                  const double* xp, const double* yp, const double* zp, const double* nxl, const double* nyl,
                  const double* nzl, const double* area, double* gx, double* gy, double* gz) {
  Grid g{itot, jtot, ktot, 1.0 / dx, 1.0 / dy, 1.0 / dz};
  spread_ind_all(g, faithful != 0, npts, xp, yp, zp, nxl, nyl, nzl, area, 1.0 / (dx * dy * dz), gx, gy, gz);
  return 0;
}

int or_spread(int itot, int jtot, int ktot, double dx, double dy, double dz, int faithful, long npts,
              const double* xp, const double* yp, const double* zp, const double* fxl, const double* fyl,
              const double* fzl, const double* area, double* fx, double* fy, double* fz) {
  Grid g{itot, jtot, ktot, 1.0 / dx, 1.0 / dy, 1.0 / dz};
  double dVi = 1.0 / (dx * dy * dz);
  spread_all(g, faithful != 0, 1, npts, xp, yp, zp, fxl, fyl, fzl, area, dVi, fx, fy, fz);
  return 0;
}

void or_update_pos(long npts, double dt, double lz, double* xp, double* yp, double* zp, const double* ul,
                   const double* vl, const double* wl) {
  for (long l = 0; l < npts; ++l) {
    xp[l] = xp[l] + (ul[l] * dt);
    yp[l] = yp[l] + (vl[l] * dt);
    zp[l] = zp[l] + (wl[l] * dt);
    if (zp[l] < 0.) zp[l] = 0.;
    else if (zp[l] > lz) zp[l] = lz;
  }
}

void or_update_pos_capsules(int ncap, const long* off, double dt, double lx, double ly, double lz, double* xp,
                            double* yp, double* zp, const double* ul, const double* vl, const double* wl) {
  // Update_Pos.f90:95-99 and 118-126 per point, then :131-180 per capsule:
  // sequential centroid, shift by one period when it has left the box
  or_update_pos(off[ncap], dt, lz, xp, yp, zp, ul, vl, wl);
  for (int p = 0; p < ncap; ++p) {
    const long a = off[p], b = off[p + 1];
    double x = 0., y = 0.;
    for (long l = a; l < b; ++l) { x += xp[l]; y += yp[l]; }
    x /= (double)(b - a);
    y /= (double)(b - a);
    if (x > lx) for (long l = a; l < b; ++l) xp[l] = xp[l] - lx;
    if (x < 0.) for (long l = a; l < b; ++l) xp[l] = xp[l] + lx;
    if (y > ly) for (long l = a; l < b; ++l) yp[l] = yp[l] - ly;
    if (y < 0.) for (long l = a; l < b; ++l) yp[l] = yp[l] + ly;
  }
}

void or_surf_vol(long nl, const double* x, const double* y, const double* z, const double* nx, const double* ny,
                 const double* nz, const double* area, double exy1_prev, double* out) {
  double xm = 0, ym = 0, zm = 0;
  for (long l = 0; l < nl; ++l) { xm += x[l]; ym += y[l]; zm += z[l]; }
  xm /= nl; ym /= nl; zm /= nl;
  // radial layer sums of surf_vol.f90:77-96 in closed form
  double S2 = 0, S22 = 0;
  for (int l = 1; l <= 1000; ++l) {
    double ma = (l - 1) / 1000., na = (l - .5) / 1000.;
    S2 += ma * ma;
    S22 += ma * ma * na * na;
  }
  double vol = 0, ixx = 0, ixy = 0, ixz = 0, iyy = 0, iyz = 0, izz = 0, atot = 0, rmax = -1, rmin = 1e300;
  for (long l = 0; l < nl; ++l) {
    double dxp = x[l] - xm, dyp = y[l] - ym, dzp = z[l] - zm;
    double r = std::sqrt(dxp * dxp + dyp * dyp + dzp * dzp);
    double dr = r / 1000.;
    double cs = (dxp * nx[l] + dyp * ny[l] + dzp * nz[l]) / r;
    double base = area[l] * dr * std::fabs(cs);
    vol += base * S2;
    ixx += base * S22 * (dyp * dyp + dzp * dzp);
    ixy -= base * S22 * (dxp * dyp);
    ixz -= base * S22 * (dxp * dzp);
    iyy += base * S22 * (dxp * dxp + dzp * dzp);
    iyz -= base * S22 * (dyp * dzp);
    izz += base * S22 * (dxp * dxp + dyp * dyp);
    atot += area[l];
    if (r > rmax) rmax = r;
    if (r < rmin) rmin = r;
  }
  double i1 = ixx + iyy + izz;
  double i2 = ixx * iyy + iyy * izz + ixx * izz - ixy * ixy - iyz * iyz - ixz * ixz;
  double i3 = ixx * iyy * izz - ixx * iyz * iyz - iyy * ixz * ixz - izz * ixy * ixy + 2. * ixy * ixz * iyz;
  double r = (2. * i1 * i1 * i1 - 9. * i1 * i2 + 27. * i3) / 54.;
  double q = (3. * i2 - i1 * i1) / 9.;
  double teta = std::acos(r / std::sqrt(-(q * q * q)));
  double ip1 = i1 / 3. + 2. * std::sqrt(-q) * std::cos(teta / 3.);
  double ip2 = i1 / 3. + 2. * std::sqrt(-q) * std::cos((teta + 2. * kPi) / 3.);
  double ip3 = i1 / 3. + 2. * std::sqrt(-q) * std::cos((teta + 4. * kPi) / 3.);
  double mass = (4. / 3.) * kPi;
  double ic1 = ip1 / (mass / 5.), ic2 = ip2 / (mass / 5.), ic3 = ip3 / (mass / 5.);
  double lp2 = std::sqrt(.5 * (ic1 + ic3 - ic2));
  double lp1 = std::sqrt(ic3 - lp2 * lp2);
  double lp3 = std::sqrt(ic1 - lp2 * lp2);
  double exy1 = exy1_prev;
  if (std::fabs(ip1 - ixx) < 0.0001) exy1 = std::fabs(lp2 - lp3) / (lp2 + lp3);
  else if (std::fabs(ip2 - ixx) < 0.0001) exy1 = std::fabs(lp1 - lp3) / (lp1 + lp3);
  else if (std::fabs(ip3 - ixx) < 0.0001) exy1 = std::fabs(lp1 - lp2) / (lp1 + lp2);
  out[0] = vol;
  out[1] = atot;
  out[2] = exy1;
  out[3] = std::fabs(rmax - rmin) / (rmax + rmin);
  out[4] = xm;
  out[5] = ym;
  out[6] = zm;
}

void or_collisions(long nl, const double* zp, const double* area, double dx, double dy, double col,
                   double betacol, double rep, double rad0, double* fzl) {
  double dyi = 1.0 / dy;
  for (long i = 0; i < nl; ++i) {
    double fc = 0.;
    long jm = std::lround(std::sqrt(std::fmax(rad0 * rad0 - zp[i] * zp[i], 0.)) * dyi);
    for (long j = -jm; j <= jm; ++j)
      for (long k = -jm; k <= jm; ++k) {
        double ss = std::sqrt(zp[i] * zp[i] + (j * dy) * (j * dy) + (k * dx) * (k * dx));
        if (ss < rad0)
          fc += (2. * (col / (rep * rep))) * (std::exp(2. * betacol * (rad0 - ss)) - std::exp(betacol * (rad0 - ss))) *
                std::fabs(zp[i] / ss) * (std::fmin(area[i], dx * dx) / std::fmax(area[i], dx * dx));
      }
    fzl[i] += fc;
  }
}

void or_skalak(double I1, double I2, const double* I1de, const double* I2de, double gs, double csk, double* out) {
  // membmodel.c:81-99 restated: out = W1, W2, dW1[2], dW2[2]
  membrane_law(0, 0.5 * gs, csk, I1, I2, I1de, I2de, out[0], out[1], out + 2, out + 4);
}

void or_membrane_law(int law, double I1, double I2, const double* I1de, const double* I2de, double gs, double csk,
                     double* out) {
  // membmodel.c:60-99 restated (law 0 Skalak, 1 neo-Hookean): out = W1, W2, dW1[2], dW2[2]
  membrane_law(law, 0.5 * gs, csk, I1, I2, I1de, I2de, out[0], out[1], out + 2, out + 4);
}

int or_coupling_step(int itot, int jtot, int ktot, double dx, double dy, double dz, int ncap, const int* degree,
                     const double* radius, double gs, double csk, int faithful, int nthreads, const double* u,
                     const double* v, const double* w, const double* xp, const double* yp, const double* zp,
                     double* ul, double* vl, double* wl, double* fxl, double* fyl, double* fzl, double* nx,
                     double* ny, double* nz, double* area, double* fx, double* fy, double* fz, double* t) {
  using clk = std::chrono::steady_clock;
  Grid g{itot, jtot, ktot, 1.0 / dx, 1.0 / dy, 1.0 / dz};
  std::vector<long> off(ncap + 1, 0);
  for (int c = 0; c < ncap; ++c) off[c + 1] = off[c] + 8L * (degree[c] + 1) * (degree[c] + 1);
  const long npts = off[ncap];
  int nth = nthreads_of(nthreads);
  bool fa = faithful != 0;
  // build per-degree state outside the timed stages (the reference does it at init)
  for (int c = 0; c < ncap; ++c) get_capsule(degree[c], radius[c]);
  auto t0 = clk::now();
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nth)
#endif
  for (long b = 0; b < (npts + 255) / 256; ++b) {
    long p0 = b * 256, p1 = p0 + 256 < npts ? p0 + 256 : npts;
    interp_points(g, fa, u, v, w, p0, p1, xp, yp, zp, ul, vl, wl);
  }
  auto t1 = clk::now();
  int err = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic) num_threads(nth) reduction(| : err)
#endif
  for (int c = 0; c < ncap; ++c) {
    long o = off[c];
    err |= capsule_force(degree[c], radius[c], gs, csk, 0, fa, xp + o, yp + o, zp + o, fxl + o, fyl + o, fzl + o, nx + o,
                         ny + o, nz + o, area + o, nullptr, nullptr, nullptr, nullptr);
  }
  auto t2 = clk::now();
  spread_all(g, fa, nth, npts, xp, yp, zp, fxl, fyl, fzl, area, 1.0 / (dx * dy * dz), fx, fy, fz);
  auto t3 = clk::now();
  if (t) {
    t[0] = std::chrono::duration<double>(t1 - t0).count();
    t[1] = std::chrono::duration<double>(t2 - t1).count();
    t[2] = std::chrono::duration<double>(t3 - t2).count();
  }
  return err;
}

}  // extern "C"
