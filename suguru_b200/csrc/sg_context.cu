// sg_context.cu -- the C ABI (include/sg_coupling.h): context set-up, device
// memory, per-degree tables, work lists, and the step pipeline.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "sg_ctx.h"

using namespace sg;

const double kPi = 3.14159265358979323846264338327950288;

namespace {

// Lowest SH degree whose tensor-core contractions run in BF16x6 under the
// automatic split mode.  The force takes second derivatives of the analysed
// shape, so the ~2^-17 relative error of a BF16x3 product grows about as
// L^2 in the force: measured against the FP64 oracle, BF16x3 gives
// 2e-5 (L = 8), 4e-5 to 8e-5 (L = 12 to 16) and 2.5e-4 (L = 22); BF16x6
// keeps every degree at the FP32 CUDA-core level.
constexpr int kSixTermDegree = 16;

int terms_for(const sg_ctx* c, int degree) {
  if (c->leg_terms) return c->leg_terms;
  // the bending terms take fourth derivatives of the analysed shape, which
  // amplify the product error about as L^4: FP32-level products throughout
  if (c->bend) return 6;
  return degree >= kSixTermDegree ? 6 : 3;
}

// Split mode of every tensor-core problem (by its group's degree) and the
// number of operand parts the launches stage.
void assign_terms(sg_ctx* c, std::vector<sg::LegProblem>& P) {
  c->leg_parts = 2;
  for (sg::LegProblem& p : P) {
    p.terms = terms_for(c, c->groups[p.group].L);
    if (p.terms == 6) c->leg_parts = 3;
  }
}

template <class V>
cudaError_t upload(sg_ctx* c, void*& dst, const std::vector<V>& v) {
  cudaError_t e = dalloc(c, dst, sizeof(V) * v.size());
  if (e != cudaSuccess) return e;
  return cudaMemcpy(dst, v.data(), sizeof(V) * v.size(), cudaMemcpyHostToDevice);
}

template <class V>
cudaError_t upload2(sg_ctx* c, void* (&dst)[2], const std::vector<double>& v) {
  (void)sizeof(V);
  cudaError_t e = upload(c, dst[0], v);
  if (e != cudaSuccess) return e;
  std::vector<float> f(v.begin(), v.end());
  return upload(c, dst[1], f);
}

// Per-degree FP64 tables -> device (double and float copies).
cudaError_t build_tables(sg_ctx* c, Group& g) {
  const int N = g.N, nD = g.nD, mD = g.mD, nO = g.nO, mO = g.mO;
  std::vector<double> thD(nD), wD(nD), thO(nO), wO(nO);
  host_gauss(nD, thD.data(), wD.data());
  host_gauss(nO, thO.data(), wO.data());
  std::vector<double> P((size_t)N * N), dP((size_t)N * N), d2P((size_t)N * N);
  std::vector<double> synD((size_t)N * 3 * nD * N, 0.0), anaD((size_t)N * N * nD, 0.0);
  std::vector<double> synO((size_t)N * 2 * nO * N, 0.0), anaO((size_t)N * N * nO, 0.0);
  for (int i = 0; i < nD; ++i) {
    host_legendre(thD[i], N, N, P.data(), dP.data(), d2P.data());
    for (int m = 0; m < N; ++m) {
      const double h = (m == 0) ? 0.5 : 1.0;  // sph3.f90:69-71, shsgc m=0 half weight
      for (int n = 0; n < N; ++n) {
        const double p = P[(size_t)m * N + n], d = dP[(size_t)m * N + n], e = d2P[(size_t)m * N + n];
        synD[((size_t)m * 3 * nD + 0 * nD + i) * N + n] = h * p;
        synD[((size_t)m * 3 * nD + 1 * nD + i) * N + n] = h * d;
        synD[((size_t)m * 3 * nD + 2 * nD + i) * N + n] = h * e;
        anaD[((size_t)m * N + n) * nD + i] = wD[i] * p;
      }
    }
  }
  for (int i = 0; i < nO; ++i) {
    host_legendre(thO[i], N, N, P.data(), dP.data(), nullptr);
    for (int m = 0; m < N; ++m) {
      const double h = (m == 0) ? 0.5 : 1.0;
      for (int n = 0; n < N; ++n) {
        synO[((size_t)m * 2 * nO + 0 * nO + i) * N + n] = h * P[(size_t)m * N + n];
        synO[((size_t)m * 2 * nO + 1 * nO + i) * N + n] = h * dP[(size_t)m * N + n];
        anaO[((size_t)m * N + n) * nO + i] = wO[i] * P[(size_t)m * N + n];
      }
    }
  }
  std::vector<double> latD((size_t)nD * 4), latO((size_t)nO * 4);
  for (int i = 0; i < nD; ++i) {
    latD[4 * i] = std::sin(thD[i]);
    latD[4 * i + 1] = std::cos(thD[i]);
    latD[4 * i + 2] = wD[i] / std::sin(thD[i]) * (2.0 * kPi / mD);  // wgtdsinf, sph.f90:130
    latD[4 * i + 3] = thD[i];
  }
  for (int i = 0; i < nO; ++i) {
    latO[4 * i] = std::sin(thO[i]);
    latO[4 * i + 1] = std::cos(thO[i]);
    latO[4 * i + 2] = wO[i] / std::sin(thO[i]) * (2.0 * kPi / mO);
    latO[4 * i + 3] = thO[i];
  }
  auto trig = [&](int nlon) {
    std::vector<double> t((size_t)2 * N * nlon);
    for (int m = 0; m < N; ++m)
      for (int j = 0; j < nlon; ++j) {
        const double a = 2.0 * kPi * (double)(((long long)m * j) % nlon) / nlon;
        t[(size_t)m * nlon + j] = std::cos(a);
        t[(size_t)N * nlon + (size_t)m * nlon + j] = std::sin(a);
      }
    return t;
  };
  g.h_tab[0] = synD;
  g.h_tab[1] = anaD;
  g.h_tab[2] = synO;
  g.h_tab[3] = anaO;
  cudaError_t e;
  if ((e = upload2<double>(c, g.tab.syn_D, synD)) != cudaSuccess) return e;
  if ((e = upload2<double>(c, g.tab.ana_D, anaD)) != cudaSuccess) return e;
  if ((e = upload2<double>(c, g.tab.syn_O, synO)) != cudaSuccess) return e;
  if ((e = upload2<double>(c, g.tab.ana_O, anaO)) != cudaSuccess) return e;
  if ((e = upload2<double>(c, g.tab.latD, latD)) != cudaSuccess) return e;
  if ((e = upload2<double>(c, g.tab.latO, latO)) != cudaSuccess) return e;
  if ((e = upload2<double>(c, g.tab.trigD, trig(mD))) != cudaSuccess) return e;
  if ((e = upload2<double>(c, g.tab.trigO, trig(mO))) != cudaSuccess) return e;
  return cudaSuccess;
}

void add_problem(std::vector<LegProblem>& P, std::vector<LegWork>& W, const LegProblem& p, int& maxJ, int& maxK) {
  const int id = (int)P.size();
  P.push_back(p);
  for (int m = 0; m < p.M; ++m)
    for (int q0 = 0; q0 < p.Q; q0 += 32) W.push_back(LegWork{id, m, q0});
  maxJ = std::max(maxJ, p.J);
  maxK = std::max(maxK, p.K);
}

LegProblem prob(const void* A, long long sAc, long long sAr, long long sAm, const void* B, long long sBm, void* D,
                long long sDc, long long sDr, long long sDm, int rpc, int ncap, int M, int J, int K, int tri,
                int group, int kind) {
  LegProblem p{};
  p.A = A; p.sAc = sAc; p.sAr = sAr; p.sAm = sAm;
  p.B = B; p.sBm = sBm;
  p.D = D; p.sDc = sDc; p.sDr = sDr; p.sDm = sDm;
  p.rpc = rpc; p.Q = rpc * ncap; p.M = M; p.J = J; p.K = K;
  p.tri = tri; p.group = group; p.kind = kind;
  p.next[0] = p.next[1] = -1;
  return p;
}

// The per-group constants the kernels read (tables, buffers) to the device.
int upload_groups(sg_ctx* c) {
  std::vector<GroupDev> gdev(c->groups.size());
  for (size_t gi = 0; gi < c->groups.size(); ++gi) {
    const Group& gr = c->groups[gi];
    GroupDev& d = gdev[gi];
    d.L = gr.L; d.N = gr.N; d.nD = gr.nD; d.mD = gr.mD; d.nO = gr.nO; d.mO = gr.mO;
    for (int q = 0; q < 2; ++q) {
      d.latD[q] = gr.tab.latD[q]; d.latO[q] = gr.tab.latO[q];
      d.trigD[q] = gr.tab.trigD[q]; d.trigO[q] = gr.tab.trigO[q];
    }
    d.buf = gr.buf;
  }
  if (!gdev.empty())
    SG_TRY(cudaMemcpy(c->d_groups, gdev.data(), sizeof(GroupDev) * gdev.size(), cudaMemcpyHostToDevice), "groups");
  return SG_OK;
}

// Bending set-up (first sg_set_capsule_bending with a nonzero modulus): per
// degree group the FP64 table of the third and fourth theta derivatives
// (kind 4: syn_B[m][kind nD + i][n], m = 0 halved as the other synthesis
// tables, sph3.f90:72-102), the buffer GB of their series, and the synthesis
// problem S1b (A = the shape's coefficients, as S1), with its work lists for
// the CUDA-core and the tensor-core launch.
int bend_setup(sg_ctx* c) {
  if (c->bend_ready) return SG_OK;
  const size_t E = c->esz;
  const int pi = c->mixed ? 1 : 0;
  std::vector<LegProblem> P = c->h_probs;
  std::vector<LegWork> W, WT;
  int maxJ = 0, maxK = 0;
  std::vector<int> ids;
  for (size_t gi = 0; gi < c->groups.size(); ++gi) {
    Group& gr = c->groups[gi];
    const int N = gr.N, nD = gr.nD, n = (int)gr.caps.size();
    std::vector<double> th(nD), wq(nD), d3((size_t)N * N), d4((size_t)N * N);
    host_gauss(nD, th.data(), wq.data());
    std::vector<double> synB((size_t)N * 2 * nD * N, 0.0);
    for (int i = 0; i < nD; ++i) {
      host_legendre_d34(th[i], N, N, d3.data(), d4.data());
      for (int m = 0; m < N; ++m) {
        const double h = (m == 0) ? 0.5 : 1.0;
        for (int q = 0; q < N; ++q) {
          synB[((size_t)m * 2 * nD + 0 * nD + i) * N + q] = h * d3[(size_t)m * N + q];
          synB[((size_t)m * 2 * nD + 1 * nD + i) * N + q] = h * d4[(size_t)m * N + q];
        }
      }
    }
    gr.h_tab[4] = synB;
    SG_TRY(upload2<double>(c, gr.tab.syn_B, synB), "bending tables");
    SG_TRY(dalloc(c, gr.buf.GB, E * (size_t)n * 12 * N * nD), "alloc");
    const long long LN = N, LD = nD;
    ids.push_back((int)P.size());
    add_problem(P, W, prob(gr.buf.Cpos, 6 * LN * LN, LN * LN, LN, gr.tab.syn_B[pi], 2 * LD * LN, gr.buf.GB,
                           6 * LN * 2 * LD, LN * 2 * LD, 2 * LD, 6, n, N, 2 * nD, N, 1, (int)gi, 4),
                maxJ, maxK);
  }
  if (c->mixed) {
    std::vector<uint16_t> img;
    std::vector<size_t> off;
    LegLevels lv{};
    for (int id : ids) {
      LegProblem& p = P[id];
      p.Jp = (p.J + 15) / 16 * 16;
      p.Kp = (p.K + 15) / 16 * 16;
      p.sBimg = 3LL * p.Jp * p.Kp;
      off.push_back(img.size());
      img.resize(img.size() + (size_t)p.M * p.sBimg);
      const std::vector<double>& hb = c->groups[p.group].h_tab[4];
      host_umma_image(hb.data(), p.sBm, p.M, p.J, p.K, p.Jp, p.Kp, img.data() + off.back());
      auto al4 = [](const void* ptr) { return ((uintptr_t)ptr & 15u) == 0; };
      p.vecA = (al4(p.A) && p.sAc % 4 == 0 && p.sAr % 4 == 0 && p.sAm % 4 == 0 && p.K % 8 == 0) ? 1 : 0;
      p.vecD = (al4(p.D) && p.sDc % 4 == 0 && p.sDr % 4 == 0 && p.sDm % 4 == 0 && p.J % 4 == 0) ? 1 : 0;
      lv.jp[0] = std::max(lv.jp[0], p.Jp);
      lv.kp[0] = std::max(lv.kp[0], p.Kp);
      lv.a_kp = std::max(lv.a_kp, p.Kp);
      for (int m = 0; m < p.M; ++m)
        for (int q0 = 0; q0 < p.Q; q0 += 128) WT.push_back(LegWork{id, m, q0});
    }
    void* dimg = nullptr;
    SG_TRY(upload(c, dimg, img), "umma images");
    for (size_t k = 0; k < ids.size(); ++k) P[ids[k]].Bimg = (const uint16_t*)dimg + off[k];
    c->lvB = lv;
    void* tmp = nullptr;
    SG_TRY(upload(c, tmp, WT), "work");
    c->d_lwBT = (LegWork*)tmp;
    c->nlwBT = (int)WT.size();
  }
  void* tmp = nullptr;
  SG_TRY(upload(c, tmp, W), "work");
  c->d_lwB = (LegWork*)tmp;
  c->nlwB = (int)W.size();
  c->maxJB = maxJ;
  c->maxKB = maxK;
  c->h_probs = P;
  assign_terms(c, c->h_probs);
  SG_TRY(upload(c, tmp, c->h_probs), "problems");
  c->d_probs = (LegProblem*)tmp;
  SG_RET(upload_groups(c));
  c->bend_ready = true;
  return SG_OK;
}

// Work items of the persistent pointwise kernels: every capsule split into
// `split` row ranges (each item stages the capsule's whole input block),
// largest degree first so that the heaviest items start early.  More items
// than capsules keep every SM busy when there are few capsules per SM.
int set_point_split(sg_ctx* c, int split) {
  if (split < 1 || split > kMaxPointSplit) return fail(c, SG_ERR_ARG, "point split out of range");
  std::vector<RowWork> wpos, wmem, wsh;
  std::vector<int> gorder(c->groups.size());
  for (size_t gi = 0; gi < gorder.size(); ++gi) gorder[gi] = (int)gi;
  std::sort(gorder.begin(), gorder.end(), [&](int a, int b) { return c->groups[a].L > c->groups[b].L; });
  for (int q = 0; q < split; ++q)  // item q of every capsule, then item q+1: large items spread out
    for (int gi : gorder)
      for (int k : c->groups[gi].caps) {
        const Group& gr = c->groups[gi];
        const int pD = std::min(split, gr.nD), pO = std::min(split, gr.nO);
        if (q < pD) {
          const int r0 = gr.nD * q / pD, r1 = gr.nD * (q + 1) / pD;
          wpos.push_back(RowWork{k, r0, r1 - r0, gi});
          wmem.push_back(RowWork{k, r0, r1 - r0, gi});
        }
        if (q < pO) {
          const int r0 = gr.nO * q / pO, r1 = gr.nO * (q + 1) / pO;
          wsh.push_back(RowWork{k, r0, r1 - r0, gi});
        }
      }
  c->nwpos = (int)wpos.size();
  c->nwmem = (int)wmem.size();
  c->nwsh = (int)wsh.size();
  c->nwfin = c->nwmem;
  SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
  SG_TRY(cudaMemcpy(c->d_wpos, wpos.data(), sizeof(RowWork) * wpos.size(), cudaMemcpyHostToDevice), "work");
  SG_TRY(cudaMemcpy(c->d_wmem, wmem.data(), sizeof(RowWork) * wmem.size(), cudaMemcpyHostToDevice), "work");
  SG_TRY(cudaMemcpy(c->d_wsh, wsh.data(), sizeof(RowWork) * wsh.size(), cudaMemcpyHostToDevice), "work");
  SG_TRY(cudaMemcpy(c->d_wfin, wmem.data(), sizeof(RowWork) * wmem.size(), cudaMemcpyHostToDevice), "work");
  c->point_split = split;
  return SG_OK;
}

int setup(sg_ctx* c) {
  const sg_config& cfg = c->cfg;
  c->mixed = cfg.precision == SG_PREC_MIXED;
  c->esz = c->mixed ? 4 : 8;
  const size_t E = c->esz;
  const int pi = c->mixed ? 1 : 0;
  SG_TRY(cudaSetDevice(cfg.device), "cudaSetDevice");
  if (cfg.stream) {
    c->st = (cudaStream_t)cfg.stream;
  } else {
    SG_TRY(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking), "cudaStreamCreate");
    c->own_stream = true;
  }
  // FP32 spreads on 16 x 16 x 8 tiles (fewer points straddle a tile edge);
  // FP64 keeps 1024-cell tiles for its three-limb shared accumulators
  const int shape = (c->mixed && cfg.itot >= 16 && cfg.jtot >= 16) ? 1 : -1;
  const unsigned allowed = c->mixed ? kAllTileShapes : kFp64TileShapes;
  if (!make_ib_grid(cfg.itot, cfg.jtot, cfg.ktot, cfg.lx, cfg.ly, cfg.lz, c->grid, shape, allowed) &&
      !make_ib_grid(cfg.itot, cfg.jtot, cfg.ktot, cfg.lx, cfg.ly, cfg.lz, c->grid, -1, allowed))
    return fail(c, SG_ERR_CONFIG,
                "grid out of range: need itot, jtot >= 8, (itot+2)(jtot+2)(ktot+2) < 2^31, and a tile shape whose "
                "last tile in x and y is not 1 or 2 cells wide (FP64: 32x8x4 or 8x8x4)");
  const IBGrid& g = c->grid;
  c->nfield = (long long)g.ldi * g.ldj * g.ldk;
  // capsules, offsets, degree groups
  const int ncap = cfg.ncap;
  c->off.assign(ncap + 1, 0);
  std::map<int, int> gid;
  for (int k = 0; k < ncap; ++k) {
    const int L = c->degree[k];
    c->off[k + 1] = c->off[k] + 8LL * (L + 1) * (L + 1);
    if (!gid.count(L)) {
      gid[L] = (int)c->groups.size();
      Group gr;
      gr.L = L; gr.N = L + 1; gr.nD = 2 * (L + 1); gr.mD = 4 * (L + 1); gr.nO = L + 1; gr.mO = 2 * (L + 1);
      c->groups.push_back(gr);
    }
    c->groups[gid[L]].caps.push_back(k);
  }
  c->npts = (long)c->off[ncap];
  std::vector<CapInfo> caps(ncap);
  for (size_t gi = 0; gi < c->groups.size(); ++gi) {
    Group& gr = c->groups[gi];
    c->nmax = std::max(c->nmax, gr.N);
    for (size_t q = 0; q < gr.caps.size(); ++q) {
      const int k = gr.caps[q];
      caps[k].L = gr.L; caps[k].N = gr.N; caps[k].group = (int)gi; caps[k].law = SG_LAW_SKALAK;
      caps[k].pt_off = c->off[k]; caps[k].gidx = (long long)q; caps[k].R = c->radius[k];
      caps[k].gs = cfg.gs; caps[k].csk = cfg.csk;
    }
    cudaError_t e = build_tables(c, gr);
    if (e != cudaSuccess) return cuda_fail(c, e, "tables");
    const long long n = (long long)gr.caps.size(), N = gr.N;
    SG_TRY(dalloc(c, gr.buf.Fpos, E * n * 6 * N * gr.nD), "alloc");
    SG_TRY(dalloc(c, gr.buf.Cpos, E * n * 6 * N * N), "alloc");
    SG_TRY(dalloc(c, gr.buf.G, E * n * 6 * N * 3 * gr.nD), "alloc");
    SG_TRY(dalloc(c, gr.buf.Fout, E * n * 12 * N * gr.nD), "alloc");
    SG_TRY(dalloc(c, gr.buf.Cout, E * n * 12 * N * N), "alloc");
    SG_TRY(dalloc(c, gr.buf.GO, E * n * 12 * N * 2 * gr.nO), "alloc");
    SG_TRY(dalloc(c, gr.buf.Fsh, E * n * 8 * N * gr.nO), "alloc");
    SG_TRY(dalloc(c, gr.buf.Csh, E * n * 8 * N * N), "alloc");
    SG_TRY(dalloc(c, gr.buf.GF, E * n * 14 * N * gr.nD), "alloc");
  }
  void* tmp = nullptr;
  SG_TRY(upload(c, tmp, caps), "caps");
  c->d_caps = (CapInfo*)tmp;
  c->h_caps = caps;
  SG_TRY(dalloc(c, c->d_groups, sizeof(GroupDev) * std::max<size_t>(c->groups.size(), 1)), "alloc");
  SG_RET(upload_groups(c));
  // capsule work lists of the persistent pointwise kernels (set_point_split)
  const size_t maxitems = (size_t)kMaxPointSplit * std::max(ncap, 1);
  SG_TRY(dalloc(c, c->d_wpos, sizeof(RowWork) * maxitems), "alloc");
  SG_TRY(dalloc(c, c->d_cen, sizeof(double) * 3 * std::max(c->cfg.ncap, 1)), "alloc");
  {
    // the fused force stage's capsule order: largest degree first, then index
    std::vector<int> order(c->cfg.ncap);
    for (int k = 0; k < c->cfg.ncap; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return c->h_caps[a].N > c->h_caps[b].N; });
    void* tmp = nullptr;
    if (order.empty()) order.push_back(0);
    SG_TRY(upload(c, tmp, order), "order");
    c->d_order = (int*)tmp;
  }
  SG_TRY(dalloc(c, c->d_wmem, sizeof(RowWork) * maxitems), "alloc");
  SG_TRY(dalloc(c, c->d_wsh, sizeof(RowWork) * maxitems), "alloc");
  SG_TRY(dalloc(c, c->d_wfin, sizeof(RowWork) * maxitems), "alloc");
  SG_RET(set_point_split(c, 2));
  // Legendre problems per stage
  std::vector<LegProblem> P;
  std::vector<LegWork> W[6];
  for (size_t gi = 0; gi < c->groups.size(); ++gi) {
    const Group& gr = c->groups[gi];
    const int n = (int)gr.caps.size();
    const long long N = gr.N, nD = gr.nD, nO = gr.nO;
    const SpecBuffers& b = gr.buf;
    const int G = (int)gi;
    // S0: analysis of the displacement (force grid, truncated to degree < N)
    add_problem(P, W[0], prob(b.Fpos, 6 * N * nD, N * nD, nD, gr.tab.ana_D[pi], N * nD, b.Cpos, 6 * N * N, N * N, N,
                              6, n, N, N, nD, 0, G, 1), c->maxJ[0], c->maxK[0]);
    // S1: synthesis of P, dP, d2P series on the dealias grid
    add_problem(P, W[1], prob(b.Cpos, 6 * N * N, N * N, N, gr.tab.syn_D[pi], 3 * nD * N, b.G, 6 * N * 3 * nD,
                              N * 3 * nD, 3 * nD, 6, n, N, 3 * nD, N, 1, G, 0), c->maxJ[1], c->maxK[1]);
    // S2: analysis of force and normals (dealias grid, truncated)
    add_problem(P, W[2], prob(b.Fout, 12 * N * nD, N * nD, nD, gr.tab.ana_D[pi], N * nD, b.Cout, 12 * N * N, N * N, N,
                              12, n, N, N, nD, 0, G, 1), c->maxJ[2], c->maxK[2]);
    // S3: synthesis on the SH grid: normals (rows 0-5) and shape (rows 6-11)
    add_problem(P, W[3], prob((const char*)b.Cout + E * 6 * N * N, 12 * N * N, N * N, N, gr.tab.syn_O[pi],
                              2 * nO * N, b.GO, 12 * N * 2 * nO, N * 2 * nO, 2 * nO, 6, n, N, 2 * nO, N, 1, G, 2),
                c->maxJ[3], c->maxK[3]);
    add_problem(P, W[3], prob(b.Cpos, 6 * N * N, N * N, N, gr.tab.syn_O[pi], 2 * nO * N,
                              (char*)b.GO + E * 6 * N * 2 * nO, 12 * N * 2 * nO, N * 2 * nO, 2 * nO, 6, n, N, 2 * nO,
                              N, 1, G, 2),
                c->maxJ[3], c->maxK[3]);
    // S4: analysis on the SH grid of renormalised normals and surface metric
    add_problem(P, W[4], prob(b.Fsh, 8 * N * nO, N * nO, nO, gr.tab.ana_O[pi], N * nO, b.Csh, 8 * N * N, N * N, N, 8,
                              n, N, N, nO, 0, G, 3), c->maxJ[4], c->maxK[4]);
    // S5: synthesis on the force grid (P only): force rows 0-5, normals+surfmet rows 6-13
    add_problem(P, W[5], prob(b.Cout, 12 * N * N, N * N, N, gr.tab.syn_D[pi], 3 * nD * N, b.GF, 14 * N * nD, N * nD,
                              nD, 6, n, N, nD, N, 1, G, 0), c->maxJ[5], c->maxK[5]);
    add_problem(P, W[5], prob(b.Csh, 8 * N * N, N * N, N, gr.tab.syn_D[pi], 3 * nD * N,
                              (char*)b.GF + E * 6 * N * nD, 14 * N * nD, N * nD, nD, 8, n, N, nD, N, 1, G, 0),
                c->maxJ[5], c->maxK[5]);
  }
  // tensor-core path (FP32 data): three launches of chained contractions.
  // Per group the problems above are, in order, S0 S1 S2 S3a S3b S4 S5a S5b;
  // S2 is split into its force rows (S2f) and normal rows (S2n) so that each
  // half chains into the synthesis that consumes it:
  //   launch 0: S0 -> {S1, S3b}      launch 1: S2n -> S3a, S2f -> S5a
  //   launch 2: S4 -> S5b
  // With the surrogate on, S5a runs in launch 2 instead, after the surrogate
  // force has replaced the analysed force rows.
  std::vector<int> roots[3];
  if (c->mixed) {
    const size_t ng = c->groups.size();
    for (size_t gi = 0; gi < ng; ++gi) {
      const Group& gr = c->groups[gi];
      const long long N = gr.N, nD = gr.nD;
      const int base = 8 * (int)gi;
      LegProblem f = P[base + 2], nrm = P[base + 2];
      f.rpc = 6;
      f.Q = 6 * (int)gr.caps.size();
      nrm.rpc = 6;
      nrm.Q = f.Q;
      nrm.A = (const char*)nrm.A + E * 6 * N * nD;
      nrm.D = (char*)nrm.D + E * 6 * N * N;
      const int iF = (int)P.size(), iN = iF + 1;
      P.push_back(f);
      P.push_back(nrm);
      P[base + 0].next[0] = base + 1;  // S0 -> S1
      P[base + 0].next[1] = base + 4;  // S0 -> S3b
      P[iN].next[0] = base + 3;        // S2n -> S3a
      if (!cfg.surrogate) P[iF].next[0] = base + 6;  // S2f -> S5a
      P[base + 5].next[0] = base + 7;  // S4 -> S5b
      roots[0].push_back(base + 0);
      roots[1].push_back(iN);
      roots[1].push_back(iF);
      roots[2].push_back(base + 5);
      if (cfg.surrogate) roots[2].push_back(base + 6);
    }
    for (int f = 0; f < 3; ++f) c->leg_roots[f] = roots[f];
  }
  // tensor-core operands: the three bf16 parts of every problem's table, and
  // work lists of 128-row tiles of the root problems (FP32 data only)
  if (c->mixed) {
    std::vector<uint16_t> img;
    std::vector<size_t> img_off(P.size());
    for (size_t pi2 = 0; pi2 < P.size(); ++pi2) {
      LegProblem& p = P[pi2];
      p.Jp = (p.J + 15) / 16 * 16;
      p.Kp = (p.K + 15) / 16 * 16;
      p.sBimg = 3LL * p.Jp * p.Kp;
      img_off[pi2] = img.size();
      img.resize(img.size() + (size_t)p.M * p.sBimg);
      const std::vector<double>& hb = c->groups[p.group].h_tab[p.kind];
      host_umma_image(hb.data(), p.sBm, p.M, p.J, p.K, p.Jp, p.Kp, img.data() + img_off[pi2]);
      auto al4 = [](const void* ptr) { return ((uintptr_t)ptr & 15u) == 0; };
      p.vecA = (al4(p.A) && p.sAc % 4 == 0 && p.sAr % 4 == 0 && p.sAm % 4 == 0 && p.K % 8 == 0) ? 1 : 0;
      p.vecD = (al4(p.D) && p.sDc % 4 == 0 && p.sDr % 4 == 0 && p.sDm % 4 == 0 && p.J % 4 == 0) ? 1 : 0;
    }
    void* dimg = nullptr;
    SG_TRY(upload(c, dimg, img), "umma images");
    for (size_t pi2 = 0; pi2 < P.size(); ++pi2) P[pi2].Bimg = (const uint16_t*)dimg + img_off[pi2];
    for (int f = 0; f < 3; ++f) {
      // work lists on 128-row and on 64-row tiles (the launches use the
      // 128-row list unless sg_set_legendre_tile_rows or the autotuner switch)
      for (int t = 0; t < 2; ++t) {
        const int tm = t ? 64 : 128;
        std::vector<LegWork> WT;
        for (int r : roots[f])
          for (int m = 0; m < P[r].M; ++m)
            for (int q0 = 0; q0 < P[r].Q; q0 += tm)
              WT.push_back(LegWork{r, m, q0, P[r].next[0], P[r].next[0] >= 0 ? P[r].next[1] : -1});
        c->nlwT[t][f] = (int)WT.size();
        SG_TRY(upload(c, tmp, WT), "work");
        c->d_lwT[t][f] = (LegWork*)tmp;
      }
      c->tmF[f] = 128;
      for (int r : roots[f]) {
        const LegProblem& p = P[r];
        const int chain[3] = {r, p.next[0], p.next[0] >= 0 ? p.next[1] : -1};
        LegLevels& lv = c->lvF[f];
        for (int l = 0; l < 3; ++l) {
          const int q = chain[l];
          if (q < 0) continue;
          lv.jp[l] = std::max(lv.jp[l], P[q].Jp);
          lv.kp[l] = std::max(lv.kp[l], P[q].Kp);
          lv.a_kp = std::max(lv.a_kp, P[q].Kp);
        }
      }
      c->nlwF[f] = c->nlwT[0][f];
      c->d_lwF[f] = c->d_lwT[0][f];
    }
    c->leg_tc = true;
    assign_terms(c, P);
  }
  c->h_probs = P;
  SG_TRY(upload(c, tmp, P), "problems");
  c->d_probs = (LegProblem*)tmp;
  if (c->mixed) {
    // the fused force stage: the per-group problems 8 g .. 8 g + 7 with their
    // FP32 tables; its staged A rows take rpc M K floats at most
    for (size_t q = 0; q < 8 * c->groups.size(); ++q)
      c->fused_cf = std::max(c->fused_cf, (size_t)P[q].rpc * P[q].M * P[q].K);
  }
  for (int s = 0; s < 6; ++s) {
    c->nlw[s] = (int)W[s].size();
    SG_TRY(upload(c, tmp, W[s]), "work");
    c->d_lw[s] = (LegWork*)tmp;
  }
  SG_TRY(dalloc(c, c->d_err, sizeof(int)), "alloc");
  SG_TRY(cudaMemset(c->d_err, 0, sizeof(int)), "memset");
  SG_TRY(cudaMallocHost(&c->h_err, sizeof(int)), "cudaMallocHost");
  *c->h_err = 0;
  SG_TRY(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, cfg.device), "attribute");
  SG_RET(sur_setup(c));
  // binning work
  const long np = std::max(c->npts, 1L);
  SG_TRY(dalloc(c, c->ibw.pos, (c->mixed ? sizeof(PosRec<float>) : sizeof(PosRec<double>)) * np), "alloc");
  SG_TRY(dalloc(c, c->ibw.frc, (c->mixed ? sizeof(ForceRec<float>) : sizeof(ForceRec<double>)) * np), "alloc");
  SG_TRY(dalloc(c, c->ibw.entries, sizeof(int) * 8 * np), "alloc");
  c->max_tiles = g.ntiles;
  for (int sh = 0; sh < kNumTileShapes; ++sh) {
    IBGrid t{};
    if (make_ib_grid(cfg.itot, cfg.jtot, cfg.ktot, cfg.lx, cfg.ly, cfg.lz, t, sh))
      c->max_tiles = std::max(c->max_tiles, t.ntiles);
  }
  SG_TRY(dalloc(c, c->ibw.counts, sizeof(int) * c->max_tiles), "alloc");
  SG_TRY(dalloc(c, c->ibw.starts, sizeof(int) * (c->max_tiles + 1)), "alloc");
  SG_TRY(dalloc(c, c->ibw.fill, sizeof(int) * c->max_tiles), "alloc");
  SG_TRY(cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking), "cudaStreamCreate");
  SG_TRY(cudaEventCreateWithFlags(&c->ev_bin, cudaEventDisableTiming), "cudaEventCreate");
  SG_TRY(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming), "cudaEventCreate");
  if (cfg.mem == SG_MEM_HOST) {
    SG_TRY(cudaStreamCreateWithFlags(&c->st3, cudaStreamNonBlocking), "cudaStreamCreate");
    SG_TRY(cudaEventCreateWithFlags(&c->ev_frc, cudaEventDisableTiming), "cudaEventCreate");
    SG_TRY(cudaEventCreateWithFlags(&c->ev_join3, cudaEventDisableTiming), "cudaEventCreate");
  }
  if (cfg.mem == SG_MEM_HOST) {
    SG_TRY(dalloc(c, c->s_u, E * c->nfield), "alloc");
    SG_TRY(dalloc(c, c->s_v, E * c->nfield), "alloc");
    SG_TRY(dalloc(c, c->s_w, E * c->nfield), "alloc");
    for (int q = 0; q < 3; ++q) SG_TRY(dalloc(c, c->s_f[q], E * c->nfield), "alloc");
    SG_TRY(dalloc(c, c->s_X, sizeof(double) * np), "alloc");
    SG_TRY(dalloc(c, c->s_Y, sizeof(double) * np), "alloc");
    SG_TRY(dalloc(c, c->s_Z, sizeof(double) * np), "alloc");
    for (int q = 0; q < 10; ++q) SG_TRY(dalloc(c, c->s_lag[q], E * np), "alloc");
    SG_TRY(dalloc(c, c->s_out, sizeof(double) * 7 * std::max(ncap, 1)), "alloc");
    SG_TRY(dalloc(c, c->s_exy, sizeof(double) * std::max(ncap, 1)), "alloc");
  }
  SG_TRY(cudaDeviceSynchronize(), "setup");
  return SG_OK;
}

// ------------------------------------------------------------ pipeline ----
template <class T>
int dev_bin(sg_ctx* c, const double* X, const double* Y, const double* Z, cudaStream_t st) {
  SG_TRY(launch_bin<T>(c->grid, c->npts, X, Y, Z, c->ibw, st), "bin");
  c->launches += c->npts > 0 ? 3 : 1;
  return SG_OK;
}

template <class T>
int dev_interp(sg_ctx* c, const T* u, const T* v, const T* w, T* U, T* V, T* W, cudaStream_t st) {
  SG_TRY(launch_interp<T>(c->grid, c->npts, c->ibw, u, v, w, U, V, W, st), "interp");
  c->launches += 1;
  return SG_OK;
}

// Events around one contraction launch when the step is profiled (the
// SG_STAGE_CONTRACT time is their sum).
int con_mark(sg_ctx* c, int end) {
  if (!c->profiling || c->capturing || !c->ev_con[0][0] || c->ncon >= sg_ctx::kMaxContract) return SG_OK;
  SG_TRY(cudaEventRecord(c->ev_con[end][c->ncon], c->st), "event");
  if (end) ++c->ncon;
  return SG_OK;
}

template <class T>
int dev_legendre(sg_ctx* c, int s) {
  if (sizeof(T) == 4 && c->leg_tc) {
    // stages 0, 2, 4 launch the chained products; 1, 3, 5 ran inside them
    if (s % 2) return SG_OK;
    const int f = s / 2;
    SG_RET(con_mark(c, 0));
    SG_TRY(launch_legendre_mma(c->d_probs, c->d_lwF[f], c->nlwF[f], c->lvF[f], c->leg_parts, c->tmF[f],
                               c->d_err, c->num_sms, c->st),
           "legendre (tensor cores)");
    SG_RET(con_mark(c, 1));
    c->launches += 1;
  } else {
    SG_RET(con_mark(c, 0));
    SG_TRY(launch_legendre<T>(c->d_probs, c->d_lw[s], c->nlw[s], c->maxJ[s], c->maxK[s], c->st), "legendre");
    SG_RET(con_mark(c, 1));
    c->launches += 1;
  }
  return SG_OK;
}

template <class T>
int dev_forces(sg_ctx* c, const double* X, const double* Y, const double* Z, T* FX, T* FY, T* FZ, T* NX, T* NY,
               T* NZ, T* A) {
  const int nc = c->cfg.ncap;
  c->ncon = 0;
  if (nc == 0) return SG_OK;
  if constexpr (sizeof(T) == 4) {
    if (c->fused && !c->bend && !sur_flags(c)) {
      SG_TRY(launch_force_fused(c->d_order, nc, c->d_caps, c->d_groups, c->d_probs, X, Y, Z, c->d_cen, FX, FY, FZ, NX,
                                NY, NZ, A, c->ibw.frc, c->grid.dvi, c->nmax, c->fused_cf, c->st),
             "force (fused)");
      c->launches += 1;
      return SG_OK;
    }
  }
  SG_TRY(launch_posfwd<T>(c->d_wpos, c->nwpos, c->d_caps, c->d_groups, X, Y, Z, nc, c->d_cen, c->nmax, c->st),
         "posfwd");
  SG_RET(dev_legendre<T>(c, 0));
  const bool f32 = sizeof(T) == 4;
  if (f32) SG_RET(sur_step_pre(c));  // surrogate force and its residual check
  SG_RET(dev_legendre<T>(c, 1));
  if (c->bend) {
    // the third and fourth derivative series of the shape (problem S1b)
    SG_RET(con_mark(c, 0));
    if (f32 && c->leg_tc)
      SG_TRY(launch_legendre_mma(c->d_probs, c->d_lwBT, c->nlwBT, c->lvB, c->leg_parts, 128, c->d_err, c->num_sms,
                                 c->st),
             "legendre (bending)");
    else
      SG_TRY(launch_legendre<T>(c->d_probs, c->d_lwB, c->nlwB, c->maxJB, c->maxKB, c->st), "legendre (bending)");
    SG_RET(con_mark(c, 1));
    c->launches += 1;
    SG_TRY(launch_membrane_bend<T>(c->d_wmem, c->nwmem, c->d_caps, c->d_groups, f32 ? sur_flags(c) : nullptr,
                                   c->nmax, c->st),
           "membrane (bending)");
  } else {
    SG_TRY(launch_membrane<T>(c->d_wmem, c->nwmem, c->d_caps, c->d_groups, f32 ? sur_flags(c) : nullptr, c->nmax,
                              c->d_err, c->st),
           "membrane");
  }
  SG_RET(dev_legendre<T>(c, 2));
  if (f32) SG_RET(sur_step_post(c));
  SG_RET(dev_legendre<T>(c, 3));
  SG_TRY(launch_shgrid<T>(c->d_wsh, c->nwsh, c->d_caps, c->d_groups, c->nmax, c->d_err, c->st), "shgrid");
  SG_RET(dev_legendre<T>(c, 4));
  SG_RET(dev_legendre<T>(c, 5));
  SG_TRY(launch_final<T>(c->d_wfin, c->nwfin, c->d_caps, c->d_groups, FX, FY, FZ, NX, NY, NZ, A, c->ibw.frc,
                         c->grid.dvi, c->nmax, c->d_err, c->st),
         "final");
  c->launches += 5;  // centroids, posfwd, membrane, shgrid, final (Legendre launches counted above)
  return SG_OK;
}

// have_rec: the force records were written by this step's final synthesis;
// otherwise they are packed from the caller's force and area arrays first.
template <class T>
int dev_spread(sg_ctx* c, const T* FX, const T* FY, const T* FZ, const T* A, T* fx, T* fy, T* fz, bool have_rec) {
  if (!have_rec) {
    SG_TRY(launch_pack_forces<T>(c->grid, c->npts, FX, FY, FZ, A, c->ibw, c->st), "pack forces");
    c->launches += c->npts > 0 ? 1 : 0;
  }
  SG_TRY(launch_spread<T>(c->grid, c->ibw, fx, fy, fz, c->st), "spread");
  c->launches += 1;
  return SG_OK;
}

// Reports a bounded device wait that expired (flag copied to pinned memory
// at the end of each step) once the stream has been synchronised.
int check_err(sg_ctx* c) {
  if (c->h_err && *c->h_err) {
    *c->h_err = 0;
    SG_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st), "memset");
    return fail(c, SG_ERR_TIMEOUT, "a tensor-core completion wait timed out");
  }
  return SG_OK;
}

int finish(sg_ctx* c) {
  if (c->capturing) return SG_OK;
  if (!c->cfg.async || c->cfg.mem == SG_MEM_HOST) {
    SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
    SG_RET(check_err(c));
  }
  return SG_OK;
}

int h2d(sg_ctx* c, void* dst, const void* src, size_t bytes, cudaStream_t st = nullptr) {
  SG_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st ? st : c->st), "h2d");
  return SG_OK;
}
int d2h(sg_ctx* c, void* dst, const void* src, size_t bytes, cudaStream_t st = nullptr) {
  SG_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st ? st : c->st), "d2h");
  return SG_OK;
}


template <class T>
int run_step(sg_ctx* c, int what, const void* u, const void* v, const void* w, const double* X, const double* Y,
             const double* Z, void* U, void* V, void* W, void* FX, void* FY, void* FZ, void* NX, void* NY, void* NZ,
             void* A, void* fx, void* fy, void* fz) {
  // what: bit0 interp, bit1 forces, bit2 spread (spread reads FX.. and A as inputs when bit1 is clear)
  const bool host = c->cfg.mem == SG_MEM_HOST;
  const size_t pb = sizeof(double) * c->npts, lb = sizeof(T) * c->npts, fb = sizeof(T) * c->nfield;
  c->launches = 0;
  const double *dX = X, *dY = Y, *dZ = Z;
  const T *du = (const T*)u, *dv = (const T*)v, *dw = (const T*)w;
  T* L[10] = {(T*)U, (T*)V, (T*)W, (T*)FX, (T*)FY, (T*)FZ, (T*)NX, (T*)NY, (T*)NZ, (T*)A};
  T *dfx = (T*)fx, *dfy = (T*)fy, *dfz = (T*)fz;
  // Full step on two streams (when not profiling): binning and the
  // interpolation branch (velocity upload, interp, velocity download) run on
  // st2, the force branch (forces, spread, their downloads) on st.  The force
  // stage reads only the positions, so it runs beside the binning and the
  // interpolation; the spread waits for the binning, and st waits for st2
  // before the step ends.  In host memory the velocity upload on one stream
  // also overlaps the downloads on the other (the spread does not read the
  // velocity).  In host memory the force downloads go to a third stream that
  // forks after the force stage, so that they run beside the spread.  A
  // captured graph takes the same forks and joins.
  const bool dual = c->st2 && (what & 1) && (what & 6) && !c->profiling;
  cudaStream_t sB = dual ? c->st2 : c->st;
  if (host) {
    SG_RET(h2d(c, c->s_X, X, pb));
    SG_RET(h2d(c, c->s_Y, Y, pb));
    SG_RET(h2d(c, c->s_Z, Z, pb));
    dX = c->s_X; dY = c->s_Y; dZ = c->s_Z;
    for (int q = 0; q < 10; ++q) L[q] = (T*)c->s_lag[q];
    if ((what & 4) && !(what & 2)) {
      SG_RET(h2d(c, L[3], FX, lb));
      SG_RET(h2d(c, L[4], FY, lb));
      SG_RET(h2d(c, L[5], FZ, lb));
      SG_RET(h2d(c, L[9], A, lb));
    }
    dfx = (T*)c->s_f[0]; dfy = (T*)c->s_f[1]; dfz = (T*)c->s_f[2];
  }
  if (dual) {  // st2 starts after everything queued on st so far (positions included)
    SG_TRY(cudaEventRecord(c->ev_join, c->st), "event");
    SG_TRY(cudaStreamWaitEvent(sB, c->ev_join, 0), "stream wait");
  }
  auto mark = [&](int k) -> int {
    if (c->profiling && !c->capturing) SG_TRY(cudaEventRecord(c->ev[k], c->st), "event");
    return SG_OK;
  };
  SG_RET(mark(0));
  if (what & 5) SG_RET(dev_bin<T>(c, dX, dY, dZ, sB));
  if (dual) SG_TRY(cudaEventRecord(c->ev_bin, sB), "event");
  SG_RET(mark(1));
  if (what & 1) {
    if (host) {
      SG_RET(h2d(c, c->s_u, u, fb, sB));
      SG_RET(h2d(c, c->s_v, v, fb, sB));
      SG_RET(h2d(c, c->s_w, w, fb, sB));
      du = (const T*)c->s_u; dv = (const T*)c->s_v; dw = (const T*)c->s_w;
    }
    SG_RET(dev_interp<T>(c, du, dv, dw, L[0], L[1], L[2], sB));
    if (host) {
      SG_RET(d2h(c, U, L[0], lb, sB));
      SG_RET(d2h(c, V, L[1], lb, sB));
      SG_RET(d2h(c, W, L[2], lb, sB));
    }
  }
  if (dual) SG_TRY(cudaEventRecord(c->ev_join, sB), "event");
  SG_RET(mark(2));
  if (what & 2) {
    SG_RET(dev_forces<T>(c, dX, dY, dZ, L[3], L[4], L[5], L[6], L[7], L[8], L[9]));
    if (c->wall_in_step && (what & 4)) {  // call collisions between complagrforces and lagr2eulr (main.f90:229-233)
      SG_TRY(launch_collisions<T>(c->npts, c->wall, dZ, L[9], L[5], c->ibw.frc, c->grid.dvi, c->st), "collisions");
      c->launches += c->npts > 0 ? 1 : 0;
    }
    if (host) {
      // beside the spread when one follows: the download direction then has no gap while it runs
      const bool side = dual && (what & 4) && c->st3;
      if (side) {
        SG_TRY(cudaEventRecord(c->ev_frc, c->st), "event");
        SG_TRY(cudaStreamWaitEvent(c->st3, c->ev_frc, 0), "stream wait");
      }
      void* outs[7] = {FX, FY, FZ, NX, NY, NZ, A};
      for (int q = 0; q < 7; ++q) SG_RET(d2h(c, outs[q], L[3 + q], lb, side ? c->st3 : nullptr));
      if (side) {
        SG_TRY(cudaEventRecord(c->ev_join3, c->st3), "event");
        c->join3 = true;
      }
    }
  }
  SG_RET(mark(3));
  if (what & 4) {
    if (dual) SG_TRY(cudaStreamWaitEvent(c->st, c->ev_bin, 0), "stream wait");
    SG_RET(dev_spread<T>(c, L[3], L[4], L[5], L[9], dfx, dfy, dfz, (what & 2) != 0));
    if (host) {
      SG_RET(d2h(c, fx, dfx, fb));
      SG_RET(d2h(c, fy, dfy, fb));
      SG_RET(d2h(c, fz, dfz, fb));
    }
  }
  SG_RET(mark(4));
  c->ev_used[0] = (what & 5) != 0;
  c->ev_used[1] = (what & 1) != 0;
  c->ev_used[2] = (what & 2) != 0;
  c->ev_used[3] = (what & 4) != 0;
  if (dual) SG_TRY(cudaStreamWaitEvent(c->st, c->ev_join, 0), "stream wait");
  if (c->join3) {
    SG_TRY(cudaStreamWaitEvent(c->st, c->ev_join3, 0), "stream wait");
    c->join3 = false;
  }
  if (what & 2)  // bounded waits of the force kernels
    SG_TRY(cudaMemcpyAsync(c->h_err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st), "error flag");
  SG_TRY(cudaGetLastError(), "step");
  return finish(c);
}

}  // namespace

int sg::run_forces_only(sg_ctx* c, const double* X, const double* Y, const double* Z, void* const* lag) {
  const bool host = c->cfg.mem == SG_MEM_HOST;
  const size_t pb = sizeof(double) * c->npts;
  const double *dX = X, *dY = Y, *dZ = Z;
  if (host) {
    SG_RET(h2d(c, c->s_X, X, pb));
    SG_RET(h2d(c, c->s_Y, Y, pb));
    SG_RET(h2d(c, c->s_Z, Z, pb));
    dX = c->s_X; dY = c->s_Y; dZ = c->s_Z;
  }
  c->launches = 0;
  if (c->mixed) {
    float* L[7];
    for (int q = 0; q < 7; ++q) L[q] = (float*)lag[q];
    SG_RET(dev_forces<float>(c, dX, dY, dZ, L[0], L[1], L[2], L[3], L[4], L[5], L[6]));
  } else {
    double* L[7];
    for (int q = 0; q < 7; ++q) L[q] = (double*)lag[q];
    SG_RET(dev_forces<double>(c, dX, dY, dZ, L[0], L[1], L[2], L[3], L[4], L[5], L[6]));
  }
  SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
  return check_err(c);
}

namespace {

int check_ptrs(sg_ctx* c, std::initializer_list<const void*> ps) {
  if (c->npts == 0) return SG_OK;
  for (const void* p : ps)
    if (!p) return fail(c, SG_ERR_ARG, "null array argument");
  return SG_OK;
}

}  // namespace

// ================================================================ C ABI ===
extern "C" {

int sg_create(const sg_config* cfg, sg_ctx** out) {
  if (!cfg || !out) return SG_ERR_ARG;
  *out = nullptr;
  sg_ctx* c = new sg_ctx();
  c->cfg = *cfg;
  int rc = SG_OK;
  if (cfg->ncap < 0 || (cfg->ncap > 0 && (!cfg->degree || !cfg->radius))) {
    rc = fail(c, SG_ERR_CONFIG, "ncap < 0 or missing degree/radius arrays");
  } else if (cfg->precision != SG_PREC_FP64 && cfg->precision != SG_PREC_MIXED) {
    rc = fail(c, SG_ERR_CONFIG, "precision must be SG_PREC_FP64 or SG_PREC_MIXED");
  } else if (cfg->mem != SG_MEM_HOST && cfg->mem != SG_MEM_DEVICE) {
    rc = fail(c, SG_ERR_CONFIG, "mem must be SG_MEM_HOST or SG_MEM_DEVICE");
  } else if (!(cfg->lx > 0 && cfg->ly > 0 && cfg->lz > 0)) {
    rc = fail(c, SG_ERR_CONFIG, "domain lengths must be positive");
  } else if (cfg->surrogate && cfg->precision != SG_PREC_MIXED) {
    rc = fail(c, SG_ERR_CONFIG, "the surrogate runs on the mixed path only");
  } else {
    c->degree.assign(cfg->degree, cfg->degree + cfg->ncap);
    c->radius.assign(cfg->radius, cfg->radius + cfg->ncap);
    for (int k = 0; k < cfg->ncap && rc == SG_OK; ++k) {
      if (c->degree[k] < 2 || c->degree[k] > 31) rc = fail(c, SG_ERR_CONFIG, "SH degree must be in [2, 31]");
      if (!(c->radius[k] > 0)) rc = fail(c, SG_ERR_CONFIG, "capsule radius must be positive");
    }
    c->cfg.degree = nullptr;
    c->cfg.radius = nullptr;
    if (rc == SG_OK) rc = setup(c);
  }
  *out = c;  // returned even on failure so sg_last_error can report; caller destroys
  return rc;
}

void sg_destroy(sg_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->cfg.device);
  if (c->st) cudaStreamSynchronize(c->st);
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  if (c->graph) cudaGraphDestroy(c->graph);
  poisson_free(c);
  for (void* p : c->allocs) cudaFree(p);
  for (int k = 0; k <= sg_ctx::kMarkStages; ++k)
    if (c->ev[k]) cudaEventDestroy(c->ev[k]);
  for (int e = 0; e < 2; ++e)
    for (int k = 0; k < sg_ctx::kMaxContract; ++k)
      if (c->ev_con[e][k]) cudaEventDestroy(c->ev_con[e][k]);
  if (c->own_stream && c->st) cudaStreamDestroy(c->st);
  if (c->st2) {
    cudaStreamSynchronize(c->st2);
    cudaStreamDestroy(c->st2);
  }
  if (c->ev_bin) cudaEventDestroy(c->ev_bin);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->st3) {
    cudaStreamSynchronize(c->st3);
    cudaStreamDestroy(c->st3);
  }
  if (c->ev_frc) cudaEventDestroy(c->ev_frc);
  if (c->ev_join3) cudaEventDestroy(c->ev_join3);
  if (c->h_err) cudaFreeHost(c->h_err);
  if (c->h_sur_count) cudaFreeHost(c->h_sur_count);
  delete c;
}

const char* sg_last_error(const sg_ctx* c) { return c ? c->err.c_str() : "null context"; }

int sg_synchronize(sg_ctx* c) {
  if (!c) return SG_ERR_ARG;
  SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
  return check_err(c);
}

int sg_interp(sg_ctx* c, const void* u, const void* v, const void* w, const double* X, const double* Y,
              const double* Z, void* U, void* V, void* W) {
  if (!c) return SG_ERR_ARG;
  SG_RET(check_ptrs(c, {u, v, w, X, Y, Z, U, V, W}));
  if (c->mixed)
    return run_step<float>(c, 1, u, v, w, X, Y, Z, U, V, W, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0);
  return run_step<double>(c, 1, u, v, w, X, Y, Z, U, V, W, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0);
}

int sg_membrane_force(sg_ctx* c, const double* X, const double* Y, const double* Z, void* FX, void* FY, void* FZ,
                      void* NX, void* NY, void* NZ, void* AREA) {
  if (!c) return SG_ERR_ARG;
  SG_RET(check_ptrs(c, {X, Y, Z, FX, FY, FZ, NX, NY, NZ, AREA}));
  if (c->mixed)
    return run_step<float>(c, 2, 0, 0, 0, X, Y, Z, 0, 0, 0, FX, FY, FZ, NX, NY, NZ, AREA, 0, 0, 0);
  return run_step<double>(c, 2, 0, 0, 0, X, Y, Z, 0, 0, 0, FX, FY, FZ, NX, NY, NZ, AREA, 0, 0, 0);
}

int sg_spread(sg_ctx* c, const double* X, const double* Y, const double* Z, const void* FX, const void* FY,
              const void* FZ, const void* AREA, void* fx, void* fy, void* fz) {
  if (!c) return SG_ERR_ARG;
  if (!fx || !fy || !fz) return fail(c, SG_ERR_ARG, "null field argument");
  SG_RET(check_ptrs(c, {X, Y, Z, FX, FY, FZ, AREA}));
  if (c->mixed)
    return run_step<float>(c, 4, 0, 0, 0, X, Y, Z, 0, 0, 0, (void*)FX, (void*)FY, (void*)FZ, 0, 0, 0, (void*)AREA,
                           fx, fy, fz);
  return run_step<double>(c, 4, 0, 0, 0, X, Y, Z, 0, 0, 0, (void*)FX, (void*)FY, (void*)FZ, 0, 0, 0, (void*)AREA, fx,
                          fy, fz);
}

int sg_step(sg_ctx* c, const void* u, const void* v, const void* w, const double* X, const double* Y,
            const double* Z, void* U, void* V, void* W, void* FX, void* FY, void* FZ, void* NX, void* NY, void* NZ,
            void* AREA, void* fx, void* fy, void* fz) {
  if (!c) return SG_ERR_ARG;
  if (!fx || !fy || !fz) return fail(c, SG_ERR_ARG, "null field argument");
  SG_RET(check_ptrs(c, {u, v, w, X, Y, Z, U, V, W, FX, FY, FZ, NX, NY, NZ, AREA}));
  if (c->mixed) return run_step<float>(c, 7, u, v, w, X, Y, Z, U, V, W, FX, FY, FZ, NX, NY, NZ, AREA, fx, fy, fz);
  return run_step<double>(c, 7, u, v, w, X, Y, Z, U, V, W, FX, FY, FZ, NX, NY, NZ, AREA, fx, fy, fz);
}

int sg_update_pos(sg_ctx* c, double dt, double* X, double* Y, double* Z, const void* U, const void* V,
                  const void* W) {
  if (!c) return SG_ERR_ARG;
  SG_RET(check_ptrs(c, {X, Y, Z, U, V, W}));
  const bool host = c->cfg.mem == SG_MEM_HOST;
  const size_t pb = sizeof(double) * c->npts, lb = c->esz * c->npts;
  double *dX = X, *dY = Y, *dZ = Z;
  const void *dU = U, *dV = V, *dW = W;
  if (host) {
    SG_RET(h2d(c, c->s_X, X, pb));
    SG_RET(h2d(c, c->s_Y, Y, pb));
    SG_RET(h2d(c, c->s_Z, Z, pb));
    SG_RET(h2d(c, c->s_lag[0], U, lb));
    SG_RET(h2d(c, c->s_lag[1], V, lb));
    SG_RET(h2d(c, c->s_lag[2], W, lb));
    dX = c->s_X; dY = c->s_Y; dZ = c->s_Z;
    dU = c->s_lag[0]; dV = c->s_lag[1]; dW = c->s_lag[2];
  }
  const sg_config& f = c->cfg;
  cudaError_t e = c->mixed ? launch_update_pos<float>(f.ncap, c->d_caps, dt, f.lx, f.ly, f.lz, dX, dY, dZ,
                                                      (const float*)dU, (const float*)dV, (const float*)dW, c->st)
                           : launch_update_pos<double>(f.ncap, c->d_caps, dt, f.lx, f.ly, f.lz, dX, dY, dZ,
                                                       (const double*)dU, (const double*)dV, (const double*)dW, c->st);
  if (e != cudaSuccess) return cuda_fail(c, e, "update_pos");
  if (host) {
    SG_RET(d2h(c, X, dX, pb));
    SG_RET(d2h(c, Y, dY, pb));
    SG_RET(d2h(c, Z, dZ, pb));
  }
  return finish(c);
}

int sg_set_wall_collisions(sg_ctx* c, int in_step, double col, double betacol, double rad0, double rep) {
  if (!c) return SG_ERR_ARG;
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph first");
  if (!std::isfinite(col) || !std::isfinite(betacol) || !(rad0 > 0.0) || !std::isfinite(rad0) || !(rep > 0.0) ||
      !std::isfinite(rep))
    return fail(c, SG_ERR_ARG, "wall collision parameters must be finite, rad0 and rep positive");
  c->wall = sg::WallParams{col, betacol, rad0, rep, c->cfg.lx / c->cfg.itot, c->cfg.ly / c->cfg.jtot};
  c->wall_set = true;
  c->wall_in_step = in_step != 0;
  return SG_OK;
}

int sg_collisions(sg_ctx* c, const double* Z, const void* AREA, void* FZ) {
  if (!c) return SG_ERR_ARG;
  if (!c->wall_set) return fail(c, SG_ERR_STATE, "wall collision parameters not set (sg_set_wall_collisions)");
  SG_RET(check_ptrs(c, {Z, AREA, FZ}));
  const bool host = c->cfg.mem == SG_MEM_HOST;
  const size_t pb = sizeof(double) * c->npts, lb = c->esz * c->npts;
  const double* dZ = Z;
  const void* dA = AREA;
  void* dF = FZ;
  if (host) {
    SG_RET(h2d(c, c->s_Z, Z, pb));
    SG_RET(h2d(c, c->s_lag[9], AREA, lb));
    SG_RET(h2d(c, c->s_lag[5], FZ, lb));
    dZ = c->s_Z; dA = c->s_lag[9]; dF = c->s_lag[5];
  }
  cudaError_t e = c->mixed ? launch_collisions<float>(c->npts, c->wall, dZ, (const float*)dA, (float*)dF, nullptr,
                                                      c->grid.dvi, c->st)
                           : launch_collisions<double>(c->npts, c->wall, dZ, (const double*)dA, (double*)dF, nullptr,
                                                       c->grid.dvi, c->st);
  if (e != cudaSuccess) return cuda_fail(c, e, "collisions");
  if (host) SG_RET(d2h(c, FZ, dF, lb));
  return finish(c);
}

int sg_set_indicator_params(sg_ctx* c, double visc0, double lambda, double thetainc, double ta, double rep) {
  if (!c) return SG_ERR_ARG;
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph first");
  SG_RET(indicator_setup(c, visc0, lambda, thetainc, ta, rep));
  SG_TRY(cudaDeviceSynchronize(), "indicator setup");
  return SG_OK;
}

int sg_indicator(sg_ctx* c, const double* X, const double* Y, const double* Z, const void* NX, const void* NY,
                 const void* NZ, const void* AREA, void* indic, void* visc, void* fy, void* fz) {
  if (!c) return SG_ERR_ARG;
  if (!c->ind.ready) return fail(c, SG_ERR_STATE, "indicator parameters not set (sg_set_indicator_params)");
  if (!indic) return fail(c, SG_ERR_ARG, "null indicator field");
  SG_RET(check_ptrs(c, {X, Y, Z, NX, NY, NZ, AREA}));
  const bool host = c->cfg.mem == SG_MEM_HOST;
  const size_t pb = sizeof(double) * c->npts, lb = c->esz * c->npts, fb = c->esz * c->nfield;
  const double *dX = X, *dY = Y, *dZ = Z;
  const void *dN[3] = {NX, NY, NZ}, *dA = AREA;
  void *dI = indic, *dV = visc, *dFy = fy, *dFz = fz;
  if (host) {
    SG_RET(h2d(c, c->s_X, X, pb));
    SG_RET(h2d(c, c->s_Y, Y, pb));
    SG_RET(h2d(c, c->s_Z, Z, pb));
    for (int q = 0; q < 3; ++q) {
      SG_RET(h2d(c, c->s_lag[6 + q], dN[q], lb));
      dN[q] = c->s_lag[6 + q];
    }
    SG_RET(h2d(c, c->s_lag[9], AREA, lb));
    dX = c->s_X; dY = c->s_Y; dZ = c->s_Z; dA = c->s_lag[9];
    dI = c->s_f[0];
    dV = visc ? c->s_f[1] : nullptr;
    if (fy) SG_RET(h2d(c, c->s_u, fy, fb));
    if (fz) SG_RET(h2d(c, c->s_v, fz, fb));
    dFy = fy ? c->s_u : nullptr;
    dFz = fz ? c->s_v : nullptr;
  }
  c->launches = 0;
  if (c->mixed)
    SG_RET(indicator_run<float>(c, dX, dY, dZ, (const float*)dN[0], (const float*)dN[1], (const float*)dN[2],
                                (const float*)dA, (float*)dI, (float*)dV, (float*)dFy, (float*)dFz));
  else
    SG_RET(indicator_run<double>(c, dX, dY, dZ, (const double*)dN[0], (const double*)dN[1], (const double*)dN[2],
                                 (const double*)dA, (double*)dI, (double*)dV, (double*)dFy, (double*)dFz));
  if (host) {
    SG_RET(d2h(c, indic, dI, fb));
    if (visc) SG_RET(d2h(c, visc, dV, fb));
    if (fy) SG_RET(d2h(c, fy, dFy, fb));
    if (fz) SG_RET(d2h(c, fz, dFz, fb));
  }
  return finish(c);
}

int sg_set_flow_params(sg_ctx* c, double rep, double vb2, double vt2) {
  if (!c) return SG_ERR_ARG;
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph first");
  SG_RET(flow_setup(c, rep, vb2, vt2));
  SG_TRY(cudaDeviceSynchronize(), "flow setup");
  return SG_OK;
}

int sg_flow_step(sg_ctx* c, double dt, const double* uo, const double* vo, const double* wo, const double* uoo,
                 const double* voo, const double* woo, double* p, const double* fx, const double* fy,
                 const double* fz, double* u, double* v, double* w) {
  if (!c) return SG_ERR_ARG;
  if (!c->flow.ready) return fail(c, SG_ERR_STATE, "flow parameters not set (sg_set_flow_params)");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(c, SG_ERR_ARG, "dt must be positive and finite");
  SG_RET(check_ptrs(c, {uo, vo, wo, uoo, voo, woo, p, fx, fy, fz, u, v, w}));
  const bool host = c->cfg.mem == SG_MEM_HOST;
  const size_t fb = sizeof(double) * c->nfield;
  const double* in[10] = {uo, vo, wo, uoo, voo, woo, p, fx, fy, fz};
  double* out[3] = {u, v, w};
  const double* din[10];
  double* dout[3];
  for (int q = 0; q < 10; ++q) din[q] = in[q];
  for (int q = 0; q < 3; ++q) dout[q] = out[q];
  if (host) {
    for (int q = 0; q < 10; ++q) {
      SG_RET(h2d(c, c->flow.stage[q], in[q], fb));
      din[q] = (const double*)c->flow.stage[q];
    }
    for (int q = 0; q < 3; ++q) dout[q] = (double*)c->flow.stage[10 + q];
  }
  c->launches = 0;
  SG_RET(flow_run(c, dt, din[0], din[1], din[2], din[3], din[4], din[5], (double*)din[6], din[7], din[8], din[9],
                  dout[0], dout[1], dout[2]));
  if (host) {
    SG_RET(d2h(c, p, din[6], fb));
    for (int q = 0; q < 3; ++q) SG_RET(d2h(c, out[q], dout[q], fb));
  }
  return finish(c);
}

int sg_overlap_lid(sg_ctx* c, int nf, int nr, const double* u, const double* v, const double* w, const double* p,
                   const double* indic, double* ub, double* vb, double* wb, double* pb, double* indb) {
  if (!c) return SG_ERR_ARG;
  const sg_config& g = c->cfg;
  if (nr < 2) return fail(c, SG_ERR_ARG, "overlap mesh: nr (main cell / fine cell) must be at least 2");
  if (nf < 0 || nf + 1 > g.ktot + 1) return fail(c, SG_ERR_ARG, "overlap mesh: need 0 <= nf and nf + 1 <= kmax + 1");
  SG_RET(check_ptrs(c, {u, v, w, p, indic, ub, vb, wb, pb, indb}));
  const long ldi = g.itot + 2, plane = ldi * (g.jtot + 2);
  const int ni = g.itot * nr + 2, nj = g.jtot * nr + 2;
  const size_t nlid = (size_t)ni * nj;
  LidArgs a{};
  a.ldi = ldi;
  a.plane = plane;
  a.ni = ni;
  a.nj = nj;
  // param.f90:25-26, 40-41: dx = 1/(itot/lx), dxc = 1/(itotc/lx), itotc = itot nr
  a.dx = 1.0 / ((double)g.itot / g.lx);
  a.dy = 1.0 / ((double)g.jtot / g.ly);
  a.dxc = 1.0 / ((double)(g.itot * nr) / g.lx);
  a.dyc = 1.0 / ((double)(g.jtot * nr) / g.ly);
  a.offx = (0.5 * (1.0 - (1.0 / nr))) * a.dx;
  a.offy = (0.5 * (1.0 - (1.0 / nr))) * a.dy;
  const double* in[5] = {u, v, w, p, indic};
  double* out[5] = {ub, vb, wb, pb, indb};
  const bool host = g.mem == SG_MEM_HOST;
  if (host) {
    // only planes nf and nf + 1 are read: those, and the lid, are staged on the device
    if (!c->ovl_in) SG_TRY(dalloc(c, c->ovl_in, sizeof(double) * 10 * plane), "alloc");
    if (c->ovl_out_n < nlid) {
      SG_TRY(dalloc(c, c->ovl_out, sizeof(double) * 5 * nlid), "alloc");
      c->ovl_out_n = nlid;
    }
    for (int f = 0; f < 5; ++f) {
      SG_RET(h2d(c, c->ovl_in + 2 * f * plane, in[f] + (long)nf * plane, sizeof(double) * 2 * plane));
      a.f[f] = c->ovl_in + 2 * f * plane;
      a.o[f] = c->ovl_out + f * nlid;
    }
  } else {
    for (int f = 0; f < 5; ++f) {
      a.f[f] = in[f] + (long)nf * plane;
      a.o[f] = out[f];
    }
  }
  c->launches = 1;
  SG_TRY(launch_overlap_lid(a, c->st), "overlap lid");
  if (host)
    for (int f = 0; f < 5; ++f) SG_RET(d2h(c, out[f], a.o[f], sizeof(double) * nlid));
  return finish(c);
}

int sg_surf_vol(sg_ctx* c, const double* X, const double* Y, const double* Z, const void* NX, const void* NY,
                const void* NZ, const void* AREA, const double* exy1_prev, double* out) {
  if (!c) return SG_ERR_ARG;
  if (!out) return fail(c, SG_ERR_ARG, "null output");
  SG_RET(check_ptrs(c, {X, Y, Z, NX, NY, NZ, AREA}));
  const bool host = c->cfg.mem == SG_MEM_HOST;
  const size_t pb = sizeof(double) * c->npts, lb = c->esz * c->npts;
  const double *dX = X, *dY = Y, *dZ = Z, *dexy = exy1_prev;
  const void *dNX = NX, *dNY = NY, *dNZ = NZ, *dA = AREA;
  double* dout = out;
  if (host) {
    SG_RET(h2d(c, c->s_X, X, pb));
    SG_RET(h2d(c, c->s_Y, Y, pb));
    SG_RET(h2d(c, c->s_Z, Z, pb));
    SG_RET(h2d(c, c->s_lag[6], NX, lb));
    SG_RET(h2d(c, c->s_lag[7], NY, lb));
    SG_RET(h2d(c, c->s_lag[8], NZ, lb));
    SG_RET(h2d(c, c->s_lag[9], AREA, lb));
    if (exy1_prev) SG_RET(h2d(c, c->s_exy, exy1_prev, sizeof(double) * c->cfg.ncap));
    dX = c->s_X; dY = c->s_Y; dZ = c->s_Z;
    dNX = c->s_lag[6]; dNY = c->s_lag[7]; dNZ = c->s_lag[8]; dA = c->s_lag[9];
    dexy = exy1_prev ? c->s_exy : nullptr;
    dout = c->s_out;
  }
  cudaError_t e = c->mixed ? launch_surf_vol<float>(c->cfg.ncap, c->d_caps, dX, dY, dZ, (const float*)dNX,
                                                    (const float*)dNY, (const float*)dNZ, (const float*)dA, dexy,
                                                    dout, c->st)
                           : launch_surf_vol<double>(c->cfg.ncap, c->d_caps, dX, dY, dZ, (const double*)dNX,
                                                     (const double*)dNY, (const double*)dNZ, (const double*)dA, dexy,
                                                     dout, c->st);
  if (e != cudaSuccess) return cuda_fail(c, e, "surf_vol");
  if (host) SG_RET(d2h(c, out, c->s_out, sizeof(double) * 7 * c->cfg.ncap));
  return finish(c);
}

int sg_gauss(int nlat, double* theta, double* weights) {
  if (nlat < 1 || !theta || !weights) return SG_ERR_ARG;
  host_gauss(nlat, theta, weights);
  return SG_OK;
}

int sg_legendre(double theta, int mm, int nn, double* P, double* dP, double* d2P) {
  if (mm < 1 || nn < 1) return SG_ERR_ARG;
  host_legendre(theta, mm, nn, P, dP, d2P);
  return SG_OK;
}

int sg_last_launch_count(const sg_ctx* c) { return c ? c->launches : 0; }

int sg_set_profiling(sg_ctx* c, int on) {
  if (!c) return SG_ERR_ARG;
  if (on && !c->ev[0]) {
    for (int k = 0; k <= sg_ctx::kMarkStages; ++k) SG_TRY(cudaEventCreate(&c->ev[k]), "cudaEventCreate");
    for (int e = 0; e < 2; ++e)
      for (int k = 0; k < sg_ctx::kMaxContract; ++k) SG_TRY(cudaEventCreate(&c->ev_con[e][k]), "cudaEventCreate");
  }
  c->profiling = on != 0;
  return SG_OK;
}

int sg_set_fused_force(sg_ctx* c, int on) {
  if (!c) return SG_ERR_ARG;
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph first");
  if (!c->mixed && on) return fail(c, SG_ERR_CONFIG, "the fused force stage is the mixed-precision path's");
  c->fused = on != 0;
  return SG_OK;
}

int sg_get_fused_force(sg_ctx* c) { return c ? (c->fused ? 1 : 0) : -1; }

int sg_set_capsule_bending(sg_ctx* c, const double* eb) {
  if (!c) return SG_ERR_ARG;
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph first");
  bool any = false;
  for (int k = 0; k < c->cfg.ncap; ++k) {
    const double v = eb ? eb[k] : 0.0;
    if (!std::isfinite(v)) return fail(c, SG_ERR_ARG, "bending modulus must be finite");
    any = any || v != 0.0;
  }
  SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
  if (any) SG_RET(bend_setup(c));
  for (int k = 0; k < c->cfg.ncap; ++k) c->h_caps[k].eb = eb ? eb[k] : 0.0;
  c->bend = any;
  assign_terms(c, c->h_probs);
  SG_TRY(cudaMemcpy(c->d_probs, c->h_probs.data(), sizeof(LegProblem) * c->h_probs.size(), cudaMemcpyHostToDevice),
         "problems");
  SG_TRY(cudaMemcpy(c->d_caps, c->h_caps.data(), sizeof(CapInfo) * c->h_caps.size(), cudaMemcpyHostToDevice),
         "upload");
  return SG_OK;
}

int sg_set_tile_shape(sg_ctx* c, int shape) {
  if (!c) return SG_ERR_ARG;
  if (shape < -1 || shape >= kNumTileShapes) return fail(c, SG_ERR_ARG, "tile shape out of range");
  if (shape >= 0 && !c->mixed) {
    const TileShape& t = kTileShapes[shape];
    if (t.TX * t.TY * t.TZ > 1024) return fail(c, SG_ERR_ARG, "FP64 spreading takes tiles of at most 1024 cells");
  }
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph before changing the tile shape");
  IBGrid g{};
  const sg_config& cfg = c->cfg;
  if (!make_ib_grid(cfg.itot, cfg.jtot, cfg.ktot, cfg.lx, cfg.ly, cfg.lz, g, shape,
                    c->mixed ? kAllTileShapes : kFp64TileShapes) ||
      g.ntiles > c->max_tiles)
    return fail(c, SG_ERR_ARG, "tile shape not valid for this grid");
  c->grid = g;
  return SG_OK;
}

int sg_set_legendre_terms(sg_ctx* c, int terms) {
  if (!c) return SG_ERR_ARG;
  if (terms != 0 && terms != 3 && terms != 6) return fail(c, SG_ERR_ARG, "terms must be 0 (automatic), 3 or 6");
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph first");
  if (!c->mixed) return fail(c, SG_ERR_CONFIG, "the split modes belong to the mixed-precision path");
  c->leg_terms = terms;
  if (c->h_probs.empty()) return SG_OK;
  assign_terms(c, c->h_probs);
  SG_TRY(cudaStreamSynchronize(c->st), "sync");
  SG_TRY(cudaMemcpy(c->d_probs, c->h_probs.data(), sizeof(LegProblem) * c->h_probs.size(), cudaMemcpyHostToDevice),
         "problems");
  return SG_OK;
}

int sg_get_legendre_terms(sg_ctx* c, int degree) {
  if (!c || degree < 0) return -1;
  return terms_for(c, degree);
}

int sg_set_legendre_tile_rows(sg_ctx* c, int rows) {
  if (!c) return SG_ERR_ARG;
  if (rows != 64 && rows != 128) return fail(c, SG_ERR_ARG, "tile rows must be 64 or 128");
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph first");
  if (!c->mixed) return fail(c, SG_ERR_CONFIG, "the tensor-core path is the mixed-precision path");
  const int t = rows == 64 ? 1 : 0;
  for (int f = 0; f < 3; ++f) {
    c->tmF[f] = rows;
    c->nlwF[f] = c->nlwT[t][f];
    c->d_lwF[f] = c->d_lwT[t][f];
  }
  return SG_OK;
}

int sg_get_legendre_tile_rows(sg_ctx* c) { return c ? c->tmF[0] : -1; }

int sg_set_tensor_cores(sg_ctx* c, int on) {
  if (!c) return SG_ERR_ARG;
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph first");
  if (on && !c->mixed) return fail(c, SG_ERR_CONFIG, "the tensor-core path is the mixed-precision path");
  c->leg_tc = on != 0 && c->nlwF[0] > 0;
  return SG_OK;
}

int sg_set_point_split(sg_ctx* c, int split) {
  if (!c) return SG_ERR_ARG;
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph before changing the schedule");
  return set_point_split(c, split);
}

int sg_get_point_split(const sg_ctx* c) { return c ? c->point_split : 0; }

int sg_get_tile_shape(const sg_ctx* c, int* shape, int* tx, int* ty, int* tz) {
  if (!c) return SG_ERR_ARG;
  if (shape) *shape = c->grid.shape;
  if (tx) *tx = c->grid.TX;
  if (ty) *ty = c->grid.TY;
  if (tz) *tz = c->grid.TZ;
  return SG_OK;
}

int sg_autotune(sg_ctx* c, const void* u, const void* v, const void* w, const double* X, const double* Y,
                const double* Z, void* U, void* V, void* W, void* FX, void* FY, void* FZ, void* NX, void* NY,
                void* NZ, void* AREA, void* fx, void* fy, void* fz, int reps, int* best_shape, float* best_ms) {
  if (!c) return SG_ERR_ARG;
  if (reps < 1) return fail(c, SG_ERR_ARG, "reps must be >= 1");
  if (c->graph) return fail(c, SG_ERR_STATE, "release the captured graph before tuning");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  SG_TRY(cudaEventCreate(&e0), "cudaEventCreate");
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(c, SG_ERR_CUDA, "cudaEventCreate");
  }
  const int async = c->cfg.async;
  c->cfg.async = 1;  // queue the repetitions back to back
  int rc = SG_OK;
  auto time_step = [&](float* ms) -> int {
    int r = sg_step(c, u, v, w, X, Y, Z, U, V, W, FX, FY, FZ, NX, NY, NZ, AREA, fx, fy, fz);  // warm-up
    if (r == SG_OK && cudaEventRecord(e0, c->st) != cudaSuccess) r = fail(c, SG_ERR_CUDA, "event");
    for (int k = 0; k < reps && r == SG_OK; ++k)
      r = sg_step(c, u, v, w, X, Y, Z, U, V, W, FX, FY, FZ, NX, NY, NZ, AREA, fx, fy, fz);
    if (r == SG_OK && (cudaEventRecord(e1, c->st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                       cudaEventElapsedTime(ms, e0, e1) != cudaSuccess))
      r = fail(c, SG_ERR_CUDA, "autotune timing");
    *ms /= (float)reps;
    return r;
  };
  // 1) spreading tile shape
  int best = -1;
  float bms = 0.f;
  for (int sh = 0; sh < kNumTileShapes && rc == SG_OK; ++sh) {
    if (sg_set_tile_shape(c, sh) != SG_OK) continue;  // not valid for this precision or grid
    float ms = 0.f;
    rc = time_step(&ms);
    if (rc == SG_OK && (best < 0 || ms < bms)) {
      best = sh;
      bms = ms;
    }
  }
  if (rc == SG_OK && best >= 0) rc = sg_set_tile_shape(c, best);
  // 2) work items per capsule of the persistent pointwise kernels
  int bsplit = c->point_split;
  for (int sp = 1; sp <= kMaxPointSplit && rc == SG_OK && best >= 0; sp *= 2) {
    rc = set_point_split(c, sp);
    float ms = 0.f;
    if (rc == SG_OK) rc = time_step(&ms);
    if (rc == SG_OK && ms < bms) {
      bsplit = sp;
      bms = ms;
    }
  }
  if (rc == SG_OK && best >= 0) rc = set_point_split(c, bsplit);
  // 3) tile rows of the tensor-core Legendre launches (mixed path)
  if (rc == SG_OK && best >= 0 && c->leg_tc) {
    int brows = c->tmF[0];
    for (int rows : {128, 64}) {
      if (rc != SG_OK) break;
      rc = sg_set_legendre_tile_rows(c, rows);
      float ms = 0.f;
      if (rc == SG_OK) rc = time_step(&ms);
      if (rc == SG_OK && ms < bms) {
        brows = rows;
        bms = ms;
      }
    }
    if (rc == SG_OK) rc = sg_set_legendre_tile_rows(c, brows);
  }
  c->cfg.async = async;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != SG_OK) return rc;
  if (best < 0) return fail(c, SG_ERR_STATE, "no tile shape is valid for this grid");
  if (best_shape) *best_shape = best;
  if (best_ms) *best_ms = bms;
  return SG_OK;
}

int sg_graph_capture(sg_ctx* c, const void* u, const void* v, const void* w, const double* X, const double* Y,
                     const double* Z, void* U, void* V, void* W, void* FX, void* FY, void* FZ, void* NX, void* NY,
                     void* NZ, void* AREA, void* fx, void* fy, void* fz) {
  if (!c) return SG_ERR_ARG;
  if (c->cfg.mem != SG_MEM_DEVICE) return fail(c, SG_ERR_STATE, "graph capture needs device memory mode");
  if (c->graph) return fail(c, SG_ERR_STATE, "a graph is already captured");
  if (!c->st) return fail(c, SG_ERR_STATE, "no stream");
  SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
  SG_TRY(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  c->capturing = true;
  const int rc = sg_step(c, u, v, w, X, Y, Z, U, V, W, FX, FY, FZ, NX, NY, NZ, AREA, fx, fy, fz);
  c->capturing = false;
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->st, &g);
  if (rc != SG_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
  cudaGraphExec_t x = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&x, g, 0);
  if (ei != cudaSuccess) {
    cudaGraphDestroy(g);
    return cuda_fail(c, ei, "cudaGraphInstantiate");
  }
  c->graph = g;
  c->graph_exec = x;
  c->graph_launches = c->launches;
  return SG_OK;
}

int sg_graph_launch(sg_ctx* c) {
  if (!c) return SG_ERR_ARG;
  if (!c->graph_exec) return fail(c, SG_ERR_STATE, "no captured graph");
  SG_TRY(cudaGraphLaunch(c->graph_exec, c->st), "cudaGraphLaunch");
  c->launches = c->graph_launches;
  return finish(c);
}

int sg_graph_release(sg_ctx* c) {
  if (!c) return SG_ERR_ARG;
  if (c->graph_exec) SG_TRY(cudaStreamSynchronize(c->st), "synchronize");
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  if (c->graph) cudaGraphDestroy(c->graph);
  c->graph_exec = nullptr;
  c->graph = nullptr;
  return SG_OK;
}

int sg_stage_times(sg_ctx* c, float* ms, int n) {
  if (!c || !ms) return SG_ERR_ARG;
  if (!c->profiling) return fail(c, SG_ERR_STATE, "profiling is off");
  SG_TRY(cudaEventSynchronize(c->ev[sg_ctx::kMarkStages]), "event sync");
  for (int k = 0; k < n && k < sg_ctx::kMarkStages; ++k) {
    float t = 0.f;
    if (c->ev_used[k]) SG_TRY(cudaEventElapsedTime(&t, c->ev[k], c->ev[k + 1]), "elapsed");
    ms[k] = t;
  }
  if (n > SG_STAGE_CONTRACT) {
    float sum = 0.f;
    for (int k = 0; k < c->ncon && c->ev_used[SG_STAGE_MEMBRANE]; ++k) {
      float t = 0.f;
      SG_TRY(cudaEventElapsedTime(&t, c->ev_con[0][k], c->ev_con[1][k]), "elapsed");
      sum += t;
    }
    ms[SG_STAGE_CONTRACT] = sum;
  }
  return SG_OK;
}

int sg_contraction_work(const sg_ctx* c, double* out) {
  if (!c || !out) return SG_ERR_ARG;
  out[0] = out[1] = out[2] = 0.0;
  if (c->cfg.ncap == 0) return SG_OK;
  // algorithmic multiply-adds of one problem: rows x sum over m of the
  // products that are not zero by the triangular structure (synthesis: terms
  // n >= m of the K = N coefficients; analysis: outputs n >= m of J = N)
  auto useful = [](const LegProblem& p) {
    double s = 0;
    for (int m = 0; m < p.M; ++m) {
      const int k = p.tri ? std::max(p.K - m, 0) : p.K;
      const int j = (p.kind == 1 || p.kind == 3) ? std::max(p.J - m, 0) : p.J;
      s += (double)j * k;
    }
    return 2.0 * p.Q * s;
  };
  if (c->leg_tc) {
    for (int f = 0; f < 3; ++f) {
      const int tm = c->tmF[f];
      for (int r : c->leg_roots[f]) {
        const LegProblem& p = c->h_probs[r];
        const int chain[3] = {r, p.next[0], p.next[0] >= 0 ? p.next[1] : -1};
        for (int q : chain) {
          if (q < 0) continue;
          const LegProblem& pq = c->h_probs[q];
          out[0] += useful(pq);
          const double tiles = (double)((pq.Q + tm - 1) / tm);
          double mk = 0;  // issued K per m (the kernel skips whole K steps below m in a synthesis)
          for (int m = 0; m < pq.M; ++m) mk += pq.Kp - (pq.tri ? 16 * (m >> 4) : 0);
          out[1] += 2.0 * tiles * tm * pq.Jp * mk * pq.terms;
        }
      }
    }
    out[2] = 3;
  } else {
    // CUDA-core path: the six stages over every problem of the context
    // (the tensor-core split problems appended after them are not launched)
    const size_t nplain = c->h_probs.size() - (c->mixed ? 2 * c->groups.size() : 0);
    for (size_t i = 0; i < nplain; ++i) out[0] += useful(c->h_probs[i]);
    out[2] = 6;
  }
  return SG_OK;
}

}  // extern "C"
