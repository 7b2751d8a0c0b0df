/* Oracle part 1: 1D tables, simplex interpolation, reference-element levels,
 * per-panel refined levels and the level-resolved direct SLP/DLP sums.
 * TEST INFRASTRUCTURE ONLY (see orc_common.h). */
#include "orc_common.h"
#include <map>
#include <mutex>
#ifdef __AVX2__
#include <immintrin.h>
#endif
#include "vr_table.h"
#include <algorithm>
#include <cfloat>
#include <stdexcept>

namespace orc {

int lu_factor(int n, double* A, int* piv) {
  for (int k = 0; k < n; ++k) {
    int p = k;
    double pm = std::fabs(A[k + (size_t)k * n]);
    for (int i = k + 1; i < n; ++i) {
      double v = std::fabs(A[i + (size_t)k * n]);
      if (v > pm) { pm = v; p = i; }
    }
    piv[k] = p;
    if (pm == 0.0) return k + 1;
    if (p != k)
      for (int j = 0; j < n; ++j) std::swap(A[k + (size_t)j * n], A[p + (size_t)j * n]);
    double inv = 1.0 / A[k + (size_t)k * n];
    for (int i = k + 1; i < n; ++i) A[i + (size_t)k * n] *= inv;
    for (int j = k + 1; j < n; ++j) {
      double akj = A[k + (size_t)j * n];
      if (akj == 0.0) continue;
      double* cj = A + (size_t)j * n;
      const double* ck = A + (size_t)k * n;
      for (int i = k + 1; i < n; ++i) cj[i] -= ck[i] * akj;
    }
  }
  return 0;
}

void lu_solve(int n, const double* LU, const int* piv, double* B, int nrhs) {
  for (int r = 0; r < nrhs; ++r) {
    double* b = B + (size_t)r * n;
    for (int k = 0; k < n; ++k)
      if (piv[k] != k) std::swap(b[k], b[piv[k]]);
    for (int k = 0; k < n; ++k) {
      double bk = b[k];
      const double* ck = LU + (size_t)k * n;
      for (int i = k + 1; i < n; ++i) b[i] -= ck[i] * bk;
    }
    for (int k = n - 1; k >= 0; --k) {
      b[k] /= LU[k + (size_t)k * n];
      double bk = b[k];
      const double* ck = LU + (size_t)k * n;
      for (int i = 0; i < k; ++i) b[i] -= ck[i] * bk;
    }
  }
}

/* utils/gauss.m:1-37: Legendre-Gauss nodes by the (damped) Newton iteration
 * of lgwt.m with its initial guess, weights, and Fornberg's differentiation
 * matrix.  Nodes are returned ascending (x = y(end:-1:1)); the weights keep
 * the iteration's order, as gauss.m does (they are symmetric). */
void gauss(int N, double* x, double* w, double* D) {
  if (N == 1) {
    x[0] = 0.0; w[0] = 2.0;
    if (D) D[0] = 0.0;
    return;
  }
  int n = N - 1, N1 = n + 1, N2 = n + 2;
  std::vector<double> y(N1), y0(N1, 2.0), L((size_t)N1 * N2), Lp(N1);
  for (int k = 0; k <= n; ++k) {
    double xu = -1.0 + 2.0 * k / (double)n;
    y[k] = std::cos((2.0 * k + 1.0) * PI / (2.0 * n + 2.0)) +
           (0.27 / N1) * std::sin(PI * xu * n / N2);
  }
  const double eps = DBL_EPSILON;
  for (int it = 0; it < 1000; ++it) {
    double md = 0.0;
    for (int k = 0; k < N1; ++k) md = std::max(md, std::fabs(y[k] - y0[k]));
    if (!(md > eps)) break;
    for (int i = 0; i < N1; ++i) {
      L[i] = 1.0;
      L[i + (size_t)N1] = y[i];
    }
    for (int k = 2; k <= N1; ++k)
      for (int i = 0; i < N1; ++i)
        L[i + (size_t)k * N1] = ((2.0 * k - 1.0) * y[i] * L[i + (size_t)(k - 1) * N1] -
                                 (k - 1.0) * L[i + (size_t)(k - 2) * N1]) / k;
    for (int i = 0; i < N1; ++i)
      Lp[i] = N2 * (L[i + (size_t)(N1 - 1) * N1] - y[i] * L[i + (size_t)(N2 - 1) * N1]) /
              (1.0 - y[i] * y[i]);
    for (int i = 0; i < N1; ++i) {
      y0[i] = y[i];
      y[i] = y0[i] - L[i + (size_t)(N2 - 1) * N1] / Lp[i];
    }
  }
  for (int i = 0; i < N1; ++i) {
    x[i] = y[N1 - 1 - i];
    w[i] = 2.0 / ((1.0 - y[i] * y[i]) * Lp[i] * Lp[i]) * ((double)N2 / N1) * ((double)N2 / N1);
  }
  if (D) {
    std::vector<double> a(N);
    for (int k = 0; k < N; ++k) {
      double p = 1.0;
      for (int i = 0; i < N; ++i)
        if (i != k) p *= (x[k] - x[i]);
      a[k] = p;
    }
    for (int k = 0; k < N; ++k) {
      double s = 0.0;
      for (int i = 0; i < N; ++i) {
        if (i == k) continue;
        D[i + (size_t)k * N] = (a[i] / a[k]) / (x[i] - x[k]);
        s += 1.0 / (x[k] - x[i]);
      }
      D[k + (size_t)k * N] = s;
    }
  }
}

void bary_weights(int n, const double* x, double* wb) {
  for (int j = 0; j < n; ++j) {
    double p = 1.0;
    for (int k = 0; k < n; ++k)
      if (k != j) p *= (x[j] - x[k]);
    wb[j] = 1.0 / p;
  }
}

void legendre_vals2coefs(int n, const double* x, const double* w, double* U) {
  for (int i = 0; i < n; ++i) {
    double p0 = 1.0, p1 = x[i];
    for (int k = 0; k < n; ++k) {
      double pk;
      if (k == 0) pk = 1.0;
      else if (k == 1) pk = x[i];
      else {
        pk = ((2.0 * k - 1.0) * x[i] * p1 - (k - 1.0) * p0) / k;
        p0 = p1; p1 = pk;
      }
      U[k + (size_t)i * n] = (2.0 * k + 1.0) / 2.0 * w[i] * pk;
    }
  }
}

int npols_of(int korder) { return (korder + 1) * (korder + 2) / 2; }

/* Orthogonal polynomials on the simplex in collapsed coordinates:
 * P_{a,b}(u,v) = L_a(2u+v-1, 1-v) * P_b^{(2a+1,0)}(2v-1), where
 * L_a(s,t) = t^a P_a(s/t) is the homogenised Legendre polynomial.  Ordered by
 * total degree a+b, then b.  Any basis of the degree-korder polynomials gives
 * the same interpolation matrix pols*umatr; this one is well conditioned. */
void koorn_pols(double u, double v, int korder, double* pols) {
  double s = 2.0 * u + v - 1.0, t = 1.0 - v, z = 2.0 * v - 1.0;
  double La[64];
  La[0] = 1.0;
  if (korder >= 1) La[1] = s;
  for (int a = 1; a < korder; ++a)
    La[a + 1] = ((2.0 * a + 1.0) * s * La[a] - a * t * t * La[a - 1]) / (a + 1.0);
  int idx = 0;
  for (int deg = 0; deg <= korder; ++deg) {
    for (int b = 0; b <= deg; ++b) {
      int a = deg - b;
      double alpha = 2.0 * a + 1.0;
      /* Jacobi P_b^{(alpha,0)}(z) */
      double p0 = 1.0, p1 = 0.5 * (alpha + 2.0) * z + 0.5 * alpha, pb;
      if (b == 0) pb = p0;
      else if (b == 1) pb = p1;
      else {
        for (int j = 1; j < b; ++j) {
          double jj = j + 1.0; /* computing P_{j+1} */
          double c1 = 2.0 * jj * (jj + alpha) * (2.0 * jj + alpha - 2.0);
          double c2 = (2.0 * jj + alpha - 1.0) * (alpha * alpha);
          double c3 = (2.0 * jj + alpha - 2.0) * (2.0 * jj + alpha - 1.0) * (2.0 * jj + alpha);
          double c4 = 2.0 * (jj + alpha - 1.0) * (jj - 1.0) * (2.0 * jj + alpha);
          double p2 = ((c2 + c3 * z) * p1 - c4 * p0) / c1;
          p0 = p1; p1 = p2;
        }
        pb = p1;
      }
      pols[idx++] = La[a] * pb;
    }
  }
}

void vr_nodes(int deg, double* uv, double* w) {
  if (deg < 0 || deg > QOL_VR_MAXDEG) throw std::runtime_error("VR degree out of table");
  int o = qol_vr_offset[deg], n = qol_vr_offset[deg + 1] - o;
  for (int i = 0; i < n; ++i) {
    if (uv) { uv[2 * i] = qol_vr_uv[2 * (o + i)]; uv[2 * i + 1] = qol_vr_uv[2 * (o + i) + 1]; }
    if (w) w[i] = qol_vr_w[o + i];
  }
}

void koorn_umatr(int korder, double* umatr, double* vmatr) {
  int np = npols_of(korder);
  std::vector<double> uv(2 * np), V((size_t)np * np), p(np);
  vr_nodes(korder, uv.data(), nullptr);
  for (int i = 0; i < np; ++i) {
    koorn_pols(uv[2 * i], uv[2 * i + 1], korder, p.data());
    for (int k = 0; k < np; ++k) V[i + (size_t)k * np] = p[k];
  }
  if (vmatr) std::copy(V.begin(), V.end(), vmatr);
  std::vector<int> piv(np);
  std::vector<double> I((size_t)np * np, 0.0);
  for (int i = 0; i < np; ++i) I[i + (size_t)i * np] = 1.0;
  if (lu_factor(np, V.data(), piv.data())) throw std::runtime_error("singular VR vandermonde");
  lu_solve(np, V.data(), piv.data(), I.data(), np);
  std::copy(I.begin(), I.end(), umatr);
}

void interp_matrix(int korder, int n, const double* uv, double* M) {
  int np = npols_of(korder);
  std::vector<double> um((size_t)np * np), p(np);
  koorn_umatr(korder, um.data(), nullptr);
  for (int i = 0; i < n; ++i) {
    koorn_pols(uv[2 * i], uv[2 * i + 1], korder, p.data());
    for (int j = 0; j < np; ++j) {
      double s = 0.0;
      for (int k = 0; k < np; ++k) s += p[k] * um[k + (size_t)j * np];
      M[i + (size_t)j * n] = s;
    }
  }
}

/* cc_subidx_at (patch_refine_mod.f90:264-311): which of the 64 level-4
 * sub-triangles the cc level keeps (1-based). */
static const int CC_SUBIDX[39] = {1,  2,  3,  4,  7,  8,  9,  10, 11, 13, 14, 16, 17,
                                  27, 32, 33, 34, 35, 37, 40, 41, 42, 43, 44, 46, 47,
                                  48, 49, 50, 52, 53, 55, 58, 59, 60, 61, 62, 63, 64};
static const int CC_NSUB = 39;
static const double CC_EXTRA_SCALE = 0.625, CC_EXTRA_OFFSET = 0.4375;

/* ref_square_regroup (patch_refine_mod.f90:313-421) */
static void square_regroup(RefElem& R, int ilev, i8 n1, int korder, bool is_cc) {
  RefLevel& L = R.lev[ilev - 1];
  i8 nsub_old = L.nsub, npairable = nsub_old, ncell;
  if (is_cc) { npairable = nsub_old - 4; ncell = 8; }
  else ncell = (i8)1 << (ilev - 1);
  double side = 1.0 / (double)ncell;
  int qg = korder + 1;
  if (qg < 8) qg = korder + 3;
  double fac = 0.0;
  for (double wv : R.lev[0].wt) fac += wv;
  fac *= 2.0;
  std::vector<double> uv_old = L.uv, wt_old = L.wt;
  std::vector<i8> cellcnt((size_t)ncell * ncell, 0), singles;
  auto cell_of = [&](i8 q, i8& ic, i8& jc) {
    i8 i0 = (q - 1) * n1;
    double cu = 0.0, cv = 0.0;
    for (i8 i = 0; i < n1; ++i) cu += uv_old[2 * (i0 + i)];
    for (i8 i = 0; i < n1; ++i) cv += uv_old[2 * (i0 + i) + 1];
    cu /= (double)n1; cv /= (double)n1;
    ic = std::min(std::max((i8)(cu / side), (i8)0), ncell - 1);
    jc = std::min(std::max((i8)(cv / side), (i8)0), ncell - 1);
  };
  for (i8 q = 1; q <= npairable; ++q) {
    i8 ic, jc; cell_of(q, ic, jc);
    if (++cellcnt[ic + ncell * jc] > 2) throw std::runtime_error("square regroup: >2 in a cell");
  }
  for (i8 q = 1; q <= npairable; ++q) {
    i8 ic, jc; cell_of(q, ic, jc);
    if (cellcnt[ic + ncell * jc] == 1) singles.push_back(q);
  }
  for (i8 q = npairable + 1; q <= nsub_old; ++q) singles.push_back(q);
  i8 npair = 0;
  for (i8 c = 0; c < ncell * ncell; ++c) if (cellcnt[c] == 2) ++npair;
  i8 nsingle = (i8)singles.size();
  i8 n = npair * qg * qg + nsingle * n1, nsub = npair + nsingle;
  L.uv.assign(2 * n, 0.0); L.wt.assign(n, 0.0);
  L.suboff.assign(nsub + 1, 0); L.subtyp.assign(nsub, 0);
  for (i8 k = 0; k < npair; ++k) L.subtyp[k] = 1;
  std::vector<double> tq(qg), wq(qg);
  gauss(qg, tq.data(), wq.data(), nullptr);
  std::vector<double> u01(qg), w01(qg);
  for (int i = 0; i < qg; ++i) { u01[i] = 0.5 * (tq[i] + 1.0); w01[i] = 0.5 * wq[i]; }
  i8 row = 0, k = 0;
  for (i8 jc = 0; jc < ncell; ++jc)
    for (i8 ic = 0; ic < ncell; ++ic) {
      if (cellcnt[ic + ncell * jc] != 2) continue;
      for (int j = 0; j < qg; ++j)
        for (int i = 0; i < qg; ++i) {
          L.uv[2 * row] = ((double)ic + u01[i]) * side;
          L.uv[2 * row + 1] = ((double)jc + u01[j]) * side;
          L.wt[row] = w01[i] * w01[j] * side * side * fac;
          ++row;
        }
      ++k; L.suboff[k] = row;
    }
  for (i8 s = 0; s < nsingle; ++s) {
    i8 i0 = (singles[s] - 1) * n1;
    for (i8 j = 0; j < n1; ++j) {
      L.uv[2 * row] = uv_old[2 * (i0 + j)];
      L.uv[2 * row + 1] = uv_old[2 * (i0 + j) + 1];
      L.wt[row] = wt_old[i0 + j];
      ++row;
    }
    ++k; L.suboff[k] = row;
  }
  L.n = n; L.nsub = nsub;
}

/* 4-way split of a level's node set (patch_refine_mod.f90:216-240):
 * copies (u0,v0), (-u0,-v0), (u0,v0+2), (u0+2,v0) of uv0 = 2uv-1, then mapped
 * by ((x-1)/2+1)/2, each weight quartered. */
static void split4(const std::vector<double>& uvp, const std::vector<double>& wtp,
                   std::vector<double>& uv, std::vector<double>& wt) {
  i8 np = (i8)wtp.size();
  uv.assign(8 * np, 0.0); wt.assign(4 * np, 0.0);
  for (i8 i = 0; i < np; ++i) {
    double u0 = 2.0 * uvp[2 * i] - 1.0, v0 = 2.0 * uvp[2 * i + 1] - 1.0;
    double cu[4] = {u0, -u0, u0, u0 + 2.0}, cv[4] = {v0, -v0, v0 + 2.0, v0};
    for (int b = 0; b < 4; ++b) {
      uv[2 * (b * np + i)] = cu[b];
      uv[2 * (b * np + i) + 1] = cv[b];
      wt[b * np + i] = 0.25 * wtp[i];
    }
  }
  for (i8 i = 0; i < 4 * np; ++i) {
    uv[2 * i] = ((uv[2 * i] - 1.0) * 0.5 + 1.0) * 0.5;
    uv[2 * i + 1] = ((uv[2 * i + 1] - 1.0) * 0.5 + 1.0) * 0.5;
  }
}

void build_ref(int korder, int order, int nlevel, bool sqmode, RefElem& R) {
  int npols = npols_of(korder);
  R.korder = korder; R.npols = npols; R.order = order; R.nlevel = nlevel; R.sqmode = sqmode;
  R.lev.assign(nlevel, RefLevel());
  i8 n1 = (i8)order * (order + 1) / 2;
  for (int ilev = 1; ilev <= nlevel; ++ilev) {
    RefLevel& L = R.lev[ilev - 1];
    if (ilev == 1) {
      L.uv.assign(2 * n1, 0.0); L.wt.assign(n1, 0.0);
      vr_nodes(order - 1, L.uv.data(), L.wt.data());
      L.n = n1; L.nsub = 1;
    } else if (ilev == nlevel && nlevel == 4) {
      std::vector<double> uvt, wtt;
      split4(R.lev[ilev - 2].uv, R.lev[ilev - 2].wt, uvt, wtt);
      i8 ncc = CC_NSUB + 4;
      L.n = ncc * n1; L.nsub = ncc;
      L.uv.assign(2 * L.n, 0.0); L.wt.assign(L.n, 0.0);
      for (int q = 1; q <= CC_NSUB; ++q)
        for (i8 i = 1; i <= n1; ++i) {
          i8 isrc = (CC_SUBIDX[q - 1] - 1) * n1 + i - 1, idst = (q - 1) * n1 + i - 1;
          L.uv[2 * idst] = uvt[2 * isrc]; L.uv[2 * idst + 1] = uvt[2 * isrc + 1];
          L.wt[idst] = wtt[isrc];
        }
      const RefLevel& L2 = R.lev[1];
      for (int q = 1; q <= 4; ++q)
        for (i8 i = 1; i <= n1; ++i) {
          i8 isrc = (q - 1) * n1 + i - 1, idst = (CC_NSUB + q - 1) * n1 + i - 1;
          L.uv[2 * idst] = (L2.uv[2 * isrc] - 0.5) * CC_EXTRA_SCALE + CC_EXTRA_OFFSET;
          L.uv[2 * idst + 1] = (L2.uv[2 * isrc + 1] - 0.5) * CC_EXTRA_SCALE + CC_EXTRA_OFFSET;
          L.wt[idst] = CC_EXTRA_SCALE * CC_EXTRA_SCALE * L2.wt[isrc];
        }
    } else {
      split4(R.lev[ilev - 2].uv, R.lev[ilev - 2].wt, L.uv, L.wt);
      L.n = 4 * R.lev[ilev - 2].n; L.nsub = 4 * R.lev[ilev - 2].nsub;
    }
  }
  for (int ilev = 1; ilev <= nlevel; ++ilev) {
    RefLevel& L = R.lev[ilev - 1];
    if (sqmode && ilev >= 2) {
      square_regroup(R, ilev, n1, korder, ilev == nlevel && nlevel == 4);
    } else {
      L.suboff.assign(L.nsub + 1, 0); L.subtyp.assign(L.nsub, 0);
      for (i8 i = 0; i <= L.nsub; ++i) L.suboff[i] = i * n1;
    }
    L.interp.assign((size_t)L.n * npols, 0.0);
    interp_matrix(korder, (int)L.n, L.uv.data(), L.interp.data());
    L.interp_t.assign((size_t)L.n * npols, 0.0);
    for (i8 q = 0; q < L.n; ++q)
      for (int k = 0; k < npols; ++k) L.interp_t[(size_t)q * npols + k] = L.interp[q + (size_t)L.n * k];
  }
}

void build_panel_levels(const RefElem& R, const double* sx, const double* rts,
                        const double* rps, double dist, std::vector<PanelLevel>& lv) {
  int np = R.npols;
  double dist2 = dist * dist;
  std::vector<double> srcT((size_t)np * 9);
  for (int j = 0; j < np; ++j)
    for (int d = 0; d < 3; ++d) {
      srcT[j + (size_t)d * np] = sx[3 * j + d];
      srcT[j + (size_t)(3 + d) * np] = rts[3 * j + d];
      srcT[j + (size_t)(6 + d) * np] = rps[3 * j + d];
    }
  lv.assign(R.nlevel, PanelLevel());
  for (int il = 0; il < R.nlevel; ++il) {
    const RefLevel& L = R.lev[il];
    PanelLevel& P = lv[il];
    i8 n = L.n, nsub = L.nsub;
    P.n = n; P.nsub = nsub;
    P.sx.assign(3 * n, 0.0); P.snx.assign(3 * n, 0.0); P.sw.assign(n, 0.0);
    P.qpoint.assign(3 * nsub, 0.0); P.qradii2.assign(nsub, 0.0);
    std::vector<double> geo((size_t)n * 9, 0.0);
    for (int c = 0; c < 9; ++c)
      for (int k = 0; k < np; ++k) {
        double b = srcT[k + (size_t)c * np];
        const double* a = L.interp.data() + (size_t)k * n;
        double* g = geo.data() + (size_t)c * n;
        for (i8 i = 0; i < n; ++i) g[i] += a[i] * b;
      }
    for (i8 i = 0; i < n; ++i) {
      double g[9];
      for (int c = 0; c < 9; ++c) g[c] = geo[i + (size_t)c * n];
      P.sx[3 * i] = g[0]; P.sx[3 * i + 1] = g[1]; P.sx[3 * i + 2] = g[2];
      double nx = g[7] * g[5] - g[8] * g[4];
      double ny = g[8] * g[3] - g[6] * g[5];
      double nz = g[6] * g[4] - g[7] * g[3];
      double sp = std::sqrt(nx * nx + ny * ny + nz * nz);
      P.snx[3 * i] = nx / sp; P.snx[3 * i + 1] = ny / sp; P.snx[3 * i + 2] = nz / sp;
      P.sw[i] = sp * L.wt[i];
    }
    for (i8 k = 0; k < nsub; ++k) {
      i8 i0 = L.suboff[k], nk = L.suboff[k + 1] - i0;
      double swsum = 0.0, q[3] = {0, 0, 0};
      for (i8 i = i0; i < i0 + nk; ++i) swsum += P.sw[i];
      for (int d = 0; d < 3; ++d) {
        double s = 0.0;
        for (i8 i = i0; i < i0 + nk; ++i) s += P.sx[3 * i + d] * P.sw[i];
        q[d] = s / swsum;
      }
      double rmax2 = 0.0;
      for (i8 i = i0; i < i0 + nk; ++i) {
        double d2 = 0.0;
        for (int d = 0; d < 3; ++d) { double t = P.sx[3 * i + d] - q[d]; d2 += t * t; }
        rmax2 = std::max(rmax2, d2);
      }
      for (int d = 0; d < 3; ++d) P.qpoint[3 * k + d] = q[d];
      P.qradii2[k] = (L.subtyp[k] == 1) ? dist2 * std::max(rmax2, 0.5 * swsum)
                                         : dist2 * std::max(rmax2, swsum);
    }
  }
}

int g_orc_simd = 0;

#ifdef __AVX2__
/* isimd = 256: four targets a lane group, the scalar formula's operations in
 * the same order (separate multiplies and adds, IEEE sqrt and division), so
 * the same bits */
static void sdlpmat_avx2(i8 m, const double* tx, i8 n, const double* sx, const double* snx, const double* sw,
                         double* A, double* B) {
  const double pi4inv = 1.0 / (4.0 * PI);
  const i8 m4 = m & ~(i8)3;
  std::vector<double> xs(m), ys(m), zs(m);
  for (i8 i = 0; i < m; ++i) { xs[i] = tx[3 * i]; ys[i] = tx[3 * i + 1]; zs[i] = tx[3 * i + 2]; }
  const __m256d tiny = _mm256_set1_pd(1.0e-28), zero = _mm256_setzero_pd();
  for (i8 j = 0; j < n; ++j) {
    const double w4 = sw[j] * pi4inv;
    const __m256d vw = _mm256_set1_pd(w4), sxj = _mm256_set1_pd(sx[3 * j]), syj = _mm256_set1_pd(sx[3 * j + 1]),
                  szj = _mm256_set1_pd(sx[3 * j + 2]), nxj = _mm256_set1_pd(snx[3 * j]),
                  nyj = _mm256_set1_pd(snx[3 * j + 1]), nzj = _mm256_set1_pd(snx[3 * j + 2]);
    for (i8 i = 0; i < m4; i += 4) {
      const __m256d dx = _mm256_sub_pd(_mm256_loadu_pd(&xs[i]), sxj), dy = _mm256_sub_pd(_mm256_loadu_pd(&ys[i]), syj),
                    dz = _mm256_sub_pd(_mm256_loadu_pd(&zs[i]), szj);
      const __m256d rr = _mm256_add_pd(_mm256_add_pd(_mm256_mul_pd(dx, dx), _mm256_mul_pd(dy, dy)), _mm256_mul_pd(dz, dz));
      const __m256d ok = _mm256_cmp_pd(rr, tiny, _CMP_GT_OQ);
      const __m256d r = _mm256_sqrt_pd(rr);
      if (A) _mm256_storeu_pd(&A[i + m * j], _mm256_blendv_pd(zero, _mm256_div_pd(vw, r), ok));
      if (B) {
        const __m256d dn = _mm256_add_pd(_mm256_add_pd(_mm256_mul_pd(dx, nxj), _mm256_mul_pd(dy, nyj)), _mm256_mul_pd(dz, nzj));
        _mm256_storeu_pd(&B[i + m * j], _mm256_blendv_pd(zero, _mm256_div_pd(_mm256_mul_pd(vw, dn), _mm256_mul_pd(r, rr)), ok));
      }
    }
    for (i8 i = m4; i < m; ++i) {
      double dx = xs[i] - sx[3 * j], dy = ys[i] - sx[3 * j + 1], dz = zs[i] - sx[3 * j + 2];
      double rr = dx * dx + dy * dy + dz * dz;
      if (rr > 1.0e-28) {
        double r = std::sqrt(rr);
        if (A) A[i + m * j] = w4 / r;
        if (B) B[i + m * j] = w4 * (dx * snx[3 * j] + dy * snx[3 * j + 1] + dz * snx[3 * j + 2]) / (r * rr);
      } else {
        if (A) A[i + m * j] = 0.0;
        if (B) B[i + m * j] = 0.0;
      }
    }
  }
}
#endif

void sdlpmat(i8 m, const double* tx, i8 n, const double* sx, const double* snx,
             const double* sw, double* A, double* B) {
#ifdef __AVX2__
  if (g_orc_simd == 256) { sdlpmat_avx2(m, tx, n, sx, snx, sw, A, B); return; }
#endif
  const double pi4inv = 1.0 / (4.0 * PI);
  for (i8 j = 0; j < n; ++j) {
    double w4 = sw[j] * pi4inv;
    for (i8 i = 0; i < m; ++i) {
      double dx = tx[3 * i] - sx[3 * j], dy = tx[3 * i + 1] - sx[3 * j + 1],
             dz = tx[3 * i + 2] - sx[3 * j + 2];
      double rr = dx * dx + dy * dy + dz * dz;
      if (rr > 1.0e-28) {
        double r = std::sqrt(rr);
        if (A) A[i + m * j] = w4 / r;
        if (B) B[i + m * j] = w4 * (dx * snx[3 * j] + dy * snx[3 * j + 1] + dz * snx[3 * j + 2]) / (r * rr);
      } else {
        if (A) A[i + m * j] = 0.0;
        if (B) B[i + m * j] = 0.0;
      }
    }
  }
}

int g_orc_refine = 0;

const RefElem& ref_cached(int korder, int order, int nlevel, bool sqmode) {
  static std::mutex mu;
  static std::map<long long, RefElem*> refs;
  const long long key = korder + 1000LL * order + 1000000LL * nlevel + (sqmode ? 1000000000LL : 0);
  std::lock_guard<std::mutex> g(mu);
  auto it = refs.find(key);
  if (it != refs.end()) return *it->second;
  RefElem* R = new RefElem();
  build_ref(korder, order, nlevel, sqmode, *R);
  refs[key] = R;
  return *R;
}

/* walk (patch_refine_mod.f90:740-771): from the whole patch down the
 * quadtree of the first ntree levels (children of sub-patch q: 4q..4q+3), a
 * sub-patch whose ball excludes x joins the cut, one that contains it is
 * split, and containment at the last tree level fails the walk */
static bool cut_walk(const std::vector<PanelLevel>& lv, int ntree, const double* x,
                     std::vector<std::pair<int, i8>>& cut) {
  std::vector<i8> act(1, 0), nxt;
  cut.clear();
  for (int il = 0; il < ntree; ++il) {
    nxt.clear();
    const PanelLevel& P = lv[il];
    for (i8 q : act) {
      double d2 = 0.0;
      for (int d = 0; d < 3; ++d) { double t = x[d] - P.qpoint[3 * q + d]; d2 += t * t; }
      if (d2 > P.qradii2[q]) cut.push_back({il, q});
      else if (il == ntree - 1) return false;
      else for (int b = 0; b < 4; ++b) nxt.push_back(4 * q + b);
    }
    if (nxt.empty()) break;
    act.swap(nxt);
  }
  return true;
}

/* adaptive_pass (patch_refine_mod.f90:617-718): the targets the walk resolves
 * get the kernel on their cut's nodes contracted with the matching rows of
 * each level's interpmat (cut_gI, :720-738), summed node by node in cut
 * order; the rest stay in irem */
static void adaptive_cuts(const RefElem& R, const std::vector<PanelLevel>& lv, i8 m, const double* tx,
                          double* As, double* Ad, std::vector<i8>& irem, i8& nrem, i8* level_of) {
  const int np = R.npols, ntree = R.nlevel - 1;
  const i8 n1 = R.lev[0].n;
  std::vector<std::pair<int, i8>> cut;
  std::vector<double> a(n1), b(n1), ss(np), sd(np);
  i8 keep = 0;
  for (i8 jj = 0; jj < nrem; ++jj) {
    const i8 t = irem[jj];
    if (!cut_walk(lv, ntree, tx + 3 * t, cut)) { irem[keep++] = t; continue; }
    std::fill(ss.begin(), ss.end(), 0.0);
    std::fill(sd.begin(), sd.end(), 0.0);
    for (const auto& c : cut) {
      const PanelLevel& P = lv[c.first];
      const i8 i0 = c.second * n1;
      sdlpmat(1, tx + 3 * t, n1, P.sx.data() + 3 * i0, P.snx.data() + 3 * i0, P.sw.data() + i0, a.data(), b.data());
      const double* It = R.lev[c.first].interp_t.data() + (size_t)i0 * np;
      for (i8 q = 0; q < n1; ++q)
        for (int k = 0; k < np; ++k) { ss[k] += a[q] * It[(size_t)q * np + k]; sd[k] += b[q] * It[(size_t)q * np + k]; }
    }
    for (int k = 0; k < np; ++k) { As[t + m * k] = ss[k]; Ad[t + m * k] = sd[k]; }
    if (level_of) level_of[t] = 0;
  }
  nrem = keep;
}

void sdlpmat_levels(const RefElem& R, const std::vector<PanelLevel>& lv, i8 m,
                    const double* tx, double* As, double* Ad, i8* idxs, i8* ms,
                    i8* level_of) {
  int np = R.npols;
  std::vector<i8> irem(m), ibat, inext;
  for (i8 j = 0; j < m; ++j) irem[j] = j;
  i8 nrem = m;
  int il0 = 0;
  if (g_orc_refine == 1 && R.nlevel >= 3) { /* the walk, then one_level at the finest level */
    adaptive_cuts(R, lv, m, tx, As, Ad, irem, nrem, level_of);
    il0 = R.nlevel - 1;
  }
  for (int il = il0; il < R.nlevel && nrem > 0; ++il) {
    const PanelLevel& P = lv[il];
    ibat.clear(); inext.clear();
    for (i8 jj = 0; jj < nrem; ++jj) {
      i8 j = irem[jj];
      bool outside = true;
      for (i8 k = 0; k < P.nsub; ++k) {
        double d2 = 0.0;
        for (int d = 0; d < 3; ++d) { double t = P.qpoint[3 * k + d] - tx[3 * j + d]; d2 += t * t; }
        if (d2 < P.qradii2[k]) { outside = false; break; }
      }
      if (outside) ibat.push_back(j); else inext.push_back(j);
    }
    i8 nbat = (i8)ibat.size();
    if (nbat > 0) {
      i8 nl = P.n;
      std::vector<double> txb(3 * nbat), Ab((size_t)nbat * nl), Bb((size_t)nbat * nl);
      for (i8 i = 0; i < nbat; ++i)
        for (int d = 0; d < 3; ++d) txb[3 * i + d] = tx[3 * ibat[i] + d];
      sdlpmat(nbat, txb.data(), nl, P.sx.data(), P.snx.data(), P.sw.data(), Ab.data(), Bb.data());
      /* contraction with interpmat (the reference's dgemm), each output
       * summed over the level nodes in node order; the loop over the hd
       * outputs innermost (contiguous, vectorisable) */
      const double* It = R.lev[il].interp_t.data();
      std::vector<double> ss(np), sd(np);
      for (i8 i = 0; i < nbat; ++i) {
        i8 t = ibat[i];
        std::fill(ss.begin(), ss.end(), 0.0);
        std::fill(sd.begin(), sd.end(), 0.0);
        for (i8 q = 0; q < nl; ++q) {
          const double a = Ab[i + nbat * q], b = Bb[i + nbat * q];
          const double* Iq = It + (size_t)q * np;
          for (int k = 0; k < np; ++k) { ss[k] += a * Iq[k]; sd[k] += b * Iq[k]; }
        }
        for (int k = 0; k < np; ++k) { As[t + m * k] = ss[k]; Ad[t + m * k] = sd[k]; }
        if (level_of) level_of[t] = il + 1;
      }
    }
    nrem = (i8)inext.size();
    for (i8 jj = 0; jj < nrem; ++jj) irem[jj] = inext[jj];
  }
  *ms = nrem;
  for (i8 jj = 0; jj < nrem; ++jj) {
    idxs[jj] = irem[jj] + 1;
    if (level_of) level_of[irem[jj]] = R.nlevel + 1;
  }
}

} // namespace orc
