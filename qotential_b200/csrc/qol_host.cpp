/* Host-side per-order tables of the library: Gauss-Legendre data, the
 * Vioreanu-Rokhlin table, simplex interpolation and the reference-element
 * refinement levels (src/patch_refine_mod.f90:100-421).  Built once per order
 * on the host, uploaded to the device and cached. */
#include "qol_host.h"
#include "vr_table.h"
#include <algorithm>
#include <cfloat>
#include <cstdlib>
#include <stdexcept>

namespace qolh {
static const double QOL_PI_H = 3.14159265358979323846;

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
  }
}

void surface_eval(int nmode, const double* modes, int nfp, double t, double p, double* x) {
  double R = 0.0, Z = 0.0;
  for (int k = 0; k < nmode; ++k) {
    const double ang = modes[4 * k] * p - nfp * modes[4 * k + 1] * t;
    R = R + modes[4 * k + 2] * std::cos(ang);
    Z = Z + modes[4 * k + 3] * std::sin(ang);
  }
  x[0] = R * std::cos(t); x[1] = R * std::sin(t); x[2] = Z;
}

std::vector<Chart> surface_charts(int nmode, const double* modes, int nfp, int mp, int np, int nterms, bool split) {
  const double ASPECT = 1.65;
  std::vector<double> x0(nterms), w0(nterms);
  gauss(nterms, x0.data(), w0.data(), nullptr);
  const double ts1 = QOL_PI_H / np, ts2 = QOL_PI_H / mp;
  std::vector<Chart> cl;
  for (int j = 1; j <= np; ++j)
    for (int i = 1; i <= mp; ++i) {
      auto ev = [&](double t1, double t2, double* x) {
        surface_eval(nmode, modes, nfp, (t1 + 2.0 * j) * ts1, (t2 + 2.0 * i) * ts2, x);
      };
      double xll[3], xul[3], xlr[3];
      ev(x0[0], x0[0], xll); ev(x0[0], x0[nterms - 1], xul); ev(x0[nterms - 1], x0[0], xlr);
      double dt = 0.0, dp = 0.0;
      for (int d = 0; d < 3; ++d) { dt += (xll[d] - xlr[d]) * (xll[d] - xlr[d]); dp += (xll[d] - xul[d]) * (xll[d] - xul[d]); }
      dt = std::sqrt(dt); dp = std::sqrt(dp);
      const Chart base{1.0, 0.0, 1.0, 0.0, (double)j, (double)i};
      if (split && dt / dp > ASPECT) {
        Chart c1 = base, c2 = base; c1.a1 = 0.5; c1.b1 = -0.5; c2.a1 = 0.5; c2.b1 = 0.5;
        cl.push_back(c1); cl.push_back(c2);
      } else if (split && dp / dt > ASPECT) {
        Chart c1 = base, c2 = base; c1.a2 = 0.5; c1.b2 = -0.5; c2.a2 = 0.5; c2.b2 = 0.5;
        cl.push_back(c1); cl.push_back(c2);
      } else {
        cl.push_back(base);
      }
    }
  return cl;
}

namespace {
/* a chart's point: t1, t2 in [-1, 1] -> the surface at toroidal
 * ((a1 t1 + b1) + 2 jj) ts1, poloidal ((a2 t2 + b2) + 2 ii) ts2 */
struct ChartMap {
  int nmode, nfp;
  const double* modes;
  double ts1, ts2;
  void point(const Chart& c, double t1, double t2, double* x) const {
    surface_eval(nmode, modes, nfp, ((c.a1 * t1 + c.b1) + 2.0 * c.jj) * ts1, ((c.a2 * t2 + c.b2) + 2.0 * c.ii) * ts2,
                 x);
  }
};

double dist3(const double* a, const double* b) {
  return std::sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
}

/* the chart's parameter box [t1lo, t1hi, t2lo, t2hi] in units of ts1, ts2 */
void chart_box(const Chart& c, double ts1, double ts2, double* bx) {
  bx[0] = ((c.b1 - c.a1) + 2.0 * c.jj) * ts1;
  bx[1] = ((c.b1 + c.a1) + 2.0 * c.jj) * ts1;
  bx[2] = ((c.b2 - c.a2) + 2.0 * c.ii) * ts2;
  bx[3] = ((c.b2 + c.a2) + 2.0 * c.ii) * ts2;
}

/* the four quarters of a chart, (-,-), (+,-), (-,+), (+,+) in (t1, t2) */
void quarters(const Chart& c, Chart* q) {
  for (int k = 0; k < 4; ++k) {
    q[k] = c;
    q[k].a1 = c.a1 / 2.0;
    q[k].a2 = c.a2 / 2.0;
    q[k].b1 = c.b1 + ((k & 1) ? c.a1 / 2.0 : -c.a1 / 2.0);
    q[k].b2 = c.b2 + ((k & 2) ? c.a2 / 2.0 : -c.a2 / 2.0);
  }
}

/* A X = B in place (A p x p, B p x q, column-major), partial pivoting by
 * rows of the augmented system */
void solve_inplace(double* A, int p, double* B, int q) {
  for (int k = 0; k < p; ++k) {
    int ipv = k;
    double pmax = std::fabs(A[k + k * p]);
    for (int i = k + 1; i < p; ++i)
      if (std::fabs(A[i + k * p]) > pmax) { pmax = std::fabs(A[i + k * p]); ipv = i; }
    if (ipv != k) {
      for (int j = 0; j < p; ++j) std::swap(A[k + j * p], A[ipv + j * p]);
      for (int j = 0; j < q; ++j) std::swap(B[k + j * p], B[ipv + j * p]);
    }
    for (int i = k + 1; i < p; ++i) {
      const double f = A[i + k * p] / A[k + k * p];
      A[i + k * p] = f;
      for (int j = k + 1; j < p; ++j) A[i + j * p] -= f * A[k + j * p];
      for (int j = 0; j < q; ++j) B[i + j * p] -= f * B[k + j * p];
    }
  }
  for (int j = 0; j < q; ++j)
    for (int i = p - 1; i >= 0; --i) {
      double v = B[i + j * p];
      for (int k = i + 1; k < p; ++k) v -= A[i + k * p] * B[k + j * p];
      B[i + j * p] = v / A[i + i * p];
    }
}

/* panel_resolution (:338-416): the mean curvature H of the chart on its p x p
 * Gauss grid (node a + b p at (t1, t2) = (x0[b], x0[a])), from spectral
 * first and second derivatives (D), expanded in the tensor Legendre basis
 * (C = V^-1 H V^-T); the 2-norm share of the coefficients of degree p-2 or
 * p-1 in either direction */
double curvature_tail(const ChartMap& S, const Chart& c, int p, const std::vector<double>& x0,
                      const std::vector<double>& D, const std::vector<double>& V) {
  const int n2 = p * p;
  std::vector<double> X(3 * n2), r1(3 * n2), r2(3 * n2), r11(3 * n2), r12(3 * n2), r22(3 * n2), H(n2), Cf(n2),
      Tt(n2), A(n2);
  for (int b = 0; b < p; ++b)
    for (int a = 0; a < p; ++a) S.point(c, x0[b], x0[a], &X[3 * (a + b * p)]);
  auto along_t2 = [&](const std::vector<double>& f, std::vector<double>& g) { /* d/d(index a) */
    for (int b = 0; b < p; ++b)
      for (int a = 0; a < p; ++a)
        for (int d = 0; d < 3; ++d) {
          double v = 0.0;
          for (int k = 0; k < p; ++k) v += D[a + k * p] * f[3 * (k + b * p) + d];
          g[3 * (a + b * p) + d] = v;
        }
  };
  auto along_t1 = [&](const std::vector<double>& f, std::vector<double>& g) { /* d/d(index b) */
    for (int b = 0; b < p; ++b)
      for (int a = 0; a < p; ++a)
        for (int d = 0; d < 3; ++d) {
          double v = 0.0;
          for (int k = 0; k < p; ++k) v += D[b + k * p] * f[3 * (a + k * p) + d];
          g[3 * (a + b * p) + d] = v;
        }
  };
  along_t1(X, r1); along_t2(X, r2);
  along_t1(r1, r11); along_t1(r2, r12); along_t2(r2, r22);
  for (int k = 0; k < n2; ++k) {
    const double* u = &r1[3 * k];
    const double* v = &r2[3 * k];
    double nv[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
    double nn = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
    if (nn <= 0.0) nn = 1.0;
    for (double& t : nv) t /= nn;
    const double E = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const double F = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
    const double G = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const double L = nv[0] * r11[3 * k] + nv[1] * r11[3 * k + 1] + nv[2] * r11[3 * k + 2];
    const double M = nv[0] * r12[3 * k] + nv[1] * r12[3 * k + 1] + nv[2] * r12[3 * k + 2];
    const double N = nv[0] * r22[3 * k] + nv[1] * r22[3 * k + 1] + nv[2] * r22[3 * k + 2];
    double den = 2.0 * (E * G - F * F);
    if (den == 0.0) den = 1.0;
    H[k] = (E * N - 2.0 * F * M + G * L) / den;
  }
  Cf = H;
  A = V;
  solve_inplace(A.data(), p, Cf.data(), p);
  for (int a = 0; a < p; ++a)
    for (int b = 0; b < p; ++b) Tt[b + a * p] = Cf[a + b * p];
  A = V;
  solve_inplace(A.data(), p, Tt.data(), p);
  double tail = 0.0, tot = 0.0;
  for (int a = 0; a < p; ++a)
    for (int b = 0; b < p; ++b) {
      const double z = Tt[b + a * p];
      tot += z * z;
      if (a >= p - 2 || b >= p - 2) tail += z * z;
    }
  return std::sqrt(tail / (tot > 0.0 ? tot : 1.0));
}
} // namespace

bool surface_charts_adaptive(int nmode, const double* modes, int nfp, int mp, int np, int p, double restol,
                             long long cap, std::vector<Chart>& L) {
  const double ASPECT = 1.65;
  const int ASPECT_PASSES = 8, CURV_LEVELS = 12, BALANCE_SWEEPS = 20;
  if (cap <= 0) cap = 200000;
  std::vector<double> x0(p), w0(p), D((size_t)p * p), V((size_t)p * p);
  gauss(p, x0.data(), w0.data(), D.data());
  for (int i = 0; i < p; ++i) { /* Legendre Vandermonde V[i + k p] = P_k(x0_i) */
    V[i] = 1.0;
    if (p > 1) V[i + p] = x0[i];
    for (int k = 1; k < p - 1; ++k)
      V[i + (k + 1) * p] = ((2.0 * k + 1.0) * x0[i] * V[i + k * p] - k * V[i + (k - 1) * p]) / (k + 1.0);
  }
  const ChartMap S{nmode, nfp, modes, QOL_PI_H / np, QOL_PI_H / mp};
  L.clear();
  for (int j = 1; j <= np; ++j)
    for (int i = 1; i <= mp; ++i) L.push_back(Chart{1.0, 0.0, 1.0, 0.0, (double)j, (double)i});
  if ((long long)L.size() > cap) return false;
  /* 1. aspect: halve along the longer side, the second half appended (and
   * tested again within the same pass) */
  for (int pass = 0; pass < ASPECT_PASSES; ++pass) {
    int nsplit = 0;
    for (size_t k = 0; k < L.size(); ++k) {
      const Chart c = L[k];
      double xll[3], xul[3], xlr[3];
      S.point(c, x0[0], x0[0], xll);
      S.point(c, x0[0], x0[p - 1], xul);
      S.point(c, x0[p - 1], x0[0], xlr);
      const double dt = dist3(xll, xlr), dp = dist3(xll, xul);
      if (dt / dp > ASPECT || dp / dt > ASPECT) {
        if ((long long)L.size() >= cap) return false;
        Chart lo = c, hi = c;
        if (dt / dp > ASPECT) { lo.a1 = hi.a1 = c.a1 / 2.0; lo.b1 = c.b1 - c.a1 / 2.0; hi.b1 = c.b1 + c.a1 / 2.0; }
        else { lo.a2 = hi.a2 = c.a2 / 2.0; lo.b2 = c.b2 - c.a2 / 2.0; hi.b2 = c.b2 + c.a2 / 2.0; }
        L[k] = lo;
        L.push_back(hi);
        ++nsplit;
      }
    }
    if (!nsplit) break;
  }
  if (restol <= 0.0) return true;
  /* 2. curvature: quarter a chart while its curvature tail exceeds restol;
   * a chart that passes is not tested again */
  std::vector<char> done(L.size(), 0);
  for (int pass = 0; pass < CURV_LEVELS; ++pass) {
    int nsplit = 0;
    const size_t n0 = L.size();
    for (size_t k = 0; k < n0; ++k) {
      if (done[k]) continue;
      if (curvature_tail(S, L[k], p, x0, D, V) <= restol) { done[k] = 1; continue; }
      if ((long long)L.size() + 3 > cap) return false;
      Chart q[4];
      quarters(L[k], q);
      L[k] = q[0];
      for (int t = 1; t < 4; ++t) { L.push_back(q[t]); done.push_back(0); }
      ++nsplit;
    }
    if (!nsplit) break;
  }
  /* 3. 2:1 balance: quarter a chart whose face is longer than twice a face
   * neighbour's (periodic in both panel indices) */
  const double ts1 = S.ts1, ts2 = S.ts2;
  for (int pass = 0; pass < BALANCE_SWEEPS; ++pass) {
    const size_t n0 = L.size();
    std::vector<char> split(n0, 0);
    for (size_t k = 0; k < n0; ++k) {
      double bk[4];
      chart_box(L[k], ts1, ts2, bk);
      for (size_t q = 0; q < n0; ++q) {
        if (q == k) continue;
        const double dj = std::fabs(L[q].jj - L[k].jj), di = std::fabs(L[q].ii - L[k].ii);
        if (dj > 1.5 && std::fabs(dj - np) > 1.5) continue;
        if (di > 1.5 && std::fabs(di - mp) > 1.5) continue;
        double bq[4];
        chart_box(L[q], ts1, ts2, bq);
        const double du = 1e-9 * ts1, dv = 1e-9 * ts2;
        if ((std::fabs(bk[1] - bq[0]) < du || std::fabs(bk[0] - bq[1]) < du) &&
            std::fmin(bk[3], bq[3]) - std::fmax(bk[2], bq[2]) > dv) {
          if (bk[3] - bk[2] > 2.0 * (bq[3] - bq[2]) + dv) split[k] = 1;
        } else if ((std::fabs(bk[3] - bq[2]) < dv || std::fabs(bk[2] - bq[3]) < dv) &&
                   std::fmin(bk[1], bq[1]) - std::fmax(bk[0], bq[0]) > du) {
          if (bk[1] - bk[0] > 2.0 * (bq[1] - bq[0]) + du) split[k] = 1;
        }
      }
    }
    int nsplit = 0;
    for (size_t k = 0; k < n0; ++k) {
      if (!split[k]) continue;
      if ((long long)L.size() + 3 > cap) return false;
      Chart q[4];
      quarters(L[k], q);
      L[k] = q[0];
      for (int t = 1; t < 4; ++t) L.push_back(q[t]);
      ++nsplit;
    }
    if (!nsplit) break;
  }
  return true;
}

void surface_interp_tables(int p, std::vector<double>& tables) {
  const int hd = p * (p + 1) / 2;
  std::vector<double> x0(p), w0(p), uv(2 * hd);
  gauss(p, x0.data(), w0.data(), nullptr);
  vr_nodes(p - 1, uv.data(), nullptr);
  tables.assign((size_t)4 * hd * p * p, 0.0);
  auto lag = [&](double t, int j) { /* Lagrange basis j at t */
    double num = 1.0, den = 1.0;
    for (int k = 0; k < p; ++k)
      if (k != j) { num *= (t - x0[k]); den *= (x0[j] - x0[k]); }
    return num / den;
  };
  for (int key = 0; key < 4; ++key)
    for (int i = 0; i < hd; ++i) {
      const double u = 2.0 * uv[2 * i] - 1.0, v = 2.0 * uv[2 * i + 1] - 1.0;
      const double t1 = key == 0 ? u : key == 1 ? -u : key == 2 ? v : -v;
      const double t2 = key == 0 ? v : key == 1 ? -v : key == 2 ? -u : u;
      for (int b = 0; b < p; ++b)
        for (int a = 0; a < p; ++a)
          tables[((size_t)key * hd + i) * p * p + a + (size_t)b * p] = lag(t1, b) * lag(t2, a);
    }
}

void xlate_schedule(int L, int lanes, std::vector<uint32_t>& tab, int& steps, std::vector<uint32_t>& red,
                    int& slots) {
  struct Out { int idx; std::vector<uint32_t> terms; };
  std::vector<Out> outs;
  for (int n = 0; n < L; ++n)
    for (int k = 0; k <= n; ++k) {
      Out o;
      o.idx = n * (n + 1) / 2 + k;
      for (int lam = 0; lam <= n; ++lam) {
        const int nu = n - lam;
        for (int mu = std::max(-lam, k - nu); mu <= std::min(lam, k + nu); ++mu) {
          const int kr = k - mu, am = std::abs(mu), ar = std::abs(kr);
          const int neg = ((mu < 0 && (am & 1)) ? 1 : 0) ^ ((kr < 0 && (ar & 1)) ? 1 : 0);
          uint32_t w = (uint32_t)(lam * (lam + 1) / 2 + am) | ((uint32_t)(nu * (nu + 1) / 2 + ar) << 8) |
                       ((uint32_t)(mu < 0) << 26) | ((uint32_t)(kr < 0) << 27) | ((uint32_t)neg << 28) |
                       (1u << 29);
          o.terms.push_back(w);
        }
      }
      outs.push_back(std::move(o));
    }
  /* pieces of at most P terms (P = total / lanes, at least 8), each with its
   * own partial-sum slot; slots of an output are consecutive */
  size_t total = 0;
  for (const Out& o : outs) total += o.terms.size();
  const int P = std::max<int>(8, (int)((total + lanes - 1) / lanes));
  struct Piece { int slot, cost; std::vector<uint32_t> terms; };
  std::vector<Piece> pieces;
  red.assign(2 * outs.size(), 0u);
  slots = 0;
  for (const Out& o : outs) {
    const int c = (int)o.terms.size(), k = (c + P - 1) / P;
    red[2 * o.idx] = (uint32_t)slots;
    red[2 * o.idx + 1] = (uint32_t)k;
    for (int q = 0; q < k; ++q) {
      const int lo = (int)((long long)c * q / k), hi = (int)((long long)c * (q + 1) / k);
      Piece pc;
      pc.slot = slots++;
      pc.terms.assign(o.terms.begin() + lo, o.terms.begin() + hi);
      for (uint32_t& w : pc.terms) w |= (uint32_t)pc.slot << 16;
      pc.terms.back() |= 1u << 30; /* last term: flush to the slot */
      pc.cost = hi - lo;
      pieces.push_back(std::move(pc));
    }
  }
  /* longest first; ties by slot, lanes by load then index */
  std::vector<int> ord(pieces.size());
  for (size_t i = 0; i < ord.size(); ++i) ord[i] = (int)i;
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return pieces[a].cost > pieces[b].cost; });
  std::vector<std::vector<int>> lanep(lanes); /* pieces of each lane, in order */
  std::vector<int> load(lanes, 0);
  for (int pi : ord) {
    int best = 0;
    for (int q = 1; q < lanes; ++q)
      if (load[q] < load[best]) best = q;
    load[best] += pieces[pi].cost;
    lanep[best].push_back(pi);
  }
  steps = 0;
  for (int q = 0; q < lanes; ++q) steps = std::max(steps, load[q]);
  tab.assign((size_t)steps * lanes, 0u);
  /* Order of the terms inside each piece (any order sums the same terms): at
   * every step the 8 lanes of a quarter-warp should read M entries (14 doubles
   * apart, so 16-byte bank group 7 em + k mod 8) with distinct em mod 8 or the
   * same em, and R(x) entries (2 doubles apart) with distinct ex mod 8 or the
   * same ex; greedy per step, lanes in order, fewest clashes first (an M clash
   * costs its 6 loads, an R(x) clash 1), ties to the earlier term. */
  for (int g0 = 0; g0 < lanes; g0 += 8) {
    const int g1 = std::min(lanes, g0 + 8);
    std::vector<int> pc(lanes, 0);                /* current piece of the lane */
    std::vector<std::vector<uint32_t>> rem(lanes); /* its terms not yet placed */
    for (int q = g0; q < g1; ++q)
      if (!lanep[q].empty()) rem[q] = pieces[lanep[q][0]].terms;
    for (int s2 = 0; s2 < steps; ++s2) {
      std::vector<uint32_t> chosen;
      for (int q = g0; q < g1; ++q) {
        if (rem[q].empty()) continue; /* this lane is done */
        int bi = 0, bc = 1 << 30;
        for (int c = 0; c < (int)rem[q].size(); ++c) {
          const uint32_t em = rem[q][c] & 255, ex = (rem[q][c] >> 8) & 255;
          int cost = 0;
          for (uint32_t w : chosen) {
            const uint32_t em2 = w & 255, ex2 = (w >> 8) & 255;
            if (em2 != em && (em2 & 7) == (em & 7)) cost += 6;
            if (ex2 != ex && (ex2 & 7) == (ex & 7)) cost += 1;
          }
          if (cost < bc) { bc = cost; bi = c; }
        }
        uint32_t w = rem[q][bi] & ~(1u << 30);
        rem[q].erase(rem[q].begin() + bi);
        if (rem[q].empty()) { /* the piece's last term flushes it; then the next piece */
          w |= 1u << 30;
          if (++pc[q] < (int)lanep[q].size()) rem[q] = pieces[lanep[q][pc[q]]].terms;
        }
        chosen.push_back(w);
        tab[(size_t)s2 * lanes + q] = w;
      }
    }
  }
}

} // namespace qolh
