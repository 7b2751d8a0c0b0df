/* Oracle part 2: the RRQ close-panel correction (rrq_r64,
 * src/lap3d_close_mod.f90:622-881), restated.  TEST INFRASTRUCTURE ONLY.
 *
 * In-repo reference structure followed here:
 *  - frame: alpha = 1.25/sqrt(2 sum sw) (:709), rotation R from the vertex
 *    triangle and the origin shift c = c0 - (1.25 sx3min/alpha) R(3,:)
 *    (:503-509);
 *  - basis: the solid harmonics Im Y_l^m, 1<=m<=l<=nterms, evaluated with the
 *    harmonic axis along the frame's first axis ((X,Y,Z) = (y,z,x), :583-597);
 *  - D system: Mmatrix with its diagonal blocks zeroed (MD, :851-858) is the
 *    real form of the quaternion system  sum_j W_j grad h_k(y_j) = J_k,
 *    Ad_j = Sc W_j;  S system Msl^T As = Ocl + Fm^T Ad (:861-863).
 *  - line integrals of 1/r (Ichi) and 1/r^3 (Ialpha) kernels over the three
 *    edges with nquad Gauss nodes and singularity-swap weights w1, w3
 *    (:336-470, :797).
 *
 * Restated from the published mathematics (the LineQuaaadrature and
 * QuatApproximation submodules are not vendored):
 *  - the moments J_k = int_G E(y-x) n grad h_k dS (E = (y-x)/(4 pi r^3),
 *    quaternion products) follow from Cartan's homotopy formula for the closed
 *    2-form E dsigma grad p with p homogeneous about the target:
 *    int_G E n grad p = (1/(l-1)) oint E (rho x dy) grad p, l = deg p >= 2, and
 *    int_G E n dS = (-Omega/(4pi), (1/4pi) oint dy/r) for the l = 1 part;
 *    the homogeneous split is done exactly by the segment integrals
 *    Phi(y) = int_0^1 [grad h(x+t rho) - grad h(x)]/t dt and
 *    Psi(y) = int_0^1 grad h(x+t rho) dt (Gauss-Legendre, exact for the
 *    polynomial degree), which equals the local-to-local translation of the
 *    reference applied node by node;
 *  - Green's identity for the S moments: S[d_n h] = D[h] - h(x) D[1]
 *    + (1/4pi) oint (rho x dy).Psi / r;
 *  - singularity-swap quadrature (af Klinteberg & Tornberg, BIT 2021): complex
 *    root t0 of |gamma(t)-x|^2 by Newton on the Legendre interpolant, exact
 *    moments of |t-t0|^{-1}, |t-t0|^{-3} by recurrence, Bjorck-Pereyra dual
 *    Vandermonde solve;
 *  - the solid angle Omega = int_G (y-x).n/r^3 dS by the Dirac-string line
 *    integral oint (rho x s).dy/(r (r - s.rho)) with s pointing away from the
 *    panel (the exterior/interior flag decides for targets on the panel),
 *    integrated on a mesh graded towards the nearest edge point.
 */
#include "orc_common.h"
#include <algorithm>
#include <stdexcept>

namespace orc {

/* experiment switches (test hook; 0 = the documented behaviour) */
int g_orc_flags = 0;

/* ---------------- solid harmonics ---------------- */
/* Schmidt-normalised regular solid harmonics S_l^m, m>=1, in harmonic
 * coordinates (X,Y,Z) = (y,z,x) of the frame; outputs h = Im S_l^m and its
 * frame gradient for k = l(l-1)/2 + m-1, 1<=m<=l<=L. */
static void harm_eval(int L, double x, double y, double z, double* h, double* gx,
                      double* gy, double* gz) {
  const double X = y, Y = z, Z = x;
  const double r2 = X * X + Y * Y + Z * Z;
  /* (X+iY)^{m} C_m tracked with its derivative */
  cplx Pm(1.0, 0.0);      /* C_{m-1} (X+iY)^{m-1} */
  cplx Pm1(0.0, 0.0);     /* (m-1) C_{m-1} (X+iY)^{m-2} */
  const cplx w(X, Y);
  for (int m = 1; m <= L; ++m) {
    double cm = std::sqrt((2.0 * m - 1.0) / (2.0 * m));
    /* S_m^m = cm (X+iY) S_{m-1}^{m-1}; d/dX = cm [S_{m-1} + (X+iY) dS_{m-1}/dX] */
    cplx Smm = cm * w * Pm;
    cplx dSmm = cm * (Pm + w * Pm1); /* derivative w.r.t. (X+iY): d/dX; d/dY = i d/dX */
    Pm1 = dSmm; Pm = Smm;
    /* column m: value + gradient (gX, gY, gZ) */
    cplx s2 = 0.0, s2x = 0.0, s2y = 0.0, s2z = 0.0;        /* S_{l-2} */
    cplx s1 = Smm, s1x = dSmm, s1y = cplx(0, 1) * dSmm, s1z = 0.0; /* S_{l-1} */
    for (int l = m; l <= L; ++l) {
      cplx s, sx, sy, sz;
      if (l == m) {
        s = s1; sx = s1x; sy = s1y; sz = s1z;
      } else {
        double a = (2.0 * l - 1.0);
        double b = std::sqrt((double)(l + m - 1) * (double)(l - m - 1));
        double c = 1.0 / std::sqrt((double)(l - m) * (double)(l + m));
        s = (a * Z * s1 - b * r2 * s2) * c;
        sx = (a * Z * s1x - b * (2.0 * X * s2 + r2 * s2x)) * c;
        sy = (a * Z * s1y - b * (2.0 * Y * s2 + r2 * s2y)) * c;
        sz = (a * (s1 + Z * s1z) - b * (2.0 * Z * s2 + r2 * s2z)) * c;
        s2 = s1; s2x = s1x; s2y = s1y; s2z = s1z;
        s1 = s; s1x = sx; s1y = sy; s1z = sz;
      }
      int k = l * (l - 1) / 2 + (m - 1);
      if (h) h[k] = s.imag();
      gx[k] = sz.imag(); gy[k] = sx.imag(); gz[k] = sy.imag();
    }
  }
}

/* ---------------- small vector helpers ---------------- */
static inline void cross(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* Legendre series of degree n-1 and its derivative at complex t */
template <class T>
static void leg_eval(int n, const double* c /* n */, T t, T& f, T& fp) {
  T p0 = 1.0, p1 = t, d0 = 0.0, d1 = 1.0;
  f = c[0] * p0; fp = 0.0;
  if (n > 1) { f += c[1] * p1; fp += c[1] * d1; }
  for (int k = 1; k + 1 < n; ++k) {
    T p2 = ((2.0 * k + 1.0) * t * p1 - (double)k * p0) / (k + 1.0);
    T d2 = d0 + (2.0 * k + 1.0) * p1;
    f += c[k + 1] * p2; fp += c[k + 1] * d2;
    p0 = p1; p1 = p2; d0 = d1; d1 = d2;
  }
}

/* ---------------- singularity swap ---------------- */
/* Bjorck-Pereyra solve of sum_i x_i^k z_i = b_k, k = 0..n-1 (Golub & Van
 * Loan, Alg. 4.6.2); b is overwritten with z. */
static void bjorck_pereyra_dual(int n, const double* x, double* b) {
  int N = n - 1;
  for (int k = 0; k < N; ++k)
    for (int i = N; i >= k + 1; --i) b[i] -= x[k] * b[i - 1];
  for (int k = N - 1; k >= 0; --k) {
    for (int i = k + 1; i <= N; ++i) b[i] /= (x[i] - x[i - k - 1]);
    for (int i = k; i <= N - 1; ++i) b[i] -= b[i + 1];
  }
}

struct EdgeRoot {
  bool ok = false;
  cplx t0 = 0.0;
};

/* complex root of |gamma(t)-x|^2 nearest the edge, Newton on the Legendre
 * interpolant; gamma given by coefficients cf (3 x n: cf[d*n+k]). */
static EdgeRoot edge_root(int n, const double* cf, const double* tg, const double* bx,
                          const double* x) {
  EdgeRoot R;
  int ib = 0;
  double best = 1e300;
  for (int i = 0; i < n; ++i) {
    double d2 = 0.0;
    for (int d = 0; d < 3; ++d) { double t = bx[3 * i + d] - x[d]; d2 += t * t; }
    if (d2 < best) { best = d2; ib = i; }
  }
  /* local linearisation at the nearest node */
  double g[3], gp[3];
  for (int d = 0; d < 3; ++d) {
    double f, fp;
    leg_eval<double>(n, cf + d * n, tg[ib], f, fp);
    g[d] = f - x[d]; gp[d] = fp;
  }
  double aa = dot3(gp, gp), bb = dot3(g, gp), cc = dot3(g, g);
  double disc = std::max(aa * cc - bb * bb, 0.0);
  cplx t = cplx(tg[ib] - bb / aa, std::sqrt(disc) / aa);
  for (int it = 0; it < 40; ++it) {
    cplx F = 0.0, Fp = 0.0;
    for (int d = 0; d < 3; ++d) {
      cplx f, fp;
      leg_eval<cplx>(n, cf + d * n, t, f, fp);
      f -= x[d];
      F += f * f; Fp += 2.0 * f * fp;
    }
    if (std::abs(Fp) == 0.0) return R;
    cplx dt = F / Fp;
    t -= dt;
    if (std::abs(dt) < 1e-14 * std::max(1.0, std::abs(t))) {
      R.ok = std::isfinite(t.real()) && std::isfinite(t.imag());
      R.t0 = cplx(t.real(), std::fabs(t.imag()));
      return R;
    }
  }
  return R;
}

static double bernstein_radius(cplx t0) {
  cplx s = std::sqrt(t0 - 1.0) * std::sqrt(t0 + 1.0);
  return std::max(std::abs(t0 + s), std::abs(t0 - s));
}

static const double RHO_SSQ = 100.0; /* rrq_r64 :654 */
static const double RHO_REC = 3.0;   /* recurrence moments inside, 48-pt GL outside */

/* modified weights w1, w3 on the nquad Gauss nodes of one edge for target x */
static void ssq_weights(int n, const double* tg, const double* wg, const EdgeRoot& R,
                        const double* gl48x, const double* gl48w, double* w1, double* w3) {
  double a = R.t0.real(), b = std::fabs(R.t0.imag());
  /* a real root on the edge itself (the target on the boundary curve) has no
   * finite moments: plain Gauss there; a real root beyond an endpoint (the
   * target on the curve's continuation, e.g. a node of a neighbouring panel
   * near a shared vertex) keeps the singularity swap */
  bool use = R.ok && bernstein_radius(R.t0) < RHO_SSQ && (b > 0.0 || std::fabs(a) > 1.0);
  if (g_orc_flags & 4) use = false;
  if (!use) {
    for (int i = 0; i < n; ++i) { w1[i] = wg[i]; w3[i] = wg[i]; }
    return;
  }
  double Q[64], P[64];
  if (bernstein_radius(R.t0) < RHO_REC) {
    double s1 = std::sqrt((1.0 - a) * (1.0 - a) + b * b);
    double sm = std::sqrt((1.0 + a) * (1.0 + a) + b * b);
    double t02 = a * a + b * b;
    /* Q0 = int dt/s and P0 = int dt/s^3 over [-1,1], s = |t - t0|: for a root
     * beyond an endpoint in the cancellation-free forms (valid down to b = 0),
     * otherwise asinh((1-a)/b) + asinh((1+a)/b) and [(t-a)/(b^2 s)] */
    if (a > 1.0) {
      Q[0] = std::log((sm + 1.0 + a) / (s1 + a - 1.0));
      P[0] = 1.0 / (s1 * (s1 + a - 1.0)) - 1.0 / (sm * (sm + a + 1.0));
    } else if (a < -1.0) {
      Q[0] = std::log((s1 + 1.0 - a) / (sm - 1.0 - a));
      P[0] = 1.0 / (sm * (sm - a - 1.0)) - 1.0 / (s1 * (s1 - a + 1.0));
    } else {
      Q[0] = std::asinh((1.0 - a) / b) + std::asinh((1.0 + a) / b);
      P[0] = ((1.0 - a) / s1 + (1.0 + a) / sm) / (b * b);
    }
    for (int k = 1; k < n; ++k) {
      double bnd = s1 - ((k - 1) % 2 == 0 ? 1.0 : -1.0) * sm; /* [t^{k-1} s]_{-1}^{1} */
      double v = (2.0 * k - 1.0) * a * Q[k - 1] + bnd;
      if (k >= 2) v -= (k - 1.0) * t02 * Q[k - 2];
      Q[k] = v / k;
    }
    for (int k = 1; k < n; ++k) {
      double bnd = 1.0 / s1 - ((k - 1) % 2 == 0 ? 1.0 : -1.0) / sm; /* [t^{k-1}/s] */
      double v = a * P[k - 1] - bnd;
      if (k >= 2) v += (k - 1.0) * Q[k - 2];
      P[k] = v;
    }
  } else {
    for (int k = 0; k < n; ++k) { Q[k] = 0.0; P[k] = 0.0; }
    for (int q = 0; q < 48; ++q) {
      double t = gl48x[q];
      double s2 = (t - a) * (t - a) + b * b, s = std::sqrt(s2);
      double f1 = gl48w[q] / s, f3 = f1 / s2, tk = 1.0;
      for (int k = 0; k < n; ++k) { Q[k] += tk * f1; P[k] += tk * f3; tk *= t; }
    }
  }
  bjorck_pereyra_dual(n, tg, Q);
  bjorck_pereyra_dual(n, tg, P);
  for (int i = 0; i < n; ++i) {
    double s = std::sqrt((tg[i] - a) * (tg[i] - a) + b * b);
    w1[i] = Q[i] * s;
    w3[i] = P[i] * s * s * s;
  }
}

/* ---------------- per-panel precompute ---------------- */
struct RRQPanel {
  int nterms, hdim, nquad, nbd, ng;
  double R[9], c[3], alpha;
  std::vector<double> cfp;        /* Legendre coefs of the interpolant's edges (frame), 3 edges x 3 x nquad */
  std::vector<double> bx, bt, cf; /* boundary (frame) 3 x nbd, d/dt 3 x nbd, Legendre coefs 3 edges x 3 x nquad */
  std::vector<double> PD, PS, B;  /* hdim x 4hdim, hdim x hdim, hdim x hdim */
  std::vector<double> tq, wq, tgl, wgl, gl48x, gl48w, tsa, wsa;
  std::vector<double> scf; /* Koornwinder coefficients of the frame node positions, 3 x hdim */
  bool exterior;
  bool keep_systems = false;      /* keep copies of the two systems before factoring (conditioning checks) */
  std::vector<double> Dsys, Ssys; /* A^T (4hd x 4hd) and Msl^T (hd x hd), column-major */
};

static void circum_frame(const double* v1, const double* v2, const double* v3, double* R,
                         double* c0) {
  double a[3], b[3], n[3], e1[3], e2[3];
  for (int d = 0; d < 3; ++d) { a[d] = v2[d] - v1[d]; b[d] = v3[d] - v1[d]; }
  cross(a, b, n);
  double nn = std::sqrt(dot3(n, n));
  for (int d = 0; d < 3; ++d) n[d] /= nn;
  double la = std::sqrt(dot3(a, a));
  for (int d = 0; d < 3; ++d) e1[d] = a[d] / la;
  cross(n, e1, e2);
  for (int d = 0; d < 3; ++d) { R[0 + 3 * d] = e1[d]; R[1 + 3 * d] = e2[d]; R[2 + 3 * d] = n[d]; }
  /* circumcentre: v1 + [ |a|^2 b - |b|^2 a ] x (a x b) / (2 |a x b|^2) */
  double axb[3], p[3], q[3];
  cross(a, b, axb);
  double aa = dot3(a, a), bb = dot3(b, b), den = 2.0 * dot3(axb, axb);
  for (int d = 0; d < 3; ++d) p[d] = aa * b[d] - bb * a[d];
  cross(p, axb, q);
  for (int d = 0; d < 3; ++d) c0[d] = v1[d] + q[d] / den;
}

static inline void to_frame(const RRQPanel& P, const double* x, double* y) {
  double d[3] = {x[0] - P.c[0], x[1] - P.c[1], x[2] - P.c[2]};
  for (int i = 0; i < 3; ++i)
    y[i] = P.alpha * (P.R[i + 0] * d[0] + P.R[i + 3] * d[1] + P.R[i + 6] * d[2]);
}

static void build_rrq_panel(const RRQConfig& cfg, const double* sx, const double* snx,
                            const double* sw, const double* sxbd_chart, const double* rv_chart,
                            RRQPanel& P) {
  const int L = cfg.nterms, nq = cfg.nquad, hd = L * (L + 1) / 2, korder = L - 1;
  P.nterms = L; P.hdim = hd; P.nquad = nq; P.nbd = 3 * nq; P.exterior = cfg.exterior;
  P.tgl.resize(nq); P.wgl.resize(nq);
  std::vector<double> Dgl((size_t)nq * nq), Leg((size_t)nq * nq);
  gauss(nq, P.tgl.data(), P.wgl.data(), Dgl.data());
  legendre_vals2coefs(nq, P.tgl.data(), P.wgl.data(), Leg.data());
  P.gl48x.resize(48); P.gl48w.resize(48);
  gauss(48, P.gl48x.data(), P.gl48w.data(), nullptr);
  P.tsa.resize(16); P.wsa.resize(16);
  gauss(16, P.tsa.data(), P.wsa.data(), nullptr);
  P.ng = std::max(1, (L + 1) / 2);
  P.tq.resize(P.ng); P.wq.resize(P.ng);
  gauss(P.ng, P.tq.data(), P.wq.data(), nullptr);
  for (int g = 0; g < P.ng; ++g) { P.tq[g] = 0.5 * (P.tq[g] + 1.0); P.wq[g] *= 0.5; }

  /* interpolant through the VR nodes */
  std::vector<double> bnd_uv(2 * (3 * nq + 3));
  const double th1 = 2.0 * PI / 3.0, th2 = 4.0 * PI / 3.0, thi1 = 1.0 / th1;
  for (int e = 0; e < 3; ++e)
    for (int q = 0; q < nq; ++q) {
      double tt = e * th1 + 0.5 * (1.0 + P.tgl[q]) * th1;
      double u = 0.0, v = 0.0;
      if (tt < th1) v = 1.0 - thi1 * tt;
      else if (tt < th2) u = thi1 * (tt - th1);
      else { u = 1.0 - thi1 * (tt - th2); v = thi1 * (tt - th2); }
      bnd_uv[2 * (e * nq + q)] = u; bnd_uv[2 * (e * nq + q) + 1] = v;
    }
  double vert_uv[6] = {0, 0, 1, 0, 0, 1};
  for (int i = 0; i < 6; ++i) bnd_uv[2 * 3 * nq + i] = vert_uv[i];
  std::vector<double> Mb((size_t)(3 * nq + 3) * hd);
  interp_matrix(korder, 3 * nq + 3, bnd_uv.data(), Mb.data());
  std::vector<double> braw(3 * (3 * nq + 3), 0.0);
  for (int i = 0; i < 3 * nq + 3; ++i)
    for (int d = 0; d < 3; ++d) {
      double s = 0.0;
      for (int j = 0; j < hd; ++j) s += Mb[i + (size_t)(3 * nq + 3) * j] * sx[3 * j + d];
      braw[3 * i + d] = s;
    }
  double rv[9];
  if (cfg.ichart == 1) {
    for (int i = 0; i < 9; ++i) rv[i] = rv_chart[i];
    for (int i = 0; i < 3 * 3 * nq; ++i) braw[i] = sxbd_chart[i];
  } else {
    for (int i = 0; i < 9; ++i) rv[i] = braw[3 * 3 * nq + i];
  }
  double c0[3];
  circum_frame(rv, rv + 3, rv + 6, P.R, c0);
  if (g_orc_flags & 1) for (int d = 0; d < 3; ++d) { P.R[2 + 3 * d] = -P.R[2 + 3 * d]; P.R[1 + 3 * d] = -P.R[1 + 3 * d]; }
  double swsum = 0.0;
  for (int j = 0; j < hd; ++j) swsum += sw[j];
  P.alpha = 1.25 / std::sqrt(2.0 * swsum);
  /* origin shift below the lowest node (lap3d_close_mod.f90:503-509) */
  double zmin = 1e300;
  for (int j = 0; j < hd; ++j) {
    double d[3] = {sx[3 * j] - c0[0], sx[3 * j + 1] - c0[1], sx[3 * j + 2] - c0[2]};
    double z = P.alpha * (P.R[2] * d[0] + P.R[5] * d[1] + P.R[8] * d[2]);
    zmin = std::min(zmin, z);
  }
  double sx3min = (g_orc_flags & 2) ? 0.0 : std::max(0.0, -zmin);
  for (int d = 0; d < 3; ++d) P.c[d] = c0[d] - (1.25 * sx3min / P.alpha) * P.R[2 + 3 * d];

  /* the interpolant's own edges in the frame (used for the solid angle) */
  {
    std::vector<double> Dg2((size_t)nq * nq), Lg2((size_t)nq * nq), t2(nq), w2(nq);
    gauss(nq, t2.data(), w2.data(), nullptr);
    legendre_vals2coefs(nq, t2.data(), w2.data(), Lg2.data());
    std::vector<double> pb(3 * 3 * nq);
    for (int i = 0; i < 3 * nq; ++i) {
      double s3[3] = {0, 0, 0};
      for (int j = 0; j < hd; ++j)
        for (int d = 0; d < 3; ++d) s3[d] += Mb[i + (size_t)(3 * nq + 3) * j] * sx[3 * j + d];
      to_frame(P, s3, &pb[3 * i]);
    }
    P.cfp.assign(9 * nq, 0.0);
    for (int e = 0; e < 3; ++e)
      for (int d = 0; d < 3; ++d)
        for (int q = 0; q < nq; ++q) {
          double sc = 0.0;
          for (int k = 0; k < nq; ++k) sc += Lg2[q + (size_t)nq * k] * pb[3 * (e * nq + k) + d];
          P.cfp[e * 3 * nq + d * nq + q] = sc;
        }
  }
  /* boundary in the frame, its t-derivative per edge (t in [-1,1]) */
  P.bx.assign(3 * P.nbd, 0.0); P.bt.assign(3 * P.nbd, 0.0); P.cf.assign(9 * nq, 0.0);
  for (int i = 0; i < P.nbd; ++i) to_frame(P, &braw[3 * i], &P.bx[3 * i]);
  for (int e = 0; e < 3; ++e)
    for (int d = 0; d < 3; ++d) {
      for (int q = 0; q < nq; ++q) {
        double s = 0.0, sc = 0.0;
        for (int k = 0; k < nq; ++k) {
          s += Dgl[q + (size_t)nq * k] * P.bx[3 * (e * nq + k) + d];
          sc += Leg[q + (size_t)nq * k] * P.bx[3 * (e * nq + k) + d];
        }
        P.bt[3 * (e * nq + q) + d] = s;
        P.cf[e * 3 * nq + d * nq + q] = sc;
      }
    }

  /* basis at the nodes, quaternion system and the S system */
  std::vector<double> H((size_t)hd * hd), G1((size_t)hd * hd), G2((size_t)hd * hd),
      G3((size_t)hd * hd), Msl((size_t)hd * hd);
  for (int j = 0; j < hd; ++j) {
    double y[3], nrm[3];
    to_frame(P, &sx[3 * j], y);
    for (int i = 0; i < 3; ++i)
      nrm[i] = P.R[i] * snx[3 * j] + P.R[i + 3] * snx[3 * j + 1] + P.R[i + 6] * snx[3 * j + 2];
    std::vector<double> h(hd), gx(hd), gy(hd), gz(hd);
    harm_eval(L, y[0], y[1], y[2], h.data(), gx.data(), gy.data(), gz.data());
    for (int k = 0; k < hd; ++k) {
      H[j + (size_t)hd * k] = h[k];
      G1[j + (size_t)hd * k] = gx[k]; G2[j + (size_t)hd * k] = gy[k]; G3[j + (size_t)hd * k] = gz[k];
      Msl[j + (size_t)hd * k] = nrm[0] * gx[k] + nrm[1] * gy[k] + nrm[2] * gz[k];
    }
  }
  /* A (4hd x 4hd): rows (s,x,y,z) x k, cols (w0,w1,w2,w3) x j
   *  s: [0,-a,-b,-c]  x: [a,0,c,-b]  y: [b,-c,0,a]  z: [c,b,-a,0]
   * (the real form of W v for W = (w0,w), v = (0,(a,b,c)): (-w.v, w0 v + w x v))
   * with a(k,j) = d_x h_k(y_j) etc.  We need rows 0..hd-1 of A^{-1}:
   * solve A^T Z = I_{:,0:hd}. */
  const int N4 = 4 * hd;
  std::vector<double> AT((size_t)N4 * N4, 0.0);
  auto Aset = [&](int rb, int cb, const std::vector<double>& G, double sgn) {
    for (int k = 0; k < hd; ++k)
      for (int j = 0; j < hd; ++j) {
        int row = rb * hd + k, col = cb * hd + j;
        AT[col + (size_t)N4 * row] = sgn * G[j + (size_t)hd * k]; /* transpose */
      }
  };
  Aset(0, 1, G1, -1); Aset(0, 2, G2, -1); Aset(0, 3, G3, -1);
  Aset(1, 0, G1, +1); Aset(1, 2, G3, +1); Aset(1, 3, G2, -1);
  Aset(2, 0, G2, +1); Aset(2, 1, G3, -1); Aset(2, 3, G1, +1);
  Aset(3, 0, G3, +1); Aset(3, 1, G2, +1); Aset(3, 2, G1, -1);
  if (P.keep_systems) P.Dsys = AT;
  std::vector<int> piv(N4);
  if (lu_factor(N4, AT.data(), piv.data())) throw std::runtime_error("singular RRQ D system");
  std::vector<double> Z((size_t)N4 * hd, 0.0);
  for (int j = 0; j < hd; ++j) Z[j + (size_t)N4 * j] = 1.0;
  lu_solve(N4, AT.data(), piv.data(), Z.data(), hd);
  P.PD.assign((size_t)hd * N4, 0.0); /* PD(j, q) = Z(q, j) */
  for (int j = 0; j < hd; ++j)
    for (int q = 0; q < N4; ++q) P.PD[j + (size_t)hd * q] = Z[q + (size_t)N4 * j];
  /* PS = (Msl^T)^{-1}, B = PS * H^T with H^T(k,j) = h_k(y_j) */
  std::vector<double> MT((size_t)hd * hd);
  for (int k = 0; k < hd; ++k)
    for (int j = 0; j < hd; ++j) MT[k + (size_t)hd * j] = Msl[j + (size_t)hd * k];
  if (P.keep_systems) P.Ssys = MT;
  std::vector<int> piv2(hd);
  if (lu_factor(hd, MT.data(), piv2.data())) throw std::runtime_error("singular RRQ S system");
  P.PS.assign((size_t)hd * hd, 0.0);
  for (int j = 0; j < hd; ++j) P.PS[j + (size_t)hd * j] = 1.0;
  lu_solve(hd, MT.data(), piv2.data(), P.PS.data(), hd);
  P.B.assign((size_t)hd * hd, 0.0);
  for (int j = 0; j < hd; ++j)
    for (int i = 0; i < hd; ++i) {
      double s = 0.0;
      for (int k = 0; k < hd; ++k) s += P.PS[i + (size_t)hd * k] * H[j + (size_t)hd * k];
      P.B[i + (size_t)hd * j] = s;
    }
  std::vector<double> um((size_t)hd * hd);
  koorn_umatr(korder, um.data(), nullptr);
  P.scf.assign(3 * hd, 0.0);
  for (int j = 0; j < hd; ++j) {
    double y[3];
    to_frame(P, &sx[3 * j], y);
    for (int k = 0; k < hd; ++k)
      for (int d = 0; d < 3; ++d) P.scf[d * hd + k] += um[k + (size_t)hd * j] * y[d];
  }
}

/* edge point and derivative at parameter t from the Legendre coefficients */
static inline void edge_at(const RRQPanel& P, int e, double t, double* y, double* yp) {
  const std::vector<double>& cf = (g_orc_flags & 8) ? P.cfp : P.cf;
  for (int d = 0; d < 3; ++d) leg_eval<double>(P.nquad, &cf[e * 3 * P.nquad + d * P.nquad], t, y[d], yp[d]);
}

/* side of the target relative to the panel: +1 above (along R(3,:)), -1
 * below, 0 on the panel surface.  Newton on the in-plane coordinates of the
 * interpolated surface. */
static int panel_side(const RRQPanel& P, const double* xt, int* inside = nullptr) {
  const int hd = P.hdim, korder = P.nterms - 1;
  /* start from the in-plane nearest VR node, then Newton on (u,v) */
  std::vector<double> uvn(2 * hd), p(hd), pu(hd), pv(hd);
  vr_nodes(korder, uvn.data(), nullptr);
  int ib = 0; double best = 1e300;
  for (int j = 0; j < hd; ++j) {
    double f0 = 0, f1 = 0;
    koorn_pols(uvn[2 * j], uvn[2 * j + 1], korder, p.data());
    for (int k = 0; k < hd; ++k) { f0 += p[k] * P.scf[k]; f1 += p[k] * P.scf[hd + k]; }
    double d0 = f0 - xt[0], d1 = f1 - xt[1];
    if (d0 * d0 + d1 * d1 < best) { best = d0 * d0 + d1 * d1; ib = j; }
  }
  double uv[2] = {uvn[2 * ib], uvn[2 * ib + 1]};
  double zs = 0.0;
  for (int it = 0; it < 40; ++it) {
    const double h = 1e-7;
    koorn_pols(uv[0], uv[1], korder, p.data());
    koorn_pols(uv[0] + h, uv[1], korder, pu.data());
    koorn_pols(uv[0], uv[1] + h, korder, pv.data());
    double f0 = 0, f1 = 0, fu0 = 0, fu1 = 0, fv0 = 0, fv1 = 0;
    zs = 0.0;
    for (int k = 0; k < hd; ++k) {
      f0 += p[k] * P.scf[k]; f1 += p[k] * P.scf[hd + k]; zs += p[k] * P.scf[2 * hd + k];
      fu0 += pu[k] * P.scf[k]; fu1 += pu[k] * P.scf[hd + k];
      fv0 += pv[k] * P.scf[k]; fv1 += pv[k] * P.scf[hd + k];
    }
    double J00 = (fu0 - f0) / h, J10 = (fu1 - f1) / h, J01 = (fv0 - f0) / h, J11 = (fv1 - f1) / h;
    double r0 = f0 - xt[0], r1 = f1 - xt[1];
    double det = J00 * J11 - J01 * J10;
    if (det == 0.0) break;
    double du = (J11 * r0 - J01 * r1) / det, dv = (-J10 * r0 + J00 * r1) / det;
    uv[0] -= du; uv[1] -= dv;
    if (std::fabs(du) + std::fabs(dv) < 1e-14) break;
  }
  koorn_pols(uv[0], uv[1], korder, p.data());
  zs = 0.0;
  for (int k = 0; k < hd; ++k) zs += p[k] * P.scf[2 * hd + k];
  double hgt = xt[2] - zs;
  if (inside) {
    const double tol = 1e-10;
    *inside = (uv[0] >= -tol && uv[1] >= -tol && uv[0] + uv[1] <= 1.0 + tol) ? 1 : 0;
  }
  if (std::fabs(hgt) <= 1e-12) return 0;
  return hgt > 0 ? 1 : -1;
}

/* smallest (r - s.rho)/r over 32 samples per edge: how close the string
 * x + lambda s (lambda > 0) passes to the boundary, seen from x */
static double string_clearance(const RRQPanel& P, const double* xt, double sdir) {
  double cmin = 2.0;
  for (int e = 0; e < 3; ++e)
    for (int q = 0; q < 32; ++q) {
      double t = -1.0 + (2.0 * q + 1.0) / 32.0, y[3], yp[3];
      for (int d = 0; d < 3; ++d) leg_eval<double>(P.nquad, &P.cf[e * 3 * P.nquad + d * P.nquad], t, y[d], yp[d]);
      double rho[3] = {y[0] - xt[0], y[1] - xt[1], y[2] - xt[2]};
      double r = std::sqrt(dot3(rho, rho));
      double c = (r - sdir * rho[2]) / r;
      if (c < cmin) cmin = c;
    }
  return cmin;
}

/* Dirac-string direction: away from the panel when the target projects
 * inside the triangle (the exterior/interior flag decides on the panel);
 * otherwise both directions avoid the panel and the one passing farther from
 * the boundary is used. */
static double string_direction(const RRQPanel& P, const double* xt, bool exterior) {
  int inside = 1;
  int side = panel_side(P, xt, &inside);
  if (inside) return side == 0 ? (exterior ? 1.0 : -1.0) : (double)side;
  double cu = string_clearance(P, xt, 1.0), cd = string_clearance(P, xt, -1.0);
  return cu >= cd ? 1.0 : -1.0;
}

/* solid angle Omega = int_G (y-x).n/r^3 dS by the string formula along s */
static double solid_angle(const RRQPanel& P, const double* xt, const EdgeRoot* roots, const double* s) {
  double tot = 0.0;
  for (int e = 0; e < 3; ++e) {
    /* graded breakpoints towards the nearest parameter */
    double ts = 0.0, dd = 2.0;
    if (roots[e].ok) {
      ts = std::min(1.0, std::max(-1.0, roots[e].t0.real()));
      dd = std::max(std::fabs(roots[e].t0.imag()), 1e-15);
    }
    std::vector<double> br;
    br.push_back(-1.0); br.push_back(1.0);
    if (!roots[e].ok) {
      for (int k = 1; k < 16; ++k) br.push_back(-1.0 + k / 8.0);
    } else if (dd < 1.0) {
      for (double h = 0.5 * dd; h < 2.0; h *= 2.0) {
        if (ts - h > -1.0) br.push_back(ts - h);
        if (ts + h < 1.0) br.push_back(ts + h);
      }
    }
    std::sort(br.begin(), br.end());
    for (size_t ib = 0; ib + 1 < br.size(); ++ib) {
      double a = br[ib], b = br[ib + 1];
      if (!(b > a)) continue;
      double hm = 0.5 * (b - a), cm = 0.5 * (a + b);
      for (int q = 0; q < 16; ++q) {
        double t = cm + hm * P.tsa[q], y[3], yp[3];
        edge_at(P, e, t, y, yp);
        double rho[3] = {y[0] - xt[0], y[1] - xt[1], y[2] - xt[2]};
        double r = std::sqrt(dot3(rho, rho));
        double sr = dot3(s, rho), c[3];
        cross(rho, s, c);
        double den;
        if (sr > 0) den = dot3(c, c) / (r + sr); else den = r - sr;
        tot += hm * P.wsa[q] * dot3(c, yp) / (r * den);
      }
    }
  }
  return tot;
}

static void quat_mul_pure(const double* u, const double* v, double* q) {
  /* (0,u)(0,v) = (-u.v, u x v) */
  q[0] = -dot3(u, v);
  q[1] = u[1] * v[2] - u[2] * v[1];
  q[2] = u[2] * v[0] - u[0] * v[2];
  q[3] = u[0] * v[1] - u[1] * v[0];
}

/* one target's RRQ weights in physical scaling: As (hd), Ad (hd), Om (4hd), Ial */
static void rrq_target(const RRQPanel& P, const RRQConfig& cfg, const std::vector<double>& sxf,
                       const double* x, double* As, double* Ad, double* Om, double* Ial) {
  const int hd = P.hdim, nq = P.nquad, L = P.nterms;
  double xt[3];
  to_frame(P, x, xt);
  EdgeRoot roots[3];
  std::vector<double> w1(P.nbd), w3(P.nbd);
  for (int e = 0; e < 3; ++e) {
    roots[e] = edge_root(nq, &P.cf[e * 3 * nq], P.tgl.data(), &P.bx[3 * e * nq], xt);
    ssq_weights(nq, P.tgl.data(), P.wgl.data(), roots[e], P.gl48x.data(), P.gl48w.data(),
                &w1[e * nq], &w3[e * nq]);
  }
  (void)sxf;
  double sdir = string_direction(P, xt, cfg.exterior);
  double sv[3] = {0.0, 0.0, sdir};
  double Omega = solid_angle(P, xt, roots, sv);
  const double i4p = 1.0 / (4.0 * PI);

  /* per boundary node weights */
  std::vector<double> cD(3 * P.nbd), cS(3 * P.nbd);
  double lint[3] = {0, 0, 0};
  for (int i = 0; i < P.nbd; ++i) {
    const double* y = &P.bx[3 * i];
    const double* yp = &P.bt[3 * i];
    double rho[3] = {y[0] - xt[0], y[1] - xt[1], y[2] - xt[2]};
    double r = std::sqrt(dot3(rho, rho));
    double rxy[3], rrx[3];
    cross(rho, yp, rxy);
    cross(rho, rxy, rrx);
    double f1 = w1[i] / r, f3 = w3[i] / (r * r * r);
    for (int d = 0; d < 3; ++d) {
      cD[3 * i + d] = f3 * rrx[d];
      cS[3 * i + d] = f1 * rxy[d];
      lint[d] += f1 * yp[d];
    }
  }
  std::vector<double> hx(hd), gxx(hd), gyx(hd), gzx(hd), gx(hd), gy(hd), gz(hd);
  harm_eval(L, xt[0], xt[1], xt[2], hx.data(), gxx.data(), gyx.data(), gzx.data());
  std::vector<double> JD(4 * hd, 0.0), RS(hd, 0.0);
  double sumcD[3] = {0, 0, 0};
  for (int i = 0; i < P.nbd; ++i) {
    const double* y = &P.bx[3 * i];
    double rho[3] = {y[0] - xt[0], y[1] - xt[1], y[2] - xt[2]};
    for (int g = 0; g < P.ng; ++g) {
      double t = P.tq[g];
      double z[3] = {xt[0] + t * rho[0], xt[1] + t * rho[1], xt[2] + t * rho[2]};
      harm_eval(L, z[0], z[1], z[2], nullptr, gx.data(), gy.data(), gz.data());
      double aD = P.wq[g] / t, aS = P.wq[g];
      double uD[3] = {aD * cD[3 * i], aD * cD[3 * i + 1], aD * cD[3 * i + 2]};
      double uS[3] = {aS * cS[3 * i], aS * cS[3 * i + 1], aS * cS[3 * i + 2]};
      for (int d = 0; d < 3; ++d) sumcD[d] += uD[d];
      for (int k = 0; k < hd; ++k) {
        double v[3] = {gx[k], gy[k], gz[k]}, q[4];
        quat_mul_pure(uD, v, q);
        JD[k] += q[0]; JD[hd + k] += q[1]; JD[2 * hd + k] += q[2]; JD[3 * hd + k] += q[3];
        RS[k] += dot3(uS, v);
      }
    }
  }
  /* Q grad h(x) - (sum cD) grad h(x), then scale the line part by 1/(4pi) */
  for (int k = 0; k < hd; ++k) {
    double v[3] = {gxx[k], gyx[k], gzx[k]}, q[4], qq[4];
    quat_mul_pure(sumcD, v, q);
    /* Q = (-Omega/4pi, lint/4pi) times (0,v): (-l.v, s v + l x v) */
    double l[3] = {lint[0] * i4p, lint[1] * i4p, lint[2] * i4p};
    double s0 = -Omega * i4p;
    qq[0] = -dot3(l, v);
    qq[1] = s0 * v[0] + (l[1] * v[2] - l[2] * v[1]);
    qq[2] = s0 * v[1] + (l[2] * v[0] - l[0] * v[2]);
    qq[3] = s0 * v[2] + (l[0] * v[1] - l[1] * v[0]);
    for (int c = 0; c < 4; ++c) JD[c * hd + k] = (JD[c * hd + k] - q[c]) * i4p + qq[c];
    RS[k] = RS[k] * i4p + hx[k] * Omega * i4p;
  }
  const int N4 = 4 * hd;
  std::vector<double> adv(hd, 0.0);
  for (int j = 0; j < hd; ++j) {
    double s = 0.0;
    for (int q = 0; q < N4; ++q) s += P.PD[j + (size_t)hd * q] * JD[q];
    adv[j] = s;
  }
  for (int j = 0; j < hd; ++j) {
    double s = 0.0;
    for (int k = 0; k < hd; ++k) s += P.PS[j + (size_t)hd * k] * RS[k];
    for (int k = 0; k < hd; ++k) s += P.B[j + (size_t)hd * k] * adv[k];
    As[j] = s / P.alpha;
    Ad[j] = adv[j];
  }
  if (Om)
    for (int q = 0; q < N4; ++q) Om[q] = (q < hd ? JD[q] : -JD[q]) / P.alpha;
  if (Ial) *Ial = Omega;
}

void rrq(const RRQConfig& cfg, i8 m, const double* tx, const double* sx, const double* snx,
         const double* sw, const double* rts, const double* rps, const double* sxbd_chart,
         const double* rv_chart, double* As, double* Ad, double* Omega, double* Ialpha,
         i8* level_of) {
  const int L = cfg.nterms, hd = L * (L + 1) / 2;
  for (i8 i = 0; i < m * hd; ++i) { As[i] = 0.0; Ad[i] = 0.0; }
  if (Omega) for (i8 i = 0; i < m * 4 * hd; ++i) Omega[i] = 0.0;
  if (Ialpha) for (i8 i = 0; i < m; ++i) Ialpha[i] = 0.0;
  const RefElem& R = ref_cached(L - 1, cfg.orderff, 4, g_orc_refine == 0);
  std::vector<PanelLevel> lv;
  build_panel_levels(R, sx, rts, rps, cfg.distff, lv);
  std::vector<i8> idxs(m);
  i8 ms = 0;
  if (cfg.force) {
    ms = m;
    for (i8 i = 0; i < m; ++i) { idxs[i] = i + 1; if (level_of) level_of[i] = 5; }
  } else {
    sdlpmat_levels(R, lv, m, tx, As, Ad, idxs.data(), &ms, level_of);
  }
  if (ms == 0) return;
  RRQPanel P;
  build_rrq_panel(cfg, sx, snx, sw, sxbd_chart, rv_chart, P);
  std::vector<double> sxf(3 * hd);
  for (int j = 0; j < hd; ++j) to_frame(P, &sx[3 * j], &sxf[3 * j]);
  std::vector<double> as(hd), ad(hd), om(4 * hd);
  for (i8 jj = 0; jj < ms; ++jj) {
    i8 t = idxs[jj] - 1;
    double ial;
    rrq_target(P, cfg, sxf, &tx[3 * t], as.data(), ad.data(), om.data(), &ial);
    for (int k = 0; k < hd; ++k) { As[t + m * k] = as[k]; Ad[t + m * k] = ad[k]; }
    if (Omega) for (int q = 0; q < 4 * hd; ++q) Omega[q + (size_t)4 * hd * t] = om[q];
    if (Ialpha) Ialpha[t] = ial;
  }
}


/* the panel's two linear systems, as factored by build_rrq_panel: the D
 * system A^T (4hd x 4hd) and the S system Msl^T (hd x hd), column-major
 * (lap3d_close_mod.f90:851-863).  Conditioning checks of the tests use it. */
void panel_systems(const RRQConfig& cfg, const double* sx, const double* snx, const double* sw, double* DT,
                   double* MT) {
  RRQPanel P;
  P.keep_systems = true;
  build_rrq_panel(cfg, sx, snx, sw, nullptr, nullptr, P);
  std::copy(P.Dsys.begin(), P.Dsys.end(), DT);
  std::copy(P.Ssys.begin(), P.Ssys.end(), MT);
}

/* debug hook: per-edge roots and the solid angle on the graded mesh and on
 * a uniform 512-interval mesh, for one panel and one target */
void debug_target(const RRQConfig& cfg, const double* sx, const double* snx, const double* sw,
                  const double* x, double* out) {
  RRQPanel P;
  build_rrq_panel(cfg, sx, snx, sw, nullptr, nullptr, P);
  double xt[3];
  to_frame(P, x, xt);
  EdgeRoot roots[3];
  for (int e = 0; e < 3; ++e) {
    roots[e] = edge_root(P.nquad, &P.cf[e * 3 * P.nquad], P.tgl.data(), &P.bx[3 * e * P.nquad], xt);
    out[3 * e] = roots[e].ok; out[3 * e + 1] = roots[e].t0.real(); out[3 * e + 2] = roots[e].t0.imag();
  }
  double sv[3] = {0.0, 0.0, string_direction(P, xt, true)};
  out[9] = sv[2];
  out[10] = solid_angle(P, xt, roots, sv);
  EdgeRoot bad[3];
  double tot = 0.0;
  for (int e = 0; e < 3; ++e)
    for (int ib = 0; ib < 512; ++ib) {
      double a = -1.0 + 2.0 * ib / 512.0, b = a + 2.0 / 512.0, hm = 0.5 * (b - a), cm = 0.5 * (a + b);
      for (int q = 0; q < 16; ++q) {
        double t = cm + hm * P.tsa[q], y[3], yp[3];
        edge_at(P, e, t, y, yp);
        double rho[3] = {y[0] - xt[0], y[1] - xt[1], y[2] - xt[2]};
        double r = std::sqrt(dot3(rho, rho)), sr = dot3(sv, rho), c[3];
        cross(rho, sv, c);
        double den = sr > 0 ? dot3(c, c) / (r + sr) : r - sr;
        tot += hm * P.wsa[q] * dot3(c, yp) / (r * den);
      }
    }
  (void)bad;
  out[11] = tot;
  out[12] = xt[0]; out[13] = xt[1]; out[14] = xt[2];
}

} // namespace orc
