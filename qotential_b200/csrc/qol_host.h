/* Host-side tables for the qol_b200 library (see qol_host.cpp). */
#ifndef QOL_HOST_H
#define QOL_HOST_H
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

namespace qolh {
typedef long long i8;
typedef std::complex<double> cplx;
static const double PI = 3.14159265358979323846264338327950288;

/* ---------------- small dense helpers ---------------- */
/* LU with partial pivoting, in place, column-major n x n; returns 0 if ok. */
int lu_factor(int n, double* A, int* piv);
/* Solve A X = B with the factors from lu_factor, B is n x nrhs column-major. */
void lu_solve(int n, const double* LU, const int* piv, double* B, int nrhs);

/* ---------------- 1D tables ---------------- */
/* Gauss-Legendre on [-1,1] (utils/gauss.m:1-37 restated): nodes ascending,
 * weights, and the spectral differentiation matrix D (n x n col-major, may be
 * null). */
void gauss(int n, double* x, double* w, double* D);
/* barycentric Lagrange weights 1/prod_{k!=j}(x_j-x_k) */
void bary_weights(int n, const double* x, double* wb);
/* Legendre values->coefficients matrix U(k,i) = (2k+1)/2 w_i P_k(x_i) */
void legendre_vals2coefs(int n, const double* x, const double* w, double* U);

/* ---------------- simplex interpolation ---------------- */
int npols_of(int korder);
/* orthogonal (Koornwinder/Dubiner) polynomials on the simplex
 * (0,0),(1,0),(0,1), total degree <= korder; pols[npols] */
void koorn_pols(double u, double v, int korder, double* pols);
/* VR nodes (2 x npts) and weights of degree deg */
void vr_nodes(int deg, double* uv, double* w);
/* umatr (vals->coefs) and vmatr (coefs->vals) at the VR nodes of degree korder */
void koorn_umatr(int korder, double* umatr, double* vmatr);
/* interpolation matrix n x npols from VR(korder) nodes to points uv */
void interp_matrix(int korder, int n, const double* uv, double* M);

/* ---------------- reference element levels ---------------- */
struct RefLevel {
  i8 n = 0, nsub = 0;
  std::vector<double> uv, wt, interp; /* interp n x npols col-major */
  std::vector<i8> suboff, subtyp;
};
struct RefElem {
  int korder = -1, npols = -1, order = -1, nlevel = -1;
  bool sqmode = true;
  std::vector<RefLevel> lev;
};
/* build_patch_ref_r64 + ref_square_regroup + cc_subidx_at
 * (src/patch_refine_mod.f90:100-262, 264-311, 313-421) */
void build_ref(int korder, int order, int nlevel, bool sqmode, RefElem& R);

/* ---------------- harmonic translation schedule ---------------- */
/* Work list of the regular-solid-harmonic translation
 *   T_n^k = sum_{lam=0..n} sum_mu M_lam^mu R_{n-lam}^{k-mu}(x),  0 <= k <= n <= L-1,
 * over `lanes` threads.  Each output's terms are cut into pieces of at most
 * max(8, total/lanes) terms; every piece sums into its own partial slot (slots
 * of one output consecutive: red[2o] first slot, red[2o+1] count, o =
 * n(n+1)/2+k); pieces go to lanes longest first (ties by slot, lanes by load
 * then index) and each lane runs its pieces back to back.  tab[s*lanes +
 * lane] is one term: bits 0-7 the M entry lam(lam+1)/2+|mu|, 8-15 the R entry
 * nu(nu+1)/2+|k-mu|, 16-25 the slot, 26 conj M (mu < 0), 27 conj R (k-mu < 0),
 * 28 negate ((-1)^|mu| (-1)^|k-mu| = -1), 29 valid, 30 last term of its piece. */
/* Fourier surface (VMEC convention of utils/stellarator_geo_mex.c surf_eval,
 * :91-102): R = sum rc cos(m p - nfp n t), Z = sum zs sin(m p - nfp n t),
 * x = (R cos t, R sin t, Z); modes (m, n, rc, zs) x nmode */
void surface_eval(int nmode, const double* modes, int nfp, double t, double p, double* x);
/* one chart of the mp x np (t, p) grid: t = ((a1 s + b1) + 2 jj) pi/np,
 * p = ((a2 s + b2) + 2 ii) pi/mp for s in [-1, 1] (build_charts,
 * utils/stellarator_geo_mex.c:125-160; split at aspect 1.65 when requested) */
struct Chart { double a1, b1, a2, b2, jj, ii; };
std::vector<Chart> surface_charts(int nmode, const double* modes, int nfp, int mp, int np, int nterms, bool split);
/* build_charts_adaptive (utils/stellarator_geo_mex.c:427-546): aspect passes,
 * then, for restol > 0, curvature refinement (the Legendre tail of the mean
 * curvature on the chart's p x p Gauss grid above restol) and 2:1 balance.
 * false when the list would exceed cap charts. */
bool surface_charts_adaptive(int nmode, const double* modes, int nfp, int mp, int np, int p, double restol,
                             long long cap, std::vector<Chart>& out);
/* Lagrange interpolation from the p Gauss nodes, tensor form: M (hd x p^2,
 * row-major, column m = a + b p) for the VR nodes of degree p-1 under the
 * four chart orientations (geo_core, :636-750): keys lA (u, v), rA (-u, -v),
 * lB (v, -u), rB (-v, u) with (u, v) = 2 uv - 1 */
void surface_interp_tables(int p, std::vector<double>& tables /* 4 x hd x p^2 */);
void xlate_schedule(int L, int lanes, std::vector<uint32_t>& tab, int& steps, std::vector<uint32_t>& red,
                    int& slots);

} // namespace qolh
#endif
