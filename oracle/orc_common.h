/* Oracle: CPU restatement of the RRQ near-field hot path of haiszhu/qotential.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the library (qotential_b200/) links,
 * imports or calls this code; only tests/, __graft_entry__.smoke() and the
 * bench's CPU-baseline leg do, and only as the checker / timed CPU baseline.
 *
 * All arithmetic is FP64, integers int64, arrays column-major with the
 * reference's layouts.  Each routine cites the reference file:line it restates.
 * Routines whose reference source lives in the un-vendored LineQuaaadrature /
 * QuatApproximation submodules are restated from the published mathematics
 * (see the comments at each one).
 */
#ifndef ORC_COMMON_H
#define ORC_COMMON_H
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

namespace orc {
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
  std::vector<double> interp_t;       /* the same, row-major (npols per node: the contraction's order) */
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

/* one panel's refined levels (build_patch_levels_r64, patch_refine_mod.f90:423-502) */
struct PanelLevel {
  i8 n = 0, nsub = 0;
  std::vector<double> sx, snx, sw, qpoint, qradii2;
};
void build_panel_levels(const RefElem& R, const double* sx, const double* rts,
                        const double* rps, double dist, std::vector<PanelLevel>& lv);

/* SLP/DLP kernel rows: S = w/(4 pi r), D = w (x-y).n/(4 pi r^3), zero for
 * r^2 <= 1e-28 (utils/f/ckernels_expts.c:52-123 formulas) */
void sdlpmat(i8 m, const double* tx, i8 n, const double* sx, const double* snx,
             const double* sw, double* A, double* B);

/* the patch refinement of the reference test's iadap switch
 * (test/stellarator_grf.f90:46-47 over patch_refine_mod.f90:53-56):
 * 0 square-regrouped levels (PR_SQUARE, the default), 1 the adaptive tree walk
 * on plain 4-split levels (PR_ADAPTIVE), 3 plain 4-split levels, level walk */
extern int g_orc_refine;
/* build_patch_ref_r64's cached reference element (patch_refine_mod.f90:100-121
 * returns early for the element it already holds), one per (korder, order,
 * nlevel, square mode) */
const RefElem& ref_cached(int korder, int order, int nlevel, bool sqmode);

/* lap3dsdlpmat_levels_r64 (patch_refine_mod.f90:516-615); with g_orc_refine
 * == 1 and nlevel >= 3 its adaptive branch (adaptive_pass, walk, cut_gI,
 * one_level at the finest level: :532-539, 617-771) */
void sdlpmat_levels(const RefElem& R, const std::vector<PanelLevel>& lv, i8 m,
                    const double* tx, double* As, double* Ad, i8* idxs, i8* ms,
                    i8* level_of /* nullable: per target level 1..4, 0 = an adaptive cut, 5 = unresolved */);

/* ---------------- RRQ ---------------- */
struct RRQConfig {
  int nterms, nquad, orderff;
  double distff;
  bool exterior;
  int ichart;
  bool force = false; /* test hook: send every target through the RRQ branch */
};
/* rrq_r64 (src/lap3d_close_mod.f90:622-881) restated.
 * sxbd_chart (3 x 3nquad) / rv_chart (3x3) are used when ichart == 1. */
void rrq(const RRQConfig& cfg, i8 m, const double* tx, const double* sx,
         const double* snx, const double* sw, const double* rts, const double* rps,
         const double* sxbd_chart, const double* rv_chart, double* As, double* Ad,
         double* Omega, double* Ialpha, i8* level_of);

/* kernel-matrix evaluation: 0 scalar, 256 AVX2 over 4 targets (the
 * reference's isimd = 256 path, src/patch_refine_mod.f90:575-591); both give
 * the same bits */
extern int g_orc_simd;
/* experiment switches, 0 in normal use (test hook) */
extern int g_orc_flags;
void panel_systems(const RRQConfig& cfg, const double* sx, const double* snx, const double* sw, double* DT,
                   double* MT);
void debug_target(const RRQConfig& cfg, const double* sx, const double* snx, const double* sw,
                  const double* x, double* out);

} // namespace orc
#endif
