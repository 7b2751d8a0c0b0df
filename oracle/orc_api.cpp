/* Oracle C API (ctypes-facing).  TEST INFRASTRUCTURE ONLY: called from
 * tests/, __graft_entry__.smoke() and the bench's CPU-baseline leg, never by
 * the library. */
#include "orc_common.h"
#include <algorithm>
#include <cstdio>
#include <exception>
#include <map>
#include <mutex>
#include <omp.h>

using namespace orc;

namespace {
const RefElem& ref_for(int korder, int orderff, int nlevel, bool sq) { return ref_cached(korder, orderff, nlevel, sq); }
bool square() { return g_orc_refine == 0; }
} // namespace

extern "C" {

int orc_gauss(int n, double* x, double* w, double* D) {
  gauss(n, x, w, D);
  return 0;
}

int orc_debug_target(int nterms, int nquad, int orderff, const double* sx, const double* snx, const double* sw,
                     const double* x, double* out) {
  RRQConfig cfg{nterms, nquad, orderff, 1.4, true, 0};
  debug_target(cfg, sx, snx, sw, x, out);
  return 0;
}
/* the D and S systems of one panel's RRQ precompute (conditioning checks) */
int orc_rrq_panel_systems(int nterms, const double* sx, const double* snx, const double* sw, double* DT, double* MT) {
  RRQConfig cfg{nterms, nterms + 2, nterms + 2, 1.4, true, 0};
  try {
    panel_systems(cfg, sx, snx, sw, DT, MT);
  } catch (const std::exception&) {
    return 4;
  }
  return 0;
}
int orc_set_flags(int f) { orc::g_orc_flags = f; return 0; }
/* the reference test's iadap: 0 square levels, 1 adaptive tree walk, 3 plain levels */
int orc_set_refine(int iadap) {
  if (iadap != 0 && iadap != 1 && iadap != 3) return 1;
  orc::g_orc_refine = iadap;
  return 0;
}
/* isimd for the kernel-matrix sums: 0 scalar, 256 AVX2 (same results) */
int orc_set_simd(int isimd) { orc::g_orc_simd = isimd == 256 ? 256 : 0; return 0; }

int orc_vr_nodes_export(int deg, double* uv, double* w) {
  vr_nodes(deg, uv, w);
  return 0;
}

/* simplex_precomp_r64 (src/lap3d_close_mod.f90:115-133) */
int orc_simplex_precomp(int nquad, int korder, int kpols, double* tgl, double* wgl,
                        double* Dgl, double* wb, double* Leg, double* umatr, double* vmatr) {
  if (kpols != npols_of(korder)) return 3;
  gauss(nquad, tgl, wgl, Dgl);
  bary_weights(nquad, tgl, wb);
  legendre_vals2coefs(nquad, tgl, wgl, Leg);
  koorn_umatr(korder, umatr, vmatr);
  return 0;
}

int orc_ref_level_sizes(int korder, int orderff, int nlevel, int sq, long long* n, long long* nsub) {
  const RefElem& R = ref_for(korder, orderff, nlevel, sq != 0);
  for (int l = 0; l < nlevel; ++l) { n[l] = R.lev[l].n; nsub[l] = R.lev[l].nsub; }
  return 0;
}

int orc_ref_level_get(int korder, int orderff, int nlevel, int sq, int lev, double* uv,
                      double* wt, double* interp, long long* suboff, long long* subtyp) {
  const RefElem& R = ref_for(korder, orderff, nlevel, sq != 0);
  const RefLevel& L = R.lev[lev];
  if (uv) std::copy(L.uv.begin(), L.uv.end(), uv);
  if (wt) std::copy(L.wt.begin(), L.wt.end(), wt);
  if (interp) std::copy(L.interp.begin(), L.interp.end(), interp);
  if (suboff) std::copy(L.suboff.begin(), L.suboff.end(), suboff);
  if (subtyp) std::copy(L.subtyp.begin(), L.subtyp.end(), subtyp);
  return 0;
}

/* build_patch_levels_r64 for one panel, flattened level by level */
int orc_panel_levels(int korder, int npols, const double* sx, const double* rts,
                     const double* rps, int order, double dist, int nlevel, double* osx,
                     double* osnx, double* osw, double* oqp, double* oqr2) {
  if (npols != npols_of(korder)) return 3;
  const RefElem& R = ref_for(korder, order, nlevel, square());
  std::vector<PanelLevel> lv;
  build_panel_levels(R, sx, rts, rps, dist, lv);
  long long on = 0, os = 0;
  for (int l = 0; l < nlevel; ++l) {
    const PanelLevel& P = lv[l];
    std::copy(P.sx.begin(), P.sx.end(), osx + 3 * on);
    std::copy(P.snx.begin(), P.snx.end(), osnx + 3 * on);
    std::copy(P.sw.begin(), P.sw.end(), osw + on);
    std::copy(P.qpoint.begin(), P.qpoint.end(), oqp + 3 * os);
    std::copy(P.qradii2.begin(), P.qradii2.end(), oqr2 + os);
    on += P.n; os += P.nsub;
  }
  return 0;
}

/* build + lap3dsdlpmat_levels_r64 for one panel (patch_refine_mod.f90:423-615) */
int orc_sdlpmat_levels(int korder, int npols, const double* sx, const double* rts,
                       const double* rps, int order, double dist, int nlevel, long long m,
                       const double* tx, double* As, double* Ad, long long* idxs,
                       long long* ms, long long* level_of) {
  if (npols != npols_of(korder)) return 3;
  const RefElem& R = ref_for(korder, order, nlevel, square());
  std::vector<PanelLevel> lv;
  build_panel_levels(R, sx, rts, rps, dist, lv);
  for (long long i = 0; i < m * npols; ++i) { As[i] = 0.0; Ad[i] = 0.0; }
  sdlpmat_levels(R, lv, m, tx, As, Ad, idxs, ms, level_of);
  return 0;
}

int orc_sdlpmat(long long m, const double* tx, long long n, const double* sx,
                const double* snx, const double* sw, double* A, double* B) {
  sdlpmat(m, tx, n, sx, snx, sw, A, B);
  return 0;
}

/* rrq_r64 (src/lap3d_close_mod.f90:622-881) */
int orc_rrq(long long m, const double* tx, long long n, const double* sx, const double* snx,
            const double* sw, const double* rts, const double* rps, int nterms, int nquad,
            int orderff, double distff, int exterior, int ichart, const double* sxbd_chart,
            const double* rv_chart, double* As, double* Ad, double* Omega, double* Ialpha,
            long long* level_of) {
  if (n != (long long)nterms * (nterms + 1) / 2) return 3;
  try {
    RRQConfig cfg{nterms, nquad, orderff, distff, exterior != 0, ichart};
    cfg.force = (exterior & 2) != 0;
    cfg.exterior = (exterior & 1) != 0;
    rrq(cfg, m, tx, sx, snx, sw, rts, rps, sxbd_chart, rv_chart, As, Ad, Omega, Ialpha, level_of);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "orc_rrq: %s\n", e.what());
    return 5;
  }
  return 0;
}

/* getnearquad_lap_rrq_r64 (src/lap3d_close_mod.f90:884-960): per panel rrq
 * minus the self-masked naive block, COO in block column-major order. */
int orc_getnearquad(long long npan, int nterms, long long hdim, int nquad, long long nsrc,
                    const double* sx, const double* snx, const double* sw, const double* rts,
                    const double* rps, long long ntcx, const double* tcx, const long long* tcxrow,
                    const long long* tcxi, int orderff, double distff, long long iside,
                    long long nnz, long long* sparsei, long long* sparsej, double* sparsevs,
                    double* sparsevd, int nthreads, long long* level_hist, long long* pair_level) {
  if (hdim != (long long)nterms * (nterms + 1) / 2 || npan * hdim != nsrc) return 1;
  if (tcxi[0] != 1 || tcxi[npan] != ntcx + 1) return 1;
  for (long long k = 0; k < npan; ++k) if (tcxi[k + 1] < tcxi[k]) return 1;
  if ((tcxi[npan] - 1) * hdim > nnz) return 2;
  bool exterior = (iside % 10) == 0;
  RRQConfig cfg{nterms, nquad, orderff, distff, exterior, 0};
  (void)ref_for(nterms - 1, orderff, 4, square());
  int err = 0;
  long long hist[6] = {0, 0, 0, 0, 0, 0};
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : hist[:6])
  for (long long k = 0; k < npan; ++k) {
    long long jlo = tcxi[k] - 1, m = tcxi[k + 1] - tcxi[k];
    if (m <= 0) continue;
    long long idxlo = k * hdim;
    std::vector<double> As(m * hdim), Ad(m * hdim), An(m * hdim), Bn(m * hdim);
    std::vector<long long> lvl(m, 0);
    try {
      rrq(cfg, m, tcx + 3 * jlo, sx + 3 * idxlo, snx + 3 * idxlo, sw + idxlo, rts + 3 * idxlo,
          rps + 3 * idxlo, nullptr, nullptr, As.data(), Ad.data(), nullptr, nullptr, lvl.data());
    } catch (...) {
#pragma omp atomic write
      err = 5;
      continue;
    }
    sdlpmat(m, tcx + 3 * jlo, hdim, sx + 3 * idxlo, snx + 3 * idxlo, sw + idxlo, An.data(), Bn.data());
    for (long long i = 0; i < m; ++i) {
      long long row = tcxrow[jlo + i];
      if (row >= idxlo + 1 && row <= idxlo + hdim) {
        long long c = row - idxlo - 1;
        An[i + m * c] = 0.0; Bn[i + m * c] = 0.0;
      }
      hist[std::min<long long>(lvl[i], 5)]++;
      if (pair_level) pair_level[jlo + i] = lvl[i];
    }
    for (long long j = 0; j < hdim; ++j)
      for (long long i = 0; i < m; ++i) {
        long long o = jlo * hdim + j * m + i;
        sparsei[o] = tcxrow[jlo + i];
        sparsej[o] = idxlo + j + 1;
        sparsevs[o] = As[i + m * j] - An[i + m * j];
        sparsevd[o] = Ad[i + m * j] - Bn[i + m * j];
      }
  }
  if (level_hist) for (int i = 0; i < 6; ++i) level_hist[i] = hist[i];
  return err;
}

/* ball count + CSR fill of the GRF driver (stellarator_grf_core_mod.f90:652-693,
 * 774-806): targets are surface nodes inside 1.75 sqrt(area) of the panel's
 * node mean, in source order. */
int orc_ballcount(long long npan, long long hdim, long long nsrc, const double* sx,
                  const double* sw, long long* counts, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < npan; ++k) {
    double qp[3] = {0, 0, 0}, s = 0.0;
    for (long long i = 0; i < hdim; ++i) {
      for (int d = 0; d < 3; ++d) qp[d] += sx[3 * (k * hdim + i) + d];
      s += sw[k * hdim + i];
    }
    double qr = 1.75 * std::sqrt(s);
    for (int d = 0; d < 3; ++d) qp[d] /= (double)hdim;
    long long c = 0;
    for (long long j = 0; j < nsrc; ++j) {
      double a = sx[3 * j] - qp[0], b = sx[3 * j + 1] - qp[1], e = sx[3 * j + 2] - qp[2];
      if (a * a + b * b + e * e < qr * qr) ++c;
    }
    counts[k] = c;
  }
  return 0;
}

int orc_ballfill(long long npan, long long hdim, long long nsrc, const double* sx,
                 const double* sw, const long long* offs, long long* csr_idx, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < npan; ++k) {
    double qp[3] = {0, 0, 0}, s = 0.0;
    for (long long i = 0; i < hdim; ++i) {
      for (int d = 0; d < 3; ++d) qp[d] += sx[3 * (k * hdim + i) + d];
      s += sw[k * hdim + i];
    }
    double qr = 1.75 * std::sqrt(s);
    for (int d = 0; d < 3; ++d) qp[d] /= (double)hdim;
    long long c = offs[k];
    for (long long j = 0; j < nsrc; ++j) {
      double a = sx[3 * j] - qp[0], b = sx[3 * j + 1] - qp[1], e = sx[3 * j + 2] - qp[2];
      if (a * a + b * b + e * e < qr * qr) csr_idx[c++] = j + 1;
    }
  }
  return 0;
}

/* blocked Direct far field u_i = sum_j S_ij ubn_j - D_ij ub_j, self term zero
 * (stellarator_grf_core_mod.f90:566-606) */
int orc_direct_farfield(long long nsrc, const double* sx, const double* snx, const double* sw,
                        const double* ub, const double* ubn, double* u, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const double pi4inv = 1.0 / (4.0 * PI);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < nsrc; ++i) {
    double acc = 0.0;
    for (long long j = 0; j < nsrc; ++j) {
      double dx = sx[3 * i] - sx[3 * j], dy = sx[3 * i + 1] - sx[3 * j + 1],
             dz = sx[3 * i + 2] - sx[3 * j + 2];
      double rr = dx * dx + dy * dy + dz * dz;
      if (rr > 1.0e-28) {
        double w4 = sw[j] * pi4inv, r = std::sqrt(rr);
        double a = w4 / r;
        double b = w4 * (dx * snx[3 * j] + dy * snx[3 * j + 1] + dz * snx[3 * j + 2]) / (r * rr);
        acc = acc + a * ubn[j] - b * ub[j];
      }
    }
    u[i] = acc;
  }
  return 0;
}

/* the GRF near phase (stellarator_grf_core_mod.f90:760-899): per panel
 * rrq minus naive block contracted with (ubn, ub) into csr_val, then the serial
 * scatter in panel order.  xbuf (3 x (3 nquad + 3) per panel) carries the chart
 * boundary when ichart == 1. */
int orc_grf_near(long long npan, int nterms, int nquad, int orderff, double distff,
                 int exterior, int ichart, const double* xbuf, const double* sx,
                 const double* snx, const double* sw, const double* rts, const double* rps,
                 const double* ub, const double* ubn, const long long* offs,
                 const long long* csr_idx, double* u, double* csr_val, int nthreads,
                 long long* level_hist) {
  long long hdim = (long long)nterms * (nterms + 1) / 2, nbd = 3LL * nquad;
  RRQConfig cfg{nterms, nquad, orderff, distff, exterior != 0, ichart};
  (void)ref_for(nterms - 1, orderff, 4, square());
  int err = 0;
  long long hist[6] = {0, 0, 0, 0, 0, 0};
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : hist[:6])
  for (long long k = 0; k < npan; ++k) {
    long long o0 = offs[k], m = offs[k + 1] - offs[k];
    if (m == 0) continue;
    long long i0 = k * hdim;
    std::vector<double> tc(3 * m), S(m * hdim), K(m * hdim), An(m * hdim), Bn(m * hdim);
    std::vector<long long> lvl(m, 0);
    for (long long j = 0; j < m; ++j)
      for (int d = 0; d < 3; ++d) tc[3 * j + d] = sx[3 * (csr_idx[o0 + j] - 1) + d];
    const double* xb = xbuf ? xbuf + (size_t)k * 3 * (nbd + 3) : nullptr;
    try {
      rrq(cfg, m, tc.data(), sx + 3 * i0, snx + 3 * i0, sw + i0, rts + 3 * i0, rps + 3 * i0,
          xb, xb ? xb + 3 * nbd : nullptr, S.data(), K.data(), nullptr, nullptr, lvl.data());
    } catch (...) {
#pragma omp atomic write
      err = 5;
      continue;
    }
    sdlpmat(m, tc.data(), hdim, sx + 3 * i0, snx + 3 * i0, sw + i0, An.data(), Bn.data());
    for (long long j = 0; j < m; ++j) {
      csr_val[o0 + j] = 0.0;
      hist[std::min<long long>(lvl[j], 5)]++;
    }
    for (long long i2 = 0; i2 < hdim; ++i2)
      for (long long j = 0; j < m; ++j)
        csr_val[o0 + j] = csr_val[o0 + j] + (S[j + m * i2] - An[j + m * i2]) * ubn[i0 + i2] -
                          (K[j + m * i2] - Bn[j + m * i2]) * ub[i0 + i2];
  }
  if (err) return err;
  for (long long k = 0; k < npan; ++k)
    for (long long j = offs[k]; j < offs[k + 1]; ++j) u[csr_idx[j] - 1] += csr_val[j];
  if (level_hist) for (int i = 0; i < 6; ++i) level_hist[i] = hist[i];
  return 0;
}

} // extern "C"
