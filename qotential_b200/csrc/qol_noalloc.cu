/* qol_rrq_noalloc: the single-panel close correction (the work of qol_rrq)
 * for callers that cannot allocate GPU memory.
 *
 * Some callers cannot call cudaMalloc: codes embedded in a host application
 * that owns all GPU memory through its own pool allocator (a cudaMalloc there
 * fails under the pool's cap or fragments it), and codes on a latency-critical
 * path where cudaMalloc's implicit device-wide synchronisation is not allowed.
 * This entry point allocates no GPU memory: its workspace (refined levels,
 * per-panel RRQ matrices, per-target moments) and the per-order tables live in
 * one file-scope device array of QOL_NOALLOC_SCRATCH_BYTES (16 MiB) that every
 * GPU loading the library holds until exit.  The caller passes every input and
 * output as device memory.
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/qol_b200.h"
#include "qol_dev.cuh"
#include "qol_host.h"
#include "qol_kernels.h"

#define QOL_NOALLOC_SCRATCH_BYTES (16u << 20)

static __device__ __align__(256) unsigned char g_noalloc_scratch[QOL_NOALLOC_SCRATCH_BYTES];

namespace {

struct NoAllocDev {
  bool ready = false;
  unsigned char* base = nullptr; /* device address of g_noalloc_scratch on this device */
  long long key = -1;            /* order whose tables are resident */
  size_t table_bytes = 0;
  OrderTab T{};
};

std::mutex g_na_mu;
NoAllocDev g_na[64];
thread_local char g_na_msg[256];

int na_fail(int code, const char* msg) {
  std::snprintf(g_na_msg, sizeof g_na_msg, "%s", msg);
  return code;
}

#define NA_CK(x)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (x);                                                             \
    if (e_ != cudaSuccess) {                                                          \
      std::snprintf(g_na_msg, sizeof g_na_msg, "%s: %s", #x, cudaGetErrorString(e_)); \
      return QOL_ERR_CUDA;                                                            \
    }                                                                                 \
  } while (0)

/* first call on a device: the scratch array's device address (host code only
 * sees a stand-in for the symbol) and the harmonic recurrence coefficients */
int na_setup(int dev, cudaStream_t st) {
  NoAllocDev& D = g_na[dev];
  if (D.ready) return 0;
  void* p = nullptr;
  NA_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
  D.base = (unsigned char*)p;
  std::vector<double> hb((QOL_MAXL + 2) * (QOL_MAXL + 2), 0.0), hc(hb.size(), 0.0), hcm(QOL_MAXL + 2, 0.0);
  for (int m = 1; m <= QOL_MAXL; ++m) {
    hcm[m] = std::sqrt((2.0 * m - 1.0) / (2.0 * m));
    for (int l = m + 1; l <= QOL_MAXL; ++l) {
      hb[l * (QOL_MAXL + 2) + m] = std::sqrt((double)(l + m - 1) * (double)(l - m - 1));
      hc[l * (QOL_MAXL + 2) + m] = 1.0 / std::sqrt((double)(l - m) * (double)(l + m));
    }
  }
  NA_CK(qol_upload_harm_coefs(hb.data(), hc.data(), hcm.data(), st));
  D.ready = true;
  return 0;
}

/* the per-order tables, staged on the host and copied into the front of the
 * scratch array (same content as the other entry points' tables) */
int na_tables(NoAllocDev& D, int nterms, int orderff, int nquad, cudaStream_t st) {
  long long key = nterms + 100LL * orderff + 10000LL * nquad;
  if (D.key == key) return 0;
  const int korder = nterms - 1, hd = nterms * (nterms + 1) / 2;
  qolh::RefElem R;
  try {
    qolh::build_ref(korder, orderff, 4, true, R);
  } catch (...) {
    return na_fail(QOL_ERR_ORDER, "qol_rrq_noalloc: unsupported order");
  }
  std::vector<unsigned char> stage;
  auto put = [&](const void* src, size_t bytes) {
    size_t off = (stage.size() + 255) & ~(size_t)255;
    stage.resize(off + bytes);
    std::memcpy(stage.data() + off, src, bytes);
    return off;
  };
  OrderTab T{};
  T.korder = korder; T.hd = hd; T.nterms = nterms; T.orderff = orderff; T.nquad = nquad; T.nlevel = 4;
  T.ng = (nterms + 1) / 2 > 1 ? (nterms + 1) / 2 : 1;
  size_t o_interp[4], o_wt[4], o_so[4], o_st[4];
  for (int l = 0; l < 4; ++l) {
    const qolh::RefLevel& L = R.lev[l];
    T.n[l] = (int)L.n; T.nsub[l] = (int)L.nsub;
    const int ncw = 32 * ((hd + 31) / 32); /* zero-padded 16-byte rows */
    T.ncw = ncw;
    std::vector<double> rm((size_t)L.n * ncw, 0.0);
    for (long long i = 0; i < L.n; ++i)
      for (int k = 0; k < hd; ++k) rm[(size_t)i * ncw + k] = L.interp[i + (size_t)L.n * k];
    std::vector<int> stp(L.subtyp.begin(), L.subtyp.end());
    o_interp[l] = put(rm.data(), sizeof(double) * rm.size());
    o_wt[l] = put(L.wt.data(), sizeof(double) * L.wt.size());
    o_so[l] = put(L.suboff.data(), sizeof(long long) * L.suboff.size());
    o_st[l] = put(stp.data(), sizeof(int) * stp.size());
  }
  std::vector<double> tgl(nquad), wgl(nquad), Dgl(nquad * nquad), Leg(nquad * nquad);
  qolh::gauss(nquad, tgl.data(), wgl.data(), Dgl.data());
  qolh::legendre_vals2coefs(nquad, tgl.data(), wgl.data(), Leg.data());
  std::vector<double> g48x(48), g48w(48), g16x(16), g16w(16), tq(T.ng), wq(T.ng);
  qolh::gauss(48, g48x.data(), g48w.data(), nullptr);
  qolh::gauss(16, g16x.data(), g16w.data(), nullptr);
  qolh::gauss(T.ng, tq.data(), wq.data(), nullptr);
  for (int g = 0; g < T.ng; ++g) { tq[g] = 0.5 * (tq[g] + 1.0); wq[g] *= 0.5; }
  std::vector<double> buv(2 * (3 * nquad + 3));
  const double th1 = 2.0 * QOL_PI / 3.0, th2 = 4.0 * QOL_PI / 3.0, thi1 = 1.0 / th1;
  for (int e = 0; e < 3; ++e)
    for (int q = 0; q < nquad; ++q) {
      double tt = e * th1 + 0.5 * (1.0 + tgl[q]) * th1, u = 0.0, v = 0.0;
      if (tt < th1) v = 1.0 - thi1 * tt;
      else if (tt < th2) u = thi1 * (tt - th1);
      else { u = 1.0 - thi1 * (tt - th2); v = thi1 * (tt - th2); }
      buv[2 * (e * nquad + q)] = u; buv[2 * (e * nquad + q) + 1] = v;
    }
  const double vuv[6] = {0, 0, 1, 0, 0, 1};
  for (int i = 0; i < 6; ++i) buv[2 * 3 * nquad + i] = vuv[i];
  std::vector<double> Mcm((size_t)(3 * nquad + 3) * hd), Mb((size_t)(3 * nquad + 3) * hd);
  qolh::interp_matrix(korder, 3 * nquad + 3, buv.data(), Mcm.data());
  for (int i = 0; i < 3 * nquad + 3; ++i)
    for (int j = 0; j < hd; ++j) Mb[(size_t)i * hd + j] = Mcm[i + (size_t)(3 * nquad + 3) * j];
  std::vector<double> um((size_t)hd * hd), vr(2 * hd);
  qolh::koorn_umatr(korder, um.data(), nullptr);
  qolh::vr_nodes(korder, vr.data(), nullptr);
  size_t o_tgl = put(tgl.data(), 8 * tgl.size()), o_wgl = put(wgl.data(), 8 * wgl.size());
  size_t o_Dgl = put(Dgl.data(), 8 * Dgl.size()), o_Leg = put(Leg.data(), 8 * Leg.size());
  size_t o_48x = put(g48x.data(), 8 * 48), o_48w = put(g48w.data(), 8 * 48);
  size_t o_16x = put(g16x.data(), 8 * 16), o_16w = put(g16w.data(), 8 * 16);
  size_t o_tq = put(tq.data(), 8 * tq.size()), o_wq = put(wq.data(), 8 * wq.size());
  size_t o_Mb = put(Mb.data(), 8 * Mb.size()), o_um = put(um.data(), 8 * um.size());
  size_t o_vr = put(vr.data(), 8 * vr.size());
  std::vector<uint32_t> xs, xr;
  qolh::xlate_schedule(nterms, QOL_MOM_THREADS, xs, T.xsteps, xr, T.xslots);
  size_t o_xs = put(xs.data(), sizeof(uint32_t) * xs.size());
  size_t o_xr = put(xr.data(), sizeof(uint32_t) * xr.size());
  std::vector<double> tgi((size_t)nquad * nquad, 0.0); /* Bjorck-Pereyra node-difference reciprocals */
  for (int k = 0; k + 1 < nquad; ++k)
    for (int i = k + 1; i < nquad; ++i) tgi[(size_t)k * nquad + i] = 1.0 / (tgl[i] - tgl[i - k - 1]);
  size_t o_tgi = put(tgi.data(), sizeof(double) * tgi.size());
  size_t bytes = (stage.size() + 255) & ~(size_t)255;
  if (bytes > QOL_NOALLOC_SCRATCH_BYTES / 2)
    return na_fail(QOL_ERR_LIMIT, "qol_rrq_noalloc: tables of this order exceed half of the 16 MiB scratch");
  /* the copy overwrites the front of the scratch: until it has landed no
   * order's tables are resident, so a failed copy leaves none marked */
  D.key = -1;
  NA_CK(cudaMemcpyAsync(D.base, stage.data(), stage.size(), cudaMemcpyHostToDevice, st));
  NA_CK(cudaStreamSynchronize(st));
  auto dp = [&](size_t off) { return (const void*)(D.base + off); };
  for (int l = 0; l < 4; ++l) {
    T.interp[l] = (const double*)dp(o_interp[l]);
    T.wt[l] = (const double*)dp(o_wt[l]);
    T.suboff[l] = (const long long*)dp(o_so[l]);
    T.subtyp[l] = (const int*)dp(o_st[l]);
  }
  T.tgl = (const double*)dp(o_tgl); T.wgl = (const double*)dp(o_wgl);
  T.Dgl = (const double*)dp(o_Dgl); T.Leg = (const double*)dp(o_Leg);
  T.gl48x = (const double*)dp(o_48x); T.gl48w = (const double*)dp(o_48w);
  T.gl16x = (const double*)dp(o_16x); T.gl16w = (const double*)dp(o_16w);
  T.tq = (const double*)dp(o_tq); T.wq = (const double*)dp(o_wq);
  T.Mb = (const double*)dp(o_Mb); T.umatr = (const double*)dp(o_um); T.vruv = (const double*)dp(o_vr);
  T.xsched = (const unsigned*)dp(o_xs);
  T.xred = (const unsigned*)dp(o_xr);
  T.tginv = (const double*)dp(o_tgi);
  D.T = T;
  D.table_bytes = bytes;
  D.key = key;
  return 0;
}

/* every array argument must be device (or managed) memory of the current
 * device: a host pointer handed to the kernels would fault the GPU */
int na_check_device_ptr(const void* p, int dev, const char* name) {
  cudaPointerAttributes a{};
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError(); /* clear the error the query left */
    std::snprintf(g_na_msg, sizeof g_na_msg, "qol_rrq_noalloc: %s is not a CUDA pointer", name);
    return QOL_ERR_ARG;
  }
  if (a.type == cudaMemoryTypeManaged) return 0;
  if (a.type != cudaMemoryTypeDevice || a.device != dev) {
    std::snprintf(g_na_msg, sizeof g_na_msg, "qol_rrq_noalloc: %s must be device memory of the current device", name);
    return QOL_ERR_ARG;
  }
  return 0;
}

} // namespace

extern "C" const char* qol_noalloc_last_error(void) { return g_na_msg; }

extern "C" int qol_rrq_noalloc(qol_int m, const double* tx, qol_int n, const double* sx, const double* snx,
                               const double* sw, const double* rts, const double* rps, qol_int order, qol_int nquad,
                               qol_int orderff, double distff, qol_int exterior, double* As, double* Ad,
                               void* stream) {
  std::lock_guard<std::mutex> g(g_na_mu);
  const qol_int hd = order * (order + 1) / 2;
  if (n != hd) return na_fail(QOL_ERR_NPOLS, "qol_rrq_noalloc: n must equal order*(order+1)/2");
  if (m < 0 || (m > 0 && (!tx || !sx || !snx || !sw || !rts || !rps || !As || !Ad)))
    return na_fail(QOL_ERR_ARG, "qol_rrq_noalloc: bad arguments");
  if (order < 2 || order > QOL_MAXL || nquad < 2 || nquad > QOL_MAXNQ || orderff < 2 || orderff > 21)
    return na_fail(QOL_ERR_ORDER, "qol_rrq_noalloc: unsupported order");
  if (m == 0) return 0;
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0;
  NA_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return na_fail(QOL_ERR_ARG, "qol_rrq_noalloc: device index out of range");
  {
    const void* ptrs[8] = {tx, sx, snx, sw, rts, rps, As, Ad};
    const char* names[8] = {"tx", "sx", "snx", "sw", "rts", "rps", "As", "Ad"};
    for (int i = 0; i < 8; ++i) {
      int prc = na_check_device_ptr(ptrs[i], dev, names[i]);
      if (prc) return prc;
    }
  }
  int rc = na_setup(dev, st);
  if (rc) return rc;
  NoAllocDev& D = g_na[dev];
  if ((rc = na_tables(D, (int)order, (int)orderff, (int)nquad, st))) return rc;
  OrderTab T = D.T;
  T.dist = distff;
  const int nq = (int)nquad, nbd = 3 * nq;
  /* workspace after the tables; sizes checked against the scratch */
  size_t used = D.table_bytes;
  bool over = false;
  auto take = [&](size_t bytes) -> unsigned char* {
    size_t off = (used + 255) & ~(size_t)255;
    used = off + bytes;
    if (used > QOL_NOALLOC_SCRATCH_BYTES) over = true;
    return D.base + off;
  };
  LevelWS W{};
  for (int l = 0; l < 4; ++l) {
    W.node[l] = (double*)take(sizeof(double) * (size_t)T.n[l] * 7);
    W.sub[l] = (double*)take(sizeof(double) * (size_t)T.nsub[l] * 4);
  }
  PairWS G{};
  G.level = (signed char*)take((size_t)m);
  G.grp = (int*)take(sizeof(int) * (size_t)m);
  G.cnt = (int*)take(sizeof(int) * 8);
  G.off = (int*)take(sizeof(int) * 8);
  long long* rrq_off = (long long*)take(sizeof(long long) * 2);
  long long* dxi = (long long*)take(sizeof(long long) * 2);
  long long* drow = (long long*)take(sizeof(long long) * (size_t)m);
  RRQWS R{};
  R.npan = 1;
  R.rrq_off = rrq_off;
  R.frame = (double*)take(sizeof(double) * RRQ_FRAME);
  R.bx = (double*)take(sizeof(double) * 3 * nbd);
  R.bt = (double*)take(sizeof(double) * 3 * nbd);
  R.cf = (double*)take(sizeof(double) * 9 * nq);
  R.scf = (double*)take(sizeof(double) * 3 * hd);
  R.sxf = (double*)take(sizeof(double) * 3 * hd);
  R.hmat = (double*)take(sizeof(double) * hd * hd);
  R.smat = (double*)take(sizeof(double) * hd * hd);
  R.PD = (double*)take(sizeof(double) * 4 * hd * hd);
  R.B = (double*)take(sizeof(double) * hd * hd);
  R.JD = (double*)take(sizeof(double) * (size_t)m * 4 * hd);
  R.RS = (double*)take(sizeof(double) * (size_t)m * hd);
  R.line = (double*)take(sizeof(double) * (size_t)m * (6 * nbd + 4));
  R.edge = (double*)take(sizeof(double) * (size_t)m * 3 * (2 * nq + 3));
  R.pair = (int2*)take(sizeof(int2) * (size_t)(m > 0 ? m : 1));
  R.side = (signed char*)take((size_t)(m > 0 ? m : 1));
  if (over) {
    std::snprintf(g_na_msg, sizeof g_na_msg,
                  "qol_rrq_noalloc: m = %lld targets at order %lld need %zu bytes of scratch; the static scratch "
                  "holds %u bytes", (long long)m, (long long)order, used, (unsigned)QOL_NOALLOC_SCRATCH_BYTES);
    return QOL_ERR_LIMIT;
  }
  /* the scratch keeps the previous call's contents: clear what starts at zero */
  const long long xi[2] = {1, m + 1};
  NA_CK(cudaMemcpyAsync(dxi, xi, sizeof xi, cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemsetAsync(drow, 0, sizeof(long long) * (size_t)m, st));
  NA_CK(cudaMemsetAsync(G.cnt, 0, sizeof(int) * 8, st));
  NA_CK(cudaMemsetAsync(G.off, 0, sizeof(int) * 8, st));
  NA_CK(cudaMemsetAsync(As, 0, sizeof(double) * (size_t)m * hd, st));
  NA_CK(cudaMemsetAsync(Ad, 0, sizeof(double) * (size_t)m * hd, st));
  PanelIn P{sx, snx, sw, rts, rps};
  PairIn Q{tx, drow, dxi};
  OutCOO O{As, Ad, nullptr, 0};
  NA_CK(qol_launch_levels(T, P, W, 1, st));
  NA_CK(qol_launch_classify(T, Q, W, G, 1, st));
  NA_CK(qol_launch_scan(1, T.nlevel + 1, G.cnt, rrq_off, st));
  long long nrrq = 0;
  NA_CK(cudaMemcpyAsync(&nrrq, rrq_off + 1, sizeof(long long), cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
  R.nrrq = nrrq;
  R.glo = 0; R.ghi = nrrq; R.plo = 0; R.phi = 1;
  NA_CK(qol_launch_direct(T, P, Q, W, G, O, 1, st));
  if (nrrq > 0) {
    NA_CK(qol_launch_rrq_pairs(T, Q, G, R, 1, st));
    NA_CK(qol_launch_rrq_panel(T, P, G, R, 1, nullptr, st));
    NA_CK(qol_launch_rrq_target(T, Q, G, R, exterior != 0, st));
    NA_CK(qol_launch_rrq_apply(T, P, Q, G, R, O, st));
  }
  return 0;
}
