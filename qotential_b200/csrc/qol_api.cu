/* qol_b200 C ABI: context, per-order device tables, workspace, orchestration
 * of the hot-path kernels, and the qol_* entry points (see include/qol_b200.h
 * for the reference interface each one replaces). */
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <functional>
#include <thread>
#include <emmintrin.h>
#include <sys/mman.h>
#include <unistd.h>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/qol_b200.h"
#include "qol_dev.cuh"
#include "qol_host.h"
#include "qol_kernels.h"

namespace {

/* g_mu serialises the entry points, except qol_getnearquad_lap_rrq_dev,
 * which holds it only to set up and then runs under its stream's lock (calls
 * on different streams run concurrently); g_tab_mu guards the per-order
 * tables (their creation and the autotuner's one write), which every call
 * reads.  Lock order: g_mu, g_ctx_mu, a stream's lock, g_tab_mu. */
std::recursive_mutex g_mu;
std::recursive_mutex g_tab_mu;
thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(x)                                                                              \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess) return fail(QOL_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

/* ---------------- device arena ---------------- */
struct Arena {
  char* base = nullptr;
  size_t cap = 0, used = 0;
  ~Arena() { if (base) cudaFree(base); }
  int reserve(size_t bytes) {
    if (bytes <= cap) return 0;
    if (base) { cudaFree(base); base = nullptr; cap = 0; }
    size_t want = bytes + bytes / 8;
    if (cudaMalloc(&base, want) != cudaSuccess) {
      cudaGetLastError();
      return fail(QOL_ERR_CUDA, "device allocation of %zu bytes failed", want);
    }
    cap = want;
    return 0;
  }
  void reset() { used = 0; }
  void release() {
    if (base) cudaFree(base);
    base = nullptr;
    cap = used = 0;
  }
  template <class T>
  T* take(size_t n) {
    size_t off = (used + 255) & ~(size_t)255;
    used = off + n * sizeof(T);
    return (T*)(base + off);
  }
};

/* ---------------- per-order tables ---------------- */
struct OrderCache {
  OrderTab T{};
  std::vector<void*> bufs;
  ~OrderCache() { for (void* p : bufs) cudaFree(p); }
  template <class V>
  const typename V::value_type* up(const V& v) {
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(typename V::value_type) * std::max<size_t>(1, v.size())) != cudaSuccess) return nullptr;
    cudaMemcpy(p, v.data(), sizeof(typename V::value_type) * v.size(), cudaMemcpyHostToDevice);
    bufs.push_back(p);
    return (const typename V::value_type*)p;
  }
};

std::map<long long, std::unique_ptr<OrderCache>> g_orders;
bool g_coefs_uploaded = false;
Arena g_arena, g_arena2, g_arena_io, g_arena_grf; /* pipeline, per-pair RRQ storage, host-entry buffers, GRF */
std::vector<std::unique_ptr<Arena>> g_batch_arenas; /* the batched entry: two a job, one for its queue */
/* per-phase device milliseconds of the pipeline (diagnostics) */
int g_ktime_on = 0;
int g_sum_precision = 0; /* 0 FP64 (the drop-in), 1 FP32 level sums */
int g_autotune = 1;      /* measure the panel kernel's cluster size once per order */
/* learned level selector: off (0) or on (1), its BF16-rounded weights on the
 * device, the confidence threshold, and the decision counters of the calls */
int g_sel_mode = 0;
float g_sel_conf = 0.9f;
double g_sel_tol = 1e-8;  /* mode 2: the two-level check's row-error tolerance */
int g_force_level = 0;    /* labelling runs: direct pairs all on this level (0: off) */
/* patch refinement, the reference test's iadap (test/stellarator_grf.f90:46-47
 * over patch_refine_mod.f90:53-56): 0 square-regrouped levels (PR_SQUARE, the
 * default), 1 the adaptive tree walk on plain 4-split levels (PR_ADAPTIVE),
 * 3 plain 4-split levels with the level walk */
int g_refine = 0;
float* g_sel_w = nullptr;
unsigned long long* g_sel_cnt = nullptr; /* accepted, low confidence, check failed, pairs */
double g_ktime[QOL_NPHASE] = {};
long long g_kcalls = 0;
cudaStream_t g_stream = nullptr;

int ensure_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(QOL_ERR_CUDA, "no CUDA device available (the library has no CPU path)");
  }
  if (!g_stream) CK(cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking));
  if (!g_coefs_uploaded) {
    std::vector<double> hb((QOL_MAXL + 2) * (QOL_MAXL + 2), 0.0), hc(hb.size(), 0.0), hcm(QOL_MAXL + 2, 0.0);
    for (int m = 1; m <= QOL_MAXL; ++m) {
      hcm[m] = std::sqrt((2.0 * m - 1.0) / (2.0 * m));
      for (int l = m + 1; l <= QOL_MAXL; ++l) {
        hb[l * (QOL_MAXL + 2) + m] = std::sqrt((double)(l + m - 1) * (double)(l - m - 1));
        hc[l * (QOL_MAXL + 2) + m] = 1.0 / std::sqrt((double)(l - m) * (double)(l + m));
      }
    }
    CK(qol_upload_harm_coefs(hb.data(), hc.data(), hcm.data(), g_stream));
    g_coefs_uploaded = true;
  }
  return 0;
}

/* build (or fetch) the device tables for one (nterms, orderff, nquad) */
int order_tables(int nterms, int orderff, int nquad, OrderCache** out, int refine = -1) {
  std::lock_guard<std::recursive_mutex> tl(g_tab_mu);
  if (refine < 0) refine = g_refine;
  if (nterms < 2 || nterms > QOL_MAXL || orderff < 2 || orderff - 1 > 20 || nquad < 2 || nquad > QOL_MAXNQ ||
      nterms - 1 > 20)
    return fail(QOL_ERR_ORDER, "unsupported order nterms=%d orderff=%d nquad=%d", nterms, orderff, nquad);
  long long key = nterms + 100LL * orderff + 10000LL * nquad + 1000000LL * refine;
  auto it = g_orders.find(key);
  if (it != g_orders.end()) { *out = it->second.get(); return 0; }
  std::unique_ptr<OrderCache> C(new OrderCache());
  OrderTab& T = C->T;
  const int korder = nterms - 1, hd = nterms * (nterms + 1) / 2;
  qolh::RefElem R;
  try {
    qolh::build_ref(korder, orderff, 4, refine == 0, R);
  } catch (const std::exception& e) {
    return fail(QOL_ERR_ORDER, "reference element: %s", e.what());
  }
  T.korder = korder; T.hd = hd; T.nterms = nterms; T.orderff = orderff; T.nquad = nquad; T.nlevel = 4;
  T.adaptive = refine == 1;
  T.ng = std::max(1, (nterms + 1) / 2);
  for (int l = 0; l < 4; ++l) {
    const qolh::RefLevel& L = R.lev[l];
    T.n[l] = (int)L.n; T.nsub[l] = (int)L.nsub;
    std::vector<int> st(L.subtyp.begin(), L.subtyp.end());
    /* zero-padded rows of ncw columns, and their TF32 split of the FP32
     * rounding (round to nearest, ties away: the device's cvt.rna.tf32.f32) */
    auto tf32 = [](float x) {
      uint32_t u;
      std::memcpy(&u, &x, 4);
      u = (u + 0x1000u) & ~0x1FFFu;
      return u;
    };
    const int ncw = 32 * ((hd + 31) / 32);
    std::vector<double> rp((size_t)L.n * ncw, 0.0);
    /* the TF32 parts as the tcgen05.mma B operand (K-major, no swizzle):
     * tiles of 32 rows (zero padded), each [row quad][column][4 rows of the
     * quad], so a column's 8-column groups are 128-byte core matrices */
    const long long npad = (L.n + 31) / 32 * 32;
    std::vector<uint32_t> rh((size_t)npad * ncw, 0u), rl(rh.size(), 0u);
    for (long long i = 0; i < L.n; ++i)
      for (int k = 0; k < hd; ++k) {
        const size_t e = (size_t)i * ncw + k;
        rp[e] = L.interp[i + (size_t)L.n * k];
        const float f = (float)rp[e];
        const size_t fe = (size_t)(i / 32) * 32 * ncw + ((size_t)((i % 32) / 4) * ncw + k) * 4 + (i % 4);
        rh[fe] = tf32(f);
        float h;
        std::memcpy(&h, &rh[fe], 4);
        rl[fe] = tf32(f - h);
      }
    /* the selector check's sketch vectors on this level's nodes: I_l v for 4
     * fixed +-1 vectors v over the hd node values (a hash of (node, vector)) */
    auto sign = [](int k, int v) {
      uint32_t h = (uint32_t)(4 * k + v + 1) * 0x9E3779B1u;
      h ^= h >> 15; h *= 0x85EBCA77u; h ^= h >> 13;
      return (h & 1u) ? -1.0 : 1.0;
    };
    std::vector<double> sk((size_t)L.n * 4, 0.0);
    for (long long i = 0; i < L.n; ++i)
      for (int v = 0; v < 4; ++v) {
        double a = 0.0;
        for (int k = 0; k < hd; ++k) a += L.interp[i + (size_t)L.n * k] * sign(k, v);
        sk[(size_t)i * 4 + v] = a;
      }
    T.sk[l] = C->up(sk);
    T.ncw = ncw;
    T.interp[l] = C->up(rp);
    T.interp_hi[l] = C->up(rh);
    T.interp_lo[l] = C->up(rl);
    T.wt[l] = C->up(L.wt);
    T.suboff[l] = C->up(L.suboff);
    T.subtyp[l] = C->up(st);
  }
  std::vector<double> tgl(nquad), wgl(nquad), Dgl(nquad * nquad), Leg(nquad * nquad);
  qolh::gauss(nquad, tgl.data(), wgl.data(), Dgl.data());
  qolh::legendre_vals2coefs(nquad, tgl.data(), wgl.data(), Leg.data());
  std::vector<double> g48x(48), g48w(48), g16x(16), g16w(16), tq(T.ng), wq(T.ng);
  qolh::gauss(48, g48x.data(), g48w.data(), nullptr);
  qolh::gauss(16, g16x.data(), g16w.data(), nullptr);
  qolh::gauss(T.ng, tq.data(), wq.data(), nullptr);
  for (int g = 0; g < T.ng; ++g) { tq[g] = 0.5 * (tq[g] + 1.0); wq[g] *= 0.5; }
  /* boundary nodes of the three edges (tpar2uv parametrisation,
   * stellarator_grf_core_mod.f90:1069-1085) and the three vertices */
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
  double vuv[6] = {0, 0, 1, 0, 0, 1};
  for (int i = 0; i < 6; ++i) buv[2 * 3 * nquad + i] = vuv[i];
  std::vector<double> Mcm((size_t)(3 * nquad + 3) * hd), Mb((size_t)(3 * nquad + 3) * hd);
  qolh::interp_matrix(korder, 3 * nquad + 3, buv.data(), Mcm.data());
  for (int i = 0; i < 3 * nquad + 3; ++i)
    for (int j = 0; j < hd; ++j) Mb[(size_t)i * hd + j] = Mcm[i + (size_t)(3 * nquad + 3) * j];
  std::vector<double> um((size_t)hd * hd), vr(2 * hd);
  qolh::koorn_umatr(korder, um.data(), nullptr);
  qolh::vr_nodes(korder, vr.data(), nullptr);
  T.tgl = C->up(tgl); T.wgl = C->up(wgl); T.Dgl = C->up(Dgl); T.Leg = C->up(Leg);
  T.gl48x = C->up(g48x); T.gl48w = C->up(g48w); T.gl16x = C->up(g16x); T.gl16w = C->up(g16w);
  T.tq = C->up(tq); T.wq = C->up(wq); T.Mb = C->up(Mb); T.umatr = C->up(um); T.vruv = C->up(vr);
  std::vector<uint32_t> xs;
  std::vector<uint32_t> xr;
  qolh::xlate_schedule(nterms, QOL_MOM_THREADS, xs, T.xsteps, xr, T.xslots);
  T.xsched = C->up(xs);
  T.xred = C->up(xr);
  std::vector<double> tgi((size_t)nquad * nquad, 0.0); /* Bjorck-Pereyra node-difference reciprocals */
  for (int k = 0; k + 1 < nquad; ++k)
    for (int i = k + 1; i < nquad; ++i) tgi[(size_t)k * nquad + i] = 1.0 / (tgl[i] - tgl[i - k - 1]);
  T.tginv = C->up(tgi);
  if (!T.tgl || !T.Mb || !T.vruv || !T.xsched || !T.xred || !T.tginv)
    return fail(QOL_ERR_CUDA, "table upload failed");
  *out = C.get();
  g_orders[key] = std::move(C);
  return 0;
}

/* ---------------- the pipeline on device pointers ---------------- */
/* events recorded in stream order; the interval from ev[k] to ev[k+1]
 * belongs to phase ph[k] (-1: none) */
struct Timing {
  std::vector<cudaEvent_t> ev;
  std::vector<int> ph, sid; /* phase that starts at the event, stream index */
  bool on = false;
};

/* after the stream passed every event: accumulate into timeinfo (the
 * reference's slots) and the per-phase totals, release the events */
void finish_timing(Timing& tm, double* timeinfo) {
  if (!tm.on) return;
  double ms[QOL_NPHASE] = {};
  for (size_t k = 0; k < tm.ev.size(); ++k) { /* a phase ends at the next event on its stream */
    if (tm.ph[k] < 0) continue;
    size_t k2 = k + 1;
    while (k2 < tm.ev.size() && tm.sid[k2] != tm.sid[k]) ++k2;
    float t = 0.f;
    if (k2 < tm.ev.size() && cudaEventElapsedTime(&t, tm.ev[k], tm.ev[k2]) == cudaSuccess) ms[tm.ph[k]] += t;
  }
  if (timeinfo) {
    timeinfo[0] += 1e-3 * ms[0];                   /* patch levels */
    timeinfo[1] += 1e-3 * ms[3];                   /* per-panel RRQ precompute */
    timeinfo[2] += 1e-3 * (ms[1] + ms[2] + ms[9]); /* classification (selector) + level sums */
    timeinfo[5] += 1e-3 * (ms[4] + ms[5] + ms[6]); /* SSQ / solid angle / moments */
    timeinfo[7] += 1e-3 * (ms[7] + ms[8]);         /* solves + COO */
  }
  for (int i = 0; i < QOL_NPHASE; ++i) g_ktime[i] += ms[i];
  g_kcalls += 1;
  for (cudaEvent_t e : tm.ev) cudaEventDestroy(e);
  tm.ev.clear();
  tm.ph.clear();
  tm.sid.clear();
  tm.on = false;
}

struct Job {
  int npan, nterms, nquad, orderff, exterior, subtract_naive;
  double distff;
  long long ntcx;
  PanelIn P;
  PairIn Q;
  double *vs, *vd, *omega, *ialpha;
  long long *si, *sj;
  const double* chart;
  /* optional: the pipeline after classification over these panel chunks
   * (boundaries, first 0, last npan), alternating between the caller's
   * stream and a second one; after_chunk(c, s) once chunk c's values are
   * queued on stream s */
  const std::vector<long long>* chunk_pan;
  std::function<void(int, cudaStream_t)> after_chunk;
};

/* the second stream of chunked calls, one per device, created on first use */
int aux_stream(cudaStream_t* out) {
  static cudaStream_t s[64] = {};
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(QOL_ERR_CUDA, "device ordinal %d out of range", dev);
  if (!s[dev]) CK(cudaStreamCreateWithFlags(&s[dev], cudaStreamNonBlocking));
  *out = s[dev];
  return 0;
}

/* the back stage's launches on one stream of the device entry, captured as a
 * CUDA graph and replayed while every launch argument is unchanged (the same
 * order tables, workspace, buffers and sizes: a solver's repeated calls) */
struct BackKey {
  OrderTab T;
  PanelIn P;
  PairIn Q;
  LevelWS W;
  PairWS G;
  RRQWS R;
  OutCOO O;
  const double* chart;
  long long *si, *sj;
  long long nrrq;
  int npan, exterior, direct_done;
};
struct BackGraph {
  BackKey key;
  cudaGraphExec_t exec = nullptr;
  void drop() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
  }
};
std::atomic<long long> g_graph_captures{0}, g_graph_replays{0};
std::atomic<int> g_graphs_on{1}; /* qol_set_graphs */

/* one pipeline call, in two stages: front() sizes and lays out the
 * workspace, computes the refined levels, classifies the pairs and sizes the
 * per-pair RRQ storage (one host read of the RRQ count); back() runs the level
 * sums (unless done elsewhere: the batched entry's persistent kernel), the
 * RRQ phases and the COO indices */
struct PipeRun {
  const Job& J;
  cudaStream_t st;
  double* timeinfo;
  Arena* A1;
  Arena* A2;
  OrderCache* C = nullptr;
  OrderTab T{};
  int hd = 0, npan = 0, nq = 0, nbd = 0;
  long long ntcx = 0, nrrq = 0;
  LevelWS W{};
  PairWS G{};
  RRQWS R{};
  OutCOO O{};
  long long* rrq_off = nullptr;
  std::vector<long long> off_h;
  Timing tm;
  cudaStream_t st2 = nullptr;
  BackGraph* graph = nullptr; /* the stream's cached back stage (device entry), or none */
  PipeRun(const Job& j, cudaStream_t s, double* ti, Arena* a1 = &g_arena, Arena* a2 = &g_arena2)
      : J(j), st(s), timeinfo(ti), A1(a1), A2(a2) {}
  void rec(int phase, int sidx = 0) {
    if (!tm.on) return;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, sidx ? st2 : st);
    tm.ev.push_back(e);
    tm.ph.push_back(phase);
    tm.sid.push_back(sidx);
  }
  int front();
  int back(long long* hist_out, std::vector<int>* grp_out, int* cnt_out, bool direct_done);
  int launches(bool direct_done);
  bool back_graph(bool direct_done);
};

int PipeRun::front() {
  C = nullptr;
  int rc = 0;
  {
    std::lock_guard<std::recursive_mutex> tl(g_tab_mu);
    if ((rc = order_tables(J.nterms, J.orderff, J.nquad, &C))) return rc;
    T = C->T;
  }
  {
    int cs[8], nt[8];
    if (qol_panel_shapes(T.hd, T.nquad, cs, nt, 8) == 0) /* hdim 136 (nterms 16): no cluster of the panel kernel fits */
      return fail(QOL_ERR_ORDER, "nterms=%d (hdim %d): the per-panel RRQ precompute has no launch shape; nterms <= 15",
                  J.nterms, T.hd);
  }
  T.dist = J.distff;
  T.sum_fp32 = g_sum_precision == 1;
  T.force_level = g_force_level;
  hd = T.hd; npan = J.npan; nq = T.nquad; nbd = 3 * nq;
  ntcx = J.ntcx;
  /* workspace size */
  size_t need = 0;
  auto add = [&](size_t bytes) { need += (bytes + 255) & ~(size_t)255; };
  for (int l = 0; l < 4; ++l) { add(sizeof(double) * (size_t)npan * T.n[l] * 7); add(sizeof(double) * (size_t)npan * T.nsub[l] * 4); }
  add(ntcx); add(sizeof(int) * ntcx); add(sizeof(int) * (size_t)npan * 8 * 2);
  add(sizeof(long long) * (npan + 1));
  add(sizeof(double) * (size_t)npan * (RRQ_FRAME + 6 * nbd + 9 * nq + 6 * hd));
  add(sizeof(double) * (size_t)npan * hd * hd * 7);
  rc = A1->reserve(need + 4096);
  if (rc) return rc;
  A1->reset();
  W = LevelWS{};
  for (int l = 0; l < 4; ++l) {
    W.node[l] = A1->take<double>((size_t)npan * T.n[l] * 7);
    W.sub[l] = A1->take<double>((size_t)npan * T.nsub[l] * 4);
  }
  G = PairWS{};
  G.level = A1->take<signed char>(ntcx);
  G.grp = A1->take<int>(ntcx);
  G.cnt = A1->take<int>((size_t)npan * 8);
  G.off = A1->take<int>((size_t)npan * 8);
  R = RRQWS{};
  R.npan = npan;
  rrq_off = A1->take<long long>(npan + 1);
  R.rrq_off = rrq_off;
  R.frame = A1->take<double>((size_t)npan * RRQ_FRAME);
  R.bx = A1->take<double>((size_t)npan * 3 * nbd);
  R.bt = A1->take<double>((size_t)npan * 3 * nbd);
  R.cf = A1->take<double>((size_t)npan * 9 * nq);
  R.scf = A1->take<double>((size_t)npan * 3 * hd);
  R.sxf = A1->take<double>((size_t)npan * 3 * hd);
  R.hmat = A1->take<double>((size_t)npan * hd * hd);
  R.smat = A1->take<double>((size_t)npan * hd * hd);
  R.PD = A1->take<double>((size_t)npan * 4 * hd * hd);
  R.B = A1->take<double>((size_t)npan * hd * hd);
  R.ialpha = J.ialpha;
  CK(cudaMemsetAsync(G.cnt, 0, sizeof(int) * (size_t)npan * 8, st));
  CK(cudaMemsetAsync(G.off, 0, sizeof(int) * (size_t)npan * 8, st));
  tm.on = timeinfo || g_ktime_on;
  st2 = st; /* chunked calls: odd chunks run here */
  rec(0);
  CK(qol_launch_levels(T, J.P, W, npan, st));
  rec(1);
  if (g_sel_mode && g_sel_w && !g_force_level && !g_refine) { /* confident, checked predictions first; the walk for the rest */
    rec(9);
    CK(qol_launch_sel_infer(T, J.P, J.Q, W, G, npan, g_sel_w, g_sel_conf, g_sel_cnt, g_sel_mode, st));
    if (g_sel_mode == 2) CK(qol_launch_sel_check(T, J.P, J.Q, W, G, npan, g_sel_tol, g_sel_cnt, st));
    rec(1);
    CK(qol_launch_classify(T, J.Q, W, G, npan, st, 1));
  } else {
    CK(qol_launch_classify(T, J.Q, W, G, npan, st));
  }
  CK(qol_launch_scan(npan, T.nlevel + 1, G.cnt, rrq_off, st));
  /* RRQ pair offsets per panel (all of them when the per-pair phase is chunked) */
  off_h.assign(J.chunk_pan ? npan + 1 : 1, 0);
  CK(cudaMemcpyAsync(off_h.data(), J.chunk_pan ? rrq_off : rrq_off + npan, sizeof(long long) * off_h.size(),
                     cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (g_sel_mode && g_sel_w && !g_force_level && !g_refine) { /* the inference's waits on the tensor cores are bounded */
    unsigned werr = 0;
    CK(qol_sel_wait_error(&werr, st));
    if (werr) return fail(QOL_ERR_CUDA, "selector inference: a wait on the tensor cores timed out");
  }
  nrrq = off_h.back();
  R.nrrq = nrrq;
  /* per-pair RRQ moment storage (separate arena: its size is known only now) */
  rc = A2->reserve(sizeof(double) * (size_t)std::max<long long>(nrrq, 1) * (5 * hd + 6 * nbd + 4 + 3 * (2 * nq + 3) + 2) +
                        8192);
  if (rc) return rc;
  A2->reset();
  R.JD = A2->take<double>((size_t)std::max<long long>(nrrq, 1) * 4 * hd);
  R.RS = A2->take<double>((size_t)std::max<long long>(nrrq, 1) * hd);
  R.line = A2->take<double>((size_t)std::max<long long>(nrrq, 1) * (6 * nbd + 4));
  R.edge = A2->take<double>((size_t)std::max<long long>(nrrq, 1) * 3 * (2 * nq + 3));
  R.pair = A2->take<int2>((size_t)std::max<long long>(nrrq, 1));
  R.side = A2->take<signed char>((size_t)std::max<long long>(nrrq, 1));
  O = OutCOO{};
  O.vs = J.vs; O.vd = J.vd; O.omega = J.omega; O.subtract_naive = J.subtract_naive;
  /* the panel kernel's (cluster size, threads) shape, measured once per order
   * on the first call with enough panels: each shape on the first 512 panels,
   * one warm-up and the faster of two timed launches; every shape gives the same results
   * (the same arithmetic split over more or fewer CTAs), the fastest is kept
   * with the order's tables */
  std::lock_guard<std::recursive_mutex> tl(g_tab_mu); /* the tuner writes the order's tables */
  if (nrrq > 0 && g_autotune && !C->T.panel_cs && npan >= 256) {
    int cs[8], nt[8];
    const int ns = qol_panel_shapes(hd, nq, cs, nt, 8);
    int best = 0;
    if (ns > 1) {
      cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
      cudaError_t te = cudaEventCreate(&e0);
      if (te == cudaSuccess) te = cudaEventCreate(&e1);
      if (te == cudaSuccess) te = cudaEventCreate(&e2);
      float bms = 0.f;
      for (int i = 0; i < ns && te == cudaSuccess; ++i) { /* one warm-up, the faster of two timed launches */
        OrderTab Tt = T;
        Tt.panel_cs = cs[i];
        Tt.panel_nt = nt[i];
        const int np2 = std::min(npan, 512);
        float ms = 0.f, ms2 = 0.f;
        if ((te = qol_launch_rrq_panel(Tt, J.P, G, R, np2, J.chart, st)) != cudaSuccess ||
            (te = cudaEventRecord(e0, st)) != cudaSuccess ||
            (te = qol_launch_rrq_panel(Tt, J.P, G, R, np2, J.chart, st)) != cudaSuccess ||
            (te = cudaEventRecord(e1, st)) != cudaSuccess ||
            (te = qol_launch_rrq_panel(Tt, J.P, G, R, np2, J.chart, st)) != cudaSuccess ||
            (te = cudaEventRecord(e2, st)) != cudaSuccess || (te = cudaEventSynchronize(e2)) != cudaSuccess ||
            (te = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess ||
            (te = cudaEventElapsedTime(&ms2, e1, e2)) != cudaSuccess)
          break;
        ms = std::min(ms, ms2);
        if (i == 0 || ms < bms) { best = i; bms = ms; }
      }
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
      if (e2) cudaEventDestroy(e2);
      CK(te);
    }
    if (ns > 0) {
      C->T.panel_cs = T.panel_cs = cs[best];
      C->T.panel_nt = T.panel_nt = nt[best];
    }
  }
  return 0;
}

int PipeRun::launches(bool direct_done) {
  int rc = 0;
  /* one pass over all panels, or (host entry) panel chunks whose every phase
   * runs before the next chunk's, so that chunk c's values are final early
   * and leave the GPU while later chunks compute */
  const bool chunked = J.chunk_pan != nullptr;
  if (!chunked) {
    if (!direct_done) {
      rec(2);
      CK(qol_launch_direct(T, J.P, J.Q, W, G, O, npan, st));
      CK(qol_launch_direct_cut(T, J.P, J.Q, W, G, O, npan, st));
    }
    rec(3);
    if (nrrq > 0) CK(qol_launch_rrq_panel(T, J.P, G, R, npan, J.chart, st));
  }
  if (nrrq > 0) CK(qol_launch_rrq_pairs(T, J.Q, G, R, npan, st));
  const int nch = chunked ? (int)J.chunk_pan->size() - 1 : 1;
  cudaEvent_t fork = nullptr, join = nullptr;
  if (chunked && nch > 1) { /* a chunk's kernels fill the SMs the other's tail leaves idle */
    if ((rc = aux_stream(&st2))) return rc;
    CK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    CK(cudaEventRecord(fork, st));
    CK(cudaStreamWaitEvent(st2, fork, 0));
  }
  for (int c = 0; c < nch; ++c) {
    const long long a = chunked ? (*J.chunk_pan)[c] : 0, b = chunked ? (*J.chunk_pan)[c + 1] : npan;
    const int si = (c & 1) && st2 != st ? 1 : 0;
    const cudaStream_t sc = si ? st2 : st;
    R.plo = (int)a; R.phi = (int)b;
    R.glo = chunked ? off_h[a] : 0;
    R.ghi = chunked ? off_h[b] : nrrq;
    if (chunked && b > a) {
      rec(2, si);
      CK(qol_launch_direct(T, J.P, J.Q, W, G, O, (int)(b - a), sc, (int)a));
      CK(qol_launch_direct_cut(T, J.P, J.Q, W, G, O, (int)(b - a), sc, (int)a));
      rec(3, si);
      if (R.ghi > R.glo) CK(qol_launch_rrq_panel(T, J.P, G, R, (int)(b - a), J.chart, sc));
    }
    if (R.ghi > R.glo) {
      rec(4, si);
      CK(qol_launch_rrq_ssq(T, J.Q, G, R, sc));
      rec(5, si);
      CK(qol_launch_rrq_geom(T, J.Q, G, R, J.exterior, sc));
      rec(6, si);
      CK(qol_launch_rrq_moments(T, J.Q, G, R, sc));
      rec(7, si);
      CK(qol_launch_rrq_apply(T, J.P, J.Q, G, R, O, sc));
    }
    rec(-1, si);
    if (J.after_chunk) J.after_chunk(c, sc);
  }
  if (join) { /* the caller's stream waits for the second one */
    CK(cudaEventRecord(join, st2));
    CK(cudaStreamWaitEvent(st, join, 0));
    cudaEventDestroy(fork);
    cudaEventDestroy(join);
  }
  rec(8);
  if (J.si) CK(qol_launch_coo_index(T, J.Q, J.si, J.sj, npan, st));
  rec(-1);
  return 0;
}

/* the back stage as a CUDA graph (device entry, one pass, no per-phase
 * timing, FP64 level sums, a created stream): replays the stream's graph when
 * every launch argument is the one it was captured with, else captures the
 * launches and keeps the graph; false when that is not possible here (the
 * launches then run directly) */
bool PipeRun::back_graph(bool direct_done) {
  if (!graph || !g_graphs_on.load() || J.chunk_pan || tm.on || T.sum_fp32 || st == nullptr) return false;
  R.plo = 0; R.phi = npan; R.glo = 0; R.ghi = nrrq; /* the one pass's ranges, as launches() sets them */
  BackKey k;
  std::memset(&k, 0, sizeof k);
  std::memcpy(&k.T, &T, sizeof T);
  std::memcpy(&k.P, &J.P, sizeof J.P);
  std::memcpy(&k.Q, &J.Q, sizeof J.Q);
  std::memcpy(&k.W, &W, sizeof W);
  std::memcpy(&k.G, &G, sizeof G);
  std::memcpy(&k.R, &R, sizeof R);
  k.O.vs = O.vs; k.O.vd = O.vd; k.O.omega = O.omega; k.O.subtract_naive = O.subtract_naive;
  k.chart = J.chart; k.si = J.si; k.sj = J.sj; k.nrrq = nrrq;
  k.npan = npan; k.exterior = J.exterior; k.direct_done = direct_done;
  if (graph->exec && std::memcmp(&graph->key, &k, sizeof k) == 0) {
    if (cudaGraphLaunch(graph->exec, st) == cudaSuccess) {
      ++g_graph_replays;
      return true;
    }
    cudaGetLastError();
    graph->drop();
    return false;
  }
  graph->drop();
  if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const int lrc = launches(direct_done);
  cudaGraph_t gr = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(st, &gr);
  cudaGraphExec_t ex = nullptr;
  bool ok = lrc == 0 && ce == cudaSuccess && gr && cudaGraphInstantiate(&ex, gr, 0) == cudaSuccess;
  if (gr) cudaGraphDestroy(gr);
  if (ok && cudaGraphLaunch(ex, st) != cudaSuccess) ok = false;
  if (!ok) {
    if (ex) cudaGraphExecDestroy(ex);
    cudaGetLastError();
    return false;
  }
  graph->exec = ex;
  std::memcpy(&graph->key, &k, sizeof k);
  ++g_graph_captures;
  return true;
}

int PipeRun::back(long long* hist_out, std::vector<int>* grp_out, int* cnt_out, bool direct_done) {
  int rc = 0;
  if (!back_graph(direct_done) && (rc = launches(direct_done))) return rc;
  if (T.sum_fp32) { /* the FP32 level-sum kernel's waits are bounded: a timeout is reported here */
    unsigned werr = 0;
    CK(qol_wait_error(&werr, st));
    if (werr) return fail(QOL_ERR_CUDA, "FP32 level sums: a wait on the tensor cores timed out");
  }
  if (hist_out || grp_out || cnt_out || tm.on) {
    CK(cudaStreamSynchronize(st));
  }
  if (hist_out || cnt_out) {
    std::vector<int> cnt((size_t)npan * 8);
    CK(cudaMemcpy(cnt.data(), G.cnt, sizeof(int) * cnt.size(), cudaMemcpyDeviceToHost));
    if (hist_out) {
      for (int i = 0; i < 6; ++i) hist_out[i] = 0;
      for (int p = 0; p < npan; ++p) {
        for (int l = 1; l <= 5; ++l) hist_out[l] += cnt[(size_t)p * 8 + l];
        hist_out[0] += cnt[(size_t)p * 8 + QOL_LV_CUT]; /* adaptive cuts */
      }
    }
    if (cnt_out) for (int l = 0; l < 8; ++l) cnt_out[l] = cnt[l];
  }
  if (grp_out) {
    grp_out->resize(ntcx);
    CK(cudaMemcpy(grp_out->data(), G.grp, sizeof(int) * ntcx, cudaMemcpyDeviceToHost));
  }
  finish_timing(tm, timeinfo);
  return 0;
}

int run_pipeline(const Job& J, cudaStream_t st, double* timeinfo, long long* hist_out, std::vector<int>* grp_out,
                 int* cnt_out, Arena* a1 = &g_arena, Arena* a2 = &g_arena2, BackGraph* graph = nullptr) {
  PipeRun P(J, st, timeinfo, a1, a2);
  P.graph = graph;
  int rc = P.front();
  if (rc) return rc;
  return P.back(hist_out, grp_out, cnt_out, false);
}

/* the device entry's workspace per (device, stream): calls on one stream share
 * it and are ordered by its lock; calls on different streams run concurrently */
struct StreamCtx {
  std::mutex mu;
  Arena a1, a2;
  BackGraph graph; /* its back stage, captured over a1 and a2 */
};
std::mutex g_ctx_mu;
std::map<std::pair<int, cudaStream_t>, std::unique_ptr<StreamCtx>> g_ctx;
StreamCtx* stream_ctx(cudaStream_t st) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> g(g_ctx_mu);
  std::unique_ptr<StreamCtx>& c = g_ctx[std::make_pair(dev, st)];
  if (!c) c.reset(new StreamCtx());
  return c.get();
}

/* ---------------- patch-level handles ---------------- */
struct Slot {
  bool live = false;
  long long generation = 1, npols = 0, korder = 0, order = 0, nlevel = 0;
  double dist = 0.0;
  std::vector<double> sx, rts, rps;
};
Slot g_slots[QOL_MAX_HANDLES];

bool decode_handle(long long h, int* slot) {
  if (h <= 0) return false;
  long long s = (h - 1) % QOL_MAX_HANDLES + 1;
  long long gen = (h - s) / QOL_MAX_HANDLES;
  *slot = (int)(s - 1);
  return g_slots[s - 1].live && g_slots[s - 1].generation == gen;
}

template <class T>
int dcopy_in(T** d, const T* h, size_t n, cudaStream_t st) {
  T* p = g_arena.take<T>(std::max<size_t>(n, 1));
  if (n) CK(cudaMemcpyAsync(p, h, sizeof(T) * n, cudaMemcpyHostToDevice, st));
  *d = p;
  return 0;
}

int tables_match(int nquad, int korder, const double* tgl, const double* wgl, const double* umatr) {
  int hd = (korder + 1) * (korder + 2) / 2;
  std::vector<double> t(nquad), w(nquad), um((size_t)hd * hd);
  qolh::gauss(nquad, t.data(), w.data(), nullptr);
  qolh::koorn_umatr(korder, um.data(), nullptr);
  for (int i = 0; i < nquad; ++i)
    if (std::fabs(t[i] - tgl[i]) > 1e-13 || std::fabs(w[i] - wgl[i]) > 1e-13) return 0;
  if (umatr)
    for (size_t i = 0; i < um.size(); ++i)
      if (std::fabs(um[i] - umatr[i]) > 1e-9 * (1.0 + std::fabs(um[i]))) return 0;
  return 1;
}

/* ---------------- host-buffer output: staged, overlapped copies ---------------- */
/* The host-pointer entry point runs the pipeline over panel chunks; each
 * chunk's COO values leave the GPU on a copy stream while the next chunk
 * computes, through a ring of pinned staging buffers that host threads empty
 * into the caller's arrays.  The COO indices are a layout function of
 * tcxrow/tcxi (k_coo_index computes the same), so that entry point fills them
 * on host threads while the GPU works instead of moving them over the link. */
/* small pieces: the ring (24 x 2 MiB) can stay in the host's last-level cache
 * between the DMA write and the copy out */
constexpr size_t kStageBytes = (size_t)2 << 20;
/* wall-clock milestones of the last host-pointer call, ms from its start:
 * inputs queued, all chunks queued, value copies queued, values landed,
 * every host task done, end, indices filled */
double g_host_ms[7] = {0, 0, 0, 0, 0, 0, 0};
inline double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}
constexpr int kNStage = 24;

struct StageRing {
  void* buf[kNStage] = {};
  cudaEvent_t ev[kNStage] = {};
  cudaStream_t cs = nullptr;
  bool ok = false;
  int init() {
    if (ok) return 0;
    for (int b = 0; b < kNStage; ++b) {
      CK(cudaMallocHost(&buf[b], kStageBytes));
      CK(cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming));
    }
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    ok = true;
    return 0;
  }
} g_ring;

/* host threads draining a task queue in order (the index fills are queued
 * first and run while the GPU computes, then the value pages are mapped,
 * the staging copies follow); finish() runs what is queued and joins */
class Workers {
 public:
  explicit Workers(int n) {
    for (int i = 0; i < n; ++i) th_.emplace_back([this] { loop(); });
  }
  ~Workers() { finish(); }
  void submit(std::function<void()> f) {
    {
      std::lock_guard<std::mutex> g(mu_);
      q_.push_back(std::move(f));
    }
    cv_.notify_one();
  }
  void finish() {
    {
      std::lock_guard<std::mutex> g(mu_);
      if (closed_) return;
      closed_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }

 private:
  void loop() {
    for (;;) {
      std::function<void()> f;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return closed_ || !q_.empty(); });
        if (q_.empty()) return;
        f = std::move(q_.front());
        q_.pop_front();
      }
      f();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::function<void()>> q_;
  bool closed_ = false;
};

/* staging buffers free for a new device-to-host copy */
class FreeList {
 public:
  FreeList() { for (int b = 0; b < kNStage; ++b) free_.push_back(b); }
  int take() {
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return !free_.empty(); });
    int b = free_.back();
    free_.pop_back();
    return b;
  }
  void give(int b) {
    {
      std::lock_guard<std::mutex> g(mu_);
      free_.push_back(b);
    }
    cv_.notify_one();
  }

 private:
  std::mutex mu_;
  std::condition_variable cv_;
  std::vector<int> free_;
};

/* chunks recorded on the compute stream so far (the copy side waits on it
 * before it waits on a chunk's event, which must already be recorded) */
class Progress {
 public:
  void set(int n) {
    {
      std::lock_guard<std::mutex> g(mu_);
      n_ = n;
    }
    cv_.notify_all();
  }
  void abort() {
    {
      std::lock_guard<std::mutex> g(mu_);
      abort_ = true;
    }
    cv_.notify_all();
  }
  bool wait(int c) { /* false when aborted first */
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return abort_ || n_ > c; });
    return n_ > c;
  }

 private:
  std::mutex mu_;
  std::condition_variable cv_;
  int n_ = 0;
  bool abort_ = false;
};

/* map the pages of [p, p+n) writable before the values arrive (the kernel
 * zeroes fresh pages on first write; done here it overlaps the GPU work).
 * Advisory: contents are unchanged and a kernel without it is skipped. */
#ifndef MADV_POPULATE_WRITE
#define MADV_POPULATE_WRITE 23
#endif
void prefault(void* p, size_t n) {
  static const size_t pg = (size_t)sysconf(_SC_PAGESIZE);
  const size_t a = ((size_t)p + pg - 1) & ~(pg - 1), b = ((size_t)p + n) & ~(pg - 1);
  if (b > a) madvise((void*)a, b - a, MADV_POPULATE_WRITE);
}

/* The output arrays are written once and not read back here: streaming
 * (non-temporal) stores skip the read of each destination line that an
 * ordinary store makes, which is a third of the host memory traffic. */
void copy_out(void* dst, const void* src, size_t n /* a multiple of 8 */) {
  char* d = (char*)dst;
  const char* s = (const char*)src;
  if (n >= 8 && ((uintptr_t)d & 15)) {
    long long v;
    std::memcpy(&v, s, 8);
    _mm_stream_si64((long long*)d, v);
    d += 8; s += 8; n -= 8;
  }
  for (; n >= 64; n -= 64, d += 64, s += 64) {
    const __m128i a = _mm_loadu_si128((const __m128i*)s), b = _mm_loadu_si128((const __m128i*)(s + 16));
    const __m128i c = _mm_loadu_si128((const __m128i*)(s + 32)), e = _mm_loadu_si128((const __m128i*)(s + 48));
    _mm_stream_si128((__m128i*)d, a);
    _mm_stream_si128((__m128i*)(d + 16), b);
    _mm_stream_si128((__m128i*)(d + 32), c);
    _mm_stream_si128((__m128i*)(d + 48), e);
  }
  for (; n >= 8; n -= 8, d += 8, s += 8) {
    long long v;
    std::memcpy(&v, s, 8);
    _mm_stream_si64((long long*)d, v);
  }
  _mm_sfence();
}

/* COO indices of panels [k0, k1) (reference order (tcxi(k)-1) hd + (j-1) m + i) */
void fill_indices(long long k0, long long k1, int hd, const long long* tcxi, const long long* tcxrow, long long* si,
                  long long* sj) {
  for (long long k = k0; k < k1; ++k) {
    const long long p0 = tcxi[k] - 1, m = tcxi[k + 1] - tcxi[k];
    long long* oi = si + (size_t)p0 * hd;
    long long* oj = sj + (size_t)p0 * hd;
    const long long* row = tcxrow + p0;
    for (int j = 0; j < hd; ++j) {
      const long long col = k * hd + j + 1;
      long long* a = oi + (size_t)j * m;
      long long* b = oj + (size_t)j * m;
      for (long long i = 0; i < m; ++i) { _mm_stream_si64(a + i, row[i]); _mm_stream_si64(b + i, col); }
    }
  }
  _mm_sfence();
}

} // namespace

/* ===================================================================== */
/* C ABI                                                                 */
/* ===================================================================== */
extern "C" {

const char* qol_last_error(void) { return g_err.c_str(); }

int qol_kernel_times(int enable, double* ms, qol_int* calls) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (ms) for (int i = 0; i < QOL_NPHASE; ++i) ms[i] = g_ktime[i];
  if (calls) *calls = g_kcalls;
  if (enable >= 0) {
    g_ktime_on = enable;
    for (int i = 0; i < QOL_NPHASE; ++i) g_ktime[i] = 0.0;
    g_kcalls = 0;
  }
  return 0;
}
int qol_version(void) { return 100; }

int qol_set_autotune(int on) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (on != 0 && on != 1) return fail(QOL_ERR_ARG, "autotune must be 0 or 1");
  g_autotune = on;
  return 0;
}

int qol_panel_shape(qol_int nterms, qol_int orderff, qol_int nquad, int* cs, int* nt) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  std::lock_guard<std::recursive_mutex> tl(g_tab_mu);
  if (!cs || !nt) return fail(QOL_ERR_ARG, "null argument");
  *cs = 0; *nt = 0;
  const long long key = nterms + 100LL * orderff + 10000LL * nquad;
  auto it = g_orders.find(key);
  if (it != g_orders.end()) { *cs = it->second->T.panel_cs; *nt = it->second->T.panel_nt; }
  return 0;
}

int qol_set_sum_precision(int mode) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (mode != 0 && mode != 1) return fail(QOL_ERR_ARG, "sum precision must be 0 (FP64) or 1 (FP32 level sums)");
  g_sum_precision = mode;
  return 0;
}

/* ---------------- learned level selector (no reference counterpart) ---------------- */
static_assert(QOL_SELECTOR_NW == QOL_SEL_NW, "selector weight count");
/* features and plain-walk levels of every near pair (the training data) */
int qol_selector_features(qol_int npan, qol_int nterms, qol_int nquad, const double* sx, const double* snx,
                          const double* sw, const double* rts, const double* rps, qol_int ntcx, const double* tcx,
                          const qol_int* tcxrow, const qol_int* tcxi, qol_int orderff, double distff, float* feat,
                          signed char* level) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (!sx || !snx || !sw || !rts || !rps || !tcx || !tcxrow || !tcxi || !feat || !level || npan <= 0 || ntcx < 0)
    return fail(QOL_ERR_ARG, "qol_selector_features: null argument or bad size");
  if (tcxi[0] != 1 || tcxi[npan] != ntcx + 1) return fail(QOL_ERR_LAYOUT, "tcxi must be one-based and cover tcx");
  OrderCache* C = nullptr;
  int rc = order_tables((int)nterms, (int)orderff, (int)nquad, &C);
  if (rc) return rc;
  OrderTab T = C->T;
  T.dist = distff;
  const int hd = T.hd;
  const long long nsrc = (long long)npan * hd;
  if ((rc = ensure_device())) return rc;
  cudaStream_t st = g_stream;
  std::vector<void*> bufs;
  auto dal = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) return nullptr;
    bufs.push_back(p);
    return p;
  };
  auto done = [&](int r) {
    for (void* p : bufs) cudaFree(p);
    return r;
  };
  double* dsx = (double*)dal(sizeof(double) * 3 * nsrc);
  double* dsnx = (double*)dal(sizeof(double) * 3 * nsrc);
  double* dsw = (double*)dal(sizeof(double) * nsrc);
  double* drts = (double*)dal(sizeof(double) * 3 * nsrc);
  double* drps = (double*)dal(sizeof(double) * 3 * nsrc);
  double* dtcx = (double*)dal(sizeof(double) * 3 * std::max<qol_int>(ntcx, 1));
  long long* drow = (long long*)dal(sizeof(long long) * std::max<qol_int>(ntcx, 1));
  long long* dxi = (long long*)dal(sizeof(long long) * (npan + 1));
  float* dfeat = (float*)dal(sizeof(float) * QOL_SEL_F * std::max<qol_int>(ntcx, 1));
  LevelWS W{};
  for (int l = 0; l < 4; ++l) {
    W.node[l] = (double*)dal(sizeof(double) * (size_t)npan * T.n[l] * 7);
    W.sub[l] = (double*)dal(sizeof(double) * (size_t)npan * T.nsub[l] * 4);
  }
  PairWS G{};
  G.level = (signed char*)dal(std::max<qol_int>(ntcx, 1));
  G.grp = (int*)dal(sizeof(int) * std::max<qol_int>(ntcx, 1));
  G.cnt = (int*)dal(sizeof(int) * (size_t)npan * 8);
  G.off = (int*)dal(sizeof(int) * (size_t)npan * 8);
  for (void* p : bufs)
    if (!p) return done(fail(QOL_ERR_CUDA, "qol_selector_features: device allocation failed"));
  auto ck = [&](cudaError_t e) { return e == cudaSuccess ? 0 : fail(QOL_ERR_CUDA, "%s", cudaGetErrorString(e)); };
  if ((rc = ck(cudaMemcpyAsync(dsx, sx, sizeof(double) * 3 * nsrc, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemcpyAsync(dsnx, snx, sizeof(double) * 3 * nsrc, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemcpyAsync(dsw, sw, sizeof(double) * nsrc, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemcpyAsync(drts, rts, sizeof(double) * 3 * nsrc, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemcpyAsync(drps, rps, sizeof(double) * 3 * nsrc, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemcpyAsync(dtcx, tcx, sizeof(double) * 3 * ntcx, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemcpyAsync(drow, tcxrow, sizeof(long long) * ntcx, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemcpyAsync(dxi, tcxi, sizeof(long long) * (npan + 1), cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemsetAsync(G.cnt, 0, sizeof(int) * (size_t)npan * 8, st))))
    return done(rc);
  const PanelIn P{dsx, dsnx, dsw, drts, drps};
  const PairIn Q{dtcx, drow, dxi};
  if ((rc = ck(qol_launch_levels(T, P, W, (int)npan, st))) || (rc = ck(qol_launch_classify(T, Q, W, G, (int)npan, st))) ||
      (rc = ck(qol_launch_sel_features(hd, P, Q, (int)npan, dfeat, st))) ||
      (rc = ck(cudaMemcpyAsync(feat, dfeat, sizeof(float) * QOL_SEL_F * ntcx, cudaMemcpyDeviceToHost, st))) ||
      (rc = ck(cudaMemcpyAsync(level, G.level, ntcx, cudaMemcpyDeviceToHost, st))) ||
      (rc = ck(cudaStreamSynchronize(st))))
    return done(rc);
  return done(0);
}

namespace {
/* device copies of a training set and the optimiser state */
struct SelTrain {
  float *feat = nullptr, *w = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *slot = nullptr;
  signed char* lab = nullptr;
  int* idx = nullptr;
  double* sloss = nullptr;
  ~SelTrain() {
    for (void* p : {(void*)feat, (void*)w, (void*)m, (void*)v, (void*)grad, (void*)slot, (void*)lab, (void*)idx,
                    (void*)sloss})
      if (p) cudaFree(p);
  }
};
int sel_check(qol_int n, const float* feat, const signed char* label, const float* w) {
  if (n <= 0 || !feat || !label || !w) return fail(QOL_ERR_ARG, "selector: null argument or empty set");
  for (qol_int i = 0; i < n; ++i)
    if (label[i] < 0 || label[i] >= QOL_SEL_C) return fail(QOL_ERR_ARG, "selector: labels must be 0..%d", QOL_SEL_C - 1);
  return 0;
}
} // namespace

/* mean cross-entropy gradient and loss over n samples (no update) */
int qol_selector_grad(qol_int n, const float* feat, const signed char* label, const float* w, float* grad,
                      double* loss) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  int rc = sel_check(n, feat, label, w);
  if (rc) return rc;
  if (!grad || !loss) return fail(QOL_ERR_ARG, "qol_selector_grad: null argument");
  if ((rc = ensure_device())) return rc;
  cudaStream_t st = g_stream;
  const int nslot = (int)((n + 255) / 256);
  SelTrain D;
  std::vector<int> idx(n);
  for (qol_int i = 0; i < n; ++i) idx[i] = (int)i;
  auto ck = [&](cudaError_t e) { return e == cudaSuccess ? 0 : fail(QOL_ERR_CUDA, "%s", cudaGetErrorString(e)); };
  if ((rc = ck(cudaMalloc(&D.feat, sizeof(float) * QOL_SEL_F * n))) || (rc = ck(cudaMalloc(&D.lab, n))) ||
      (rc = ck(cudaMalloc(&D.idx, sizeof(int) * n))) || (rc = ck(cudaMalloc(&D.w, sizeof(float) * QOL_SEL_NW))) ||
      (rc = ck(cudaMalloc(&D.grad, sizeof(float) * QOL_SEL_NW))) ||
      (rc = ck(cudaMalloc(&D.slot, sizeof(float) * QOL_SEL_NW * (size_t)nslot))) ||
      (rc = ck(cudaMalloc(&D.sloss, sizeof(double) * nslot))))
    return rc;
  std::vector<double> sl(nslot);
  if ((rc = ck(cudaMemcpyAsync(D.feat, feat, sizeof(float) * QOL_SEL_F * n, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemcpyAsync(D.lab, label, n, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemcpyAsync(D.idx, idx.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemcpyAsync(D.w, w, sizeof(float) * QOL_SEL_NW, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(qol_launch_sel_grad(D.feat, D.lab, D.idx, 0, n, D.w, D.slot, D.sloss, nslot, st))) ||
      (rc = ck(qol_launch_sel_update(D.slot, nslot, 1.0f / (float)n, D.grad, D.w, nullptr, nullptr, 0.0f, 1, st))) ||
      (rc = ck(cudaMemcpyAsync(grad, D.grad, sizeof(float) * QOL_SEL_NW, cudaMemcpyDeviceToHost, st))) ||
      (rc = ck(cudaMemcpyAsync(sl.data(), D.sloss, sizeof(double) * nslot, cudaMemcpyDeviceToHost, st))) ||
      (rc = ck(cudaStreamSynchronize(st))))
    return rc;
  double acc = 0.0;
  for (double v : sl) acc += v;
  *loss = acc / (double)n;
  return 0;
}

/* Adam on the mean cross-entropy: epochs over a seeded shuffle, batches of
 * `batch` samples (a multiple of 256); w holds the initial weights and
 * receives the trained ones; loss[e] = mean loss seen during epoch e */
int qol_selector_train(qol_int n, const float* feat, const signed char* label, qol_int epochs, qol_int batch, double lr,
                       unsigned long long seed, float* w, double* loss) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  int rc = sel_check(n, feat, label, w);
  if (rc) return rc;
  if (epochs <= 0 || batch < 256 || batch % 256 || !(lr > 0.0) || !loss)
    return fail(QOL_ERR_ARG, "qol_selector_train: epochs > 0, batch a positive multiple of 256, lr > 0");
  if ((rc = ensure_device())) return rc;
  cudaStream_t st = g_stream;
  const int nslot = (int)(batch / 256);
  SelTrain D;
  auto ck = [&](cudaError_t e) { return e == cudaSuccess ? 0 : fail(QOL_ERR_CUDA, "%s", cudaGetErrorString(e)); };
  if ((rc = ck(cudaMalloc(&D.feat, sizeof(float) * QOL_SEL_F * n))) || (rc = ck(cudaMalloc(&D.lab, n))) ||
      (rc = ck(cudaMalloc(&D.idx, sizeof(int) * n))) || (rc = ck(cudaMalloc(&D.w, sizeof(float) * QOL_SEL_NW))) ||
      (rc = ck(cudaMalloc(&D.m, sizeof(float) * QOL_SEL_NW))) ||
      (rc = ck(cudaMalloc(&D.v, sizeof(float) * QOL_SEL_NW))) ||
      (rc = ck(cudaMalloc(&D.slot, sizeof(float) * QOL_SEL_NW * (size_t)nslot))) ||
      (rc = ck(cudaMalloc(&D.sloss, sizeof(double) * nslot))))
    return rc;
  if ((rc = ck(cudaMemcpyAsync(D.feat, feat, sizeof(float) * QOL_SEL_F * n, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemcpyAsync(D.lab, label, n, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemcpyAsync(D.w, w, sizeof(float) * QOL_SEL_NW, cudaMemcpyHostToDevice, st))) ||
      (rc = ck(cudaMemsetAsync(D.m, 0, sizeof(float) * QOL_SEL_NW, st))) ||
      (rc = ck(cudaMemsetAsync(D.v, 0, sizeof(float) * QOL_SEL_NW, st))))
    return rc;
  std::vector<int> idx(n);
  for (qol_int i = 0; i < n; ++i) idx[i] = (int)i;
  unsigned long long sm = seed;
  auto next = [&]() { /* splitmix64 */
    unsigned long long z = (sm += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  std::vector<double> sl(nslot);
  int it = 0;
  for (qol_int e = 0; e < epochs; ++e) {
    for (qol_int i = n - 1; i > 0; --i) std::swap(idx[i], idx[(qol_int)(next() % (unsigned long long)(i + 1))]);
    if ((rc = ck(cudaMemcpyAsync(D.idx, idx.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st)))) return rc;
    double eloss = 0.0;
    for (qol_int b0 = 0; b0 < n; b0 += batch) {
      const qol_int b1 = std::min<qol_int>(n, b0 + batch);
      const int ns = (int)((b1 - b0 + 255) / 256);
      if ((rc = ck(qol_launch_sel_grad(D.feat, D.lab, D.idx, b0, b1, D.w, D.slot, D.sloss, ns, st))) ||
          (rc = ck(qol_launch_sel_update(D.slot, ns, 1.0f / (float)(b1 - b0), nullptr, D.w, D.m, D.v, (float)lr, ++it,
                                         st))) ||
          (rc = ck(cudaMemcpyAsync(sl.data(), D.sloss, sizeof(double) * ns, cudaMemcpyDeviceToHost, st))) ||
          (rc = ck(cudaStreamSynchronize(st))))
        return rc;
      for (int q = 0; q < ns; ++q) eloss += sl[q];
    }
    loss[e] = eloss / (double)n;
  }
  if ((rc = ck(cudaMemcpy(w, D.w, sizeof(float) * QOL_SEL_NW, cudaMemcpyDeviceToHost)))) return rc;
  return 0;
}

/* mode 0: plain ball-test walk; mode 1: the learned selector with weights w
 * (FP32, used rounded to BF16), confidence threshold conf in (0, 1] and the
 * ball check; mode 2: the same with the two-level check at the tolerance of
 * qol_selector_set_tol */
int qol_selector_set(int mode, const float* w, double conf) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (mode == 0) { g_sel_mode = 0; return 0; }
  if ((mode != 1 && mode != 2) || !w || !(conf > 0.0 && conf <= 1.0))
    return fail(QOL_ERR_ARG, "qol_selector_set: mode 0, 1 or 2, weights and a confidence in (0, 1]");
  std::vector<float> wb(QOL_SEL_NW);
  for (int i = 0; i < QOL_SEL_NW; ++i) { /* round to nearest even BF16 */
    uint32_t u;
    std::memcpy(&u, &w[i], 4);
    if ((u & 0x7F800000u) != 0x7F800000u) u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
    else u &= 0xFFFF0000u;
    std::memcpy(&wb[i], &u, 4);
  }
  auto ck = [&](cudaError_t e) { return e == cudaSuccess ? 0 : fail(QOL_ERR_CUDA, "%s", cudaGetErrorString(e)); };
  int rc = 0;
  if (!g_sel_w && ((rc = ck(cudaMalloc(&g_sel_w, sizeof(float) * QOL_SEL_NW))) ||
                   (rc = ck(cudaMalloc(&g_sel_cnt, sizeof(unsigned long long) * 4))) ||
                   (rc = ck(cudaMemset(g_sel_cnt, 0, sizeof(unsigned long long) * 4)))))
    return rc;
  if ((rc = ck(cudaMemcpy(g_sel_w, wb.data(), sizeof(float) * QOL_SEL_NW, cudaMemcpyHostToDevice)))) return rc;
  g_sel_mode = mode;
  g_sel_conf = (float)conf;
  return 0;
}

/* patch refinement mode of the calls that follow: the reference test's iadap
 * (0 square levels, 1 adaptive tree walk, 3 plain levels); 2 or any other
 * value is refused (PR_SQUARE and PR_ADAPTIVE cannot be combined,
 * patch_refine_mod.f90:116-117) */
int qol_set_patch_refine(int iadap) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (iadap != 0 && iadap != 1 && iadap != 3)
    return fail(QOL_ERR_ARG, "qol_set_patch_refine: iadap 0 (square), 1 (adaptive) or 3 (plain levels)");
  g_refine = iadap;
  return 0;
}

/* the two-level check's tolerance on a row's error (single-layer rows over
 * the panel's diameter, double-layer rows as they are; 1-norm scale) */
int qol_selector_set_tol(double tol) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (!(tol > 0.0 && tol < 1.0)) return fail(QOL_ERR_ARG, "qol_selector_set_tol: tol in (0, 1)");
  g_sel_tol = tol;
  return 0;
}

/* labelling: level 1..4 puts every pair that the plain walk resolves by a
 * direct sum on that level in the calls that follow (RRQ pairs unchanged,
 * the selector off); 0 restores the walk */
int qol_selector_force_level(int level) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (level < 0 || level > 4) return fail(QOL_ERR_ARG, "qol_selector_force_level: level 0..4");
  g_force_level = level;
  return 0;
}

/* the selector's decisions since the last call: accepted, low confidence,
 * check failed (the last two went to the plain walk); resets them */
int qol_selector_stats(qol_int* counts3) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (!counts3) return fail(QOL_ERR_ARG, "null argument");
  unsigned long long c[4] = {};
  if (g_sel_cnt) {
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(c, g_sel_cnt, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemset(g_sel_cnt, 0, sizeof(c)) != cudaSuccess)
      return fail(QOL_ERR_CUDA, "selector counters");
  }
  for (int i = 0; i < 3; ++i) counts3[i] = (qol_int)c[i];
  return 0;
}

int qol_level_sizes(qol_int nterms, qol_int orderff, qol_int* n4, qol_int* nsub4) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  qolh::RefElem R;
  try {
    qolh::build_ref((int)nterms - 1, (int)orderff, 4, g_refine == 0, R);
  } catch (const std::exception& e) {
    return fail(QOL_ERR_ORDER, "reference element: %s", e.what());
  }
  for (int l = 0; l < 4; ++l) { n4[l] = R.lev[l].n; nsub4[l] = R.lev[l].nsub; }
  return 0;
}

/* the reference element's level `level` (0..3) for the current refinement
 * mode: uv (2 x n), wt (n), suboff (nsub + 1), subtyp (nsub); with uv == NULL
 * only the sizes (diagnostics: tests compare the tables with an independent
 * restatement) */
int qol_ref_level_table(qol_int nterms, qol_int orderff, qol_int level, qol_int* n, qol_int* nsub, double* uv,
                        double* wt, qol_int* suboff, qol_int* subtyp) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (!n || !nsub || level < 0 || level > 3) return fail(QOL_ERR_ARG, "qol_ref_level_table: bad arguments");
  qolh::RefElem R;
  try {
    qolh::build_ref((int)nterms - 1, (int)orderff, 4, g_refine == 0, R);
  } catch (const std::exception& e) {
    return fail(QOL_ERR_ORDER, "reference element: %s", e.what());
  }
  const qolh::RefLevel& L = R.lev[level];
  *n = L.n; *nsub = L.nsub;
  if (!uv) return 0;
  if (!wt || !suboff || !subtyp) return fail(QOL_ERR_ARG, "qol_ref_level_table: null output");
  std::copy(L.uv.begin(), L.uv.end(), uv);
  std::copy(L.wt.begin(), L.wt.end(), wt);
  for (size_t i = 0; i < L.suboff.size(); ++i) suboff[i] = L.suboff[i];
  for (size_t i = 0; i < L.subtyp.size(); ++i) subtyp[i] = L.subtyp[i];
  return 0;
}

int qol_probe_fp64_peak(double* tflops) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  int rc = ensure_device();
  if (rc) return rc;
  int dev = 0, nsm = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  double* out = nullptr;
  const int blocks = nsm * 8, iters = 1 << 16;
  CK(cudaMalloc(&out, sizeof(double) * blocks));
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a)); CK(cudaEventCreate(&b));
  double best = 0.0;
  for (int rep = 0; rep < 6; ++rep) {
    CK(cudaEventRecord(a, g_stream));
    CK(qol_launch_fp64_peak(out, blocks, iters, g_stream));
    CK(cudaEventRecord(b, g_stream));
    CK(cudaEventSynchronize(b));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, a, b));
    double fl = 2.0 * 8.0 * (double)iters * blocks * 256.0;
    if (rep > 0) best = std::max(best, fl / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(a); cudaEventDestroy(b); cudaFree(out);
  *tflops = best;
  return 0;
}

int qol_simplex_precomp(qol_int nquad, qol_int korder, qol_int kpols, double* tgl, double* wgl, double* Dgl,
                        double* w_bclag, double* Legmat, double* umatr, double* vmatr) {
  if (nquad < 1 || korder < 0 || korder > 20 || !tgl || !wgl || !Dgl || !w_bclag || !Legmat || !umatr || !vmatr)
    return fail(QOL_ERR_ARG, "qol_simplex_precomp: bad arguments");
  if (kpols != (korder + 1) * (korder + 2) / 2) return fail(QOL_ERR_NPOLS, "kpols mismatch");
  qolh::gauss((int)nquad, tgl, wgl, Dgl);
  qolh::bary_weights((int)nquad, tgl, w_bclag);
  qolh::legendre_vals2coefs((int)nquad, tgl, wgl, Legmat);
  qolh::koorn_umatr((int)korder, umatr, vmatr);
  return 0;
}

int qol_build_patch_levels(qol_int korder, qol_int npols, const double* sx, const double* rts, const double* rps,
                           qol_int order, double dist, qol_int nlevel, qol_int* lv, qol_int* ier) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (lv) *lv = 0;
  if (!sx || !rts || !rps || !lv || !ier) return fail(QOL_ERR_ARG, "null argument");
  if (npols != (korder + 1) * (korder + 2) / 2) { *ier = 3; return fail(QOL_ERR_NPOLS, "npols mismatch"); }
  if (nlevel != 4) { *ier = 1; return fail(QOL_ERR_ORDER, "only nlevel = 4 (the reference's NLEVEL) is supported"); }
  for (int s = 0; s < QOL_MAX_HANDLES; ++s) {
    Slot& S = g_slots[s];
    if (S.live) continue;
    S.live = true; S.npols = npols; S.korder = korder; S.order = order; S.nlevel = nlevel; S.dist = dist;
    S.sx.assign(sx, sx + 3 * npols); S.rts.assign(rts, rts + 3 * npols); S.rps.assign(rps, rps + 3 * npols);
    *lv = S.generation * QOL_MAX_HANDLES + (s + 1);
    *ier = 0;
    return 0;
  }
  *ier = 1;
  return fail(QOL_ERR_NOSLOT, "no free patch-level slot");
}

int qol_lap3dsdlpmat_levels(qol_int m, const double* tx, qol_int npols, qol_int lv, qol_int isimd, double* As,
                            double* Ad, qol_int* idxs, qol_int* ms, qol_int* ier) {
  (void)isimd;
  std::lock_guard<std::recursive_mutex> g(g_mu);
  int s;
  if (!ier || !ms) return fail(QOL_ERR_ARG, "null argument");
  if (!decode_handle(lv, &s)) { *ms = 0; *ier = 2; return fail(QOL_ERR_HANDLE, "bad handle"); }
  Slot& S = g_slots[s];
  if (npols != S.npols) { *ms = 0; *ier = 3; return fail(QOL_ERR_NPOLS, "npols mismatch"); }
  if (m < 0 || (m > 0 && (!tx || !As || !Ad || !idxs))) return fail(QOL_ERR_ARG, "bad arguments");
  int rc = ensure_device();
  if (rc) return rc;
  *ier = 0;
  if (m == 0) { *ms = 0; return 0; }
  const int nterms = (int)S.korder + 1;
  OrderCache* C = nullptr;
  rc = order_tables(nterms, (int)S.order, nterms + 2, &C);
  if (rc) return rc;
  /* inputs: one panel, the caller's targets; As/Ad copied in so that rows of
   * unresolved targets keep their values (intent(inout) in the reference) */
  cudaStream_t st = g_stream;
  size_t need = sizeof(double) * (size_t)(m * 3 + 9 * npols + 2 * m * npols + npols) + sizeof(long long) * (m + 4) +
                16 * 256;
  if ((rc = g_arena.reserve(need + (64 << 20)))) return rc;
  g_arena.reset();
  double *dsx, *drts, *drps, *dtx, *dAs, *dAd, *dsnx, *dsw;
  long long *drow, *dxi;
  std::vector<double> zeros(3 * npols, 0.0), ones(npols, 1.0);
  std::vector<long long> rows(m, 0), xi = {1, m + 1};
  if ((rc = dcopy_in(&dsx, S.sx.data(), 3 * npols, st)) || (rc = dcopy_in(&drts, S.rts.data(), 3 * npols, st)) ||
      (rc = dcopy_in(&drps, S.rps.data(), 3 * npols, st)) || (rc = dcopy_in(&dsnx, zeros.data(), 3 * npols, st)) ||
      (rc = dcopy_in(&dsw, ones.data(), npols, st)) || (rc = dcopy_in(&dtx, tx, 3 * m, st)) ||
      (rc = dcopy_in(&dAs, As, m * npols, st)) || (rc = dcopy_in(&dAd, Ad, m * npols, st)) ||
      (rc = dcopy_in(&drow, (const long long*)rows.data(), m, st)) || (rc = dcopy_in(&dxi, (const long long*)xi.data(), 2, st)))
    return rc;
  /* the pipeline's own arena use starts after these buffers: run levels +
   * classify + direct through a dedicated small pipeline */
  OrderTab T = C->T;
  T.dist = S.dist;
  LevelWS W{};
  for (int l = 0; l < 4; ++l) {
    W.node[l] = g_arena.take<double>((size_t)T.n[l] * 7);
    W.sub[l] = g_arena.take<double>((size_t)T.nsub[l] * 4);
  }
  PairWS G{};
  G.level = g_arena.take<signed char>(m);
  G.grp = g_arena.take<int>(m);
  G.cnt = g_arena.take<int>(8);
  G.off = g_arena.take<int>(8);
  CK(cudaMemsetAsync(G.cnt, 0, sizeof(int) * 8, st));
  CK(cudaMemsetAsync(G.off, 0, sizeof(int) * 8, st));
  PanelIn P{dsx, dsnx, dsw, drts, drps};
  PairIn Q{dtx, drow, dxi};
  OutCOO O{dAs, dAd, nullptr, 0};
  CK(qol_launch_levels(T, P, W, 1, st));
  CK(qol_launch_classify(T, Q, W, G, 1, st));
  CK(qol_launch_direct(T, P, Q, W, G, O, 1, st));
  CK(qol_launch_direct_cut(T, P, Q, W, G, O, 1, st));
  int cnt[8], off[8];
  std::vector<int> grp(m);
  CK(cudaMemcpyAsync(cnt, G.cnt, sizeof cnt, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(off, G.off, sizeof off, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(grp.data(), G.grp, sizeof(int) * m, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(As, dAs, sizeof(double) * m * npols, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(Ad, dAd, sizeof(double) * m * npols, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  *ms = cnt[T.nlevel + 1];
  for (int i = 0; i < cnt[T.nlevel + 1]; ++i) idxs[i] = grp[off[T.nlevel + 1] + i] + 1;
  return 0;
}

int qol_clear_patch_levels(qol_int lv, qol_int* ier) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  int s;
  if (!ier) return fail(QOL_ERR_ARG, "null argument");
  if (!decode_handle(lv, &s)) { *ier = 2; return fail(QOL_ERR_HANDLE, "bad handle"); }
  g_slots[s].live = false; g_slots[s].npols = 0; g_slots[s].generation += 1;
  g_slots[s].sx.clear(); g_slots[s].rts.clear(); g_slots[s].rps.clear();
  *ier = 0;
  return 0;
}

int qol_clear_patch_levels_all(qol_int* ier) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  for (int s = 0; s < QOL_MAX_HANDLES; ++s)
    if (g_slots[s].live) {
      g_slots[s].live = false; g_slots[s].npols = 0; g_slots[s].generation += 1;
    }
  if (ier) *ier = 0;
  return 0;
}

static int validate_near(qol_int npan, qol_int nterms, qol_int hdim, qol_int nsrc, qol_int ntcx, const qol_int* tcxi,
                         qol_int nnz) {
  if (npan < 0 || ntcx < 0 || nnz < 0) return fail(QOL_ERR_ARG, "negative size");
  if (hdim != nterms * (nterms + 1) / 2 || npan * hdim != nsrc)
    return fail(QOL_ERR_LAYOUT, "the panel order, hdim, npan, and nsrc are inconsistent");
  if (tcxi[0] != 1 || tcxi[npan] != ntcx + 1)
    return fail(QOL_ERR_LAYOUT, "tcxi must be monotone, one-based, and cover tcx exactly");
  for (qol_int k = 0; k < npan; ++k)
    if (tcxi[k + 1] < tcxi[k]) return fail(QOL_ERR_LAYOUT, "tcxi must be monotone, one-based, and cover tcx exactly");
  if ((tcxi[npan] - 1) * hdim > nnz) return fail(QOL_ERR_NNZ, "nnz is too small for the requested panel-target interactions");
  return 0;
}

int qol_getnearquad_lap_rrq_dev(qol_int npan, qol_int nterms, qol_int hdim, qol_int nquad, qol_int nsrc,
                                const double* sx, const double* snx, const double* sw, const double* rts,
                                const double* rps, qol_int ntcx, const double* tcx, const qol_int* tcxrow,
                                const qol_int* tcxi, qol_int orderff, double distff, qol_int iside, qol_int nnz,
                                qol_int* sparsei, qol_int* sparsej, double* sparsevs, double* sparsevd,
                                void* stream, int sync, qol_int* level_hist) {
  std::unique_lock<std::recursive_mutex> g(g_mu);
  int rc = ensure_device();
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream; /* 0 = the legacy default stream */
  /* the call runs on its stream's workspace under the stream's lock; with the
   * per-phase kernel timing on it also keeps the global lock (the timings add
   * into one set of totals) */
  StreamCtx* cx = stream_ctx(st);
  if (!cx) return fail(QOL_ERR_CUDA, "no current device");
  if (!g_ktime_on) g.unlock();
  std::unique_lock<std::mutex> sl(cx->mu);
  std::vector<long long> xi(npan + 1);
  CK(cudaMemcpyAsync(xi.data(), tcxi, sizeof(long long) * (npan + 1), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if ((rc = validate_near(npan, nterms, hdim, nsrc, ntcx, xi.data(), nnz))) return rc;
  if (npan == 0 || ntcx == 0) return 0;
  Job J{};
  J.npan = (int)npan; J.nterms = (int)nterms; J.nquad = (int)nquad; J.orderff = (int)orderff;
  J.exterior = (iside % 10) == 0; J.subtract_naive = 1; J.distff = distff; J.ntcx = ntcx;
  J.P = PanelIn{sx, snx, sw, rts, rps};
  J.Q = PairIn{tcx, (const long long*)tcxrow, (const long long*)tcxi};
  J.vs = sparsevs; J.vd = sparsevd; J.si = (long long*)sparsei; J.sj = (long long*)sparsej;
  rc = run_pipeline(J, st, nullptr, level_hist, nullptr, nullptr, &cx->a1, &cx->a2, &cx->graph);
  if (rc) return rc;
  if (sync) CK(cudaStreamSynchronize(st));
  return 0;
}

int qol_set_graphs(int enable) {
  if (enable != 0 && enable != 1) return fail(QOL_ERR_ARG, "qol_set_graphs: 0 or 1");
  g_graphs_on.store(enable);
  return 0;
}

int qol_graph_stats(qol_int* captures, qol_int* replays) {
  if (!captures || !replays) return fail(QOL_ERR_ARG, "null argument");
  *captures = g_graph_captures.load();
  *replays = g_graph_replays.load();
  return 0;
}

int qol_release_workspace(void) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(QOL_ERR_CUDA, "qol_release_workspace: device sync");
  for (Arena* a : {&g_arena, &g_arena2, &g_arena_io, &g_arena_grf}) a->release();
  g_batch_arenas.clear();
  std::lock_guard<std::mutex> cg(g_ctx_mu);
  for (auto& kv : g_ctx) { /* a call still running on that stream finishes first */
    std::lock_guard<std::mutex> sl(kv.second->mu);
    kv.second->graph.drop(); /* it launches into the workspace freed here */
    kv.second->a1.release();
    kv.second->a2.release();
  }
  return 0;
}

int qol_getnearquad_lap_rrq_batch_dev(qol_int njob, const qol_near_job* jobs, void* stream, qol_int* level_hist) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (njob < 0 || (njob > 0 && !jobs)) return fail(QOL_ERR_ARG, "bad arguments");
  int rc = ensure_device();
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  /* per job: validation (the CSR offsets read back), the pipeline job, two arenas */
  std::vector<std::unique_ptr<Arena>>& arenas = g_batch_arenas;
  while (arenas.size() < 2 * (size_t)njob + 1) arenas.emplace_back(new Arena());
  std::vector<Job> Js((size_t)njob);
  std::vector<char> live((size_t)njob, 0);
  for (qol_int k = 0; k < njob; ++k) {
    const qol_near_job& q = jobs[k];
    std::vector<long long> xi(q.npan + 1);
    CK(cudaMemcpyAsync(xi.data(), q.tcxi, sizeof(long long) * (q.npan + 1), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if ((rc = validate_near(q.npan, q.nterms, q.hdim, q.nsrc, q.ntcx, xi.data(), q.nnz))) return rc;
    if (level_hist) for (int i = 0; i < 6; ++i) level_hist[6 * k + i] = 0;
    if (q.npan == 0 || q.ntcx == 0) continue;
    Job& J = Js[k];
    J.npan = (int)q.npan; J.nterms = (int)q.nterms; J.nquad = (int)q.nquad; J.orderff = (int)q.orderff;
    J.exterior = (q.iside % 10) == 0; J.subtract_naive = 1; J.distff = q.distff; J.ntcx = q.ntcx;
    J.P = PanelIn{q.sx, q.snx, q.sw, q.rts, q.rps};
    J.Q = PairIn{q.tcx, (const long long*)q.tcxrow, (const long long*)q.tcxi};
    J.vs = q.sparsevs; J.vd = q.sparsevd; J.si = (long long*)q.sparsei; J.sj = (long long*)q.sparsej;
    live[k] = 1;
  }
  /* front of every job, each on its own workspace */
  std::vector<std::unique_ptr<PipeRun>> runs((size_t)njob);
  for (qol_int k = 0; k < njob; ++k) {
    if (!live[k]) continue;
    runs[k].reset(new PipeRun(Js[k], st, nullptr, arenas[2 * k].get(), arenas[2 * k + 1].get()));
    if ((rc = runs[k]->front())) return rc;
  }
  /* the level sums of all jobs: one persistent launch over the level-binned queue */
  if (g_sum_precision == 1) {
    for (qol_int k = 0; k < njob; ++k)
      if (live[k]) {
        PipeRun& P = *runs[k];
        CK(qol_launch_direct(P.T, P.J.P, P.J.Q, P.W, P.G, P.O, P.npan, st));
      }
  } else {
    std::vector<DirectJob> dj;
    std::vector<int> items;
    int nbmax = 1;
    for (qol_int k = 0; k < njob; ++k)
      if (live[k]) {
        PipeRun& P = *runs[k];
        dj.push_back(DirectJob{P.T, P.J.P, P.J.Q, P.W, P.G, P.O});
        nbmax = std::max(nbmax, P.T.ncw / 32);
      }
    for (int l = 3; l >= 0; --l) /* finest level first */
      for (size_t j = 0, k = 0; k < (size_t)njob; ++k) {
        if (!live[k]) continue;
        for (int p = 0; p < runs[k]->npan; ++p) { items.push_back((int)j); items.push_back(p); items.push_back(l); }
        ++j;
      }
    Arena& A = *arenas[2 * njob];
    const size_t need = sizeof(DirectJob) * dj.size() + sizeof(int) * (items.size() + 1) + 3 * 256;
    if ((rc = A.reserve(need))) return rc;
    A.reset();
    DirectJob* ddj = A.take<DirectJob>(dj.size());
    int* ditems = A.take<int>(items.size());
    int* dhead = A.take<int>(1);
    CK(cudaMemcpyAsync(ddj, dj.data(), sizeof(DirectJob) * dj.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ditems, items.data(), sizeof(int) * items.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(dhead, 0, sizeof(int), st));
    CK(qol_launch_direct_queue(ddj, nbmax, ditems, (int)(items.size() / 3), dhead, st));
    CK(cudaStreamSynchronize(st)); /* the host vectors above are the copies' sources */
  }
  for (qol_int k = 0; k < njob; ++k)
    if (live[k]) {
      PipeRun& P = *runs[k];
      CK(qol_launch_direct_cut(P.T, P.J.P, P.J.Q, P.W, P.G, P.O, P.npan, st));
    }
  /* the rest of every job (one stream: the per-pair RRQ kernels fill the GPU;
   * jobs on separate streams measured 3 % slower) */
  for (qol_int k = 0; k < njob; ++k) {
    if (!live[k]) continue;
    if ((rc = runs[k]->back(nullptr, nullptr, nullptr, true))) return rc;
  }
  CK(cudaStreamSynchronize(st));
  if (level_hist)
    for (qol_int k = 0; k < njob; ++k) {
      if (!live[k]) continue;
      const PipeRun& P = *runs[k];
      std::vector<int> cnt((size_t)P.npan * 8);
      CK(cudaMemcpy(cnt.data(), P.G.cnt, sizeof(int) * cnt.size(), cudaMemcpyDeviceToHost));
      for (int p = 0; p < P.npan; ++p) {
        for (int l = 1; l <= 5; ++l) level_hist[6 * k + l] += cnt[(size_t)p * 8 + l];
        level_hist[6 * k] += cnt[(size_t)p * 8 + QOL_LV_CUT];
      }
    }
  return 0;
}

int qol_getnearquad_lap_rrq(qol_int npan, qol_int nterms, qol_int hdim, qol_int nquad, qol_int nsrc, const double* sx,
                            const double* snx, const double* sw, const double* rts, const double* rps, qol_int ntcx,
                            const double* tcx, const qol_int* tcxrow, const qol_int* tcxi, qol_int orderff,
                            double distff, qol_int iside, qol_int isimd, qol_int nnz, qol_int* sparsei,
                            qol_int* sparsej, double* sparsevs, double* sparsevd, double* timeinfo) {
  (void)isimd;
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (!sx || !snx || !sw || !rts || !rps || !tcxi || (ntcx > 0 && (!tcx || !tcxrow)))
    return fail(QOL_ERR_ARG, "null argument");
  int rc = validate_near(npan, nterms, hdim, nsrc, ntcx, tcxi, nnz);
  if (rc) return rc;
  if ((rc = ensure_device())) return rc;
  if (npan == 0 || ntcx == 0) return 0;
  if ((rc = g_ring.init())) return rc;
  const auto tstart = std::chrono::steady_clock::now();
  cudaStream_t st = g_stream;
  const int hd = (int)hdim;
  const size_t nout = (size_t)ntcx * hdim;
  /* panel chunks (up to kMaxChunks on large calls): the pipeline runs chunk by
   * chunk and each chunk's values leave the GPU while later chunks compute.
   * Target counts follow a tapered schedule: a half-size first chunk (its
   * values are the first that can leave), full-size ones, then a half- and a
   * quarter-size last pair (what is left to copy after the last kernel) */
  constexpr int kMaxChunks = 12;
  const int nch = (int)std::max<qol_int>(1, std::min<qol_int>(kMaxChunks, npan / 192));
  std::vector<double> wcum(nch + 1, 0.0);
  for (int c = 0; c < nch; ++c) {
    double w = 1.0;
    if (nch >= 4) w = c == 0 ? 0.5 : (c == nch - 2 ? 0.5 : (c == nch - 1 ? 0.25 : 1.0));
    wcum[c + 1] = wcum[c] + w;
  }
  std::vector<long long> cb(nch + 1, 0);
  cb[nch] = npan;
  for (int c = 1; c < nch; ++c) {
    const qol_int want = (qol_int)((double)ntcx * wcum[c] / wcum[nch]);
    qol_int k = std::lower_bound(tcxi, tcxi + npan + 1, want + 1) - tcxi;
    cb[c] = std::min<qol_int>(npan, std::max<qol_int>(cb[c - 1], k));
  }
  size_t bytes = sizeof(double) * (size_t)(nsrc * 13 + ntcx * 3) + sizeof(long long) * (ntcx + npan + 1) +
                 sizeof(double) * 2 * nout + 16 * 256;
  if ((rc = g_arena_io.reserve(bytes))) return rc;
  g_arena_io.reset();
  double* dsx = g_arena_io.take<double>(3 * nsrc);
  double* dsnx = g_arena_io.take<double>(3 * nsrc);
  double* dsw = g_arena_io.take<double>(nsrc);
  double* drts = g_arena_io.take<double>(3 * nsrc);
  double* drps = g_arena_io.take<double>(3 * nsrc);
  double* dtcx = g_arena_io.take<double>(3 * ntcx);
  long long* drow = g_arena_io.take<long long>(ntcx);
  long long* dxi = g_arena_io.take<long long>(npan + 1);
  double* dval = g_arena_io.take<double>(2 * nout); /* vs then vd */
  int out = 0;
  const unsigned hw = std::thread::hardware_concurrency();
  /* leave two cores to the launching thread and the copy thread */
  const int nthr = (int)std::min(16u, std::max(2u, hw > 4 ? hw - 2 : 2u));
  /* inputs through the pinned ring: host threads copy pieces of the caller's
   * (pageable) arrays into free ring buffers and queue each piece's DMA on the
   * compute stream; the kernels are queued once every piece has landed */
  {
    struct Piece {
      char* d;
      const char* h;
      size_t n;
    };
    std::vector<Piece> pcs;
    auto add = [&](void* d, const void* h, size_t n) {
      for (size_t off = 0; off < n; off += kStageBytes)
        pcs.push_back({(char*)d + off, (const char*)h + off, std::min(kStageBytes, n - off)});
    };
    add(dsx, sx, sizeof(double) * 3 * nsrc);
    add(dsnx, snx, sizeof(double) * 3 * nsrc);
    add(dsw, sw, sizeof(double) * nsrc);
    add(drts, rts, sizeof(double) * 3 * nsrc);
    add(drps, rps, sizeof(double) * 3 * nsrc);
    add(dtcx, tcx, sizeof(double) * 3 * ntcx);
    add(drow, tcxrow, sizeof(long long) * ntcx);
    add(dxi, tcxi, sizeof(long long) * (npan + 1));
    FreeList ifl;
    std::atomic<int> ierr{0};
    {
      Workers IW(nthr);
      for (const Piece& pc : pcs)
        IW.submit([&, pc] {
          const int b = ifl.take();
          std::memcpy(g_ring.buf[b], pc.h, pc.n);
          if (cudaMemcpyAsync(pc.d, g_ring.buf[b], pc.n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
              cudaEventRecord(g_ring.ev[b], st) != cudaSuccess || cudaEventSynchronize(g_ring.ev[b]) != cudaSuccess)
            ierr = 1;
          ifl.give(b);
        });
    } /* joins the threads: every piece has landed */
    if (ierr) {
      cudaStreamSynchronize(st);
      return fail(QOL_ERR_CUDA, "input copy through the staging ring failed");
    }
  }
  g_host_ms[0] = ms_since(tstart);
  std::atomic<int> werr{0};
  {
    Workers W(nthr);
    /* COO indices on the host, overlapping the device work */
    const long long per = std::max<long long>(1, ntcx / (4 * nthr));
    std::atomic<int> fills_left{0};
    std::vector<std::pair<qol_int, qol_int>> fills;
    for (qol_int k0 = 0; k0 < npan;) {
      qol_int k1 = k0 + 1;
      while (k1 < npan && tcxi[k1] - tcxi[k0] < per) ++k1;
      fills.emplace_back(k0, k1);
      k0 = k1;
    }
    fills_left = (int)fills.size();
    for (auto kk : fills)
      W.submit([=, &fills_left] {
        fill_indices(kk.first, kk.second, hd, tcxi, tcxrow, sparsei, sparsej);
        if (--fills_left == 0) g_host_ms[6] = ms_since(tstart);
      });
    /* then the value arrays' pages, in chunk order */
    for (int c = 0; c < nch; ++c) {
      const size_t t0 = (size_t)(tcxi[cb[c]] - 1) * hd, t1 = (size_t)(tcxi[cb[c + 1]] - 1) * hd;
      for (size_t o = t0; o < t1; o += (size_t)4 << 20) {
        const size_t n = std::min((size_t)4 << 20, t1 - o);
        for (double* arr : {sparsevs, sparsevd}) W.submit([=] { prefault(arr + o, n * sizeof(double)); });
      }
    }
    /* values: chunk c leaves the GPU once the compute stream passed its event */
    std::vector<cudaEvent_t> cev(nch, nullptr);
    for (int c = 0; c < nch && !out; ++c)
      if (cudaEventCreateWithFlags(&cev[c], cudaEventDisableTiming) != cudaSuccess)
        out = fail(QOL_ERR_CUDA, "event creation failed");
    Progress prog;
    FreeList fl;
    std::atomic<int> cerr{0};
    std::thread copier([&] {
      double* hdst[2] = {sparsevs, sparsevd};
      for (int c = 0; c < nch; ++c) {
        if (!prog.wait(c)) return;
        if (cudaStreamWaitEvent(g_ring.cs, cev[c], 0) != cudaSuccess) { cerr = 1; return; }
        const size_t t0 = (size_t)(tcxi[cb[c]] - 1), t1 = (size_t)(tcxi[cb[c + 1]] - 1);
        for (int a = 0; a < 2; ++a) {
          const char* src = (const char*)(dval + a * nout + t0 * hd);
          char* dst = (char*)(hdst[a] + t0 * hd);
          const size_t tot = (t1 - t0) * hd * sizeof(double);
          for (size_t off = 0; off < tot; off += kStageBytes) {
            const size_t n = std::min(kStageBytes, tot - off);
            const int b = fl.take();
            if (cudaMemcpyAsync(g_ring.buf[b], src + off, n, cudaMemcpyDeviceToHost, g_ring.cs) != cudaSuccess ||
                cudaEventRecord(g_ring.ev[b], g_ring.cs) != cudaSuccess) {
              cerr = 1;
              fl.give(b);
              return;
            }
            W.submit([&, b, dst, off, n] {
              if (cudaEventSynchronize(g_ring.ev[b]) == cudaSuccess) copy_out(dst + off, g_ring.buf[b], n);
              else werr = 1;
              fl.give(b);
            });
          }
        }
      }
    });
    if (!out) {
      Job J{};
      J.npan = (int)npan; J.nterms = (int)nterms; J.nquad = (int)nquad; J.orderff = (int)orderff;
      J.exterior = (iside % 10) == 0; J.subtract_naive = 1; J.distff = distff; J.ntcx = ntcx;
      J.P = PanelIn{dsx, dsnx, dsw, drts, drps};
      J.Q = PairIn{dtcx, drow, dxi};
      J.vs = dval; J.vd = dval + nout;
      J.si = nullptr; J.sj = nullptr;
      J.chunk_pan = &cb;
      J.after_chunk = [&](int c, cudaStream_t sc) {
        if (cudaEventRecord(cev[c], sc) == cudaSuccess) prog.set(c + 1);
        else cerr = 1;
      };
      out = run_pipeline(J, st, timeinfo, nullptr, nullptr, nullptr);
    }
    if (out || cerr) prog.abort();
    g_host_ms[1] = ms_since(tstart);
    copier.join();
    g_host_ms[2] = ms_since(tstart);
    cudaStreamSynchronize(g_ring.cs);
    g_host_ms[3] = ms_since(tstart);
    W.finish();
    g_host_ms[4] = ms_since(tstart);
    cudaStreamSynchronize(st);
    for (cudaEvent_t e : cev) if (e) cudaEventDestroy(e);
    if (!out && (cerr || werr)) out = fail(QOL_ERR_CUDA, "device-to-host copy of the COO values failed");
  }
  g_host_ms[5] = ms_since(tstart);
  return out;
}

int qol_last_host_times(double* ms7) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (!ms7) return fail(QOL_ERR_ARG, "null argument");
  for (int i = 0; i < 7; ++i) ms7[i] = g_host_ms[i];
  return 0;
}

/* GRF near phase (stellarator_grf_core_mod.f90:652-899): ball lists of the
 * surface's own nodes, the RRQ corrections of every near pair, contracted with
 * the density (ubn, ub) and scattered into u in panel order. */
/* the GRF near phase of panels [plo, phi) for nrhs densities (ub, ubn, u:
 * nsrc x nrhs, column-major): the near search and the corrections once, their
 * application once a density */
static int grf_near_impl(qol_int npan, qol_int nterms, qol_int nquad, qol_int orderff, double distff, qol_int iside,
                         qol_int nsrc, const double* sx, const double* snx, const double* sw, const double* rts,
                         const double* rps, const double* xbuf, qol_int nrhs, const double* ub, const double* ubn,
                         qol_int plo, qol_int phi, double* u, qol_int* nnear, qol_int* level_hist, double* timeinfo) {
  const qol_int hd = nterms * (nterms + 1) / 2;
  if (!sx || !snx || !sw || !rts || !rps || !ub || !ubn || !u) return fail(QOL_ERR_ARG, "null argument");
  if (npan < 0 || nsrc != npan * hd) return fail(QOL_ERR_LAYOUT, "the panel order, npan and nsrc are inconsistent");
  if (plo < 0 || phi < plo || phi > npan) return fail(QOL_ERR_ARG, "panel range outside [0, npan]");
  if (nrhs < 1) return fail(QOL_ERR_ARG, "nrhs must be positive");
  int rc = ensure_device();
  if (rc) return rc;
  if (nnear) *nnear = 0;
  if (level_hist) for (int i = 0; i < 6; ++i) level_hist[i] = 0;
  const qol_int nloc = phi - plo; /* this call's panels [plo, phi): ball lists, corrections, scatter */
  if (nloc == 0) return 0;
  cudaStream_t st = g_stream;
  const int nbd = 3 * (int)nquad;
  size_t need = sizeof(double) * (size_t)(16 * nsrc + 3 * (nrhs - 1) * nsrc + 4 * npan + 6 * ((nsrc + 255) / 256) +
                                          (xbuf ? 3 * (nbd + 3) * npan : 0)) +
                sizeof(long long) * (size_t)(3 * nloc + 3) + 16 * 256;
  if ((rc = g_arena_io.reserve(need))) return rc;
  g_arena_io.reset();
  double* dsx = g_arena_io.take<double>(3 * nsrc);
  double* dsnx = g_arena_io.take<double>(3 * nsrc);
  double* dsw = g_arena_io.take<double>(nsrc);
  double* drts = g_arena_io.take<double>(3 * nsrc);
  double* drps = g_arena_io.take<double>(3 * nsrc);
  double* dub = g_arena_io.take<double>(nsrc * nrhs);
  double* dubn = g_arena_io.take<double>(nsrc * nrhs);
  double* du = g_arena_io.take<double>(nsrc * nrhs);
  double* dball = g_arena_io.take<double>(4 * npan);
  double* dbox = g_arena_io.take<double>(6 * (size_t)((nsrc + 255) / 256)); /* node-chunk boxes of the near search */
  double* dchart = xbuf ? g_arena_io.take<double>((size_t)3 * (nbd + 3) * nloc) : nullptr;
  long long* dcnt = g_arena_io.take<long long>(nloc);
  long long* doff = g_arena_io.take<long long>(nloc + 1); /* 0-based offsets */
  long long* dxi = g_arena_io.take<long long>(nloc + 1);  /* 1-based, the pipeline's tcxi */
  CK(cudaMemcpyAsync(dsx, sx, sizeof(double) * 3 * nsrc, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dsnx, snx, sizeof(double) * 3 * nsrc, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dsw, sw, sizeof(double) * nsrc, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(drts, rts, sizeof(double) * 3 * nsrc, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(drps, rps, sizeof(double) * 3 * nsrc, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dub, ub, sizeof(double) * nsrc * nrhs, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dubn, ubn, sizeof(double) * nsrc * nrhs, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(du, u, sizeof(double) * nsrc * nrhs, cudaMemcpyHostToDevice, st));
  if (xbuf)
    CK(cudaMemcpyAsync(dchart, xbuf + (size_t)3 * (nbd + 3) * plo, sizeof(double) * 3 * (nbd + 3) * nloc,
                       cudaMemcpyHostToDevice, st));
  CK(qol_launch_grf_balls((int)npan, (int)hd, nsrc, dsx, dsw, dball, dbox, dcnt, (int)plo, (int)phi, st));
  std::vector<long long> cnt(nloc), off(nloc + 1), xi(nloc + 1);
  CK(cudaMemcpyAsync(cnt.data(), dcnt, sizeof(long long) * nloc, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  off[0] = 0;
  for (qol_int k = 0; k < nloc; ++k) off[k + 1] = off[k] + cnt[k];
  for (qol_int k = 0; k <= nloc; ++k) xi[k] = off[k] + 1;
  const long long nn = off[nloc];
  if (nnear) *nnear = nn;
  CK(cudaMemcpyAsync(doff, off.data(), sizeof(long long) * (nloc + 1), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dxi, xi.data(), sizeof(long long) * (nloc + 1), cudaMemcpyHostToDevice, st));
  if (nn > 0) {
    need = sizeof(double) * (size_t)nn * (3 + 1 + 2 * hd) + sizeof(long long) * (size_t)nn * 2 + 8 * 256;
    if ((rc = g_arena_grf.reserve(need))) return rc;
    g_arena_grf.reset();
    long long* didx = g_arena_grf.take<long long>(nn);
    long long* dloc = plo ? g_arena_grf.take<long long>(nn) : didx; /* rows in the range's own numbering */
    double* dtcx = g_arena_grf.take<double>(3 * nn);
    double* dval = g_arena_grf.take<double>(nn);
    double* dvs = g_arena_grf.take<double>((size_t)nn * hd);
    double* dvd = g_arena_grf.take<double>((size_t)nn * hd);
    const double* ball = dball + 4 * (size_t)plo;
    CK(qol_launch_grf_csr((int)nloc, nsrc, dsx, ball, dbox, doff, didx, dtcx, plo ? dloc : nullptr,
                          (long long)plo * hd, st));
    Job J{};
    J.npan = (int)nloc; J.nterms = (int)nterms; J.nquad = (int)nquad; J.orderff = (int)orderff;
    J.exterior = (iside % 10) == 0; J.subtract_naive = 1; J.distff = distff; J.ntcx = nn;
    const size_t o = (size_t)plo * hd; /* the range's panels; the self-pair mask compares their rows */
    J.P = PanelIn{dsx + 3 * o, dsnx + 3 * o, dsw + o, drts + 3 * o, drps + 3 * o};
    J.Q = PairIn{dtcx, dloc, dxi};
    J.vs = dvs; J.vd = dvd; J.si = nullptr; J.sj = nullptr;
    J.chart = dchart;
    long long hist[6] = {0, 0, 0, 0, 0, 0};
    if ((rc = run_pipeline(J, st, timeinfo, hist, nullptr, nullptr))) return rc;
    if (level_hist) for (int i = 0; i < 6; ++i) level_hist[i] = hist[i];
    for (qol_int r = 0; r < nrhs; ++r) {
      const size_t ro = (size_t)r * nsrc;
      CK(qol_launch_grf_apply((int)nloc, (int)hd, nsrc, dsx, ball, doff, didx, dvs, dvd, dub + ro + o, dubn + ro + o,
                              dval, du + ro, st));
    }
  }
  CK(cudaMemcpyAsync(u, du, sizeof(double) * nsrc * nrhs, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return 0;
}

int qol_grf_near_range(qol_int npan, qol_int nterms, qol_int nquad, qol_int orderff, double distff, qol_int iside,
                       qol_int nsrc, const double* sx, const double* snx, const double* sw, const double* rts,
                       const double* rps, const double* xbuf, const double* ub, const double* ubn, qol_int plo,
                       qol_int phi, double* u, qol_int* nnear, qol_int* level_hist, double* timeinfo) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  return grf_near_impl(npan, nterms, nquad, orderff, distff, iside, nsrc, sx, snx, sw, rts, rps, xbuf, 1, ub, ubn, plo,
                       phi, u, nnear, level_hist, timeinfo);
}

int qol_grf_near_multi(qol_int npan, qol_int nterms, qol_int nquad, qol_int orderff, double distff, qol_int iside,
                       qol_int nsrc, const double* sx, const double* snx, const double* sw, const double* rts,
                       const double* rps, const double* xbuf, qol_int nrhs, const double* ub, const double* ubn,
                       double* u, qol_int* nnear, qol_int* level_hist, double* timeinfo) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  return grf_near_impl(npan, nterms, nquad, orderff, distff, iside, nsrc, sx, snx, sw, rts, rps, xbuf, nrhs, ub, ubn, 0,
                       npan, u, nnear, level_hist, timeinfo);
}

/* the blocked Direct far field u_i = sum_j S_ij ubn_j - D_ij ub_j with zero
 * self term (stellarator_grf_core_mod.f90:566-606) */
int qol_grf_near(qol_int npan, qol_int nterms, qol_int nquad, qol_int orderff, double distff, qol_int iside,
                 qol_int nsrc, const double* sx, const double* snx, const double* sw, const double* rts,
                 const double* rps, const double* xbuf, const double* ub, const double* ubn, double* u,
                 qol_int* nnear, qol_int* level_hist, double* timeinfo) {
  return qol_grf_near_range(npan, nterms, nquad, orderff, distff, iside, nsrc, sx, snx, sw, rts, rps, xbuf, ub, ubn,
                            0, npan, u, nnear, level_hist, timeinfo);
}

/* the GPU geometry generator over a chart list (geo_core, :636-750) */
static int panels_of_charts(const std::vector<qolh::Chart>& cl, qol_int nmode, const double* modes, qol_int nfp,
                            qol_int mp, qol_int np, qol_int nterms, qol_int* ntri, double* sx, double* snx,
                            double* sw, double* rts, double* rps) {
  const qol_int nchart = (qol_int)cl.size(), nt = 2 * nchart;
  if (!sx) { *ntri = nt; return 0; } /* the size query (as stellarator_geo_ntri) */
  if (!snx || !sw || !rts || !rps) return fail(QOL_ERR_ARG, "null output");
  if (*ntri < nt) return fail(QOL_ERR_NNZ, "ntri is smaller than the panel count");
  *ntri = nt;
  int rc = ensure_device();
  if (rc) return rc;
  const int p = (int)nterms, hd = p * (p + 1) / 2;
  const size_t nsrc = (size_t)nt * hd;
  std::vector<double> x0(p), w0(p), Dm((size_t)p * p), uv(2 * hd), wts(hd), tables, chv(6 * (size_t)nchart);
  qolh::gauss(p, x0.data(), w0.data(), Dm.data());
  qolh::vr_nodes(p - 1, uv.data(), wts.data());
  qolh::surface_interp_tables(p, tables);
  for (qol_int c = 0; c < nchart; ++c) {
    const qolh::Chart& h = cl[c];
    const double v[6] = {h.a1, h.b1, h.a2, h.b2, h.jj, h.ii};
    for (int k = 0; k < 6; ++k) chv[6 * c + k] = v[k];
  }
  cudaStream_t st = g_stream;
  const size_t need = sizeof(double) * (4 * (size_t)nmode + chv.size() + 2 * (size_t)p + Dm.size() + hd +
                                        tables.size() + 13 * nsrc) + 16 * 256;
  if ((rc = g_arena_io.reserve(need))) return rc;
  g_arena_io.reset();
  double* dmodes = g_arena_io.take<double>(4 * (size_t)nmode);
  double* dch = g_arena_io.take<double>(chv.size());
  double* dx0 = g_arena_io.take<double>(p);
  double* dD = g_arena_io.take<double>(Dm.size());
  double* dw = g_arena_io.take<double>(hd);
  double* dtab = g_arena_io.take<double>(tables.size());
  double* dsx = g_arena_io.take<double>(3 * nsrc);
  double* dsnx = g_arena_io.take<double>(3 * nsrc);
  double* dsw = g_arena_io.take<double>(nsrc);
  double* drts = g_arena_io.take<double>(3 * nsrc);
  double* drps = g_arena_io.take<double>(3 * nsrc);
  CK(cudaMemcpyAsync(dmodes, modes, sizeof(double) * 4 * nmode, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dch, chv.data(), sizeof(double) * chv.size(), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dx0, x0.data(), sizeof(double) * p, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dD, Dm.data(), sizeof(double) * Dm.size(), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dw, wts.data(), sizeof(double) * hd, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dtab, tables.data(), sizeof(double) * tables.size(), cudaMemcpyHostToDevice, st));
  const double pi = 3.14159265358979323846;
  CK(qol_launch_surface_panels((int)nchart, (int)nmode, dmodes, (int)nfp, p, dch, pi / (double)np, pi / (double)mp,
                               dx0, dD, dw, dtab, dsx, dsnx, dsw, drts, drps, st));
  CK(cudaMemcpyAsync(sx, dsx, sizeof(double) * 3 * nsrc, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(snx, dsnx, sizeof(double) * 3 * nsrc, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(sw, dsw, sizeof(double) * nsrc, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(rts, drts, sizeof(double) * 3 * nsrc, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(rps, drps, sizeof(double) * 3 * nsrc, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return 0;
}

int qol_surface_panels(qol_int nmode, const double* modes, qol_int nfp, qol_int mp, qol_int np, qol_int nterms,
                       qol_int split, qol_int* ntri, double* sx, double* snx, double* sw, double* rts,
                       double* rps) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (!modes || !ntri || nmode < 1 || mp < 1 || np < 1) return fail(QOL_ERR_ARG, "bad arguments");
  if (nterms < 2 || nterms > 16) return fail(QOL_ERR_ORDER, "nterms outside 2..16");
  const std::vector<qolh::Chart> cl =
      qolh::surface_charts((int)nmode, modes, (int)nfp, (int)mp, (int)np, (int)nterms, split != 0);
  return panels_of_charts(cl, nmode, modes, nfp, mp, np, nterms, ntri, sx, snx, sw, rts, rps);
}

int qol_surface_charts(qol_int nmode, const double* modes, qol_int nfp, qol_int mp, qol_int np, qol_int p,
                       double restol, qol_int cap, qol_int* nchart, double* charts) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (!modes || !nchart || nmode < 1 || mp < 1 || np < 1) return fail(QOL_ERR_ARG, "bad arguments");
  if (p < 2 || p > 16) return fail(QOL_ERR_ORDER, "p outside 2..16");
  std::vector<qolh::Chart> cl;
  if (!qolh::surface_charts_adaptive((int)nmode, modes, (int)nfp, (int)mp, (int)np, (int)p, restol, cap, cl))
    return fail(QOL_ERR_NNZ, "qol_surface_charts: more than cap charts");
  if (charts) {
    if (*nchart < (qol_int)cl.size()) return fail(QOL_ERR_NNZ, "nchart is smaller than the chart count");
    for (size_t k = 0; k < cl.size(); ++k) {
      const double v[6] = {cl[k].a1, cl[k].b1, cl[k].a2, cl[k].b2, cl[k].jj, cl[k].ii};
      for (int d = 0; d < 6; ++d) charts[6 * k + d] = v[d];
    }
  }
  *nchart = (qol_int)cl.size();
  return 0;
}

int qol_surface_panels_charts(qol_int nmode, const double* modes, qol_int nfp, qol_int mp, qol_int np,
                              qol_int nterms, qol_int nchart, const double* charts, qol_int* ntri, double* sx,
                              double* snx, double* sw, double* rts, double* rps) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (!modes || !ntri || !charts || nmode < 1 || mp < 1 || np < 1 || nchart < 1)
    return fail(QOL_ERR_ARG, "bad arguments");
  if (nterms < 2 || nterms > 16) return fail(QOL_ERR_ORDER, "nterms outside 2..16");
  std::vector<qolh::Chart> cl((size_t)nchart);
  for (qol_int k = 0; k < nchart; ++k)
    cl[k] = qolh::Chart{charts[6 * k], charts[6 * k + 1], charts[6 * k + 2], charts[6 * k + 3], charts[6 * k + 4],
                        charts[6 * k + 5]};
  return panels_of_charts(cl, nmode, modes, nfp, mp, np, nterms, ntri, sx, snx, sw, rts, rps);
}

int qol_interp_matrix(qol_int korder, qol_int n, const double* uv, double* M) {
  if (korder < 0 || korder > 20 || n < 0 || (n > 0 && (!uv || !M))) return fail(QOL_ERR_ARG, "bad arguments");
  qolh::interp_matrix((int)korder, (int)n, uv, M);
  return 0;
}

int qol_direct_farfield_range(qol_int nsrc, const double* sx, const double* snx, const double* sw,
                              const double* ub, const double* ubn, qol_int tlo, qol_int thi, double* u) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (!sx || !snx || !sw || !ub || !ubn || !u) return fail(QOL_ERR_ARG, "null argument");
  if (nsrc < 0) return fail(QOL_ERR_ARG, "negative size");
  if (tlo < 0 || thi < tlo || thi > nsrc) return fail(QOL_ERR_ARG, "target range outside [0, nsrc]");
  int rc = ensure_device();
  if (rc) return rc;
  if (thi == tlo) return 0;
  cudaStream_t st = g_stream;
  if ((rc = g_arena_io.reserve(sizeof(double) * (size_t)10 * nsrc + 8 * 256))) return rc;
  g_arena_io.reset();
  double* dsx = g_arena_io.take<double>(3 * nsrc);
  double* dsnx = g_arena_io.take<double>(3 * nsrc);
  double* dsw = g_arena_io.take<double>(nsrc);
  double* dub = g_arena_io.take<double>(nsrc);
  double* dubn = g_arena_io.take<double>(nsrc);
  double* du = g_arena_io.take<double>(nsrc);
  CK(cudaMemcpyAsync(dsx, sx, sizeof(double) * 3 * nsrc, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dsnx, snx, sizeof(double) * 3 * nsrc, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dsw, sw, sizeof(double) * nsrc, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dub, ub, sizeof(double) * nsrc, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dubn, ubn, sizeof(double) * nsrc, cudaMemcpyHostToDevice, st));
  CK(qol_launch_direct_far(nsrc, dsx, dsnx, dsw, dub, dubn, du, tlo, thi, st));
  CK(cudaMemcpyAsync(u + tlo, du + tlo, sizeof(double) * (thi - tlo), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return 0;
}

int qol_direct_farfield(qol_int nsrc, const double* sx, const double* snx, const double* sw, const double* ub,
                        const double* ubn, double* u) {
  return qol_direct_farfield_range(nsrc, sx, snx, sw, ub, ubn, 0, nsrc, u);
}

int qol_rrq(qol_int m, const double* tx, qol_int n, const double* sx, const double* snx, const double* sw,
            const double* rts, const double* rps, qol_int order, qol_int nquad, qol_int orderff, double distff,
            qol_int exterior, qol_int isimd, qol_int ichart, const double* sxbd_chart, const double* rv_chart,
            const double* tgl, const double* wgl, const double* Dgl, const double* w_bclag, const double* Legmat,
            const double* umatr, const double* vmatr, double* As, double* Ad, double* Omega,
            double* IalphaAsvestas, double* timeinfo) {
  (void)isimd; (void)Dgl; (void)w_bclag; (void)Legmat; (void)vmatr;
  std::lock_guard<std::recursive_mutex> g(g_mu);
  const qol_int hd = order * (order + 1) / 2;
  if (n != hd) return fail(QOL_ERR_NPOLS, "n must equal order*(order+1)/2");
  if (m < 0 || !sx || !snx || !sw || !rts || !rps || (m > 0 && (!tx || !As || !Ad)))
    return fail(QOL_ERR_ARG, "bad arguments");
  if (tgl && wgl && !tables_match((int)nquad, (int)order - 1, tgl, wgl, umatr))
    return fail(QOL_ERR_TABLES, "precomputed tables differ from qol_simplex_precomp's");
  int rc = ensure_device();
  if (rc) return rc;
  if (m == 0) return 0;
  cudaStream_t st = g_stream;
  const int nbd = 3 * (int)nquad;
  size_t bytes = sizeof(double) * (size_t)(13 * n + 3 * m + 2 * m * n + 4 * hd * m + m + 3 * (nbd + 3)) +
                 sizeof(long long) * (m + 2) + 16 * 256;
  char* buf = nullptr;
  if (cudaMalloc(&buf, bytes) != cudaSuccess) { cudaGetLastError(); return fail(QOL_ERR_CUDA, "device allocation failed"); }
  size_t used = 0;
  auto take = [&](size_t b) { size_t o = (used + 255) & ~(size_t)255; used = o + b; return buf + o; };
  double* dsx = (double*)take(sizeof(double) * 3 * n);
  double* dsnx = (double*)take(sizeof(double) * 3 * n);
  double* dsw = (double*)take(sizeof(double) * n);
  double* drts = (double*)take(sizeof(double) * 3 * n);
  double* drps = (double*)take(sizeof(double) * 3 * n);
  double* dtx = (double*)take(sizeof(double) * 3 * m);
  double* dAs = (double*)take(sizeof(double) * m * n);
  double* dAd = (double*)take(sizeof(double) * m * n);
  double* dOm = (double*)take(sizeof(double) * 4 * hd * m);
  double* dIa = (double*)take(sizeof(double) * m);
  double* dch = (double*)take(sizeof(double) * 3 * (nbd + 3));
  long long* drow = (long long*)take(sizeof(long long) * m);
  long long* dxi = (long long*)take(sizeof(long long) * 2);
  std::vector<long long> xi = {1, m + 1};
  std::vector<double> chart;
  if (ichart == 1) {
    if (!sxbd_chart || !rv_chart) { cudaFree(buf); return fail(QOL_ERR_ARG, "ichart = 1 needs sxbd_chart and rv_chart"); }
    chart.assign(sxbd_chart, sxbd_chart + 3 * nbd);
    chart.insert(chart.end(), rv_chart, rv_chart + 9);
  }
  int out = 0;
  do {
#define CKB(x)                                                                        \
  {                                                                                   \
    cudaError_t e_ = (x);                                                             \
    if (e_ != cudaSuccess) { out = fail(QOL_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); break; } \
  }
    CKB(cudaMemcpyAsync(dsx, sx, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    CKB(cudaMemcpyAsync(dsnx, snx, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    CKB(cudaMemcpyAsync(dsw, sw, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    CKB(cudaMemcpyAsync(drts, rts, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    CKB(cudaMemcpyAsync(drps, rps, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    CKB(cudaMemcpyAsync(dtx, tx, sizeof(double) * 3 * m, cudaMemcpyHostToDevice, st));
    CKB(cudaMemsetAsync(drow, 0, sizeof(long long) * m, st));
    CKB(cudaMemcpyAsync(dxi, xi.data(), sizeof(long long) * 2, cudaMemcpyHostToDevice, st));
    CKB(cudaMemsetAsync(dAs, 0, sizeof(double) * m * n, st));
    CKB(cudaMemsetAsync(dAd, 0, sizeof(double) * m * n, st));
    CKB(cudaMemsetAsync(dOm, 0, sizeof(double) * 4 * hd * m, st));
    CKB(cudaMemsetAsync(dIa, 0, sizeof(double) * m, st));
    if (ichart == 1) CKB(cudaMemcpyAsync(dch, chart.data(), sizeof(double) * chart.size(), cudaMemcpyHostToDevice, st));
    Job J{};
    J.npan = 1; J.nterms = (int)order; J.nquad = (int)nquad; J.orderff = (int)orderff;
    J.exterior = exterior != 0; J.subtract_naive = 0; J.distff = distff; J.ntcx = m;
    J.P = PanelIn{dsx, dsnx, dsw, drts, drps};
    J.Q = PairIn{dtx, drow, dxi};
    J.vs = dAs; J.vd = dAd; J.omega = dOm; J.ialpha = dIa; J.si = nullptr; J.sj = nullptr;
    J.chart = ichart == 1 ? dch : nullptr;
    out = run_pipeline(J, st, timeinfo, nullptr, nullptr, nullptr);
    if (out) break;
    CKB(cudaMemcpyAsync(As, dAs, sizeof(double) * m * n, cudaMemcpyDeviceToHost, st));
    CKB(cudaMemcpyAsync(Ad, dAd, sizeof(double) * m * n, cudaMemcpyDeviceToHost, st));
    if (Omega) CKB(cudaMemcpyAsync(Omega, dOm, sizeof(double) * 4 * hd * m, cudaMemcpyDeviceToHost, st));
    if (IalphaAsvestas) CKB(cudaMemcpyAsync(IalphaAsvestas, dIa, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
    CKB(cudaStreamSynchronize(st));
#undef CKB
  } while (0);
  cudaFree(buf);
  return out;
}

/* ---------------- reference-symbol aliases ---------------- */
void qol_simplex_precomp_mex_(const qol_int* nquad, const qol_int* korder, const qol_int* kpols, double* tgl,
                              double* wgl, double* Dgl, double* w_bclag, double* Legmat, double* umatr,
                              double* vmatr) {
  qol_simplex_precomp(*nquad, *korder, *kpols, tgl, wgl, Dgl, w_bclag, Legmat, umatr, vmatr);
}
void qol_build_patch_levels_mex_(const qol_int* korder, const qol_int* npols, const double* sx, const double* rts,
                                 const double* rps, const qol_int* order, const double* dist, const qol_int* nlevel,
                                 qol_int* lv, qol_int* ier) {
  qol_build_patch_levels(*korder, *npols, sx, rts, rps, *order, *dist, *nlevel, lv, ier);
}
void qol_lap3dsdlpmat_levels_mex_(const qol_int* m, const double* tx, const qol_int* npols, const qol_int* lv,
                                  const qol_int* isimd, double* As, double* Ad, qol_int* idxs, qol_int* ms,
                                  qol_int* ier) {
  qol_lap3dsdlpmat_levels(*m, tx, *npols, *lv, *isimd, As, Ad, idxs, ms, ier);
}
void qol_clear_patch_levels_mex_(const qol_int* lv, qol_int* ier) { qol_clear_patch_levels(*lv, ier); }
void qol_clear_patch_levels_all_mex_(qol_int* ier) { qol_clear_patch_levels_all(ier); }
void qol_getnearquad_lap_rrq_mex_(const qol_int* npan, const qol_int* nterms, const qol_int* hdim,
                                  const qol_int* nquad, const qol_int* nsrc, const double* sx, const double* snx,
                                  const double* sw, const double* rts, const double* rps, const qol_int* ntcx,
                                  const double* tcx, const qol_int* tcxrow, const qol_int* tcxi,
                                  const qol_int* orderff, const double* distff, const qol_int* iside,
                                  const qol_int* isimd, const qol_int* nnz, qol_int* sparsei, qol_int* sparsej,
                                  double* sparsevs, double* sparsevd, double* timeinfo) {
  qol_getnearquad_lap_rrq(*npan, *nterms, *hdim, *nquad, *nsrc, sx, snx, sw, rts, rps, *ntcx, tcx, tcxrow, tcxi,
                          *orderff, *distff, *iside, *isimd, *nnz, sparsei, sparsej, sparsevs, sparsevd, timeinfo);
}
void qol_rrq_mex_(const qol_int* m, const double* tx, const qol_int* n, const double* sx, const double* snx,
                  const double* sw, const double* rts, const double* rps, const qol_int* order, const qol_int* nquad,
                  const qol_int* orderff, const double* distff, const qol_int* exterior, const qol_int* isimd,
                  const qol_int* ichart, const double* sxbd_chart, const double* rv_chart, const double* tgl,
                  const double* wgl, const double* Dgl, const double* w_bclag, const double* Legmat,
                  const double* umatr, const double* vmatr, double* As, double* Ad, double* Omega,
                  double* IalphaAsvestas, double* timeinfo) {
  qol_rrq(*m, tx, *n, sx, snx, sw, rts, rps, *order, *nquad, *orderff, *distff, *exterior, *isimd, *ichart,
          sxbd_chart, rv_chart, tgl, wgl, Dgl, w_bclag, Legmat, umatr, vmatr, As, Ad, Omega, IalphaAsvestas,
          timeinfo);
}

} // extern "C"
