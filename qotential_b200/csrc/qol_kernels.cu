/* qol_b200 kernels: the RRQ near-field hot path on sm_100a, FP64.
 *
 *   k_level_nodes,   build_patch_levels_r64 (patch_refine_mod.f90:423-502)
 *   k_level_subs
 *   k_classify       ball tests of lap3dsdlpmat_levels_r64 (:516-551)
 *   k_direct         level kernel sums fused with the interpmat contraction
 *                    (:553-600) and the naive-block subtraction of
 *                    getnearquad_lap_rrq_r64 (lap3d_close_mod.f90:935-956)
 *   k_rrq_panel_blk  per-panel RRQ precompute (lap3d_close_mod.f90:472-620,
 *                    843-863): frame, boundary, harmonic basis, inverse of the
 *                    quaternion system and of the S system (blocked
 *                    Gauss-Jordan, trailing updates on the FP64 tensor path)
 *   k_rrq_geom       per-pair SSQ weights, string direction, solid angle,
 *                    boundary weights (:789-832), one warp per pair
 *   k_rrq_moments    per-pair harmonic moments (:832-841) by solid-harmonic
 *                    translation, one warp per pair
 *   k_rrq_apply      the two solves as per-panel matrix products (:843-870)
 *   k_coo_index      COO row/column indices (:948-956)
 */
#include "qol_dev.cuh"
#include "qol_kernels.h"
#include <cmath>
#include <cooperative_groups.h>
namespace cg = cooperative_groups;

__constant__ double c_hb[QOL_MAXL + 2][QOL_MAXL + 2]; /* sqrt((l+m-1)(l-m-1)) */
__constant__ double c_hc[QOL_MAXL + 2][QOL_MAXL + 2]; /* 1/sqrt((l-m)(l+m)) */
__constant__ double c_hcm[QOL_MAXL + 2];               /* sqrt((2m-1)/(2m)) */
/* regular solid harmonics R_l^m (k_rrq_moments) */
__constant__ double c_rq[QOL_MAXL + 2][QOL_MAXL + 2]; /* 1/((l+m)(l-m)), l > m */
__constant__ double c_rn[QOL_MAXL + 2][QOL_MAXL + 2]; /* sqrt((l-m)!(l+m)!) */
__constant__ double c_rd[QOL_MAXL + 2];               /* 1/(2m) */
__constant__ double c_rinv[QOL_MAXL + 2];             /* 1/l, 0 at l = 0 */
/* three-term recurrences without divisions (k_rrq_geom) */
__constant__ double c_la[QOL_MAXNQ + 2];            /* (2k+1)/(k+1) */
__constant__ double c_lb[QOL_MAXNQ + 2];            /* k/(k+1) */
__constant__ double c_rk[QOL_MAXNQ + 2];            /* 1/k, 0 at k = 0 */
__device__ double g_jq[QOL_MAXL + 1][QOL_MAXL + 1][4]; /* Jacobi P^(2a+1,0)_b: (c2, c3, c4)/c1 */

cudaError_t qol_upload_harm_coefs(const double* hb, const double* hc, const double* hcm, cudaStream_t st) {
  cudaError_t err = cudaSuccess;
  auto keep = [&](cudaError_t e) { if (err == cudaSuccess) err = e; };
  keep(cudaMemcpyToSymbolAsync(c_hb, hb, sizeof(double) * (QOL_MAXL + 2) * (QOL_MAXL + 2), 0,
                          cudaMemcpyHostToDevice, st));
  keep(cudaMemcpyToSymbolAsync(c_hc, hc, sizeof(double) * (QOL_MAXL + 2) * (QOL_MAXL + 2), 0,
                          cudaMemcpyHostToDevice, st));
  keep(cudaMemcpyToSymbolAsync(c_hcm, hcm, sizeof(double) * (QOL_MAXL + 2), 0, cudaMemcpyHostToDevice, st));
  const int M = QOL_MAXL + 2;
  double rq[M][M] = {}, rn[M][M] = {}, rd[M] = {}, rinv[M] = {};
  double fact[2 * M];
  fact[0] = 1.0;
  for (int i = 1; i < 2 * M; ++i) fact[i] = fact[i - 1] * i;
  for (int l = 0; l < M; ++l) {
    if (l > 0) { rd[l] = 1.0 / (2.0 * l); rinv[l] = 1.0 / l; }
    for (int m = 0; m <= l; ++m) {
      if (l > m) rq[l][m] = 1.0 / ((double)(l + m) * (double)(l - m));
      rn[l][m] = std::sqrt(fact[l - m] * fact[l + m]);
    }
  }
  keep(cudaMemcpyToSymbolAsync(c_rq, rq, sizeof(rq), 0, cudaMemcpyHostToDevice, st));
  keep(cudaMemcpyToSymbolAsync(c_rn, rn, sizeof(rn), 0, cudaMemcpyHostToDevice, st));
  keep(cudaMemcpyToSymbolAsync(c_rd, rd, sizeof(rd), 0, cudaMemcpyHostToDevice, st));
  keep(cudaMemcpyToSymbolAsync(c_rinv, rinv, sizeof(rinv), 0, cudaMemcpyHostToDevice, st));
  double la[QOL_MAXNQ + 2] = {}, lb[QOL_MAXNQ + 2] = {};
  for (int k = 0; k < QOL_MAXNQ + 2; ++k) { la[k] = (2.0 * k + 1.0) / (k + 1.0); lb[k] = k / (k + 1.0); }
  keep(cudaMemcpyToSymbolAsync(c_la, la, sizeof(la), 0, cudaMemcpyHostToDevice, st));
  keep(cudaMemcpyToSymbolAsync(c_lb, lb, sizeof(lb), 0, cudaMemcpyHostToDevice, st));
  double rk[QOL_MAXNQ + 2] = {};
  for (int k = 1; k < QOL_MAXNQ + 2; ++k) rk[k] = 1.0 / k;
  keep(cudaMemcpyToSymbolAsync(c_rk, rk, sizeof(rk), 0, cudaMemcpyHostToDevice, st));
  static double jq[QOL_MAXL + 1][QOL_MAXL + 1][4];
  for (int a = 0; a <= QOL_MAXL; ++a)
    for (int b = 0; b <= QOL_MAXL; ++b) {
      const double al = 2.0 * a + 1.0, j = b;
      const double c1 = 2.0 * j * (j + al) * (2.0 * j + al - 2.0);
      const double c2 = (2.0 * j + al - 1.0) * (al * al);
      const double c3 = (2.0 * j + al - 2.0) * (2.0 * j + al - 1.0) * (2.0 * j + al);
      const double c4 = 2.0 * (j + al - 1.0) * (j - 1.0) * (2.0 * j + al);
      jq[a][b][0] = b >= 2 ? c2 / c1 : 0.0;
      jq[a][b][1] = b >= 2 ? c3 / c1 : 0.0;
      jq[a][b][2] = b >= 2 ? c4 / c1 : 0.0;
      jq[a][b][3] = 0.0;
    }
  keep(cudaMemcpyToSymbolAsync(g_jq, jq, sizeof(jq), 0, cudaMemcpyHostToDevice, st));
  keep(cudaStreamSynchronize(st)); /* the host tables above are locals */
  return err;
}

/* ===================================================================== */
/* K2: level of every (target, panel) pair, grouped per panel by level   */
/* ===================================================================== */
/* walk (patch_refine_mod.f90:740-771) over the quadtree of the first
 * nlevel-1 levels of plain 4-split sub-patches (children of q: 4q..4q+3): a
 * sub-patch whose ball excludes x joins the cut (bit: the sub-patch's index
 * after all coarser levels' sub-patches), one that contains it is split, and
 * containment at the last tree level fails the walk */
__device__ __forceinline__ bool cut_walk(const OrderTab& T, const LevelWS& W, int pan, const double* x,
                                         unsigned& cut) {
  unsigned act = 1u;
  int off = 0;
  cut = 0u;
  const int ntree = T.nlevel - 1;
  for (int il = 0; il < ntree; ++il) {
    const double* qp = W.sub[il] + (size_t)pan * T.nsub[il] * 4;
    unsigned nxt = 0u;
    for (int q = 0; q < T.nsub[il]; ++q) {
      if (!((act >> q) & 1u)) continue;
      const double a = x[0] - qp[4 * q], b = x[1] - qp[4 * q + 1], c = x[2] - qp[4 * q + 2];
      if (a * a + b * b + c * c > qp[4 * q + 3]) cut |= 1u << (off + q);
      else if (il == ntree - 1) return false;
      else nxt |= 0xFu << (4 * q);
    }
    if (!nxt) break;
    act = nxt;
    off += T.nsub[il];
  }
  return true;
}

__global__ void __launch_bounds__(128) k_classify(OrderTab T, PairIn Q, LevelWS W, PairWS G, int preset) {
  const int pan = blockIdx.x;
  const long long p0 = Q.tcxi[pan] - 1, m = Q.tcxi[pan + 1] - Q.tcxi[pan];
  __shared__ int cnt[8], warpc[4][8];
  __shared__ int base_l[8];
  if (threadIdx.x < 8) cnt[threadIdx.x] = 0;
  __syncthreads();
  /* pass 1: counts per level */
  for (long long t0 = 0; t0 < m; t0 += blockDim.x) {
    long long t = t0 + threadIdx.x;
    int lv = 0;
    if (t < m) {
      const double* x = Q.tcx + 3 * (p0 + t);
      const int pre = preset ? (int)G.level[p0 + t] : 0; /* a level the selector already accepted */
      lv = pre ? pre : T.nlevel + 1;
      if (T.adaptive && !pre) { /* the walk, then the finest level's balls (one_level at nlevel) */
        unsigned cut;
        if (cut_walk(T, W, pan, x, cut)) lv = QOL_LV_CUT;
        else {
          const int l = T.nlevel - 1;
          const double* qp = W.sub[l] + (size_t)pan * T.nsub[l] * 4;
          bool outside = true;
          for (int s = 0; s < T.nsub[l]; ++s) {
            double a = qp[4 * s] - x[0], b = qp[4 * s + 1] - x[1], c = qp[4 * s + 2] - x[2];
            if (a * a + b * b + c * c < qp[4 * s + 3]) { outside = false; break; }
          }
          lv = outside ? T.nlevel : T.nlevel + 1;
        }
      }
      for (int l = 0; l < T.nlevel && !pre && !T.adaptive; ++l) {
        const double* qp = W.sub[l] + (size_t)pan * T.nsub[l] * 4;
        bool outside = true;
        for (int s = 0; s < T.nsub[l]; ++s) {
          double a = qp[4 * s] - x[0], b = qp[4 * s + 1] - x[1], c = qp[4 * s + 2] - x[2];
          if (a * a + b * b + c * c < qp[4 * s + 3]) { outside = false; break; }
        }
        if (outside) { lv = l + 1; break; }
      }
      if (T.force_level > 0 && !pre && lv <= T.nlevel) lv = T.force_level;
      G.level[p0 + t] = (signed char)lv;
      atomicAdd(&cnt[lv], 1);
    }
  }
  __syncthreads();
  const int lmax = T.adaptive ? QOL_LV_CUT : T.nlevel + 1; /* the pair classes */
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int l = 1; l <= lmax; ++l) {
      base_l[l] = acc;
      G.cnt[(size_t)pan * 8 + l] = cnt[l];
      G.off[(size_t)pan * 8 + l] = acc;
      acc += cnt[l];
    }
  }
  __syncthreads();
  /* pass 2: deterministic compaction in target order */
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (long long t0 = 0; t0 < m; t0 += blockDim.x) {
    long long t = t0 + threadIdx.x;
    int lv = (t < m) ? (int)G.level[p0 + t] : 0;
    for (int l = 1; l <= lmax; ++l) {
      unsigned b = __ballot_sync(0xffffffffu, lv == l);
      if (lane == 0) warpc[wid][l] = __popc(b);
      __syncthreads();
      int before = 0;
      for (int w = 0; w < wid; ++w) before += warpc[w][l];
      int tot = 0;
      for (int w = 0; w < 4; ++w) tot += warpc[w][l];
      if (lv == l) {
        int pos = base_l[l] + before + __popc(b & ((1u << lane) - 1u));
        G.grp[p0 + pos] = (int)t;
      }
      __syncthreads();
      if (threadIdx.x == 0) base_l[l] += tot;
      __syncthreads();
    }
  }
}

/* ===================================================================== */
/* K3: level-resolved pairs: kernel rows on the level nodes contracted   */
/* with interpmat, minus the self-masked naive block, written as COO     */
/* values.  One CTA per (panel, level); chunks of 32 targets.            */
/* ===================================================================== */
#define DTT 32           /* targets per chunk */
#define DNT 32           /* level nodes per tile (8 DMMA k-steps) */
#define DKS (DTT + 4)    /* kernel-tile row stride: fragment loads hit 16 distinct bank pairs */
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
/* both addresses 16-byte aligned; .cg: through L2 only */
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
/* D = A (8x4, row) B (4x8, col) + D, FP64 tensor path; per lane a = A[lane/4][lane%4],
 * b = B[lane%4][lane/4], d = D[lane/4][2 (lane%4) + {0,1}] */
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}


/* ===================================================================== */
/* K1: refined levels of every panel                                     */
/* ===================================================================== */
/* Level nodes as one batched contraction per level: G_p (n_l x 9) = I_l (n_l x
 * hd) S_p (hd x 9), S_p = [x | x_t | x_p] at panel p's nodes.  LV_P panels per
 * CTA share the interpolation rows (B holds their 9 LV_P columns), each CTA
 * takes a chunk of at most LV_M rows of one level; FP64 tensor path
 * (m8n8k4), one m-block of 8 rows at a time per warp.  Epilogue per (node,
 * panel): normal x_p cross x_t normalised, area element |.| wt, the 7-field
 * SoA record. */
#define LV_P 8
#define LV_M 512
#define LV_CS (9 * LV_P + 4) /* B row stride (doubles, 12 mod 16): conflict-free fragment loads */
#define LV_ES (9 * LV_P + 1) /* epilogue staging row stride */
__global__ void __launch_bounds__(256, 2) k_level_nodes(OrderTab T, PanelIn P, LevelWS W, int npan) {
  const int hd = T.hd, KP = (hd + 3) & ~3, ncw = T.ncw;
  const int p0 = blockIdx.x * LV_P;
  int l = 0, c = blockIdx.y;
  for (; l < T.nlevel; ++l) {
    const int nc = (T.n[l] + LV_M - 1) / LV_M;
    if (c < nc) break;
    c -= nc;
  }
  if (l >= T.nlevel) return;
  const int n = T.n[l], r0 = c * LV_M, r1 = min(n, r0 + LV_M);
  const double* I = T.interp[l]; /* n x ncw, zero columns hd .. ncw-1 */
  const double* wt = T.wt[l];
  extern __shared__ __align__(16) double lsm[];
  double* S = lsm;                  /* KP x LV_CS */
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double* E = lsm + KP * LV_CS + w * 8 * LV_ES; /* this warp's 8 x LV_ES staging */
  for (int e = threadIdx.x; e < KP * 9 * LV_P; e += blockDim.x) {
    const int k = e / (9 * LV_P), col = e % (9 * LV_P), p = col / 9, f = col % 9;
    double v = 0.0;
    if (k < hd && p0 + p < npan) {
      const size_t g = (size_t)(p0 + p) * hd + k;
      const double* src = f < 3 ? P.sx : (f < 6 ? P.rts : P.rps);
      v = src[3 * g + f % 3];
    }
    S[k * LV_CS + col] = v;
  }
  __syncthreads();
  const int g = lane >> 2, t4 = lane & 3;
  const int nmb = (r1 - r0 + 7) / 8;
  for (int mb = w; mb < nmb; mb += 8) {
    const int row = r0 + 8 * mb + g;
    const bool rv = row < r1;
    const double* Ir = I + (size_t)(rv ? row : r0) * ncw + t4;
    double acc[9][2];
#pragma unroll
    for (int j = 0; j < 9; ++j) { acc[j][0] = 0.0; acc[j][1] = 0.0; }
#pragma unroll 4
    for (int ks = 0; ks < KP / 4; ++ks) {
      const double a = rv ? __ldg(Ir + 4 * ks) : 0.0;
      const double* Sb = S + (4 * ks + t4) * LV_CS + g;
#pragma unroll
      for (int j = 0; j < 9; ++j) dmma(acc[j][0], acc[j][1], a, Sb[8 * j]);
    }
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      E[g * LV_ES + 8 * j + 2 * t4] = acc[j][0];
      E[g * LV_ES + 8 * j + 2 * t4 + 1] = acc[j][1];
    }
    __syncwarp();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int it = lane + 32 * h, gi = it & 7, p = it >> 3, i = r0 + 8 * mb + gi;
      if (i < r1 && p0 + p < npan) {
        const double* v = E + gi * LV_ES + 9 * p;
        const double nx = v[7] * v[5] - v[8] * v[4];
        const double ny = v[8] * v[3] - v[6] * v[5];
        const double nz = v[6] * v[4] - v[7] * v[3];
        const double sp = sqrt(nx * nx + ny * ny + nz * nz);
        double* base = W.node[l] + (size_t)(p0 + p) * n * 7;
        base[0 * n + i] = v[0];
        base[1 * n + i] = v[1];
        base[2 * n + i] = v[2];
        base[3 * n + i] = nx / sp;
        base[4 * n + i] = ny / sp;
        base[5 * n + i] = nz / sp;
        base[6 * n + i] = sp * wt[i];
      }
    }
    __syncwarp();
  }
}
constexpr size_t level_nodes_smem(int hd) { return sizeof(double) * (((hd + 3) & ~3) * LV_CS + 8 * 8 * LV_ES); }

/* sub-patch centroids and squared near radii: one thread per (panel, level,
 * sub-patch), sums in node order as the reference's loop
 * (patch_refine_mod.f90:423-502) */
__global__ void __launch_bounds__(128) k_level_subs(OrderTab T, LevelWS W, int npan) {
  int nsubt = 0;
  for (int l = 0; l < T.nlevel; ++l) nsubt += T.nsub[l];
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)npan * nsubt) return;
  const int pan = (int)(e / nsubt);
  int s = (int)(e % nsubt), l = 0;
  while (s >= T.nsub[l]) { s -= T.nsub[l]; ++l; }
  const int n = T.n[l], ns = T.nsub[l];
  const double* base = W.node[l] + (size_t)pan * n * 7;
  const long long i0 = T.suboff[l][s], i1 = T.suboff[l][s + 1];
  double swsum = 0.0, q[3];
  for (long long i = i0; i < i1; ++i) swsum += base[6 * n + i];
  for (int d = 0; d < 3; ++d) {
    double acc = 0.0;
    for (long long i = i0; i < i1; ++i) acc += base[d * n + i] * base[6 * n + i];
    q[d] = acc / swsum;
  }
  double rmax2 = 0.0;
  for (long long i = i0; i < i1; ++i) {
    double d2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      const double t = base[d * n + i] - q[d];
      d2 += t * t;
    }
    rmax2 = fmax(rmax2, d2);
  }
  double* qp = W.sub[l] + ((size_t)pan * ns + s) * 4;
  qp[0] = q[0]; qp[1] = q[1]; qp[2] = q[2];
  const double d2 = T.dist * T.dist;
  qp[3] = (T.subtyp[l][s] == 1) ? d2 * fmax(rmax2, 0.5 * swsum) : d2 * fmax(rmax2, swsum);
}

/* the level sums of one (panel, level) item, by all threads of the CTA, in
 * chunks of DTT targets.  Tiles of DNT level nodes, double-buffered in shared
 * memory: the node data and interpolation rows of tile t+1 arrive by async
 * copy while the FP64 tensor path accumulates S and D (targets x hd) += K It
 * over tile t; then the kernel values KS, KD of tile t+1 are formed from the
 * staged nodes.  Warp w: targets 16 (w>>2) .. +15, columns 8 NB (w&3) .., NB
 * column blocks of 8.  dsm: direct_smem<NB>() bytes of dynamic shared memory */
template <int NB>
__device__ __forceinline__ void direct_item(const OrderTab& T, const PanelIn& P, const PairIn& Q, const LevelWS& W,
                                            const PairWS& G, const OutCOO& O, int pan, int l, double* dsm) {
  if (l >= T.nlevel) return;
  const int cntl = G.cnt[(size_t)pan * 8 + l + 1];
  if (cntl == 0) return;
  const int offl = G.off[(size_t)pan * 8 + l + 1];
  const int hd = T.hd, n = T.n[l];
  const long long p0 = Q.tcxi[pan] - 1, m = Q.tcxi[pan + 1] - Q.tcxi[pan];
  const double* node = W.node[l] + (size_t)pan * n * 7;
  const double* I = T.interp[l]; /* rows of NCW = T.ncw columns */
  constexpr int NCW = 32 * NB; /* padded columns */
  constexpr int ICS = NCW + 4; /* interpolation-tile row stride */
  constexpr int STG = 2 * DNT * DKS + DNT * ICS + 8 * DNT; /* doubles per stage: KS, KD, It, nodes (7 x DNT, padded) */
  double* tg = dsm + 2 * STG; /* DTT x 3 */
  int* tloc = (int*)(tg + 3 * DTT);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int tb0 = 16 * (w >> 2), cb0 = 8 * NB * (w & 3);
  const int fr = lane >> 2, fc = lane & 3;
  const double i4p = 1.0 / (4.0 * QOL_PI);
  const int ntile = (n + DNT - 1) / DNT;
  /* async copies of tile t into stage s: interpolation rows and the 7 node fields */
  auto fetch = [&](int t, int s) {
    double* It = dsm + s * STG + 2 * DNT * DKS;
    double* nd = It + DNT * ICS;
    const int n0 = t * DNT;
    for (int e = threadIdx.x; e < DNT * NCW / 2; e += blockDim.x) { /* 16-byte pieces */
      const int nn = e / (NCW / 2), c = 2 * (e % (NCW / 2)), i = n0 + nn;
      if (i < n) cp_async16(&It[nn * ICS + c], I + (size_t)i * NCW + c);
      else { It[nn * ICS + c] = 0.0; It[nn * ICS + c + 1] = 0.0; }
    }
    for (int e = threadIdx.x; e < 7 * DNT; e += blockDim.x) {
      const int f = e / DNT, nn = e % DNT, i = n0 + nn;
      if (i < n) cp_async8(&nd[f * DNT + nn], node + (size_t)f * n + i);
      else nd[f * DNT + nn] = 0.0;
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  /* kernel values of tile t (its nodes already staged in stage s) */
  auto kvals = [&](int t, int s, int nt) {
    double* KS = dsm + s * STG;
    double* KD = KS + DNT * DKS;
    const double* nd = KD + DNT * DKS + DNT * ICS;
    const int n0 = t * DNT;
    for (int e = threadIdx.x; e < DNT * DTT; e += blockDim.x) {
      const int nn = e / DTT, tt = e % DTT;
      double sv = 0.0, dv = 0.0;
      if (n0 + nn < n && tt < nt)
        sdl_kernel(tg[3 * tt] - nd[nn], tg[3 * tt + 1] - nd[DNT + nn], tg[3 * tt + 2] - nd[2 * DNT + nn],
                   nd[3 * DNT + nn], nd[4 * DNT + nn], nd[5 * DNT + nn], nd[6 * DNT + nn] * i4p, sv, dv);
      KS[nn * DKS + tt] = sv;
      KD[nn * DKS + tt] = dv;
    }
  };
  for (int c0 = 0; c0 < cntl; c0 += DTT) {
    const int nt = min(DTT, cntl - c0);
    __syncthreads();
    fetch(0, 0);
    if (threadIdx.x < DTT) {
      const int tl = threadIdx.x < nt ? G.grp[p0 + offl + c0 + threadIdx.x] : -1;
      tloc[threadIdx.x] = tl;
      for (int d = 0; d < 3; ++d) tg[3 * threadIdx.x + d] = tl >= 0 ? Q.tcx[3 * (p0 + tl) + d] : 0.0;
    }
    cp_async_wait_all();
    __syncthreads();
    kvals(0, 0, nt);
    __syncthreads();
    double cS[2][NB][2], cD[2][NB][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < NB; ++b) { cS[a][b][0] = cS[a][b][1] = 0.0; cD[a][b][0] = cD[a][b][1] = 0.0; }
    for (int t = 0; t < ntile; ++t) {
      const int s = t & 1;
      if (t + 1 < ntile) fetch(t + 1, s ^ 1);
      const double* KS = dsm + s * STG;
      const double* KD = KS + DNT * DKS;
      const double* It = KD + DNT * DKS;
      const int nn_max = min(DNT, n - t * DNT);
#pragma unroll 2
      for (int ks = 0; ks < DNT / 4; ++ks) {
        if (4 * ks >= nn_max) break;
        const int kr = 4 * ks + fc;
        const double aS0 = KS[kr * DKS + tb0 + fr], aS1 = KS[kr * DKS + tb0 + 8 + fr];
        const double aD0 = KD[kr * DKS + tb0 + fr], aD1 = KD[kr * DKS + tb0 + 8 + fr];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          const double bv = It[kr * ICS + cb0 + 8 * b + fr];
          dmma(cS[0][b][0], cS[0][b][1], aS0, bv);
          dmma(cS[1][b][0], cS[1][b][1], aS1, bv);
          dmma(cD[0][b][0], cD[0][b][1], aD0, bv);
          dmma(cD[1][b][0], cD[1][b][1], aD1, bv);
        }
      }
      if (t + 1 < ntile) {
        cp_async_wait_all();
        __syncthreads(); /* tile t+1's nodes staged; stage s^1's kernel values no longer read */
        kvals(t + 1, s ^ 1, nt);
      }
      __syncthreads(); /* tile t+1's kernel values visible; stage s free for tile t+2 */
    }
    /* naive block and the COO write */
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const int tt = tb0 + 8 * a + fr;
      if (tt >= nt) continue;
      const int tl = tloc[tt];
      const long long row = Q.tcxrow[p0 + tl];
      const double x0 = tg[3 * tt], x1 = tg[3 * tt + 1], x2 = tg[3 * tt + 2];
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int k = cb0 + 8 * b + 2 * fc + h;
          if (k >= hd) continue;
          double vs = cS[a][b][h], vd = cD[a][b][h];
          if (O.subtract_naive) {
            const size_t gj = (size_t)pan * hd + k;
            double ns = 0.0, nd = 0.0;
            if (row != (long long)gj + 1)
              sdl_kernel(x0 - P.sx[3 * gj], x1 - P.sx[3 * gj + 1], x2 - P.sx[3 * gj + 2], P.snx[3 * gj],
                         P.snx[3 * gj + 1], P.snx[3 * gj + 2], P.sw[gj] * i4p, ns, nd);
            vs -= ns; vd -= nd;
          }
          const size_t o = (size_t)p0 * hd + (size_t)k * m + tl;
          O.vs[o] = vs;
          O.vd[o] = vd;
        }
    }
  }
}
/* level sums of the adaptive cuts (adaptive_pass, patch_refine_mod.f90:617-718,
 * with cut_gI :720-738): one warp per pair, lanes over the hd output columns.
 * The cut's sub-patches in walk order (level by level, sub-patch order), their
 * nodes 32 at a time (one kernel value a lane, then shuffled), each node's
 * interpmat row contracted into the columns; minus the self-masked naive
 * block and written as COO values as k_direct does. */
#define CUT_MAXC 5 /* columns a lane: hd <= 160 */
__global__ void __launch_bounds__(256) k_direct_cut(OrderTab T, PanelIn P, PairIn Q, LevelWS W, PairWS G, OutCOO O,
                                                    int pan0) {
  const int pan = pan0 + blockIdx.x;
  const int cnt = G.cnt[(size_t)pan * 8 + QOL_LV_CUT];
  if (cnt == 0) return;
  const int off = G.off[(size_t)pan * 8 + QOL_LV_CUT];
  const long long p0 = Q.tcxi[pan] - 1, m = Q.tcxi[pan + 1] - Q.tcxi[pan];
  const int hd = T.hd, ncw = T.ncw, n1 = T.n[0];
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const double i4p = 1.0 / (4.0 * QOL_PI);
  for (int i = threadIdx.x >> 5; i < cnt; i += nw) {
    const int tl = G.grp[p0 + off + i];
    const double x[3] = {Q.tcx[3 * (p0 + tl)], Q.tcx[3 * (p0 + tl) + 1], Q.tcx[3 * (p0 + tl) + 2]};
    unsigned cut;
    cut_walk(T, W, pan, x, cut);
    double aS[CUT_MAXC], aD[CUT_MAXC];
#pragma unroll
    for (int j = 0; j < CUT_MAXC; ++j) aS[j] = aD[j] = 0.0;
    int lbase = 0;
    for (int il = 0; il < T.nlevel - 1; ++il) {
      const int n = T.n[il];
      const double* node = W.node[il] + (size_t)pan * n * 7;
      const double* I = T.interp[il];
      for (int q = 0; q < T.nsub[il]; ++q) {
        if (!((cut >> (lbase + q)) & 1u)) continue;
        const int kend = (q + 1) * n1;
        for (int k0 = q * n1; k0 < kend; k0 += 32) {
          const int k = k0 + lane;
          double sv = 0.0, dv = 0.0;
          if (k < kend)
            sdl_kernel(x[0] - node[k], x[1] - node[n + k], x[2] - node[2 * n + k], node[3 * n + k], node[4 * n + k],
                       node[5 * n + k], node[6 * n + k] * i4p, sv, dv);
          const int nk = min(32, kend - k0);
          for (int kk = 0; kk < nk; ++kk) {
            const double s = __shfl_sync(0xffffffffu, sv, kk), d = __shfl_sync(0xffffffffu, dv, kk);
            const double* Ir = I + (size_t)(k0 + kk) * ncw;
#pragma unroll
            for (int j = 0; j < CUT_MAXC; ++j) {
              const int c = lane + 32 * j;
              if (c < hd) {
                const double iv = Ir[c];
                aS[j] = fma(s, iv, aS[j]);
                aD[j] = fma(d, iv, aD[j]);
              }
            }
          }
        }
      }
      lbase += T.nsub[il];
    }
    const long long row = Q.tcxrow[p0 + tl];
#pragma unroll
    for (int j = 0; j < CUT_MAXC; ++j) {
      const int c = lane + 32 * j;
      if (c >= hd) continue;
      double vs = aS[j], vd = aD[j];
      if (O.subtract_naive) {
        const size_t gj = (size_t)pan * hd + c;
        double ns = 0.0, nd = 0.0;
        if (row != (long long)gj + 1)
          sdl_kernel(x[0] - P.sx[3 * gj], x[1] - P.sx[3 * gj + 1], x[2] - P.sx[3 * gj + 2], P.snx[3 * gj],
                     P.snx[3 * gj + 1], P.snx[3 * gj + 2], P.sw[gj] * i4p, ns, nd);
        vs -= ns; vd -= nd;
      }
      const size_t o = (size_t)p0 * hd + (size_t)c * m + tl;
      O.vs[o] = vs;
      O.vd[o] = vd;
    }
  }
}

/* one CTA per (panel, level) */
template <int NB>
__global__ void __launch_bounds__(256, 2) k_direct(OrderTab T, PanelIn P, PairIn Q, LevelWS W, PairWS G,
                                                   OutCOO O, int pan0) {
  extern __shared__ __align__(16) double dsm[];
  direct_item<NB>(T, P, Q, W, G, O, pan0 + blockIdx.x, blockIdx.y, dsm); /* panels pan0 .. pan0 + gridDim.x - 1 */
}

/* the level sums of many pipeline jobs (surfaces, orders) in one persistent
 * launch: every CTA takes the next (job, panel, level) item from a device
 * queue (items[3 i .. 3 i + 2], ordered by the host: finest level first, so
 * the longest items start first) until the queue is empty, and runs the same
 * item code as k_direct, so the values are k_direct's bit for bit */
template <int NBMAX>
__global__ void __launch_bounds__(256, 2) k_direct_queue(const DirectJob* jobs, const int* items, int nitems,
                                                         int* head) {
  extern __shared__ __align__(16) double dsm[];
  __shared__ int s_it;
  for (;;) {
    __syncthreads(); /* the previous item is done with shared memory */
    if (threadIdx.x == 0) s_it = atomicAdd(head, 1);
    __syncthreads();
    const int it = s_it;
    if (it >= nitems) return;
    const DirectJob& D = jobs[items[3 * it]];
    const int pan = items[3 * it + 1], l = items[3 * it + 2];
    switch (D.T.ncw / 32) {
      case 1: direct_item<1>(D.T, D.P, D.Q, D.W, D.G, D.O, pan, l, dsm); break;
      case 2: if (NBMAX >= 2) direct_item<(NBMAX >= 2 ? 2 : 1)>(D.T, D.P, D.Q, D.W, D.G, D.O, pan, l, dsm); break;
      case 3: if (NBMAX >= 3) direct_item<(NBMAX >= 3 ? 3 : 1)>(D.T, D.P, D.Q, D.W, D.G, D.O, pan, l, dsm); break;
      case 4: if (NBMAX >= 4) direct_item<(NBMAX >= 4 ? 4 : 1)>(D.T, D.P, D.Q, D.W, D.G, D.O, pan, l, dsm); break;
      case 5: if (NBMAX >= 5) direct_item<(NBMAX >= 5 ? 5 : 1)>(D.T, D.P, D.Q, D.W, D.G, D.O, pan, l, dsm); break;
      default: break;
    }
  }
}

template <int NB>
constexpr size_t direct_smem() {
  return sizeof(double) * (2 * (2 * DNT * DKS + DNT * (32 * NB + 4) + 8 * DNT) + 3 * DTT) + sizeof(int) * DTT;
}

/* ---------------------------------------------------------------------
 * FP32 form of the level sums (the precision variant) on the fifth-
 * generation tensor cores: kernel values in FP32 from coordinates taken
 * relative to the panel's first node (so that the FP32 differences keep
 * their relative accuracy), the contraction with the interpolation rows by
 * tcgen05.mma kind::tf32 with the 3xTF32 split (a b ~ a_lo b_hi + a_hi b_lo
 * + a_hi b_hi, a_hi = TF32 rounding of a, a_lo = TF32 rounding of the rest),
 * accumulated in FP32 in tensor memory over UG tiles of UNT nodes and as
 * compensated (Kahan) FP32 sums in registers across those groups, in FP64
 * from there on; the naive block in FP64.
 *
 * One CTA of UTHREADS threads per (panel, level), the finest level first,
 * chunks of UTT = 64 targets.  The MMA's 128 rows are the single-layer rows
 * of the chunk's targets (rows 0..63) and their double-layer rows (64..127),
 * its N the padded interpolation columns (ncw), its K the level nodes, UNT
 * to a tile.  Shared-memory operands in the K-major canonical layout without
 * swizzle (core matrices of 8 rows x 16 bytes): A as [node quad][row][4],
 * B as [node quad][column][4] (the host lays the interpolation tables out
 * so, tile after tile, and one bulk copy a part moves a tile).  UNS
 * pipeline stages: while the tensor cores work on tile t, the threads
 * compute tile t+1's kernel values and thread 0 has its interpolation rows
 * copied (an mbarrier counts their bytes); a stage is released by the
 * tcgen05.commit of the MMAs that read it, and two accumulator buffers in
 * tensor memory alternate between groups, so one is added into the FP64
 * registers while the MMAs fill the other.  Every wait
 * on an mbarrier is bounded (about a second); after a timeout the CTA sets
 * g_qol_wait_err, waits (bounded) for its MMAs in flight, frees its tensor
 * memory and returns.
 * --------------------------------------------------------------------- */
#define UTT 64        /* targets per chunk */
#define UNT 32        /* level nodes per tile (4 MMA k-steps of 8) */
#define UNS 3         /* pipeline stages */
#define UG 1          /* tiles per FP32 accumulation group */
#define UTHREADS 512
__device__ unsigned g_qol_wait_err; /* nonzero: a bounded wait of the FP32 level-sum kernel timed out */

/* TF32 rounding of an FP32 bit pattern: to nearest, ties away from zero (the
 * rounding of cvt.rna.tf32.f32), done on the integer pipes */
__device__ __forceinline__ unsigned tf32_rna_bits(unsigned u) { return (u + 0x1000u) & 0xFFFFE000u; }
/* hi = TF32 rounding of x, lo = TF32 rounding of x - hi */
__device__ __forceinline__ void tf32_split(float x, float& hi, float& lo) {
  hi = __uint_as_float(tf32_rna_bits(__float_as_uint(x)));
  lo = __uint_as_float(tf32_rna_bits(__float_as_uint(x - hi)));
}
/* D[tmem] (+)= A B, TF32 operands from shared memory, FP32 accumulate;
 * acc = 0 overwrites D */
__device__ __forceinline__ void umma_tf32(unsigned d, unsigned long long a, unsigned long long b, unsigned idesc,
                                          unsigned acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
/* 8 consecutive FP32 columns of this warp's 32 tensor-memory lanes, one lane
 * a thread, added into the compensated sums (a, c)[0..7] (the wait takes the
 * registers, so nothing reads them before the load has completed) */
__device__ __forceinline__ void tmem_add8(unsigned taddr, float* a, float* c) {
  unsigned v[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n"
               : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7])
               :
               : "memory");
#pragma unroll
  for (int e = 0; e < 8; ++e) { /* compensated (Kahan) FP32 sum: a + c carries about twice FP32's precision */
    const float y = __uint_as_float(v[e]) - c[e];
    const float t = a[e] + y;
    c[e] = __fsub_rn(__fsub_rn(t, a[e]), y);
    a[e] = t;
  }
}template <int NB>
struct UmmaShape {
  static constexpr int NCW = 32 * NB;                 /* MMA N: padded interpolation columns */
  static constexpr int ABYTES = 128 * UNT * 4;        /* one TF32 part of the A tile */
  static constexpr int BBYTES = NCW * UNT * 4;        /* one TF32 part of the B tile */
  static constexpr int NDOFF = 2 * ABYTES + 2 * BBYTES; /* the tile's node values: 7 x UNT floats */
  static constexpr int STG = (NDOFF + 7 * UNT * 4 + 1023) / 1024 * 1024;
  static constexpr unsigned NCOL = 2 * NCW <= 32 ? 32u : 2 * NCW <= 64 ? 64u : 2 * NCW <= 128 ? 128u
                                 : 2 * NCW <= 256 ? 256u : 512u; /* two accumulator buffers, a power of 2 */
  /* instruction descriptor: FP32 accumulator, TF32 A and B, both K-major, N, M = 128 */
  static constexpr unsigned IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(NCW >> 3) << 17) | (8u << 24);
  /* after the stages: 2 UNS mbarriers, the tensor-memory address, and per
   * target of the chunk its FP64 coordinates, row and local id */
  static constexpr size_t SMEM = (size_t)UNS * STG + 16 * UNS + 16 + (size_t)UTT * (24 + 8 + 4);
};
/* global -> shared bulk copy (no tensor map), completing on the mbarrier bar */
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

template <int NB>
__global__ void __launch_bounds__(UTHREADS, 1) k_direct_umma(OrderTab T, PanelIn P, PairIn Q, LevelWS W, PairWS G,
                                                            OutCOO O, int pan0) {
  using U = UmmaShape<NB>;
  constexpr int NCW = U::NCW, ABYTES = U::ABYTES, BBYTES = U::BBYTES, STG = U::STG;
  constexpr int ACOL = NCW / 4; /* accumulator columns of a thread */
  const int pan = pan0 + blockIdx.x, l = T.nlevel - 1 - (int)blockIdx.y; /* panels pan0 .., the finest level first */
  if (l < 0) return;
  const int cntl = G.cnt[(size_t)pan * 8 + l + 1];
  if (cntl == 0) return;
  extern __shared__ __align__(1024) unsigned char usm[];
  unsigned long long* mbar = reinterpret_cast<unsigned long long*>(usm + UNS * STG);
  unsigned* tslot = reinterpret_cast<unsigned*>(mbar + 2 * UNS);
  double* tg = reinterpret_cast<double*>(tslot + 4); /* UTT x 3 */
  long long* trow = reinterpret_cast<long long*>(tg + 3 * UTT);
  int* tloc = reinterpret_cast<int*>(trow + UTT);
  double* accs = reinterpret_cast<double*>(usm); /* [layer][NCW][UTT], the epilogue's sums: overlays the stages */
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned sbase = (unsigned)__cvta_generic_to_shared(usm);
  const unsigned md0 = (unsigned)__cvta_generic_to_shared(mbar); /* per stage: its MMAs are done */
  const unsigned bf0 = md0 + 8 * UNS;                             /* per stage: its interpolation rows have landed */
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     (unsigned)__cvta_generic_to_shared(tslot)),
                 "r"(U::NCOL)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < 2 * UNS; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(md0 + 8 * s) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const unsigned tmem = *tslot;

  const int offl = G.off[(size_t)pan * 8 + l + 1];
  const int hd = T.hd, n = T.n[l];
  const long long p0 = Q.tcxi[pan] - 1, m = Q.tcxi[pan + 1] - Q.tcxi[pan];
  const double* node = W.node[l] + (size_t)pan * n * 7;
  const unsigned* Ihg = T.interp_hi[l]; /* tiles of UNT rows in the B layout above */
  const unsigned* Ilg = T.interp_lo[l];
  const double i4p = 1.0 / (4.0 * QOL_PI);
  const double* pc = P.sx + (size_t)pan * hd * 3; /* the panel's first node */
  const double c0x = pc[0], c0y = pc[1], c0z = pc[2];
  const int ntile = (n + UNT - 1) / UNT;
  /* kernel values: target kr of the chunk, node quad kq of every tile */
  const int kr = tid % UTT, kq = tid / UTT;
  /* accumulators: tensor-memory lane quarter aq (rows 32 aq .. 32 aq + 31:
   * single layer for aq < 2), column quarter ac; row ar of the chunk */
  const int aq = warp & 3, ac = warp >> 2;
  const int ar = 32 * (aq & 1) + lane;
  const unsigned trow_t = tmem + ((unsigned)(32 * aq) << 16) + (unsigned)(ac * ACOL);
  /* node staging: field nf, node nn of a tile */
  const int nf = tid / UNT, nn = tid % UNT;
  auto node_load = [&](int t) -> double {
    const int i = t * UNT + nn;
    return (nf < 7 && i < n) ? node[(size_t)nf * n + i] : 0.0;
  };
  auto node_store = [&](int s, double v) {
    if (nf < 7) {
      float* nd = reinterpret_cast<float*>(usm + s * STG + U::NDOFF);
      const double c = nf == 0 ? c0x : nf == 1 ? c0y : nf == 2 ? c0z : 0.0;
      nd[nf * UNT + nn] = (float)(nf == 6 ? v * i4p : v - c);
    }
  };
  unsigned nfe = 0; /* thread 0: tiles whose interpolation rows were requested */
  auto fetch = [&](unsigned u, int t) { /* thread 0: tile t (the CTA's tile u) into stage u % UNS, one bulk copy a part */
    const unsigned s = u % UNS, bar = bf0 + 8 * s, dst = sbase + s * STG + 2 * ABYTES;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(2 * BBYTES) : "memory");
    bulk_g2s(dst, Ihg + (size_t)t * (BBYTES / 4), BBYTES, bar);
    bulk_g2s(dst + BBYTES, Ilg + (size_t)t * (BBYTES / 4), BBYTES, bar);
    nfe = u + 1;
  };
  auto drain = [&](int buf, float* acc, float* cmp) {
#pragma unroll
    for (int j = 0; j < NB; ++j) tmem_add8(trow_t + (unsigned)(buf * NCW + 8 * j), acc + 8 * j, cmp + 8 * j);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  };

  /* branches depend only on values every thread agrees on (a wait's outcome
   * is collected into to and made common at the next barrier), so every
   * thread reaches the barriers and the warp-wide tensor-memory loads */
  unsigned tc = 0; /* tiles committed by this CTA: tile u used stage u % UNS in its phase (u / UNS) & 1 */
  int to = 0;      /* a wait timed out */
  for (int c0 = 0; c0 < cntl && !to; c0 += UTT) {
    const int nt = min(UTT, cntl - c0);
    __syncthreads(); /* the previous chunk's epilogue is done with the stages and the target data */
    if (tid < UTT) {
      const int tl = tid < nt ? G.grp[p0 + offl + c0 + tid] : -1;
      tloc[tid] = tl;
      trow[tid] = tl >= 0 ? Q.tcxrow[p0 + tl] : 0;
      for (int d = 0; d < 3; ++d) tg[3 * tid + d] = tl >= 0 ? Q.tcx[3 * (p0 + tl) + d] : 0.0;
    }
    if (tid == 0) fetch(tc, 0);
    node_store(tc % UNS, node_load(0));
    __syncthreads(); /* target data and tile 0's node values staged */
    const bool kv = kr < nt;
    const float xr = (float)(tg[3 * kr] - c0x), yr = (float)(tg[3 * kr + 1] - c0y), zr = (float)(tg[3 * kr + 2] - c0z);
    float acc[ACOL], cmp[ACOL]; /* compensated FP32 sums across the groups: acc - cmp */
#pragma unroll
    for (int j = 0; j < ACOL; ++j) acc[j] = cmp[j] = 0.0f;
    for (int t = 0; t < ntile; ++t, ++tc) {
      const int s = tc % UNS, s1 = (tc + 1) % UNS;
      double nv = 0.0;
      if (t + 1 < ntile) {
        /* stage s1 is free once tile tc + 1 - UNS's MMAs are done: thread 0
         * waits for that before its copy into s1, and the barrier below
         * orders every other thread's writes into s1 after its wait */
        if (tid == 0) {
          if (tc + 1 >= UNS) to |= !mbar_wait_bounded(md0 + 8 * s1, ((tc + 1 - UNS) / UNS) & 1);
          fetch(tc + 1, t + 1);
        }
        nv = node_load(t + 1);
      }
      { /* tile t's kernel values: target kr, nodes 4 kq .. 4 kq + 3, as TF32 parts */
        const float* nd = reinterpret_cast<const float*>(usm + s * STG + U::NDOFF);
        const float4 X = *reinterpret_cast<const float4*>(nd + 4 * kq);
        const float4 Y = *reinterpret_cast<const float4*>(nd + UNT + 4 * kq);
        const float4 Z = *reinterpret_cast<const float4*>(nd + 2 * UNT + 4 * kq);
        const float4 NX = *reinterpret_cast<const float4*>(nd + 3 * UNT + 4 * kq);
        const float4 NY = *reinterpret_cast<const float4*>(nd + 4 * UNT + 4 * kq);
        const float4 NZ = *reinterpret_cast<const float4*>(nd + 5 * UNT + 4 * kq);
        const float4 WW = *reinterpret_cast<const float4*>(nd + 6 * UNT + 4 * kq);
        const float xs[4] = {X.x, X.y, X.z, X.w}, ys[4] = {Y.x, Y.y, Y.z, Y.w}, zs[4] = {Z.x, Z.y, Z.z, Z.w};
        const float nxs[4] = {NX.x, NX.y, NX.z, NX.w}, nys[4] = {NY.x, NY.y, NY.z, NY.w};
        const float nzs[4] = {NZ.x, NZ.y, NZ.z, NZ.w}, ws[4] = {WW.x, WW.y, WW.z, WW.w};
        float sh[4], sl[4], dh[4], dl[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float dx = xr - xs[i], dy = yr - ys[i], dz = zr - zs[i];
          const float rr = dx * dx + dy * dy + dz * dz;
          float sv = 0.0f, dv = 0.0f;
          if (kv && rr > 1.0e-28f) {
            const float ri = rsqrtf(rr);
            sv = ws[i] * ri;
            dv = sv * ri * ri * (dx * nxs[i] + dy * nys[i] + dz * nzs[i]);
          }
          tf32_split(sv, sh[i], sl[i]);
          tf32_split(dv, dh[i], dl[i]);
        }
        unsigned char* A = usm + s * STG;
        const int oS = (kq * 128 + kr) * 16, oD = (kq * 128 + UTT + kr) * 16;
        *reinterpret_cast<float4*>(A + oS) = make_float4(sh[0], sh[1], sh[2], sh[3]);
        *reinterpret_cast<float4*>(A + ABYTES + oS) = make_float4(sl[0], sl[1], sl[2], sl[3]);
        *reinterpret_cast<float4*>(A + oD) = make_float4(dh[0], dh[1], dh[2], dh[3]);
        *reinterpret_cast<float4*>(A + ABYTES + oD) = make_float4(dl[0], dl[1], dl[2], dl[3]);
      }
      if (t + 1 < ntile) node_store(s1, nv);
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); /* the A tile visible to the tensor cores */
      to = __syncthreads_or(to);
      if (to) break;
      if (tid == 0) {
        to |= !mbar_wait_bounded(bf0 + 8 * s, (tc / UNS) & 1); /* tile t's interpolation rows have landed */
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        /* descriptors of stage 0 advanced by (bytes >> 4): the start address is
         * the low 14 bits and every shared address here is below 256 KB */
        const unsigned long long a0 = umma_desc(sbase, 2048, 128) + (unsigned)(s * STG >> 4);
        const unsigned long long b0 = umma_desc(sbase + 2 * ABYTES, 16 * NCW, 128) + (unsigned)(s * STG >> 4);
        const unsigned d = tmem + (unsigned)(((t / UG) & 1) * NCW);
#pragma unroll
        for (int ks = 0; ks < UNT / 8; ++ks) {
          const unsigned long long ah = a0 + 256 * ks, al = ah + (ABYTES >> 4);
          const unsigned long long bh = b0 + 2 * NCW * ks, bl = bh + (BBYTES >> 4);
          umma_tf32(d, al, bh, U::IDESC, (t % UG) | ks);
          umma_tf32(d, ah, bl, U::IDESC, 1u);
          umma_tf32(d, ah, bh, U::IDESC, 1u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(md0 + 8 * s)
                     : "memory");
      }
      if (t % UG == 0 && t > 0) { /* group t / UG - 1 is complete with tile tc - 1: add it up */
        to |= !mbar_wait_bounded(md0 + 8 * ((tc - 1) % UNS), ((tc - 1) / UNS) & 1);
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        drain((t / UG - 1) & 1, acc, cmp);
      }
    }
    if (__syncthreads_or(to)) { to = 1; break; }
    to |= !mbar_wait_bounded(md0 + 8 * ((tc - 1) % UNS), ((tc - 1) / UNS) & 1); /* the last group */
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    drain(((ntile - 1) / UG) & 1, acc, cmp);
    to = __syncthreads_or(to); /* every MMA and copy of the chunk is complete: the stages are free */
    if (to) break;
#pragma unroll
    for (int j = 0; j < ACOL; ++j) accs[((aq < 2 ? 0 : NCW) + ac * ACOL + j) * UTT + ar] = (double)acc[j] - (double)cmp[j];
    __syncthreads();
    /* naive block (FP64) and the COO write, a thread per (column, target):
     * consecutive threads take consecutive targets of a column */
    for (int e = tid; e < hd * nt; e += UTHREADS) {
      const int k = e / nt, r = e - k * nt;
      double vs = accs[k * UTT + r], vd = accs[(NCW + k) * UTT + r];
      if (O.subtract_naive) {
        const size_t gj = (size_t)pan * hd + k;
        double ns = 0.0, ndv = 0.0;
        if (trow[r] != (long long)gj + 1)
          sdl_kernel(tg[3 * r] - P.sx[3 * gj], tg[3 * r + 1] - P.sx[3 * gj + 1], tg[3 * r + 2] - P.sx[3 * gj + 2],
                     P.snx[3 * gj], P.snx[3 * gj + 1], P.snx[3 * gj + 2], P.sw[gj] * i4p, ns, ndv);
        vs -= ns; vd -= ndv;
      }
      const size_t o = (size_t)p0 * hd + (size_t)k * m + tloc[r];
      O.vs[o] = vs;
      O.vd[o] = vd;
    }
  }
  if (to) { /* a wait timed out: flag it, let the MMAs and copies in flight finish (bounded), free the tensor memory */
    if (tid == 0) {
      atomicOr(&g_qol_wait_err, 1u);
      if (tc > 0) mbar_wait_bounded(md0 + 8 * ((tc - 1) % UNS), ((tc - 1) / UNS) & 1);
      for (unsigned u = tc; u < nfe; ++u) mbar_wait_bounded(bf0 + 8 * (u % UNS), (u / UNS) & 1);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(U::NCOL) : "memory");
  }
}

/* ===================================================================== */
/* harmonic column evaluation (shared by K4 and K5)                      */
/* ===================================================================== */
/* column m of the Schmidt solid harmonics at frame point (x,y,z); calls
 * f(l, k, h, gx, gy, gz) for l = m..L with the sin-type value and frame
 * gradient.  Same recurrences as the oracle. */
template <class F>
__device__ __forceinline__ void harm_column(int L, int m, double x, double y, double z, F f) {
  const double X = y, Y = z, Z = x;
  const double r2 = X * X + Y * Y + Z * Z;
  cd Pm = mk(1.0, 0.0), Pm1 = mk(0.0, 0.0);
  const cd w = mk(X, Y);
  for (int mm = 1; mm <= m; ++mm) {
    double cm = c_hcm[mm];
    cd Smm = cscale(cm, cmul(w, Pm));
    cd dSmm = cscale(cm, cadd(Pm, cmul(w, Pm1)));
    Pm1 = dSmm; Pm = Smm;
  }
  cd s1 = Pm, s1x = Pm1, s1y = mk(-Pm1.im, Pm1.re), s1z = mk(0.0, 0.0);
  cd s2 = mk(0.0, 0.0), s2x = s2, s2y = s2, s2z = s2;
  f(m, m * (m - 1) / 2 + (m - 1), s1.im, s1z.im, s1x.im, s1y.im);
  for (int l = m + 1; l <= L; ++l) {
    double a = (2.0 * l - 1.0), b = c_hb[l][m], c = c_hc[l][m];
    cd s, sx, sy, sz;
    s = cscale(c, csub(cscale(a * Z, s1), cscale(b * r2, s2)));
    sx = cscale(c, csub(cscale(a * Z, s1x), cscale(b, cadd(cscale(2.0 * X, s2), cscale(r2, s2x)))));
    sy = cscale(c, csub(cscale(a * Z, s1y), cscale(b, cadd(cscale(2.0 * Y, s2), cscale(r2, s2y)))));
    sz = cscale(c, csub(cscale(a, cadd(s1, cscale(Z, s1z))), cscale(b, cadd(cscale(2.0 * Z, s2), cscale(r2, s2z)))));
    s2 = s1; s2x = s1x; s2y = s1y; s2z = s1z;
    s1 = s; s1x = sx; s1y = sy; s1z = sz;
    f(l, l * (l - 1) / 2 + (m - 1), s.im, sz.im, sx.im, sy.im);
  }
}

/* ===================================================================== */
/* K4: per-panel RRQ precompute                                          */
/* ===================================================================== */
__device__ __forceinline__ void qmul(const double* a, const double* b, double* c) {
  c[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  c[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  c[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
  c[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}

/* per-panel RRQ frame and boundary (every thread of the CTA calls it): the panel's nodes into s_sx, the boundary and vertices
 * from the interpolant (or the caller's chart) into s_raw, the frame
 * (R, c, alpha: lap3d_close_mod.f90:503-509, alpha = 1.25/sqrt(2 sum sw)
 * :709) into s_fr; rank 0 of the cluster writes the per-panel outputs (frame,
 * boundary in the frame, its t-derivative and Legendre coefficients, the
 * Koornwinder coefficients of the frame node positions). */
__device__ void panel_frame_setup(const OrderTab& T, const PanelIn& P, const RRQWS& R, const double* chart, int pan,
                                  int rank, double* s_sx, double* s_raw, double* s_fr) {
  const int hd = T.hd, nq = T.nquad, nbd = 3 * nq;
  for (int e = threadIdx.x; e < 3 * hd; e += blockDim.x) s_sx[e] = P.sx[(size_t)pan * hd * 3 + e];
  __syncthreads();
  /* boundary + vertices from the interpolant, or the caller's chart */
  for (int i = threadIdx.x; i < nbd + 3; i += blockDim.x) {
    double a[3] = {0.0, 0.0, 0.0};
    if (chart) {
      for (int d = 0; d < 3; ++d) a[d] = chart[(size_t)pan * 3 * (nbd + 3) + 3 * i + d];
    } else {
      for (int j = 0; j < hd; ++j) {
        double mb = T.Mb[(size_t)i * hd + j];
        a[0] += mb * s_sx[3 * j]; a[1] += mb * s_sx[3 * j + 1]; a[2] += mb * s_sx[3 * j + 2];
      }
    }
    s_raw[3 * i] = a[0]; s_raw[3 * i + 1] = a[1]; s_raw[3 * i + 2] = a[2];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    /* frame from the vertex triangle: e1 along v2-v1, e3 its normal, origin
     * the circumcentre shifted below the lowest node */
    const double* v1 = &s_raw[3 * nbd];
    const double* v2 = v1 + 3;
    const double* v3 = v1 + 6;
    double a[3], b[3], nn[3], e1[3], e2[3];
    for (int d = 0; d < 3; ++d) { a[d] = v2[d] - v1[d]; b[d] = v3[d] - v1[d]; }
    cross3(a, b, nn);
    double nl = sqrt(dot3(nn, nn));
    for (int d = 0; d < 3; ++d) nn[d] /= nl;
    double la = sqrt(dot3(a, a));
    for (int d = 0; d < 3; ++d) e1[d] = a[d] / la;
    cross3(nn, e1, e2);
    double Rm[9];
    for (int d = 0; d < 3; ++d) { Rm[0 + 3 * d] = e1[d]; Rm[1 + 3 * d] = e2[d]; Rm[2 + 3 * d] = nn[d]; }
    double axb[3], pp[3], qq[3], cc[3];
    cross3(a, b, axb);
    double aa = dot3(a, a), bb = dot3(b, b), den = 2.0 * dot3(axb, axb);
    for (int d = 0; d < 3; ++d) pp[d] = aa * b[d] - bb * a[d];
    cross3(pp, axb, qq);
    for (int d = 0; d < 3; ++d) cc[d] = v1[d] + qq[d] / den;
    double swsum = 0.0;
    for (int j = 0; j < hd; ++j) swsum += P.sw[(size_t)pan * hd + j];
    double alpha = 1.25 / sqrt(2.0 * swsum);
    double zmin = 1e300;
    for (int j = 0; j < hd; ++j) {
      double d0 = s_sx[3 * j] - cc[0], d1 = s_sx[3 * j + 1] - cc[1], d2 = s_sx[3 * j + 2] - cc[2];
      double zz = alpha * (Rm[2] * d0 + Rm[5] * d1 + Rm[8] * d2);
      zmin = fmin(zmin, zz);
    }
    double sx3min = fmax(0.0, -zmin);
    for (int i = 0; i < 9; ++i) s_fr[i] = Rm[i];
    for (int d = 0; d < 3; ++d) s_fr[9 + d] = cc[d] - (1.25 * sx3min / alpha) * Rm[2 + 3 * d];
    s_fr[12] = alpha;
  }
  __syncthreads();
  const double alpha = s_fr[12];
  auto tofr = [&](const double* x, double* y) {
    double d0 = x[0] - s_fr[9], d1 = x[1] - s_fr[10], d2 = x[2] - s_fr[11];
    for (int i = 0; i < 3; ++i) y[i] = alpha * (s_fr[i] * d0 + s_fr[i + 3] * d1 + s_fr[i + 6] * d2);
  };
  if (rank == 0) { /* per-panel outputs: frame, boundary, Legendre coefficients, node coefficients */
    double* fr = R.frame + (size_t)pan * RRQ_FRAME;
    double* bx = R.bx + (size_t)pan * 3 * nbd;
    double* bt = R.bt + (size_t)pan * 3 * nbd;
    double* cf = R.cf + (size_t)pan * 9 * nq;
    double* scf = R.scf + (size_t)pan * 3 * hd;
    for (int i = threadIdx.x; i < RRQ_FRAME; i += blockDim.x) fr[i] = i < 13 ? s_fr[i] : 0.0;
    for (int i = threadIdx.x; i < nbd; i += blockDim.x) {
      double y[3];
      tofr(&s_raw[3 * i], y);
      for (int d = 0; d < 3; ++d) { bx[3 * i + d] = y[d]; s_raw[3 * i + d] = y[d]; }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 3 * 3 * nq; e += blockDim.x) {
      int ed = e / (3 * nq), r = e % (3 * nq), d = r / nq, q = r % nq;
      double s = 0.0, sc = 0.0;
      for (int k = 0; k < nq; ++k) {
        double v = s_raw[3 * (ed * nq + k) + d];
        s += T.Dgl[q + nq * k] * v;
        sc += T.Leg[q + nq * k] * v;
      }
      bt[3 * (ed * nq + q) + d] = s;
      cf[ed * 3 * nq + d * nq + q] = sc;
    }
    for (int e = threadIdx.x; e < 3 * hd; e += blockDim.x) {
      int d = e / hd, k = e % hd;
      double s = 0.0;
      for (int j = 0; j < hd; ++j) {
        double y[3];
        tofr(&s_sx[3 * j], y);
        s += T.umatr[k + (size_t)hd * j] * y[d];
      }
      scf[d * hd + k] = s;
    }
    for (int j = threadIdx.x; j < hd; j += blockDim.x) {
      double y[3];
      tofr(&s_sx[3 * j], y);
      for (int d = 0; d < 3; ++d) R.sxf[(size_t)pan * 3 * hd + 3 * j + d] = y[d];
    }
  }
}

/* B = PS H^T for rows c0 .. c0 + nc - 1 of one panel: B[i][j] = sum_k PS[i][k]
 * h_k(y_j) on the FP64 tensor path (m8n8k4): PS rows (A) and H rows (B^T)
 * staged in K tiles in the CTA's shared memory (room doubles, all dead by
 * now), zero padded; warp w takes the column blocks w, w + NW, .. with every
 * row block.  PS (global) must be complete and visible: the caller fences and
 * synchronises the cluster first. */
__device__ void panel_b_epilogue(const RRQWS& R, int hd, int pan, int c0, int nc, int room, double* psm) {
  const double* PS = R.smat + (size_t)pan * hd * hd;
  const double* H = R.hmat + (size_t)pan * hd * hd;
  {
    double* B = R.B + (size_t)pan * hd * hd;
    const int MBn = (nc + 7) / 8, NBn = (hd + 7) / 8, rows = 8 * (MBn + NBn), KP = (hd + 3) & ~3;
    auto skf = [](int kt) { return (kt % 16 == 4 || kt % 16 == 12) ? kt : kt + 4; }; /* conflict-free strides */
    int KT = KP;
    while (KT > 4 && rows * skf(KT) > room) KT -= 4;
    const int SK = skf(KT);
    double* sP = psm;                         /* 8 MBn x SK */
    double* sH = psm + (size_t)8 * MBn * SK;  /* 8 NBn x SK */
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int NT = blockDim.x, NW = NT / 32;
    constexpr int MBX = 9, NBX = 2; /* row blocks <= 9, column blocks a warp <= 2 */
    double acc[NBX][MBX][2];
#pragma unroll
    for (int u = 0; u < NBX; ++u)
#pragma unroll
      for (int v = 0; v < MBX; ++v) { acc[u][v][0] = 0.0; acc[u][v][1] = 0.0; }
    for (int k0 = 0; k0 < KP; k0 += KT) {
      __syncthreads();
      for (int e = threadIdx.x; e < 8 * MBn * KT; e += NT) {
        const int i = e / KT, kk = e % KT, k = k0 + kk;
        sP[i * SK + kk] = (i < nc && k < hd) ? PS[(size_t)(c0 + i) * hd + k] : 0.0;
      }
      for (int e = threadIdx.x; e < 8 * NBn * KT; e += NT) {
        const int j = e / KT, kk = e % KT, k = k0 + kk;
        sH[j * SK + kk] = (j < hd && k < hd) ? H[(size_t)j * hd + k] : 0.0;
      }
      __syncthreads();
      const int kst = min(KT, KP - k0) / 4;
      for (int ks = 0; ks < kst; ++ks) {
        const int kc = 4 * ks + (lane & 3);
#pragma unroll
        for (int u = 0; u < NBX; ++u) {
          const int nb = wid + NW * u;
          if (nb >= NBn) continue;
          const double bv = sH[(8 * nb + (lane >> 2)) * SK + kc];
#pragma unroll
          for (int v = 0; v < MBX; ++v)
            if (v < MBn) dmma(acc[u][v][0], acc[u][v][1], sP[(8 * v + (lane >> 2)) * SK + kc], bv);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < NBX; ++u) {
      const int nb = wid + NW * u;
      if (nb >= NBn) continue;
#pragma unroll
      for (int v = 0; v < MBX; ++v) {
        const int i = 8 * v + (lane >> 2);
        if (v >= MBn || i >= nc) continue;
#pragma unroll
        for (int h2 = 0; h2 < 2; ++h2) {
          const int j = 8 * nb + 2 * (lane & 3) + h2;
          if (j < hd) B[(size_t)(c0 + i) * hd + j] = acc[u][v][h2];
        }
      }
    }
  }
}

/* ---------------------------------------------------------------------
 * Per-panel RRQ precompute: the inverses of the quaternion system V (hd x hd,
 * V[j][k] = (0, grad h_k(y_j)), the real form of the reference's MD,
 * lap3d_close_mod.f90:851-858) and of the real S system MS (Msl^T, :861-863)
 * by a blocked Gauss-Jordan elimination with row pivoting (largest quaternion
 * norm / magnitude among the unused rows of the pivot column, no row moves;
 * the inverse is X^-1[k][c] = X[pi(k)][pi^-1(c)] with pi the pivot sequence),
 * one cluster of CS CTAs a panel, each CTA holding ncol of the columns of
 * both systems in shared memory (orders up to nterms 16 with CS <= 8).
 * Columns are taken PB_NB = 8 at a time.  The CTA owning a block eliminates
 * within the block's 8 columns alone (the panel phase: 8 column steps,
 * register-resident, one named barrier a step) and publishes the block M and
 * its pivot rows P to every CTA of the cluster through distributed shared
 * memory; every CTA then applies the block's 8 steps to its other columns at
 * once, X[:, J] <- X[:, J] (rows P set to 0) + M X[P, J], on the FP64 tensor
 * path (mma m8n8k4): for the quaternion system the real GEMM (4 hd x 32)
 * (32 x ncol) with A the left-multiplication matrices of M's entries, built
 * in the fragment loads (entry c^d of M[i][b], sign from a table), B the
 * pivot rows' components; for the real system the GEMM (hd x 8) (8 x ncol).
 * Two cluster barriers a block (12 blocks at hdim 91).  Then PD, PS and
 * B = PS H^T (tensor path).
 * Shared memory per CTA (doubles): Xq 4 planes of hq x RS (V's columns of this
 * CTA, component-major), Xr hr x RS (MS's columns), Mq hq x 8 x 4 and Mr
 * hr x 8 (the published block), the step's pivot column (two buffers),
 * pivot bookkeeping.  hq = hd rounded up to 2 (8 real rows), hr to 8, ncol =
 * ceil(hd / CS) rounded up to 8, RS = ncol + 1.
 * --------------------------------------------------------------------- */
constexpr int PB_NB = 8;
constexpr int PB_MAXT = 512; /* threads a CTA: two warps per 8-column tile, at most 8 tiles */
/* barrier of the first nthreads threads of the CTA (a multiple of 32) */
__device__ __forceinline__ void named_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(nthreads) : "memory");
}
__host__ __device__ constexpr int pblk_ncol(int hd, int CS) { return (((hd + CS - 1) / CS) + 7) & ~7; }
__host__ __device__ constexpr int pblk_hq(int hd) { return (hd + 1) & ~1; }
__host__ __device__ constexpr int pblk_hr(int hd) { return (hd + 7) & ~7; }
/* row stride of the matrices: odd, so a column's rows fall in distinct banks */
__host__ __device__ constexpr int pblk_rs(int hd, int CS) { return pblk_ncol(hd, CS) + 1; }
/* plane stride of V's components: 8 (mod 16) doubles, so the four components
 * of a tensor-core tile row fall in different banks */
__host__ __device__ constexpr int pblk_plane(int hd, int CS) {
  return pblk_hq(hd) * pblk_rs(hd, CS) + ((8 - (pblk_hq(hd) * pblk_rs(hd, CS)) % 16) + 16) % 16;
}
__host__ __device__ constexpr size_t pblk_smem_bytes(int hd, int CS) {
  return sizeof(double) * ((size_t)4 * pblk_plane(hd, CS) + (size_t)pblk_hr(hd) * pblk_rs(hd, CS) +
                           (size_t)pblk_hq(hd) * PB_NB * 4 + (size_t)pblk_hr(hd) * PB_NB +
                           2 * ((size_t)pblk_hq(hd) * 4 + pblk_hr(hd) + 8)) +
         sizeof(int) * ((size_t)2 * pblk_hq(hd) + 2 * pblk_hr(hd) + 4 * (size_t)hd + 4);
}
__host__ __device__ constexpr int pblk_threads(int hd, int CS) {
  return 64 * (pblk_ncol(hd, CS) / 8) > PB_MAXT ? PB_MAXT
         : (64 * (pblk_ncol(hd, CS) / 8) < 32 * PB_NB ? 32 * PB_NB : 64 * (pblk_ncol(hd, CS) / 8));
}
/* sign of entry (c, d) of the left-multiplication matrix of a quaternion a,
 * whose entry is sign * a[c ^ d]: rows (+---), (++-+), (+++-), (+-++) */
__device__ __forceinline__ double lmul_sign(int c, int d) {
  return ((0x284Eu >> (4 * c + d)) & 1u) ? -1.0 : 1.0;
}

template <int CS, int PB_MAXS /* row slots of a lane in the panel phase: hq <= 32 PB_MAXS */>
__global__ void __launch_bounds__(PB_MAXT, 1) k_rrq_panel_blk(OrderTab T, PanelIn P, PairWS G, RRQWS R,
                                                                const double* chart /* nullable */) {
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int pan = R.plo + (int)(blockIdx.x / CS);
  if (G.cnt[(size_t)pan * 8 + T.nlevel + 1] == 0 && !R.all_panels) return; /* whole cluster */
  const int hd = T.hd, nq = T.nquad, nbd = 3 * nq, L = T.nterms;
  const int ncol = pblk_ncol(hd, CS), hq = pblk_hq(hd), hr = pblk_hr(hd), PL = pblk_plane(hd, CS);
  const int RS = pblk_rs(hd, CS); /* row stride of Xq's planes and of Xr */
  const int c0 = rank * ncol; /* this CTA's columns c0 .. c0 + ncol - 1 (those < hd valid) */
  const int NT = blockDim.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, NW = NT >> 5;
  extern __shared__ __align__(16) double psm[];
  double* Xq = psm;                           /* [comp][row][col], plane stride PL */
  double* Xr = Xq + 4 * (size_t)PL;           /* [row][col] */
  double* Mq = Xr + (size_t)hr * RS;          /* [row][b][comp] */
  double* Mr = Mq + (size_t)hq * PB_NB * 4;   /* [row][b] */
  double* fq = Mr + (size_t)hr * PB_NB;       /* the step's pivot columns, 2 buffers: [buf][V comp][row], MS */
  int* usedq = (int*)(fq + 2 * ((size_t)4 * hq + hr + 8));
  int* usedr = usedq + hq;
  int* isPq = usedr + hr; /* rows of the current block's pivots */
  int* isPr = isPq + hq;
  int* pivq = isPr + hr;  /* pivot row of each column, V then MS */
  int* pivr = pivq + hd;
  int* posq = pivr + hd;  /* inverse permutations */
  int* posr = posq + hd;
  int* pidx = posr + hd;  /* the step's pivot rows (V, MS), 2 buffers */
  /* geometry staging aliases the block buffers (free until the first block) */
  double* s_sx = Mq;
  double* s_raw = s_sx + 3 * hd;
  double* s_fr = s_raw + 3 * (nbd + 3);
  panel_frame_setup(T, P, R, chart, pan, rank, s_sx, s_raw, s_fr);
  const double alpha = s_fr[12];
  /* zero the matrices (padding rows and columns stay zero) and the bookkeeping */
  for (int e = tid; e < 4 * PL + hr * RS; e += NT) Xq[e] = 0.0;
  for (int e = tid; e < hq; e += NT) usedq[e] = e >= hd; /* padding rows never pivot */
  for (int e = tid; e < hr; e += NT) usedr[e] = e >= hd;
  __syncthreads();
  /* basis at the nodes: V[j][k] = (0, grad h_k(y_j)) for this CTA's harmonics
   * k, MS[k][j] = n_j . grad h_k(y_j) for this CTA's nodes j, H rows of its nodes */
  double* H = R.hmat + (size_t)pan * hd * hd; /* H[j*hd+k] = h_k(y_j) */
  for (int e = tid; e < hd * L; e += NT) {
    const int j = e / L, m = e % L + 1;
    double y[3], nrm[3];
    {
      const double d0 = s_sx[3 * j] - s_fr[9], d1 = s_sx[3 * j + 1] - s_fr[10], d2 = s_sx[3 * j + 2] - s_fr[11];
#pragma unroll
      for (int i = 0; i < 3; ++i) y[i] = alpha * (s_fr[i] * d0 + s_fr[i + 3] * d1 + s_fr[i + 6] * d2);
    }
    const double* sn = P.snx + ((size_t)pan * hd + j) * 3;
#pragma unroll
    for (int i = 0; i < 3; ++i) nrm[i] = s_fr[i] * sn[0] + s_fr[i + 3] * sn[1] + s_fr[i + 6] * sn[2];
    const bool ownj = j >= c0 && j < c0 + ncol;
    harm_column(L, m, y[0], y[1], y[2], [&](int l, int k, double h, double gx, double gy, double gz) {
        if (k >= c0 && k < c0 + ncol) {
          const int lc = k - c0;
          Xq[PL + (size_t)j * RS + lc] = gx;
          Xq[2 * PL + (size_t)j * RS + lc] = gy;
          Xq[3 * PL + (size_t)j * RS + lc] = gz;
        }
        if (ownj) {
          Xr[(size_t)k * RS + (j - c0)] = nrm[0] * gx + nrm[1] * gy + nrm[2] * gz;
          H[(size_t)j * hd + k] = h;
        }
      });
  }
  __syncthreads();
  double* Mq_r[CS];
  double* Mr_r[CS];
  int* pivq_r[CS];
#pragma unroll
  for (int r = 0; r < CS; ++r) {
    Mq_r[r] = cl.map_shared_rank(Mq, r);
    Mr_r[r] = cl.map_shared_rank(Mr, r);
    pivq_r[r] = cl.map_shared_rank(pivq, r);
  }
  const int nblk = (hd + PB_NB - 1) / PB_NB;
  for (int blk = 0; blk < nblk; ++blk) {
    const int k0 = blk * PB_NB, owner = k0 / ncol, lb0 = k0 - owner * ncol;
    const int nbk = min(PB_NB, hd - k0);
    if (rank == owner) {
      /* panel phase: the unblocked steps on the block's 8 columns alone, held
       * in registers by warps 0..7 (warp c: local block column c of both
       * systems, lane l: rows l, l + 32, ..).  Step j: warp j picks the pivot
       * rows of its column (largest norm / magnitude among the unused rows,
       * smallest row on ties: the unblocked rule), publishes the pivots and its
       * whole column (the elimination factors) in shared memory (two buffers
       * by step parity) and one named barrier of the 8 warps later every warp
       * scales its entry of the pivot rows and eliminates its column. */
      if (wid < PB_NB) {
        const int c = wid, lcol = lb0 + c;
        double xq[PB_MAXS][4], xr[PB_MAXS];
#pragma unroll
        for (int sl = 0; sl < PB_MAXS; ++sl) {
          const int r = lane + 32 * sl;
#pragma unroll
          for (int cc = 0; cc < 4; ++cc) xq[sl][cc] = r < hq ? Xq[cc * PL + (size_t)r * RS + lcol] : 0.0;
          xr[sl] = r < hr ? Xr[(size_t)r * RS + lcol] : 0.0;
        }
        /* rows pivoted in earlier blocks, and then in this one: bit masks */
        unsigned long long uq[3] = {0ull, 0ull, 0ull}, ur[3] = {0ull, 0ull, 0ull};
        for (int r = lane; r < 192; r += 32) {
          const bool a1 = r >= hd || usedq[min(r, hq - 1)] != 0, a2 = r >= hd || usedr[min(r, hr - 1)] != 0;
          const unsigned m1 = __ballot_sync(0xffffffffu, a1), m2 = __ballot_sync(0xffffffffu, a2);
          const int w64 = (r - lane) >> 6, sh = ((r - lane) & 63);
#pragma unroll
          for (int w = 0; w < 3; ++w)
            if (w64 == w) { uq[w] |= (unsigned long long)m1 << sh; ur[w] |= (unsigned long long)m2 << sh; }
        }
#define PB_USED(m, r) ((((r) < 64 ? m[0] : ((r) < 128 ? m[1] : m[2])) >> ((r) & 63)) & 1ull)
        for (int j = 0; j < nbk; ++j) {
          double* fb = fq + (size_t)(j & 1) * (4 * hq + hr + 8); /* the step's factors: [comp][row], MS, inverses */
          if (c == j) {
            /* pivot rows of this column */
            double bv = -1.0, bw = -1.0;
            int bi = hd, bj = hd;
#pragma unroll
            for (int sl = 0; sl < PB_MAXS; ++sl) {
              const int r = lane + 32 * sl;
              if (r < hd && !PB_USED(uq, r)) {
                const double v = xq[sl][0] * xq[sl][0] + xq[sl][1] * xq[sl][1] + xq[sl][2] * xq[sl][2] +
                                 xq[sl][3] * xq[sl][3];
                if (v > bv) { bv = v; bi = r; }
              }
              if (r < hd && !PB_USED(ur, r)) {
                const double v = fabs(xr[sl]);
                if (v > bw) { bw = v; bj = r; }
              }
            }
            for (int o = 16; o > 0; o >>= 1) {
              const double v2 = __shfl_xor_sync(0xffffffffu, bv, o);
              const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
              if (v2 > bv || (v2 == bv && i2 < bi)) { bv = v2; bi = i2; }
              const double w2 = __shfl_xor_sync(0xffffffffu, bw, o);
              const int j2 = __shfl_xor_sync(0xffffffffu, bj, o);
              if (w2 > bw || (w2 == bw && j2 < bj)) { bw = w2; bj = j2; }
            }
            if (bi >= hd) { /* a NaN column: the first unused row (results NaN, indices in range) */
              bi = 0;
              while (bi < hd - 1 && PB_USED(uq, bi)) ++bi;
            }
            if (bj >= hd) {
              bj = 0;
              while (bj < hd - 1 && PB_USED(ur, bj)) ++bj;
            }
#pragma unroll
            for (int sl = 0; sl < PB_MAXS; ++sl) {
              const int r = lane + 32 * sl;
              if (r < hq)
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) fb[cc * hq + r] = xq[sl][cc];
              if (r < hr) fb[4 * hq + r] = xr[sl];
            }
            __syncwarp();
            if (lane == 0) { /* the pivot inverses, once: conj(f)/|f|^2 and 1/f */
              const double f0 = fb[bi], f1 = fb[hq + bi], f2 = fb[2 * hq + bi], f3 = fb[3 * hq + bi];
              const double n2i = 1.0 / (f0 * f0 + f1 * f1 + f2 * f2 + f3 * f3);
              double* pvb = fb + 4 * hq + hr; /* after the step's columns */
              pvb[0] = f0 * n2i; pvb[1] = -f1 * n2i; pvb[2] = -f2 * n2i; pvb[3] = -f3 * n2i;
              pvb[4] = 1.0 / fb[4 * hq + bj];
              pidx[2 * (j & 1)] = bi; pidx[2 * (j & 1) + 1] = bj; pivq[k0 + j] = bi; pivr[k0 + j] = bj;
            }
          }
          named_bar(1, 32 * PB_NB);
          const int p = pidx[2 * (j & 1)], p2 = pidx[2 * (j & 1) + 1];
          const double* pvb = fb + 4 * hq + hr;
          const double pi4[4] = {pvb[0], pvb[1], pvb[2], pvb[3]};
          const double rinv = pvb[4];
          /* this column's entries of the pivot rows, scaled */
          double rq4[4], rr1;
          {
            const int sp = p >> 5, lp = p & 31, sp2 = p2 >> 5, lp2 = p2 & 31;
            double v[4] = {0.0, 0.0, 0.0, 0.0}, w = 0.0;
#pragma unroll
            for (int sl = 0; sl < PB_MAXS; ++sl) {
              if (sl == sp)
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) v[cc] = xq[sl][cc];
              if (sl == sp2) w = xr[sl];
            }
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) v[cc] = __shfl_sync(0xffffffffu, v[cc], lp);
            w = __shfl_sync(0xffffffffu, w, lp2);
            if (c == j) {
#pragma unroll
              for (int cc = 0; cc < 4; ++cc) rq4[cc] = pi4[cc];
              rr1 = rinv;
            } else {
              qmul(pi4, v, rq4);
              rr1 = rinv * w;
            }
          }
          /* eliminate: row p takes the scaled entry, the others subtract */
#pragma unroll
          for (int sl = 0; sl < PB_MAXS; ++sl) {
            const int r = lane + 32 * sl;
            if (r < hq) {
              if (r == p) {
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) xq[sl][cc] = rq4[cc];
              } else {
                const double f[4] = {fb[r], fb[hq + r], fb[2 * hq + r], fb[3 * hq + r]};
                double t[4];
                if (c == j) {
                  qmul(f, pi4, t);
#pragma unroll
                  for (int cc = 0; cc < 4; ++cc) xq[sl][cc] = -t[cc];
                } else {
                  qmul(f, rq4, t);
#pragma unroll
                  for (int cc = 0; cc < 4; ++cc) xq[sl][cc] -= t[cc];
                }
              }
            }
            if (r < hr) {
              if (r == p2) xr[sl] = rr1;
              else if (c == j) xr[sl] = -fb[4 * hq + r] * rinv;
              else xr[sl] -= fb[4 * hq + r] * rr1;
            }
          }
#pragma unroll
          for (int w = 0; w < 3; ++w) {
            if ((p >> 6) == w) uq[w] |= 1ull << (p & 63);
            if ((p2 >> 6) == w) ur[w] |= 1ull << (p2 & 63);
          }
        }
#pragma unroll
        for (int sl = 0; sl < PB_MAXS; ++sl) {
          const int r = lane + 32 * sl;
          if (r < hq)
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) Xq[cc * PL + (size_t)r * RS + lcol] = xq[sl][cc];
          if (r < hr) Xr[(size_t)r * RS + lcol] = xr[sl];
        }
      }
      __syncthreads();
#undef PB_USED
      /* publish the block and its pivot rows to every CTA of the cluster */
      for (int e = tid; e < hq * PB_NB * 4; e += NT) {
        const int c = e & 3, b = (e >> 2) & 7, i = e >> 5;
        const double v = Xq[c * PL + (size_t)i * RS + lb0 + b];
#pragma unroll
        for (int r = 0; r < CS; ++r) Mq_r[r][e] = v;
      }
      for (int e = tid; e < hr * PB_NB; e += NT) {
        const double v = Xr[(size_t)(e >> 3) * RS + lb0 + (e & 7)];
#pragma unroll
        for (int r = 0; r < CS; ++r) Mr_r[r][e] = v;
      }
      if (tid < nbk) {
#pragma unroll
        for (int r = 0; r < CS; ++r) { pivq_r[r][k0 + tid] = pivq[k0 + tid]; pivq_r[r][hd + k0 + tid] = pivr[k0 + tid]; }
      }
    }
    cl.sync();
    /* this block's pivot rows */
    for (int e = tid; e < hq; e += NT) {
      int f = 0;
      for (int j = 0; j < nbk; ++j) f |= pivq[k0 + j] == e;
      isPq[e] = f;
      if (f) usedq[e] = 1;
    }
    for (int e = tid; e < hr; e += NT) {
      int f = 0;
      for (int j = 0; j < nbk; ++j) f |= pivr[k0 + j] == e;
      isPr[e] = f;
      if (f) usedr[e] = 1;
    }
    __syncthreads();
    /* trailing update of this CTA's other columns: warp w takes column tile
     * w % ntl and every G-th row tile, B fragments (the pivot rows) read
     * before any tile is stored */
    {
      const int ntl = ncol / 8, skip = rank == owner ? lb0 / 8 : -1;
      const int Gq = NW >= ntl ? NW / ntl : 1;
      const bool act = wid < Gq * ntl;
      const int nt = wid % ntl, g0 = wid / ntl;
      const int J = 8 * nt + (lane >> 2);
      double bq[PB_NB], br2[2];
      const int d = lane & 3;
#pragma unroll
      for (int ks = 0; ks < PB_NB; ++ks) {
        const int prow = ks < nbk ? pivq[k0 + ks] : 0;
        bq[ks] = (act && ks < nbk) ? Xq[d * PL + (size_t)prow * RS + J] : 0.0;
      }
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        const int b = 4 * ks + d;
        const int prow = b < nbk ? pivr[k0 + b] : 0;
        br2[ks] = (act && b < nbk) ? Xr[(size_t)prow * RS + J] : 0.0;
      }
      __syncthreads();
      if (act && nt != skip) {
        /* quaternion system: row tiles of 8 real rows = 2 quaternion rows */
        const int cc = (lane >> 2) & 3, ci = cc ^ d;
        const double sg = lmul_sign(cc, d);
        const int jc = 8 * nt + 2 * (lane & 3);
        for (int mt = g0; mt < hq / 2; mt += Gq) {
          const int i = 2 * mt + (lane >> 4);
          double* xr = Xq + cc * PL + (size_t)i * RS + jc;
          const bool zp = isPq[i] != 0;
          double a0 = zp ? 0.0 : xr[0], a1 = zp ? 0.0 : xr[1];
          const double* mrow = Mq + (size_t)i * PB_NB * 4;
#pragma unroll
          for (int ks = 0; ks < PB_NB; ++ks) dmma(a0, a1, sg * mrow[4 * ks + ci], bq[ks]);
          xr[0] = a0; xr[1] = a1;
        }
        /* real system */
        for (int mt = g0; mt < hr / 8; mt += Gq) {
          const int i = 8 * mt + (lane >> 2);
          double* xr = Xr + (size_t)i * RS + jc;
          const bool zp = isPr[i] != 0;
          double a0 = zp ? 0.0 : xr[0], a1 = zp ? 0.0 : xr[1];
#pragma unroll
          for (int ks = 0; ks < 2; ++ks) dmma(a0, a1, Mr[(size_t)i * PB_NB + 4 * ks + d], br2[ks]);
          xr[0] = a0; xr[1] = a1;
        }
      }
    }
    cl.sync(); /* every CTA is done with the block before the next is published */
  }
  /* inverse positions of the pivot sequences (every CTA holds all pivots) */
  for (int k = tid; k < hd; k += NT) { posq[pivq[k]] = k; posr[pivr[k]] = k; }
  __syncthreads();
  double* PD = R.PD + (size_t)pan * hd * 4 * hd;
  double* PS = R.smat + (size_t)pan * hd * hd;
  const int nc = min(ncol, hd - c0);
  for (int e = tid; e < hd * nc; e += NT) {
    const int i = e / nc, tc = e % nc, gc = c0 + tc;
    const int jq = pivq[gc], kq = posq[i];
    double* d = PD + (size_t)jq * 4 * hd + kq;
    d[0] = Xq[(size_t)i * RS + tc];
    d[hd] = -Xq[PL + (size_t)i * RS + tc];
    d[2 * hd] = -Xq[2 * PL + (size_t)i * RS + tc];
    d[3 * hd] = -Xq[3 * PL + (size_t)i * RS + tc];
    PS[(size_t)posr[i] * hd + pivr[gc]] = Xr[(size_t)i * RS + tc];
  }
  __threadfence();
  cl.sync();
  panel_b_epilogue(R, hd, pan, c0, nc, (int)(pblk_smem_bytes(hd, CS) / sizeof(double)), psm);
}

/* ===================================================================== */
/* K5: per-pair RRQ moments, one warp per pair                           */
/* ===================================================================== */
#define RRQ_WARPS 4
struct WarpSM {
  double w1[3 * QOL_MAXNQ], w3[3 * QOL_MAXNQ];
  double br[3][112];
  int nbr[3];
};


/* the three coordinate series (3 x n Legendre coefficients) of one edge and
 * their derivatives at t, one recurrence for all three, no divisions */
__device__ __forceinline__ void leg_eval3(int n, const double* c, double t, double* y, double* yp) {
  double p0 = 1.0, p1 = t, d0 = 0.0, d1 = 1.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) { y[d] = c[d * n]; yp[d] = 0.0; }
  if (n > 1)
#pragma unroll
    for (int d = 0; d < 3; ++d) { y[d] += c[d * n + 1] * p1; yp[d] += c[d * n + 1] * d1; }
  for (int k = 1; k + 1 < n; ++k) {
    const double p2 = c_la[k] * t * p1 - c_lb[k] * p0;
    const double d2 = d0 + (2.0 * k + 1.0) * p1;
#pragma unroll
    for (int d = 0; d < 3; ++d) { y[d] += c[d * n + k + 1] * p2; yp[d] += c[d * n + k + 1] * d2; }
    p0 = p1; p1 = p2; d0 = d1; d1 = d2;
  }
}


/* the panel's Koornwinder expansion (coefficients scf, 3 x hd) at (u, v),
 * (u + h, v) and (u, v + h): f[3 c + p] = coordinate c at point p.  Column a:
 * the Legendre factor L_a((2u + v - 1)/(1 - v)) (1 - v)^a by its three-term
 * recurrence (advanced one step per column), the Jacobi P_b^(2a+1,0)(2v - 1)
 * by its recurrence down the column; terms summed in column order */
__device__ void koorn_eval3_thread(int korder, int hd, const double* scf, double u, double v, double h,
                                   double* f /* 9 */) {
  double acc[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) acc[i] = 0.0;
  const double us[3] = {u, u + h, u}, vs[3] = {v, v, v + h};
  double sv[3], tt[3], zv[3], L0[3], L1[3];
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    sv[p] = 2.0 * us[p] + vs[p] - 1.0;
    const double t = 1.0 - vs[p];
    tt[p] = t * t;
    zv[p] = 2.0 * vs[p] - 1.0;
    L0[p] = 1.0; L1[p] = sv[p];
  }
  for (int a = 0; a <= korder; ++a) {
    double La[3];
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      if (a <= 1) La[p] = a == 0 ? 1.0 : sv[p];
      else {
        const double L2 = c_la[a - 1] * sv[p] * L1[p] - c_lb[a - 1] * tt[p] * L0[p];
        L0[p] = L1[p]; L1[p] = L2; La[p] = L2;
      }
    }
    const double alpha = 2.0 * a + 1.0;
    double p0[3], p1[3];
#pragma unroll
    for (int p = 0; p < 3; ++p) { p0[p] = 1.0; p1[p] = 0.5 * (alpha + 2.0) * zv[p] + 0.5 * alpha; }
    const double* jq = &g_jq[a][0][0];
    for (int b = 0; b <= korder - a; ++b) {
      double pb[3];
      if (b == 0) {
#pragma unroll
        for (int p = 0; p < 3; ++p) pb[p] = p0[p];
      } else if (b == 1) {
#pragma unroll
        for (int p = 0; p < 3; ++p) pb[p] = p1[p];
      } else {
        const double A = jq[4 * b], B = jq[4 * b + 1], C = jq[4 * b + 2];
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const double p2 = (A + B * zv[p]) * p1[p] - C * p0[p];
          p0[p] = p1[p]; p1[p] = p2; pb[p] = p2;
        }
      }
      const int deg = a + b, idx = deg * (deg + 1) / 2 + b;
      const double s0 = scf[idx], s1 = scf[hd + idx], s2 = scf[2 * hd + idx];
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        const double val = La[p] * pb[p];
        acc[p] += val * s0;
        acc[3 + p] += val * s1;
        acc[6 + p] += val * s2;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) f[i] = acc[i];
}

/* side test of every RRQ pair of the launch, one thread per pair: the
 * target's projection onto the panel by Newton from the nearest node's
 * (u, v) (finite-difference Jacobian), its height over
 * the panel and whether the projection lies inside the triangle:
 * R.side = side (-1, 0, 1; 0 within 1e-12) + 4 inside */
__global__ void __launch_bounds__(128) k_rrq_side(OrderTab T, PairIn Q, RRQWS R) {
  const long long gidx = R.glo + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gidx >= R.ghi) return;
  const int2 pr = R.pair[gidx];
  const int pan = pr.x, tl = pr.y, hd = T.hd;
  const long long p0 = Q.tcxi[pan] - 1;
  const double* fr = R.frame + (size_t)pan * RRQ_FRAME;
  const double* scf = R.scf + (size_t)pan * 3 * hd;
  const double* sxf = R.sxf + (size_t)pan * 3 * hd;
  const double alpha = fr[12];
  double xt[3];
  {
    const double* x = Q.tcx + 3 * (p0 + tl);
    const double d0 = x[0] - fr[9], d1 = x[1] - fr[10], d2 = x[2] - fr[11];
    for (int i = 0; i < 3; ++i) xt[i] = alpha * (fr[i] * d0 + fr[i + 3] * d1 + fr[i + 6] * d2);
  }
  double best = 1e300;
  int ib = hd;
  for (int j = 0; j < hd; ++j) { /* the nearest node in the frame's plane (first on ties) */
    const double d0 = sxf[3 * j] - xt[0], d1 = sxf[3 * j + 1] - xt[1], d2 = d0 * d0 + d1 * d1;
    if (d2 < best) { best = d2; ib = j; }
  }
  double u = T.vruv[2 * ib], v = T.vruv[2 * ib + 1];
  double f[9];
  const double h = 1e-7;
  for (int it = 0; it < 40; ++it) {
    koorn_eval3_thread(T.korder, hd, scf, u, v, h, f);
    const double J00 = (f[1] - f[0]) / h, J10 = (f[4] - f[3]) / h, J01 = (f[2] - f[0]) / h, J11 = (f[5] - f[3]) / h;
    const double r0 = f[0] - xt[0], r1 = f[3] - xt[1];
    const double det = J00 * J11 - J01 * J10;
    if (det == 0.0) break;
    const double du = (J11 * r0 - J01 * r1) / det, dv = (-J10 * r0 + J00 * r1) / det;
    u -= du; v -= dv;
    if (fabs(du) + fabs(dv) < 1e-14) break;
  }
  koorn_eval3_thread(T.korder, hd, scf, u, v, 0.0, f);
  const double tol = 1e-10;
  const int inside = (u >= -tol && v >= -tol && u + v <= 1.0 + tol) ? 1 : 0;
  const double hgt = xt[2] - f[6];
  const int side = fabs(hgt) <= 1e-12 ? 0 : (hgt > 0 ? 1 : -1);
  R.side[gidx] = (signed char)(side + 4 * inside);
}

/* singularity-swap root and modified weights, one thread per (RRQ pair,
 * edge): writes w1 (nq), w3 (nq), ok, Re t0, Im t0 to the pair's edge record */
__global__ void __launch_bounds__(128) k_rrq_ssq(OrderTab T, PairIn Q, PairWS G, RRQWS R) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 3 * (R.ghi - R.glo)) return;
  const long long gidx = R.glo + tid / 3;
  const int e = (int)(tid % 3);
  const int2 pr = R.pair[gidx]; /* (panel, local target) */
  const int pan = pr.x, tl = pr.y;
  const long long p0 = Q.tcxi[pan] - 1;
  const int nq = T.nquad, nbd = 3 * nq;
  const double* fr = R.frame + (size_t)pan * RRQ_FRAME;
  const double* bx = R.bx + (size_t)pan * 3 * nbd;
  const double* cf = R.cf + (size_t)pan * 9 * nq;
  const double alpha = fr[12];
  double xt[3];
  {
    const double* x = Q.tcx + 3 * (p0 + tl);
    double d0 = x[0] - fr[9], d1 = x[1] - fr[10], d2 = x[2] - fr[11];
    for (int i = 0; i < 3; ++i) xt[i] = alpha * (fr[i] * d0 + fr[i + 3] * d1 + fr[i + 6] * d2);
  }
  double* er = R.edge + ((size_t)gidx * 3 + e) * (2 * nq + 3);
  cd t0 = mk(0.0, 0.0);
  bool ok = edge_root_dev(nq, cf + e * 3 * nq, T.tgl, bx + 3 * e * nq, xt, c_la, c_lb, t0);
  ssq_weights_dev(nq, T.tgl, T.wgl, ok, t0, T.gl48x, T.gl48w, T.tginv, c_rk, er, er + nq);
  er[2 * nq] = ok ? 1.0 : 0.0;
  er[2 * nq + 1] = t0.re;
  er[2 * nq + 2] = t0.im;
}

__global__ void __launch_bounds__(32 * RRQ_WARPS) k_rrq_geom(OrderTab T, PairIn Q, PairWS G, RRQWS R, int exterior) {
  __shared__ WarpSM S[RRQ_WARPS];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long gidx = R.glo + (long long)blockIdx.x * RRQ_WARPS + wid;
  if (gidx >= R.ghi) return;
  WarpSM& W = S[wid];
  const int2 pr = R.pair[gidx]; /* (panel, local target) */
  const int pan = pr.x, tl = pr.y;
  const long long p0 = Q.tcxi[pan] - 1;
  const int nq = T.nquad, nbd = 3 * nq;
  const double* fr = R.frame + (size_t)pan * RRQ_FRAME;
  const double* bx = R.bx + (size_t)pan * 3 * nbd;
  const double* bt = R.bt + (size_t)pan * 3 * nbd;
  const double* cf = R.cf + (size_t)pan * 9 * nq;
  const double alpha = fr[12];
  double xt[3];
  {
    const double* x = Q.tcx + 3 * (p0 + tl);
    double d0 = x[0] - fr[9], d1 = x[1] - fr[10], d2 = x[2] - fr[11];
    for (int i = 0; i < 3; ++i) xt[i] = alpha * (fr[i] * d0 + fr[i + 3] * d1 + fr[i + 6] * d2);
  }
  const double xt0 = xt[0], xt1 = xt[1], xt2 = xt[2];
  /* singularity-swap weights (from k_rrq_ssq) and graded breakpoints, one
   * lane per edge */
  for (int e2 = lane; e2 < 3 * 2 * nq; e2 += 32) { /* the weights, all lanes */
    const int e = e2 / (2 * nq), r = e2 % (2 * nq);
    const double v = R.edge[((size_t)gidx * 3 + e) * (2 * nq + 3) + r];
    if (r < nq) W.w1[e * nq + r] = v;
    else W.w3[e * nq + r - nq] = v;
  }
  if (lane < 3) {
    const int e = lane;
    const double* er = R.edge + ((size_t)gidx * 3 + e) * (2 * nq + 3);
    const bool ok = er[2 * nq] != 0.0;
    const cd t0 = mk(er[2 * nq + 1], er[2 * nq + 2]);
    double ts = 0.0, dd = 2.0;
    if (ok) { ts = fmin(1.0, fmax(-1.0, t0.re)); dd = fmax(fabs(t0.im), 1e-15); }
    double left[54], right[54];
    int nl = 0, nr = 0;
    if (!ok) {
      for (int k = 1; k < 16; ++k) right[nr++] = -1.0 + k / 8.0;
    } else if (dd < 1.0) {
      for (double h = 0.5 * dd; h < 2.0; h *= 2.0) {
        if (ts - h > -1.0 && nl < 54) left[nl++] = ts - h;
        if (ts + h < 1.0 && nr < 54) right[nr++] = ts + h;
      }
    }
    int c = 0;
    W.br[e][c++] = -1.0;
    for (int k = nl - 1; k >= 0; --k) W.br[e][c++] = left[k];
    for (int k = 0; k < nr; ++k) W.br[e][c++] = right[k];
    W.br[e][c++] = 1.0;
    W.nbr[e] = c;
  }
  /* Dirac-string direction: away from the panel when the target projects
   * inside the triangle; otherwise the one passing farther from the boundary */
  double sdir;
  {
    const int sd = R.side[gidx]; /* from k_rrq_side */
    const int inside = sd >= 3 ? 1 : 0, side = sd - 4 * inside;
    sdir = side == 0 ? (exterior ? 1.0 : -1.0) : (double)side;
    if (!inside) {
      double cu = 2.0, cdn = 2.0;
      for (int pnt = lane; pnt < 96; pnt += 32) {
        int e = pnt >> 5, q = pnt & 31;
        double t = -1.0 + (2.0 * q + 1.0) / 32.0, y[3], yp[3];
        leg_eval3(nq, cf + e * 3 * nq, t, y, yp);
        double rho[3] = {y[0] - xt0, y[1] - xt1, y[2] - xt2};
        double r = sqrt(dot3(rho, rho));
        cu = fmin(cu, (r - rho[2]) / r);
        cdn = fmin(cdn, (r + rho[2]) / r);
      }
      for (int o = 16; o > 0; o >>= 1) {
        cu = fmin(cu, __shfl_xor_sync(0xffffffffu, cu, o));
        cdn = fmin(cdn, __shfl_xor_sync(0xffffffffu, cdn, o));
      }
      sdir = cu >= cdn ? 1.0 : -1.0;
    }
  }
  __syncwarp();
  /* solid angle: points of the graded meshes over the lanes */
  double Omega;
  {
    double tot = 0.0;
    /* the three edges' points as one list over the lanes */
    const int p0n = 16 * (W.nbr[0] - 1), p1n = p0n + 16 * (W.nbr[1] - 1), p2n = p1n + 16 * (W.nbr[2] - 1);
    for (int pg = lane; pg < p2n; pg += 32) {
      {
        const int e = pg < p0n ? 0 : (pg < p1n ? 1 : 2), pnt = pg - (e == 0 ? 0 : (e == 1 ? p0n : p1n));
        int ib = pnt >> 4, q = pnt & 15;
        double a = W.br[e][ib], b = W.br[e][ib + 1];
        if (!(b > a)) continue;
        double hm = 0.5 * (b - a), cm = 0.5 * (a + b), t = cm + hm * T.gl16x[q];
        double y[3], yp[3];
        leg_eval3(nq, cf + e * 3 * nq, t, y, yp);
        double rho[3] = {y[0] - xt0, y[1] - xt1, y[2] - xt2};
        double r = sqrt(dot3(rho, rho));
        double s3[3] = {0.0, 0.0, sdir}, c[3];
        double sr = sdir * rho[2];
        cross3(rho, s3, c);
        double den = sr > 0 ? dot3(c, c) / (r + sr) : r - sr;
        tot += hm * T.gl16w[q] * dot3(c, yp) / (r * den);
      }
    }
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    Omega = tot;
  }
  /* per boundary node weights (1/4pi folded in), written with the solid
   * angle to the pair's line record: cD (3 nbd), cS (3 nbd), lint (3), Omega */
  const double i4p = 1.0 / (4.0 * QOL_PI);
  double* rec = R.line + (size_t)gidx * (6 * nbd + 4);
  double lint[3] = {0, 0, 0};
  for (int i = lane; i < nbd; i += 32) {
    const double* y = bx + 3 * i;
    const double* yp = bt + 3 * i;
    double rho[3] = {y[0] - xt0, y[1] - xt1, y[2] - xt2};
    double r = sqrt(dot3(rho, rho));
    double rxy[3], rrx[3];
    cross3(rho, yp, rxy);
    cross3(rho, rxy, rrx);
    double f1 = W.w1[i] / r, f3 = W.w3[i] / (r * r * r);
    for (int d = 0; d < 3; ++d) {
      rec[3 * i + d] = f3 * rrx[d] * i4p;
      rec[3 * nbd + 3 * i + d] = f1 * rxy[d] * i4p;
      lint[d] += f1 * yp[d];
    }
  }
  for (int d = 0; d < 3; ++d)
    for (int o = 16; o > 0; o >>= 1) lint[d] += __shfl_xor_sync(0xffffffffu, lint[d], o);
  if (lane == 0) {
    rec[6 * nbd + 0] = lint[0]; rec[6 * nbd + 1] = lint[1]; rec[6 * nbd + 2] = lint[2];
    rec[6 * nbd + 3] = Omega;
    if (R.ialpha) R.ialpha[tl] = Omega; /* single-panel calls (qol_rrq) */
  }
}

/* ---------------------------------------------------------------------
 * Harmonic moments by translation.
 *
 * Regular solid harmonics R_l^m = r^l P_l^m(cos th) e^{i m phi} / (l+m)!
 * (no Condon-Shortley phase) in the harmonic coordinates (X,Y,Z) = (p1,p2,p0)
 * of a frame point p.  The sin-type basis of the RRQ systems is
 * h_{l,m} = N_lm Im R_l^m, N_lm = sqrt((l-m)!(l+m)!), and
 *   R_m^m = R_{m-1}^{m-1} (X+iY)/(2m),
 *   R_l^m = ((2l-1) Z R_{l-1}^m - r^2 R_{l-2}^m) / ((l+m)(l-m)),
 *   d_Z R_l^m = R_{l-1}^m,  d_X R_l^m = (R_{l-1}^{m-1} - R_{l-1}^{m+1})/2,
 *   d_Y R_l^m = i (R_{l-1}^{m-1} + R_{l-1}^{m+1})/2,
 *   R_l^m(x+rho) = sum_{lam,mu} R_lam^mu(rho) R_{l-lam}^{m-mu}(x)  (addition
 *   theorem), R_l^{-m} = (-1)^m conj(R_l^m).
 * The reference's moments (lap3d_close_mod.f90:832-841) integrate grad h_k
 * along the segments x -> y_i to the boundary nodes:
 *   Phi_k(y) = int_0^1 [grad h_k(x+t rho) - grad h_k(x)]/t dt,
 *   Psi_k(y) = int_0^1 grad h_k(x+t rho) dt.
 * The degree-lam part of grad h_k(x+rho) in rho integrates to 1/lam (Phi) and
 * 1/(lam+1) (Psi), so with the node sums
 *   M_lam^mu[d] = sum_i c_i[d] R_lam^mu(rho_i) / lam   (D weights cD)
 *                                            / (lam+1) (S weights cS)
 * every moment is a translation T_n^k = sum M_lam^mu R_{n-lam}^{k-mu}(x) of
 * degree n = l-1 and the three derivative rules above.  Same quadrature as
 * the point-wise segment rule (that rule is exact for these polynomials),
 * a fraction of the arithmetic.
 * --------------------------------------------------------------------- */

#define MOM_T QOL_MOM_THREADS /* threads per RRQ pair */
#define MOM_NC 16 /* boundary nodes per chunk */
#define MOM_CS (MOM_NC + 1)

__host__ __device__ constexpr int mom_rows(int L) { return L * (L + 1); }
__host__ __device__ constexpr int mom_rec(int nbd) { return (6 * nbd + 4 + 1) & ~1; }
/* doubles of shared memory of one pair after the line record: the node chunk,
 * later M (entries 14 doubles apart), R(x), the translation's partial sums
 * (12 per slot, component-major); T reuses M's space once the translation is done */
__host__ __device__ constexpr int mom_region(int L, int slots) {
  return mom_rows(L) * MOM_CS > 7 * mom_rows(L) + (L + 1) * (L + 2) + 12 * slots
             ? mom_rows(L) * MOM_CS
             : 7 * mom_rows(L) + (L + 1) * (L + 2) + 12 * slots;
}

/* one CTA of MOM_T threads per RRQ pair.
 * (A) R_lam^mu(rho_i), lam <= L-1, mu >= 0, chunks of MOM_NC nodes: thread
 *     (g, j) evaluates node c0+j over the column pair (g, L-1-g) (L <= 16: at
 *     most 8 pairs), the two columns as two recurrence chains in flight, into
 *     ch[row][j], row = 2 entry(lam,mu) + re/im.
 * (B) each thread contracts its rows e = tid + MOM_T r with the 6 weights.
 * (C) R(x) up to degree L.
 * (D) the translation, pieces of the term lists per thread (qolh::xlate_schedule),
 *     partial sums per piece, then their fixed-order sum per output.
 * (E) the moments of every h_{l,m}. */
template <int LB>
__global__ void __launch_bounds__(MOM_T, 7) k_rrq_moments(OrderTab T, PairIn Q, PairWS G, RRQWS R) {
  constexpr int RPT = (LB * (LB + 1) + MOM_T - 1) / MOM_T; /* real rows of M per thread */
  extern __shared__ __align__(16) double mom_sm[];
  /* c_rq and c_rn are read from constant memory (a warp reads at most two
   * entries at a time), which leaves shared memory to more resident pairs */
  __shared__ double s_rd[QOL_MAXL + 2], s_ri[QOL_MAXL + 2];
  const int tid = threadIdx.x;
  for (int e = tid; e < QOL_MAXL + 2; e += MOM_T) { s_rd[e] = c_rd[e]; s_ri[e] = c_rinv[e]; }
  const long long gidx = R.glo + blockIdx.x;
  if (gidx >= R.ghi) return; /* uniform over the CTA */
  const int2 pr = R.pair[gidx]; /* (panel, local target) */
  const int pan = pr.x, tl = pr.y;
  const long long p0 = Q.tcxi[pan] - 1;
  const int hd = T.hd, nq = T.nquad, nbd = 3 * nq, L = T.nterms;
  const double* fr = R.frame + (size_t)pan * RRQ_FRAME;
  const double* bx = R.bx + (size_t)pan * 3 * nbd;
  const double alpha = fr[12];
  double xt0, xt1, xt2;
  {
    const double* x = Q.tcx + 3 * (p0 + tl);
    double d0 = x[0] - fr[9], d1 = x[1] - fr[10], d2 = x[2] - fr[11];
    xt0 = alpha * (fr[0] * d0 + fr[3] * d1 + fr[6] * d2);
    xt1 = alpha * (fr[1] * d0 + fr[4] * d1 + fr[7] * d2);
    xt2 = alpha * (fr[2] * d0 + fr[5] * d1 + fr[8] * d2);
  }
  double* rec = mom_sm;
  double* ch = rec + mom_rec(nbd);
  {
    const double* grec = R.line + (size_t)gidx * (6 * nbd + 4);
    for (int e = tid; e < 6 * nbd + 4; e += MOM_T) rec[e] = grec[e];
  }
  __syncthreads();
  const double* cD = rec;
  const double* cS = rec + 3 * nbd;
  const int NE = mom_rows(L);
  double acc[RPT][6];
#pragma unroll
  for (int r = 0; r < RPT; ++r)
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[r][c] = 0.0;
  int erow[RPT];
#pragma unroll
  for (int r = 0; r < RPT; ++r) erow[r] = min(tid + MOM_T * r, NE - 1) * MOM_CS;
  const int np = (L + 1) / 2, pa = tid >> 4, jn = tid & 15, qa = L - 1 - pa;
  for (int c0 = 0; c0 < nbd; c0 += MOM_NC) {
    if (tid < MOM_NC) { /* the diagonal R_m^m, m < L, of node c0 + tid, once, into its rows */
      const int i = min(c0 + tid, nbd - 1);
      const double X = bx[3 * i + 1] - xt1, Y = bx[3 * i + 2] - xt2;
      double dr = 1.0, di = 0.0;
      ch[0 * MOM_CS + tid] = 1.0;
      ch[1 * MOM_CS + tid] = 0.0;
      for (int mm = 1; mm < L; ++mm) {
        const double t = dr * X - di * Y;
        di = (dr * Y + di * X) * s_rd[mm];
        dr = t * s_rd[mm];
        const int row = mm * (mm + 1) + 2 * mm;
        ch[row * MOM_CS + tid] = dr;
        ch[(row + 1) * MOM_CS + tid] = di;
      }
    }
    __syncthreads();
    if (pa < np) {
      const int i = min(c0 + jn, nbd - 1);
      const double Z = bx[3 * i] - xt0, X = bx[3 * i + 1] - xt1, Y = bx[3 * i + 2] - xt2;
      const double r2 = X * X + Y * Y + Z * Z;
      /* columns pa (L-pa entries) and qa (L-qa entries, none when qa == pa), from
       * their diagonal entries */
      const int n1 = L - pa, n2 = qa > pa ? L - qa : 0;
      const int dpa = pa * (pa + 1) + 2 * pa, dqa = qa * (qa + 1) + 2 * qa;
      double ur = ch[dpa * MOM_CS + jn], ui = ch[(dpa + 1) * MOM_CS + jn], vr = 0.0, vi = 0.0;
      double sr = n2 ? ch[dqa * MOM_CS + jn] : 0.0, si = n2 ? ch[(dqa + 1) * MOM_CS + jn] : 0.0, tr = 0.0, ti = 0.0;
      for (int e = 0; e < n1; ++e) {
        if (e > 0) {
          const int l = pa + e;
          const double q = c_rq[l][pa], a = (2.0 * l - 1.0) * Z;
          const double nr = (a * ur - r2 * vr) * q, ni = (a * ui - r2 * vi) * q;
          vr = ur; vi = ui; ur = nr; ui = ni;
        }
        const int row = (pa + e) * (pa + e + 1) + 2 * pa;
        ch[row * MOM_CS + jn] = ur;
        ch[(row + 1) * MOM_CS + jn] = ui;
        if (e < n2) {
          if (e > 0) {
            const int l = qa + e;
            const double q = c_rq[l][qa], a = (2.0 * l - 1.0) * Z;
            const double nr = (a * sr - r2 * tr) * q, ni = (a * si - r2 * ti) * q;
            tr = sr; ti = si; sr = nr; si = ni;
          }
          const int row2 = (qa + e) * (qa + e + 1) + 2 * qa;
          ch[row2 * MOM_CS + jn] = sr;
          ch[(row2 + 1) * MOM_CS + jn] = si;
        }
      }
    }
    __syncthreads();
    const int nj = min(MOM_NC, nbd - c0);
    for (int jj = 0; jj < nj; ++jj) {
      const int ii = c0 + jj;
      const double w0 = cD[3 * ii], w1 = cD[3 * ii + 1], w2 = cD[3 * ii + 2];
      const double w3 = cS[3 * ii], w4 = cS[3 * ii + 1], w5 = cS[3 * ii + 2];
#pragma unroll
      for (int r = 0; r < RPT; ++r) {
        const double v = ch[erow[r] + jj];
        acc[r][0] += v * w0; acc[r][1] += v * w1; acc[r][2] += v * w2;
        acc[r][3] += v * w3; acc[r][4] += v * w4; acc[r][5] += v * w5;
      }
    }
    __syncthreads();
  }
  /* M[entry][6 components][re,im] (entries 14 doubles apart) with the 1/lam
   * (D) and 1/(lam+1) (S) segment weights; then R(x) up to degree L */
  double* Mt = ch;
  double* Rx = ch + 7 * NE;
  double* Pp = Rx + (L + 1) * (L + 2);
  double* Tt = ch; /* after the translation */
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const int e = tid + MOM_T * r;
    if (e < NE) {
      const int ent = e >> 1, ri = e & 1;
      int lam = 0;
      while ((lam + 1) * (lam + 2) / 2 <= ent) ++lam;
      const double wD = s_ri[lam], wS = s_ri[lam + 1];
      double* dst = Mt + ent * 14 + ri;
      dst[0] = acc[r][0] * wD; dst[2] = acc[r][1] * wD; dst[4] = acc[r][2] * wD;
      dst[6] = acc[r][3] * wS; dst[8] = acc[r][4] * wS; dst[10] = acc[r][5] * wS;
    }
  }
  if (tid <= L) { /* column m = tid of R(x) */
    const int m = tid;
    const double Z = xt0, X = xt1, Y = xt2, r2 = X * X + Y * Y + Z * Z;
    double dr = 1.0, di = 0.0;
    for (int mm = 1; mm <= m; ++mm) {
      const double t = dr * X - di * Y;
      di = (dr * Y + di * X) * s_rd[mm];
      dr = t * s_rd[mm];
    }
    double ar = dr, ai = di, br = 0.0, bi = 0.0;
    for (int l = m; l <= L; ++l) {
      if (l > m) {
        const double q = c_rq[l][m], a = (2.0 * l - 1.0) * Z;
        const double nr = (a * ar - r2 * br) * q, ni = (a * ai - r2 * bi) * q;
        br = ar; bi = ai; ar = nr; ai = ni;
      }
      const int ent = l * (l + 1) / 2 + m;
      Rx[2 * ent] = ar; Rx[2 * ent + 1] = ai;
    }
  }
  __syncthreads();
  /* (D) this thread's pieces of the translation, each flushed to its slot */
  {
    double a[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) a[c] = 0.0;
    const unsigned* tab = T.xsched + tid;
    const int nst = T.xsteps;
    unsigned wn = nst > 0 ? __ldg(tab) : 0u;
    for (int s = 0; s < nst; ++s) {
      const unsigned w = wn;
      if (s + 1 < nst) wn = __ldg(tab + MOM_T * (s + 1));
      if (!(w & (1u << 29))) break; /* a thread's terms are contiguous from step 0 */
      const int em = w & 255, ex = (w >> 8) & 255;
      const double2 rv = *reinterpret_cast<const double2*>(Rx + 2 * ex);
      double c = rv.x, d = rv.y;
      if (w & (1u << 28)) { c = -c; d = -d; }
      if (w & (1u << 27)) d = -d;
      double p = d, q = c;
      if (w & (1u << 26)) { p = -d; q = -c; }
      const double2* mv = reinterpret_cast<const double2*>(Mt + em * 14);
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double2 v = mv[k];
        a[2 * k] += v.x * c - v.y * p;
        a[2 * k + 1] += v.y * q + v.x * d;
      }
      if (w & (1u << 30)) { /* slots component-major: Pp[c * xslots + slot] */
        double* dst = Pp + ((w >> 16) & 1023);
#pragma unroll
        for (int c2 = 0; c2 < 12; ++c2) { dst[c2 * T.xslots] = a[c2]; a[c2] = 0.0; }
      }
    }
  }
  __syncthreads();
  for (int o = tid; o < NE / 2; o += MOM_T) { /* T_o = sum of its pieces, in slot order */
    const int ps = (int)T.xred[2 * o], npc = (int)T.xred[2 * o + 1];
    double t[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) t[c] = Pp[c * T.xslots + ps];
    for (int q = 1; q < npc; ++q)
#pragma unroll
      for (int c = 0; c < 12; ++c) t[c] += Pp[c * T.xslots + ps + q];
#pragma unroll
    for (int c = 0; c < 12; ++c) Tt[12 * o + c] = t[c];
  }
  __syncthreads();
  /* (E) the moments of h_{l,m}: T of degree l-1 at orders m-1, m, m+1, and
   * the x point: (s0, lint/4pi) (x) (0, grad h(x)) and h(x) Omega/4pi */
  const double i4p = 1.0 / (4.0 * QOL_PI);
  const double lint0 = rec[6 * nbd], lint1 = rec[6 * nbd + 1], lint2 = rec[6 * nbd + 2], Omega = rec[6 * nbd + 3];
  const double s0 = -Omega * i4p;
  const double wv0 = lint0 * i4p, wv1 = lint1 * i4p, wv2 = lint2 * i4p;
  double* JD = R.JD + (size_t)gidx * 4 * hd;
  double* RS = R.RS + (size_t)gidx * hd;
  for (int k = tid; k < hd; k += MOM_T) {
    int l = 1;
    while ((l + 1) * l / 2 <= k) ++l;
    const int m = k - l * (l - 1) / 2 + 1, n = l - 1;
    const double Nf = c_rn[l][m];
    /* P[d][c]: component c (x,y,z frame) of the d-weighted moment */
    double PD[3][3], PS[3][3];
    const double* t0 = Tt + (n * (n + 1) / 2 + (m - 1)) * 12; /* order m-1 (always <= n) */
    const bool h1 = m <= n, h2 = m + 1 <= n;
    const double* t1 = Tt + (n * (n + 1) / 2 + m) * 12;
    const double* t2 = Tt + (n * (n + 1) / 2 + m + 1) * 12;
#pragma unroll
    for (int d = 0; d < 6; ++d) {
      const double ar = t0[2 * d], ai = t0[2 * d + 1];
      const double zi = h1 ? t1[2 * d + 1] : 0.0;
      const double br = h2 ? t2[2 * d] : 0.0, bi = h2 ? t2[2 * d + 1] : 0.0;
      double* P = d < 3 ? PD[d] : PS[d - 3];
      P[0] = Nf * zi;
      P[1] = 0.5 * Nf * (ai - bi);
      P[2] = 0.5 * Nf * (ar + br);
    }
    /* h(x) and grad h(x) */
    const double hx = Nf * Rx[2 * (l * (l + 1) / 2 + m) + 1];
    const double* q0 = Rx + 2 * (n * (n + 1) / 2 + (m - 1));
    const double gzi = h1 ? Rx[2 * (n * (n + 1) / 2 + m) + 1] : 0.0;
    const double q2r = h2 ? Rx[2 * (n * (n + 1) / 2 + m + 1)] : 0.0;
    const double q2i = h2 ? Rx[2 * (n * (n + 1) / 2 + m + 1) + 1] : 0.0;
    const double gx = Nf * gzi, gy = 0.5 * Nf * (q0[1] - q2i), gz = 0.5 * Nf * (q0[0] + q2r);
    JD[0 * hd + k] = -(PD[0][0] + PD[1][1] + PD[2][2]) - (wv0 * gx + wv1 * gy + wv2 * gz);
    JD[1 * hd + k] = (PD[1][2] - PD[2][1]) + s0 * gx + (wv1 * gz - wv2 * gy);
    JD[2 * hd + k] = (PD[2][0] - PD[0][2]) + s0 * gy + (wv2 * gx - wv0 * gz);
    JD[3 * hd + k] = (PD[0][1] - PD[1][0]) + s0 * gz + (wv0 * gy - wv1 * gx);
    RS[k] = (PS[0][0] + PS[1][1] + PS[2][2]) + hx * Omega * i4p;
  }
}

/* ===================================================================== */
/* K6: RRQ solves as matrix products per panel + naive subtraction + COO */
/* ===================================================================== */
#define AT 64  /* RRQ targets per chunk: 8 warps x 8 */
#define AK 32  /* inner-dimension tile */
#define AKS 36 /* tile row stride (doubles): m8n8k4 fragment loads hit 16 distinct bank pairs */
/* Out[t][j] += sum_k A[t][k] Bt[j][k] over k < K on the FP64 tensor path, for the
 * chunk's targets t (warp w: 8w..8w+7) and all NB column blocks of 8;
 * load(k0, sA_tile, sB_tile) fills the K tile [k0, k0+AK) (A: AT x AKS, Bt: 8NB x AKS,
 * zero outside the data) */
template <int NB, class Load>
__device__ __forceinline__ void apply_dmma(int K, double (&acc)[NB][2], double* sAt, double* sBt, Load load) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int fr = lane >> 2, fc = lane & 3;
  for (int k0 = 0; k0 < K; k0 += AK) {
    __syncthreads();
    load(k0, sAt, sBt);
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
#pragma unroll 2
    for (int ks = 0; ks < AK / 4; ++ks) {
      const double a = sAt[(8 * w + fr) * AKS + 4 * ks + fc];
#pragma unroll
      for (int b = 0; b < NB; ++b) dmma(acc[b][0], acc[b][1], a, sBt[(8 * b + fr) * AKS + 4 * ks + fc]);
    }
  }
}
__device__ __forceinline__ void cp_or_zero(double* dst, const double* src, bool ok) {
  if (ok) cp_async8(dst, src);
  else *dst = 0.0;
}

/* per panel, chunks of AT RRQ targets: Ad = PD JD, As = (PS RS + B Ad) / alpha,
 * naive-block subtraction and the COO values (and Omega for qol_rrq) */
template <int NB>
__global__ void __launch_bounds__(256, 2) k_rrq_apply(OrderTab T, PanelIn P, PairIn Q, PairWS G, RRQWS R, OutCOO O) {
  const int pan = R.plo + blockIdx.x;
  const int cnt = G.cnt[(size_t)pan * 8 + T.nlevel + 1];
  if (cnt == 0) return;
  const int hd = T.hd, N4 = 4 * hd;
  const long long p0 = Q.tcxi[pan] - 1, m = Q.tcxi[pan + 1] - Q.tcxi[pan];
  const int offl = G.off[(size_t)pan * 8 + T.nlevel + 1];
  const long long g0 = R.rrq_off[pan];
  const double* PD = R.PD + (size_t)pan * hd * N4;
  const double* PS = R.smat + (size_t)pan * hd * hd;
  const double* B = R.B + (size_t)pan * hd * hd;
  const double alpha = R.frame[(size_t)pan * RRQ_FRAME + 12];
  extern __shared__ __align__(16) double sm[];
  double* sAt = sm;                 /* AT x AKS */
  double* sBt = sAt + AT * AKS;     /* 8NB x AKS */
  double* sAd = sBt + 8 * NB * AKS; /* AT x hd: Ad of the chunk */
  __shared__ int tloc[AT];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int fr = lane >> 2, fc = lane & 3;
  const double i4p = 1.0 / (4.0 * QOL_PI);
  for (int c0 = 0; c0 < cnt; c0 += AT) {
    const int nt = min(AT, cnt - c0);
    __syncthreads();
    if (threadIdx.x < AT) tloc[threadIdx.x] = threadIdx.x < nt ? G.grp[p0 + offl + c0 + threadIdx.x] : 0;
    double acc[NB][2];
#pragma unroll
    for (int b = 0; b < NB; ++b) { acc[b][0] = 0.0; acc[b][1] = 0.0; }
    const double* JD = R.JD + (size_t)(g0 + c0) * N4;
    const double* RS = R.RS + (size_t)(g0 + c0) * hd;
    /* Ad[t][j] = sum_q JD[t][q] PD[j][q] */
    apply_dmma<NB>(N4, acc, sAt, sBt, [&](int k0, double* a, double* bt) {
      /* 16-byte pieces: N4 is even, so a piece never straddles the row end */
      for (int e = threadIdx.x; e < AT * AK / 2; e += blockDim.x) {
        const int t = e / (AK / 2), k = 2 * (e % (AK / 2));
        if (t < nt && k0 + k < N4) cp_async16(&a[t * AKS + k], JD + (size_t)t * N4 + k0 + k);
        else { a[t * AKS + k] = 0.0; a[t * AKS + k + 1] = 0.0; }
      }
      for (int e = threadIdx.x; e < 8 * NB * AK / 2; e += blockDim.x) {
        const int j = e / (AK / 2), k = 2 * (e % (AK / 2));
        if (j < hd && k0 + k < N4) cp_async16(&bt[j * AKS + k], PD + (size_t)j * N4 + k0 + k);
        else { bt[j * AKS + k] = 0.0; bt[j * AKS + k + 1] = 0.0; }
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    });
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int t = 8 * w + fr, j = 8 * b + 2 * fc + h;
        if (j < hd) sAd[t * hd + j] = acc[b][h];
        acc[b][h] = 0.0;
      }
    __syncthreads();
    /* As[t][i] = sum_k RS[t][k] PS[i][k] + sum_j Ad[t][j] B[i][j] */
    apply_dmma<NB>(2 * hd, acc, sAt, sBt, [&](int k0, double* a, double* bt) {
      for (int e = threadIdx.x; e < AT * AK; e += blockDim.x) {
        const int t = e / AK, k = e % AK, kk = k0 + k;
        if (kk < hd) cp_or_zero(&a[t * AKS + k], RS + (size_t)t * hd + kk, t < nt);
        else a[t * AKS + k] = (kk < 2 * hd) ? sAd[t * hd + kk - hd] : 0.0;
      }
      for (int e = threadIdx.x; e < 8 * NB * AK; e += blockDim.x) {
        const int i = e / AK, k = e % AK, kk = k0 + k;
        const bool ok = i < hd && kk < 2 * hd;
        cp_or_zero(&bt[i * AKS + k], kk < hd ? PS + (size_t)i * hd + kk : B + (size_t)i * hd + (kk - hd), ok);
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    });
    /* naive block, COO values */
    const int t = 8 * w + fr;
    if (t < nt) {
      const int tl = tloc[t];
      const long long row = Q.tcxrow[p0 + tl];
      const double* x = Q.tcx + 3 * (p0 + tl);
      const double x0 = x[0], x1 = x[1], x2 = x[2];
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int j = 8 * b + 2 * fc + h;
          if (j >= hd) continue;
          double vs = acc[b][h] / alpha, vd = sAd[t * hd + j];
          if (O.subtract_naive) {
            const size_t gj = (size_t)pan * hd + j;
            double ns = 0.0, nd = 0.0;
            if (row != (long long)gj + 1)
              sdl_kernel(x0 - P.sx[3 * gj], x1 - P.sx[3 * gj + 1], x2 - P.sx[3 * gj + 2], P.snx[3 * gj],
                         P.snx[3 * gj + 1], P.snx[3 * gj + 2], P.sw[gj] * i4p, ns, nd);
            vs -= ns; vd -= nd;
          }
          const size_t o = (size_t)p0 * hd + (size_t)j * m + tl;
          O.vs[o] = vs;
          O.vd[o] = vd;
        }
    }
    /* Omega (reference layout, qol_rrq only): (J_s, -J_x, -J_y, -J_z)/alpha */
    if (O.omega)
      for (int e = threadIdx.x; e < N4 * nt; e += blockDim.x) {
        int tt = e / N4, q = e % N4;
        double v = R.JD[(size_t)(g0 + c0 + tt) * N4 + q];
        O.omega[(size_t)tloc[tt] * N4 + q] = (q < hd ? v : -v) / alpha;
      }
  }
}
template <int NB>
constexpr size_t apply_smem(int hd) {
  return sizeof(double) * ((size_t)AT * AKS + (size_t)8 * NB * AKS + (size_t)AT * hd);
}

/* ===================================================================== */
/* K7: COO row/column indices (block column-major per panel)            */
/* ===================================================================== */
/* (panel, local target) of every RRQ pair, in RRQ pair order */
__global__ void __launch_bounds__(128) k_rrq_pairs(OrderTab T, PairIn Q, PairWS G, RRQWS R) {
  const int pan = blockIdx.x;
  const long long g0 = R.rrq_off[pan], n = R.rrq_off[pan + 1] - g0;
  const long long p0 = Q.tcxi[pan] - 1;
  const int* grp = G.grp + p0 + G.off[(size_t)pan * 8 + T.nlevel + 1];
  for (long long j = threadIdx.x; j < n; j += blockDim.x) R.pair[g0 + j] = make_int2(pan, grp[j]);
}

__global__ void __launch_bounds__(256) k_coo_index(OrderTab T, PairIn Q, long long* si, long long* sj) {
  const int pan = blockIdx.x, hd = T.hd;
  const long long p0 = Q.tcxi[pan] - 1, m = Q.tcxi[pan + 1] - Q.tcxi[pan];
  const long long* row = Q.tcxrow + p0;
  long long* oi = si + (size_t)p0 * hd;
  long long* oj = sj + (size_t)p0 * hd;
  const long long c1 = (long long)pan * hd + 1;
  if (m * hd < (1LL << 31)) { /* the usual block: 32-bit index arithmetic */
    const int mi = (int)m, tot = mi * hd;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      const int j = e / mi, i = e - j * mi;
      oi[e] = __ldg(row + i);
      oj[e] = c1 + j;
    }
  } else {
    for (long long e = threadIdx.x; e < m * hd; e += blockDim.x) {
      const long long j = e / m, i = e - j * m;
      oi[e] = __ldg(row + i);
      oj[e] = c1 + j;
    }
  }
}

/* ===================================================================== */
/* small scan of per-panel RRQ counts                                    */
/* ===================================================================== */
__global__ void k_scan_rrq(int npan, int lev, const int* cnt, long long* off) {
  __shared__ long long part[1024];
  const int nth = blockDim.x, tid = threadIdx.x;
  const int per = (npan + nth - 1) / nth;
  const int a = tid * per, b = min(npan, a + per);
  long long s = 0;
  for (int i = a; i < b; ++i) s += cnt[(size_t)i * 8 + lev];
  part[tid] = s;
  __syncthreads();
  if (tid == 0) {
    long long acc = 0;
    for (int i = 0; i < nth; ++i) { long long v = part[i]; part[i] = acc; acc += v; }
    off[npan] = acc;
  }
  __syncthreads();
  long long acc = part[tid];
  for (int i = a; i < b; ++i) { off[i] = acc; acc += cnt[(size_t)i * 8 + lev]; }
}

/* ===================================================================== */
/* launchers                                                             */
/* ===================================================================== */
cudaError_t qol_launch_levels(const OrderTab& T, const PanelIn& P, const LevelWS& W, int npan, cudaStream_t st) {
  if (npan <= 0) return cudaSuccess;
  if (T.ncw < ((T.hd + 3) & ~3)) return cudaErrorInvalidValue; /* the padded rows cover the k-steps */
  int nch = 0, nsubt = 0;
  for (int l = 0; l < T.nlevel; ++l) {
    nch += (T.n[l] + LV_M - 1) / LV_M;
    nsubt += T.nsub[l];
  }
  const size_t smem = level_nodes_smem(T.hd);
  cudaFuncSetAttribute(k_level_nodes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_level_nodes<<<dim3((npan + LV_P - 1) / LV_P, nch), 256, smem, st>>>(T, P, W, npan);
  const long long nt = (long long)npan * nsubt;
  k_level_subs<<<(unsigned)((nt + 127) / 128), 128, 0, st>>>(T, W, npan);
  return cudaGetLastError();
}
cudaError_t qol_launch_classify(const OrderTab& T, const PairIn& Q, const LevelWS& W, const PairWS& G, int npan,
                                cudaStream_t st, int preset) {
  k_classify<<<npan, 128, 0, st>>>(T, Q, W, G, preset);
  return cudaGetLastError();
}
cudaError_t qol_launch_direct(const OrderTab& T, const PanelIn& P, const PairIn& Q, const LevelWS& W,
                              const PairWS& G, const OutCOO& O, int npan, cudaStream_t st, int pan0) {
  if (npan <= 0) return cudaSuccess;
  dim3 grid(npan, T.nlevel);
  auto go = [&](auto kern, size_t smem) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<grid, 256, smem, st>>>(T, P, Q, W, G, O, pan0);
  };
  const int nb = T.ncw / 32; /* the padded interpolation rows fix the column blocks */
  if (nb < 1 || nb > 5 || T.ncw != 32 * ((T.hd + 31) / 32)) return cudaErrorInvalidValue;
  if (T.sum_fp32) { /* the precision variant: UTHREADS threads a CTA */
    auto gu = [&](auto kern, size_t smem) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      kern<<<grid, UTHREADS, smem, st>>>(T, P, Q, W, G, O, pan0);
    };
    switch (nb) {
      case 1: gu(k_direct_umma<1>, UmmaShape<1>::SMEM); break;
      case 2: gu(k_direct_umma<2>, UmmaShape<2>::SMEM); break;
      case 3: gu(k_direct_umma<3>, UmmaShape<3>::SMEM); break;
      case 4: gu(k_direct_umma<4>, UmmaShape<4>::SMEM); break;
      case 5: gu(k_direct_umma<5>, UmmaShape<5>::SMEM); break;
    }
    return cudaGetLastError();
  }
  switch (nb) {
    case 1: go(k_direct<1>, direct_smem<1>()); break;
    case 2: go(k_direct<2>, direct_smem<2>()); break;
    case 3: go(k_direct<3>, direct_smem<3>()); break;
    case 4: go(k_direct<4>, direct_smem<4>()); break;
    case 5: go(k_direct<5>, direct_smem<5>()); break;
  }
  return cudaGetLastError();
}
cudaError_t qol_wait_error(unsigned* flag, cudaStream_t st) {
  cudaError_t e = cudaMemcpyFromSymbolAsync(flag, g_qol_wait_err, sizeof(unsigned), 0, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && *flag) {
    const unsigned z = 0;
    e = cudaMemcpyToSymbolAsync(g_qol_wait_err, &z, sizeof z, 0, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  return e;
}
cudaError_t qol_launch_direct_queue(const DirectJob* jobs, int nbmax, const int* items, int nitems, int* head,
                                    cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const unsigned grid = (unsigned)std::min(2 * nsm, nitems); /* two resident CTAs an SM */
  auto go = [&](auto kern, size_t smem) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<grid, 256, smem, st>>>(jobs, items, nitems, head);
  };
  switch (nbmax) {
    case 1: go(k_direct_queue<1>, direct_smem<1>()); break;
    case 2: go(k_direct_queue<2>, direct_smem<2>()); break;
    case 3: go(k_direct_queue<3>, direct_smem<3>()); break;
    case 4: go(k_direct_queue<4>, direct_smem<4>()); break;
    case 5: go(k_direct_queue<5>, direct_smem<5>()); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t qol_launch_direct_cut(const OrderTab& T, const PanelIn& P, const PairIn& Q, const LevelWS& W,
                                  const PairWS& G, const OutCOO& O, int npan, cudaStream_t st, int pan0) {
  if (npan <= 0 || !T.adaptive) return cudaSuccess;
  if (T.hd > 32 * CUT_MAXC || T.nlevel != 4 || T.nsub[T.nlevel - 2] > 32) return cudaErrorInvalidValue;
  k_direct_cut<<<npan, 256, 0, st>>>(T, P, Q, W, G, O, pan0);
  return cudaGetLastError();
}
cudaError_t qol_launch_scan(int npan, int lev, const int* cnt, long long* off, cudaStream_t st) {
  k_scan_rrq<<<1, 1024, 0, st>>>(npan, lev, cnt, off);
  return cudaGetLastError();
}
/* the blocked panel kernel's cluster sizes for hd: every CS whose columns fit
 * (shared memory <= 227 KB, at most 9 column tiles a CTA), smallest first */
static int pblk_cluster_sizes(int hd, int* out) {
  int n = 0;
  for (int cs : {1, 2, 4, 8}) {
    if (pblk_ncol(hd, cs) > 64 || pblk_smem_bytes(hd, cs) > 227 * 1024) continue;
    if (cs > 1 && pblk_ncol(hd, cs) * (cs - 1) >= hd) continue; /* every CTA owns a valid column */
    out[n++] = cs;
  }
  return n;
}
cudaError_t qol_launch_rrq_panel(const OrderTab& T, const PanelIn& P, const PairWS& G, const RRQWS& R, int npan,
                                 const double* chart, cudaStream_t st) {
  if (npan <= 0) return cudaSuccess;
  int sizes[4];
  const int nsz = pblk_cluster_sizes(T.hd, sizes);
  if (nsz == 0) return cudaErrorInvalidConfiguration;
  /* a cluster size chosen by measurement (qol_panel_shapes lists them), else the smallest */
  int cs = sizes[0];
  if (T.panel_cs)
    for (int i = 0; i < nsz; ++i)
      if (sizes[i] == T.panel_cs) cs = T.panel_cs;
  const size_t smem = pblk_smem_bytes(T.hd, cs);
  const int nt = pblk_threads(T.hd, cs);
  auto go = [&](auto kern) -> cudaError_t {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (cs > 1) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(npan * cs));
    cfg.blockDim = dim3((unsigned)nt);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, T, P, G, R, chart);
  };
  const bool wide = pblk_hq(T.hd) > 96;
  switch (cs) {
    case 1: return wide ? go(k_rrq_panel_blk<1, 5>) : go(k_rrq_panel_blk<1, 3>);
    case 2: return wide ? go(k_rrq_panel_blk<2, 5>) : go(k_rrq_panel_blk<2, 3>);
    case 4: return wide ? go(k_rrq_panel_blk<4, 5>) : go(k_rrq_panel_blk<4, 3>);
    default: return wide ? go(k_rrq_panel_blk<8, 5>) : go(k_rrq_panel_blk<8, 3>);
  }
}
int qol_panel_shapes(int hd, int nquad, int* cs, int* nt, int cap) {
  (void)nquad;
  int sizes[4];
  const int n = pblk_cluster_sizes(hd, sizes);
  int k = 0;
  for (int i = 0; i < n && k < cap; ++i, ++k) { cs[k] = sizes[i]; nt[k] = pblk_threads(hd, sizes[i]); }
  return k;
}
cudaError_t qol_launch_rrq_pairs(const OrderTab& T, const PairIn& Q, const PairWS& G, const RRQWS& R, int npan,
                                 cudaStream_t st) {
  if (npan <= 0 || R.nrrq == 0) return cudaSuccess;
  k_rrq_pairs<<<npan, 128, 0, st>>>(T, Q, G, R);
  return cudaGetLastError();
}
cudaError_t qol_launch_rrq_ssq(const OrderTab& T, const PairIn& Q, const PairWS& G, const RRQWS& R, cudaStream_t st) {
  const long long n = R.ghi - R.glo;
  if (n <= 0) return cudaSuccess;
  k_rrq_ssq<<<(unsigned)((3 * n + 127) / 128), 128, 0, st>>>(T, Q, G, R);
  return cudaGetLastError();
}
cudaError_t qol_launch_rrq_geom(const OrderTab& T, const PairIn& Q, const PairWS& G, const RRQWS& R, int exterior,
                                cudaStream_t st) {
  const long long n = R.ghi - R.glo;
  if (n <= 0) return cudaSuccess;
  k_rrq_side<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(T, Q, R);
  long long nb = (n + RRQ_WARPS - 1) / RRQ_WARPS;
  k_rrq_geom<<<(unsigned)nb, 32 * RRQ_WARPS, 0, st>>>(T, Q, G, R, exterior);
  return cudaGetLastError();
}
cudaError_t qol_launch_rrq_target(const OrderTab& T, const PairIn& Q, const PairWS& G, const RRQWS& R, int exterior,
                                  cudaStream_t st) {
  cudaError_t e = qol_launch_rrq_ssq(T, Q, G, R, st);
  if (e == cudaSuccess) e = qol_launch_rrq_geom(T, Q, G, R, exterior, st);
  if (e == cudaSuccess) e = qol_launch_rrq_moments(T, Q, G, R, st);
  return e;
}
cudaError_t qol_launch_rrq_moments(const OrderTab& T, const PairIn& Q, const PairWS& G, const RRQWS& R,
                                   cudaStream_t st) {
  const long long n = R.ghi - R.glo;
  if (n <= 0) return cudaSuccess;
  const size_t smem = sizeof(double) * (mom_rec(3 * T.nquad) + mom_region(T.nterms, T.xslots));
  auto go = [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<(unsigned)n, MOM_T, smem, st>>>(T, Q, G, R);
  };
  if (T.nterms <= 4) go(k_rrq_moments<4>);
  else if (T.nterms <= 6) go(k_rrq_moments<6>);
  else if (T.nterms <= 8) go(k_rrq_moments<8>);
  else if (T.nterms <= 10) go(k_rrq_moments<10>);
  else if (T.nterms <= 12) go(k_rrq_moments<12>);
  else if (T.nterms <= 14) go(k_rrq_moments<14>);
  else go(k_rrq_moments<16>);
  return cudaGetLastError();
}
cudaError_t qol_launch_rrq_apply(const OrderTab& T, const PanelIn& P, const PairIn& Q, const PairWS& G,
                                 const RRQWS& R, const OutCOO& O, cudaStream_t st) {
  const int npan = R.phi - R.plo;
  if (npan <= 0) return cudaSuccess;
  auto go = [&](auto kern, size_t smem) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<npan, 256, smem, st>>>(T, P, Q, G, R, O);
  };
  switch ((T.hd + 7) / 8) { /* column blocks of 8 */
    case 1: go(k_rrq_apply<1>, apply_smem<1>(T.hd)); break;
    case 2: go(k_rrq_apply<2>, apply_smem<2>(T.hd)); break;
    case 3: go(k_rrq_apply<3>, apply_smem<3>(T.hd)); break;
    case 4: go(k_rrq_apply<4>, apply_smem<4>(T.hd)); break;
    case 5: go(k_rrq_apply<5>, apply_smem<5>(T.hd)); break;
    case 6: go(k_rrq_apply<6>, apply_smem<6>(T.hd)); break;
    case 7: go(k_rrq_apply<7>, apply_smem<7>(T.hd)); break;
    case 8: go(k_rrq_apply<8>, apply_smem<8>(T.hd)); break;
    case 9: go(k_rrq_apply<9>, apply_smem<9>(T.hd)); break;
    case 10: go(k_rrq_apply<10>, apply_smem<10>(T.hd)); break;
    case 11: go(k_rrq_apply<11>, apply_smem<11>(T.hd)); break;
    case 12: go(k_rrq_apply<12>, apply_smem<12>(T.hd)); break;
    case 13: go(k_rrq_apply<13>, apply_smem<13>(T.hd)); break;
    case 14: go(k_rrq_apply<14>, apply_smem<14>(T.hd)); break;
    case 15: go(k_rrq_apply<15>, apply_smem<15>(T.hd)); break;
    case 16: go(k_rrq_apply<16>, apply_smem<16>(T.hd)); break;
    default: go(k_rrq_apply<17>, apply_smem<17>(T.hd)); break;
  }
  return cudaGetLastError();
}
cudaError_t qol_launch_coo_index(const OrderTab& T, const PairIn& Q, long long* si, long long* sj, int npan,
                                 cudaStream_t st) {
  k_coo_index<<<npan, 256, 0, st>>>(T, Q, si, sj);
  return cudaGetLastError();
}


/* ===================================================================== */
/* surface panels (the reference's geometry generator, geo_core,          */
/* utils/stellarator_geo_mex.c:636-750): one CTA per chart, p^2 threads   */
/* ===================================================================== */
/* chart c: (a1, b1, a2, b2, jj, ii) at charts[6c..]; the Fourier surface
 * sampled on the p x p Gauss grid of the chart, its t- and p-derivatives by
 * the spectral differentiation matrix D, and the chart's two triangles'
 * Vioreanu-Rokhlin nodes by tensor Lagrange interpolation (tables: 4
 * orientations x hd x p^2); outputs in the reference layout, triangle 2c + s */
__global__ void __launch_bounds__(256) k_surface_panels(int nmode, const double* modes, int nfp, int p, int hd,
                                                        const double* charts, double ts1, double ts2,
                                                        const double* x0, const double* D, const double* wts,
                                                        const double* tables, double* sx, double* snx, double* sw,
                                                        double* rts, double* rps) {
  extern __shared__ double gsm[];
  const int P2 = p * p, c = blockIdx.x, tid = threadIdx.x;
  double* G = gsm;           /* p^2 x 9: x, x_t, x_p */
  const double* ch = charts + 6 * (size_t)c;
  if (tid < P2) {
    const int a = tid % p, b = tid / p;
    const double uu = ((ch[0] * x0[b] + ch[1]) + 2.0 * ch[4]) * ts1;
    const double vv = ((ch[2] * x0[a] + ch[3]) + 2.0 * ch[5]) * ts2;
    double R = 0.0, Z = 0.0;
    for (int k = 0; k < nmode; ++k) {
      const double ang = modes[4 * k] * vv - nfp * modes[4 * k + 1] * uu;
      R = R + modes[4 * k + 2] * cos(ang);
      Z = Z + modes[4 * k + 3] * sin(ang);
    }
    G[9 * tid] = R * cos(uu); G[9 * tid + 1] = R * sin(uu); G[9 * tid + 2] = Z;
  }
  __syncthreads();
  if (tid < P2) { /* node m = a + b p: d/da along the row, d/db along the column */
    const int a = tid % p, b = tid / p;
    double ta[3] = {0.0, 0.0, 0.0}, tb[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < p; ++k) {
      const double da = D[a + (size_t)p * k], db = D[b + (size_t)p * k]; /* D[row][k], column-major */
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        ta[d] += da * G[9 * (k + b * p) + d];
        tb[d] += db * G[9 * (a + k * p) + d];
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) { G[9 * tid + 3 + d] = ta[d]; G[9 * tid + 6 + d] = tb[d]; }
  }
  __syncthreads();
  double d1 = 0.0, d2 = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double e1 = G[d] - G[9 * (P2 - 1) + d], e2 = G[9 * (p - 1) + d] - G[9 * (P2 - p) + d];
    d1 += e1 * e1; d2 += e2 * e2;
  }
  const int key0 = d1 + 1e-13 > d2 ? 0 : 2; /* (lA, rA) or (lB, rB) */
  for (int e = tid; e < 2 * hd; e += blockDim.x) {
    const int s = e / hd, i = e % hd, key = key0 + s;
    const double* M = tables + ((size_t)key * hd + i) * P2;
    double acc[9];
#pragma unroll
    for (int f = 0; f < 9; ++f) acc[f] = 0.0;
    for (int m = 0; m < P2; ++m) {
      const double w = M[m];
#pragma unroll
      for (int f = 0; f < 9; ++f) acc[f] += w * G[9 * m + f];
    }
    /* xt = d/d(row index) = acc[3..5], xp = acc[6..8] (geometry.panels' rts, rps) */
    const double n0 = acc[7] * acc[5] - acc[8] * acc[4], n1 = acc[8] * acc[3] - acc[6] * acc[5],
                 n2 = acc[6] * acc[4] - acc[7] * acc[3];
    const double sp = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    const size_t o = (size_t)(2 * c + s) * hd + i;
    sx[3 * o] = acc[0]; sx[3 * o + 1] = acc[1]; sx[3 * o + 2] = acc[2];
    snx[3 * o] = n0 / sp; snx[3 * o + 1] = n1 / sp; snx[3 * o + 2] = n2 / sp;
    rts[3 * o] = 2.0 * acc[3]; rts[3 * o + 1] = 2.0 * acc[4]; rts[3 * o + 2] = 2.0 * acc[5];
    rps[3 * o] = 2.0 * acc[6]; rps[3 * o + 1] = 2.0 * acc[7]; rps[3 * o + 2] = 2.0 * acc[8];
    sw[o] = sp * wts[i] * 4.0;
  }
}
cudaError_t qol_launch_surface_panels(int nchart, int nmode, const double* modes, int nfp, int p,
                                      const double* charts, double ts1, double ts2, const double* x0,
                                      const double* D, const double* wts, const double* tables, double* sx,
                                      double* snx, double* sw, double* rts, double* rps, cudaStream_t st) {
  if (nchart <= 0) return cudaSuccess;
  const int hd = p * (p + 1) / 2;
  const size_t smem = sizeof(double) * 9 * (size_t)p * p;
  k_surface_panels<<<nchart, 256, smem, st>>>(nmode, modes, nfp, p, hd, charts, ts1, ts2, x0, D, wts, tables, sx,
                                               snx, sw, rts, rps);
  return cudaGetLastError();
}

/* ===================================================================== */
/* FP64 FMA throughput probe (roofline denominator for the FP64 kernels)  */
/* ===================================================================== */
__global__ void __launch_bounds__(256) k_fp64_peak(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-3, x1 = x0 + 1.0, x2 = x0 + 2.0, x3 = x0 + 3.0;
  double x4 = x0 + 4.0, x5 = x0 + 5.0, x6 = x0 + 6.0, x7 = x0 + 7.0;
  for (int i = 0; i < iters; ++i) {
    x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
    x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
  }
  double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 12345.678) out[blockIdx.x] = s; /* keep the chains alive */
}

cudaError_t qol_launch_fp64_peak(double* out, int blocks, int iters, cudaStream_t st) {
  k_fp64_peak<<<blocks, 256, 0, st>>>(out, iters, 0.999999999, 1e-9);
  return cudaGetLastError();
}
/* ===================================================================== */
/* GRF near phase (stellarator_grf_core_mod.f90:652-899) and the Direct    */
/* far field (:566-606) on the GPU                                        */
/* ===================================================================== */
/* ball of panel k: centre = mean of its hd nodes (summed in node order),
 * radius 1.75 sqrt(sum sw); stored (qx, qy, qz, qr^2) */
__global__ void k_ball_centers(int npan, int hd, const double* sx, const double* sw, double* ball) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npan) return;
  double qp0 = 0.0, qp1 = 0.0, qp2 = 0.0, s = 0.0;
  for (int i = 0; i < hd; ++i) {
    const size_t j = (size_t)k * hd + i;
    qp0 = __dadd_rn(qp0, sx[3 * j]); qp1 = __dadd_rn(qp1, sx[3 * j + 1]); qp2 = __dadd_rn(qp2, sx[3 * j + 2]);
    s = __dadd_rn(s, sw[j]);
  }
  const double qr = __dmul_rn(1.75, sqrt(s));
  ball[4 * k] = qp0 / (double)hd;
  ball[4 * k + 1] = qp1 / (double)hd;
  ball[4 * k + 2] = qp2 / (double)hd;
  ball[4 * k + 3] = __dmul_rn(qr, qr);
}
/* the ball test exactly as written in the reference (no fused multiply-adds) */
__device__ __forceinline__ bool in_ball(const double* x, const double* b) {
  const double a = __dadd_rn(x[0], -b[0]), c = __dadd_rn(x[1], -b[1]), e = __dadd_rn(x[2], -b[2]);
  return __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(c, c)), __dmul_rn(e, e)) < b[3];
}
/* Near search by node chunks: the nodes in source order are cut into chunks of
 * BALL_CH; a chunk's axis-aligned bounding box is tested against a panel's
 * ball first (conservatively: the box distance is at most any node's) and only
 * the nodes of chunks that can reach the ball get the exact test.  Sources of
 * consecutive panels are neighbours on the surface, so a ball reaches a few
 * chunks; the panel's list stays in source order (chunks in order, nodes in
 * order within a chunk): the reference's CSR, without a sort. */
#define BALL_CH 256
__global__ void __launch_bounds__(BALL_CH) k_chunk_boxes(long long nsrc, const double* sx, double* box) {
  __shared__ double red[6][BALL_CH / 32];
  const long long j = (long long)blockIdx.x * BALL_CH + threadIdx.x;
  double v[6];
  if (j < nsrc) {
    for (int d = 0; d < 3; ++d) { v[d] = sx[3 * j + d]; v[3 + d] = v[d]; }
  } else {
    for (int d = 0; d < 3; ++d) { v[d] = 1e300; v[3 + d] = -1e300; }
  }
  for (int o = 16; o > 0; o >>= 1)
    for (int d = 0; d < 3; ++d) {
      v[d] = fmin(v[d], __shfl_xor_sync(0xffffffffu, v[d], o));
      v[3 + d] = fmax(v[3 + d], __shfl_xor_sync(0xffffffffu, v[3 + d], o));
    }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
    for (int d = 0; d < 6; ++d) red[d][w] = v[d];
  __syncthreads();
  if (threadIdx.x < 6) {
    const int d = threadIdx.x;
    double r = red[d][0];
    for (int q = 1; q < BALL_CH / 32; ++q) r = d < 3 ? fmin(r, red[d][q]) : fmax(r, red[d][q]);
    box[6 * (size_t)blockIdx.x + d] = r;
  }
}
__device__ __forceinline__ bool ball_reaches_box(const double* b, const double* box) {
  double d2 = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double t = fmax(fmax(box[d] - b[d], b[d] - box[3 + d]), 0.0);
    d2 += t * t;
  }
  return d2 <= b[3] * (1.0 + 1e-12);
}
/* this CTA's chunks that reach ball b among chunks [c0, c0 + blockDim.x),
 * in order, into list[0 .. return) */
__device__ int reaching_chunks(const double* b, const double* box, long long nchunk, long long c0, int* list,
                               int* wcnt) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const long long c = c0 + threadIdx.x;
  const bool hit = c < nchunk && ball_reaches_box(b, box + 6 * c);
  const unsigned m = __ballot_sync(0xffffffffu, hit);
  if (lane == 0) wcnt[w] = __popc(m);
  __syncthreads();
  int before = 0, total = 0;
  for (int q = 0; q < nw; ++q) { if (q < w) before += wcnt[q]; total += wcnt[q]; }
  if (hit) list[before + __popc(m & ((1u << lane) - 1u))] = (int)(c - c0);
  __syncthreads();
  return total;
}
/* near sources per panel (CTA per panel) */
__global__ void __launch_bounds__(BALL_CH) k_ball_count(long long nsrc, const double* sx, const double* ball,
                                                        const double* box, long long* counts) {
  const int k = blockIdx.x;
  __shared__ double b[4];
  __shared__ long long part[BALL_CH / 32];
  __shared__ int list[BALL_CH], wcnt[BALL_CH / 32];
  if (threadIdx.x < 4) b[threadIdx.x] = ball[4 * k + threadIdx.x];
  __syncthreads();
  const long long nchunk = (nsrc + BALL_CH - 1) / BALL_CH;
  long long c = 0;
  for (long long c0 = 0; c0 < nchunk; c0 += BALL_CH) {
    const int nl = reaching_chunks(b, box, nchunk, c0, list, wcnt);
    for (int q = 0; q < nl; ++q) {
      const long long j = (c0 + list[q]) * BALL_CH + threadIdx.x;
      c += (j < nsrc && in_ball(sx + 3 * j, b)) ? 1 : 0;
    }
    __syncthreads();
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
    counts[k] = t;
  }
}
/* their 1-based indices in source order (the reference's CSR), the target
 * coordinates gathered alongside */
__global__ void __launch_bounds__(BALL_CH) k_ball_fill(long long nsrc, const double* sx, const double* ball,
                                                       const double* box, const long long* offs, long long* csr_idx,
                                                       double* tcx, long long* csr_loc /* nullable */,
                                                       long long row_shift) {
  const int k = blockIdx.x;
  __shared__ double b[4];
  __shared__ int wcnt[BALL_CH / 32], list[BALL_CH], lcnt[BALL_CH / 32];
  if (threadIdx.x < 4) b[threadIdx.x] = ball[4 * k + threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const long long nchunk = (nsrc + BALL_CH - 1) / BALL_CH;
  long long base = offs[k];
  for (long long c0 = 0; c0 < nchunk; c0 += BALL_CH) {
    const int nl = reaching_chunks(b, box, nchunk, c0, list, lcnt);
    for (int q = 0; q < nl; ++q) {
      const long long j = (c0 + list[q]) * BALL_CH + threadIdx.x;
      const bool hit = j < nsrc && in_ball(sx + 3 * j, b);
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if (lane == 0) wcnt[w] = __popc(m);
      __syncthreads();
      int before = 0, total = 0;
      for (int qq = 0; qq < nw; ++qq) { if (qq < w) before += wcnt[qq]; total += wcnt[qq]; }
      if (hit) {
        const long long pos = base + before + __popc(m & ((1u << lane) - 1u));
        csr_idx[pos] = j + 1;
        if (csr_loc) csr_loc[pos] = j + 1 - row_shift; /* the pipeline's numbering of a panel range */
        tcx[3 * pos] = sx[3 * j]; tcx[3 * pos + 1] = sx[3 * j + 1]; tcx[3 * pos + 2] = sx[3 * j + 2];
      }
      base += total;
      __syncthreads();
    }
  }
}
/* csr_val[o0+j] = sum_k (S - S_naive)[j][k] ubn_k - (D - D_naive)[j][k] ub_k over
 * the panel's hd nodes, in node order (the COO values are already minus the
 * naive block) */
__global__ void __launch_bounds__(256) k_grf_fill(int hd, const long long* offs, const double* vs, const double* vd,
                                                  const double* ub, const double* ubn, double* csr_val) {
  const int k = blockIdx.x;
  const long long o0 = offs[k], m = offs[k + 1] - o0;
  for (long long j = threadIdx.x; j < m; j += blockDim.x) {
    double v = 0.0;
    for (int i = 0; i < hd; ++i) {
      const size_t o = (size_t)o0 * hd + (size_t)i * m + j;
      v = v + vs[o] * ubn[(size_t)k * hd + i] - vd[o] * ub[(size_t)k * hd + i];
    }
    csr_val[o0 + j] = v;
  }
}
/* u[t] += csr_val of every panel whose ball holds t, in panel order (the
 * reference's serial scatter), one thread per source node, no atomics */
#define GRF_PT 512 /* panels per shared-memory tile */
__global__ void __launch_bounds__(256) k_grf_scatter(int npan, long long nsrc, const double* sx, const double* ball,
                                                     const long long* offs, const long long* csr_idx,
                                                     const double* csr_val, double* u) {
  __shared__ double sb[GRF_PT * 4];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double x[3] = {0.0, 0.0, 0.0};
  if (t < nsrc) { x[0] = sx[3 * t]; x[1] = sx[3 * t + 1]; x[2] = sx[3 * t + 2]; }
  double acc = t < nsrc ? u[t] : 0.0;
  for (int k0 = 0; k0 < npan; k0 += GRF_PT) {
    const int nk = min(GRF_PT, npan - k0);
    __syncthreads();
    for (int e = threadIdx.x; e < 4 * nk; e += blockDim.x) sb[e] = ball[4 * (size_t)k0 + e];
    __syncthreads();
    if (t < nsrc)
      for (int kk = 0; kk < nk; ++kk) {
        if (!in_ball(x, sb + 4 * kk)) continue;
        /* position of t+1 in the panel's sorted list */
        long long lo = offs[k0 + kk], hi = offs[k0 + kk + 1] - 1;
        while (lo < hi) {
          const long long mid = (lo + hi) >> 1;
          if (csr_idx[mid] < t + 1) lo = mid + 1; else hi = mid;
        }
        if (lo < offs[k0 + kk + 1] && csr_idx[lo] == t + 1) acc += csr_val[lo];
      }
  }
  if (t < nsrc) u[t] = acc;
}
/* u_i = sum_j S_ij ubn_j - D_ij ub_j over all sources, zero self term, in
 * source order (the reference's blocked Direct far field) */
#define FAR_TILE 256
__global__ void __launch_bounds__(256) k_direct_far(long long nsrc, const double* sx, const double* snx,
                                                    const double* sw, const double* ub, const double* ubn, double* u,
                                                    long long tlo, long long thi) {
  __shared__ double sj[FAR_TILE][8]; /* x, y, z, nx, ny, nz, w/4pi ubn, w/4pi ub */
  const long long i = tlo + (long long)blockIdx.x * blockDim.x + threadIdx.x; /* targets [tlo, thi) */
  const double i4p = 1.0 / (4.0 * QOL_PI);
  double x0 = 0.0, x1 = 0.0, x2 = 0.0;
  if (i < thi) { x0 = sx[3 * i]; x1 = sx[3 * i + 1]; x2 = sx[3 * i + 2]; }
  double acc = 0.0;
  for (long long j0 = 0; j0 < nsrc; j0 += FAR_TILE) {
    const int nj = (int)min((long long)FAR_TILE, nsrc - j0);
    __syncthreads();
    for (int e = threadIdx.x; e < nj; e += blockDim.x) {
      const long long j = j0 + e;
      sj[e][0] = sx[3 * j]; sj[e][1] = sx[3 * j + 1]; sj[e][2] = sx[3 * j + 2];
      sj[e][3] = snx[3 * j]; sj[e][4] = snx[3 * j + 1]; sj[e][5] = snx[3 * j + 2];
      sj[e][6] = sw[j] * i4p * ubn[j]; sj[e][7] = sw[j] * i4p * ub[j];
    }
    __syncthreads();
    for (int e = 0; e < nj; ++e) {
      const double dx = x0 - sj[e][0], dy = x1 - sj[e][1], dz = x2 - sj[e][2];
      const double rr = dx * dx + dy * dy + dz * dz;
      if (rr > 1.0e-28) {
        const double ri = rsqrt(rr);
        acc += ri * (sj[e][6] - sj[e][7] * ri * ri * (dx * sj[e][3] + dy * sj[e][4] + dz * sj[e][5]));
      }
    }
  }
  if (i < thi) u[i] = acc;
}

cudaError_t qol_launch_grf_balls(int npan, int hd, long long nsrc, const double* sx, const double* sw, double* ball,
                                 double* box, long long* counts, int plo, int phi, cudaStream_t st) {
  k_ball_centers<<<(npan + 127) / 128, 128, 0, st>>>(npan, hd, sx, sw, ball);
  const long long nchunk = (nsrc + BALL_CH - 1) / BALL_CH;
  if (nchunk > 0) k_chunk_boxes<<<(unsigned)nchunk, BALL_CH, 0, st>>>(nsrc, sx, box);
  if (phi > plo) k_ball_count<<<phi - plo, BALL_CH, 0, st>>>(nsrc, sx, ball + 4 * (size_t)plo, box, counts);
  return cudaGetLastError();
}
cudaError_t qol_launch_grf_csr(int npan, long long nsrc, const double* sx, const double* ball, const double* box,
                               const long long* offs, long long* csr_idx, double* tcx, long long* csr_loc,
                               long long row_shift, cudaStream_t st) {
  k_ball_fill<<<npan, BALL_CH, 0, st>>>(nsrc, sx, ball, box, offs, csr_idx, tcx, csr_loc, row_shift);
  return cudaGetLastError();
}
cudaError_t qol_launch_grf_apply(int npan, int hd, long long nsrc, const double* sx, const double* ball,
                                 const long long* offs, const long long* csr_idx, const double* vs, const double* vd,
                                 const double* ub, const double* ubn, double* csr_val, double* u, cudaStream_t st) {
  k_grf_fill<<<npan, 256, 0, st>>>(hd, offs, vs, vd, ub, ubn, csr_val);
  k_grf_scatter<<<(unsigned)((nsrc + 255) / 256), 256, 0, st>>>(npan, nsrc, sx, ball, offs, csr_idx, csr_val, u);
  return cudaGetLastError();
}
cudaError_t qol_launch_direct_far(long long nsrc, const double* sx, const double* snx, const double* sw,
                                  const double* ub, const double* ubn, double* u, long long tlo, long long thi,
                                  cudaStream_t st) {
  if (thi <= tlo) return cudaSuccess;
  k_direct_far<<<(unsigned)((thi - tlo + 255) / 256), 256, 0, st>>>(nsrc, sx, snx, sw, ub, ubn, u, tlo, thi);
  return cudaGetLastError();
}
