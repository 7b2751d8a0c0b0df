/* Learned level selector (no reference counterpart): an MLP 8 -> 64 -> 64 -> 5
 * on per-pair geometry features predicts a (target, panel) pair's level:
 * classes 0..3 = direct sums on refined level 1..4, class 4 = RRQ.  Two
 * label sets and two acceptance rules (the mode):
 *   mode 1 - labels are the levels the plain ball tests of
 *     lap3dsdlpmat_levels_r64 (patch_refine_mod.f90:516-551) give; a
 *     confident direct prediction l is used only when the target lies
 *     outside every level-l sub-patch ball (the plain criterion at that
 *     level), an RRQ prediction only when the walk gives RRQ;
 *   mode 2 - labels are the lowest level whose row is within a tolerance of
 *     the finest level's, capped at the walk's level (error-judged,
 *     qotential_b200/selector.py); a confident prediction l below the walk's
 *     level is used only when the two-level check below estimates its row
 *     error within that tolerance; otherwise the walk's level is kept, and
 *     pairs the walk sends to RRQ stay RRQ (close to the panel the direct
 *     sums may converge to another value than RRQ's).
 * Pairs of low confidence, or whose check fails, keep the plain walk.
 *
 * The two-level check (k_sel_check): sketch sums s_v = sum_q K(x, y_q) w_q
 * (I_l v)_q over the level-l nodes and over the nodes of level l + 1, for the
 * single- and double-layer kernels and 4 fixed +-1 vectors v over the
 * panel's node values, so s_v is the row of that level applied to v.  The
 * difference e = max_v max(|dS_v| / D, |dD_v|) (D = sqrt(sum w), the panel's
 * diameter; single-layer rows scale with length) estimates the level-l row's
 * error; the prediction passes when QOL_SEL_BETA e <= tol.
 *
 * Features (FP32, from a per-panel descriptor computed in FP64 with fixed
 * reduction order): centroid c = sum w y / sum w, diameter D = sqrt(sum w),
 * mean normal nb, in-plane axes e1 (first node direction), e2 = nb x e1,
 * curvature k = max |n_j - nb|, aspect a = sqrt(l1 / l2) of the in-plane
 * second moments.  With d = x - c:
 *   f0 log10(|d| / D), f1 tanh(d.e1 / D), f2 tanh(d.e2 / D), f3 d.nb / |d|,
 *   f4 log10(|d.nb| / D), f5 k, f6 ln a, f7 log10(min_j |x - y_j| / D)
 * (logs of arguments clamped below at 1e-12).
 *
 * Weights: W1[f][i] (8 x 64), b1, W2[i][j] (64 x 64), b2, W3[j][k] (64 x 5),
 * b3, in that order.  Training and inference compute with BF16 operands
 * (the weights, the features and the hidden activations rounded to BF16) and
 * FP32 sums; training keeps FP32 master weights for the Adam step and takes
 * the gradient with respect to the rounded weights. */
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "qol_dev.cuh"
#include "qol_kernels.h"

namespace {

constexpr int F = QOL_SEL_F, H = QOL_SEL_H, NC = QOL_SEL_C;
constexpr int OW1 = 0, OB1 = OW1 + F * H, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H, OB3 = OW3 + H * NC;
static_assert(OB3 + NC == QOL_SEL_NW, "weight layout");

/* the BF16 rounding (nearest, ties to even) of x, as a float: the operands
 * of the MLP (weights, features, hidden activations) are BF16 values, its sums
 * FP32 */
__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

/* the panel descriptor: c(3), nb(3), e1(3), e2(3), D, kappa, ln(aspect); one
 * warp, lanes over the panel's nodes, shuffle sums in a fixed order */
__device__ void sel_panel(int hd, const double* sx, const double* snx, const double* sw, double* dsc) {
  const int lane = threadIdx.x & 31;
  auto wsum = [&](double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
  };
  auto wmax = [&](double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
  };
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0, n0 = 0, n1 = 0, n2 = 0;
  for (int j = lane; j < hd; j += 32) {
    const double w = sw[j];
    s0 += w; s1 += w * sx[3 * j]; s2 += w * sx[3 * j + 1]; s3 += w * sx[3 * j + 2];
    n0 += w * snx[3 * j]; n1 += w * snx[3 * j + 1]; n2 += w * snx[3 * j + 2];
  }
  s0 = wsum(s0); s1 = wsum(s1); s2 = wsum(s2); s3 = wsum(s3);
  n0 = wsum(n0); n1 = wsum(n1); n2 = wsum(n2);
  const double c0 = s1 / s0, c1 = s2 / s0, c2 = s3 / s0;
  const double nl = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
  n0 /= nl; n1 /= nl; n2 /= nl;
  double a0 = sx[0] - c0, a1 = sx[1] - c1, a2 = sx[2] - c2;
  const double an = a0 * n0 + a1 * n1 + a2 * n2;
  a0 -= an * n0; a1 -= an * n1; a2 -= an * n2;
  const double al = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
  a0 /= al; a1 /= al; a2 /= al;
  const double b0 = n1 * a2 - n2 * a1, b1 = n2 * a0 - n0 * a2, b2 = n0 * a1 - n1 * a0;
  double kap = 0, ixx = 0, iyy = 0, ixy = 0;
  for (int j = lane; j < hd; j += 32) {
    const double d0 = snx[3 * j] - n0, d1 = snx[3 * j + 1] - n1, d2 = snx[3 * j + 2] - n2;
    kap = fmax(kap, sqrt(d0 * d0 + d1 * d1 + d2 * d2));
    const double y0 = sx[3 * j] - c0, y1 = sx[3 * j + 1] - c1, y2 = sx[3 * j + 2] - c2;
    const double u = y0 * a0 + y1 * a1 + y2 * a2, v = y0 * b0 + y1 * b1 + y2 * b2, w = sw[j];
    ixx += w * u * u; iyy += w * v * v; ixy += w * u * v;
  }
  kap = wmax(kap); ixx = wsum(ixx); iyy = wsum(iyy); ixy = wsum(ixy);
  const double tr = 0.5 * (ixx + iyy), dt = sqrt(0.25 * (ixx - iyy) * (ixx - iyy) + ixy * ixy);
  const double l1 = tr + dt, l2 = fmax(tr - dt, 1e-300);
  if (lane == 0) {
    dsc[0] = c0; dsc[1] = c1; dsc[2] = c2; dsc[3] = n0; dsc[4] = n1; dsc[5] = n2;
    dsc[6] = a0; dsc[7] = a1; dsc[8] = a2; dsc[9] = b0; dsc[10] = b1; dsc[11] = b2;
    dsc[12] = sqrt(s0); dsc[13] = kap; dsc[14] = 0.5 * log(l1 / l2);
  }
}

__device__ __forceinline__ double lg10c(double v) { return log10(fmax(v, 1e-12)); }

/* the 8 features of target x against the panel (descriptor dsc, nodes sx) */
__device__ void sel_features(const double* x, const double* dsc, int hd, const double* sx, float* f) {
  const double D = dsc[12];
  const double d0 = x[0] - dsc[0], d1 = x[1] - dsc[1], d2 = x[2] - dsc[2];
  const double r = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  const double u = d0 * dsc[6] + d1 * dsc[7] + d2 * dsc[8], v = d0 * dsc[9] + d1 * dsc[10] + d2 * dsc[11];
  const double h = d0 * dsc[3] + d1 * dsc[4] + d2 * dsc[5];
  double m2 = 1e300;
  for (int j = 0; j < hd; ++j) {
    const double e0 = x[0] - sx[3 * j], e1 = x[1] - sx[3 * j + 1], e2 = x[2] - sx[3 * j + 2];
    m2 = fmin(m2, e0 * e0 + e1 * e1 + e2 * e2);
  }
  f[0] = (float)lg10c(r / D);
  f[1] = (float)tanh(u / D);
  f[2] = (float)tanh(v / D);
  f[3] = (float)(r > 0.0 ? h / r : 0.0);
  f[4] = (float)lg10c(fabs(h) / D);
  f[5] = (float)dsc[13];
  f[6] = (float)dsc[14];
  f[7] = (float)lg10c(sqrt(m2) / D);
}

/* per panel: descriptor into shared memory, node coordinates staged */
__device__ void sel_stage(int pan, int hd, const PanelIn& P, double* s_sx, double* dsc) {
  for (int e = threadIdx.x; e < 3 * hd; e += blockDim.x) s_sx[e] = P.sx[(size_t)pan * hd * 3 + e];
  if (threadIdx.x < 32)
    sel_panel(hd, P.sx + (size_t)pan * hd * 3, P.snx + (size_t)pan * hd * 3, P.sw + (size_t)pan * hd, dsc);
  __syncthreads();
}

/* features of every pair of the panel (dataset for training) */
__global__ void __launch_bounds__(128) k_sel_features(int hd, PanelIn P, PairIn Q, float* feat) {
  const int pan = blockIdx.x;
  extern __shared__ double ssm[];
  double* dsc = ssm;        /* 16 */
  double* s_sx = ssm + 16;  /* 3 hd */
  sel_stage(pan, hd, P, s_sx, dsc);
  const long long p0 = Q.tcxi[pan] - 1, m = Q.tcxi[pan + 1] - Q.tcxi[pan];
  for (long long t = threadIdx.x; t < m; t += blockDim.x) {
    float f[F];
    sel_features(Q.tcx + 3 * (p0 + t), dsc, hd, s_sx, f);
#pragma unroll
    for (int c = 0; c < F; ++c) feat[(size_t)(p0 + t) * F + c] = f[c];
  }
}

/* ---------------------------------------------------------------------
 * Inference on the fifth-generation tensor cores.  One CTA of SI_T = 128
 * threads per panel, tiles of 128 pairs, a pair a thread: its row of every
 * matrix and its lane of tensor memory.  The three layers are
 * tcgen05.mma kind::f16 products with BF16 operands in shared memory
 * (K-major, no swizzle: core matrices of 8 rows x 16 bytes) and FP32
 * accumulators in SI_TMEM columns of tensor memory, which every layer
 * reuses: X (128 x 16, the 8 features and zeros) times W1 (N 64), then H1
 * (128 x 64) times W2 (N 64, four K steps of 16), then H2 times W3 (N 16: the
 * 5 classes and zeros).  After each layer every thread reads its row back 8
 * columns at a time, adds the bias, takes the ReLU and rounds to BF16 into
 * the next layer's A row: BF16 features, weights and hidden activations with
 * FP32 sums, as in training (k_sel_grad).  Thread 0 issues each layer's MMAs
 * and waits for their commit (bounded, about a second); the outcome is agreed
 * at a barrier, and after a timeout the CTA sets g_sel_wait_err, leaves the
 * rest of the panel to the plain walk (level 0) and frees its tensor memory.
 * --------------------------------------------------------------------- */
#define SI_T 128   /* threads, pairs a tile, the MMAs' M */
#define SI_TMEM 64u
__device__ unsigned g_sel_wait_err; /* nonzero: a bounded wait of k_sel_infer timed out */

/* byte offset of element (r, k) of a K-major BF16 operand of `rows` rows */
__device__ __forceinline__ unsigned kmaj_off(int r, int k, int rows) {
  return (unsigned)((k >> 3) * (rows >> 3) * 128 + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
/* D[tmem] (+)= A B, BF16 operands from shared memory, FP32 accumulate; acc = 0 overwrites D */
__device__ __forceinline__ void umma_bf16(unsigned d, unsigned long long a, unsigned long long b, unsigned idesc,
                                          unsigned acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
/* instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N = n, M = 128 */
__host__ __device__ constexpr unsigned si_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(n >> 3) << 17) | (8u << 24);
}
/* 8 consecutive FP32 columns of this thread's tensor-memory lane (the wait
 * takes the registers, so nothing reads them before the load has completed) */
__device__ __forceinline__ void tmem_ld8(unsigned taddr, float* v) {
  unsigned r0, r1, r2, r3, r4, r5, r6, r7;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3), "=r"(r4), "=r"(r5), "=r"(r6), "=r"(r7)
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n"
               : "+r"(r0), "+r"(r1), "+r"(r2), "+r"(r3), "+r"(r4), "+r"(r5), "+r"(r6), "+r"(r7)
               :
               : "memory");
  v[0] = __uint_as_float(r0); v[1] = __uint_as_float(r1); v[2] = __uint_as_float(r2); v[3] = __uint_as_float(r3);
  v[4] = __uint_as_float(r4); v[5] = __uint_as_float(r5); v[6] = __uint_as_float(r6); v[7] = __uint_as_float(r7);
}
__device__ __forceinline__ unsigned pack_bf2(float lo, float hi) {
  return (unsigned)__bfloat16_as_ushort(__float2bfloat16_rn(lo)) |
         ((unsigned)__bfloat16_as_ushort(__float2bfloat16_rn(hi)) << 16);
}
/* dynamic shared memory of k_sel_infer: the descriptor and node coordinates,
 * then (1024-aligned) the A tile (128 x 64), W1 (64 x 16), W2 (64 x 64), W3
 * (16 x 64) as BF16, the biases (64 + 64 + 8 floats), the mbarrier and the
 * tensor-memory address */
__host__ __device__ constexpr size_t si_head(int hd) { return (sizeof(double) * (16 + 3 * (size_t)hd) + 1023) & ~(size_t)1023; }
__host__ __device__ constexpr size_t si_smem(int hd) { return si_head(hd) + 16384 + 2048 + 8192 + 2048 + 4 * 136 + 16; }

/* learned level decision of every pair of the panel: G.level = accepted level
 * (1..nlevel+1), a candidate -l for the two-level check (mode 2) or 0 (the
 * plain walk decides); counters [accepted, low confidence, check failed] */
__global__ void __launch_bounds__(SI_T) k_sel_infer(OrderTab T, PanelIn P, PairIn Q, LevelWS W, PairWS G,
                                                    const float* wbf, float conf, unsigned long long* cnt, int mode) {
  const int pan = blockIdx.x, hd = T.hd, tid = threadIdx.x, warp = tid >> 5;
  extern __shared__ __align__(16) double ssm[];
  double* dsc = ssm;
  double* s_sx = ssm + 16;
  unsigned char* XA = reinterpret_cast<unsigned char*>(ssm) + si_head(hd);
  unsigned char* B1 = XA + 16384;
  unsigned char* B2 = B1 + 2048;
  unsigned char* B3 = B2 + 8192;
  float* bias = reinterpret_cast<float*>(B3 + 2048); /* b1 [0, 64), b2 [64, 128), b3 [128, 136) */
  unsigned long long* mbar = reinterpret_cast<unsigned long long*>(bias + 136);
  unsigned* tslot = reinterpret_cast<unsigned*>(mbar + 1);
  __shared__ unsigned long long sc[3];
  const unsigned mb = (unsigned)__cvta_generic_to_shared(mbar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     (unsigned)__cvta_generic_to_shared(tslot)),
                 "r"(SI_TMEM)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (tid < 3) sc[tid] = 0;
  /* the weights as B operands (rows = outputs, K = inputs): W1[c][i] at (i, c),
   * W2[i][j] at (j, i), W3[j][k] at (k, j); zero rows and columns pad K to 16
   * and N to 16 */
  for (int e = tid; e < 64 * 16; e += SI_T) {
    const int i = e >> 4, c = e & 15;
    *reinterpret_cast<__nv_bfloat16*>(B1 + kmaj_off(i, c, 64)) = __float2bfloat16_rn(c < F ? wbf[OW1 + c * H + i] : 0.0f);
  }
  for (int e = tid; e < 64 * 64; e += SI_T) {
    const int j = e >> 6, i = e & 63;
    *reinterpret_cast<__nv_bfloat16*>(B2 + kmaj_off(j, i, 64)) = __float2bfloat16_rn(wbf[OW2 + i * H + j]);
  }
  for (int e = tid; e < 16 * 64; e += SI_T) {
    const int k = e >> 6, j = e & 63;
    *reinterpret_cast<__nv_bfloat16*>(B3 + kmaj_off(k, j, 16)) = __float2bfloat16_rn(k < NC ? wbf[OW3 + j * NC + k] : 0.0f);
  }
  for (int e = tid; e < 136; e += SI_T)
    bias[e] = e < 64 ? wbf[OB1 + e] : e < 128 ? wbf[OB2 + e - 64] : (e - 128 < NC ? wbf[OB3 + e - 128] : 0.0f);
  sel_stage(pan, hd, P, s_sx, dsc); /* ends with a barrier */
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const unsigned tmem = *tslot;
  const unsigned trow = tmem + ((unsigned)(32 * warp) << 16); /* this thread's lane: row tid */
  const unsigned sa = (unsigned)__cvta_generic_to_shared(XA), sb1 = sa + 16384, sb2 = sb1 + 2048, sb3 = sb2 + 8192;
  const long long p0 = Q.tcxi[pan] - 1, m = Q.tcxi[pan + 1] - Q.tcxi[pan];
  unsigned a = 0, lo = 0, ck = 0, ph = 0;
  int to = 0;
  /* the operands written (generic proxy) become visible to the tensor cores;
   * thread 0 issues, all agree on the commit's arrival */
  auto layer = [&](int which) -> bool {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    int bad = 0;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      if (which == 1) {
        umma_bf16(tmem, umma_desc(sa, 2048, 128), umma_desc(sb1, 1024, 128), si_idesc(64), 0u);
      } else {
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
          if (which == 2)
            umma_bf16(tmem, umma_desc(sa + 4096 * ks, 2048, 128), umma_desc(sb2 + 2048 * ks, 1024, 128), si_idesc(64),
                      (unsigned)ks);
          else
            umma_bf16(tmem, umma_desc(sa + 4096 * ks, 2048, 128), umma_desc(sb3 + 512 * ks, 256, 128), si_idesc(16),
                      (unsigned)ks);
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mb)
                   : "memory");
      bad = !mbar_wait_bounded(mb, ph & 1);
    }
    ++ph;
    to = __syncthreads_or(bad);
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    return !to;
  };
  /* this thread's row of the layer's sums, biased, ReLU, BF16: the next A row */
  auto hidden = [&](const float* b) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      float v[8];
      tmem_ld8(trow + 8 * q, v);
      uint4 o;
      o.x = pack_bf2(fmaxf(v[0] + b[8 * q + 0], 0.0f), fmaxf(v[1] + b[8 * q + 1], 0.0f));
      o.y = pack_bf2(fmaxf(v[2] + b[8 * q + 2], 0.0f), fmaxf(v[3] + b[8 * q + 3], 0.0f));
      o.z = pack_bf2(fmaxf(v[4] + b[8 * q + 4], 0.0f), fmaxf(v[5] + b[8 * q + 5], 0.0f));
      o.w = pack_bf2(fmaxf(v[6] + b[8 * q + 6], 0.0f), fmaxf(v[7] + b[8 * q + 7], 0.0f));
      *reinterpret_cast<uint4*>(XA + kmaj_off(tid, 8 * q, SI_T)) = o;
    }
  };
  for (long long t0 = 0; t0 < m && !to; t0 += SI_T) {
    const long long t = t0 + tid;
    const bool valid = t < m;
    if (valid) G.level[p0 + t] = 0; /* the plain walk, unless decided below */
    const double* x = Q.tcx + 3 * (p0 + (valid ? t : 0));
    float f[F];
    if (valid) sel_features(x, dsc, hd, s_sx, f);
    else
#pragma unroll
      for (int c = 0; c < F; ++c) f[c] = 0.0f;
    *reinterpret_cast<uint4*>(XA + kmaj_off(tid, 0, SI_T)) =
        make_uint4(pack_bf2(f[0], f[1]), pack_bf2(f[2], f[3]), pack_bf2(f[4], f[5]), pack_bf2(f[6], f[7]));
    *reinterpret_cast<uint4*>(XA + kmaj_off(tid, 8, SI_T)) = make_uint4(0u, 0u, 0u, 0u);
    if (!layer(1)) break;
    hidden(bias);
    if (!layer(2)) break;
    hidden(bias + 64);
    if (!layer(3)) break;
    float z[8];
    tmem_ld8(trow, z);
    if (!valid) continue;
#pragma unroll
    for (int k = 0; k < NC; ++k) z[k] += bias[128 + k];
    int best = 0;
#pragma unroll
    for (int k = 1; k < NC; ++k) best = z[k] > z[best] ? k : best;
    float den = 0.0f;
#pragma unroll
    for (int k = 0; k < NC; ++k) den += __expf(z[k] - z[best]);
    const float prob = 1.0f / den;
    /* outside every ball of level index l (the plain criterion at that level) */
    auto outside = [&](int l) {
      const double* qp = W.sub[l] + (size_t)pan * T.nsub[l] * 4;
      for (int s = 0; s < T.nsub[l]; ++s) {
        const double b0 = qp[4 * s] - x[0], b1 = qp[4 * s + 1] - x[1], b2 = qp[4 * s + 2] - x[2];
        if (b0 * b0 + b1 * b1 + b2 * b2 < qp[4 * s + 3]) return false;
      }
      return true;
    };
    /* the walk's level: RRQ (nlevel + 1) when inside a ball at every level */
    auto walk = [&]() {
      for (int l = 0; l < T.nlevel; ++l)
        if (outside(l)) return l + 1;
      return T.nlevel + 1;
    };
    int lv = 0;
    if (prob < conf) ++lo;
    else if (mode == 2) {
      /* a level below the walk's, for the two-level check; the walk's own
       * level otherwise (RRQ pairs stay RRQ: near the panel the direct sums
       * can converge to a value other than RRQ's, which no check of their
       * convergence sees) */
      const int w = walk();
      if (w <= T.nlevel && best + 1 < w) lv = -(best + 1);
      else lv = w, ++a;
    } else if (best >= T.nlevel) { /* RRQ: when the walk gives it */
      if (walk() > T.nlevel) lv = T.nlevel + 1, ++a;
      else ++ck;
    } else if (outside(best)) lv = best + 1, ++a;
    else ++ck;
    G.level[p0 + t] = (signed char)lv;
  }
  if (to && tid == 0) {
    atomicOr(&g_sel_wait_err, 1u);
    mbar_wait_bounded(mb, (ph - 1) & 1); /* the MMAs in flight (bounded again) */
  }
  atomicAdd(&sc[0], (unsigned long long)a);
  atomicAdd(&sc[1], (unsigned long long)lo);
  atomicAdd(&sc[2], (unsigned long long)ck);
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (tid < 3) atomicAdd(&cnt[tid], sc[tid]);
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(SI_TMEM) : "memory");
  }
}

/* the two-level check of the direct-level candidates (G.level = -l, l =
 * 1..nlevel-1): accepted -> l, rejected -> 0 (the plain walk); counters
 * [accepted, -, check failed].  One CTA per (panel, candidate level);
 * candidates are gathered SC_C at a time in target order, SC_J per thread,
 * the nodes of both levels (coordinates, normal, weight, the 4 sketch values)
 * staged SC_NT at a time in shared memory and read as 16-byte pairs by every
 * thread; each thread sums its nodes in node order (deterministic). */
#ifndef QOL_SC_T
#define QOL_SC_T 128 /* check threads a CTA */
#endif
#ifndef QOL_SC_J
#define QOL_SC_J 1   /* candidates a thread */
#endif
#ifndef QOL_SC_MINB
#define QOL_SC_MINB 8 /* resident CTAs an SM (64 registers a thread) */
#endif
constexpr int SC_T = QOL_SC_T, SC_J = QOL_SC_J, SC_C = SC_T * SC_J, SC_NT = 64, SC_F = 12; /* fields a staged node, padded */

/* the sketch sums of one level's nodes for the thread's targets, added
 * (sign + 1) to or subtracted (sign - 1) from S and Dd */
__device__ __forceinline__ void sk_level(const double* node, const double* skv, int n, const double (&x)[SC_J][3],
                                         const bool (&on)[SC_J], double (&S)[SC_J][4], double (&Dd)[SC_J][4],
                                         double* nd, double w4s) {
  const int tid = threadIdx.x;
  for (int n0 = 0; n0 < n; n0 += SC_NT) {
    __syncthreads();
    for (int e = tid; e < 11 * SC_NT; e += SC_T) {
      const int f = e / SC_NT, q = e % SC_NT, i = n0 + q;
      nd[q * SC_F + f] = i < n ? (f < 7 ? node[(size_t)f * n + i] : skv[(size_t)i * 4 + f - 7]) : 0.0;
    }
    __syncthreads();
    const int nn = min(SC_NT, n - n0);
    for (int q = 0; q < nn; ++q) {
      const double2* r = reinterpret_cast<const double2*>(nd + q * SC_F);
      const double2 p01 = r[0], p2n0 = r[1], n12 = r[2], wk0 = r[3], k12 = r[4], k3 = r[5];
      const double w4 = wk0.x * w4s;
#pragma unroll
      for (int j = 0; j < SC_J; ++j) {
        if (!on[j]) continue;
        double sv, dv;
        sdl_kernel(x[j][0] - p01.x, x[j][1] - p01.y, x[j][2] - p2n0.x, p2n0.y, n12.x, n12.y, w4, sv, dv);
        S[j][0] = fma(sv, wk0.y, S[j][0]); Dd[j][0] = fma(dv, wk0.y, Dd[j][0]);
        S[j][1] = fma(sv, k12.x, S[j][1]); Dd[j][1] = fma(dv, k12.x, Dd[j][1]);
        S[j][2] = fma(sv, k12.y, S[j][2]); Dd[j][2] = fma(dv, k12.y, Dd[j][2]);
        S[j][3] = fma(sv, k3.x, S[j][3]);  Dd[j][3] = fma(dv, k3.x, Dd[j][3]);
      }
    }
  }
}

__global__ void __launch_bounds__(SC_T, QOL_SC_MINB) k_sel_check(OrderTab T, PanelIn P, PairIn Q, LevelWS W, PairWS G, double tol,
                                                    unsigned long long* cnt) {
  const int pan = blockIdx.x, l = blockIdx.y + 1, hd = T.hd; /* candidate level l, checked against l + 1 */
  const long long p0 = Q.tcxi[pan] - 1, m = Q.tcxi[pan + 1] - Q.tcxi[pan];
  if (m <= 0) return;
  __shared__ __align__(16) double nd[SC_NT * SC_F];
  __shared__ int cand[2 * SC_C];
  __shared__ int ncand, wc[SC_T / 32];
  __shared__ double sdiam;
  __shared__ unsigned long long sc[2];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid < 32) {
    double sw = 0.0;
    for (int j = lane; j < hd; j += 32) sw += P.sw[(size_t)pan * hd + j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sw += __shfl_xor_sync(0xffffffffu, sw, o);
    if (lane == 0) sdiam = sqrt(sw);
  }
  if (tid < 2) sc[tid] = 0;
  if (tid == 0) ncand = 0;
  __syncthreads();
  const double Dp = sdiam, i4p = 1.0 / (4.0 * QOL_PI);
  const int la = l - 1, lb = l, na = T.n[la], nb_ = T.n[lb];
  const double* nodea = W.node[la] + (size_t)pan * na * 7;
  const double* nodeb = W.node[lb] + (size_t)pan * nb_ * 7;
  for (long long w0 = 0;; w0 += SC_T) {
    const bool more = w0 < m;
    if (more) { /* append this window's candidates in target order */
      const long long t = w0 + tid;
      const bool c = t < m && G.level[p0 + t] == -l;
      const unsigned b = __ballot_sync(0xffffffffu, c);
      if (lane == 0) wc[wid] = __popc(b);
      __syncthreads();
      int before = ncand;
      for (int w = 0; w < wid; ++w) before += wc[w];
      if (c) cand[before + __popc(b & ((1u << lane) - 1u))] = (int)t;
      __syncthreads();
      if (tid == 0) {
        int tot = 0;
        for (int w = 0; w < SC_T / 32; ++w) tot += wc[w];
        ncand += tot;
      }
      __syncthreads();
    }
    const int nc = ncand;
    if (nc >= SC_C || (!more && nc > 0)) {
      const int nb = min(nc, SC_C);
      int my[SC_J];
      double x[SC_J][3];
      bool on[SC_J];
#pragma unroll
      for (int j = 0; j < SC_J; ++j) {
        const int k = tid + j * SC_T;
        my[j] = k < nb ? cand[k] : -1;
        on[j] = my[j] >= 0;
        const double* xp = Q.tcx + 3 * (p0 + (on[j] ? my[j] : 0));
        x[j][0] = xp[0]; x[j][1] = xp[1]; x[j][2] = xp[2];
      }
      double S[SC_J][4], Dd[SC_J][4]; /* level l's sketch sums minus level l + 1's */
#pragma unroll
      for (int j = 0; j < SC_J; ++j)
#pragma unroll
        for (int v = 0; v < 4; ++v) S[j][v] = Dd[j][v] = 0.0;
      sk_level(nodea, T.sk[la], na, x, on, S, Dd, nd, i4p);
      sk_level(nodeb, T.sk[lb], nb_, x, on, S, Dd, nd, -i4p);
#pragma unroll
      for (int j = 0; j < SC_J; ++j) {
        if (!on[j]) continue;
        double e = 0.0;
#pragma unroll
        for (int v = 0; v < 4; ++v) e = fmax(e, fmax(fabs(S[j][v]) / Dp, fabs(Dd[j][v])));
        const bool ok = QOL_SEL_BETA * e <= tol;
        G.level[p0 + my[j]] = (signed char)(ok ? l : 0);
        atomicAdd(&sc[ok ? 0 : 1], 1ull);
      }
      __syncthreads(); /* every thread has read its candidates: move the rest to the front */
      const int rest = nc - nb;
      int keep[SC_J];
#pragma unroll
      for (int j = 0; j < SC_J; ++j) keep[j] = tid + j * SC_T < rest ? cand[nb + tid + j * SC_T] : 0;
      __syncthreads();
#pragma unroll
      for (int j = 0; j < SC_J; ++j)
        if (tid + j * SC_T < rest) cand[tid + j * SC_T] = keep[j];
      if (tid == 0) ncand = rest;
      __syncthreads();
    }
    if (!more && ncand == 0) break;
  }
  __syncthreads();
  if (tid == 0) {
    atomicAdd(&cnt[0], sc[0]);
    atomicAdd(&cnt[2], sc[1]);
  }
}

/* training: one CTA of 256 samples, forward and backward; its partial
 * gradient (sums over its samples, fixed order) into slot[blockIdx.x] and its
 * loss sum into sloss[blockIdx.x].  Samples idx[n0 + 256 b + t] (t < 256) below
 * n1; the rest contribute nothing. */
constexpr int GT = 256, GS = 65; /* samples per CTA, row stride of the per-sample arrays */
__global__ void __launch_bounds__(GT) k_sel_grad(const float* feat, const signed char* lab, const int* idx, long long n0,
                                                 long long n1, const float* wg, float* slot, double* sloss) {
  extern __shared__ float fsm[];
  float* w = fsm;                  /* QOL_SEL_NW */
  float* X = w + QOL_SEL_NW + 3;   /* GT x 9 */
  float* H1 = X + GT * 9;          /* GT x GS: h1, then dh1 */
  float* H2 = H1 + GT * GS;        /* GT x GS: h2, then dh2 */
  float* DZ = H2 + GT * GS;        /* GT x 6 */
  __shared__ double red[GT / 32];
  const int t = threadIdx.x;
  for (int e = t; e < QOL_SEL_NW; e += GT) w[e] = bf(wg[e]); /* BF16 operands of the FP32 master weights */
  const long long gi = n0 + (long long)blockIdx.x * GT + t;
  const bool ok = gi < n1;
  const int s = ok ? idx[gi] : 0;
  float x[F];
#pragma unroll
  for (int c = 0; c < F; ++c) x[c] = ok ? bf(feat[(size_t)s * F + c]) : 0.0f;
#pragma unroll
  for (int c = 0; c < F; ++c) X[t * 9 + c] = x[c];
  __syncthreads();
  /* forward */
  for (int i = 0; i < H; ++i) {
    float a = w[OB1 + i];
#pragma unroll
    for (int c = 0; c < F; ++c) a = fmaf(w[OW1 + c * H + i], x[c], a);
    H1[t * GS + i] = bf(fmaxf(a, 0.0f));
  }
  float z[NC];
#pragma unroll
  for (int k = 0; k < NC; ++k) z[k] = w[OB3 + k];
  for (int j = 0; j < H; ++j) {
    float a = w[OB2 + j];
    for (int i = 0; i < H; ++i) a = fmaf(w[OW2 + i * H + j], H1[t * GS + i], a);
    a = bf(fmaxf(a, 0.0f));
    H2[t * GS + j] = a;
#pragma unroll
    for (int k = 0; k < NC; ++k) z[k] = fmaf(w[OW3 + j * NC + k], a, z[k]);
  }
  float zm = z[0];
#pragma unroll
  for (int k = 1; k < NC; ++k) zm = fmaxf(zm, z[k]);
  float den = 0.0f;
#pragma unroll
  for (int k = 0; k < NC; ++k) den += expf(z[k] - zm);
  const int y = ok ? (int)lab[s] : 0;
  double loss = ok ? (double)(logf(den) + zm - z[y]) : 0.0;
#pragma unroll
  for (int k = 0; k < NC; ++k) DZ[t * 6 + k] = ok ? expf(z[k] - zm) / den - (k == y ? 1.0f : 0.0f) : 0.0f;
  __syncthreads();
  float* g = slot + (size_t)blockIdx.x * QOL_SEL_NW;
  /* dW3, db3 */
  for (int e = t; e < H * NC + NC; e += GT) {
    float acc = 0.0f;
    if (e < H * NC) {
      const int j = e / NC, k = e % NC;
      for (int u = 0; u < GT; ++u) acc = fmaf(H2[u * GS + j], DZ[u * 6 + k], acc);
      g[OW3 + e] = acc;
    } else {
      const int k = e - H * NC;
      for (int u = 0; u < GT; ++u) acc += DZ[u * 6 + k];
      g[OB3 + k] = acc;
    }
  }
  __syncthreads();
  /* dh2 = relu'(h2) W3 dz, in place */
  for (int j = 0; j < H; ++j) {
    float a = 0.0f;
#pragma unroll
    for (int k = 0; k < NC; ++k) a = fmaf(w[OW3 + j * NC + k], DZ[t * 6 + k], a);
    H2[t * GS + j] = H2[t * GS + j] > 0.0f ? a : 0.0f;
  }
  __syncthreads();
  /* dW2[i][j] = sum_u h1[u][i] dh2[u][j]; db2 */
  for (int e = t; e < H * H; e += GT) {
    const int i = e / H, j = e % H;
    float acc = 0.0f;
    for (int u = 0; u < GT; ++u) acc = fmaf(H1[u * GS + i], H2[u * GS + j], acc);
    g[OW2 + e] = acc;
  }
  if (t < H) {
    float acc = 0.0f;
    for (int u = 0; u < GT; ++u) acc += H2[u * GS + t];
    g[OB2 + t] = acc;
  }
  __syncthreads();
  /* dh1 = relu'(h1) W2 dh2, in place */
  for (int i = 0; i < H; ++i) {
    float a = 0.0f;
    for (int j = 0; j < H; ++j) a = fmaf(w[OW2 + i * H + j], H2[t * GS + j], a);
    H1[t * GS + i] = H1[t * GS + i] > 0.0f ? a : 0.0f;
  }
  __syncthreads();
  /* dW1[c][i] = sum_u x[u][c] dh1[u][i]; db1 */
  for (int e = t; e < F * H; e += GT) {
    const int c = e / H, i = e % H;
    float acc = 0.0f;
    for (int u = 0; u < GT; ++u) acc = fmaf(X[u * 9 + c], H1[u * GS + i], acc);
    g[OW1 + e] = acc;
  }
  if (t < H) {
    float acc = 0.0f;
    for (int u = 0; u < GT; ++u) acc += H1[u * GS + t];
    g[OB1 + t] = acc;
  }
  /* loss: warp sums, then the CTA's in warp order */
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
  if ((t & 31) == 0) red[t >> 5] = loss;
  __syncthreads();
  if (t == 0) {
    double sacc = 0.0;
    for (int q = 0; q < GT / 32; ++q) sacc += red[q];
    sloss[blockIdx.x] = sacc;
  }
}

/* the batch gradient (slot sums in CTA order, / nvalid) into grad, and, with
 * lr > 0, one Adam step on w (moments m, v; step number it >= 1) */
__global__ void __launch_bounds__(256) k_sel_update(const float* slot, int nslot, float inv_n, float* grad, float* w,
                                                    float* m, float* v, float lr, int it) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= QOL_SEL_NW) return;
  float gsum = 0.0f;
  for (int b = 0; b < nslot; ++b) gsum += slot[(size_t)b * QOL_SEL_NW + p];
  const float gr = gsum * inv_n;
  if (grad) grad[p] = gr;
  if (lr > 0.0f) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float mm = b1 * m[p] + (1.0f - b1) * gr, vv = b2 * v[p] + (1.0f - b2) * gr * gr;
    m[p] = mm; v[p] = vv;
    const float mh = mm / (1.0f - powf(b1, (float)it)), vh = vv / (1.0f - powf(b2, (float)it));
    w[p] -= lr * mh / (sqrtf(vh) + eps);
  }
}

} // namespace

cudaError_t qol_launch_sel_features(int hd, const PanelIn& P, const PairIn& Q, int npan, float* feat,
                                    cudaStream_t st) {
  if (npan <= 0) return cudaSuccess;
  k_sel_features<<<npan, 128, sizeof(double) * (16 + 3 * hd), st>>>(hd, P, Q, feat);
  return cudaGetLastError();
}

cudaError_t qol_launch_sel_infer(const OrderTab& T, const PanelIn& P, const PairIn& Q, const LevelWS& W,
                                 const PairWS& G, int npan, const float* wbf, float conf, unsigned long long* cnt,
                                 int mode, cudaStream_t st) {
  if (npan <= 0) return cudaSuccess;
  const size_t smem = si_smem(T.hd);
  cudaError_t e = cudaFuncSetAttribute(k_sel_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_sel_infer<<<npan, SI_T, smem, st>>>(T, P, Q, W, G, wbf, conf, cnt, mode);
  return cudaGetLastError();
}
cudaError_t qol_sel_wait_error(unsigned* flag, cudaStream_t st) {
  cudaError_t e = cudaMemcpyFromSymbolAsync(flag, g_sel_wait_err, sizeof(unsigned), 0, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && *flag) {
    const unsigned z = 0;
    e = cudaMemcpyToSymbolAsync(g_sel_wait_err, &z, sizeof z, 0, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  return e;
}

cudaError_t qol_launch_sel_check(const OrderTab& T, const PanelIn& P, const PairIn& Q, const LevelWS& W,
                                 const PairWS& G, int npan, double tol, unsigned long long* cnt, cudaStream_t st) {
  if (npan <= 0) return cudaSuccess;
  if (T.nlevel < 2) return cudaSuccess;
  k_sel_check<<<dim3(npan, T.nlevel - 1), SC_T, 0, st>>>(T, P, Q, W, G, tol, cnt);
  return cudaGetLastError();
}

size_t qol_sel_grad_smem() { return sizeof(float) * (QOL_SEL_NW + 3 + GT * 9 + 2 * GT * GS + GT * 6); }

cudaError_t qol_launch_sel_grad(const float* feat, const signed char* lab, const int* idx, long long n0, long long n1,
                                const float* w, float* slot, double* sloss, int nslot, cudaStream_t st) {
  const size_t smem = qol_sel_grad_smem();
  cudaError_t e = cudaFuncSetAttribute(k_sel_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_sel_grad<<<nslot, GT, smem, st>>>(feat, lab, idx, n0, n1, w, slot, sloss);
  return cudaGetLastError();
}

cudaError_t qol_launch_sel_update(const float* slot, int nslot, float inv_n, float* grad, float* w, float* m, float* v,
                                  float lr, int it, cudaStream_t st) {
  k_sel_update<<<(QOL_SEL_NW + 255) / 256, 256, 0, st>>>(slot, nslot, inv_n, grad, w, m, v, lr, it);
  return cudaGetLastError();
}
