/* Device math for the RRQ near-field kernels (sm_100a, FP64).
 *
 * Restates, for one (target, panel) pair, the moment computation of rrq_r64
 * (src/lap3d_close_mod.f90:772-870): singularity-swap weights on the three
 * edges, the solid angle, and the harmonic-basis line moments.  The same
 * algorithm runs in the CPU oracle; here it is arranged for a warp per pair.
 */
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#define QOL_MAXL 16       /* max nterms */
#define QOL_MAXNQ 24      /* max nquad */
#define QOL_PI 3.14159265358979323846264338327950288

/* single-layer kernels S = w/(4 pi r), D = w (x-y).n/(4 pi r^3) of one source
 * node (zero when |x-y|^2 <= 1e-28, as the reference's sdlpmat) */
__device__ __forceinline__ void sdl_kernel(double dx, double dy, double dz, double nx, double ny, double nz, double w4,
                                           double& s, double& d) {
  const double rr = dx * dx + dy * dy + dz * dz;
  s = 0.0; d = 0.0;
  if (rr > 1.0e-28) {
    const double ri = rsqrt(rr);
    s = w4 * ri;
    d = s * ri * ri * (dx * nx + dy * ny + dz * nz);
  }
}

/* ---- fifth-generation tensor core (tcgen05) helpers, shared by the kernels that use it ---- */
__device__ __forceinline__ unsigned long long gtimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_test(unsigned a, unsigned parity) {
  unsigned ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
               : "=r"(ok)
               : "r"(a), "r"(parity)
               : "memory");
  return ok != 0;
}
/* wait until the phase of the given parity of the mbarrier at shared address
 * a has completed; false after about a second without it */
__device__ inline bool mbar_wait_bounded(unsigned a, unsigned parity) {
  if (mbar_test(a, parity)) return true;
  const unsigned long long t0 = gtimer_ns();
  do {
    __nanosleep(64);
    if (mbar_test(a, parity)) return true;
  } while (gtimer_ns() - t0 < 1000000000ull);
  return false;
}
/* shared-memory matrix descriptor of tcgen05.mma: K-major, no swizzle;
 * lbo: bytes between the two core matrices along K, sbo: bytes between
 * 8-row groups; bit 46: the descriptor version of sm_100 */
__device__ __forceinline__ unsigned long long umma_desc(unsigned saddr, unsigned lbo, unsigned sbo) {
  return (unsigned long long)((saddr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

struct cd {
  double re, im;
};
__device__ __forceinline__ cd mk(double a, double b) { cd r; r.re = a; r.im = b; return r; }
__device__ __forceinline__ cd cadd(cd a, cd b) { return mk(a.re + b.re, a.im + b.im); }
__device__ __forceinline__ cd csub(cd a, cd b) { return mk(a.re - b.re, a.im - b.im); }
__device__ __forceinline__ cd cmul(cd a, cd b) { return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
__device__ __forceinline__ cd cscale(double s, cd a) { return mk(s * a.re, s * a.im); }
__device__ __forceinline__ double cabs_(cd a) { return hypot(a.re, a.im); }
__device__ __forceinline__ cd cdiv(cd a, cd b) {
  double d = b.re * b.re + b.im * b.im;
  return mk((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}
__device__ __forceinline__ cd csqrt_(cd z) {
  double r = hypot(z.re, z.im);
  if (r == 0.0) return mk(0.0, 0.0);
  double t = sqrt(0.5 * (r + fabs(z.re)));
  if (z.re >= 0.0) return mk(t, z.im / (2.0 * t));
  return mk(fabs(z.im) / (2.0 * t), z.im >= 0.0 ? t : -t);
}

__device__ __forceinline__ void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ double dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* Legendre series (n coefficients) and derivative, real t */
__device__ __forceinline__ void leg_eval_r(int n, const double* c, double t, double& f, double& fp) {
  double p0 = 1.0, p1 = t, d0 = 0.0, d1 = 1.0;
  f = c[0]; fp = 0.0;
  if (n > 1) { f += c[1] * p1; fp += c[1] * d1; }
  for (int k = 1; k + 1 < n; ++k) {
    double p2 = ((2.0 * k + 1.0) * t * p1 - (double)k * p0) / (k + 1.0);
    double d2 = d0 + (2.0 * k + 1.0) * p1;
    f += c[k + 1] * p2; fp += c[k + 1] * d2;
    p0 = p1; p1 = p2; d0 = d1; d1 = d2;
  }
}
__device__ __forceinline__ void leg_eval_c(int n, const double* c, cd t, cd& f, cd& fp) {
  cd p0 = mk(1.0, 0.0), p1 = t, d0 = mk(0.0, 0.0), d1 = mk(1.0, 0.0);
  f = mk(c[0], 0.0); fp = mk(0.0, 0.0);
  if (n > 1) { f = cadd(f, cscale(c[1], p1)); fp = cadd(fp, cscale(c[1], d1)); }
  for (int k = 1; k + 1 < n; ++k) {
    cd p2 = cscale(1.0 / (k + 1.0), csub(cscale(2.0 * k + 1.0, cmul(t, p1)), cscale((double)k, p0)));
    cd d2 = cadd(d0, cscale(2.0 * k + 1.0, p1));
    f = cadd(f, cscale(c[k + 1], p2)); fp = cadd(fp, cscale(c[k + 1], d2));
    p0 = p1; p1 = p2; d0 = d1; d1 = d2;
  }
}

/* orthogonal simplex polynomials (same basis and order as the host tables) */
__device__ inline void koorn_pols_dev(double u, double v, int korder, double* pols) {
  double s = 2.0 * u + v - 1.0, t = 1.0 - v, z = 2.0 * v - 1.0;
  double La[QOL_MAXL + 2];
  La[0] = 1.0;
  if (korder >= 1) La[1] = s;
  for (int a = 1; a < korder; ++a)
    La[a + 1] = ((2.0 * a + 1.0) * s * La[a] - a * t * t * La[a - 1]) / (a + 1.0);
  int idx = 0;
  for (int deg = 0; deg <= korder; ++deg) {
    for (int b = 0; b <= deg; ++b) {
      int a = deg - b;
      double alpha = 2.0 * a + 1.0;
      double p0 = 1.0, p1 = 0.5 * (alpha + 2.0) * z + 0.5 * alpha, pb;
      if (b == 0) pb = p0;
      else if (b == 1) pb = p1;
      else {
        for (int j = 1; j < b; ++j) {
          double jj = j + 1.0;
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

/* Bjorck-Pereyra dual Vandermonde solve, b overwritten; xinv[k*n + i] =
 * 1/(x[i] - x[i-k-1]) (a per-node-set table) */
__device__ inline void bjorck_pereyra_dual_dev(int n, const double* x, const double* xinv, double* b) {
  int N = n - 1;
  for (int k = 0; k < N; ++k)
    for (int i = N; i >= k + 1; --i) b[i] -= x[k] * b[i - 1];
  for (int k = N - 1; k >= 0; --k) {
    for (int i = k + 1; i <= N; ++i) b[i] *= xinv[k * n + i];
    for (int i = k; i <= N - 1; ++i) b[i] -= b[i + 1];
  }
}

/* the three coordinate series (3 x n Legendre coefficients) at complex t,
 * one recurrence; la[k] = (2k+1)/(k+1), lb[k] = k/(k+1) */
__device__ inline void leg_eval3_c(int n, const double* c, cd t, const double* la, const double* lb, cd* f, cd* fp) {
  cd p0 = mk(1.0, 0.0), p1 = t, d0 = mk(0.0, 0.0), d1 = mk(1.0, 0.0);
  for (int d = 0; d < 3; ++d) { f[d] = mk(c[d * n], 0.0); fp[d] = mk(0.0, 0.0); }
  if (n > 1)
    for (int d = 0; d < 3; ++d) { f[d] = cadd(f[d], cscale(c[d * n + 1], p1)); fp[d] = cadd(fp[d], cscale(c[d * n + 1], d1)); }
  for (int k = 1; k + 1 < n; ++k) {
    cd p2 = csub(cscale(la[k], cmul(t, p1)), cscale(lb[k], p0));
    cd d2 = cadd(d0, cscale(2.0 * k + 1.0, p1));
    for (int d = 0; d < 3; ++d) {
      f[d] = cadd(f[d], cscale(c[d * n + k + 1], p2));
      fp[d] = cadd(fp[d], cscale(c[d * n + k + 1], d2));
    }
    p0 = p1; p1 = p2; d0 = d1; d1 = d2;
  }
}

__device__ inline double bernstein_radius_dev(cd t0) {
  cd s = cmul(csqrt_(csub(t0, mk(1.0, 0.0))), csqrt_(cadd(t0, mk(1.0, 0.0))));
  return fmax(cabs_(cadd(t0, s)), cabs_(csub(t0, s)));
}

#define QOL_RHO_SSQ 100.0
#define QOL_RHO_REC 3.0

/* root of |gamma(t)-x|^2 for one edge; returns ok flag, t0 with Im >= 0 */
__device__ inline bool edge_root_dev(int n, const double* cf /* 3 x n */, const double* tg,
                                     const double* bx /* 3 x n node positions */, const double* x,
                                     const double* la, const double* lb, cd& t0) {
  int ib = 0;
  double best = 1e300;
  for (int i = 0; i < n; ++i) {
    double a = bx[3 * i] - x[0], b = bx[3 * i + 1] - x[1], c = bx[3 * i + 2] - x[2];
    double d2 = a * a + b * b + c * c;
    if (d2 < best) { best = d2; ib = i; }
  }
  double g[3], gp[3];
  {
    cd f3[3], fp3[3];
    leg_eval3_c(n, cf, mk(tg[ib], 0.0), la, lb, f3, fp3);
    for (int d = 0; d < 3; ++d) { g[d] = f3[d].re - x[d]; gp[d] = fp3[d].re; }
  }
  double aa = dot3(gp, gp), bb = dot3(g, gp), cc = dot3(g, g);
  double disc = fmax(aa * cc - bb * bb, 0.0);
  cd t = mk(tg[ib] - bb / aa, sqrt(disc) / aa);
  for (int it = 0; it < 40; ++it) {
    cd F = mk(0.0, 0.0), Fp = mk(0.0, 0.0);
    cd f3[3], fp3[3];
    leg_eval3_c(n, cf, t, la, lb, f3, fp3);
    for (int d = 0; d < 3; ++d) {
      cd f = f3[d];
      f.re -= x[d];
      F = cadd(F, cmul(f, f));
      Fp = cadd(Fp, cscale(2.0, cmul(f, fp3[d])));
    }
    if (Fp.re == 0.0 && Fp.im == 0.0) return false;
    cd dt = cdiv(F, Fp);
    t = csub(t, dt);
    if (cabs_(dt) < 1e-14 * fmax(1.0, cabs_(t))) {
      bool ok = isfinite(t.re) && isfinite(t.im);
      t0 = mk(t.re, fabs(t.im));
      return ok;
    }
  }
  return false;
}

/* modified singularity-swap weights on one edge (see the oracle for the
 * derivation of the recurrences) */
__device__ inline void ssq_weights_dev(int n, const double* tg, const double* wg, bool ok, cd t0,
                                       const double* gl48x, const double* gl48w, const double* tginv,
                                       const double* rk /* 1/k */, double* w1, double* w3) {
  double rho = ok ? bernstein_radius_dev(t0) : 1e300;
  double a = t0.re, b = fabs(t0.im);
  /* a real root on the edge itself (target on the boundary curve): plain
   * Gauss; a real root beyond an endpoint (target on the curve's
   * continuation) keeps the singularity swap */
  bool use = ok && rho < QOL_RHO_SSQ && (b > 0.0 || fabs(a) > 1.0);
  if (!use) {
    for (int i = 0; i < n; ++i) { w1[i] = wg[i]; w3[i] = wg[i]; }
    return;
  }
  double Q[QOL_MAXNQ], P[QOL_MAXNQ];
  if (rho < QOL_RHO_REC) {
    double s1 = sqrt((1.0 - a) * (1.0 - a) + b * b);
    double sm = sqrt((1.0 + a) * (1.0 + a) + b * b);
    double t02 = a * a + b * b;
    /* int dt/s, int dt/s^3 over [-1,1]: cancellation-free forms for a root
     * beyond an endpoint (valid down to b = 0), else the asinh forms */
    if (a > 1.0) {
      Q[0] = log((sm + 1.0 + a) / (s1 + a - 1.0));
      P[0] = 1.0 / (s1 * (s1 + a - 1.0)) - 1.0 / (sm * (sm + a + 1.0));
    } else if (a < -1.0) {
      Q[0] = log((s1 + 1.0 - a) / (sm - 1.0 - a));
      P[0] = 1.0 / (sm * (sm - a - 1.0)) - 1.0 / (s1 * (s1 - a + 1.0));
    } else {
      Q[0] = asinh((1.0 - a) / b) + asinh((1.0 + a) / b);
      P[0] = ((1.0 - a) / s1 + (1.0 + a) / sm) / (b * b);
    }
    for (int k = 1; k < n; ++k) {
      double bnd = s1 - ((k - 1) % 2 == 0 ? 1.0 : -1.0) * sm;
      double v = (2.0 * k - 1.0) * a * Q[k - 1] + bnd;
      if (k >= 2) v -= (k - 1.0) * t02 * Q[k - 2];
      Q[k] = v * rk[k];
    }
    for (int k = 1; k < n; ++k) {
      double bnd = 1.0 / s1 - ((k - 1) % 2 == 0 ? 1.0 : -1.0) / sm;
      double v = a * P[k - 1] - bnd;
      if (k >= 2) v += (k - 1.0) * Q[k - 2];
      P[k] = v;
    }
  } else {
    for (int k = 0; k < n; ++k) { Q[k] = 0.0; P[k] = 0.0; }
    for (int q = 0; q < 48; ++q) {
      double t = gl48x[q];
      double s2 = (t - a) * (t - a) + b * b, s = sqrt(s2);
      double f1 = gl48w[q] / s, f3 = f1 / s2, tk = 1.0;
      for (int k = 0; k < n; ++k) { Q[k] += tk * f1; P[k] += tk * f3; tk *= t; }
    }
  }
  bjorck_pereyra_dual_dev(n, tg, tginv, Q);
  bjorck_pereyra_dual_dev(n, tg, tginv, P);
  for (int i = 0; i < n; ++i) {
    double s = sqrt((tg[i] - a) * (tg[i] - a) + b * b);
    w1[i] = Q[i] * s;
    w3[i] = P[i] * s * s * s;
  }
}
