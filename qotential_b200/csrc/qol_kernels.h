/* Device-side views passed by value to the qol_b200 kernels. */
#pragma once
#include <cuda_runtime.h>

#define RRQ_FRAME 16 /* R (9, rows e1,e2,e3 as R[i + 3*d]), c (3), alpha (1), pad */
#define QOL_MOM_THREADS 128 /* threads per RRQ pair in k_rrq_moments (lanes of its translation schedule) */

/* per-order tables (reference element, quadrature data), device pointers */
struct OrderTab {
  int korder, hd, nterms, orderff, nquad, nlevel, ng;
  double dist;
  int n[4], nsub[4];
  const double* interp[4];    /* n_l x ncw, row-major; columns hd .. ncw-1 zero (16-byte rows) */
  const unsigned* interp_hi[4], *interp_lo[4]; /* interp in FP32 as TF32 high and low parts (precision variant):
                                                  tiles of 32 rows (zero-padded), each [row quad][ncw][4] */
  int ncw;                    /* 32 ceil(hd / 32) */
  int panel_cs, panel_nt;     /* k_rrq_panel's cluster size and CTA threads (0: the default choice) */
  const double* wt[4];        /* n_l */
  const long long* suboff[4]; /* nsub_l + 1 */
  const int* subtyp[4];       /* nsub_l */
  const double *tgl, *wgl, *Dgl, *Leg; /* nquad; nquad x nquad col-major */
  const double *gl48x, *gl48w, *gl16x, *gl16w, *tq, *wq;
  const double* Mb;    /* (3 nquad + 3) x hd, row-major: boundary + vertex interpolation */
  const double* umatr; /* hd x hd col-major (vals -> coefs) */
  const double* vruv;  /* 2 x hd VR nodes of degree korder */
  const unsigned* xsched; /* xsteps x QOL_MOM_THREADS translation terms (qolh::xlate_schedule) */
  const unsigned* xred;   /* per translation output: first partial slot, slot count */
  int xslots;
  const double* tginv;    /* nquad x nquad: 1/(tgl[i] - tgl[i-k-1]) at [k*nquad + i] */
  int sum_fp32;           /* 1: level sums in FP32, 3xTF32 on tcgen05 (precision variant) */
  int xsteps;
  const double* sk[4];    /* n_l x 4: the selector check's sketch vectors on the level nodes (I_l v, v = +-1) */
  int force_level;        /* 1..nlevel: every pair the walk resolves by a direct sum takes this level (labels) */
  int adaptive;           /* 1: the adaptive tree walk over the first nlevel-1 (plain 4-split) levels */
};
/* pair class of an adaptive cut (G.level, G.cnt slot) */
#define QOL_LV_CUT 6

/* panel geometry (reference layouts: sx(3,nsrc) etc.) */
struct PanelIn {
  const double *sx, *snx, *sw, *rts, *rps;
};

/* targets in CSR-by-panel form (1-based tcxrow/tcxi as in the reference) */
struct PairIn {
  const double* tcx;
  const long long* tcxrow;
  const long long* tcxi;
};

/* refined level geometry: per level, per panel, 7 x n_l SoA (x,y,z,nx,ny,nz,w)
 * and per sub-patch (qx,qy,qz,qr2) */
struct LevelWS {
  double* node[4];
  double* sub[4];
};

/* pair classification and per-panel grouping by level */
struct PairWS {
  signed char* level; /* ntcx: 1..nlevel, nlevel+1 = RRQ */
  int* grp;           /* ntcx: local target ids grouped per panel by level */
  int* cnt;           /* npan x 8 */
  int* off;           /* npan x 8 */
};

/* RRQ workspace */
struct RRQWS {
  int npan, all_panels;
  long long nrrq;
  const long long* rrq_off; /* npan + 1 */
  double *frame, *bx, *bt, *cf, *scf, *sxf;
  double *hmat, *smat, *PD, *B; /* per panel: H, S inverse, D inverse rows, B = PS H^T */
  double *JD, *RS; /* per RRQ pair: 4hd, hd */
  double* line;    /* per RRQ pair: cD (3 nbd), cS (3 nbd), lint (3), Omega */
  double* edge;    /* per RRQ pair and edge: w1 (nq), w3 (nq), ok, Re t0, Im t0 */
  double* ialpha;  /* per RRQ pair (nullable) */
  int2* pair;      /* per RRQ pair: (panel, local target) */
  signed char* side; /* per RRQ pair: side of the panel (-1, 0, 1) + 4 when the target projects inside */
  long long glo, ghi; /* RRQ pairs [glo, ghi) of this launch (per-pair kernels) */
  int plo, phi;       /* panels [plo, phi) of this launch (k_rrq_apply) */
};

/* output: COO values (block column-major per panel) */
struct OutCOO {
  double *vs, *vd;
  double* omega; /* nullable: 4hd x m (qol_rrq single panel) */
  int subtract_naive;
};

cudaError_t qol_upload_harm_coefs(const double* hb, const double* hc, const double* hcm, cudaStream_t st);
cudaError_t qol_launch_levels(const OrderTab& T, const PanelIn& P, const LevelWS& W, int npan, cudaStream_t st);
cudaError_t qol_launch_classify(const OrderTab& T, const PairIn& Q, const LevelWS& W, const PairWS& G, int npan,
                                cudaStream_t st, int preset = 0 /* nonzero G.level entries are kept */);
/* learned level selector (qol_selector.cu): MLP F -> H -> H -> C, QOL_SEL_NW weights */
#define QOL_SEL_F 8
#define QOL_SEL_H 64
#define QOL_SEL_C 5
#define QOL_SEL_NW (QOL_SEL_F * QOL_SEL_H + QOL_SEL_H + QOL_SEL_H * QOL_SEL_H + QOL_SEL_H + QOL_SEL_H * QOL_SEL_C + QOL_SEL_C)
cudaError_t qol_launch_sel_features(int hd, const PanelIn& P, const PairIn& Q, int npan, float* feat, cudaStream_t st);
/* mode 1: a direct-level prediction is kept when the target is outside every
 * ball of that level; mode 2: it is marked a candidate (G.level = -l) for the
 * two-level check of qol_launch_sel_check */
cudaError_t qol_launch_sel_infer(const OrderTab& T, const PanelIn& P, const PairIn& Q, const LevelWS& W,
                                 const PairWS& G, int npan, const float* wbf, float conf, unsigned long long* cnt,
                                 int mode, cudaStream_t st);
/* reads (synchronising st) and clears the flag k_sel_infer sets when one of
 * its bounded waits on the tensor cores times out; *flag nonzero: it did */
cudaError_t qol_sel_wait_error(unsigned* flag, cudaStream_t st);
#define QOL_SEL_BETA 10.0 /* safety factor of the two-level check */
cudaError_t qol_launch_sel_check(const OrderTab& T, const PanelIn& P, const PairIn& Q, const LevelWS& W,
                                 const PairWS& G, int npan, double tol, unsigned long long* cnt, cudaStream_t st);
size_t qol_sel_grad_smem();
cudaError_t qol_launch_sel_grad(const float* feat, const signed char* lab, const int* idx, long long n0, long long n1,
                                const float* w, float* slot, double* sloss, int nslot, cudaStream_t st);
cudaError_t qol_launch_sel_update(const float* slot, int nslot, float inv_n, float* grad, float* w, float* m, float* v,
                                  float lr, int it, cudaStream_t st);
cudaError_t qol_launch_direct(const OrderTab& T, const PanelIn& P, const PairIn& Q, const LevelWS& W,
                              const PairWS& G, const OutCOO& O, int npan, cudaStream_t st,
                              int pan0 = 0 /* first panel of the launch */);
/* reads (synchronising st) and clears the flag the FP32 level-sum kernel
 * sets when one of its bounded waits times out; *flag nonzero: it did */
cudaError_t qol_wait_error(unsigned* flag, cudaStream_t st);
/* one pipeline job's level-sum inputs (the batched entry's persistent launch) */
struct DirectJob {
  OrderTab T;
  PanelIn P;
  PairIn Q;
  LevelWS W;
  PairWS G;
  OutCOO O;
};
/* the FP64 level sums of many jobs in one persistent launch over the (job,
 * panel, level) items (3 ints each, device memory) taken in order from a queue
 * whose head (*head, device memory) starts at 0; nbmax: the largest
 * interpolation column-block count (ncw / 32) among the jobs */
cudaError_t qol_launch_direct_queue(const DirectJob* jobs, int nbmax, const int* items, int nitems, int* head,
                                    cudaStream_t st);
/* the level sums of the adaptive cuts (pairs of class QOL_LV_CUT) */
cudaError_t qol_launch_direct_cut(const OrderTab& T, const PanelIn& P, const PairIn& Q, const LevelWS& W,
                                  const PairWS& G, const OutCOO& O, int npan, cudaStream_t st, int pan0 = 0);
cudaError_t qol_launch_scan(int npan, int lev, const int* cnt, long long* off, cudaStream_t st);
cudaError_t qol_launch_rrq_panel(const OrderTab& T, const PanelIn& P, const PairWS& G, const RRQWS& R, int npan,
                                 const double* chart, cudaStream_t st);
/* the (cluster size, CTA threads) shapes k_rrq_panel has for hdim hd (results do
 * not depend on the shape); returns how many, at most cap */
int qol_panel_shapes(int hd, int nquad, int* cs, int* nt, int cap);
cudaError_t qol_launch_rrq_pairs(const OrderTab& T, const PairIn& Q, const PairWS& G, const RRQWS& R, int npan,
                                 cudaStream_t st);
cudaError_t qol_launch_rrq_ssq(const OrderTab& T, const PairIn& Q, const PairWS& G, const RRQWS& R, cudaStream_t st);
cudaError_t qol_launch_rrq_geom(const OrderTab& T, const PairIn& Q, const PairWS& G, const RRQWS& R, int exterior,
                                cudaStream_t st);
cudaError_t qol_launch_rrq_moments(const OrderTab& T, const PairIn& Q, const PairWS& G, const RRQWS& R,
                                   cudaStream_t st);
/* ssq + geom + moments */
cudaError_t qol_launch_rrq_target(const OrderTab& T, const PairIn& Q, const PairWS& G, const RRQWS& R, int exterior,
                                  cudaStream_t st);
cudaError_t qol_launch_rrq_apply(const OrderTab& T, const PanelIn& P, const PairIn& Q, const PairWS& G,
                                 const RRQWS& R, const OutCOO& O, cudaStream_t st);
cudaError_t qol_launch_coo_index(const OrderTab& T, const PairIn& Q, long long* si, long long* sj, int npan,
                                 cudaStream_t st);
cudaError_t qol_launch_fp64_peak(double* out, int blocks, int iters, cudaStream_t st);
/* GRF near phase and Direct far field */
/* ball centres of all npan panels, node-chunk boxes (6 doubles a chunk of 256
 * nodes, ceil(nsrc / 256) chunks); near counts of panels [plo, phi) into
 * counts[0 .. phi - plo) */
cudaError_t qol_launch_grf_balls(int npan, int hd, long long nsrc, const double* sx, const double* sw, double* ball,
                                 double* box, long long* counts, int plo, int phi, cudaStream_t st);
/* CSR of npan panels (ball points at their first ball); csr_loc (nullable) gets the
 * rows minus row_shift */
cudaError_t qol_launch_grf_csr(int npan, long long nsrc, const double* sx, const double* ball, const double* box,
                               const long long* offs, long long* csr_idx, double* tcx, long long* csr_loc,
                               long long row_shift, cudaStream_t st);
cudaError_t qol_launch_grf_apply(int npan, int hd, long long nsrc, const double* sx, const double* ball,
                                 const long long* offs, const long long* csr_idx, const double* vs, const double* vd,
                                 const double* ub, const double* ubn, double* csr_val, double* u, cudaStream_t st);
/* the geometry generator: nchart charts -> 2 nchart panels (reference layout) */
cudaError_t qol_launch_surface_panels(int nchart, int nmode, const double* modes, int nfp, int p,
                                      const double* charts, double ts1, double ts2, const double* x0,
                                      const double* D, const double* wts, const double* tables, double* sx,
                                      double* snx, double* sw, double* rts, double* rps, cudaStream_t st);
/* u_i for the targets i in [tlo, thi) over all nsrc sources */
cudaError_t qol_launch_direct_far(long long nsrc, const double* sx, const double* snx, const double* sw,
                                  const double* ub, const double* ubn, double* u, long long tlo, long long thi,
                                  cudaStream_t st);
