/* qol_b200: B200-native (sm_100a) RRQ near-field hot path behind the
 * reference's qol_* operator API (haiszhu/qotential).
 *
 * Conventions (identical to the reference's Fortran interface):
 *  - integers are 64-bit (the reference is built with -fdefault-integer-8,
 *    Makefile:79-85); logicals are passed as integers (0/1);
 *  - arrays are column-major: sx(3,n) is x,y,z of node 1, then node 2, ...;
 *    As(m,n) is As[i + m*j];
 *  - indices in tcxrow, tcxi, sparsei, sparsej, idxs are 1-based;
 *  - the caller allocates every output.
 * Every entry point returns a status (0 = ok) and also writes the reference's
 * ier argument where the reference has one.  Status codes:
 *   0 QOL_OK, 1 QOL_ERR_NOSLOT / layout, 2 QOL_ERR_HANDLE / nnz too small,
 *   3 QOL_ERR_NPOLS, 5 QOL_ERR_CUDA, 6 QOL_ERR_ORDER (unsupported order: the
 *   getnearquad / GRF / rrq entries take nterms 2..15; at nterms 16, hdim 136,
 *   no thread-block cluster of the per-panel RRQ precompute fits in shared
 *   memory and the call is refused before any work),
 *   7 QOL_ERR_TABLES (precomputed tables differ from the library's),
 *   8 QOL_ERR_ARG (null pointer / negative size).
 * The library never falls back to a CPU path: without a usable GPU every
 * compute entry point returns QOL_ERR_CUDA.
 */
#ifndef QOL_B200_H
#define QOL_B200_H
#ifdef __cplusplus
extern "C" {
#endif

typedef long long qol_int;

enum {
  QOL_OK = 0,
  QOL_ERR_NOSLOT = 1,
  QOL_ERR_LAYOUT = 1,
  QOL_ERR_HANDLE = 2,
  QOL_ERR_NNZ = 2,
  QOL_ERR_NPOLS = 3,
  QOL_ERR_CUDA = 5,
  QOL_ERR_ORDER = 6,
  QOL_ERR_TABLES = 7,
  QOL_ERR_ARG = 8,
  QOL_ERR_LIMIT = 9
};

/* Replaces qol_simplex_precomp_mex (src/lap3d_close_mex.f90:48-59; body
 * simplex_precomp_r64, src/lap3d_close_mod.f90:115-133): Gauss-Legendre nodes,
 * weights and differentiation matrix on [-1,1] (nquad), barycentric weights,
 * Legendre values->coefficients matrix, and the simplex interpolation
 * matrices umatr (values->coefficients) / vmatr at the Vioreanu-Rokhlin
 * nodes of degree korder (kpols = (korder+1)(korder+2)/2).  Host only. */
int qol_simplex_precomp(qol_int nquad, qol_int korder, qol_int kpols, double* tgl, double* wgl,
                        double* Dgl, double* w_bclag, double* Legmat, double* umatr, double* vmatr);

/* Replaces qol_build_patch_levels_mex (src/patch_refine_mex.f90:198-208;
 * body build_patch_levels_r64, src/patch_refine_mod.f90:423-502): builds the
 * refined levels of one panel on the GPU and returns a handle in *lv
 * (generation*QOL_MAX_HANDLES + slot, as the reference encodes it). */
int qol_build_patch_levels(qol_int korder, qol_int npols, const double* sx, const double* rts,
                           const double* rps, qol_int order, double dist, qol_int nlevel,
                           qol_int* lv, qol_int* ier);

/* Replaces qol_lap3dsdlpmat_levels_mex (src/patch_refine_mex.f90:211-223;
 * body lap3dsdlpmat_levels_r64, src/patch_refine_mod.f90:516-615): As, Ad
 * (m x npols) for the targets resolved by a refined level, the 1-based list
 * idxs(1:ms) of unresolved targets.  isimd is accepted and ignored.
 * ier: 2 bad handle, 3 npols mismatch. */
int qol_lap3dsdlpmat_levels(qol_int m, const double* tx, qol_int npols, qol_int lv, qol_int isimd,
                            double* As, double* Ad, qol_int* idxs, qol_int* ms, qol_int* ier);

/* Replaces qol_clear_patch_levels_mex / qol_clear_patch_levels_all_mex
 * (src/patch_refine_mex.f90:226-242). */
int qol_clear_patch_levels(qol_int lv, qol_int* ier);
int qol_clear_patch_levels_all(qol_int* ier);

/* Replaces qol_rrq_mex (src/lap3d_close_mex.f90:18-45; body rrq_r64,
 * src/lap3d_close_mod.f90:622-881): exact-limit S and D close-panel
 * matrices As, Ad (m x n) of one panel for m targets, Omega (4 hdim x m),
 * IalphaAsvestas (m), timeinfo(20) accumulated (slots 1..8 as the
 * reference's phases, GPU milliseconds converted to seconds).  The
 * precomputed tables (tgl ... vmatr) must be the ones qol_simplex_precomp
 * returns (checked; QOL_ERR_TABLES otherwise). */
int qol_rrq(qol_int m, const double* tx, qol_int n, const double* sx, const double* snx,
            const double* sw, const double* rts, const double* rps, qol_int order, qol_int nquad,
            qol_int orderff, double distff, qol_int exterior, qol_int isimd, qol_int ichart,
            const double* sxbd_chart, const double* rv_chart, const double* tgl, const double* wgl,
            const double* Dgl, const double* w_bclag, const double* Legmat, const double* umatr,
            const double* vmatr, double* As, double* Ad, double* Omega, double* IalphaAsvestas,
            double* timeinfo);

/* Replaces qol_getnearquad_lap_rrq_mex (src/lap3d_close_mex.f90:62-81; body
 * getnearquad_lap_rrq_r64, src/lap3d_close_mod.f90:884-960): the sparse
 * near correction (RRQ minus the self-masked naive block) for all panels, as
 * COO triplets in the reference's order
 *   out = (tcxi(k)-1)*hdim + (j-1)*m_k + i.
 * Host pointers; the host<->device copies are part of the call.
 * Validation as qotential.mw:74-87 (status 1 layout, 2 nnz too small). */
int qol_getnearquad_lap_rrq(qol_int npan, qol_int nterms, qol_int hdim, qol_int nquad, qol_int nsrc,
                            const double* sx, const double* snx, const double* sw, const double* rts,
                            const double* rps, qol_int ntcx, const double* tcx, const qol_int* tcxrow,
                            const qol_int* tcxi, qol_int orderff, double distff, qol_int iside,
                            qol_int isimd, qol_int nnz, qol_int* sparsei, qol_int* sparsej,
                            double* sparsevs, double* sparsevd, double* timeinfo);

/* Device-pointer form of qol_getnearquad_lap_rrq for callers whose data is
 * already resident in GPU memory (no counterpart in the reference, which has
 * no device memory): same arguments, all arrays device pointers, work queued
 * on `stream` (a cudaStream_t, or 0 for the default stream); returns after
 * queuing unless sync != 0.  level_hist (host, 6 entries, nullable) receives
 * the pair count per refinement level (index 1..4) and RRQ (index 5). */
int qol_getnearquad_lap_rrq_dev(qol_int npan, qol_int nterms, qol_int hdim, qol_int nquad, qol_int nsrc,
                                const double* sx, const double* snx, const double* sw, const double* rts,
                                const double* rps, qol_int ntcx, const double* tcx, const qol_int* tcxrow,
                                const qol_int* tcxi, qol_int orderff, double distff, qol_int iside,
                                qol_int nnz, qol_int* sparsei, qol_int* sparsej, double* sparsevs,
                                double* sparsevd, void* stream, int sync, qol_int* level_hist);

/* Batched device form (no counterpart in the reference, which computes one
 * surface a call; its GRF driver loops over panels, stellarator_grf_core_mod.
 * f90:760-888): njob getnearquad problems, each with the arguments of
 * qol_getnearquad_lap_rrq_dev (device pointers), of any orders, in one call.
 * Every job's refined levels and pair classes are computed first; then the
 * FP64 level sums of all jobs run in ONE persistent kernel that takes (job,
 * panel, level) items from a device work queue ordered by level (finest, the
 * longest items, first); then every job's RRQ phases and COO indices.  The
 * outputs are each job's own qol_getnearquad_lap_rrq_dev outputs byte for
 * byte.  With the FP32 level sums (qol_set_sum_precision(1)) the level sums
 * run per job instead.  level_hist: 6 entries a job (nullable).  Returns
 * after the work on `stream` is done. */
/* Frees the device workspace the library keeps between calls (it grows to
 * the largest call's needs and is reused; the batched entry keeps one per
 * job); the next call allocates again.  No counterpart in the reference. */
int qol_release_workspace(void);
/* CUDA graphs of qol_getnearquad_lap_rrq_dev (no counterpart in the reference):
 * on a created stream (not the legacy default one), with the FP64 level sums
 * and the per-phase timing off, the launches after the host's read of the RRQ
 * count (level sums, RRQ phases, COO indices) are captured as a CUDA graph that
 * the stream keeps and replays while every launch argument is unchanged (the
 * same tables, workspace, buffers and sizes, as in a solver's repeated calls);
 * any other call recaptures it.  Counts since load of the graphs captured and
 * replayed (diagnostics). */
int qol_graph_stats(qol_int* captures, qol_int* replays);
/* 1 (default): the device entry captures and replays the graphs above; 0:
 * it launches directly (a kept graph is freed with qol_release_workspace) */
int qol_set_graphs(int enable);
typedef struct {
  qol_int npan, nterms, hdim, nquad, nsrc;
  const double *sx, *snx, *sw, *rts, *rps;
  qol_int ntcx;
  const double* tcx;
  const qol_int *tcxrow, *tcxi;
  qol_int orderff;
  double distff;
  qol_int iside, nnz;
  qol_int *sparsei, *sparsej;
  double *sparsevs, *sparsevd;
} qol_near_job;
int qol_getnearquad_lap_rrq_batch_dev(qol_int njob, const qol_near_job* jobs, void* stream, qol_int* level_hist);

/* No counterpart in the reference.  The work of qol_rrq for one panel (As, Ad;
 * no Omega/IalphaAsvestas/timeinfo) for callers that cannot allocate GPU
 * memory: codes inside a host application that owns all GPU memory through its
 * own pool (a cudaMalloc there fails under the pool's cap or fragments it) and
 * codes on a latency-critical path where cudaMalloc's implicit device-wide
 * synchronisation is not allowed.  Allocates no GPU memory: all workspace and
 * the per-order tables live in one static device array of 16 MiB, held by
 * every GPU that loads the library until exit.  Every array argument must be
 * device (or managed) memory of the current device (checked: QOL_ERR_ARG
 * otherwise); work is queued on `stream` (0 = the legacy default stream), and
 * every call waits once on the host for `stream` (it reads the number of RRQ
 * targets back before sizing the per-target launches).
 *  - The first call on a device sets up (takes the array's device address with
 *    cudaGetSymbolAddress, uploads constants).  A call with a new (order,
 *    orderff, nquad) re-uploads the tables into the array.
 *  - Calls share the array: calls that overlap on the GPU (other streams, other
 *    host threads' work still running) race.  Serialize them.
 *  - Limit: the order's tables, the refined levels of the panel and the panel's
 *    matrices (7 hdim^2 doubles), plus per target 8 (5 hdim + 24 nquad + 13)
 *    + 22 bytes, must fit in 16 MiB: at order 13 (hdim 91), nquad = orderff
 *    = 15, that is 6,646 bytes a target and at most 1,649 targets a call
 *    (5,324 at order 7); larger requests return QOL_ERR_LIMIT (9) with the
 *    bytes needed in qol_noalloc_last_error(). */
int qol_rrq_noalloc(qol_int m, const double* tx, qol_int n, const double* sx, const double* snx,
                    const double* sw, const double* rts, const double* rps, qol_int order, qol_int nquad,
                    qol_int orderff, double distff, qol_int exterior, double* As, double* Ad, void* stream);
const char* qol_noalloc_last_error(void);

/* GRF near phase of the reference's stellarator driver
 * (web/stellarator/fortran/stellarator_grf_core_mod.f90:652-899): for the
 * surface's own nodes as targets, the ball lists (1.75 sqrt(panel area) about
 * the panel's node mean, :652-693), the RRQ corrections minus the naive block
 * of every near pair, contracted per pair with the density (ubn, ub) (:860-875)
 * and added into u (nsrc, inout) in panel order (:892-896).  xbuf (nullable):
 * per panel the 3 x (3 nquad + 3) chart boundary (ichart = 1).  nnear: near
 * pairs; level_hist (nullable, 6): pairs per resolving level (5 = RRQ).
 * No qol_* counterpart in the reference (its GRF driver calls rrq_r64 itself). */
int qol_grf_near(qol_int npan, qol_int nterms, qol_int nquad, qol_int orderff, double distff, qol_int iside,
                 qol_int nsrc, const double* sx, const double* snx, const double* sw, const double* rts,
                 const double* rps, const double* xbuf, const double* ub, const double* ubn, double* u,
                 qol_int* nnear, qol_int* level_hist, double* timeinfo);
/* Direct far field of the same driver (stellarator_grf_core_mod.f90:566-606):
 * u_i = sum_j S_ij ubn_j - D_ij ub_j over all nodes, zero self term. */
int qol_direct_farfield(qol_int nsrc, const double* sx, const double* snx, const double* sw, const double* ub,
                        const double* ubn, double* u);
/* Panel and target ranges of the two GRF phases, for work split over GPUs
 * (no counterpart in the reference, which runs the driver on one host):
 * qol_grf_near_range adds into u the near corrections of panels [plo, phi)
 * only (their ball lists, RRQ/level corrections and scatter; all nodes stay
 * targets), so the ranges of a partition of [0, npan) sum to qol_grf_near's
 * corrections; qol_direct_farfield_range writes u_i for the targets
 * i in [tlo, thi) only.  xbuf, when given, holds every panel's chart. */
int qol_grf_near_range(qol_int npan, qol_int nterms, qol_int nquad, qol_int orderff, double distff, qol_int iside,
                       qol_int nsrc, const double* sx, const double* snx, const double* sw, const double* rts,
                       const double* rps, const double* xbuf, const double* ub, const double* ubn, qol_int plo,
                       qol_int phi, double* u, qol_int* nnear, qol_int* level_hist, double* timeinfo);
/* qol_grf_near for nrhs densities at once (no counterpart in the reference,
 * whose driver takes one density a run): ub, ubn and u are nsrc x nrhs,
 * column-major; the near search and the corrections are computed once and
 * applied to every density (u(:, r) += the near phase of density r). */
int qol_grf_near_multi(qol_int npan, qol_int nterms, qol_int nquad, qol_int orderff, double distff, qol_int iside,
                       qol_int nsrc, const double* sx, const double* snx, const double* sw, const double* rts,
                       const double* rps, const double* xbuf, qol_int nrhs, const double* ub, const double* ubn,
                       double* u, qol_int* nnear, qol_int* level_hist, double* timeinfo);
int qol_direct_farfield_range(qol_int nsrc, const double* sx, const double* snx, const double* sw,
                              const double* ub, const double* ubn, qol_int tlo, qol_int thi, double* u);

/* The reference's geometry generator on the GPU (utils/stellarator_geo_mex.c:
 * stellarator_geo_ntri / stellarator_geo, geo_core :636-750; build_charts
 * :125-160): a Fourier surface in the VMEC convention of surf_eval (:91-102),
 * R = sum rc cos(m p - nfp n t), Z = sum zs sin(m p - nfp n t), modes
 * (m, n, rc, zs) x nmode, cut into mp x np charts of the (t, p) torus (split at
 * aspect 1.65 when split != 0), each chart sampled on the nterms x nterms
 * Gauss grid and cut into two triangles whose Vioreanu-Rokhlin nodes of degree
 * nterms-1 are interpolated from it.  Outputs in the reference layout
 * (sx(3, nsrc), snx, sw, rts, rps; nsrc = ntri * nterms (nterms+1)/2), host
 * arrays.  With sx == NULL only *ntri is set (the size query); otherwise *ntri
 * must be at least the panel count (QOL_ERR_NNZ) and receives it. */
int qol_surface_panels(qol_int nmode, const double* modes, qol_int nfp, qol_int mp, qol_int np, qol_int nterms,
                       qol_int split, qol_int* ntri, double* sx, double* snx, double* sw, double* rts,
                       double* rps);
/* The adaptive chart list (stellarator_charts over build_charts_adaptive,
 * :427-546, 775-808): the mp x np charts split at aspect 1.65 (repeated
 * passes), then for restol > 0 quartered while the Legendre tail (the last two
 * degrees) of the chart's mean curvature on its p x p Gauss grid carries more
 * than restol of the spectrum, and quartered for 2:1 balance across faces.
 * charts: 6 doubles a chart (a1, b1, a2, b2, jj, ii: t1 -> a1 t1 + b1 in panel
 * jj, t2 -> a2 t2 + b2 in panel ii); with charts == NULL only *nchart (the
 * count); QOL_ERR_NNZ past cap charts or when *nchart is too small.
 * qol_surface_panels_charts: the GPU geometry generator over such a list
 * (stellarator_geo_charts :837-856), outputs and size query as
 * qol_surface_panels. */
int qol_surface_charts(qol_int nmode, const double* modes, qol_int nfp, qol_int mp, qol_int np, qol_int p,
                       double restol, qol_int cap, qol_int* nchart, double* charts);
int qol_surface_panels_charts(qol_int nmode, const double* modes, qol_int nfp, qol_int mp, qol_int np,
                              qol_int nterms, qol_int nchart, const double* charts, qol_int* ntri, double* sx,
                              double* snx, double* sw, double* rts, double* rps);
/* Host helper: the matrix M (n x npols, column-major) interpolating values at
 * the Vioreanu-Rokhlin nodes of degree korder to the points uv (2 x n) of the
 * reference triangle (koorn_pols_batch_r64 times umatr, as
 * stellarator_grf_core_mod.f90:1009-1015 builds its render interpolation). */
int qol_interp_matrix(qol_int korder, qol_int n, const double* uv, double* M);

/* Library status and diagnostics.  qol_kernel_times: when enabled, every
 * pipeline call records CUDA events on its stream around its phases and
 * accumulates the device milliseconds of its QOL_NPHASE phases: [0] refined
 * levels, [1] classification (with the host read of the RRQ pair count),
 * [2] level sums, [3] per-panel RRQ precompute, [4] singularity-swap roots and
 * weights, [5] string direction, solid angle and boundary weights, [6]
 * harmonic moments, [7] RRQ solves + COO values, [8] COO indices, [9] the
 * learned selector's inference and two-level check.  Returns the
 * sums (ms[QOL_NPHASE]) and the call count; enable >= 0 resets them and sets
 * the switch (-1: read only).  (No counterpart in the reference; its timeinfo
 * is the host-side analogue.) */
#define QOL_NPHASE 10
/* Precision of the level-resolved kernel sums for the calls that follow
 * (library-wide): 0 = FP64 (default; the drop-in), 1 = the precision variant:
 * kernel values in FP32, contraction with the interpolation rows on the
 * tcgen05 tensor cores (kind::tf32) with a 3xTF32 split, FP32 accumulation
 * over 32-node tiles and compensated FP32 sums across them, FP64 from the
 * chunk's end on; the naive block, the RRQ moments, solves and quaternion
 * fits stay FP64.  qol_rrq_noalloc always uses FP64.  No counterpart in the
 * reference (all FP64). */
int qol_set_sum_precision(int mode);
/* Autotuning of the per-panel precompute kernel (no counterpart in the
 * reference): with on = 1 (default) the first call of an order with at least
 * 256 panels times each (cluster size, CTA threads) shape the kernel has for
 * that order on 512 panels and keeps the fastest with the order's tables
 * (every shape gives the same results); 0 keeps the built-in choice.
 * qol_panel_shape returns the shape kept for an order (0, 0 before one is). */
int qol_set_autotune(int on);
int qol_panel_shape(qol_int nterms, qol_int orderff, qol_int nquad, int* cs, int* nt);
/* Learned level selector (no counterpart in the reference; it stands in for
 * the ball-test level walk of lap3dsdlpmat_levels_r64,
 * patch_refine_mod.f90:516-551).  An MLP 8 -> 64 -> 64 -> 5 on geometry
 * features of each (target, panel) pair predicts a level (classes 0..3:
 * direct sums on level 1..4; 4: RRQ): the level the plain walk gives (mode 1)
 * or the lowest level whose row is within a tolerance of the finest level's
 * (mode 2, error-judged labels).
 * qol_selector_features: the 8 features (FP32, row-major ntcx x 8) and the
 *   plain walk's level (1..5) of every near pair of a getnearquad input;
 * qol_selector_grad: mean cross-entropy and its gradient over n samples with
 *   weights w (QOL_SELECTOR_NW floats: W1 8x64, b1, W2 64x64, b2, W3 64x5, b3),
 *   as training computes it (BF16 operands, FP32 sums);
 * qol_selector_train: Adam on the GPU, `epochs` passes over a shuffle seeded
 *   by `seed`, batches of `batch` (a multiple of 256) samples; forward and
 *   backward with BF16 operands (weights, features, activations) and FP32
 *   sums, FP32 master weights; w in: initial, out: trained; loss[e] the mean
 *   loss of epoch e;
 * qol_selector_set: mode 1 makes the calls that follow use the selector with
 *   w rounded to BF16 (FP32 accumulation): a prediction with softmax
 *   probability >= conf of a direct level l is used when the target lies
 *   outside every level-l sub-patch ball, an RRQ prediction when the walk
 *   gives RRQ (else, and below conf, the plain walk
 *   decides); mode 2: a prediction l below the walk's level is used when the
 *   two-level check passes (else the walk's level; RRQ pairs of the walk stay
 *   RRQ, so the selector only lowers levels): the row of level l and of the
 *   next finer level applied to 4 fixed +-1 vectors, for the single- and
 *   double-layer kernels, differ by at most tol / 10, single-layer values
 *   over the panel's diameter sqrt(sum w); mode 0 restores the plain
 *   walk.  The COO indices never depend on the mode;
 * qol_selector_set_tol: the mode-2 tolerance (default 1e-8);
 * qol_selector_force_level: 1..4 computes every pair that the plain walk
 *   resolves by a direct sum on that level instead (RRQ pairs unchanged; the
 *   selector is off meanwhile), for error-judged labels; 0 restores the walk;
 * qol_selector_stats: accepted, low-confidence and check-failed pairs since
 *   the last call. */
#define QOL_SELECTOR_NW 5061
int qol_selector_features(qol_int npan, qol_int nterms, qol_int nquad, const double* sx, const double* snx,
                          const double* sw, const double* rts, const double* rps, qol_int ntcx, const double* tcx,
                          const qol_int* tcxrow, const qol_int* tcxi, qol_int orderff, double distff, float* feat,
                          signed char* level);
int qol_selector_grad(qol_int n, const float* feat, const signed char* label, const float* w, float* grad,
                      double* loss);
int qol_selector_train(qol_int n, const float* feat, const signed char* label, qol_int epochs, qol_int batch,
                       double lr, unsigned long long seed, float* w, double* loss);
/* Patch refinement of the level sums for the calls that follow (library
 * wide; replaces the reference's module switches PR_SQUARE / PR_ADAPTIVE,
 * patch_refine_mod.f90:53-56, with the codes of its GRF test's iadap
 * argument, test/stellarator_grf.f90:46-47): 0 square-regrouped levels (the
 * default, PR_SQUARE), 1 the adaptive tree walk (PR_ADAPTIVE: plain 4-split
 * levels, a per-target cut of sub-patches over the first three levels, the
 * finest level's ball test for the rest; an adaptive cut counts in
 * level_hist[0]), 3 plain 4-split levels with the level walk.  Any other
 * value: QOL_ERR_ARG (the reference refuses square + adaptive).  The learned
 * selector applies to the default levels only; a patch-level handle takes
 * the mode at evaluation.  No effect on qol_rrq_noalloc (square levels). */
int qol_set_patch_refine(int iadap);
/* Diagnostics: the reference element's level `level` (0..3) under the current
 * refinement mode -- n nodes, nsub sub-patches, uv (2 x n), wt (n), suboff
 * (nsub + 1, node offsets), subtyp (nsub; 1 = a Gauss-Legendre square); with
 * uv == NULL only n and nsub (build_patch_ref_r64's REF%lev, no counterpart in
 * the reference's API). */
int qol_ref_level_table(qol_int nterms, qol_int orderff, qol_int level, qol_int* n, qol_int* nsub, double* uv,
                        double* wt, qol_int* suboff, qol_int* subtyp);
int qol_selector_set(int mode, const float* w, double conf);
int qol_selector_set_tol(double tol);
int qol_selector_force_level(int level);
int qol_selector_stats(qol_int* counts3);
/* Wall-clock milestones (ms from the start) of the last
 * qol_getnearquad_lap_rrq call: [0] inputs queued, [1] all panel chunks
 * queued, [2] all value copies queued, [3] values landed in pinned staging,
 * [4] every host task done (indices filled, values in the caller's arrays),
 * [5] return, [6] COO indices filled.  No counterpart in the reference. */
int qol_last_host_times(double* ms7);
const char* qol_last_error(void);
int qol_kernel_times(int enable, double* ms, qol_int* calls);
int qol_version(void);
/* FP64 FMA throughput of this GPU in TFLOP/s (best of 5 timed launches of
 * independent FMA chains on every SM); the roofline denominator for the FP64
 * kernels.  No counterpart in the reference. */
int qol_probe_fp64_peak(double* tflops);
/* Node and sub-patch counts of the four refined levels for one order
 * (build_patch_ref_r64, src/patch_refine_mod.f90:100-262, square regroup on).
 * Host only. */
int qol_level_sizes(qol_int nterms, qol_int orderff, qol_int* n4, qol_int* nsub4);

/* Link-compatibility aliases for the reference's Fortran symbols (one
 * trailing underscore, all arguments by reference, matlab/qotential_mex.c
 * :1096-1105).  Same semantics as the functions above; no return value. */
void qol_simplex_precomp_mex_(const qol_int* nquad, const qol_int* korder, const qol_int* kpols,
                              double* tgl, double* wgl, double* Dgl, double* w_bclag, double* Legmat,
                              double* umatr, double* vmatr);
void qol_build_patch_levels_mex_(const qol_int* korder, const qol_int* npols, const double* sx,
                                 const double* rts, const double* rps, const qol_int* order,
                                 const double* dist, const qol_int* nlevel, qol_int* lv, qol_int* ier);
void qol_lap3dsdlpmat_levels_mex_(const qol_int* m, const double* tx, const qol_int* npols,
                                  const qol_int* lv, const qol_int* isimd, double* As, double* Ad,
                                  qol_int* idxs, qol_int* ms, qol_int* ier);
void qol_clear_patch_levels_mex_(const qol_int* lv, qol_int* ier);
void qol_clear_patch_levels_all_mex_(qol_int* ier);
void qol_getnearquad_lap_rrq_mex_(const qol_int* npan, const qol_int* nterms, const qol_int* hdim,
                                  const qol_int* nquad, const qol_int* nsrc, const double* sx,
                                  const double* snx, const double* sw, const double* rts,
                                  const double* rps, const qol_int* ntcx, const double* tcx,
                                  const qol_int* tcxrow, const qol_int* tcxi, const qol_int* orderff,
                                  const double* distff, const qol_int* iside, const qol_int* isimd,
                                  const qol_int* nnz, qol_int* sparsei, qol_int* sparsej,
                                  double* sparsevs, double* sparsevd, double* timeinfo);
void qol_rrq_mex_(const qol_int* m, const double* tx, const qol_int* n, const double* sx,
                  const double* snx, const double* sw, const double* rts, const double* rps,
                  const qol_int* order, const qol_int* nquad, const qol_int* orderff,
                  const double* distff, const qol_int* exterior, const qol_int* isimd,
                  const qol_int* ichart, const double* sxbd_chart, const double* rv_chart,
                  const double* tgl, const double* wgl, const double* Dgl, const double* w_bclag,
                  const double* Legmat, const double* umatr, const double* vmatr, double* As,
                  double* Ad, double* Omega, double* IalphaAsvestas, double* timeinfo);

#define QOL_MAX_HANDLES 16

#ifdef __cplusplus
}
#endif
#endif
