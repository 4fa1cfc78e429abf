/*
 * vpm_fmm.h — C ABI of the B200 FMM velocity step for the LSMPS vortex
 * particle method (drop-in for the velocity evaluation of
 * anggarapangestu/LSMPS_VPM_v2, src/FMM + src/velocity_calculation).
 *
 * Plain pointers and sizes only. Every function returns a status code
 * (VPM_OK = 0) and never lets an exception cross the ABI; the text of the last
 * failure is available from vpm_last_error(ctx). Calls on one context are
 * stream-ordered on the context's stream and are not re-entrant: use one
 * context per host thread. The caller owns every input and output buffer; no
 * pointer is retained after a call returns.
 *
 * Host-buffer entry points (vpm_fmm2d_field, vpm_velocity2d, ...) copy inputs
 * to the device, run, copy results back and synchronise. The *_device entry
 * points take device pointers, enqueue the whole evaluation on the context's
 * stream and return without synchronising; their device-side error word is
 * checked by vpm_ctx_sync().
 */
#ifndef VPM_FMM_H
#define VPM_FMM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (errno-style values). */
#define VPM_OK 0
#define VPM_EDEVICE 5      /* CUDA runtime error                                   */
#define VPM_ENOMEM 12      /* device allocation failed                             */
#define VPM_EINVAL 22      /* bad argument or degenerate input (e.g. all particles coincide) */
#define VPM_EOVERFLOW 75   /* a tree / list capacity was exceeded                  */
#define VPM_ETIMEDOUT 110  /* a bounded device-side wait gave up                   */

/* Arithmetic of the evaluation. */
#define VPM_PREC_FP64 0    /* plain form: FP64 everywhere                           */
#define VPM_PREC_MIXED 1   /* chosen form: FP32 near field, list-2 M2L in FP32 per
                              parent cell (orders 1..16), on the tensor cores as
                              3xTF32 products (orders 17..20), FP64 above       */
#define VPM_PREC_MIXED_FP64_M2L 2 /* FP32 near field, FP64 M2L (for comparisons)  */
#define VPM_PREC_MIXED_TC 3 /* as VPM_PREC_MIXED with the list-2 M2L on the tensor
                              cores (tcgen05, 3xTF32) at every order 1..20     */

/* Binomial coefficients of the translations. */
#define VPM_BINOM_REFERENCE 0 /* as the reference's binComb computes them in 32-bit
                                 int, wrapping for the largest orders
                                 (src/FMM/fmm2D.cpp:28-58); needed for 1e-10 parity */
#define VPM_BINOM_EXACT 1     /* true binomial coefficients                          */

typedef struct vpm_ctx vpm_ctx;

/*
 * Knobs of the evaluation. Defaults (vpm_fmm_params_default) are the
 * reference's 2D values: global.cpp:303 (expTree = 1.0), :311 (P_max = 10),
 * :312 (par_count_max = 75), :313 (src_count_max = 50); treeCell.cpp:5
 * (EPSILON_TOLERANCE = 1e-9); fast3DFMM.cpp:4 (support factor 2.0, support_3d) with
 * the 3D leaf cap src_count_max = 30 (global.cpp:779).
 */
typedef struct vpm_fmm_params {
    int32_t p;            /* expansion order, 1..30                                 */
    int32_t max_src;      /* leaf cap on active (source) particles: 2D tree and
                             3D TreeCell                                          */
    int32_t max_par;      /* leaf cap on all particles: 2D tree and 3D TreeCell     */
    int32_t leaf_cap_3d;  /* 3D leaf iff particle count < leaf_cap_3d               */
    double exp_tree_pct;  /* root box expansion, percent                            */
    double eps;           /* list distance tolerance                                */
    int32_t precision;    /* VPM_PREC_*                                             */
    int32_t binom;        /* VPM_BINOM_*                                            */
    int32_t max_depth;    /* deepest tree level the keys resolve (2D: 16 or 31)     */
    int32_t use_graph;    /* device entry points: 1 = capture the evaluation once as
                             a CUDA graph and replay it while the buffers, n and
                             the parameters are unchanged (no per-stage timings);
                             2 = one graph per stage, with the stage events
                             recorded between them (profiling)                    */
    double center_3d[3];  /* 3D domain centre joined into the root box
                             (Pars::xcenter/ycenter/zcenter, fast3DFMM.cpp:506-508) */
    double support_3d;    /* 3D far test: a cell is far from a target when
                             R > support_3d x its size; the reference's support
                             factor is 2.0 (fast3DFMM.cpp:4, fmm3D.cpp:3), the
                             default (0 is taken as 2.0); larger values trade
                             time for accuracy (4.0: <= 1e-4 against the direct
                             sum on the vortex rings of the tests); >= 1.0   */
} vpm_fmm_params;

/* Per-call figures (counts are exact; times are CUDA-event milliseconds). */
typedef struct vpm_fmm_stats {
    int64_t n;            /* particles                                              */
    int64_t n_cells;      /* cells in the tree (reference treeData.size())          */
    int64_t n_leaves;     /* leaves (reference leafList.size())                     */
    int32_t min_level;    /* reference TreeCell::min_level                          */
    int32_t max_level;    /* reference TreeCell::max_level                          */
    int64_t p2p_pairs;    /* (target, source) pairs over list 1, j != i             */
    int64_t m2l_pairs;    /* (cell, cell) pairs over lists 2 and 4                  */
    int64_t m2p_pairs;    /* (target, cell) pairs over list 3                       */
    int64_t list1_len;
    int64_t list3_len;
    float ms_tree;        /* bounding box, keys, sort, level splits                 */
    float ms_lists;       /* lists 1-4                                              */
    float ms_upward;      /* P2M + M2M                                              */
    float ms_m2l;
    float ms_eval;        /* M2P + L2P                                              */
    float ms_p2p;
    float ms_total;       /* device time of the whole evaluation                    */
    int32_t kernels;      /* kernel launches of this call                           */
    int32_t depth_retry;  /* 1 when the host entry point rebuilt with deeper keys   */
    float ms_keys_sort;   /* bounding box, keys, radix sort, gather (part of ms_tree) */
    float ms_levels;      /* level splits (part of ms_tree)                         */
    float ms_l2l;         /* L2L levels (not part of ms_m2l)                        */
    float pad_;
} vpm_fmm_stats;

/* Fill *p with the reference's 2D/3D defaults listed above. */
void vpm_fmm_params_default(vpm_fmm_params* p);

/* Create a context on CUDA device `device` (buffers, stream, events). */
int vpm_ctx_create(int device, vpm_ctx** out);
int vpm_ctx_destroy(vpm_ctx* ctx);
/* Run subsequent calls on `cuda_stream` (a cudaStream_t; NULL = the context's own stream, a
 * blocking stream, so it is ordered with work on the legacy default stream). */
int vpm_ctx_set_stream(vpm_ctx* ctx, void* cuda_stream);
/* Wait for the context's stream and report any device-side error word. */
int vpm_ctx_sync(vpm_ctx* ctx);
/* Message of the last failure on this context (static storage of the context). */
const char* vpm_last_error(vpm_ctx* ctx);

/*
 * 2D field of the point sources (x_j, y_j, q_j):
 *   E(x_i) = sum_j q_j (x_i - x_j) / |x_i - x_j|^2
 * approximated by the adaptive-quadtree FMM. Replaces
 *   TreeCell::initializeTree(pos, active)          src/FMM/treeCell.cpp:1043
 *   fmm2D::calcField(tree, pos, active, src)        src/FMM/fmm2D.cpp:907
 *   fmm2D::get_Field_x / get_Field_y                src/FMM/fmm2D.cpp:1146-1157
 * ex/ey are the reference's Ex/Ey (the velocity is u = Ey, v = -Ex).
 * Host buffers of n elements. stats may be NULL.
 * Host entry points (this one, vpm_fmm2d_potential, vpm_velocity2d) upload
 * positions and flags first and build the tree and lists while the strengths
 * (vorticity and core sizes) are still being copied; with page-locked host
 * buffers those copies overlap the tree build. The outputs come back in the
 * same round trip as the error word, so on a non-zero status they may have
 * been partly written.
 */
int vpm_fmm2d_field(vpm_ctx* ctx, const double* x, const double* y, const double* q,
                    const uint8_t* active, int64_t n, const vpm_fmm_params* prm,
                    double* ex, double* ey, vpm_fmm_stats* stats);

/*
 * 2D potential of the same sources by the same FMM:
 *   phi(x_i) = sum_j q_j log|x_i - x_j|
 * Replaces fmm2D::calcPotential (src/FMM/fmm2D.cpp:681-896) and
 * fmm2D::get_Potential (fmm2D.hpp:65), as called by the pressure Poisson
 * solver (src/pressure_poisson/pressure_poisson.cpp:216-219). FP64 in either
 * precision setting. Host buffers; stats may be NULL.
 */
int vpm_fmm2d_potential(vpm_ctx* ctx, const double* x, const double* y, const double* q,
                        const uint8_t* active, int64_t n, const vpm_fmm_params* prm, double* phi,
                        vpm_fmm_stats* stats);

/* Same with device pointers, asynchronous on the context's stream. */
int vpm_fmm2d_field_device(vpm_ctx* ctx, const double* x, const double* y, const double* q,
                           const uint8_t* active, int64_t n, const vpm_fmm_params* prm,
                           double* ex, double* ey);

/*
 * The FMM body of VelocityCalc::velocity_fmm_2d
 * (src/velocity_calculation/velocity_calc.cpp:455-578): sources
 * q = -omega s^2 / (2 pi), then u = Ey + u_inf, v = -Ex + v_inf
 * (the free stream of VelocityCalc::get_velocity, velocity_calc.cpp:226-230).
 * Host buffers.
 */
int vpm_velocity2d(vpm_ctx* ctx, const double* x, const double* y, const double* omega,
                   const double* s, const uint8_t* active, int64_t n, const vpm_fmm_params* prm,
                   double u_inf, double v_inf, double* u, double* v, vpm_fmm_stats* stats);

/*
 * Build only the tree and lists 1-4 of a 2D particle set (host buffers), for
 * the parity dumps below. Replaces TreeCell::initializeTree
 * (src/FMM/treeCell.cpp:1043) when no field is wanted.
 */
int vpm_tree2d_build(vpm_ctx* ctx, const double* x, const double* y, const uint8_t* active, int64_t n,
                     const vpm_fmm_params* prm, vpm_fmm_stats* stats);

/*
 * Stage-time history for profiling (no counterpart in the reference). With
 * enable = 1 every later timed evaluation (use_graph 0 or 2) records its 8
 * stage times into a ring of 64 entries, so evaluations can run back to back
 * without host synchronisation. A call returns the recorded entries (oldest
 * first) into ms[entry * 8 + stage], stages in the order keys+sort, levels,
 * lists, P2M+M2M, M2L, L2L, M2P+L2P, P2P, sets *count, clears the ring and
 * leaves recording on or off as `enable` says. Synchronises the stream.
 */
int vpm_stage_history(vpm_ctx* ctx, int32_t enable, int32_t max_entries, float* ms, int32_t* count);

/* Statistics of the last evaluation on this context (synchronises). */
int vpm_last_stats(vpm_ctx* ctx, vpm_fmm_stats* stats);

/*
 * Parity dumps of the tree and lists built by the last 2D call on this
 * context, in the reference's vocabulary (treeCell.hpp:16-75, 112-128):
 *   cells sorted by reference cell ID: ids[k]; ints6[6k..6k+5] = level, ix, iy,
 *   parNum, srcParNum, flags (1 = isLeaf, 2 = isActive); centers2[2k..] = centre.
 *   leaves in the reference's leafList order with each leaf's particle IDs
 *   (ascending, parIDList) as CSR.
 *   list `which` (1..4) as CSR over the reference's cells in ID order: lists 1
 *   and 3 for every leaf (TreeCell::intList, treeCell.cpp:636), lists 2 and 4
 *   for every cell at level >= 2 (TreeCell::extList, treeCell.cpp:818).
 * Call vpm_tree2d_counts first to size the outputs.
 */
int vpm_tree2d_counts(vpm_ctx* ctx, int64_t* n_cells, int64_t* n_leaves, int64_t list_len[4]);
int vpm_tree2d_cells(vpm_ctx* ctx, int64_t* ids, int32_t* ints6, double* centers2);
int vpm_tree2d_leaves(vpm_ctx* ctx, int64_t* leaf_ids, int64_t* offs, int32_t* pids);
int vpm_tree2d_list(vpm_ctx* ctx, int which, int64_t* cell_ids, int64_t* offs, int64_t* ids);

/*
 * vpm_fmm2d_field_device_static: the evaluation of vpm_fmm2d_field_device
 * (device buffers in and out; FP64, mixed or mixed with FP64 M2L) without any
 * device allocation, for callers that cannot call cudaMalloc: programs whose
 * device memory is owned by another allocator (a framework's caching
 * allocator holding the whole budget), and time-step loops that must not
 * stall on the device synchronisation that cudaMalloc and cudaFree can
 * cause. No counterpart in the reference (its FMM allocates host memory
 * freely).
 *
 * All scratch lives in one static device array of 8 MiB that every GPU
 * loading this library keeps until the process exits. Limits: n <= 8192,
 * p <= 12, at most 8192 tree cells; larger requests return VPM_EINVAL, a
 * tree that outgrows the array returns VPM_EOVERFLOW. The first call on a
 * device looks up the array's device address (with that device current);
 * make that first call before any stream capture begins. Both mixed settings
 * use the FP64 M2L with the FP32 near field. Calls share the array and
 * overwrite it; calls that overlap on the GPU race, so serialise them. Runs
 * on `cuda_stream` (a cudaStream_t, NULL = legacy default stream), then reads
 * the device error word back and waits for that stream. errbuf (may be NULL)
 * receives a message of at most errlen bytes.
 */
int vpm_fmm2d_field_device_static(const double* x, const double* y, const double* q,
                                  const uint8_t* active, int64_t n, const vpm_fmm_params* prm,
                                  double* ex, double* ey, void* cuda_stream, char* errbuf,
                                  size_t errlen);

/*
 * Batched independent 2D solves (no counterpart in the reference, which
 * evaluates one particle set per call): solve i is the particle range
 * offsets[i] .. offsets[i+1]-1 of the concatenated arrays (offsets: host
 * array of n_solves + 1 entries, offsets[0] = 0; each solve holds 0 or >= 2
 * particles). Each solve is exactly vpm_fmm2d_field on its range. Solves run
 * concurrently on up to 8 streams of sub-contexts forked from the context's
 * stream; with prm->use_graph the whole batch is captured as one CUDA graph
 * and replayed while offsets, buffers and parameters are unchanged.
 * The _device form takes device pointers and returns without synchronising
 * (vpm_ctx_sync reports the batch's errors); the host form copies in and out.
 */
int vpm_fmm2d_field_batched(vpm_ctx* ctx, int32_t n_solves, const int64_t* offsets, const double* x,
                            const double* y, const double* q, const uint8_t* active, const vpm_fmm_params* prm,
                            double* ex, double* ey);
int vpm_fmm2d_field_batched_device(vpm_ctx* ctx, int32_t n_solves, const int64_t* offsets, const double* x,
                                   const double* y, const double* q, const uint8_t* active,
                                   const vpm_fmm_params* prm, double* ex, double* ey);

/*
 * Streams the last batched call of this context ran its solves on: with
 * use_graph the count chosen by timing the batch's graph with 4, 8, 12 and 16
 * streams on its first call (no counterpart in the reference).
 */
int vpm_batch_streams(vpm_ctx* ctx, int32_t* streams);

/*
 * 3D velocity of the vortex particles (x_j, alpha_j) by the octree treecode
 * of the reference's default 3D path (VELOCITY_3D_TYPE 1):
 *   u(x_i) = sum_j alpha_j x (x_i - x_j) / |x_i - x_j|^3
 * with far cells (R^2 > (2 size)^2) through their 10-term Cartesian moments.
 * Replaces
 *   fmm3D::calcVelocityFast(pos, active, target, ax, ay, az)   src/FMM/fmm3D.cpp (fast3DFMM.cpp:32-92)
 *   FMMCell::generateTree                                     src/FMM/fast3DFMM.cpp:485-745
 *   fastFMM3Dutils::evaluateFMM                               src/FMM/fast3DFMM.cpp:318-472
 *   fmm3D::get_Field_x / _y / _z                              src/FMM/fmm3D.hpp:106-138
 * Every particle is a target, as in the reference (which ignores the target
 * flags); `target` may be NULL. precision = VPM_PREC_MIXED evaluates the P2P
 * and M2P terms in FP32 (FP64 geometry, decisions and per-target sums).
 * Leaf iff particle count < prm->leaf_cap_3d; the root box is the particle
 * box joined with prm->center_3d. Host buffers; stats may be NULL.
 */
int vpm_fmm3d_velocity(vpm_ctx* ctx, const double* x, const double* y, const double* z, const double* ax,
                       const double* ay, const double* az, const uint8_t* active, const uint8_t* target, int64_t n,
                       const vpm_fmm_params* prm, double* u, double* v, double* w, vpm_fmm_stats* stats);

/* Same with device pointers, asynchronous on the context's stream. */
int vpm_fmm3d_velocity_device(vpm_ctx* ctx, const double* x, const double* y, const double* z, const double* ax,
                              const double* ay, const double* az, const uint8_t* active, int64_t n,
                              const vpm_fmm_params* prm, double* u, double* v, double* w);

/*
 * The FMM body of VelocityCalc::velocity_fmm_3d_fast
 * (src/velocity_calculation/velocity_calc.cpp:2384-2524, all particles
 * evaluated): alpha = omega s^3 / (4 pi), then the free stream of
 * VelocityCalc::get_velocity (velocity_calc.cpp:226-236). Host buffers.
 */
int vpm_velocity3d(vpm_ctx* ctx, const double* x, const double* y, const double* z, const double* omega_x,
                   const double* omega_y, const double* omega_z, const double* s, const uint8_t* active, int64_t n,
                   const vpm_fmm_params* prm, double u_inf, double v_inf, double w_inf, double* u, double* v,
                   double* w, vpm_fmm_stats* stats);

/*
 * Octree only (FMMCell::generateTree), for the parity dumps: counts, then
 * per cell in this library's order (level-major, parents in order, octants
 * 0..7 under a parent): ints6 = nPar, chdFlag, parent index, isActive,
 * level, max_level (cell 0 only); geom4 = xc, yc, zc, size; and for every
 * leaf (cell k > 0 with chdFlag 0) its particle IDs in ascending order as
 * CSR leaf_offs[k]..leaf_offs[k+1] (n_cells + 1 offsets). Any output may be
 * NULL.
 */
int vpm_tree3d_build(vpm_ctx* ctx, const double* x, const double* y, const double* z, const uint8_t* active,
                     int64_t n, const vpm_fmm_params* prm, vpm_fmm_stats* stats);
int vpm_tree3d_counts(vpm_ctx* ctx, int64_t* n_cells, int64_t* n_leaves, int32_t* depth);
int vpm_tree3d_cells(vpm_ctx* ctx, int32_t* ints6, double* geom4, int64_t* leaf_offs, int32_t* pids);

/*
 * 3D velocity by the treecode on the shared TreeCell, the reference's
 * alternative 3D path (VELOCITY_3D_TYPE 2 with VELOCITY_CALCULATION_TYPE 2).
 * Replaces
 *   TreeCell::initializeTree(pos, active) with DIM 3   src/FMM/treeCell.cpp:1043-1243
 *   fmm3D::calcVelocity(tree, pos, active, ax, ay, az)  src/FMM/fmm3D.cpp:1064-1405
 *   fmm3D::calcVelocityNearBody(tree, pos, active, target, ax, ay, az)
 *                                                      src/FMM/fmm3D.cpp:1406-1606
 *   fmm3D::get_Field_x / _y / _z                       src/FMM/fmm3D.hpp:106-138
 * as called by VelocityCalc::velocity_fmm_3d (velocity_calc.cpp:2172-2375).
 * The root box is the particle box alone (side = max extent * (1 +
 * exp_tree_pct/100)); a cell is a leaf iff it holds at most prm->max_src
 * active and at most prm->max_par particles (the reference's 3D values are
 * 30 and 50, global.cpp:778-779; vpm_fmm_params_default gives the 2D 50/75).
 * Far iff R^2 > (2 length)^2 (10-term moments), near leaves by direct sum over
 * all their particles, inactive ones included. target = NULL evaluates every
 * particle (calcVelocity); otherwise only flagged ones, the others get zero
 * (calcVelocityNearBody). precision = VPM_PREC_MIXED as for
 * vpm_fmm3d_velocity. Returns VPM_EINVAL when the tree would go deeper than
 * level 10 (the reference's 32-bit cell IDs overflow there) and when a level-1
 * cell is a leaf of a deeper tree (the reference's traversal throws there).
 * Host buffers; stats may be NULL.
 */
int vpm_fmm3d_velocity_treecell(vpm_ctx* ctx, const double* x, const double* y, const double* z, const double* ax,
                                const double* ay, const double* az, const uint8_t* active, const uint8_t* target,
                                int64_t n, const vpm_fmm_params* prm, double* u, double* v, double* w,
                                vpm_fmm_stats* stats);

/* Same with device pointers (target may be NULL), asynchronous on the
 * context's stream; vpm_ctx_sync reports the failures found on the device. */
int vpm_fmm3d_velocity_treecell_device(vpm_ctx* ctx, const double* x, const double* y, const double* z,
                                       const double* ax, const double* ay, const double* az, const uint8_t* active,
                                       const uint8_t* target, int64_t n, const vpm_fmm_params* prm, double* u,
                                       double* v, double* w);

/*
 * 3D TreeCell only (TreeCell::initializeTree with DIM 3,
 * treeCell.cpp:1043-1243), for the parity dumps: vpm_tree3d_counts and
 * vpm_tree3d_cells then describe it (cells level-major, Morton order within a
 * level), and vpm_tree3d_cell_ids gives each cell's reference ID
 * (8^L - 1) / 7 + ix + iy 2^L + iz 4^L (treeCell.cpp:114-148, 223-250).
 */
int vpm_treecell3d_build(vpm_ctx* ctx, const double* x, const double* y, const double* z, const uint8_t* active,
                         int64_t n, const vpm_fmm_params* prm, vpm_fmm_stats* stats);
int vpm_tree3d_cell_ids(vpm_ctx* ctx, int64_t* ids);

/*
 * Learned (leaf caps, p) selector of the mixed 2D form. No counterpart in the
 * reference, which always uses caps 50/75 and p = 10 (global.cpp:311-313);
 * that pair is the selector's fallback.
 *
 * Candidates: 35 pairs (cap, p), cap in {25, 50, 100, 200, 400} (max_src =
 * cap, max_par = 3 cap / 2) times p in {4, 6, 8, 10, 12, 16, 20}, in the
 * order vpm_selector_candidates lists them.
 * Features (228 floats): log10 N, log10 root length, log10 max|q|, log10
 * target error, then for grid levels 3..9 of the root box a 32-bin histogram
 * (fractions of occupied cells) of floor(log2 particles per cell).
 * Network: 228 -> 64 -> 64 -> 64 -> 70 (GELU), FP32 parameters stored per
 * layer as W [out x in] then b [out]; outputs are the standardised log10
 * relative L2 error and log10 time of each candidate. Training (minibatch
 * Adam, masked MSE) and inference (BF16 weights) are CUDA kernels of this
 * library; the inputs and targets given to vpm_mlp_* are already normalised,
 * vpm_select2d normalises with the statistics of vpm_mlp_set_norm.
 */
int64_t vpm_mlp_param_count(void);
int vpm_selector_candidates(int32_t* caps, int32_t* ps, int32_t count);
int vpm_mlp_init(vpm_ctx* ctx, uint64_t seed);
int vpm_mlp_set_params(vpm_ctx* ctx, const float* params, int64_t count);
int vpm_mlp_get_params(vpm_ctx* ctx, float* params, int64_t count);
int vpm_mlp_set_norm(vpm_ctx* ctx, const float* in_mean, const float* in_std, const float* out_mean,
                     const float* out_std);
/* B rows of normalised inputs -> outputs (host arrays); bf16 selects the BF16 inference kernel. */
int vpm_mlp_forward(vpm_ctx* ctx, const float* X, int32_t B, float* Y, int32_t bf16);
/* Gradient (param_count floats) and value of the masked MSE over B rows; mask may be NULL. */
int vpm_mlp_grads(vpm_ctx* ctx, const float* X, const float* Y, const float* mask, int32_t B, float* grads,
                  float* loss);
/* `steps` Adam steps of `batch` rows drawn per epoch without replacement (seeded). */
int vpm_mlp_train(vpm_ctx* ctx, const float* X, const float* Y, const float* mask, int64_t rows, int32_t batch,
                  int32_t steps, float lr, uint64_t seed, float* loss_hist);
/* The 228 features of a particle set (host or device arrays); synchronises. */
int vpm_selector_features2d(vpm_ctx* ctx, const double* x, const double* y, const double* q,
                            const uint8_t* active, int64_t n, double target_err, float* feat);
int vpm_selector_features2d_device(vpm_ctx* ctx, const double* x, const double* y, const double* q,
                                   const uint8_t* active, int64_t n, double target_err, float* feat);
/* The cheapest candidate predicted to meet target_err with margin_decades to
 * spare (fallback 50/75, p = 10); pred (may be NULL) gets the 70 predictions
 * (log10 error, then log10 ms). */
int vpm_select2d(vpm_ctx* ctx, const float* feat, double target_err, double margin_decades, int32_t* max_src,
                 int32_t* max_par, int32_t* p, float* pred);

/*
 * FP64 direct sum of the 2D field at m sampled targets (device pointers,
 * int64 target indices on the device): E_t = sum over active j != t of
 * q_j (x_t - x_j) / |x_t - x_j|^2, the yardstick of the FMM's error (the
 * reference's own direct form, fmm2D::fieldDirSum, fmm2D.cpp:135-179, over
 * all sources). Asynchronous on the context's stream.
 */
int vpm_direct2d_field_device(vpm_ctx* ctx, const double* x, const double* y, const double* q,
                              const uint8_t* active, int64_t n, const int64_t* targets, int64_t m, double* ex,
                              double* ey);

/*
 * FP64 direct sum of the 3D velocity at m sampled targets (device pointers,
 * int64 target indices on the device): u_t = sum over active j != t of
 * alpha_j x (x_t - x_j) / |x_t - x_j|^3, the yardstick of the 3D treecode's
 * error (the reference's near-field kernel, fast3DFMM.cpp:437-459, over all
 * sources). Asynchronous on the context's stream.
 */
int vpm_direct3d_velocity_device(vpm_ctx* ctx, const double* x, const double* y, const double* z,
                                 const double* ax, const double* ay, const double* az, const uint8_t* active,
                                 int64_t n, const int64_t* targets, int64_t m, double* u, double* v, double* w);

/*
 * FMA-throughput microbenchmark of the device (TFLOP/s of dependent FMA
 * chains in FP64 and FP32): the pipe peaks the near-field roofline fractions
 * are quoted against. No counterpart in the reference (measurement utility).
 */
int vpm_measure_fma_peaks(vpm_ctx* ctx, double* fp64_tflops, double* fp32_tflops);

/*
 * Reciprocal-throughput microbenchmark (G reciprocals/s of dependent
 * rcp.approx.ftz.f32 chains): the special-function-unit peak that bounds the
 * FP32 near field, which issues one reciprocal per pair. No counterpart in
 * the reference (measurement utility).
 */
int vpm_measure_rcp_peak(vpm_ctx* ctx, double* grcp_per_s);

#ifdef __cplusplus
}
#endif

#endif /* VPM_FMM_H */
