/*
 * qbxfmm_api.h -- entry points of libqbxfmm.so.
 *
 * Each stage entry replaces one method of pytential's QBX expansion wrangler
 * (the sumpy-backed QBXExpansionWrangler, pytential/qbx/fmm.py:118-396, and the
 * SumpyExpansionWrangler methods it inherits) as called by drive_fmm
 * (pytential/qbx/fmm.py:414-594).  Outputs are accumulated (+=) into caller-owned
 * device buffers, so a caller can reproduce the driver's "new array per stage, then
 * sum" semantics by passing zeroed buffers, or let stages accumulate in place.
 * All calls are asynchronous on `stream` (a cudaStream_t, NULL = legacy default
 * stream) except qbxfmm_plan_create and qbxfmm_apply_host.
 */
#ifndef QBXFMM_API_H
#define QBXFMM_API_H

#include <stddef.h>
#include <stdint.h>

#include "qbxfmm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qbxfmm_plan qbxfmm_plan;

int qbxfmm_version(void);
/* message of the last failing call on this host thread */
const char* qbxfmm_last_error(void);

/* Validate kernel + geometry and copy the per-level box ranges to the host.
 * Replaces the wrangler constructor (pytential/qbx/fmm.py:141-170) and the
 * backend dispatch in QBXLayerPotentialSource._tree_indep_data_for_wrangler
 * (pytential/qbx/__init__.py:617-659). */
int qbxfmm_plan_create(const qbxfmm_kernel* kernel, const qbxfmm_geometry* geometry,
                       qbxfmm_plan** plan);
int qbxfmm_plan_destroy(qbxfmm_plan* plan);

/* Launch shapes of the 3D Helmholtz stage kernels: densities per CTA of each (0: the
 * library's built-in choice from nrhs and shared-memory limits).  Set by an autotuner
 * that times the candidates on the plan's own geometry (pytential_b200.autotune);
 * the reference has no counterpart (loopy picks its work-group shapes at code
 * generation, pytential/qbx/interactions.py:149, 273, 391, 516).  Results do not
 * depend on the choice beyond the summation order. */
typedef struct qbxfmm_tuning {
  int32_t m2qbxl_densities;   /* 1, 4, 8, 16 (FP64: two warps per center share the tables) */
  int32_t m2l_densities;      /* 1, 4, 8, 16 */
  int32_t p2e_densities;      /* P2M / P2L: 1, 4, 8, 16 (16: orders p <= 15) */
  int32_t l2qbxl_densities;   /* 1, 4 */
  int32_t tsqbx_densities;    /* 1, 4, 16 */
} qbxfmm_tuning;

int qbxfmm_plan_set_tuning(qbxfmm_plan* plan, const qbxfmm_tuning* tuning);
int qbxfmm_plan_get_tuning(const qbxfmm_plan* plan, qbxfmm_tuning* tuning);

/* Per-level FMM orders: orders[l] (0 <= orders[l] <= the kernel's fmm_order) is the
 * order of the multipole and local expansions of the boxes on tree level l; nlevels
 * must equal the geometry's.  Replaces fmm_level_to_order(kernel, kernel_args, tree,
 * level) (pytential/qbx/__init__.py:276-285; the wrangler's level_orders,
 * pytential/qbx/fmm.py:163-166, read per source level at :280-283 and :327-330).  The box expansions stay allocated at fmm_order,
 * which should be the largest level order; the stages that write them truncate each
 * box to its level's order (M2M and L2L level by level), which equals translating
 * between the two orders for every basis except the compressed-Taylor 3D Helmholtz
 * one (fmm_backend QBXFMM_BACKEND_SUMPY, rejected with QBXFMM_ERR_UNSUPPORTED).  The
 * matrix forms of the 3D Laplace translations are not used while level orders are
 * set.  orders == NULL restores fmm_order on every level.  Boxes must be numbered
 * by level (as boxtree numbers them). */
int qbxfmm_plan_set_level_orders(qbxfmm_plan* plan, const int32_t* orders, int32_t nlevels);
int qbxfmm_plan_get_level_orders(const qbxfmm_plan* plan, int32_t* orders, int32_t nlevels);

/* byte sizes of the workspace buffers, in qbxfmm_workspace field order:
 * strengths, mpoles, locals, qbx_exps, pot_nonqbx, pot_tree, translations,
 * pair_scratch (the last two are 0 when the matrix form is not available) */
int qbxfmm_workspace_sizes(const qbxfmm_plan* plan, size_t* sizes8);

/* Build the translation-class matrices of M2L / M2M / L2L into ws->translations
 * (the reference's translation-class precompute, pytential/qbx/fmm.py:155-161,
 * 399-407).  Once per plan and workspace, before qbxfmm_apply. */
int qbxfmm_precompute_translations(const qbxfmm_plan* plan, const qbxfmm_workspace* ws,
                                   void* stream);

/* get_flat_strengths_from_densities + reorder_sources
 * (pytential/qbx/__init__.py:1075-1096; pytential/qbx/fmm.py:199-200).
 * density: [nrhs][nelements * nodes_per_element] stage-1, element-major. */
int qbxfmm_form_strengths(const qbxfmm_plan* plan, const qbxfmm_upsample* up,
                          const void* density, void* strengths, void* stream);

/* form_multipoles (P2M; pytential/qbx/fmm.py:441-445) */
int qbxfmm_form_multipoles(const qbxfmm_plan* plan, const void* strengths, void* mpoles,
                           void* stream);
/* coarsen_multipoles (M2M; pytential/qbx/fmm.py:451-455) */
int qbxfmm_coarsen_multipoles(const qbxfmm_plan* plan, void* mpoles, void* stream);
/* eval_direct (P2P over list 1 at non-QBX targets; pytential/qbx/fmm.py:461-466) */
int qbxfmm_eval_direct(const qbxfmm_plan* plan, const void* strengths, void* pot_nonqbx,
                       int32_t* error_word, void* stream);
/* multipole_to_local (M2L over list 2; pytential/qbx/fmm.py:472-478) */
int qbxfmm_multipole_to_local(const qbxfmm_plan* plan, const void* mpoles, void* locals,
                              int32_t* error_word, void* stream);
/* eval_multipoles (M2P over list 3 at non-QBX targets; pytential/qbx/fmm.py:487-493) */
int qbxfmm_eval_multipoles(const qbxfmm_plan* plan, const void* mpoles, void* pot_nonqbx,
                           int32_t* error_word, void* stream);
/* form_locals (P2L over list 4; pytential/qbx/fmm.py:502-510) */
int qbxfmm_form_locals(const qbxfmm_plan* plan, const void* strengths, void* locals,
                       int32_t* error_word, void* stream);
/* refine_locals (L2L; pytential/qbx/fmm.py:519-523) */
int qbxfmm_refine_locals(const qbxfmm_plan* plan, void* locals, void* stream);
/* eval_locals (L2P at non-QBX targets; pytential/qbx/fmm.py:529-535) */
int qbxfmm_eval_locals(const qbxfmm_plan* plan, const void* locals, void* pot_nonqbx,
                       void* stream);
/* form_global_qbx_locals (P2QBXL; pytential/qbx/fmm.py:231-265,
 * pytential/qbx/interactions.py:40-167) */
int qbxfmm_form_global_qbx_locals(const qbxfmm_plan* plan, const void* strengths,
                                  void* qbx_exps, int32_t* error_word, void* stream);
/* translate_box_multipoles_to_qbx_local (M2QBXL, all source levels in one launch;
 * pytential/qbx/fmm.py:267-312, pytential/qbx/interactions.py:174-294) */
int qbxfmm_translate_box_multipoles_to_qbx_local(const qbxfmm_plan* plan, const void* mpoles,
                                                 void* qbx_exps, int32_t* error_word,
                                                 void* stream);
/* translate_box_local_to_qbx_local (L2QBXL, all levels in one launch;
 * pytential/qbx/fmm.py:314-356, pytential/qbx/interactions.py:301-412) */
int qbxfmm_translate_box_local_to_qbx_local(const qbxfmm_plan* plan, const void* locals,
                                            void* qbx_exps, void* stream);
/* eval_qbx_expansions (QBXL2P; pytential/qbx/fmm.py:358-389,
 * pytential/qbx/interactions.py:419-532); writes pot_tree entries of QBX targets */
int qbxfmm_eval_qbx_expansions(const qbxfmm_plan* plan, const void* qbx_exps, void* pot_tree,
                               void* stream);
/* eval_target_specific_qbx_locals (pytential/qbx/fmm.py:391-394; the reference's
 * native implementation is pytential/qbx/target_specific/impl.pyx:566-785): adds the
 * list-1 near field of every QBX target, evaluated per (target, source) pair, to
 * pot_tree.  Used instead of the list-1 part of form_global_qbx_locals when the
 * kernel's target_specific_qbx flag is set (Laplace). */
int qbxfmm_eval_target_specific_qbx_locals(const qbxfmm_plan* plan, const void* strengths,
                                           void* pot_tree, int32_t* error_word, void* stream);

/* Gradient of the Laplace single-layer potential (2D or 3D) at the non-QBX targets from the
 * FMM's own data of an apply (strengths in tree order, multipoles after
 * coarsen_multipoles, locals after refine_locals -- the workspace of qbxfmm_apply
 * holds them after the call): P2P over list 1, M2P over list 3, L2P of the target
 * box's local, each differentiated at the target (the derivative of the apply's
 * value with the tree held fixed), kernel scaling included.  The reference obtains
 * it from derivative target kernels in its FMM.  grad: [nrhs][dim][nfiltered_targets]
 * (written).  QBXFMM_ERR_UNSUPPORTED for other kernels and per-level orders. */
int qbxfmm_eval_target_gradients(const qbxfmm_plan* plan, const void* strengths,
                                 const void* mpoles, const void* locals, void* grad,
                                 int32_t* error_word, void* stream);

/* The same at the QBX targets: the gradient of each target's center's QBX local at
 * the target (center held fixed) from the apply's qbx_exps (after
 * translate_box_local_to_qbx_local), plus, for a plan with the target-specific near
 * field, the target-derivative of the list-1 sums (Legendre in 3D, powers of a/b in 2D)
 * from the strengths.  grad: [nrhs][dim][ntargets] in tree target order (written; zero
 * at other targets). */
int qbxfmm_eval_qbx_target_gradients(const qbxfmm_plan* plan, const void* strengths,
                                     const void* qbx_exps, void* grad, int32_t* error_word,
                                     void* stream);

/* {{{ transposed QBX stages (2D and 3D Laplace single layer, FP64, one FMM order)
 *
 * The transpose of the apply is the FMM with sources and targets exchanged over
 * the same boxes with transposed lists (the stage entries above on that geometry),
 * in which each global QBX center is a source carrying the order-q multipole of its
 * targets' values.  These four entries are that part, each the transpose of one QBX
 * stage of the apply; `plan` is the APPLY's plan (its centers, lists and sources),
 * `index` its reversed lists.  center_mpoles: [ncenters][nrhs][ncoeff(qbx_order)]
 * complex128.  Each output has one writer (no atomics).  QBXFMM_ERR_UNSUPPORTED for
 * other kernels, the mixed-precision form, per-level orders, qbx_order > 8 or
 * fmm_order > 21 (> 20 in 2D); these stage entries cover the single layer (the 3D
 * double layer runs through qbxfmm_apply_transpose). */

/* transpose of eval_qbx_expansions (fmm.py:358-389): target_values [nrhs][ntargets]
 * in tree target order -> center_mpoles (written; zero for centers without targets) */
int qbxfmm_transpose_eval_qbx_expansions(const qbxfmm_plan* plan, const void* target_values,
                                         void* center_mpoles, int32_t* error_word,
                                         void* stream);
/* transpose of translate_box_local_to_qbx_local (fmm.py:314-356): adds each center
 * multipole, shifted to its box center, into mpoles [nboxes][nrhs][ncoeff] */
int qbxfmm_transpose_translate_box_local_to_qbx_local(const qbxfmm_plan* plan,
                                                      const qbxfmm_transpose_index* index,
                                                      const void* center_mpoles, void* mpoles,
                                                      int32_t* error_word, void* stream);
/* transpose of translate_box_multipoles_to_qbx_local (fmm.py:267-312): adds the M2L
 * of each center multipole into the locals of the boxes in its box's list 3 */
int qbxfmm_transpose_translate_box_multipoles_to_qbx_local(const qbxfmm_plan* plan,
                                                           const qbxfmm_transpose_index* index,
                                                           const void* center_mpoles,
                                                           void* locals, int32_t* error_word,
                                                           void* stream);
/* transpose of form_global_qbx_locals (fmm.py:231-265) with eval_qbx_expansions:
 * adds, for every (QBX target, center) pair, the target's value times the truncated
 * expansion entry (the target-specific form) into the values of the sources of the
 * boxes in the center box's list 1.  target_values: [nrhs][ntargets] tree order;
 * source_values: [nrhs][nsources] tree source order */
int qbxfmm_transpose_form_global_qbx_locals(const qbxfmm_plan* plan,
                                            const qbxfmm_transpose_index* index,
                                            const void* target_values, void* source_values,
                                            int32_t* error_word, void* stream);

/* The whole transpose K^T r in one call, for the Laplace layer potential cq S + cd D
 * (3D: single layer, double layer or both; 2D: cd = 0): `plan` the apply's plan,
 * `transposed` the plan of its exchanged-role geometry (same boxes, transposed
 * lists, no centers, a unit single layer: charge coefficient 1; its translation
 * matrices built into ws by qbxfmm_precompute_translations), ws a workspace of
 * `transposed` (its qbx_exps unused).  target_values: [nrhs][ntargets] of the apply's
 * tree targets; strengths: the same values at its non-QBX targets,
 * [nrhs][nfiltered_targets]; center_mpoles: scratch [ncenters][nrhs][ncoeff(qbx_order)]
 * complex128; grad_scratch: [nrhs][3][nsources] doubles, needed when cd != 0 (the
 * transpose of a dipole layer is the normal derivative of the exchanged-role
 * potential at the sources), else may be NULL; out: [nrhs][nsources] at the apply's
 * sources in tree order, with the kernel scaling (written).  Runs on the transposed
 * plan's streams like qbxfmm_apply; graph-capturable. */
int qbxfmm_apply_transpose(const qbxfmm_plan* plan, const qbxfmm_plan* transposed,
                           const qbxfmm_transpose_index* index, const qbxfmm_workspace* ws,
                           const void* target_values, const void* strengths,
                           void* center_mpoles, void* grad_scratch, void* out, void* stream);

/* }}} */

/* potential assembly: scatter the non-QBX part, add the QBX part, reorder to user
 * targets, apply the kernel scaling (pytential/qbx/fmm.py:569-588,
 * pytential/qbx/__init__.py:775-793).  out: [nrhs][nuser_targets] (written). */
int qbxfmm_assemble(const qbxfmm_plan* plan, const void* pot_nonqbx, const void* pot_tree,
                    void* out, void* stream);

/* The whole apply in drive_fmm's order, from the stage-1 density to user-order
 * potentials; clears the workspace first.  Graph-capturable (no host syncs). */
int qbxfmm_apply(const qbxfmm_plan* plan, const qbxfmm_upsample* up,
                 const qbxfmm_workspace* ws, const void* density, void* out, void* stream);

/* End-to-end apply from host buffers: copies the density host->device, applies,
 * copies the potentials device->host, synchronizes, and checks the error word.
 * Pinned host buffers give asynchronous copies. */
int qbxfmm_apply_host(const qbxfmm_plan* plan, const qbxfmm_upsample* up,
                      const qbxfmm_workspace* ws, const void* density_host, void* out_host,
                      void* density_dev, void* out_dev, void* stream);

/* Size of the device array qbxfmm_apply_noalloc works in (64 MiB). */
#define QBXFMM_NOALLOC_SCRATCH_BYTES (64u << 20)

/* The whole apply (as qbxfmm_apply) for callers that cannot allocate device memory:
 * the caller passes only the density and the output; the intermediate arrays live
 * in a fixed device array of QBXFMM_NOALLOC_SCRATCH_BYTES inside the library, kept by
 * every GPU that loads it until the process exits.  No counterpart in the
 * reference (pytential allocates through its array context).  The first call on a
 * device resolves that array's address and should come before any stream capture;
 * calls that overlap on the GPU share the array and race; problems that need more
 * scratch are rejected with QBXFMM_ERR_ARG before any launch.  Uses the per-pair
 * translation kernels, so it serves 2D and 3D Laplace and 2D Helmholtz plans; 3D
 * Helmholtz plans (whose rotation and translation tables are a caller-owned buffer)
 * are rejected with QBXFMM_ERR_ARG before any launch.  The plan's device must be the
 * current device. */
int qbxfmm_apply_noalloc(const qbxfmm_plan* plan, const qbxfmm_upsample* up,
                         const void* density, void* out, void* stream);

/* The error word of the last qbxfmm_apply_noalloc on the current device (0: no kernel
 * met an out-of-range list entry), copied to *host_out after `stream` has finished
 * (synchronizes the stream).  Allocates nothing. */
int qbxfmm_noalloc_error_word(int32_t* host_out, void* stream);

/* Gradient of the 3D Laplace single-layer potential, by direct summation, at targets
 * far from the sources: grad[d][t] = -1/(4 pi) sum_s charges[s] (x_t - y_s)_d / |x_t - y_s|^3
 * (sources, targets and grad structure-of-arrays [3][n], device pointers).  Supplies the
 * target-position gradient of the adjoint apply; the reference obtains the same
 * quantity from its derivative kernels (a gradient target kernel in the FMM). */
int qbxfmm_laplace3d_grad_direct(int nsources, const double* sources, const double* charges,
                                 int ntargets, const double* targets, double* grad, void* stream);

/* The same gradient computed in FP32 arithmetic (positions relative to a per-block
 * origin, FP32 sums per tile of 256 sources added into FP64), for the mixed-precision
 * adjoint; relative error about 1e-6 for targets well away from the sources. */
int qbxfmm_laplace3d_grad_direct_f32(int nsources, const double* sources,
                                     const double* charges, int ntargets,
                                     const double* targets, double* grad, void* stream);

/* Dense QBX matrix of the 3D Laplace layer potential with charge / dipole weights
 * (replaces the reference's direct QBX evaluation and matrix builder,
 * pytential/qbx/__init__.py:797-1068 and pytential/symbolic/matrix.py:450-523):
 * K[t][s] (row-major, ntargets x nsources, written) = potential at target t of a unit
 * source s, scaled by 1/(4 pi); targets with target_center[t] >= 0 use the order
 * qbx_order QBX expansion about that center, the others the kernel itself.  Sources,
 * normals, targets and centers are structure-of-arrays [3][n] device pointers. */
int qbxfmm_laplace3d_qbx_matrix(int nsources, const double* sources, const double* normals,
                                double charge_coeff, double dipole_coeff, int ntargets,
                                const double* targets, const int32_t* target_center,
                                int ncenters, const double* centers, int qbx_order, double* K,
                                void* stream);

/* Dense QBX matrix of the 2D Helmholtz layer potential (the same reference routines as
 * qbxfmm_laplace3d_qbx_matrix): K[t][s] (row-major complex128, ntargets x nsources,
 * written) = potential at target t of a unit source s with charge weight
 * charge_re + i charge_im and dipole weight dipole_re + i dipole_im, times i/4; QBX
 * targets (target_center[t] >= 0) use the order qbx_order (<= 8) H2D expansion about
 * that center, the others H_0 / H_1 themselves.  Sources, normals, targets and centers
 * are structure-of-arrays [2][n] device pointers. */
int qbxfmm_helmholtz2d_qbx_matrix(int nsources, const double* sources, const double* normals,
                                  double k, double charge_re, double charge_im,
                                  double dipole_re, double dipole_im, int ntargets,
                                  const double* targets, const int32_t* target_center,
                                  int ncenters, const double* centers, int qbx_order, void* K,
                                  void* stream);

/* The same for the 2D Laplace layer potential (structure-of-arrays [2][n]; kernel
 * scaling -1/(2 pi), log|t - s| and its source-normal derivative; any qbx_order <= 32). */
int qbxfmm_laplace2d_qbx_matrix(int nsources, const double* sources, const double* normals,
                                double charge_coeff, double dipole_coeff, int ntargets,
                                const double* targets, const int32_t* target_center,
                                int ncenters, const double* centers, int qbx_order, double* K,
                                void* stream);

/* The same for the 3D Helmholtz layer potential (complex128 K, structure-of-arrays
 * [3][n], e^{ik r} / (4 pi r); QBX targets through the series of order qbx_order <= 8
 * of the target-specific near field, in the truncation of fmm_backend:
 * QBXFMM_BACKEND_SUMPY (the reference's default: the degree-qbx_order Taylor
 * polynomial about the center, j_n cut to its power series) or QBXFMM_BACKEND_FMMLIB
 * (the spherical-wave series). */
int qbxfmm_helmholtz3d_qbx_matrix(int nsources, const double* sources, const double* normals,
                                  double k, double charge_re, double charge_im,
                                  double dipole_re, double dipole_im, int ntargets,
                                  const double* targets, const int32_t* target_center,
                                  int ncenters, const double* centers, int qbx_order,
                                  int fmm_backend, void* K, void* stream);

/* Target-to-QBX-center association (replaces pytential's QBXTargetAssociator:
 * marking, pytential/qbx/target_assoc.py:544-633, and center finding, 243-363 and
 * 637-749, with the side requests of the table at 81-103).  Points are searched on
 * uniform cell grids: qbxfmm_cell_keys gives each point (structure-of-arrays
 * [dim][n], device) the key (ix * ncells[1] + iy) * ncells[2] + iz of its cell,
 * i = floor((x - lo) / h) clamped to [0, ncells), and the caller sorts the keys
 * (ascending) with the permutation that sorts them.  A grid's cell width h must be at
 * least the search radius: the largest source tunnel radius (source grid) and the
 * largest tolerant center radius (center grid).  In 2D ncells[2] = 1. */
typedef struct {
  double lo[3];
  double h;
  int64_t ncells[3];
} qbxfmm_cell_grid;

int qbxfmm_cell_keys(int dim, int n, const double* points, const qbxfmm_cell_grid* grid,
                     int64_t* keys, void* stream);

typedef struct {
  int32_t dim;
  int32_t ntargets;
  const double* targets;               /* [dim][ntargets] */
  const int32_t* target_sides;         /* 0, +-1 (surface), +-2 */
  int32_t nsources;                    /* 0: no marking (surface targets only) */
  const double* sources;               /* [dim][nsources] */
  const double* source_tunnel_radii;   /* [nsources] */
  const int64_t* source_keys;          /* sorted cell keys of the sources */
  const int32_t* source_order;         /* source of each sorted key */
  qbxfmm_cell_grid source_grid;
  int32_t ncenters;                    /* even: interior (-1), odd: exterior (+1) */
  const double* centers;               /* [dim][ncenters] */
  const double* center_tolerant_radii; /* r_c (1 + tolerance) */
  const int64_t* center_keys;
  const int32_t* center_order;
  qbxfmm_cell_grid center_grid;
} qbxfmm_assoc_problem;

/* target_to_center[t] = the chosen center, -1 (target needs no QBX) or -2 (a close
 * target without an admissible center: the reference's association failure).  A
 * target is close if |side| = 1 or some source lies within its tunnel radius; among
 * centers of an admissible side with |t - c| <= r_c (1 + tolerance) the one of least
 * |t - c| / (r_c (1 + tolerance)) on each side is taken (ties: lower index), then the
 * side whose center is nearer (ties: interior).  Equal to the host restatement bit
 * for bit (every distance operation separately rounded). */
int qbxfmm_associate_targets(const qbxfmm_assoc_problem* problem, int32_t* target_to_center,
                             void* stream);

#ifdef __cplusplus
}
#endif

#endif /* QBXFMM_API_H */
