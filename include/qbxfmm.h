/*
 * qbxfmm.h -- C ABI of the B200 QBX-FMM layer-potential apply.
 *
 * The entry points replace the expansion-wrangler stages that pytential's FMM
 * driver calls (pytential/qbx/fmm.py:414-594), one per stage, plus a whole-apply
 * entry.  All array arguments are plain pointers.  Device pointers are owned by the
 * caller; the library allocates no device memory.  Every call returns QBXFMM_OK or
 * a negative status; QBXFMM_ERR_CUDA leaves the CUDA error in qbxfmm_last_error().
 *
 * Data layout (all int32 indices, float64 coordinates):
 *   - coordinates are structure-of-arrays: x[dim][n];
 *   - sources and targets are in tree order (boxtree's sorted order);
 *   - strengths: [nrhs][nsources] in tree order, float64 for Laplace,
 *     complex128 (interleaved re, im) for Helmholtz;
 *   - box expansions (multipoles and locals): [nboxes][nrhs][ncoeff] complex128;
 *   - QBX expansions: [ncenters][nrhs][ncoeff_qbx] complex128;
 *   - potentials: [nrhs][n] float64 (Laplace) or complex128 (Helmholtz).
 */
#ifndef QBXFMM_H
#define QBXFMM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum qbxfmm_status {
  QBXFMM_OK = 0,
  QBXFMM_ERR_ARG = -1,          /* invalid argument (sizes, orders, null pointers) */
  QBXFMM_ERR_CUDA = -2,         /* a CUDA runtime call failed */
  QBXFMM_ERR_UNSUPPORTED = -3,  /* kernel family / order not built into this library */
  QBXFMM_ERR_DEVICE = -4        /* a kernel reported an error word (bad list entry) */
};

enum qbxfmm_family { QBXFMM_LAPLACE = 0, QBXFMM_HELMHOLTZ = 1 };

/* Which layer potential the sources carry.  The strength of each source is
 * multiplied by charge_coeff for the single-layer part and by dipole_coeff (along
 * the source normal) for the double-layer part, so S, D and D - i k S are one FMM
 * (pytential groups source kernels with the same density the same way,
 * pytential/qbx/__init__.py:526-532). */
typedef struct qbxfmm_kernel {
  int32_t family;            /* enum qbxfmm_family */
  int32_t dim;               /* 2 or 3 */
  double k_re, k_im;         /* Helmholtz wave number (ignored for Laplace) */
  double charge_coeff_re, charge_coeff_im;
  double dipole_coeff_re, dipole_coeff_im;
  int32_t qbx_order;         /* order of the QBX local expansions */
  int32_t fmm_order;         /* order of box multipole/local expansions */
  int32_t nrhs;              /* number of densities applied in one traversal */
  int32_t precision;         /* 0 = plain FP64, 1 = mixed (FP32 far field) */
  int32_t target_specific_qbx; /* 1: the list-1 near field of each QBX target is
                                  evaluated target-specifically (Legendre / line
                                  series per target and source) instead of through
                                  the center's expansion (pytential's
                                  _use_target_specific_qbx, fmm.py:391-394) */
  int32_t fmm_backend;       /* whose expansions' truncation the apply reproduces:
                                QBXFMM_BACKEND_SUMPY (0, the reference's default,
                                fmm_backend="sumpy": sumpy's default expansions, PDE-
                                compressed Cartesian Taylor in 3D) or
                                QBXFMM_BACKEND_FMMLIB (1, fmm_backend="fmmlib":
                                spherical-wave expansions), pytential/qbx/__init__.py:
                                93, 191, 617-659.  Only 3D Helmholtz truncates
                                differently; Laplace and 2D Helmholtz ignore it. */
} qbxfmm_kernel;

enum qbxfmm_backend { QBXFMM_BACKEND_SUMPY = 0, QBXFMM_BACKEND_FMMLIB = 1 };

/* Tree, traversal and QBX geometry, field names after boxtree's Tree /
 * FMMTraversalInfo and pytential's QBXFMMGeometryData
 * (pytential/qbx/geometry.py:361-899).  All pointers address the same memory
 * space (device memory for the CUDA library, host memory for the CPU checker). */
typedef struct qbxfmm_geometry {
  int32_t dim;
  int32_t nboxes, nlevels, nsources, ntargets;
  double root_extent;
  const double* box_centers;                /* [dim][nboxes] */
  const int32_t* box_levels;                /* [nboxes] */
  const int32_t* box_parent_ids;            /* [nboxes], -1 at the root */
  const int32_t* box_child_ids;             /* [2^dim][nboxes], 0 = no child */
  const int32_t* box_source_starts;         /* [nboxes] */
  const int32_t* box_source_counts_nonchild;
  const int32_t* box_source_counts_cumul;
  const double* sources;                    /* [dim][nsources], tree order */
  const double* source_normals;             /* [dim][nsources], tree order */
  const double* targets;                    /* [dim][ntargets], tree order */

  int32_t nsource_boxes;
  const int32_t* source_boxes;
  const int32_t* level_start_source_box_nrs;           /* [nlevels+1] */
  int32_t nsource_parent_boxes;
  const int32_t* source_parent_boxes;
  const int32_t* level_start_source_parent_box_nrs;    /* [nlevels+1] */
  int32_t ntarget_boxes;
  const int32_t* target_boxes;
  int32_t nttp_boxes;                                  /* target_or_target_parent */
  const int32_t* target_or_target_parent_boxes;
  const int32_t* level_start_ttp_box_nrs;              /* [nlevels+1] */
  const int32_t* list1_starts;   /* neighbor_source_boxes, by target box index */
  const int32_t* list1_lists;
  const int32_t* list2_starts;   /* from_sep_siblings, by ttp box index */
  const int32_t* list2_lists;
  const int32_t* list3_starts;   /* from_sep_smaller (all source levels), by target box index */
  const int32_t* list3_lists;
  const int32_t* list4_starts;   /* from_sep_bigger, by ttp box index */
  const int32_t* list4_lists;

  int32_t ncenters;
  const double* centers;                    /* [dim][ncenters], interleaved -,+ */
  const double* expansion_radii;            /* [ncenters] */
  int32_t nglobal_qbx_centers;
  const int32_t* global_qbx_centers;
  const int32_t* qbx_center_to_target_box;  /* [ncenters] -> target box index */
  const int32_t* center_to_targets_starts;  /* [ncenters+1] */
  const int32_t* center_to_targets_lists;   /* tree target indices */

  int32_t nfiltered_targets;                /* non-QBX targets */
  const int32_t* nonqbx_box_target_starts;  /* [nboxes] into the filtered list */
  const int32_t* nonqbx_box_target_counts_nonchild;
  const double* nonqbx_targets;             /* [dim][nfiltered_targets] */
  const int32_t* unfiltered_from_filtered_target_indices;
  const int32_t* sorted_target_ids;         /* tree target -> user target */
  const int32_t* user_source_ids;           /* tree source -> user source */

  int32_t nuser_targets;                    /* user targets = ntargets - ncenters */

  /* Work schedule for the QBX near-field kernels, derived from the lists above:
   * global QBX centers grouped by target box, cut into chunks of at most
   * QBXFMM_CENTER_CHUNK centers, ordered by decreasing list-1 work. */
  int32_t nqbx_chunks;
  const int32_t* qbx_chunk_target_box;      /* target box index per chunk */
  const int32_t* qbx_chunk_start;           /* offset into centers_by_target_box */
  const int32_t* qbx_chunk_count;
  const int32_t* centers_by_target_box;     /* [nglobal_qbx_centers] */

  /* Work schedule for the point evaluations at non-QBX targets: the filtered
   * targets of each target box cut into chunks of at most QBXFMM_CENTER_CHUNK,
   * ordered by decreasing list-1 + list-3 work. */
  int32_t nnonqbx_chunks;
  const int32_t* nonqbx_chunk_target_box;   /* target box index per chunk */
  const int32_t* nonqbx_chunk_start;        /* first filtered target of the chunk */
  const int32_t* nonqbx_chunk_count;

  /* Work schedule for the target-specific near field: (QBX target, center) pairs
   * grouped by the center's target box, in chunks of at most QBXFMM_CENTER_CHUNK. */
  int32_t ntsqbx_chunks;
  const int32_t* tsqbx_chunk_target_box;
  const int32_t* tsqbx_chunk_start;
  const int32_t* tsqbx_chunk_count;
  const int32_t* tsqbx_targets;             /* tree target index per pair */
  const int32_t* tsqbx_centers;             /* center index per pair */

  /* Translation classes for the matrix form of M2L / M2M / L2L.  A class is a
   * translation vector in units of the (source) box width; within a class every
   * translation is the same matrix (up to a per-level factor for M2L), so each
   * class is one dense matrix product over all its pairs.
   *   M2L: list-2 pairs grouped by offset (target - source) / width; with
   *        m2l_class_levels also by level, the classes of one offset consecutive.
   *   M2M: (child -> parent) pairs grouped by (parent level, child position).
   *   L2L: (parent -> child) pairs grouped by (child level, child position). */
  int32_t m2l_nclasses;
  const int32_t* m2l_class_offsets;         /* [dim][m2l_nclasses] integer offsets */
  const int32_t* m2l_class_levels;          /* [m2l_nclasses] level of each class, or NULL when
                                               classes are shared by all levels (Laplace) */
  const int32_t* m2l_class_starts;          /* [m2l_nclasses + 1] into the pair arrays */
  const int32_t* m2l_pair_src;              /* source box per pair (class order) */
  const int32_t* m2l_pair_dst;              /* target box per pair (class order) */
  const int32_t* m2l_tgt_pair_starts;       /* [nttp_boxes + 1] */
  const int32_t* m2l_tgt_pairs;             /* pair indices per target (list-2 order) */
  int32_t m2m_npairs;
  const int32_t* m2m_group_starts;          /* [nlevels * 2^dim + 1]: group = (level, child pos) */
  const int32_t* m2m_pair_src;              /* child box per pair */
  const int32_t* m2m_pair_dst;              /* parent box per pair */
  const int32_t* m2m_par_pair_starts;       /* [nsource_parent_boxes + 1] */
  const int32_t* m2m_par_pairs;             /* pair indices per source parent box */
  int32_t l2l_npairs;
  const int32_t* l2l_group_starts;          /* [nlevels * 2^dim + 1]: group = (level, child pos) */
  const int32_t* l2l_pair_src;              /* parent box per pair */
  const int32_t* l2l_pair_dst;              /* child box per pair */
} qbxfmm_geometry;

#define QBXFMM_CENTER_CHUNK 32

/* Element-local upsampling of a stage-1 density to the quad-stage-2 sources and
 * weighting by area element x quadrature weight
 * (pytential/qbx/__init__.py:1075-1096), fused with the reorder into tree order
 * (pytential/qbx/fmm.py:199-200). */
typedef struct qbxfmm_upsample {
  int32_t nelements;
  int32_t nodes_per_element;       /* stage-1 */
  int32_t quad_nodes_per_element;  /* quad stage 2 */
  const double* matrix;            /* [quad_nodes_per_element][nodes_per_element] */
  const double* quad_weights;      /* [nsources], user source order */
} qbxfmm_upsample;

/* Caller-owned device workspace for one apply (sizes for the kernel's orders and
 * nrhs; see qbxfmm_workspace_sizes). */
typedef struct qbxfmm_workspace {
  void* strengths;    /* [nrhs][nsources] tree order */
  void* mpoles;       /* [nboxes][nrhs][ncoeff(fmm_order)] complex128 */
  void* locals;       /* [nboxes][nrhs][ncoeff(fmm_order)] complex128 */
  void* qbx_exps;     /* [ncenters][nrhs][ncoeff(qbx_order)] complex128 */
  void* pot_nonqbx;   /* [nrhs][nfiltered_targets] */
  void* pot_tree;     /* [nrhs][ntargets] */
  int32_t* error_word;/* one int32, set by kernels that meet an out-of-range index */
  void* translations; /* translation-class matrices (filled by
                         qbxfmm_precompute_translations); NULL selects the
                         per-pair translation kernels */
  void* pair_scratch; /* per-pair translation results, reduced per output box */
} qbxfmm_workspace;

/* Reversed QBX lists for the transposed apply (qbxfmm_transpose_*), by box id, in
 * device memory; built on the host from the apply's geometry (every row's entries in
 * increasing box order). */
typedef struct qbxfmm_transpose_index {
  int32_t ncenter_boxes;
  const int32_t* center_boxes;       /* boxes holding global QBX centers (as target boxes) */
  const int32_t* box_center_starts;  /* [nboxes + 1] into box_centers */
  const int32_t* box_centers;        /* [nglobal_qbx_centers] grouped by box */
  int32_t nlist3_rows;
  const int32_t* list3_rows;         /* boxes in the list 3 of some center box */
  const int32_t* list3_rev_starts;   /* [nlist3_rows + 1] */
  const int32_t* list3_rev_lists;    /* the center boxes whose list 3 holds the row box */
  int32_t nlist1_rows;
  const int32_t* list1_rows;         /* source boxes in the list 1 of some center box */
  const int32_t* list1_rev_starts;   /* [nlist1_rows + 1] */
  const int32_t* list1_rev_lists;    /* the center boxes whose list 1 holds the row box */
  const int32_t* box_pair_starts;    /* [nboxes + 1] into pair_targets / pair_centers */
  const int32_t* pair_targets;       /* the (QBX target, center) pairs of each box's */
  const int32_t* pair_centers;       /*   centers: tree target index, center index */
} qbxfmm_transpose_index;

#ifdef __cplusplus
}
#endif

#endif /* QBXFMM_H */
