// Internal launcher declarations (one per wrangler stage).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace qbx {

// host-side sizes for the translation-matrix kernels, filled at plan creation
struct TransHost {
  int m2l_max_pairs = 0;                 // largest M2L class
  int m2l_npairs = 0;                    // all M2L pairs (pair-scratch rows)
  int m2m_level_max_group[64] = {0};     // largest (level, child position) group per level
  int l2l_level_max_group[64] = {0};
  int l2l_level_pairs[64] = {0};         // L2L pairs whose child is on a level
  const int32_t* lvl_source_parent = nullptr;   // host copy (owned by the plan)
};

// shape of the matrix-form translations: real (rp x kp) matrices acting on
// interleaved (re, im) vectors of ncf complex coefficients
struct TransCfg {
  int p = 0, ncf = 0, rp = 0, kp = 0;
  int m2m_mat_mod = 8;        // M2M / L2L matrix = base + group % mod (mod 0: base + group)
  size_t m2m_base = 0, l2l_base = 0;
  int m2l_div_by_width = 1;   // M2L reduction scales by 1 / box width (Laplace)
  size_t nmatrices = 0;
};

// M2L classes merged by the lattice symmetries of their offsets (laplace.cuh):
// canon_off [3][ncanon] the canonical offsets, cls_code[class] = canonical index << 4 |
// symmetry code
struct M2LSymClasses {
  int ncanon = 0;
  std::vector<int32_t> canon_off, cls_code;
};
M2LSymClasses m2l_symmetry_classes(int nclasses, const std::vector<int32_t>& offs);
// the same on the device (in the translations buffer)
struct TransAux {
  const int32_t* canon_off = nullptr;
  const int32_t* cls_code = nullptr;
};

TransCfg trans_cfg_laplace3(int p, int nm2l);
TransCfg trans_cfg_helm3(int p, int nclasses, int nlevels);
bool trans_supported(const TransCfg& c);
size_t trans_matrix_bytes(const TransCfg& c);
size_t trans_scratch_bytes(const TransCfg& c, int npairs, int nrhs);
cudaError_t launch_trans_build(const TransCfg& c, int nm2l, const int32_t* offs, double* T,
                               cudaStream_t st);
cudaError_t launch_m2l_gemm(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                            int nrhs, const double* T, const TransAux& aux, const double2* mp,
                            double2* lo, double* cpair, int32_t* err, cudaStream_t st);
cudaError_t launch_m2m_gemm(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                            int nrhs, const double* T, double2* mp, double* cpair, int32_t* err,
                            cudaStream_t st);
bool trans_mv_supported(const TransCfg& c);
cudaError_t launch_m2m_mv(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                          int nrhs, const double* T, double2* mp, int32_t* err, cudaStream_t st);
cudaError_t launch_l2l_mv(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                          int nrhs, const double* T, double2* lo, int32_t* err, cudaStream_t st);
cudaError_t launch_l2l_gemm(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                            int nrhs, const double* T, double2* lo, int32_t* err, cudaStream_t st);
cudaError_t launch_trans_reduce_m2l(const qbxfmm_geometry& g, const TransCfg& c, int nrhs,
                                    const double* cpair, double2* lo, cudaStream_t st);
cudaError_t launch_trans_reduce_m2m(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                                    int lev, int nrhs, const double* cpair, double2* mp,
                                    cudaStream_t st);
// mixed precision (3D Laplace): FP32 far field, split-TF32 translations
cudaError_t launch_p2m_mixed(const qbxfmm_geometry& g, SourceCoeffs sc, int p, int nrhs,
                             const double* s, double2* mp, cudaStream_t st);
cudaError_t launch_p2l_mixed(const qbxfmm_geometry& g, SourceCoeffs sc, int p, int nrhs,
                             const double* s, double2* lo, int32_t* err, cudaStream_t st);
cudaError_t launch_m2qbxl_mixed(const qbxfmm_geometry& g, int pf, int q, int nrhs,
                                const double2* mp, double2* qe, int32_t* err, cudaStream_t st);
void tf32_dims(const TransCfg& c, int& rp16, int& kp8);
bool tf32_supported(const TransCfg& c);
size_t tf32_matrix_bytes(const TransCfg& c);
cudaError_t launch_trans_split_tf32(const TransCfg& c, const double* T, uint32_t* T32,
                                    cudaStream_t st);
cudaError_t launch_m2l_gemm_mixed(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                                  int nrhs, const uint32_t* T32, const TransAux& aux,
                                  const double2* mp, double2* lo, double* cpair, int32_t* err,
                                  cudaStream_t st);
cudaError_t launch_m2m_gemm_mixed(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                                  int nrhs, const uint32_t* T32, double2* mp, double* cpair,
                                  int32_t* err, cudaStream_t st);
cudaError_t launch_l2l_gemm_mixed(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                                  int nrhs, const uint32_t* T32, double2* lo, int32_t* err,
                                  cudaStream_t st);
// scratch-free forms on the tiled kernel (per-level classes, 3D Helmholtz)
cudaError_t launch_m2m_direct(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                              int nrhs, const double* T, double2* mp, int32_t* err, cudaStream_t st);
cudaError_t launch_l2l_direct(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                              int nrhs, const double* T, double2* lo, int32_t* err, cudaStream_t st);

cudaError_t launch_form_strengths(const qbxfmm_geometry& g, const qbxfmm_upsample& up, int nrhs,
                                  const double* density, double* strengths, cudaStream_t st);
cudaError_t launch_p2m(const qbxfmm_geometry& g, SourceCoeffs sc, int p, int nrhs,
                       const double* s, double2* mp, cudaStream_t st);
cudaError_t launch_m2m(const qbxfmm_geometry& g, const int32_t* lvl_host, int p, int nrhs,
                       double2* mp, cudaStream_t st);
cudaError_t launch_m2l(const qbxfmm_geometry& g, int p, int nrhs, const double2* mp, double2* lo,
                       int32_t* err, cudaStream_t st);
cudaError_t launch_p2l(const qbxfmm_geometry& g, SourceCoeffs sc, int p, int nrhs,
                       const double* s, double2* lo, int32_t* err, cudaStream_t st);
cudaError_t launch_l2l(const qbxfmm_geometry& g, const int32_t* lvl_host, int p, int nrhs,
                       double2* lo, cudaStream_t st);
cudaError_t launch_eval_direct(const qbxfmm_geometry& g, SourceCoeffs sc, int nrhs,
                               const double* s, double* pot, int32_t* err, cudaStream_t st);
cudaError_t launch_eval_multipoles(const qbxfmm_geometry& g, int p, int nrhs, const double2* mp,
                                   double* pot, int32_t* err, cudaStream_t st);
cudaError_t launch_eval_locals(const qbxfmm_geometry& g, int p, int nrhs, const double2* lo,
                               double* pot, cudaStream_t st);
cudaError_t launch_p2qbxl(const qbxfmm_geometry& g, SourceCoeffs sc, int q, int nrhs,
                          const double* s, double2* qe, int32_t* err, cudaStream_t st);
cudaError_t launch_m2qbxl(const qbxfmm_geometry& g, int pf, int q, int nrhs, const double2* mp,
                          double2* qe, int32_t* err, cudaStream_t st);
cudaError_t launch_l2qbxl(const qbxfmm_geometry& g, int pf, int q, int nrhs, const double2* lo,
                          double2* qe, cudaStream_t st);
cudaError_t launch_qbxl2p(const qbxfmm_geometry& g, int q, int nrhs, const double2* qe,
                          double* pt, cudaStream_t st);
cudaError_t launch_tsqbx(const qbxfmm_geometry& g, SourceCoeffs sc, int q, int nrhs,
                         const double* s, double* pt, int32_t* err, cudaStream_t st);
cudaError_t launch_assemble(const qbxfmm_geometry& g, int nrhs, const double* pot_nonqbx,
                            const double* pot_tree, double* out, cudaStream_t st);

// 2D Helmholtz (complex128 strengths and potentials)
cudaError_t h2_launch_form_strengths(const qbxfmm_geometry& g, const qbxfmm_upsample& up, int nrhs,
                                     const double2* density, double2* strengths, cudaStream_t st);
cudaError_t h2_launch_p2m(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                          const double2* s, double2* mp, int32_t* err, cudaStream_t st);
cudaError_t h2_launch_m2m(const qbxfmm_geometry& g, const int32_t* lvl_host, HelmCoeffs hc, int p,
                          int nrhs, double2* mp, int32_t* err, cudaStream_t st);
cudaError_t h2_launch_eval_direct(const qbxfmm_geometry& g, HelmCoeffs hc, int nrhs,
                                  const double2* s, double2* pot, int32_t* err, cudaStream_t st);
cudaError_t h2_launch_m2l(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                          const double2* mp, double2* lo, int32_t* err, cudaStream_t st);
cudaError_t h2_launch_eval_multipoles(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                                      const double2* mp, double2* pot, int32_t* err, cudaStream_t st);
cudaError_t h2_launch_p2l(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                          const double2* s, double2* lo, int32_t* err, cudaStream_t st);
cudaError_t h2_launch_l2l(const qbxfmm_geometry& g, const int32_t* lvl_host, HelmCoeffs hc, int p,
                          int nrhs, double2* lo, int32_t* err, cudaStream_t st);
cudaError_t h2_launch_eval_locals(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                                  const double2* lo, double2* pot, int32_t* err, cudaStream_t st);
cudaError_t h2_launch_p2qbxl(const qbxfmm_geometry& g, HelmCoeffs hc, int q, int nrhs,
                             const double2* s, double2* qe, int32_t* err, cudaStream_t st);
cudaError_t h2_launch_m2qbxl(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int q, int nrhs,
                             const double2* mp, double2* qe, int32_t* err, cudaStream_t st);
cudaError_t h2_launch_l2qbxl(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int q, int nrhs,
                             const double2* lo, double2* qe, int32_t* err, cudaStream_t st);
cudaError_t h2_launch_qbxl2p(const qbxfmm_geometry& g, HelmCoeffs hc, int q, int nrhs,
                             const double2* qe, double2* pt, cudaStream_t st);
cudaError_t h2_launch_tsqbx(const qbxfmm_geometry& g, HelmCoeffs hc, int q, int nrhs,
                            const double2* s, double2* pt, int32_t* err, cudaStream_t st);
cudaError_t h2_launch_assemble(const qbxfmm_geometry& g, int nrhs, const double2* pot_nonqbx,
                               const double2* pot_tree, double2* out, cudaStream_t st);

// 3D Helmholtz (complex128; translations through the matrices / Gaunt table)
cudaError_t h3_launch_p2m(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                          const double2* s, double2* mp, cudaStream_t st);
cudaError_t h3_launch_p2l(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                          const double2* s, double2* lo, int32_t* err, cudaStream_t st);
cudaError_t h3_launch_eval_direct(const qbxfmm_geometry& g, HelmCoeffs hc, int nrhs,
                                  const double2* s, double2* pot, int32_t* err, cudaStream_t st);
cudaError_t h3_launch_eval_multipoles(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                                      const double2* mp, double2* pot, int32_t* err, cudaStream_t st);
cudaError_t h3_launch_eval_locals(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                                  const double2* lo, double2* pot, cudaStream_t st);
cudaError_t h3_launch_p2qbxl(const qbxfmm_geometry& g, HelmCoeffs hc, int q, int nrhs,
                             const double2* s, double2* qe, int32_t* err, cudaStream_t st);
// 3D Helmholtz M2L by rotation: per-direction rotation tables (Dtab, h3_m2l_dsize
// doubles each) and per-(length, level) coaxial tables (Ctab, h3_m2l_csize complex
// each) built by h3_launch_m2l_tables; clsmap[2 c] / [2 c + 1] = direction / coaxial
// table of M2L class c.
__host__ __device__ size_t h3_m2l_dsize(int pf);
__host__ __device__ size_t h3_m2l_csize(int pf);
cudaError_t h3_launch_m2l_tables(int pf, int ndir, int ncoax, const double* dirs,
                                 const double* coaxp, const double* start, const double* isq,
                                 const double* rt, const double* gaunt, double* Dtab,
                                 double2* Ctab, cudaStream_t st);
cudaError_t h3_launch_m2l_rot(const qbxfmm_geometry& g, int pf, int nrhs, const double2* mp,
                              double2* lo, const double* Dtab, const double2* Ctab,
                              const double* clsmap, int32_t* err, cudaStream_t st,
                              bool fp32 = false, int rb = 0);
// rot: rotation tables of h3_rotation_tables (start values, recurrence factors,
// lambda = 0 Gaunt slice)
// fp32: the mixed-precision form (FP32 arithmetic, FP64 expansions in and out)
cudaError_t h3_launch_m2qbxl(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int q, int nrhs,
                             const double2* mp, const double* rot, double2* qe, int32_t* err,
                             cudaStream_t st, bool fp32 = false);
cudaError_t h3_launch_l2qbxl(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int q, int nrhs,
                             const double2* lo, const double* rot, double2* qe, int32_t* err,
                             cudaStream_t st);
cudaError_t h3_launch_qbxl2p(const qbxfmm_geometry& g, HelmCoeffs hc, int q, int nrhs,
                             const double2* qe, double2* pt, cudaStream_t st);
cudaError_t h3_launch_tsqbx(const qbxfmm_geometry& g, HelmCoeffs hc, int q, int nrhs,
                            const double2* s, double2* pt, int32_t* err, cudaStream_t st);
cudaError_t h3_launch_assemble(const qbxfmm_geometry& g, int nrhs, const double2* pot_nonqbx,
                               const double2* pot_tree, double2* out, cudaStream_t st);
cudaError_t h3_launch_trans_build(const qbxfmm_geometry& g, const TransCfg& tc, double k,
                                  const double* gaunt, double* T, cudaStream_t st);

// transposed QBX stages (kernels_transpose.cu)
cudaError_t launch_tr_qbxl2p(const qbxfmm_geometry& g, int q, int nrhs, double cq,
                             const double* vals, double2* cmp, int32_t* err, cudaStream_t st);
cudaError_t launch_tr_l2qbxl(const qbxfmm_geometry& g, const qbxfmm_transpose_index& ix, int p,
                             int q, int nrhs, const double2* cmp, double2* mpoles, int32_t* err,
                             cudaStream_t st);
cudaError_t launch_tr_m2qbxl(const qbxfmm_geometry& g, const qbxfmm_transpose_index& ix, int p,
                             int q, int nrhs, const double2* cmp, double2* locals, int32_t* err,
                             cudaStream_t st);
cudaError_t launch_tr_p2qbxl(const qbxfmm_geometry& g, const qbxfmm_transpose_index& ix, int q,
                             int nrhs, double cq, const double* tvals, double* vals, double* grads,
                             int32_t* err, cudaStream_t st);
// 2D Laplace transposed QBX stages: which = 0 QBXL2P^T (tvals -> cmp), 1 L2QBXL^T
// (cmp -> box multipoles), 2 M2QBXL^T (cmp -> box locals), 3 P2QBXL^T (tvals -> vals)
cudaError_t launch_tr2_stages(int which, const qbxfmm_geometry& g, const qbxfmm_transpose_index* ix,
                              int p, int q, int nrhs, double cq, const double* tvals,
                              double2* cmp, double2* box_exps, double* vals, int32_t* err,
                              cudaStream_t st);
cudaError_t launch_tr_combine(const qbxfmm_geometry& g, int nrhs, double scale, double cq,
                              double cd, const double* vals, const double* grads, double* out,
                              cudaStream_t st);

// gradient of the 3D Laplace single layer at the non-QBX targets (kernels_fmmgrad.cu)
// 2D Laplace single layer: grad[r][2][n]
cudaError_t launch_grad2_targets(const qbxfmm_geometry& g, double cq, double scale, int p,
                                 int nrhs, const double* strengths, const double2* mpoles,
                                 const double2* locals, double* grad, int32_t* err,
                                 cudaStream_t st);
cudaError_t launch_grad2_qbx_targets(const qbxfmm_geometry& g, double cq, double scale, int q,
                                     int nrhs, bool target_specific, const double* strengths,
                                     const double2* qbx_exps, double* grad, int32_t* err,
                                     cudaStream_t st);
cudaError_t launch_grad_targets(const qbxfmm_geometry& g, double cq, double scale, int p,
                                int nrhs, const double* strengths, const double2* mpoles,
                                const double2* locals, double* grad, int32_t* err,
                                cudaStream_t st);

cudaError_t launch_grad_qbx_targets(const qbxfmm_geometry& g, double cq, double scale, int q,
                                    int nrhs, bool target_specific, const double* strengths,
                                    const double2* qbx_exps, double* grad, int32_t* err,
                                    cudaStream_t st);

// per-level FMM orders: zero the coefficients of boxes [b0, b1) above their level's order
cudaError_t launch_level_mask(const qbxfmm_geometry& g, int b0, int b1, const int32_t* orders,
                              int family, int ncf, int nrhs, double2* exps, cudaStream_t st);

}  // namespace qbx
