// Transposed QBX stages of the 3D Laplace single-layer apply, sm_100a.
//
// The transpose of the apply is the FMM with sources and targets exchanged over the
// same boxes and transposed lists; the QBX centers act there as sources carrying
// the order-q multipole of their targets' values.  These kernels are that part:
//
//   k_tr_qbxl2p   transpose of QBXL2P (fmm.py:358-389): per global center, the
//                 order-q multipole of its targets' values about the center
//                 (rscale = expansion radius), times the charge coefficient
//   k_tr_l2qbxl   transpose of L2QBXL (fmm.py:314-356): per box, the center
//                 multipoles of its centers shifted into the box multipole (M2M,
//                 the reciprocal of the box-to-center L2L)
//   k_tr_m2qbxl   transpose of M2QBXL (fmm.py:267-312): per box s, the M2L of the
//                 center multipoles of every center box whose list 3 holds s into
//                 the local of s
//   k_tr_p2qbxl   transpose of P2QBXL (fmm.py:231-265): per source box s, the center
//                 multipoles of every center box whose list 1 holds s evaluated at
//                 the sources of s (M2P)
//
// Each output (a box expansion, a source value) has one writer: the kernels gather
// over the reversed lists of qbxfmm_transpose_index, so results do not depend on
// scheduling.  The box stages of the transpose are the library's own P2M / M2M /
// M2L / M2P / P2L / L2L / L2P / P2P on the exchanged-role geometry.
#include "laplace.cuh"
#include "kernels.h"

namespace qbx {

namespace {

constexpr int NT = 128;
constexpr int TR_CB = 32;     // centers staged per batch in k_tr_p2qbxl

QBX_D bool box_ok(const qbxfmm_geometry& g, int b, int32_t* err)
{
  if ((unsigned)b < (unsigned)g.nboxes) return true;
  report(err, QBX_DEVERR_BAD_BOX);
  return false;
}

QBX_D bool center_ok(const qbxfmm_geometry& g, int c, int32_t* err)
{
  if ((unsigned)c < (unsigned)g.ncenters) return true;
  report(err, QBX_DEVERR_BAD_CENTER);
  return false;
}

}  // namespace

// {{{ QBXL2P^T: center multipoles from the targets' values

__global__ void __launch_bounds__(64)
k_tr_qbxl2p(qbxfmm_geometry g, int q, int ncq, int nrhs, double cq,
            const double* __restrict__ vals, double2* __restrict__ cmp, int32_t* err)
{
  extern __shared__ double2 smem2[];
  double2* tab = smem2;                         // [ncq] R table
  int ctr = g.global_qbx_centers[blockIdx.x];
  int r = blockIdx.y;
  if (!center_ok(g, ctr, err)) return;
  double cc[3];
  load_point<3>(g.centers, g.ncenters, ctr, cc);
  double rinv = 1.0 / g.expansion_radii[ctr];
  double2 acc[2] = {c2(0.0), c2(0.0)};
  int t0 = g.center_to_targets_starts[ctr], t1 = g.center_to_targets_starts[ctr + 1];
  for (int it = t0; it < t1; ++it) {
    int t = g.center_to_targets_lists[it];
    bool ok = (unsigned)t < (unsigned)g.ntargets;
    if (!ok) report(err, QBX_DEVERR_BAD_CENTER);
    double x[3] = {0.0, 0.0, 0.0};
    if (ok) load_point<3>(g.targets, g.ntargets, t, x);
    __syncthreads();
    sh3_R_table(q, (x[0] - cc[0]) * rinv, (x[1] - cc[1]) * rinv, (x[2] - cc[2]) * rinv, tab,
                threadIdx.x, blockDim.x);
    __syncthreads();
    double v = ok ? cq * vals[(size_t)r * g.ntargets + t] : 0.0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      int o = threadIdx.x + h * 64;
      if (o < ncq) acc[h] = caxpy(v, cconj(tab[o]), acc[h]);
    }
  }
  double2* M = cmp + ((size_t)ctr * nrhs + r) * ncq;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int o = threadIdx.x + h * 64;
    if (o < ncq) M[o] = acc[h];
  }
}

// }}}

// {{{ L2QBXL^T: center multipoles into the multipole of their box (M2M from the center)

// M_n^m += sum_{k <= min(n, q)} (rho_c / rho_b)^k sum_l Mc_k^l conj(R_{n-k}^{m-l}(d)),
// d = (center - box center) / rho_b: the entries of the box-to-center L2L.
__global__ void __launch_bounds__(NT)
k_tr_l2qbxl(qbxfmm_geometry g, qbxfmm_transpose_index ix, int p, int q, int ncf, int ncq,
            int nrhs, const double2* __restrict__ cmp, double2* __restrict__ mpoles, int32_t* err)
{
  extern __shared__ double2 smem2[];
  double2* tab = smem2;               // [ncf] R table of order p
  double2* Min = smem2 + ncf;         // [ncq] the center multipole
  int b = ix.center_boxes[blockIdx.x];
  int r = blockIdx.y;
  if (!box_ok(g, b, err)) return;
  double rho_b = level_width(g, g.box_levels[b]);
  double cb[3];
  load_point<3>(g.box_centers, g.nboxes, b, cb);
  double2 acc[2] = {c2(0.0), c2(0.0)};
  for (int k = ix.box_center_starts[b]; k < ix.box_center_starts[b + 1]; ++k) {
    int ctr = ix.box_centers[k];
    bool ok = center_ok(g, ctr, err);
    double cc[3] = {cb[0], cb[1], cb[2]};
    double rho_c = rho_b;
    if (ok) {
      load_point<3>(g.centers, g.ncenters, ctr, cc);
      rho_c = g.expansion_radii[ctr];
    }
    __syncthreads();
    sh3_R_table(p, (cc[0] - cb[0]) / rho_b, (cc[1] - cb[1]) / rho_b, (cc[2] - cb[2]) / rho_b,
                tab, threadIdx.x, NT);
    for (int i = threadIdx.x; i < ncq; i += NT)
      Min[i] = ok ? cmp[((size_t)ctr * nrhs + r) * ncq + i] : c2(0.0);
    __syncthreads();
    double ratio = rho_c / rho_b;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      int o = threadIdx.x + h * NT;
      if (o >= ncf) break;
      int n, m;
      decode3(o, n, m);
      double2 a = acc[h];
      double rk = 1.0;
      int kmax = n < q ? n : q;
      for (int kk = 0; kk <= kmax; ++kk, rk *= ratio)
        for (int l = -kk; l <= kk; ++l) {
          int dm = m - l;
          if (dm > n - kk || -dm > n - kk) continue;
          a = cfmac(cscale(rk, sh3_get(Min, kk, l)), sh3_get(tab, n - kk, dm), a);
        }
      acc[h] = a;
    }
  }
  double2* M = mpoles + ((size_t)b * nrhs + r) * ncf;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int o = threadIdx.x + h * NT;
    if (o < ncf) M[o] = cadd(M[o], acc[h]);
  }
}

// }}}

// {{{ M2QBXL^T: center multipoles into the locals of the list-3 boxes (M2L from the center)

// L_j^i += (-1)^j (rho_s / rho_c)^j / rho_c sum_{k <= q, |l| <= k} Mc_k^l S_{k+j}^{l+i}(d),
// d = (box center - center) / rho_c: the entries of M2QBXL with the roles exchanged.
__global__ void __launch_bounds__(NT)
k_tr_m2qbxl(qbxfmm_geometry g, qbxfmm_transpose_index ix, int p, int q, int ncf, int ncq,
            int nrhs, const double2* __restrict__ cmp, double2* __restrict__ locals, int32_t* err)
{
  extern __shared__ double2 smem2[];
  const int nS = idx3(p + q + 1, 0);
  double2* S = smem2;                 // [nS] S table of order p + q
  double2* Min = smem2 + nS;          // [ncq]
  int s = ix.list3_rows[blockIdx.x];
  int r = blockIdx.y;
  if (!box_ok(g, s, err)) return;
  double rho_s = level_width(g, g.box_levels[s]);
  double cs[3];
  load_point<3>(g.box_centers, g.nboxes, s, cs);
  double2 acc[2] = {c2(0.0), c2(0.0)};
  for (int e = ix.list3_rev_starts[blockIdx.x]; e < ix.list3_rev_starts[blockIdx.x + 1]; ++e) {
    int b = ix.list3_rev_lists[e];
    if (!box_ok(g, b, err)) continue;
    for (int k = ix.box_center_starts[b]; k < ix.box_center_starts[b + 1]; ++k) {
      int ctr = ix.box_centers[k];
      bool ok = center_ok(g, ctr, err);
      // a bad center contributes nothing: a unit vector for the table, zero multipole
      double cc[3] = {cs[0] - 1.0, cs[1], cs[2]};
      double rho_c = 1.0;
      if (ok) {
        load_point<3>(g.centers, g.ncenters, ctr, cc);
        rho_c = g.expansion_radii[ctr];
      }
      __syncthreads();
      sh3_S_table(p + q, (cs[0] - cc[0]) / rho_c, (cs[1] - cc[1]) / rho_c,
                  (cs[2] - cc[2]) / rho_c, S, threadIdx.x, NT);
      for (int i = threadIdx.x; i < ncq; i += NT)
        Min[i] = ok ? cmp[((size_t)ctr * nrhs + r) * ncq + i] : c2(0.0);
      __syncthreads();
      double ratio = rho_s / rho_c;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        int o = threadIdx.x + h * NT;
        if (o >= ncf) break;
        int j, ii;
        decode3(o, j, ii);
        double2 v = c2(0.0);
        for (int kk = 0; kk <= q; ++kk)
          for (int l = -kk; l <= kk; ++l) v = cfma(sh3_get(Min, kk, l), sh3_get(S, kk + j, l + ii), v);
        double rj = 1.0 / rho_c;
        for (int t = 0; t < j; ++t) rj *= ratio;
        acc[h] = caxpy((j & 1) ? -rj : rj, v, acc[h]);
      }
    }
  }
  double2* L = locals + ((size_t)s * nrhs + r) * ncf;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int o = threadIdx.x + h * NT;
    if (o < ncf) L[o] = cadd(L[o], acc[h]);
  }
}

// }}}

// {{{ P2QBXL^T: center multipoles evaluated at the list-1 sources (M2P)

// value += sum_{n <= q} w_m Re(Mc_n^m S_n^m((y - c) / rho)) / rho, w_0 = 1, w_{m>0} = 2,
// the S entries by the column recurrence, one thread per source.
__global__ void __launch_bounds__(NT)
k_tr_p2qbxl(qbxfmm_geometry g, qbxfmm_transpose_index ix, int q, int ncq, int nrhs,
            const double2* __restrict__ cmp, double* __restrict__ vals, int32_t* err)
{
  extern __shared__ double2 smem2[];
  double2* Ms = smem2;                                   // [TR_CB][ncq]
  __shared__ double s_c[TR_CB][4];                       // center, 1 / rho
  int s = ix.list1_rows[blockIdx.x];
  int r = blockIdx.y;
  if (!box_ok(g, s, err)) return;
  int s0 = g.box_source_starts[s], ns = g.box_source_counts_nonchild[s];
  if (s0 < 0 || ns < 0 || s0 + ns > g.nsources) {
    report(err, QBX_DEVERR_BAD_BOX);
    return;
  }
  for (int j0 = 0; j0 < ns; j0 += NT) {
    int j = s0 + j0 + threadIdx.x;
    bool active = j0 + threadIdx.x < ns;
    double y[3] = {0.0, 0.0, 0.0};
    if (active) load_point<3>(g.sources, g.nsources, j, y);
    double acc = 0.0;
    for (int e = ix.list1_rev_starts[blockIdx.x]; e < ix.list1_rev_starts[blockIdx.x + 1]; ++e) {
      int b = ix.list1_rev_lists[e];
      if (!box_ok(g, b, err)) continue;
      int k0 = ix.box_center_starts[b], k1 = ix.box_center_starts[b + 1];
      for (int kb = k0; kb < k1; kb += TR_CB) {
        int nb = min(TR_CB, k1 - kb);
        __syncthreads();
        for (int w = threadIdx.x; w < nb * ncq; w += NT) {
          int ci = w / ncq, i = w - ci * ncq;
          int ctr = ix.box_centers[kb + ci];
          Ms[w] = center_ok(g, ctr, err) ? cmp[((size_t)ctr * nrhs + r) * ncq + i] : c2(0.0);
        }
        if (threadIdx.x < nb) {
          int ctr = ix.box_centers[kb + threadIdx.x];
          double cc[3] = {0.0, 0.0, 0.0};
          double rinv = 0.0;
          if ((unsigned)ctr < (unsigned)g.ncenters) {
            load_point<3>(g.centers, g.ncenters, ctr, cc);
            rinv = 1.0 / g.expansion_radii[ctr];
          }
          s_c[threadIdx.x][0] = cc[0];
          s_c[threadIdx.x][1] = cc[1];
          s_c[threadIdx.x][2] = cc[2];
          s_c[threadIdx.x][3] = rinv;
        }
        __syncthreads();
        if (!active) continue;
        for (int ci = 0; ci < nb; ++ci) {
          double rinv = s_c[ci][3];
          if (rinv == 0.0) continue;
          double ux = (y[0] - s_c[ci][0]) * rinv, uy = (y[1] - s_c[ci][1]) * rinv,
                 uz = (y[2] - s_c[ci][2]) * rinv;
          double rinv2 = 1.0 / (ux * ux + uy * uy + uz * uz);
          const double2* M = Ms + ci * ncq;
          double2 smm = c2(sqrt(rinv2));
          double v = 0.0;
          for (int m = 0; m <= q; ++m) {
            if (m > 0) smm = cscale((2.0 * m - 1) * rinv2, cmul(smm, c2(ux, uy)));
            double2 a = smm, prev = c2(0.0);
            double w = m ? 2.0 : 1.0;
            for (int n = m; n <= q; ++n) {
              if (n > m) {
                double2 bb = cscale(rinv2, csub(cscale((2.0 * n - 1) * uz, a),
                                                cscale((double)(n + m - 1) * (n - m - 1), prev)));
                prev = a;
                a = bb;
              }
              double2 mv = M[idx3(n, m)];
              v += w * (mv.x * a.x - mv.y * a.y);
            }
          }
          acc += v * rinv;
        }
      }
    }
    if (active) vals[(size_t)r * g.nsources + j] += acc;
  }
}

// }}}

// {{{ launchers

cudaError_t launch_tr_qbxl2p(const qbxfmm_geometry& g, int q, int nrhs, double cq,
                             const double* vals, double2* cmp, int32_t* err, cudaStream_t st)
{
  if (g.nglobal_qbx_centers == 0) return cudaSuccess;
  int ncq = idx3(q + 1, 0);
  k_tr_qbxl2p<<<dim3(g.nglobal_qbx_centers, nrhs), 64, ncq * sizeof(double2), st>>>(
      g, q, ncq, nrhs, cq, vals, cmp, err);
  return cudaGetLastError();
}

cudaError_t launch_tr_l2qbxl(const qbxfmm_geometry& g, const qbxfmm_transpose_index& ix, int p,
                             int q, int nrhs, const double2* cmp, double2* mpoles, int32_t* err,
                             cudaStream_t st)
{
  if (ix.ncenter_boxes == 0) return cudaSuccess;
  int ncf = idx3(p + 1, 0), ncq = idx3(q + 1, 0);
  k_tr_l2qbxl<<<dim3(ix.ncenter_boxes, nrhs), NT, (ncf + ncq) * sizeof(double2), st>>>(
      g, ix, p, q, ncf, ncq, nrhs, cmp, mpoles, err);
  return cudaGetLastError();
}

cudaError_t launch_tr_m2qbxl(const qbxfmm_geometry& g, const qbxfmm_transpose_index& ix, int p,
                             int q, int nrhs, const double2* cmp, double2* locals, int32_t* err,
                             cudaStream_t st)
{
  if (ix.nlist3_rows == 0) return cudaSuccess;
  int ncf = idx3(p + 1, 0), ncq = idx3(q + 1, 0), nS = idx3(p + q + 1, 0);
  k_tr_m2qbxl<<<dim3(ix.nlist3_rows, nrhs), NT, (nS + ncq) * sizeof(double2), st>>>(
      g, ix, p, q, ncf, ncq, nrhs, cmp, locals, err);
  return cudaGetLastError();
}

cudaError_t launch_tr_p2qbxl(const qbxfmm_geometry& g, const qbxfmm_transpose_index& ix, int q,
                             int nrhs, const double2* cmp, double* vals, int32_t* err,
                             cudaStream_t st)
{
  if (ix.nlist1_rows == 0) return cudaSuccess;
  int ncq = idx3(q + 1, 0);
  size_t sh = (size_t)TR_CB * ncq * sizeof(double2);
  cudaError_t e = cudaFuncSetAttribute(k_tr_p2qbxl, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sh);
  if (e != cudaSuccess) return e;
  k_tr_p2qbxl<<<dim3(ix.nlist1_rows, nrhs), NT, sh, st>>>(g, ix, q, ncq, nrhs, cmp, vals, err);
  return cudaGetLastError();
}

// }}}

}  // namespace qbx
