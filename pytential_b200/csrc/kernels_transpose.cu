// Transposed QBX stages of the Laplace apply (3D single and double layer, 2D single
// layer), sm_100a.
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
//   k_tr_tsqbx    transpose of P2QBXL (fmm.py:231-265): per source box s, the
//                 (target, center) pairs of every center box whose list 1 holds s,
//                 evaluated at the sources of s in the target-specific form (the
//                 Legendre sum of the truncated expansion, symmetric in the roles),
//                 and for a dipole layer its gradient in the source position
//   k_tr_combine  cq value + cd normal . gradient at the sources (charge + dipole)
//
// Each output (a box expansion, a source value) has one writer: the kernels gather
// over the reversed lists of qbxfmm_transpose_index (M2QBXL^T and P2QBXL^T, when the
// rows are too few to fill the GPU, with a cluster of TR_CL CTAs per row whose partial
// sums rank 0 adds in rank order through distributed shared memory), so results do not
// depend on scheduling.  The box stages of the transpose are the library's own P2M / M2M /
// M2L / M2P / P2L / L2L / L2P / P2P on the exchanged-role geometry.
#include "laplace.cuh"
#include "kernels.h"

#include <algorithm>

#include <cooperative_groups.h>
namespace cg = cooperative_groups;

namespace qbx {

namespace {

constexpr int NT = 128;
constexpr int TR_CL = 8;      // CTAs per row (a cluster) in M2QBXL^T and P2QBXL^T when
                              // the rows alone would not fill the GPU
constexpr int TR_SPLIT_BELOW = 4 * 148;   // rows below which a row is split
// M2QBXL^T: threads per CTA and accumulation tasks per thread (2 ncf <= TRM_H TRM_NT:
// each output coefficient is split over the even and odd centers of a batch; fmm_order
// <= 21)
constexpr int TRM_NT = 192;
constexpr int TRM_H = 3;

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
// d = (center - box center) / rho_b: the entries of the box-to-center L2L.  Batches of
// mb centers per barrier (one table column task per thread): their R tables (rows
// 0..p, columns -q..p+q: the sums reach m - l up to p + q, zero beyond the row) and
// multipoles (rows 0..q, columns -q..q) expanded into zero-padded dense arrays, so
// the inner sums are branch-free.
__global__ void __launch_bounds__(NT)
k_tr_l2qbxl(qbxfmm_geometry g, qbxfmm_transpose_index ix, int p, int q, int ncf, int ncq,
            int nrhs, int mb, const double2* __restrict__ cmp, double2* __restrict__ mpoles,
            int32_t* err)
{
  extern __shared__ double2 smem2[];
  const int RW = p + 2 * q + 1, RS = (p + 1) * RW;    // R table: rows 0..p, columns -q..p+q
  const int MW = 2 * q + 1, MS = (q + 1) * MW;        // center multipole
  double2* R = smem2;                                 // [mb][RS]
  double2* Mp = R + (size_t)mb * RS;                  // [mb][MS]
  double* rk = reinterpret_cast<double*>(Mp + (size_t)mb * MS);   // [mb][q + 1]
  double* sd = rk + (size_t)mb * (q + 1);                          // [mb][3]
  int* sctr = reinterpret_cast<int*>(sd + (size_t)mb * 3);         // [mb]
  int b = ix.center_boxes[blockIdx.x];
  int r = blockIdx.y;
  if (!box_ok(g, b, err)) return;
  double rho_b = level_width(g, g.box_levels[b]);
  double cb[3];
  load_point<3>(g.box_centers, g.nboxes, b, cb);
  // the entries outside |m| <= n stay zero for every center
  for (int i = threadIdx.x; i < mb * (RS + MS); i += NT) R[i] = c2(0.0);
  double2 acc[2] = {c2(0.0), c2(0.0)};
  int k0 = ix.box_center_starts[b], k1 = ix.box_center_starts[b + 1];
  for (int kb = k0; kb < k1; kb += mb) {
    int nb = min(mb, k1 - kb);
    __syncthreads();
    if (threadIdx.x < nb) {
      int ctr = ix.box_centers[kb + threadIdx.x];
      bool ok = center_ok(g, ctr, err);
      double cc[3] = {cb[0], cb[1], cb[2]};
      double rho_c = rho_b;
      if (ok) {
        load_point<3>(g.centers, g.ncenters, ctr, cc);
        rho_c = g.expansion_radii[ctr];
      }
      sctr[threadIdx.x] = ok ? ctr : -1;
      for (int d = 0; d < 3; ++d) sd[threadIdx.x * 3 + d] = (cc[d] - cb[d]) / rho_b;
      double ratio = rho_c / rho_b, f = 1.0;
      for (int kk = 0; kk <= q; ++kk, f *= ratio) rk[threadIdx.x * (q + 1) + kk] = f;
    }
    __syncthreads();
    // R columns m = 0..p (negative columns down to -q by symmetry)
    for (int w = threadIdx.x; w < nb * (p + 1); w += NT) {
      int ci = w / (p + 1), m = w - ci * (p + 1);
      double x = sd[ci * 3], y = sd[ci * 3 + 1], z = sd[ci * 3 + 2];
      double r2 = x * x + y * y + z * z;
      double2 a = c2(1.0);
      for (int jj = 1; jj <= m; ++jj) a = cscale(0.5 * rcp(jj), cmul(a, c2(x, y)));
      double2 prev = c2(0.0);
      double2* T = R + (size_t)ci * RS + q;
      for (int n = m; n <= p; ++n) {
        if (n > m) {
          double2 bb = cscale(rcp(n + m) * rcp(n - m),
                              csub(cscale((2.0 * n - 1) * z, a), cscale(r2, prev)));
          prev = a;
          a = bb;
        }
        T[n * RW + m] = a;
        if (m >= 1 && m <= q) T[n * RW - m] = (m & 1) ? c2(-a.x, a.y) : c2(a.x, -a.y);
      }
    }
    for (int w = threadIdx.x; w < nb * ncq; w += NT) {
      int ci = w / ncq, i = w - ci * ncq;
      int ctr = sctr[ci];
      int kk, l;
      decode3(i, kk, l);
      double2 v = ctr >= 0 ? cmp[((size_t)ctr * nrhs + r) * ncq + i] : c2(0.0);
      double2* M = Mp + (size_t)ci * MS + q;
      M[kk * MW + l] = v;
      if (l > 0) M[kk * MW - l] = (l & 1) ? c2(-v.x, v.y) : c2(v.x, -v.y);
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      int o = threadIdx.x + h * NT;
      if (o >= ncf) break;
      int n, m;
      decode3(o, n, m);
      double2 a = acc[h];
      int kmax = n < q ? n : q;
      for (int ci = 0; ci < nb; ++ci) {
        const double2* M = Mp + (size_t)ci * MS + q;
        const double2* T = R + (size_t)ci * RS + q;
        for (int kk = 0; kk <= kmax; ++kk) {
          double2 v = c2(0.0);
          const double2* mrow = M + kk * MW;
          const double2* trow = T + (n - kk) * RW + m;
          for (int l = -kk; l <= kk; ++l) v = cfmac(mrow[l], trow[-l], v);
          a = caxpy(rk[ci * (q + 1) + kk], v, a);
        }
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
// Batches of mb centers per barrier (one S column task per thread): their S tables
// (rows 0..p+q, columns -q..p+q), multipoles (rows 0..q, columns -q..q) and
// (-1)^j ratio^j / rho_c factors in zero-padded dense shared arrays, so the inner
// sums are branch-free.
template <int CL>
__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(TRM_NT, 3)
k_tr_m2qbxl(qbxfmm_geometry g, qbxfmm_transpose_index ix, int p, int q, int ncf, int ncq,
            int nrhs, int mb, const double2* __restrict__ cmp, double2* __restrict__ locals,
            int32_t* err)
{
  const int row = blockIdx.x / CL, part = blockIdx.x - row * CL;
  extern __shared__ double2 smem2[];
  const int SW = p + 2 * q + 1, SS = (p + q + 1) * SW;   // S: rows 0..p+q, columns -q..p+q
  const int MW = 2 * q + 1, MS = (q + 1) * MW;
  double2* S = smem2;                                    // [mb][SS]
  double2* Mp = S + (size_t)mb * SS;                     // [mb][MS]
  double* fac = reinterpret_cast<double*>(Mp + (size_t)mb * MS);   // [mb][p + 1]
  double* sd = fac + (size_t)mb * (p + 1);                          // [mb][3]
  int* sctr = reinterpret_cast<int*>(sd + (size_t)mb * 3);          // [mb]
  int s = ix.list3_rows[row];
  int r = blockIdx.y;
  if (!box_ok(g, s, err)) return;          // the whole cluster (one row) leaves
  double rho_s = level_width(g, g.box_levels[s]);
  double cs[3];
  load_point<3>(g.box_centers, g.nboxes, s, cs);
  for (int i = threadIdx.x; i < mb * (SS + MS); i += TRM_NT) S[i] = c2(0.0);
  double2 acc[TRM_H];
#pragma unroll
  for (int h = 0; h < TRM_H; ++h) acc[h] = c2(0.0);
  int item = 0;                            // center batches dealt round-robin to the cluster
  for (int e = ix.list3_rev_starts[row]; e < ix.list3_rev_starts[row + 1]; ++e) {
    int b = ix.list3_rev_lists[e];
    if (!box_ok(g, b, err)) continue;
    int k0 = ix.box_center_starts[b], k1 = ix.box_center_starts[b + 1];
    for (int kb = k0; kb < k1; kb += mb) {
      if (item++ % CL != part) continue;
      int nb = min(mb, k1 - kb);
      __syncthreads();
      if (threadIdx.x < nb) {
        int ctr = ix.box_centers[kb + threadIdx.x];
        bool ok = center_ok(g, ctr, err);
        // a bad center contributes nothing: a unit vector for its table, zero factors
        double cc[3] = {cs[0] - 1.0, cs[1], cs[2]};
        double rho_c = 1.0;
        if (ok) {
          load_point<3>(g.centers, g.ncenters, ctr, cc);
          rho_c = g.expansion_radii[ctr];
        }
        sctr[threadIdx.x] = ok ? ctr : -1;
        for (int d = 0; d < 3; ++d) sd[threadIdx.x * 3 + d] = (cs[d] - cc[d]) / rho_c;
        double ratio = rho_s / rho_c, f = ok ? 1.0 / rho_c : 0.0;
        for (int j = 0; j <= p; ++j, f *= -ratio) fac[threadIdx.x * (p + 1) + j] = f;
      }
      __syncthreads();
      for (int w = threadIdx.x; w < nb * (p + q + 1); w += TRM_NT) {
        int ci = w / (p + q + 1), m = w - ci * (p + q + 1);
        double x = sd[ci * 3], y = sd[ci * 3 + 1], z = sd[ci * 3 + 2];
        double rinv2 = 1.0 / (x * x + y * y + z * z);
        double2 a = c2(sqrt(rinv2));
        for (int jj = 1; jj <= m; ++jj) a = cscale((2.0 * jj - 1) * rinv2, cmul(a, c2(x, y)));
        double2 prev = c2(0.0);
        double2* T = S + (size_t)ci * SS + q;
        for (int n = m; n <= p + q; ++n) {
          if (n > m) {
            double2 bb = cscale(rinv2, csub(cscale((2.0 * n - 1) * z, a),
                                            cscale((double)(n + m - 1) * (n - m - 1), prev)));
            prev = a;
            a = bb;
          }
          T[n * SW + m] = a;
          if (m >= 1 && m <= q) T[n * SW - m] = (m & 1) ? c2(-a.x, a.y) : c2(a.x, -a.y);
        }
      }
      for (int w = threadIdx.x; w < nb * ncq; w += TRM_NT) {
        int ci = w / ncq, i = w - ci * ncq;
        int ctr = sctr[ci];
        int kk, l;
        decode3(i, kk, l);
        double2 v = ctr >= 0 ? cmp[((size_t)ctr * nrhs + r) * ncq + i] : c2(0.0);
        double2* M = Mp + (size_t)ci * MS + q;
        M[kk * MW + l] = v;
        if (l > 0) M[kk * MW - l] = (l & 1) ? c2(-v.x, v.y) : c2(v.x, -v.y);
      }
      __syncthreads();
      // task t = (half, o): output coefficient o over the batch's centers of one parity
#pragma unroll
      for (int h = 0; h < TRM_H; ++h) {
        const int t = threadIdx.x + h * TRM_NT;
        if (t >= 2 * ncf) break;
        const int half = t >= ncf ? 1 : 0, o = t - half * ncf;
        int j, ii;
        decode3(o, j, ii);
        double2 a = acc[h];
        for (int ci = half; ci < nb; ci += 2) {
          const double2* M = Mp + (size_t)ci * MS + q;
          const double2* T = S + (size_t)ci * SS + q;
          double2 v = c2(0.0);
          for (int kk = 0; kk <= q; ++kk) {
            const double2* mrow = M + kk * MW;
            const double2* trow = T + (kk + j) * SW + ii;
            for (int l = -kk; l <= kk; ++l) v = cfma(mrow[l], trow[l], v);
          }
          a = caxpy(fac[ci * (p + 1) + j], v, a);
        }
        acc[h] = a;
      }
    }
  }
  // the two halves of each coefficient, then the cluster's CTAs, summed by rank 0 in a
  // fixed order (distributed shared memory); the partials [2][ncf] reuse the tables'
  // space (mb (SS + MS) >= 2 ncf for mb >= 2)
  cg::cluster_group cl = cg::this_cluster();
  double2* s_part = smem2;
  __syncthreads();
#pragma unroll
  for (int h = 0; h < TRM_H; ++h) {
    const int t = threadIdx.x + h * TRM_NT;
    if (t < 2 * ncf) s_part[t] = acc[h];
  }
  cl.sync();
  if (part == 0) {
    double2* L = locals + ((size_t)s * nrhs + r) * ncf;
    for (int o = threadIdx.x; o < ncf; o += TRM_NT) {
      double2 v = cadd(s_part[o], s_part[o + ncf]);
      for (int qq = 1; qq < CL; ++qq) {
        const double2* rp = cl.map_shared_rank(s_part, qq);
        v = cadd(v, cadd(rp[o], rp[o + ncf]));
      }
      L[o] = cadd(L[o], v);
    }
  }
  cl.sync();
}

// }}}

// {{{ P2QBXL^T: the list-1 sources' values from the QBX targets (target-specific form)

// For a QBX target t with center c and a source y in the list 1 of the center's box,
// a = t - c, b = y - c: the P2QBXL + QBXL2P entry (the QBX local of order Q formed
// from y, evaluated at t) is sum_{n <= Q} |a|^n / |b|^{n+1} P_n(cos g),
// cos g = a.b / (|a||b|) -- symmetric in the roles, so the transpose adds
// cq r_t times it to the value at y.  Equal to evaluating the center multipoles of
// k_tr_qbxl2p at y (the addition theorem), without forming them.  CTA = one source
// box of some center box's list 1; each thread holds up to TR_KS of its sources;
// the (target, center) pairs of the boxes that list it are staged TR_PB at a time.
constexpr int TR_KS = 4;
constexpr int TR_PB = NT;

template <int Q, bool DIP, int CL>
__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(NT)
k_tr_tsqbx(qbxfmm_geometry g, qbxfmm_transpose_index ix, int nrhs, double cq,
           const double* __restrict__ tvals, double* __restrict__ vals,
           double* __restrict__ grads, int32_t* err)
{
  __shared__ double s_c[3][TR_PB], s_ah[3][TR_PB], s_al[TR_PB], s_w[TR_PB];
  __shared__ double s_part[TR_KS][DIP ? 4 : 1][NT];
  const int row = blockIdx.x / CL, part = blockIdx.x - row * CL;
  cg::cluster_group cl = cg::this_cluster();
  int s = ix.list1_rows[row];
  int r = blockIdx.y;
  if (!box_ok(g, s, err)) return;
  int s0 = g.box_source_starts[s], ns = g.box_source_counts_nonchild[s];
  if (s0 < 0 || ns < 0 || s0 + ns > g.nsources) {
    report(err, QBX_DEVERR_BAD_BOX);
    return;
  }
  const double* tv = tvals + (size_t)r * g.ntargets;
  for (int g0 = 0; g0 < ns; g0 += NT * TR_KS) {
    double y[TR_KS][3], acc[TR_KS], gacc[DIP ? TR_KS : 1][3];
#pragma unroll
    for (int k = 0; k < TR_KS; ++k) {
      int jj = g0 + threadIdx.x + k * NT;
      acc[k] = 0.0;
      if (DIP) gacc[DIP ? k : 0][0] = gacc[DIP ? k : 0][1] = gacc[DIP ? k : 0][2] = 0.0;
      if (jj < ns) load_point<3>(g.sources, g.nsources, s0 + jj, y[k]);
      else y[k][0] = y[k][1] = y[k][2] = 0.0;
    }
    int item = 0;                          // pair batches dealt round-robin to the cluster
    for (int e = ix.list1_rev_starts[row]; e < ix.list1_rev_starts[row + 1]; ++e) {
      int b = ix.list1_rev_lists[e];
      if (!box_ok(g, b, err)) continue;
      int p0 = ix.box_pair_starts[b], p1 = ix.box_pair_starts[b + 1];
      for (int pb = p0; pb < p1; pb += TR_PB) {
        if (item++ % CL != part) continue;
        int np = min(TR_PB, p1 - pb);
        __syncthreads();
        if (threadIdx.x < np) {
          int t = ix.pair_targets[pb + threadIdx.x], ctr = ix.pair_centers[pb + threadIdx.x];
          double w = 0.0, cc[3] = {0.0, 0.0, 0.0}, a[3] = {0.0, 0.0, 0.0};
          if ((unsigned)t < (unsigned)g.ntargets && center_ok(g, ctr, err)) {
            double x[3];
            load_point<3>(g.centers, g.ncenters, ctr, cc);
            load_point<3>(g.targets, g.ntargets, t, x);
            for (int d = 0; d < 3; ++d) a[d] = x[d] - cc[d];
            w = cq * tv[t];
          } else if ((unsigned)t >= (unsigned)g.ntargets) {
            report(err, QBX_DEVERR_BAD_CENTER);
          }
          double al = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
          double ainv = al > 0.0 ? 1.0 / al : 0.0;
          for (int d = 0; d < 3; ++d) {
            s_c[d][threadIdx.x] = cc[d];
            s_ah[d][threadIdx.x] = a[d] * ainv;
          }
          s_al[threadIdx.x] = al;
          s_w[threadIdx.x] = w;
        }
        __syncthreads();
        for (int pi = 0; pi < np; ++pi) {
          double w = s_w[pi];
          if (w == 0.0) continue;
          double cx = s_c[0][pi], cy = s_c[1][pi], cz = s_c[2][pi];
          double hx = s_ah[0][pi], hy = s_ah[1][pi], hz = s_ah[2][pi], al = s_al[pi];
#pragma unroll
          for (int k = 0; k < TR_KS; ++k) {
            if (g0 + threadIdx.x + k * NT >= ns) break;
            double b0 = y[k][0] - cx, b1 = y[k][1] - cy, b2 = y[k][2] - cz;
            double binv = rsqrt(b0 * b0 + b1 * b1 + b2 * b2);
            double cg = (hx * b0 + hy * b1 + hz * b2) * binv;
            double ratio = al * binv;
            double pm1 = 1.0, pm2 = 0.0, dm1 = 0.0, rn = binv, sum = 0.0, sa = 0.0, sb = 0.0;
#pragma unroll
            for (int n = 0; n <= Q; ++n) {
              double pn = n == 0 ? 1.0
                        : n == 1 ? cg
                                 : ((2.0 * n - 1) * cg * pm1 - (n - 1.0) * pm2) * (1.0 / n);
              sum = fma(rn, pn, sum);
              if (DIP) {
                double dn = n == 0 ? 0.0 : n * pm1 + cg * dm1;
                sa = fma(-(n + 1.0) * rn, pn, sa);
                sb = fma(rn, dn, sb);
                dm1 = dn;
              }
              pm2 = pm1;
              pm1 = pn;
              rn *= ratio;
            }
            acc[k] = fma(w, sum, acc[k]);
            if (DIP) {
              // grad_b K = (sa b^ + sb (a^ - cos g b^)) / |b|
              double fb = w * binv * (sa - sb * cg), fa = w * binv * sb;
              gacc[DIP ? k : 0][0] += fb * b0 * binv + fa * hx;
              gacc[DIP ? k : 0][1] += fb * b1 * binv + fa * hy;
              gacc[DIP ? k : 0][2] += fb * b2 * binv + fa * hz;
            }
          }
        }
      }
    }
    // the cluster's partial sums for these sources, added by rank 0 in rank order
#pragma unroll
    for (int k = 0; k < TR_KS; ++k) {
      s_part[k][0][threadIdx.x] = acc[k];
      if (DIP)
        for (int d = 0; d < 3; ++d) s_part[k][DIP ? d + 1 : 0][threadIdx.x] = gacc[DIP ? k : 0][d];
    }
    cl.sync();
    if (part == 0) {
#pragma unroll
      for (int k = 0; k < TR_KS; ++k) {
        int jj = g0 + threadIdx.x + k * NT;
        if (jj >= ns) continue;
        double v = acc[k], gv[3] = {0.0, 0.0, 0.0};
        if (DIP)
          for (int d = 0; d < 3; ++d) gv[d] = gacc[DIP ? k : 0][d];
        for (int qq = 1; qq < CL; ++qq) {
          const double* rp = &cl.map_shared_rank(&s_part[0][0][0], qq)[0];
          v += rp[(k * (DIP ? 4 : 1)) * NT + threadIdx.x];
          if (DIP)
            for (int d = 0; d < 3; ++d) gv[d] += rp[(k * 4 + d + 1) * NT + threadIdx.x];
        }
        vals[(size_t)r * g.nsources + s0 + jj] += v;
        if (DIP) {
          double* gr = grads + (size_t)r * 3 * g.nsources + s0 + jj;
          gr[0] += gv[0];
          gr[g.nsources] += gv[1];
          gr[2 * (size_t)g.nsources] += gv[2];
        }
      }
    }
    cl.sync();
  }
}

// }}}

// {{{ 2D Laplace: the same four stages in the complex-analytic expansions
//   multipole  Re[M_0 log(z - c) + sum_k M_k ((z - c) / rho)^-k],
//   local      Re sum_k L_k ((z - c) / rho)^k

QBX_D double2 cdiv(double2 a, double2 b)
{
  double d = 1.0 / (b.x * b.x + b.y * b.y);
  return c2((a.x * b.x + a.y * b.y) * d, (a.y * b.x - a.x * b.y) * d);
}

// QBXL2P^T: per (global center, density) one thread, M_0 = cq sum r_t,
// M_k = -cq sum r_t u_t^k / k, u_t = (x_t - c) / rho
__global__ void __launch_bounds__(NT)
k_tr2_qbxl2p(qbxfmm_geometry g, int q, int nrhs, double cq, const double* __restrict__ vals,
             double2* __restrict__ cmp, int32_t* err)
{
  int ig = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (ig >= g.nglobal_qbx_centers) return;
  int ctr = g.global_qbx_centers[ig];
  if (!center_ok(g, ctr, err)) return;
  double cc[2];
  load_point<2>(g.centers, g.ncenters, ctr, cc);
  double rinv = 1.0 / g.expansion_radii[ctr];
  double2* M = cmp + ((size_t)ctr * nrhs + r) * (q + 1);
  for (int k = 0; k <= q; ++k) M[k] = c2(0.0);
  for (int it = g.center_to_targets_starts[ctr]; it < g.center_to_targets_starts[ctr + 1]; ++it) {
    int t = g.center_to_targets_lists[it];
    if ((unsigned)t >= (unsigned)g.ntargets) {
      report(err, QBX_DEVERR_BAD_CENTER);
      continue;
    }
    double x[2];
    load_point<2>(g.targets, g.ntargets, t, x);
    double v = cq * vals[(size_t)r * g.ntargets + t];
    double2 u = c2((x[0] - cc[0]) * rinv, (x[1] - cc[1]) * rinv), uk = u;
    M[0] = cadd(M[0], c2(v));
    for (int k = 1; k <= q; ++k) {
      M[k] = caxpy(-v * rcp(k), uk, M[k]);
      uk = cmul(uk, u);
    }
  }
}

// L2QBXL^T: per (center box, density), thread = output coefficient l <= p: the M2M of
// each center multipole (order q) to the box center
__global__ void __launch_bounds__(32)
k_tr2_l2qbxl(qbxfmm_geometry g, qbxfmm_transpose_index ix, int p, int q, int nrhs,
             const double2* __restrict__ cmp, double2* __restrict__ mpoles, int32_t* err)
{
  int b = ix.center_boxes[blockIdx.x];
  int r = blockIdx.y, l = threadIdx.x;
  if (!box_ok(g, b, err) || l > p) return;
  double rho_b = level_width(g, g.box_levels[b]);
  double cb[2];
  load_point<2>(g.box_centers, g.nboxes, b, cb);
  double2 acc = c2(0.0);
  for (int kk = ix.box_center_starts[b]; kk < ix.box_center_starts[b + 1]; ++kk) {
    int ctr = ix.box_centers[kk];
    if (!center_ok(g, ctr, err)) continue;
    double cc[2];
    load_point<2>(g.centers, g.ncenters, ctr, cc);
    double ratio = g.expansion_radii[ctr] / rho_b;
    double2 t = c2((cc[0] - cb[0]) / rho_b, (cc[1] - cb[1]) / rho_b);
    const double2* Min = cmp + ((size_t)ctr * nrhs + r) * (q + 1);
    if (l == 0) {
      acc = cadd(acc, Min[0]);
      continue;
    }
    double2 tp[24];                        // t^i, i <= l <= p <= 20
    tp[0] = c2(1.0);
    for (int i = 1; i <= l; ++i) tp[i] = cmul(tp[i - 1], t);
    acc = cfma(cscale(-rcp(l), Min[0]), tp[l], acc);
    double rk = ratio, bin = 1.0;          // C(l - 1, k - 1)
    for (int k = 1; k <= l && k <= q; ++k) {
      acc = cfma(cscale(rk * bin, Min[k]), tp[l - k], acc);
      rk *= ratio;
      bin = bin * (l - k) * rcp(k);
    }
  }
  double2* M = mpoles + ((size_t)b * nrhs + r) * (p + 1);
  M[l] = cadd(M[l], acc);
}

// M2QBXL^T: per (list-3 row s, density), thread = output coefficient l <= p: the M2L of
// each center multipole (order q, rscale rho_c) into the local of s (rscale rho_s)
__global__ void __launch_bounds__(32)
k_tr2_m2qbxl(qbxfmm_geometry g, qbxfmm_transpose_index ix, int p, int q, int nrhs,
             const double2* __restrict__ cmp, double2* __restrict__ locals, int32_t* err)
{
  int s = ix.list3_rows[blockIdx.x];
  int r = blockIdx.y, l = threadIdx.x;
  if (!box_ok(g, s, err) || l > p) return;
  double rho_s = level_width(g, g.box_levels[s]);
  double cs[2];
  load_point<2>(g.box_centers, g.nboxes, s, cs);
  double2 acc = c2(0.0);
  for (int e = ix.list3_rev_starts[blockIdx.x]; e < ix.list3_rev_starts[blockIdx.x + 1]; ++e) {
    int b = ix.list3_rev_lists[e];
    if (!box_ok(g, b, err)) continue;
    for (int kk = ix.box_center_starts[b]; kk < ix.box_center_starts[b + 1]; ++kk) {
      int ctr = ix.box_centers[kk];
      if (!center_ok(g, ctr, err)) continue;
      double cc[2];
      load_point<2>(g.centers, g.ncenters, ctr, cc);
      double rho_c = g.expansion_radii[ctr];
      double2 t = c2(cs[0] - cc[0], cs[1] - cc[1]);
      double2 tinv = cdiv(c2(1.0), cscale(1.0 / rho_c, t));
      const double2* Min = cmp + ((size_t)ctr * nrhs + r) * (q + 1);
      if (l == 0) {
        double2 v = cmul(Min[0], c2(0.5 * log(t.x * t.x + t.y * t.y), atan2(t.y, t.x)));
        double2 pw = tinv;
        for (int k = 1; k <= q; ++k) {
          v = cfma(Min[k], pw, v);
          pw = cmul(pw, tinv);
        }
        acc = cadd(acc, v);
        continue;
      }
      double2 tl = c2(1.0);
      for (int i = 0; i < l; ++i) tl = cmul(tl, tinv);
      double2 v = cscale(((l & 1) ? 1.0 : -1.0) * rcp(l), cmul(Min[0], tl));
      double2 sm = c2(0.0), pw = tinv;
      double bin = 1.0;                     // C(k + l - 1, l), 1 at k = 1
      for (int k = 1; k <= q; ++k) {
        sm = cfma(cscale(bin, Min[k]), pw, sm);
        pw = cmul(pw, tinv);
        bin = bin * (k + l) * rcp(k);       // C(k + l, l) = C(k + l - 1, l) (k + l) / k
      }
      v = cfma(cscale((l & 1) ? -1.0 : 1.0, tl), sm, v);
      double rl = 1.0, ratio = rho_s / rho_c;
      for (int i = 0; i < l; ++i) rl *= ratio;
      acc = caxpy(rl, v, acc);
    }
  }
  double2* L = locals + ((size_t)s * nrhs + r) * (p + 1);
  L[l] = cadd(L[l], acc);
}

// P2QBXL^T with QBXL2P^T, target-specific form: for a QBX target t with center c and a
// list-1 source y, a = t - c, b = y - c: log|t - y| ~ log|b| - Re sum_{n=1..Q} (a/b)^n / n
// (symmetric in the roles); per (source box row, density), thread = source
template <int Q>
__global__ void __launch_bounds__(NT)
k_tr2_tsqbx(qbxfmm_geometry g, qbxfmm_transpose_index ix, int nrhs, double cq,
            const double* __restrict__ tvals, double* __restrict__ vals, int32_t* err)
{
  __shared__ double s_c[2][NT], s_a[2][NT], s_w[NT];
  int s = ix.list1_rows[blockIdx.x];
  int r = blockIdx.y;
  if (!box_ok(g, s, err)) return;
  int s0 = g.box_source_starts[s], ns = g.box_source_counts_nonchild[s];
  if (s0 < 0 || ns < 0 || s0 + ns > g.nsources) {
    report(err, QBX_DEVERR_BAD_BOX);
    return;
  }
  const double* tv = tvals + (size_t)r * g.ntargets;
  for (int j0 = 0; j0 < ns; j0 += NT) {
    int j = s0 + j0 + threadIdx.x;
    bool active = j0 + threadIdx.x < ns;
    double y[2] = {0.0, 0.0};
    if (active) load_point<2>(g.sources, g.nsources, j, y);
    double acc = 0.0;
    for (int e = ix.list1_rev_starts[blockIdx.x]; e < ix.list1_rev_starts[blockIdx.x + 1]; ++e) {
      int b = ix.list1_rev_lists[e];
      if (!box_ok(g, b, err)) continue;
      int p0 = ix.box_pair_starts[b], p1 = ix.box_pair_starts[b + 1];
      for (int pb = p0; pb < p1; pb += NT) {
        int np = min(NT, p1 - pb);
        __syncthreads();
        if (threadIdx.x < np) {
          int t = ix.pair_targets[pb + threadIdx.x], ctr = ix.pair_centers[pb + threadIdx.x];
          double w = 0.0, cc[2] = {0.0, 0.0}, a[2] = {0.0, 0.0};
          if ((unsigned)t < (unsigned)g.ntargets && center_ok(g, ctr, err)) {
            double x[2];
            load_point<2>(g.centers, g.ncenters, ctr, cc);
            load_point<2>(g.targets, g.ntargets, t, x);
            a[0] = x[0] - cc[0];
            a[1] = x[1] - cc[1];
            w = cq * tv[t];
          } else if ((unsigned)t >= (unsigned)g.ntargets) {
            report(err, QBX_DEVERR_BAD_CENTER);
          }
          s_c[0][threadIdx.x] = cc[0];
          s_c[1][threadIdx.x] = cc[1];
          s_a[0][threadIdx.x] = a[0];
          s_a[1][threadIdx.x] = a[1];
          s_w[threadIdx.x] = w;
        }
        __syncthreads();
        if (!active) continue;
        for (int pi = 0; pi < np; ++pi) {
          double w = s_w[pi];
          if (w == 0.0) continue;
          double2 bb = c2(y[0] - s_c[0][pi], y[1] - s_c[1][pi]);
          double2 wv = cdiv(c2(s_a[0][pi], s_a[1][pi]), bb), pw = wv;
          double sl = 0.0;
#pragma unroll
          for (int n = 1; n <= Q; ++n) {
            sl += pw.x * (1.0 / n);
            pw = cmul(pw, wv);
          }
          acc = fma(w, 0.5 * log(bb.x * bb.x + bb.y * bb.y) - sl, acc);
        }
      }
    }
    if (active) vals[(size_t)r * g.nsources + j] += acc;
  }
}

template <int Q>
static cudaError_t tr2_tsqbx_q(const qbxfmm_geometry& g, const qbxfmm_transpose_index& ix,
                               int nrhs, double cq, const double* tvals, double* vals,
                               int32_t* err, cudaStream_t st)
{
  k_tr2_tsqbx<Q><<<dim3(ix.nlist1_rows, nrhs), NT, 0, st>>>(g, ix, nrhs, cq, tvals, vals, err);
  return cudaGetLastError();
}

cudaError_t launch_tr2_stages(int which, const qbxfmm_geometry& g, const qbxfmm_transpose_index* ix,
                              int p, int q, int nrhs, double cq, const double* tvals,
                              double2* cmp, double2* box_exps, double* vals, int32_t* err,
                              cudaStream_t st)
{
  if (p > 20 || q > 8) return cudaErrorInvalidValue;
  switch (which) {
    case 0:   // QBXL2P^T
      if (g.nglobal_qbx_centers == 0) return cudaSuccess;
      k_tr2_qbxl2p<<<dim3((g.nglobal_qbx_centers + NT - 1) / NT, nrhs), NT, 0, st>>>(
          g, q, nrhs, cq, tvals, cmp, err);
      return cudaGetLastError();
    case 1:   // L2QBXL^T
      if (ix->ncenter_boxes == 0) return cudaSuccess;
      k_tr2_l2qbxl<<<dim3(ix->ncenter_boxes, nrhs), 32, 0, st>>>(g, *ix, p, q, nrhs, cmp,
                                                                  box_exps, err);
      return cudaGetLastError();
    case 2:   // M2QBXL^T
      if (ix->nlist3_rows == 0) return cudaSuccess;
      k_tr2_m2qbxl<<<dim3(ix->nlist3_rows, nrhs), 32, 0, st>>>(g, *ix, p, q, nrhs, cmp, box_exps,
                                                                err);
      return cudaGetLastError();
    case 3:   // P2QBXL^T with QBXL2P^T
      if (ix->nlist1_rows == 0) return cudaSuccess;
      switch (q) {
        case 0: return tr2_tsqbx_q<0>(g, *ix, nrhs, cq, tvals, vals, err, st);
        case 1: return tr2_tsqbx_q<1>(g, *ix, nrhs, cq, tvals, vals, err, st);
        case 2: return tr2_tsqbx_q<2>(g, *ix, nrhs, cq, tvals, vals, err, st);
        case 3: return tr2_tsqbx_q<3>(g, *ix, nrhs, cq, tvals, vals, err, st);
        case 4: return tr2_tsqbx_q<4>(g, *ix, nrhs, cq, tvals, vals, err, st);
        case 5: return tr2_tsqbx_q<5>(g, *ix, nrhs, cq, tvals, vals, err, st);
        case 6: return tr2_tsqbx_q<6>(g, *ix, nrhs, cq, tvals, vals, err, st);
        case 7: return tr2_tsqbx_q<7>(g, *ix, nrhs, cq, tvals, vals, err, st);
        case 8: return tr2_tsqbx_q<8>(g, *ix, nrhs, cq, tvals, vals, err, st);
        default: return cudaErrorInvalidValue;
      }
    default: return cudaErrorInvalidValue;
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
  int mb = std::max(1, std::min(8, NT / (p + 1)));
  size_t sh = (size_t)mb * ((p + 1) * (p + 2 * q + 1) + (q + 1) * (2 * q + 1)) * sizeof(double2) +
              (size_t)mb * (q + 4) * sizeof(double) + (size_t)mb * sizeof(int);
  cudaError_t e = cudaFuncSetAttribute(k_tr_l2qbxl, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sh);
  if (e != cudaSuccess) return e;
  k_tr_l2qbxl<<<dim3(ix.ncenter_boxes, nrhs), NT, sh, st>>>(g, ix, p, q, ncf, ncq, nrhs, mb, cmp,
                                                            mpoles, err);
  return cudaGetLastError();
}

cudaError_t launch_tr_m2qbxl(const qbxfmm_geometry& g, const qbxfmm_transpose_index& ix, int p,
                             int q, int nrhs, const double2* cmp, double2* locals, int32_t* err,
                             cudaStream_t st)
{
  if (ix.nlist3_rows == 0) return cudaSuccess;
  int ncf = idx3(p + 1, 0), ncq = idx3(q + 1, 0);
  int mb = std::max(1, std::min(8, TRM_NT / (p + q + 1)));
  if (2 * ncf > TRM_H * TRM_NT || mb < 2) return cudaErrorInvalidValue;
  size_t sh = (size_t)mb * ((p + q + 1) * (p + 2 * q + 1) + (q + 1) * (2 * q + 1)) * sizeof(double2) +
              (size_t)mb * (p + 4) * sizeof(double) + (size_t)mb * sizeof(int);
  if (ix.nlist3_rows < TR_SPLIT_BELOW) {
    cudaError_t e = cudaFuncSetAttribute(k_tr_m2qbxl<TR_CL>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    if (e != cudaSuccess) return e;
    k_tr_m2qbxl<TR_CL><<<dim3(ix.nlist3_rows * TR_CL, nrhs), TRM_NT, sh, st>>>(
        g, ix, p, q, ncf, ncq, nrhs, mb, cmp, locals, err);
  } else {
    cudaError_t e = cudaFuncSetAttribute(k_tr_m2qbxl<1>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    if (e != cudaSuccess) return e;
    k_tr_m2qbxl<1><<<dim3(ix.nlist3_rows, nrhs), TRM_NT, sh, st>>>(g, ix, p, q, ncf, ncq, nrhs, mb,
                                                              cmp, locals, err);
  }
  return cudaGetLastError();
}

template <int Q>
static cudaError_t tr_tsqbx_q(const qbxfmm_geometry& g, const qbxfmm_transpose_index& ix,
                              int nrhs, double cq, const double* tvals, double* vals,
                              double* grads, int32_t* err, cudaStream_t st)
{
  const bool split = ix.nlist1_rows < TR_SPLIT_BELOW;
  const dim3 grid(ix.nlist1_rows * (split ? TR_CL : 1), nrhs);
  if (grads && split)
    k_tr_tsqbx<Q, true, TR_CL><<<grid, NT, 0, st>>>(g, ix, nrhs, cq, tvals, vals, grads, err);
  else if (grads)
    k_tr_tsqbx<Q, true, 1><<<grid, NT, 0, st>>>(g, ix, nrhs, cq, tvals, vals, grads, err);
  else if (split)
    k_tr_tsqbx<Q, false, TR_CL><<<grid, NT, 0, st>>>(g, ix, nrhs, cq, tvals, vals, nullptr, err);
  else
    k_tr_tsqbx<Q, false, 1><<<grid, NT, 0, st>>>(g, ix, nrhs, cq, tvals, vals, nullptr, err);
  return cudaGetLastError();
}

cudaError_t launch_tr_p2qbxl(const qbxfmm_geometry& g, const qbxfmm_transpose_index& ix, int q,
                             int nrhs, double cq, const double* tvals, double* vals, double* grads,
                             int32_t* err, cudaStream_t st)
{
  if (ix.nlist1_rows == 0) return cudaSuccess;
  switch (q) {
    case 0: return tr_tsqbx_q<0>(g, ix, nrhs, cq, tvals, vals, grads, err, st);
    case 1: return tr_tsqbx_q<1>(g, ix, nrhs, cq, tvals, vals, grads, err, st);
    case 2: return tr_tsqbx_q<2>(g, ix, nrhs, cq, tvals, vals, grads, err, st);
    case 3: return tr_tsqbx_q<3>(g, ix, nrhs, cq, tvals, vals, grads, err, st);
    case 4: return tr_tsqbx_q<4>(g, ix, nrhs, cq, tvals, vals, grads, err, st);
    case 5: return tr_tsqbx_q<5>(g, ix, nrhs, cq, tvals, vals, grads, err, st);
    case 6: return tr_tsqbx_q<6>(g, ix, nrhs, cq, tvals, vals, grads, err, st);
    case 7: return tr_tsqbx_q<7>(g, ix, nrhs, cq, tvals, vals, grads, err, st);
    case 8: return tr_tsqbx_q<8>(g, ix, nrhs, cq, tvals, vals, grads, err, st);
    default: return cudaErrorInvalidValue;
  }
}

// out[r][j] = scale (cq vals[r][j] + cd n_j . grads[r][.][j]) at the apply's sources
// (tree order): the transpose of a charge + dipole layer from the exchanged-role
// potential and its gradient there
__global__ void k_tr_combine(qbxfmm_geometry g, int nrhs, double scale, double cq, double cd,
                             const double* __restrict__ vals, const double* __restrict__ grads,
                             double* __restrict__ out)
{
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (j >= g.nsources) return;
  double v = cq * vals[(size_t)r * g.nsources + j];
  if (grads) {
    const double* gr = grads + (size_t)r * 3 * g.nsources + j;
    double n[3];
    load_point<3>(g.source_normals, g.nsources, j, n);
    v += cd * (n[0] * gr[0] + n[1] * gr[g.nsources] + n[2] * gr[2 * (size_t)g.nsources]);
  }
  out[(size_t)r * g.nsources + j] = scale * v;
}

cudaError_t launch_tr_combine(const qbxfmm_geometry& g, int nrhs, double scale, double cq,
                              double cd, const double* vals, const double* grads, double* out,
                              cudaStream_t st)
{
  if (g.nsources == 0) return cudaSuccess;
  k_tr_combine<<<dim3((g.nsources + 255) / 256, nrhs), 256, 0, st>>>(g, nrhs, scale, cq, cd,
                                                                     vals, grads, out);
  return cudaGetLastError();
}

// }}}

}  // namespace qbx
