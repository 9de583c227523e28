// Gradient of the Laplace single-layer potential (3D; 2D at the end of the file) at the
// non-QBX targets from the FMM's own data: the list-1 sources (P2P), the list-3
// multipoles (M2P) and the target box's local (L2P) -- the derivative of the apply's
// value at each target with the tree held fixed, for the target-position gradient of
// the adjoint.
//
// With u = (x - c) / rho and the solid harmonics of laplace.cuh,
//   d/du_z R_n^m = R_{n-1}^m,          d/du_x R_n^m = (R_{n-1}^{m-1} - R_{n-1}^{m+1}) / 2,
//   d/du_y R_n^m = i (R_{n-1}^{m-1} + R_{n-1}^{m+1}) / 2,
//   d/du_z S_n^m = -S_{n+1}^m,         d/du_x S_n^m = (S_{n+1}^{m-1} - S_{n+1}^{m+1}) / 2,
//   d/du_y S_n^m = i (S_{n+1}^{m-1} + S_{n+1}^{m+1}) / 2,
// and the conjugate symmetry of real fields, each table entry X_k^j (j >= 0) adds,
// for the row n = k + 1 (locals) or n = k - 1 (multipoles) and a = L or M there,
//   locals:      x += Re(a_{n,j+1} conj X) - [j>0] Re(a_{n,j-1} conj X)
//                y += Im(a_{n,j+1} conj X) + [j>0] Im(a_{n,j-1} conj X)
//                z += w_j Re(a_{n,j} conj X)
//   multipoles:  x += Re(a_{n,j+1} X) - [j>0] Re(a_{n,j-1} X)
//                y += -Im(a_{n,j+1} X) - [j>0] Im(a_{n,j-1} X)
//                z += -w_j Re(a_{n,j} X)
// (w_0 = 1, w_{j>0} = 2; entries outside |m| <= n <= p are zero), so one pass of the
// column recurrences gives the gradient without a table.  Each lane owns a target;
// for P2P and M2P a cluster of GSPL CTAs per chunk of <= 32 targets deals the sources
// or the list-3 boxes to its warps, and the partial gradients meet in a fixed order
// (shared memory, then distributed shared memory to CTA 0).
#include "laplace.cuh"
#include "kernels.h"

#include <cooperative_groups.h>
namespace cg = cooperative_groups;

namespace qbx {

namespace {

constexpr int NT = 128;
constexpr int NW = NT / 32;
constexpr int GSPL = 8;    // CTAs per target chunk (a cluster) in P2P / M2P

QBX_D double2 coef(const double2* a, int n, int m, int p)
{
  return (m >= 0 && m <= n && n <= p) ? a[idx3(n, m)] : c2(0.0);
}

// partial gradients of the warps of the GSPL CTAs of a cluster summed in a fixed order
// (warps in their CTA, then CTAs by rank through distributed shared memory); lane t
// of warp 0 of CTA 0 adds the total into out0..2
QBX_D void cluster_reduce_add(double g[3], double (*s_red)[3][32], double (*s_part)[32],
                              bool active, double* out0, double* out1, double* out2)
{
  cg::cluster_group cl = cg::this_cluster();
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (warp > 0)
    for (int d = 0; d < 3; ++d) s_red[warp - 1][d][lane] = g[d];
  __syncthreads();
  if (warp == 0) {
    for (int w = 1; w < NW; ++w)
      for (int d = 0; d < 3; ++d) g[d] += s_red[w - 1][d][lane];
    for (int d = 0; d < 3; ++d) s_part[d][lane] = g[d];
  }
  cl.sync();
  if (cl.block_rank() == 0 && warp == 0) {
    for (unsigned q = 1; q < cl.num_blocks(); ++q) {
      double* rp = cl.map_shared_rank(&s_part[0][0], q);
      for (int d = 0; d < 3; ++d) g[d] += rp[d * 32 + lane];
    }
    if (active) {
      *out0 += g[0];
      *out1 += g[1];
      *out2 += g[2];
    }
  }
  cl.sync();
}

}  // namespace

// {{{ P2P: -cq q (x - y) / |x - y|^3 over the list-1 sources of the target box

__global__ void __cluster_dims__(GSPL, 1, 1) __launch_bounds__(NT)
k_grad_direct(qbxfmm_geometry g, double cq, double scale, int nrhs,
              const double* __restrict__ strengths, double* __restrict__ grad, int32_t* err)
{
  __shared__ double s_red[NW - 1][3][32];
  __shared__ double s_part[3][32];
  int chunk = blockIdx.x / GSPL, part = blockIdx.x - chunk * GSPL, r = blockIdx.y;
  int itb = g.nonqbx_chunk_target_box[chunk];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int t = g.nonqbx_chunk_start[chunk] + lane;
  bool active = lane < g.nonqbx_chunk_count[chunk];
  double x[3] = {0.0, 0.0, 0.0};
  if (active) load_point<3>(g.nonqbx_targets, g.nfiltered_targets, t, x);
  const double* st = strengths + (size_t)r * g.nsources;
  double gr[3] = {0.0, 0.0, 0.0};
  // the sources of the list-1 boxes, each box's range dealt to the GSPL x NW warps
  const int stride = GSPL * NW, lead = part * NW + warp;
  for (int li = g.list1_starts[itb]; li < g.list1_starts[itb + 1]; ++li) {
    int sb = g.list1_lists[li];
    if ((unsigned)sb >= (unsigned)g.nboxes) {
      report(err, QBX_DEVERR_BAD_BOX);
      continue;
    }
    int s0 = g.box_source_starts[sb], s1 = s0 + g.box_source_counts_nonchild[sb];
    if (!active) continue;
    for (int j = s0 + lead; j < s1; j += stride) {
      double y[3];
      load_point<3>(g.sources, g.nsources, j, y);
      double dx = x[0] - y[0], dy = x[1] - y[1], dz = x[2] - y[2];
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 == 0.0) continue;
      double ri = rsqrt(r2);
      double f = -scale * cq * st[j] * ri * ri * ri;
      gr[0] = fma(f, dx, gr[0]);
      gr[1] = fma(f, dy, gr[1]);
      gr[2] = fma(f, dz, gr[2]);
    }
  }
  size_t o = (size_t)r * 3 * g.nfiltered_targets + t;
  cluster_reduce_add(gr, s_red, s_part, active, grad + o, grad + o + g.nfiltered_targets,
                     grad + o + 2 * (size_t)g.nfiltered_targets);
}

// }}}

// {{{ M2P: gradient of the list-3 multipoles at the targets (warps split the boxes)

__global__ void __cluster_dims__(GSPL, 1, 1) __launch_bounds__(NT)
k_grad_multipoles(qbxfmm_geometry g, int p, int ncf, int nrhs, double scale,
                  const double2* __restrict__ mpoles, double* __restrict__ grad, int32_t* err)
{
  extern __shared__ double2 smem2[];
  __shared__ double s_red[NW - 1][3][32];
  __shared__ double s_part[3][32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double2* M = smem2 + (size_t)warp * ncf;
  int chunk = blockIdx.x / GSPL, part = blockIdx.x - chunk * GSPL, r = blockIdx.y;
  int itb = g.nonqbx_chunk_target_box[chunk];
  int t = g.nonqbx_chunk_start[chunk] + lane;
  bool active = lane < g.nonqbx_chunk_count[chunk];
  double x[3] = {0.0, 0.0, 0.0};
  if (active) load_point<3>(g.nonqbx_targets, g.nfiltered_targets, t, x);
  double gr[3] = {0.0, 0.0, 0.0};
  for (int li = g.list3_starts[itb] + part * NW + warp; li < g.list3_starts[itb + 1];
       li += GSPL * NW) {
    int sb = g.list3_lists[li];
    if ((unsigned)sb >= (unsigned)g.nboxes) {
      report(err, QBX_DEVERR_BAD_BOX);
      continue;
    }
    __syncwarp();
    const double2* src = mpoles + ((size_t)sb * nrhs + r) * ncf;
    for (int q = lane; q < ncf; q += 32) M[q] = src[q];
    __syncwarp();
    if (!active) continue;
    double rho = level_width(g, g.box_levels[sb]);
    double cs[3];
    load_point<3>(g.box_centers, g.nboxes, sb, cs);
    double u0 = (x[0] - cs[0]) / rho, u1 = (x[1] - cs[1]) / rho, u2 = (x[2] - cs[2]) / rho;
    double rinv2 = 1.0 / (u0 * u0 + u1 * u1 + u2 * u2);
    double2 mm = c2(sqrt(rinv2));
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    // S_k^j for k = 0..p+1; row k feeds the coefficients of row n = k - 1
    for (int j = 0; j <= p + 1; ++j) {
      if (j > 0) mm = cscale((2.0 * j - 1) * rinv2, cmul(mm, c2(u0, u1)));
      double2 s = mm, prev = c2(0.0);
      double w = j ? 2.0 : 1.0;
      for (int k = j; k <= p + 1; ++k) {
        if (k > j) {
          double2 bb = cscale(rinv2, csub(cscale((2.0 * k - 1) * u2, s),
                                          cscale((double)(k + j - 1) * (k - j - 1), prev)));
          prev = s;
          s = bb;
        }
        int n = k - 1;
        if (n < 0) continue;
        double2 ap = coef(M, n, j + 1, p), am = coef(M, n, j - 1, p), a = coef(M, n, j, p);
        double2 vp = cmul(ap, s), vm = cmul(am, s), v = cmul(a, s);
        a0 += vp.x - (j > 0 ? vm.x : 0.0);
        a1 += -vp.y - (j > 0 ? vm.y : 0.0);
        a2 -= w * v.x;
      }
    }
    double f = scale / (rho * rho);
    gr[0] = fma(f, a0, gr[0]);
    gr[1] = fma(f, a1, gr[1]);
    gr[2] = fma(f, a2, gr[2]);
  }
  size_t o = (size_t)r * 3 * g.nfiltered_targets + t;
  cluster_reduce_add(gr, s_red, s_part, active, grad + o, grad + o + g.nfiltered_targets,
                     grad + o + 2 * (size_t)g.nfiltered_targets);
}

// }}}

// {{{ L2P: gradient of the target box's local at its targets

__global__ void __launch_bounds__(NT)
k_grad_locals(qbxfmm_geometry g, int p, int ncf, int nrhs, double scale,
              const double2* __restrict__ locals, double* __restrict__ grad)
{
  extern __shared__ double2 smem2[];
  double2* L = smem2;
  int itb = blockIdx.x, r = blockIdx.y;
  int tb = g.target_boxes[itb];
  int t0 = g.nonqbx_box_target_starts[tb];
  int nt = g.nonqbx_box_target_counts_nonchild[tb];
  if (nt == 0) return;
  const double2* src = locals + ((size_t)tb * nrhs + r) * ncf;
  for (int q = threadIdx.x; q < ncf; q += NT) L[q] = src[q];
  __syncthreads();
  double rho = level_width(g, g.box_levels[tb]);
  double cb[3];
  load_point<3>(g.box_centers, g.nboxes, tb, cb);
  for (int tt = threadIdx.x; tt < nt; tt += NT) {
    double x[3];
    load_point<3>(g.nonqbx_targets, g.nfiltered_targets, t0 + tt, x);
    double u0 = (x[0] - cb[0]) / rho, u1 = (x[1] - cb[1]) / rho, u2 = (x[2] - cb[2]) / rho;
    double r2 = u0 * u0 + u1 * u1 + u2 * u2;
    double2 mm = c2(1.0);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    // R_k^j for k = 0..p-1; row k feeds the coefficients of row n = k + 1
    for (int j = 0; j < p; ++j) {
      if (j > 0) mm = cscale(0.5 * rcp(j), cmul(mm, c2(u0, u1)));
      double2 a = mm, prev = c2(0.0);
      double w = j ? 2.0 : 1.0;
      for (int k = j; k < p; ++k) {
        if (k > j) {
          double2 bb = cscale(rcp(k + j) * rcp(k - j),
                              csub(cscale((2.0 * k - 1) * u2, a), cscale(r2, prev)));
          prev = a;
          a = bb;
        }
        int n = k + 1;
        double2 cp = coef(L, n, j + 1, p), cm = coef(L, n, j - 1, p), c = coef(L, n, j, p);
        double2 vp = cmulc(cp, a), vm = cmulc(cm, a), v = cmulc(c, a);   // a_n conj(R)
        a0 += vp.x - (j > 0 ? vm.x : 0.0);
        a1 += vp.y + (j > 0 ? vm.y : 0.0);
        a2 += w * v.x;
      }
    }
    double f = scale / rho;
    size_t o = (size_t)r * 3 * g.nfiltered_targets + t0 + tt;
    grad[o] += f * a0;
    grad[o + g.nfiltered_targets] += f * a1;
    grad[o + 2 * (size_t)g.nfiltered_targets] += f * a2;
  }
}

// }}}

// {{{ QBX targets: gradient of the center's QBX local, and of the target-specific near field

// one thread per global center: the streaming L2P gradient of its order-q QBX local
// at each of its targets (grad[r][0..2][t], tree target order)
__global__ void __launch_bounds__(NT)
k_grad_qbxl2p(qbxfmm_geometry g, int q, int ncq, int nrhs, double scale,
              const double2* __restrict__ qbx_exps, double* __restrict__ grad, int32_t* err)
{
  int ig = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (ig >= g.nglobal_qbx_centers) return;
  int ctr = g.global_qbx_centers[ig];
  if ((unsigned)ctr >= (unsigned)g.ncenters) {
    report(err, QBX_DEVERR_BAD_CENTER);
    return;
  }
  double cc[3];
  load_point<3>(g.centers, g.ncenters, ctr, cc);
  double rho = g.expansion_radii[ctr];
  const double2* L = qbx_exps + ((size_t)ctr * nrhs + r) * ncq;
  for (int it = g.center_to_targets_starts[ctr]; it < g.center_to_targets_starts[ctr + 1]; ++it) {
    int t = g.center_to_targets_lists[it];
    if ((unsigned)t >= (unsigned)g.ntargets) {
      report(err, QBX_DEVERR_BAD_CENTER);
      continue;
    }
    double x[3];
    load_point<3>(g.targets, g.ntargets, t, x);
    double u0 = (x[0] - cc[0]) / rho, u1 = (x[1] - cc[1]) / rho, u2 = (x[2] - cc[2]) / rho;
    double r2 = u0 * u0 + u1 * u1 + u2 * u2;
    double2 mm = c2(1.0);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int j = 0; j < q; ++j) {
      if (j > 0) mm = cscale(0.5 * rcp(j), cmul(mm, c2(u0, u1)));
      double2 a = mm, prev = c2(0.0);
      double w = j ? 2.0 : 1.0;
      for (int k = j; k < q; ++k) {
        if (k > j) {
          double2 bb = cscale(rcp(k + j) * rcp(k - j),
                              csub(cscale((2.0 * k - 1) * u2, a), cscale(r2, prev)));
          prev = a;
          a = bb;
        }
        int n = k + 1;
        double2 cp = coef(L, n, j + 1, q), cm = coef(L, n, j - 1, q), c = coef(L, n, j, q);
        double2 vp = cmulc(cp, a), vm = cmulc(cm, a), v = cmulc(c, a);
        a0 += vp.x - (j > 0 ? vm.x : 0.0);
        a1 += vp.y + (j > 0 ? vm.y : 0.0);
        a2 += w * v.x;
      }
    }
    double f = scale / rho;
    size_t o = (size_t)r * 3 * g.ntargets + t;
    grad[o] += f * a0;
    grad[o + g.ntargets] += f * a1;
    grad[o + 2 * (size_t)g.ntargets] += f * a2;
  }
}

// The target-specific near field K = sum_{n<=Q} |a|^n / |b|^{n+1} P_n(cos g),
// a = t - c, b = y - c, cos g = a^.b^, differentiated at the target:
//   grad_a K = sum_n |a|^{n-1} / |b|^{n+1} [(n P_n - cos g P_n') a^ + P_n' b^].
// CTA = one chunk of <= 32 (target, center) pairs (lane = pair), a cluster of GSPL CTAs
// dealing the list-1 sources of the center's box to its warps.
template <int Q>
__global__ void __cluster_dims__(GSPL, 1, 1) __launch_bounds__(NT)
k_grad_tsqbx(qbxfmm_geometry g, double cq, double scale, int nrhs,
             const double* __restrict__ strengths, double* __restrict__ grad, int32_t* err)
{
  __shared__ double s_red[NW - 1][3][32];
  __shared__ double s_part[3][32];
  int chunk = blockIdx.x / GSPL, part = blockIdx.x - chunk * GSPL, r = blockIdx.y;
  int itb = g.tsqbx_chunk_target_box[chunk];
  int i0 = g.tsqbx_chunk_start[chunk];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bool active = lane < g.tsqbx_chunk_count[chunk];
  int t = active ? g.tsqbx_targets[i0 + lane] : 0;
  int ctr = active ? g.tsqbx_centers[i0 + lane] : 0;
  if ((unsigned)ctr >= (unsigned)g.ncenters || (unsigned)t >= (unsigned)g.ntargets) {
    report(err, QBX_DEVERR_BAD_CENTER);
    active = false;
    t = ctr = 0;
  }
  double cc[3] = {0.0, 0.0, 0.0}, x[3] = {0.0, 0.0, 0.0};
  load_point<3>(g.centers, g.ncenters, ctr, cc);
  load_point<3>(g.targets, g.ntargets, t, x);
  double a[3] = {x[0] - cc[0], x[1] - cc[1], x[2] - cc[2]};
  double alen = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  double ainv = alen > 0.0 ? 1.0 / alen : 0.0;
  double ah[3] = {a[0] * ainv, a[1] * ainv, a[2] * ainv};
  const double* st = strengths + (size_t)r * g.nsources;
  double gr[3] = {0.0, 0.0, 0.0};
  const int stride = GSPL * NW, lead = part * NW + warp;
  for (int li = g.list1_starts[itb]; li < g.list1_starts[itb + 1]; ++li) {
    int sb = g.list1_lists[li];
    if ((unsigned)sb >= (unsigned)g.nboxes) {
      report(err, QBX_DEVERR_BAD_BOX);
      continue;
    }
    int s0 = g.box_source_starts[sb], s1 = s0 + g.box_source_counts_nonchild[sb];
    if (!active) continue;
    for (int j = s0 + lead; j < s1; j += stride) {
      double y[3];
      load_point<3>(g.sources, g.nsources, j, y);
      double b0 = y[0] - cc[0], b1 = y[1] - cc[1], b2 = y[2] - cc[2];
      double binv = rsqrt(b0 * b0 + b1 * b1 + b2 * b2);
      double bh0 = b0 * binv, bh1 = b1 * binv, bh2 = b2 * binv;
      double cg = ah[0] * bh0 + ah[1] * bh1 + ah[2] * bh2;
      double ratio = alen * binv;
      // rn = |a|^{n-1} / |b|^{n+1}, from n = 1
      double rn = binv * binv;
      double pm1 = 1.0, pm2 = 0.0, dm1 = 0.0, sa = 0.0, sb2 = 0.0;
#pragma unroll
      for (int n = 1; n <= Q; ++n) {
        double pn = n == 1 ? cg : ((2.0 * n - 1) * cg * pm1 - (n - 1.0) * pm2) * (1.0 / n);
        double dn = n * pm1 + cg * dm1;
        sa = fma(rn, n * pn - cg * dn, sa);
        sb2 = fma(rn, dn, sb2);
        pm2 = pm1;
        pm1 = pn;
        dm1 = dn;
        rn *= ratio;
      }
      double f = scale * cq * st[j];
      gr[0] = fma(f, sa * ah[0] + sb2 * bh0, gr[0]);
      gr[1] = fma(f, sa * ah[1] + sb2 * bh1, gr[1]);
      gr[2] = fma(f, sa * ah[2] + sb2 * bh2, gr[2]);
    }
  }
  size_t o = (size_t)r * 3 * g.ntargets + t;
  cluster_reduce_add(gr, s_red, s_part, active, grad + o, grad + o + g.ntargets,
                     grad + o + 2 * (size_t)g.ntargets);
}

template <int Q>
static cudaError_t grad_tsqbx_q(const qbxfmm_geometry& g, double cq, double scale, int nrhs,
                                const double* s, double* grad, int32_t* err, cudaStream_t st)
{
  k_grad_tsqbx<Q><<<dim3(g.ntsqbx_chunks * GSPL, nrhs), NT, 0, st>>>(g, cq, scale, nrhs, s, grad,
                                                                     err);
  return cudaGetLastError();
}

cudaError_t launch_grad_qbx_targets(const qbxfmm_geometry& g, double cq, double scale, int q,
                                    int nrhs, bool target_specific, const double* strengths,
                                    const double2* qbx_exps, double* grad, int32_t* err,
                                    cudaStream_t st)
{
  if (g.nglobal_qbx_centers == 0) return cudaSuccess;
  int ncq = idx3(q + 1, 0);
  k_grad_qbxl2p<<<dim3((g.nglobal_qbx_centers + NT - 1) / NT, nrhs), NT, 0, st>>>(
      g, q, ncq, nrhs, scale, qbx_exps, grad, err);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !target_specific || g.ntsqbx_chunks == 0) return e;
  switch (q) {
    case 0: return grad_tsqbx_q<0>(g, cq, scale, nrhs, strengths, grad, err, st);
    case 1: return grad_tsqbx_q<1>(g, cq, scale, nrhs, strengths, grad, err, st);
    case 2: return grad_tsqbx_q<2>(g, cq, scale, nrhs, strengths, grad, err, st);
    case 3: return grad_tsqbx_q<3>(g, cq, scale, nrhs, strengths, grad, err, st);
    case 4: return grad_tsqbx_q<4>(g, cq, scale, nrhs, strengths, grad, err, st);
    case 5: return grad_tsqbx_q<5>(g, cq, scale, nrhs, strengths, grad, err, st);
    case 6: return grad_tsqbx_q<6>(g, cq, scale, nrhs, strengths, grad, err, st);
    case 7: return grad_tsqbx_q<7>(g, cq, scale, nrhs, strengths, grad, err, st);
    case 8: return grad_tsqbx_q<8>(g, cq, scale, nrhs, strengths, grad, err, st);
    default: return cudaErrorInvalidValue;
  }
}

// }}}

cudaError_t launch_grad_targets(const qbxfmm_geometry& g, double cq, double scale, int p,
                                int nrhs, const double* strengths, const double2* mpoles,
                                const double2* locals, double* grad, int32_t* err,
                                cudaStream_t st)
{
  if (g.nfiltered_targets == 0) return cudaSuccess;
  int ncf = idx3(p + 1, 0);
  if (g.nnonqbx_chunks > 0) {
    k_grad_direct<<<dim3(g.nnonqbx_chunks * GSPL, nrhs), NT, 0, st>>>(g, cq, scale, nrhs,
                                                                      strengths, grad, err);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_grad_multipoles<<<dim3(g.nnonqbx_chunks * GSPL, nrhs), NT, (size_t)NW * ncf * sizeof(double2),
                        st>>>(
        g, p, ncf, nrhs, scale, mpoles, grad, err);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (g.ntarget_boxes > 0)
    k_grad_locals<<<dim3(g.ntarget_boxes, nrhs), NT, ncf * sizeof(double2), st>>>(
        g, p, ncf, nrhs, scale, locals, grad);
  return cudaGetLastError();
}

// {{{ 2D Laplace: grad Re f = (Re f', -Im f') for the complex-analytic f of each term
//   P2P    log|z - y|:                              f' = 1 / (z - y)
//   M2P    M_0 log(z - c) + sum_k M_k u^-k:          f' = (M_0 / u - sum_k k M_k u^(-k-1)) / rho
//   L2P    sum_k L_k u^k:                            f' = sum_k k L_k u^(k-1) / rho
//   TSQBX  log|b| - Re sum_{n<=Q} (a / b)^n / n:    d/da = -sum_n a^(n-1) / b^n
// (u = (z - c) / rho, a = t - c, b = y - c).  One thread per target; grad[r][2][n].

// non-QBX targets: CTA per target box, thread per target (P2P over list 1, M2P over
// list 3, L2P of the box's local)
__global__ void __launch_bounds__(NT)
k_grad2_targets(qbxfmm_geometry g, double cq, double scale, int p, int nrhs,
                const double* __restrict__ strengths, const double2* __restrict__ mpoles,
                const double2* __restrict__ locals, double* __restrict__ grad, int32_t* err)
{
  const int itb = blockIdx.x, r = blockIdx.y, ncf = p + 1;
  const int tb = g.target_boxes[itb];
  const int t0 = g.nonqbx_box_target_starts[tb];
  const int nt = g.nonqbx_box_target_counts_nonchild[tb];
  if (nt == 0) return;
  const double* st = strengths + (size_t)r * g.nsources;
  const double2* L = locals + ((size_t)tb * nrhs + r) * ncf;
  const double rho_b = level_width(g, g.box_levels[tb]);
  double cb[2];
  load_point<2>(g.box_centers, g.nboxes, tb, cb);
  for (int tt = threadIdx.x; tt < nt; tt += NT) {
    double x[2];
    load_point<2>(g.nonqbx_targets, g.nfiltered_targets, t0 + tt, x);
    double gx = 0.0, gy = 0.0;
    for (int li = g.list1_starts[itb]; li < g.list1_starts[itb + 1]; ++li) {
      const int sb = g.list1_lists[li];
      if ((unsigned)sb >= (unsigned)g.nboxes) {
        report(err, QBX_DEVERR_BAD_BOX);
        continue;
      }
      const int s0 = g.box_source_starts[sb], s1 = s0 + g.box_source_counts_nonchild[sb];
      for (int j = s0; j < s1; ++j) {
        double y[2];
        load_point<2>(g.sources, g.nsources, j, y);
        const double dx = x[0] - y[0], dy = x[1] - y[1], r2 = dx * dx + dy * dy;
        if (r2 == 0.0) continue;
        const double f = cq * st[j] / r2;
        gx = fma(f, dx, gx);
        gy = fma(f, dy, gy);
      }
    }
    double2 d = c2(0.0);                   // sum of f'
    for (int li = g.list3_starts[itb]; li < g.list3_starts[itb + 1]; ++li) {
      const int sb = g.list3_lists[li];
      if ((unsigned)sb >= (unsigned)g.nboxes) {
        report(err, QBX_DEVERR_BAD_BOX);
        continue;
      }
      const double2* M = mpoles + ((size_t)sb * nrhs + r) * ncf;
      const double rho = level_width(g, g.box_levels[sb]);
      double cs[2];
      load_point<2>(g.box_centers, g.nboxes, sb, cs);
      const double2 uinv = cinv(c2((x[0] - cs[0]) / rho, (x[1] - cs[1]) / rho));
      double2 e = cmul(M[0], uinv), pw = cmul(uinv, uinv);
      for (int k = 1; k <= p; ++k) {
        e = csub(e, cscale((double)k, cmul(M[k], pw)));
        pw = cmul(pw, uinv);
      }
      d = cadd(d, cscale(1.0 / rho, e));
    }
    {
      const double2 u = c2((x[0] - cb[0]) / rho_b, (x[1] - cb[1]) / rho_b);
      double2 e = c2(0.0), pw = c2(1.0);
      for (int k = 1; k <= p; ++k) {
        e = cadd(e, cscale((double)k, cmul(L[k], pw)));
        pw = cmul(pw, u);
      }
      d = cadd(d, cscale(1.0 / rho_b, e));
    }
    const size_t o = (size_t)r * 2 * g.nfiltered_targets + t0 + tt;
    grad[o] += scale * (gx + d.x);
    grad[o + g.nfiltered_targets] += scale * (gy - d.y);
  }
}

// QBX targets: thread per global center, the derivative of its QBX local at each of
// its targets (center held fixed)
__global__ void __launch_bounds__(NT)
k_grad2_qbxl2p(qbxfmm_geometry g, int q, int nrhs, double scale,
               const double2* __restrict__ qbx_exps, double* __restrict__ grad, int32_t* err)
{
  const int ig = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (ig >= g.nglobal_qbx_centers) return;
  const int ctr = g.global_qbx_centers[ig];
  if ((unsigned)ctr >= (unsigned)g.ncenters) {
    report(err, QBX_DEVERR_BAD_CENTER);
    return;
  }
  double cc[2];
  load_point<2>(g.centers, g.ncenters, ctr, cc);
  const double rho = g.expansion_radii[ctr];
  const double2* L = qbx_exps + ((size_t)ctr * nrhs + r) * (q + 1);
  for (int it = g.center_to_targets_starts[ctr]; it < g.center_to_targets_starts[ctr + 1]; ++it) {
    const int t = g.center_to_targets_lists[it];
    if ((unsigned)t >= (unsigned)g.ntargets) {
      report(err, QBX_DEVERR_BAD_CENTER);
      continue;
    }
    double x[2];
    load_point<2>(g.targets, g.ntargets, t, x);
    const double2 u = c2((x[0] - cc[0]) / rho, (x[1] - cc[1]) / rho);
    double2 e = c2(0.0), pw = c2(1.0);
    for (int k = 1; k <= q; ++k) {
      e = cadd(e, cscale((double)k, cmul(L[k], pw)));
      pw = cmul(pw, u);
    }
    const size_t o = (size_t)r * 2 * g.ntargets + t;
    grad[o] += scale * e.x / rho;
    grad[o + g.ntargets] -= scale * e.y / rho;
  }
}

// the target-specific near field: thread per (target, center) pair of a chunk, over
// the list-1 sources of the chunk's target box
__global__ void __launch_bounds__(32)
k_grad2_tsqbx(qbxfmm_geometry g, double cq, double scale, int q, int nrhs,
              const double* __restrict__ strengths, double* __restrict__ grad, int32_t* err)
{
  const int chunk = blockIdx.x, r = blockIdx.y, lane = threadIdx.x;
  const int itb = g.tsqbx_chunk_target_box[chunk];
  if (lane >= g.tsqbx_chunk_count[chunk]) return;
  const int t = g.tsqbx_targets[g.tsqbx_chunk_start[chunk] + lane];
  const int ctr = g.tsqbx_centers[g.tsqbx_chunk_start[chunk] + lane];
  if ((unsigned)ctr >= (unsigned)g.ncenters || (unsigned)t >= (unsigned)g.ntargets) {
    report(err, QBX_DEVERR_BAD_CENTER);
    return;
  }
  double cc[2], x[2];
  load_point<2>(g.centers, g.ncenters, ctr, cc);
  load_point<2>(g.targets, g.ntargets, t, x);
  const double2 a = c2(x[0] - cc[0], x[1] - cc[1]);
  const double* st = strengths + (size_t)r * g.nsources;
  double2 h = c2(0.0);                     // sum_j q_j sum_n a^(n-1) / b_j^n
  for (int li = g.list1_starts[itb]; li < g.list1_starts[itb + 1]; ++li) {
    const int sb = g.list1_lists[li];
    if ((unsigned)sb >= (unsigned)g.nboxes) {
      report(err, QBX_DEVERR_BAD_BOX);
      continue;
    }
    const int s0 = g.box_source_starts[sb], s1 = s0 + g.box_source_counts_nonchild[sb];
    for (int j = s0; j < s1; ++j) {
      double y[2];
      load_point<2>(g.sources, g.nsources, j, y);
      const double2 binv = cinv(c2(y[0] - cc[0], y[1] - cc[1]));
      const double2 w = cmul(a, binv);
      double2 term = binv, sum = c2(0.0);   // a^(n-1) / b^n from n = 1
      for (int n = 1; n <= q; ++n) {
        sum = cadd(sum, term);
        term = cmul(term, w);
      }
      h = cadd(h, cscale(st[j], sum));
    }
  }
  const size_t o = (size_t)r * 2 * g.ntargets + t;
  grad[o] -= scale * cq * h.x;
  grad[o + g.ntargets] += scale * cq * h.y;
}

cudaError_t launch_grad2_targets(const qbxfmm_geometry& g, double cq, double scale, int p,
                                 int nrhs, const double* strengths, const double2* mpoles,
                                 const double2* locals, double* grad, int32_t* err,
                                 cudaStream_t st)
{
  if (g.nfiltered_targets == 0 || g.ntarget_boxes == 0) return cudaSuccess;
  k_grad2_targets<<<dim3(g.ntarget_boxes, nrhs), NT, 0, st>>>(g, cq, scale, p, nrhs, strengths,
                                                              mpoles, locals, grad, err);
  return cudaGetLastError();
}

cudaError_t launch_grad2_qbx_targets(const qbxfmm_geometry& g, double cq, double scale, int q,
                                     int nrhs, bool target_specific, const double* strengths,
                                     const double2* qbx_exps, double* grad, int32_t* err,
                                     cudaStream_t st)
{
  if (g.nglobal_qbx_centers == 0) return cudaSuccess;
  k_grad2_qbxl2p<<<dim3((g.nglobal_qbx_centers + NT - 1) / NT, nrhs), NT, 0, st>>>(
      g, q, nrhs, scale, qbx_exps, grad, err);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !target_specific || g.ntsqbx_chunks == 0) return e;
  k_grad2_tsqbx<<<dim3(g.ntsqbx_chunks, nrhs), 32, 0, st>>>(g, cq, scale, q, nrhs, strengths,
                                                            grad, err);
  return cudaGetLastError();
}

// }}}

}  // namespace qbx
