// Gradient of the 3D Laplace single-layer potential at the non-QBX targets from the
// FMM's own data: the list-1 sources (P2P), the list-3 multipoles (M2P) and the target
// box's local (L2P) -- the derivative of the apply's value at each target with the
// tree held fixed, for the target-position gradient of the adjoint.
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

}  // namespace qbx
