// Dense QBX matrix of the 2D Helmholtz layer potential (the reference's direct QBX
// evaluation, pytential/qbx/__init__.py:797-1068, and its matrix builder,
// pytential/symbolic/matrix.py:450-523) with charge / dipole weights cq, cd:
//   QBX targets (target_center[t] = c >= 0): the order-Q H2D expansion about c applied
//     to the unit source, the series of the target-specific near field,
//       sum_{|m|<=Q} Z_m(t - c) (cq Hb_m(y - c) + (k/2) cd (conj(nu) Hb_{m-1} - nu Hb_{m+1})),
//     Z_m(a) = J_m(k|a|) e^{i m arg a}, Hb_m(b) = H_m(k|b|) e^{-i m arg b};
//   other targets: the kernel itself, cq H_0(k r) + cd k (nu.(t - y)/r) H_1(k r);
// times the kernel's scaling i/4 (H = J + iY, the first-kind Hankel function).  The
// row-major complex matrix times the tree-order source strengths is the layer
// potential at the tree targets.  CTA = 128 sources (thread = source: coalesced row
// writes) x 32 targets whose J tables sit in shared memory.
#include <string>

#include "../../include/qbxfmm_api.h"
#include "helmholtz.cuh"
#include "kernels.h"

namespace qbx {
int set_last_error(int code, const std::string& msg);

namespace {

constexpr int H2D_DS = 128;
constexpr int H2D_DTG = 32;

template <int Q>
__global__ void __launch_bounds__(H2D_DS)
k_h2_qbx_matrix(int nsrc, const double* __restrict__ src, const double* __restrict__ nrm,
                HelmCoeffs hc, int ntgt, const double* __restrict__ tgt,
                const int32_t* __restrict__ tcenter, int ncenters,
                const double* __restrict__ centers, double2* __restrict__ K)
{
  constexpr int NQ = 2 * Q + 1;
  __shared__ double2 s_zt[H2D_DTG][NQ];
  __shared__ double s_x[2][H2D_DTG], s_c[2][H2D_DTG];
  __shared__ int s_qbx[H2D_DTG];
  const int t0 = blockIdx.y * H2D_DTG;
  if (threadIdx.x < H2D_DTG) {
    const int i = threadIdx.x, t = t0 + i;
    int c = t < ntgt ? tcenter[t] : -1;
    if (c >= ncenters) c = -1;
    double x[2] = {0, 0}, cc[2] = {0, 0};
    if (t < ntgt)
      for (int d = 0; d < 2; ++d) x[d] = tgt[(size_t)d * ntgt + t];
    if (c >= 0)
      for (int d = 0; d < 2; ++d) cc[d] = centers[(size_t)d * ncenters + c];
    s_x[0][i] = x[0];
    s_x[1][i] = x[1];
    s_c[0][i] = cc[0];
    s_c[1][i] = cc[1];
    s_qbx[i] = c >= 0;
    double ax = x[0] - cc[0], ay = x[1] - cc[1];
    double alen = sqrt(ax * ax + ay * ay);
    double J[Q + 1];
    if (alen > 0.0) {
      double Yd[1];
      bessel_jy(Q, hc.k * alen, J, Yd, false);
    } else {
#pragma unroll
      for (int m = 0; m <= Q; ++m) J[m] = (m == 0) ? 1.0 : 0.0;
    }
    double2 e1 = alen > 0.0 ? c2(ax / alen, ay / alen) : c2(1.0);
    double2 e = c2(1.0);
#pragma unroll
    for (int m = 0; m <= Q; ++m) {
      s_zt[i][Q + m] = cscale(J[m], e);
      double2 w = cscale(J[m], cconj(e));
      s_zt[i][Q - m] = (m & 1) ? c2(-w.x, -w.y) : w;
      e = cmul(e, e1);
    }
  }
  __syncthreads();
  const int s = blockIdx.x * H2D_DS + threadIdx.x;
  if (s >= nsrc) return;
  const double y[2] = {src[s], src[(size_t)nsrc + s]};
  const bool chg = hc.cq.x != 0.0 || hc.cq.y != 0.0;
  const bool dip = hc.cd.x != 0.0 || hc.cd.y != 0.0;
  double nv[2] = {0, 0};
  if (dip) {
    nv[0] = nrm[s];
    nv[1] = nrm[(size_t)nsrc + s];
  }
  const double2 kd = cscale(0.5 * hc.k, hc.cd);
  const int tend = min(H2D_DTG, ntgt - t0);
  for (int i = 0; i < tend; ++i) {
    double2 v = c2(0.0);
    if (s_qbx[i]) {
      double ux = y[0] - s_c[0][i], uy = y[1] - s_c[1][i];
      double b2 = ux * ux + uy * uy;
      if (b2 != 0.0) {
        double binv = rsqrt(b2);
        double xx = hc.k * b2 * binv, xinv = 1.0 / xx;
        double2 H[Q + 2];
        H[0] = c2(j0(xx), y0(xx));
        H[1] = c2(j1(xx), y1(xx));
#pragma unroll
        for (int m = 1; m <= Q; ++m)
          H[m + 1] = c2(2.0 * m * xinv * H[m].x - H[m - 1].x, 2.0 * m * xinv * H[m].y - H[m - 1].y);
        double2 Hb[2 * Q + 3];                       // Hb_m at Hb[Q + 1 + m]
        double2 e1 = c2(ux * binv, -uy * binv);      // e^{-i arg b}
        double2 e = c2(1.0);
#pragma unroll
        for (int m = 0; m <= Q + 1; ++m) {
          Hb[Q + 1 + m] = cmul(H[m], e);
          double2 w = cmul(H[m], cconj(e));
          Hb[Q + 1 - m] = (m & 1) ? c2(-w.x, -w.y) : w;
          e = cmul(e, e1);
        }
        const double2* Zt = s_zt[i];
        if (chg) {
          double2 s0 = c2(0.0);
#pragma unroll
          for (int m = -Q; m <= Q; ++m) s0 = cfma(Zt[Q + m], Hb[Q + 1 + m], s0);
          v = cmul(hc.cq, s0);
        }
        if (dip) {
          double2 sm = c2(0.0), sp = c2(0.0);
#pragma unroll
          for (int m = -Q; m <= Q; ++m) {
            sm = cfma(Zt[Q + m], Hb[Q + m], sm);
            sp = cfma(Zt[Q + m], Hb[Q + 2 + m], sp);
          }
          double2 nu = c2(nv[0], nv[1]);
          v = cfma(kd, csub(cmul(cconj(nu), sm), cmul(nu, sp)), v);
        }
      }
    } else {
      double dx = s_x[0][i] - y[0], dy = s_x[1][i] - y[1];
      double r2 = dx * dx + dy * dy;
      if (r2 > 0.0) {
        double rr = sqrt(r2), kr = hc.k * rr;
        v = cmul(hc.cq, c2(j0(kr), y0(kr)));
        if (dip) {
          double cn = (nv[0] * dx + nv[1] * dy) / rr;
          v = cfma(cscale(cn * hc.k, hc.cd), c2(j1(kr), y1(kr)), v);
        }
      }
    }
    K[(size_t)(t0 + i) * nsrc + s] = c2(-0.25 * v.y, 0.25 * v.x);   // (i/4) v
  }
}

template <int Q>
cudaError_t launch_h2_matrix(dim3 grid, cudaStream_t st, int nsrc, const double* src,
                             const double* nrm, HelmCoeffs hc, int ntgt, const double* tgt,
                             const int32_t* tc, int ncen, const double* cen, double2* K)
{
  k_h2_qbx_matrix<Q><<<grid, H2D_DS, 0, st>>>(nsrc, src, nrm, hc, ntgt, tgt, tc, ncen, cen, K);
  return cudaGetLastError();
}

}  // namespace
}  // namespace qbx

extern "C" int qbxfmm_helmholtz2d_qbx_matrix(int nsources, const double* sources,
                                             const double* normals, double k, double charge_re,
                                             double charge_im, double dipole_re,
                                             double dipole_im, int ntargets,
                                             const double* targets, const int32_t* target_center,
                                             int ncenters, const double* centers, int qbx_order,
                                             void* K, void* stream)
{
  using namespace qbx;
  if (nsources < 0 || ntargets < 0 || ncenters < 0)
    return set_last_error(QBXFMM_ERR_ARG, "negative size");
  if (qbx_order < 0 || qbx_order > 8)
    return set_last_error(QBXFMM_ERR_UNSUPPORTED, "qbx_order must be in [0, 8]");
  if (!(k > 0.0)) return set_last_error(QBXFMM_ERR_ARG, "wave number must be positive");
  if (nsources == 0 || ntargets == 0) return QBXFMM_OK;
  const bool dip = dipole_re != 0.0 || dipole_im != 0.0;
  if (!sources || !targets || !target_center || !K || (ncenters > 0 && !centers) ||
      (dip && !normals))
    return set_last_error(QBXFMM_ERR_ARG, "null argument");
  dim3 grid((nsources + H2D_DS - 1) / H2D_DS, (ntargets + H2D_DTG - 1) / H2D_DTG);
  if (grid.y > 65535) return set_last_error(QBXFMM_ERR_UNSUPPORTED, "too many targets");
  HelmCoeffs hc;
  hc.k = k;
  hc.cq = c2(charge_re, charge_im);
  hc.cd = c2(dipole_re, dipole_im);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  double2* Kd = static_cast<double2*>(K);
  cudaError_t e;
  switch (qbx_order) {
#define QBX_H2M_CASE(QQ) \
  case QQ: e = launch_h2_matrix<QQ>(grid, st, nsources, sources, normals, hc, ntargets, targets, \
                                     target_center, ncenters, centers, Kd); break;
    QBX_H2M_CASE(0) QBX_H2M_CASE(1) QBX_H2M_CASE(2) QBX_H2M_CASE(3) QBX_H2M_CASE(4)
    QBX_H2M_CASE(5) QBX_H2M_CASE(6) QBX_H2M_CASE(7) QBX_H2M_CASE(8)
#undef QBX_H2M_CASE
    default: return set_last_error(QBXFMM_ERR_UNSUPPORTED, "qbx_order");
  }
  if (e != cudaSuccess)
    return set_last_error(QBXFMM_ERR_CUDA, std::string("helmholtz2d_qbx_matrix: ") + cudaGetErrorString(e));
  return QBXFMM_OK;
}
