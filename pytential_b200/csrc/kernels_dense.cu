// Dense QBX matrices of the 3D and 2D Laplace layer potentials (the reference's direct QBX
// evaluation, pytential/qbx/__init__.py:797-1068, and its matrix builder,
// pytential/symbolic/matrix.py:450-523): entry (t, s) is the potential at target t of
// a unit source at tree source s with the configured charge / dipole weights,
//   QBX targets (target_center[t] = c >= 0): the order-Q QBX expansion about center c,
//     a = t - c, b = s - c,
//     S: sum_{n<=Q} |a|^n / |b|^{n+1} P_n(cos g),
//     D: sum_{n<=Q} |a|^n / |b|^{n+2} [-(n+1)(nu.b^) P_n + (nu.a^ - cos g nu.b^) P_n'],
//     cos g = a.b / (|a||b|) (the series of the target-specific near field, applied to
//     every source);
//   other targets (target_center[t] < 0): the kernel itself, 1/|t-s| and
//     nu.(t-s)/|t-s|^3;
// times the kernel's scaling 1/(4 pi).  The row-major matrix times the tree-order
// source strengths (upsampled density x area element x weight) is the layer
// potential at the tree targets.  CTA = 128 sources (thread = source, so each row's
// writes are coalesced) x 32 targets staged in shared memory.
#include <string>

#include "../../include/qbxfmm_api.h"
#include "kernels.h"
#include "laplace.cuh"

namespace qbx {
int set_last_error(int code, const std::string& msg);

namespace {

constexpr int DS = 128;   // sources per CTA (one per thread)
constexpr int DTG = 32;   // targets per CTA

__global__ void __launch_bounds__(DS)
k_lap3_qbx_matrix(int nsrc, const double* __restrict__ src, const double* __restrict__ nrm,
                  double cq, double cd, int ntgt, const double* __restrict__ tgt,
                  const int32_t* __restrict__ tcenter, int ncenters,
                  const double* __restrict__ centers, int q, double* __restrict__ K)
{
  __shared__ double s_x[3][DTG], s_c[3][DTG], s_ah[3][DTG], s_al[DTG];
  __shared__ int s_qbx[DTG];
  const int t0 = blockIdx.y * DTG;
  for (int i = threadIdx.x; i < DTG; i += DS) {
    int t = t0 + i;
    int c = t < ntgt ? tcenter[t] : -1;
    if (c >= ncenters) c = -1;
    double x[3] = {0, 0, 0}, cc[3] = {0, 0, 0};
    if (t < ntgt)
      for (int d = 0; d < 3; ++d) x[d] = tgt[(size_t)d * ntgt + t];
    if (c >= 0)
      for (int d = 0; d < 3; ++d) cc[d] = centers[(size_t)d * ncenters + c];
    double a[3] = {x[0] - cc[0], x[1] - cc[1], x[2] - cc[2]};
    double al = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    double ai = al > 0.0 ? 1.0 / al : 0.0;
    for (int d = 0; d < 3; ++d) {
      s_x[d][i] = x[d];
      s_c[d][i] = cc[d];
      s_ah[d][i] = a[d] * ai;
    }
    s_al[i] = al;
    s_qbx[i] = c >= 0;
  }
  __syncthreads();
  const int s = blockIdx.x * DS + threadIdx.x;
  if (s >= nsrc) return;
  const double y[3] = {src[s], src[(size_t)nsrc + s], src[2 * (size_t)nsrc + s]};
  double nv[3] = {0, 0, 0};
  if (cd != 0.0)
    for (int d = 0; d < 3; ++d) nv[d] = nrm[(size_t)d * nsrc + s];
  const double scale = 0.25 / M_PI;
  const int tend = min(DTG, ntgt - t0);
  for (int i = 0; i < tend; ++i) {
    double v = 0.0;
    if (s_qbx[i]) {
      double b0 = y[0] - s_c[0][i], b1 = y[1] - s_c[1][i], b2 = y[2] - s_c[2][i];
      double binv = rsqrt(b0 * b0 + b1 * b1 + b2 * b2);
      double cg = (s_ah[0][i] * b0 + s_ah[1][i] * b1 + s_ah[2][i] * b2) * binv;
      double ratio = s_al[i] * binv;
      double pm1 = 1.0, pm2 = 0.0, dm1 = 0.0;
      double rn = binv, sS = 0.0, sA = 0.0, sB = 0.0;
      for (int n = 0; n <= q; ++n) {
        double pn, dn;
        if (n == 0) {
          pn = 1.0;
          dn = 0.0;
        } else if (n == 1) {
          pn = cg;
          dn = 1.0;
        } else {
          pn = ((2.0 * n - 1) * cg * pm1 - (n - 1.0) * pm2) / n;
          dn = n * pm1 + cg * dm1;
        }
        sS = fma(rn, pn, sS);
        sA = fma(-(n + 1.0) * rn, pn, sA);
        sB = fma(rn, dn, sB);
        pm2 = pm1;
        pm1 = pn;
        dm1 = dn;
        rn *= ratio;
      }
      v = cq * sS;
      if (cd != 0.0) {
        double db = (nv[0] * b0 + nv[1] * b1 + nv[2] * b2) * binv;
        double da = nv[0] * s_ah[0][i] + nv[1] * s_ah[1][i] + nv[2] * s_ah[2][i];
        v += cd * binv * (sA * db + sB * (da - cg * db));
      }
    } else {
      double dx = s_x[0][i] - y[0], dy = s_x[1][i] - y[1], dz = s_x[2][i] - y[2];
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > 0.0) {
        double rinv = rsqrt(r2);
        v = cq * rinv + cd * (nv[0] * dx + nv[1] * dy + nv[2] * dz) * rinv * rinv * rinv;
      }
    }
    K[(size_t)(t0 + i) * nsrc + s] = scale * v;
  }
}

// 2D Laplace: with a = t - c, b = s - c (complex), w = a / b, the target-specific series
//   S: log|b| - Re sum_{n=1..Q} w^n / n,   D: Re(nu / b sum_{n=0..Q} w^n)
// for QBX targets (the series of nu.(s - t)/|s - t|^2), log|t - s| and
// nu.(s - t)/|t - s|^2 for the others, times the kernel's scaling -1/(2 pi) (the 2D
// Laplace apply's sign conventions).
__global__ void __launch_bounds__(DS)
k_lap2_qbx_matrix(int nsrc, const double* __restrict__ src, const double* __restrict__ nrm,
                  double cq, double cd, int ntgt, const double* __restrict__ tgt,
                  const int32_t* __restrict__ tcenter, int ncenters,
                  const double* __restrict__ centers, int q, double* __restrict__ K)
{
  __shared__ double s_x[2][DTG], s_c[2][DTG];
  __shared__ int s_qbx[DTG];
  const int t0 = blockIdx.y * DTG;
  for (int i = threadIdx.x; i < DTG; i += DS) {
    int t = t0 + i;
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
  }
  __syncthreads();
  const int s = blockIdx.x * DS + threadIdx.x;
  if (s >= nsrc) return;
  const double y[2] = {src[s], src[(size_t)nsrc + s]};
  double nv[2] = {0, 0};
  if (cd != 0.0) {
    nv[0] = nrm[s];
    nv[1] = nrm[(size_t)nsrc + s];
  }
  const double scale = -0.5 / M_PI;
  const int tend = min(DTG, ntgt - t0);
  for (int i = 0; i < tend; ++i) {
    double v = 0.0;
    if (s_qbx[i]) {
      double2 bb = c2(y[0] - s_c[0][i], y[1] - s_c[1][i]);
      if (bb.x != 0.0 || bb.y != 0.0) {
        double2 binv = cinv(bb);
        double2 w = cmul(c2(s_x[0][i] - s_c[0][i], s_x[1][i] - s_c[1][i]), binv);
        double2 pw = w, sl = c2(0.0), sd = c2(1.0);
        for (int n = 1; n <= q; ++n) {
          sl = caxpy(1.0 / n, pw, sl);
          sd = cadd(sd, pw);
          pw = cmul(pw, w);
        }
        v = cq * (0.5 * log(bb.x * bb.x + bb.y * bb.y) - sl.x);
        if (cd != 0.0) v += cd * cmul(cmul(c2(nv[0], nv[1]), binv), sd).x;
      }
    } else {
      double dx = s_x[0][i] - y[0], dy = s_x[1][i] - y[1];
      double r2 = dx * dx + dy * dy;
      if (r2 > 0.0) {
        v = 0.5 * cq * log(r2);
        if (cd != 0.0) v -= cd * (nv[0] * dx + nv[1] * dy) / r2;
      }
    }
    K[(size_t)(t0 + i) * nsrc + s] = scale * v;
  }
}

}  // namespace
}  // namespace qbx

extern "C" int qbxfmm_laplace2d_qbx_matrix(int nsources, const double* sources,
                                           const double* normals, double charge_coeff,
                                           double dipole_coeff, int ntargets,
                                           const double* targets, const int32_t* target_center,
                                           int ncenters, const double* centers, int qbx_order,
                                           double* K, void* stream)
{
  using namespace qbx;
  if (nsources < 0 || ntargets < 0 || ncenters < 0)
    return set_last_error(QBXFMM_ERR_ARG, "negative size");
  if (qbx_order < 0 || qbx_order > 32)
    return set_last_error(QBXFMM_ERR_UNSUPPORTED, "qbx_order must be in [0, 32]");
  if (nsources == 0 || ntargets == 0) return QBXFMM_OK;
  if (!sources || !targets || !target_center || !K || (ncenters > 0 && !centers) ||
      (dipole_coeff != 0.0 && !normals))
    return set_last_error(QBXFMM_ERR_ARG, "null argument");
  dim3 grid((nsources + DS - 1) / DS, (ntargets + DTG - 1) / DTG);
  if (grid.y > 65535) return set_last_error(QBXFMM_ERR_UNSUPPORTED, "too many targets");
  k_lap2_qbx_matrix<<<grid, DS, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      nsources, sources, normals, charge_coeff, dipole_coeff, ntargets, targets, target_center,
      ncenters, centers, qbx_order, K);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_last_error(QBXFMM_ERR_CUDA, std::string("laplace2d_qbx_matrix: ") + cudaGetErrorString(e));
  return QBXFMM_OK;
}

extern "C" int qbxfmm_laplace3d_qbx_matrix(int nsources, const double* sources,
                                           const double* normals, double charge_coeff,
                                           double dipole_coeff, int ntargets,
                                           const double* targets, const int32_t* target_center,
                                           int ncenters, const double* centers, int qbx_order,
                                           double* K, void* stream)
{
  using namespace qbx;
  if (nsources < 0 || ntargets < 0 || ncenters < 0)
    return set_last_error(QBXFMM_ERR_ARG, "negative size");
  if (qbx_order < 0 || qbx_order > 16)
    return set_last_error(QBXFMM_ERR_UNSUPPORTED, "qbx_order must be in [0, 16]");
  if (nsources == 0 || ntargets == 0) return QBXFMM_OK;
  if (!sources || !targets || !target_center || !K || (ncenters > 0 && !centers) ||
      (dipole_coeff != 0.0 && !normals))
    return set_last_error(QBXFMM_ERR_ARG, "null argument");
  dim3 grid((nsources + DS - 1) / DS, (ntargets + DTG - 1) / DTG);
  if (grid.y > 65535) return set_last_error(QBXFMM_ERR_UNSUPPORTED, "too many targets");
  k_lap3_qbx_matrix<<<grid, DS, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      nsources, sources, normals, charge_coeff, dipole_coeff, ntargets, targets, target_center,
      ncenters, centers, qbx_order, K);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_last_error(QBXFMM_ERR_CUDA, std::string("laplace3d_qbx_matrix: ") + cudaGetErrorString(e));
  return QBXFMM_OK;
}
