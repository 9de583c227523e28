// Direct gradient of the 3D Laplace single-layer potential at far targets, used for
// the target-position gradient of the adjoint (the forward apply's targets are far
// from the surface there, so the sum needs no QBX):
//   grad u(x_t) = -1/(4 pi) sum_y q_y (x_t - y) / |x_t - y|^3.
// A cluster of GSPLIT CTAs per 64 targets (4 threads per target, interleaving the
// sources of a tile): CTA y of the cluster takes the y-th contiguous chunk of the
// sources, streamed through shared memory in tiles of 256; the 4 partial sums of a
// target meet in shared memory and CTA 0 adds the GSPLIT partials in a fixed order
// through distributed shared memory (deterministic; a few thousand targets still fill
// the GPU).
#include <string>
#include <type_traits>

#include <cooperative_groups.h>

#include "../../include/qbxfmm_api.h"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace qbx {
int set_last_error(int code, const std::string& msg);

constexpr int GT = 64;
constexpr int GS = 256;
constexpr int GSPLIT = 8;

namespace {

constexpr int TPT = 4;   // threads per target: they take every TPT-th source of a tile

// grad[d][t] = -1/(4 pi) sum_s q_s (x_t - y_s)_d / |x_t - y_s|^3.  CTA = GT targets x TPT
// threads; a cluster of GSPLIT CTAs splits the sources and sums its partials in CTA 0
// in a fixed order (distributed shared memory).  F32: the FP32 form of the mixed-
// precision adjoint -- sources staged as floats relative to an origin o (the CTA's
// first target), so that x - y = (x - o) - (y - o) keeps its relative accuracy for the
// far targets this entry serves, FP32 sums per tile added into FP64.
template <bool F32>
__global__ void __cluster_dims__(1, GSPLIT, 1) __launch_bounds__(GT * TPT)
k_lap3_grad_direct(int nsrc, const double* __restrict__ src, const double* __restrict__ q,
                   int ntgt, const double* __restrict__ tgt, double* __restrict__ grad)
{
  using R = typename std::conditional<F32, float, double>::type;
  __shared__ R s_y[3][GS], s_q[GS];
  __shared__ double s_part[3][TPT][GT];
  const int tl = threadIdx.x % GT, sub = threadIdx.x / GT;
  const int t = blockIdx.x * GT + tl;
  const bool active = t < ntgt;
  double o[3] = {0.0, 0.0, 0.0};
  if (F32)
    for (int d = 0; d < 3; ++d) o[d] = tgt[(size_t)d * ntgt + blockIdx.x * GT];
  R x[3] = {0, 0, 0};
  if (active)
    for (int d = 0; d < 3; ++d) x[d] = (R)(tgt[(size_t)d * ntgt + t] - o[d]);
  double g0 = 0.0, g1 = 0.0, g2 = 0.0;
  const int chunk = (nsrc + GSPLIT - 1) / GSPLIT;
  const int s0 = blockIdx.y * chunk, s1 = min(nsrc, s0 + chunk);
  for (int base = s0; base < s1; base += GS) {
    int cnt = min(GS, s1 - base);
    __syncthreads();
    for (int j = threadIdx.x; j < cnt; j += GT * TPT) {
      for (int d = 0; d < 3; ++d) s_y[d][j] = (R)(src[(size_t)d * nsrc + base + j] - o[d]);
      s_q[j] = (R)q[base + j];
    }
    __syncthreads();
    if (active) {
      // two sources per step into two sets of sums (independent dependency chains)
      R a0 = 0, a1 = 0, a2 = 0, b0 = 0, b1 = 0, b2 = 0;
      int j = sub;
      for (; j + TPT < cnt; j += 2 * TPT) {
        const int k = j + TPT;
        R dx = x[0] - s_y[0][j], dy = x[1] - s_y[1][j], dz = x[2] - s_y[2][j];
        R ex = x[0] - s_y[0][k], ey = x[1] - s_y[1][k], ez = x[2] - s_y[2][k];
        R r2 = dx * dx + dy * dy + dz * dz;
        R e2 = ex * ex + ey * ey + ez * ez;
        R ri = r2 > R(0) ? rsqrt(r2) : R(0);
        R ei = e2 > R(0) ? rsqrt(e2) : R(0);
        R f = s_q[j] * ri * ri * ri;
        R fe = s_q[k] * ei * ei * ei;
        a0 = fma(f, dx, a0);
        a1 = fma(f, dy, a1);
        a2 = fma(f, dz, a2);
        b0 = fma(fe, ex, b0);
        b1 = fma(fe, ey, b1);
        b2 = fma(fe, ez, b2);
      }
      if (j < cnt) {
        R dx = x[0] - s_y[0][j], dy = x[1] - s_y[1][j], dz = x[2] - s_y[2][j];
        R r2 = dx * dx + dy * dy + dz * dz;
        R ri = r2 > R(0) ? rsqrt(r2) : R(0);
        R f = s_q[j] * ri * ri * ri;
        a0 = fma(f, dx, a0);
        a1 = fma(f, dy, a1);
        a2 = fma(f, dz, a2);
      }
      g0 += (double)a0 + (double)b0;
      g1 += (double)a1 + (double)b1;
      g2 += (double)a2 + (double)b2;
    }
  }
  s_part[0][sub][tl] = g0;
  s_part[1][sub][tl] = g1;
  s_part[2][sub][tl] = g2;
  __syncthreads();
  if (sub == 0) {
    for (int u = 1; u < TPT; ++u) {
      g0 += s_part[0][u][tl];
      g1 += s_part[1][u][tl];
      g2 += s_part[2][u][tl];
    }
    s_part[0][0][tl] = g0;
    s_part[1][0][tl] = g1;
    s_part[2][0][tl] = g2;
  }
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();
  if (blockIdx.y == 0 && sub == 0 && active) {
    for (unsigned r = 1; r < GSPLIT; ++r) {
      const double* pr = cl.map_shared_rank(&s_part[0][0][0], r);
      g0 += pr[tl];
      g1 += pr[TPT * GT + tl];
      g2 += pr[2 * TPT * GT + tl];
    }
    const double c = -0.079577471545947667884;   // -1 / (4 pi)
    grad[t] = c * g0;
    grad[(size_t)ntgt + t] = c * g1;
    grad[2 * (size_t)ntgt + t] = c * g2;
  }
  cl.sync();
}

}  // namespace

}  // namespace qbx

extern "C" int qbxfmm_laplace3d_grad_direct_f32(int nsources, const double* sources,
                                                const double* charges, int ntargets,
                                                const double* targets, double* grad, void* stream)
{
  if (nsources < 0 || ntargets < 0 || (nsources > 0 && (!sources || !charges)) ||
      (ntargets > 0 && (!targets || !grad)))
    return qbx::set_last_error(QBXFMM_ERR_ARG, "qbxfmm_laplace3d_grad_direct_f32: bad arguments");
  if (ntargets == 0) return QBXFMM_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  dim3 grid((ntargets + qbx::GT - 1) / qbx::GT, qbx::GSPLIT);
  qbx::k_lap3_grad_direct<true><<<grid, qbx::GT * qbx::TPT, 0, st>>>(
      nsources, sources, charges, ntargets, targets, grad);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return qbx::set_last_error(QBXFMM_ERR_CUDA, std::string("qbxfmm_laplace3d_grad_direct_f32: ") +
                                                    cudaGetErrorString(e));
  return QBXFMM_OK;
}

extern "C" int qbxfmm_laplace3d_grad_direct(int nsources, const double* sources,
                                            const double* charges, int ntargets,
                                            const double* targets, double* grad, void* stream)
{
  if (nsources < 0 || ntargets < 0 || (nsources > 0 && (!sources || !charges)) ||
      (ntargets > 0 && (!targets || !grad)))
    return qbx::set_last_error(QBXFMM_ERR_ARG, "qbxfmm_laplace3d_grad_direct: bad arguments");
  if (ntargets == 0) return QBXFMM_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  dim3 grid((ntargets + qbx::GT - 1) / qbx::GT, qbx::GSPLIT);
  qbx::k_lap3_grad_direct<false><<<grid, qbx::GT * qbx::TPT, 0, st>>>(
      nsources, sources, charges, ntargets, targets, grad);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return qbx::set_last_error(QBXFMM_ERR_CUDA, std::string("qbxfmm_laplace3d_grad_direct: ") +
                                                    cudaGetErrorString(e));
  return QBXFMM_OK;
}
