// Direct gradient of the 3D Laplace single-layer potential at far targets, used for
// the target-position gradient of the adjoint (the forward apply's targets are far
// from the surface there, so the sum needs no QBX):
//   grad u(x_t) = -1/(4 pi) sum_y q_y (x_t - y) / |x_t - y|^3.
// A cluster of GSPLIT CTAs per 64 targets (thread = target): CTA y of the cluster takes
// the y-th contiguous chunk of the sources, streamed through shared memory in tiles
// of 256, and CTA 0 adds the GSPLIT partial sums in a fixed order through
// distributed shared memory (deterministic; a few thousand targets still fill the
// GPU).
#include <string>

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

__global__ void __cluster_dims__(1, GSPLIT, 1) __launch_bounds__(GT)
k_lap3_grad_direct(int nsrc, const double* __restrict__ src, const double* __restrict__ q,
                   int ntgt, const double* __restrict__ tgt, double* __restrict__ grad)
{
  __shared__ double s_y[3][GS], s_q[GS];
  __shared__ double s_part[3][GT];
  int t = blockIdx.x * GT + threadIdx.x;
  bool active = t < ntgt;
  double x[3] = {0, 0, 0};
  if (active)
    for (int d = 0; d < 3; ++d) x[d] = tgt[(size_t)d * ntgt + t];
  double g0 = 0.0, g1 = 0.0, g2 = 0.0;
  const int chunk = (nsrc + GSPLIT - 1) / GSPLIT;
  const int s0 = blockIdx.y * chunk, s1 = min(nsrc, s0 + chunk);
  for (int base = s0; base < s1; base += GS) {
    int cnt = min(GS, s1 - base);
    __syncthreads();
    for (int j = threadIdx.x; j < cnt; j += GT) {
      for (int d = 0; d < 3; ++d) s_y[d][j] = src[(size_t)d * nsrc + base + j];
      s_q[j] = q[base + j];
    }
    __syncthreads();
    if (active) {
      // two sources per step into two sets of sums (independent dependency chains)
      double h0 = 0.0, h1 = 0.0, h2 = 0.0;
      int j = 0;
      for (; j + 1 < cnt; j += 2) {
        double dx = x[0] - s_y[0][j], dy = x[1] - s_y[1][j], dz = x[2] - s_y[2][j];
        double ex = x[0] - s_y[0][j + 1], ey = x[1] - s_y[1][j + 1], ez = x[2] - s_y[2][j + 1];
        double r2 = dx * dx + dy * dy + dz * dz;
        double e2 = ex * ex + ey * ey + ez * ez;
        double ri = r2 > 0.0 ? rsqrt(r2) : 0.0;
        double ei = e2 > 0.0 ? rsqrt(e2) : 0.0;
        double f = s_q[j] * ri * ri * ri;
        double fe = s_q[j + 1] * ei * ei * ei;
        g0 = fma(f, dx, g0);
        g1 = fma(f, dy, g1);
        g2 = fma(f, dz, g2);
        h0 = fma(fe, ex, h0);
        h1 = fma(fe, ey, h1);
        h2 = fma(fe, ez, h2);
      }
      if (j < cnt) {
        double dx = x[0] - s_y[0][j], dy = x[1] - s_y[1][j], dz = x[2] - s_y[2][j];
        double r2 = dx * dx + dy * dy + dz * dz;
        double ri = r2 > 0.0 ? rsqrt(r2) : 0.0;
        double f = s_q[j] * ri * ri * ri;
        g0 = fma(f, dx, g0);
        g1 = fma(f, dy, g1);
        g2 = fma(f, dz, g2);
      }
      g0 += h0;
      g1 += h1;
      g2 += h2;
    }
  }
  s_part[0][threadIdx.x] = g0;
  s_part[1][threadIdx.x] = g1;
  s_part[2][threadIdx.x] = g2;
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();
  if (blockIdx.y == 0 && active) {
    for (unsigned r = 1; r < GSPLIT; ++r) {
      const double* pr = cl.map_shared_rank(&s_part[0][0], r);
      g0 += pr[threadIdx.x];
      g1 += pr[GT + threadIdx.x];
      g2 += pr[2 * GT + threadIdx.x];
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
  qbx::k_lap3_grad_direct<<<grid, qbx::GT, 0, st>>>(
      nsources, sources, charges, ntargets, targets, grad);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return qbx::set_last_error(QBXFMM_ERR_CUDA, std::string("qbxfmm_laplace3d_grad_direct: ") +
                                                    cudaGetErrorString(e));
  return QBXFMM_OK;
}
