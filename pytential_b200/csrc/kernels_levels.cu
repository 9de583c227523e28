// Per-level FMM orders (the reference's fmm_level_to_order, pytential/qbx/__init__.py:
// 276-285): a plan with per-level orders stores every box expansion at the largest
// order and zeroes, after each stage that writes box expansions, the coefficients
// whose degree exceeds the order of the box's level.  For the bases whose coefficients
// do not depend on the truncation order (solid harmonics, complex Taylor, H2D
// Bessel/Hankel, spherical waves) a translation computed at the largest order from a
// truncated source and then truncated to the target's order equals the translation
// between the two orders, so the result is the reference's mixed-order FMM.
#include "common.cuh"
#include "kernels.h"

namespace qbx {

namespace {

// degree of stored coefficient i: 3D Laplace (n, m >= 0) at n (n + 1) / 2 + m,
// 2D Laplace (n) at n, 2D Helmholtz (n = -p..p) at n + p, 3D Helmholtz (n, m) at n^2 + n + m
QBX_D int coeff_degree(int family, int dim, int ncf, int i)
{
  if (family == QBXFMM_LAPLACE) {
    if (dim == 2) return i;
    int n = (int)((sqrt(8.0 * i + 1.0) - 1.0) * 0.5);
    while ((n + 1) * (n + 2) / 2 <= i) ++n;
    while (n * (n + 1) / 2 > i) --n;
    return n;
  }
  if (dim == 2) return abs(i - (ncf - 1) / 2);
  int n = (int)sqrt((double)i);
  while ((n + 1) * (n + 1) <= i) ++n;
  while (n * n > i) --n;
  return n;
}

__global__ void __launch_bounds__(256)
k_level_mask(int b0, int b1, const int32_t* __restrict__ box_levels,
             const int32_t* __restrict__ orders, int nlevels, int family, int dim, int ncf,
             int nrhs, double2* __restrict__ exps)
{
  int b = b0 + blockIdx.x;
  if (b >= b1) return;
  int lev = box_levels[b];
  if (lev < 0 || lev >= nlevels) return;
  int p = orders[lev];
  double2* e = exps + (size_t)b * nrhs * ncf;
  for (int x = threadIdx.x; x < nrhs * ncf; x += blockDim.x)
    if (coeff_degree(family, dim, ncf, x % ncf) > p) e[x] = make_double2(0.0, 0.0);
}

}  // namespace

cudaError_t launch_level_mask(const qbxfmm_geometry& g, int b0, int b1, const int32_t* orders,
                              int family, int ncf, int nrhs, double2* exps, cudaStream_t st)
{
  if (b1 <= b0) return cudaSuccess;
  k_level_mask<<<b1 - b0, 256, 0, st>>>(b0, b1, g.box_levels, orders, g.nlevels, family, g.dim,
                                        ncf, nrhs, exps);
  return cudaGetLastError();
}

}  // namespace qbx
