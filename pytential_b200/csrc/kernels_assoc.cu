// Target-to-QBX-center association on the device (pytential/qbx/target_assoc.py:
// marking 544-633, center finding 243-363 and 637-749, side requests 81-103).
//
// Spatial search: uniform grids of cells no narrower than the search radius (the
// largest source tunnel radius for marking, the largest tolerant center radius for
// center finding), points sorted by cell key by the caller; a target scans the 3^dim
// cells around its own, a superset of the points within the radius.  The candidate
// tests and the choice among candidates are the reference's and do not depend on the
// visiting order, so the result equals the host restatement's bit for bit: distances
// are sqrt((d0 d0 + d1 d1) + d2 d2) of (point - target) with every operation rounded
// separately (no contraction into fused multiply-adds), as numpy evaluates
// ``norm(p - t, axis=0)``, and relative distances are one rounded division.
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/qbxfmm_api.h"

namespace qbx {

int set_last_error(int code, const std::string& msg);

namespace {

constexpr int32_t ASSOC_NO_QBX = -1;
constexpr int32_t ASSOC_FAILED = -2;

__device__ __forceinline__ int64_t cell_of(double x, double lo, double h, int64_t n)
{
  double u = floor(__ddiv_rn(__dsub_rn(x, lo), h));
  int64_t i = u < 0.0 ? 0 : (int64_t)u;
  return i >= n ? n - 1 : i;
}

__device__ __forceinline__ int64_t key_of(const qbxfmm_cell_grid& gr, const int64_t* c)
{
  return (c[0] * gr.ncells[1] + c[1]) * gr.ncells[2] + c[2];
}

__device__ __forceinline__ double dist(int dim, const double* pts, int64_t np, int64_t i,
                                       const double* t)
{
  double s = 0.0;
  for (int d = 0; d < dim; ++d) {
    double v = __dsub_rn(pts[(size_t)d * np + i], t[d]);
    double q = __dmul_rn(v, v);
    s = d == 0 ? q : __dadd_rn(s, q);
  }
  return __dsqrt_rn(s);
}

// first index in keys[0, n) with keys[i] >= k
__device__ __forceinline__ int64_t lower(const int64_t* keys, int64_t n, int64_t k)
{
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (keys[mid] < k) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void k_cell_keys(int dim, int n, const double* __restrict__ pts, qbxfmm_cell_grid gr,
                            int64_t* __restrict__ keys)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t c[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) c[d] = cell_of(pts[(size_t)d * n + i], gr.lo[d], gr.h, gr.ncells[d]);
  keys[i] = key_of(gr, c);
}

// Calls f(j) for every sorted position j of the cells around the target's cell.
template <class F>
__device__ __forceinline__ void for_neighbors(int dim, const qbxfmm_cell_grid& gr,
                                              const int64_t* keys, int64_t n, const double* t,
                                              F&& f)
{
  int64_t c0[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) c0[d] = cell_of(t[d], gr.lo[d], gr.h, gr.ncells[d]);
  int lim2 = dim == 3 ? 1 : 0;
  for (int a = -1; a <= 1; ++a) {
    int64_t x = c0[0] + a;
    if (x < 0 || x >= gr.ncells[0]) continue;
    for (int b = -1; b <= 1; ++b) {
      int64_t y = c0[1] + b;
      if (y < 0 || y >= gr.ncells[1]) continue;
      for (int e = -lim2; e <= lim2; ++e) {
        int64_t z = c0[2] + e;
        if (z < 0 || z >= gr.ncells[2]) continue;
        int64_t c[3] = {x, y, z};
        int64_t k = key_of(gr, c);
        for (int64_t j = lower(keys, n, k); j < n && keys[j] == k; ++j) f(j);
      }
    }
  }
}

__global__ void k_associate(qbxfmm_assoc_problem pb, int32_t* __restrict__ result)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pb.ntargets) return;
  const int dim = pb.dim;
  double t[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) t[d] = pb.targets[(size_t)d * pb.ntargets + i];
  const int side = pb.target_sides[i];
  // marking: surface targets always, others when inside some source's tunnel
  bool marked = side == 1 || side == -1;
  if (!marked && pb.nsources > 0) {
    for_neighbors(dim, pb.source_grid, pb.source_keys, pb.nsources, t, [&](int64_t j) {
      if (marked) return;
      int32_t s = pb.source_order[j];
      if (dist(dim, pb.sources, pb.nsources, s, t) <= pb.source_tunnel_radii[s]) marked = true;
    });
  }
  if (!marked) {
    result[i] = ASSOC_NO_QBX;
    return;
  }
  // center finding: per side the minimal relative distance (ties: lower center index),
  // then the side whose chosen center is closer (ties: interior)
  double brel[2] = {0, 0}, bd[2] = {0, 0};
  int32_t bc[2] = {-1, -1};          // [0] interior (even centers), [1] exterior (odd)
  if (pb.ncenters > 0) {
    for_neighbors(dim, pb.center_grid, pb.center_keys, pb.ncenters, t, [&](int64_t j) {
      int32_t c = pb.center_order[j];
      int cs = (c & 1) ? 1 : -1;
      if (cs * side < 0) return;
      double d = dist(dim, pb.centers, pb.ncenters, c, t);
      double rel = __ddiv_rn(d, pb.center_tolerant_radii[c]);
      if (!(rel <= 1.0)) return;
      int k = c & 1;
      if (bc[k] < 0 || rel < brel[k] || (rel == brel[k] && c < bc[k])) {
        brel[k] = rel;
        bd[k] = d;
        bc[k] = c;
      }
    });
  }
  int32_t r;
  if (bc[1] >= 0 && (bc[0] < 0 || bd[1] < bd[0])) r = bc[1];
  else if (bc[0] >= 0) r = bc[0];
  else r = ASSOC_FAILED;
  result[i] = r;
}

}  // namespace

}  // namespace qbx

extern "C" int qbxfmm_cell_keys(int dim, int n, const double* points, const qbxfmm_cell_grid* grid,
                                int64_t* keys, void* stream)
{
  if ((dim != 2 && dim != 3) || n < 0 || !grid || (n > 0 && (!points || !keys)) ||
      !(grid->h > 0.0) || grid->ncells[0] < 1 || grid->ncells[1] < 1 || grid->ncells[2] < 1 ||
      (dim == 2 && grid->ncells[2] != 1))
    return qbx::set_last_error(QBXFMM_ERR_ARG, "qbxfmm_cell_keys: bad arguments");
  if (n == 0) return QBXFMM_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  qbx::k_cell_keys<<<(n + 255) / 256, 256, 0, st>>>(dim, n, points, *grid, keys);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return qbx::set_last_error(QBXFMM_ERR_CUDA, std::string("qbxfmm_cell_keys: ") +
                                                    cudaGetErrorString(e));
  return QBXFMM_OK;
}

extern "C" int qbxfmm_associate_targets(const qbxfmm_assoc_problem* pb, int32_t* target_to_center,
                                        void* stream)
{
  if (!pb || (pb->dim != 2 && pb->dim != 3) || pb->ntargets < 0 || pb->nsources < 0 ||
      pb->ncenters < 0 || (pb->ntargets > 0 && (!pb->targets || !pb->target_sides ||
                                                 !target_to_center)) ||
      (pb->nsources > 0 && (!pb->sources || !pb->source_tunnel_radii || !pb->source_keys ||
                            !pb->source_order)) ||
      (pb->ncenters > 0 && (!pb->centers || !pb->center_tolerant_radii || !pb->center_keys ||
                            !pb->center_order)))
    return qbx::set_last_error(QBXFMM_ERR_ARG, "qbxfmm_associate_targets: bad arguments");
  if (pb->ntargets == 0) return QBXFMM_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  qbx::k_associate<<<(pb->ntargets + 127) / 128, 128, 0, st>>>(*pb, target_to_center);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return qbx::set_last_error(QBXFMM_ERR_CUDA, std::string("qbxfmm_associate_targets: ") +
                                                    cudaGetErrorString(e));
  return QBXFMM_OK;
}
