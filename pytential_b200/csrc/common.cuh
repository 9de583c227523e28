// Shared device helpers for the QBX-FMM kernels: complex arithmetic on double2,
// geometry accessors, launch error plumbing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/qbxfmm.h"

#define QBX_HD __host__ __device__ __forceinline__
#define QBX_D __device__ __forceinline__

namespace qbx {

// {{{ complex double as double2

QBX_HD double2 c2(double re, double im = 0.0) { return make_double2(re, im); }
QBX_HD double2 cadd(double2 a, double2 b) { return c2(a.x + b.x, a.y + b.y); }
QBX_HD double2 csub(double2 a, double2 b) { return c2(a.x - b.x, a.y - b.y); }
QBX_HD double2 cscale(double s, double2 a) { return c2(s * a.x, s * a.y); }
QBX_HD double2 cconj(double2 a) { return c2(a.x, -a.y); }
QBX_HD double2 cmul(double2 a, double2 b)
{
  return c2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a * conj(b)
QBX_HD double2 cmulc(double2 a, double2 b)
{
  return c2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
// acc + a * b
QBX_HD double2 cfma(double2 a, double2 b, double2 acc)
{
  return c2(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
}
// acc + a * conj(b)
QBX_HD double2 cfmac(double2 a, double2 b, double2 acc)
{
  return c2(fma(a.x, b.x, fma(a.y, b.y, acc.x)), fma(a.y, b.x, fma(-a.x, b.y, acc.y)));
}
// acc + s * a  (s real)
QBX_HD double2 caxpy(double s, double2 a, double2 acc)
{
  return c2(fma(s, a.x, acc.x), fma(s, a.y, acc.y));
}

// }}}

QBX_HD int idx3(int n, int m) { return n * (n + 1) / 2 + m; }

inline int ncoeff(int family, int dim, int order)
{
  if (family == QBXFMM_LAPLACE) return dim == 3 ? (order + 1) * (order + 2) / 2 : order + 1;
  return dim == 3 ? (order + 1) * (order + 1) : 2 * order + 1;
}

QBX_D double level_width(const qbxfmm_geometry& g, int level)
{
  return ldexp(g.root_extent, -level);
}

template <int DIM>
QBX_D void load_point(const double* __restrict__ soa, int n, int i, double* out)
{
#pragma unroll
  for (int d = 0; d < DIM; ++d) out[d] = __ldg(soa + (size_t)d * n + i);
}

// Device-side error word: the first failing kernel records a code and keeps going
// without touching out-of-range memory.
enum : int32_t { QBX_DEVERR_NONE = 0, QBX_DEVERR_BAD_BOX = 1, QBX_DEVERR_BAD_CENTER = 2 };

QBX_D void report(int32_t* err, int32_t code)
{
  if (err) atomicCAS(err, 0, code);
}

// Laplace coefficients and their ratio, resolved once per call on the host
struct SourceCoeffs {
  double cq;   // single-layer weight
  double cd;   // double-layer weight
};

}  // namespace qbx
