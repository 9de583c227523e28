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

// {{{ complex float as float2 (mixed-precision far field)

QBX_HD float2 f2(float re, float im = 0.0f) { return make_float2(re, im); }
QBX_HD float2 fadd(float2 a, float2 b) { return f2(a.x + b.x, a.y + b.y); }
QBX_HD float2 fsub(float2 a, float2 b) { return f2(a.x - b.x, a.y - b.y); }
QBX_HD float2 fscale(float s, float2 a) { return f2(s * a.x, s * a.y); }
QBX_HD float2 fconj(float2 a) { return f2(a.x, -a.y); }
QBX_HD float2 fmul(float2 a, float2 b)
{
  return f2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// acc + a * b
QBX_HD float2 ffma(float2 a, float2 b, float2 acc)
{
  return f2(fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y)));
}
// acc + s * a  (s real)
QBX_HD float2 faxpy(float s, float2 a, float2 acc) { return f2(fmaf(s, a.x, acc.x), fmaf(s, a.y, acc.y)); }
QBX_HD float2 tof(double2 a) { return f2((float)a.x, (float)a.y); }
QBX_HD double2 tod(float2 a) { return c2((double)a.x, (double)a.y); }

// the double2 names for float2, so that kernels templated on the real type R (and
// its complex type, cplx_t<R>) read the same in both precisions
QBX_HD float2 cadd(float2 a, float2 b) { return fadd(a, b); }
QBX_HD float2 cscale(float s, float2 a) { return fscale(s, a); }
QBX_HD float2 cconj(float2 a) { return fconj(a); }
QBX_HD float2 cmul(float2 a, float2 b) { return fmul(a, b); }
QBX_HD float2 cfma(float2 a, float2 b, float2 acc) { return ffma(a, b, acc); }
QBX_HD float2 caxpy(float s, float2 a, float2 acc) { return faxpy(s, a, acc); }

template <typename R> struct cplx_of;
template <> struct cplx_of<double> { using type = double2; };
template <> struct cplx_of<float> { using type = float2; };
template <typename R> using cplx_t = typename cplx_of<R>::type;
template <typename R> QBX_HD cplx_t<R> cmake(R re, R im = R(0));
template <> QBX_HD double2 cmake<double>(double re, double im) { return c2(re, im); }
template <> QBX_HD float2 cmake<float>(float re, float im) { return f2(re, im); }
QBX_HD double2 cto(double2 a, double2) { return a; }
QBX_HD float2 cto(double2 a, float2) { return tof(a); }
QBX_HD double2 c2d(double2 a) { return a; }
QBX_HD double2 c2d(float2 a) { return tod(a); }

// }}}

QBX_HD int idx3(int n, int m) { return n * (n + 1) / 2 + m; }

// reciprocals of small integers (c_rcp[i] = 1/i, c_rcp[0] = 0): keeps float64
// divisions out of the expansion recurrences
static __constant__ double c_rcp[128] = {0.0, 1.0 / 1, 1.0 / 2, 1.0 / 3, 1.0 / 4, 1.0 / 5, 1.0 / 6, 1.0 / 7, 1.0 / 8, 1.0 / 9, 1.0 / 10, 1.0 / 11, 1.0 / 12, 1.0 / 13, 1.0 / 14, 1.0 / 15, 1.0 / 16, 1.0 / 17, 1.0 / 18, 1.0 / 19, 1.0 / 20, 1.0 / 21, 1.0 / 22, 1.0 / 23, 1.0 / 24, 1.0 / 25, 1.0 / 26, 1.0 / 27, 1.0 / 28, 1.0 / 29, 1.0 / 30, 1.0 / 31, 1.0 / 32, 1.0 / 33, 1.0 / 34, 1.0 / 35, 1.0 / 36, 1.0 / 37, 1.0 / 38, 1.0 / 39, 1.0 / 40, 1.0 / 41, 1.0 / 42, 1.0 / 43, 1.0 / 44, 1.0 / 45, 1.0 / 46, 1.0 / 47, 1.0 / 48, 1.0 / 49, 1.0 / 50, 1.0 / 51, 1.0 / 52, 1.0 / 53, 1.0 / 54, 1.0 / 55, 1.0 / 56, 1.0 / 57, 1.0 / 58, 1.0 / 59, 1.0 / 60, 1.0 / 61, 1.0 / 62, 1.0 / 63, 1.0 / 64, 1.0 / 65, 1.0 / 66, 1.0 / 67, 1.0 / 68, 1.0 / 69, 1.0 / 70, 1.0 / 71, 1.0 / 72, 1.0 / 73, 1.0 / 74, 1.0 / 75, 1.0 / 76, 1.0 / 77, 1.0 / 78, 1.0 / 79, 1.0 / 80, 1.0 / 81, 1.0 / 82, 1.0 / 83, 1.0 / 84, 1.0 / 85, 1.0 / 86, 1.0 / 87, 1.0 / 88, 1.0 / 89, 1.0 / 90, 1.0 / 91, 1.0 / 92, 1.0 / 93, 1.0 / 94, 1.0 / 95, 1.0 / 96, 1.0 / 97, 1.0 / 98, 1.0 / 99, 1.0 / 100, 1.0 / 101, 1.0 / 102, 1.0 / 103, 1.0 / 104, 1.0 / 105, 1.0 / 106, 1.0 / 107, 1.0 / 108, 1.0 / 109, 1.0 / 110, 1.0 / 111, 1.0 / 112, 1.0 / 113, 1.0 / 114, 1.0 / 115, 1.0 / 116, 1.0 / 117, 1.0 / 118, 1.0 / 119, 1.0 / 120, 1.0 / 121, 1.0 / 122, 1.0 / 123, 1.0 / 124, 1.0 / 125, 1.0 / 126, 1.0 / 127};

QBX_D double rcp(int i) { return c_rcp[i]; }

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
// device error word codes: an out-of-range list entry (box, center), or a bulk copy
// whose completion wait ran out
enum : int32_t {
  QBX_DEVERR_NONE = 0,
  QBX_DEVERR_BAD_BOX = 1,
  QBX_DEVERR_BAD_CENTER = 2,
  QBX_DEVERR_COPY_TIMEOUT = 3
};

QBX_D void report(int32_t* err, int32_t code)
{
  if (err) atomicCAS(err, 0, code);
}

// Laplace source weights, resolved once per call on the host
struct SourceCoeffs {
  double cq;   // single-layer weight
  double cd;   // double-layer weight
};

// Helmholtz source weights (complex) and wave number
struct HelmCoeffs {
  double2 cq;
  double2 cd;
  double k;
  int taylor = 0;   // 3D: the reference's default truncation (sumpy's compressed Taylor
                    // expansions: regular waves with j_n cut to its power series)
  // launch shapes picked by the plan's tuning (qbxfmm_tuning; 0: built-in choice):
  // densities per CTA of M2QBXL, M2L, P2M / P2L, L2QBXL, the target-specific near field
  int rb_rot = 0, rb_m2l = 0, rb_p2e = 0, rb_l2q = 0, rb_ts = 0;
};

}  // namespace qbx
