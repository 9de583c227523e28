// Laplace expansion arithmetic (2D complex-analytic, 3D solid harmonics), float64.
//
// 3D: R_n^m(v) = r^n P_n^m(cos t) e^{imp} / (n+m)!, S_n^m(v) = (n-m)! P_n^m e^{imp} / r^{n+1}
// (no Condon-Shortley phase), negative m via X_n^{-m} = (-1)^m conj(X_n^m).  With
// 1/|x-y| = sum conj(R_n^m(y)) S_n^m(x), multipoles are M = sum q conj(R(y-c)) and
// locals phi(x) = sum L conj(R(x-c)) with L = sum q S(y-c).  Coefficients are
// scaled by rscale^n (multipoles divided, locals multiplied).  Gradients:
//   d.grad R_n^m = dz R_{n-1}^m + (dx+i dy)/2 R_{n-1}^{m-1} - (dx-i dy)/2 R_{n-1}^{m+1}
//   d.grad S_n^m = -dz S_{n+1}^m + (dx+i dy)/2 S_{n+1}^{m-1} - (dx-i dy)/2 S_{n+1}^{m+1}
// 2D: multipole Re[M_0 log(z-c) + sum_k M_k (z-c)^-k], local Re sum L_k (z-c)^k.
#pragma once

#include "common.cuh"

namespace qbx {

// decode a 3D coefficient index -> (n, m) for the triangular layout idx3(n, m)
QBX_HD void decode3(int c, int& n, int& m)
{
  n = (int)((sqrt(8.0 * c + 1.0) - 1.0) * 0.5);
  while ((n + 1) * (n + 2) / 2 <= c) ++n;
  while (n * (n + 1) / 2 > c) --n;
  m = c - n * (n + 1) / 2;
}

// {{{ 3D M2L offset symmetries
//
// The 16 isometries that map the box lattice to itself and the z axis to itself,
// sigma = R^q C^s Z^t (R: quarter turn about z, (x, y) -> (-y, x); C: y -> -y;
// Z: z -> -z; code q | s << 2 | t << 3), act on the stored coefficients (m >= 0) by
// one phase and an optional conjugation each: from S_n^m(R v) = i^m S_n^m(v),
// S_n^m(C v) = conj S_n^m(v), S_n^m(Z v) = (-1)^(n+m) S_n^m(v), the M2L matrix of the
// offset sigma d is
//   T(sigma d) M = Phi_out( T(d) Phi_in(M) ),
//   Phi_in(M)_k^l  = i^(2t(k+l) + (s ? -lq : lq)) conj^s(M_k^l),
//   Phi_out(L)_j^i = i^(2t(j+i) + iq) conj^s(L_j^i),
// so every list-2 offset uses the matrix of one canonical offset (dx >= dy >= 0,
// dz >= 0).

// largest real entry count (2 x coefficients) the class kernels' op tables hold
constexpr int M2L_SYM_MAXR = 1024;

// triangular index -> (n, m), single precision start (exact for c < 2^20)
QBX_D void coef_nm3(int c, int& n, int& m)
{
  int nn = (int)((sqrtf(8.0f * c + 1.0f) - 1.0f) * 0.5f);
  while ((nn + 1) * (nn + 2) / 2 <= c) ++nn;
  while (nn * (nn + 1) / 2 > c) --nn;
  n = nn;
  m = c - nn * (nn + 1) / 2;
}

// key of the stored coefficient c: (n + m) mod 2 | (m mod 4) << 1 (all the maps need)
QBX_D int m2l_sym_key(int c)
{
  int n, m;
  coef_nm3(c, n, m);
  return ((n + m) & 1) | ((m & 3) << 1);
}

// Each map sends a coefficient (a, b) to i^e conj^s(a + ib): entry `part` of the result
// is +-a or +-b.  Returned: bit 0 = take the other entry of the coefficient (k ^ 1),
// bit 1 = negate.  Phi_in (out = false) or Phi_out (out = true) of the coefficient
// with key `key`.
QBX_D int m2l_sym_op(int key, int sym, bool out, int part)
{
  const int q = sym & 3, s = (sym >> 2) & 1, t = (sym >> 3) & 1;
  const int m4 = key >> 1;
  const int e = (2 * t * (key & 1) + ((s && !out) ? -m4 * q : m4 * q)) & 3;
  int neg;
  if (part == 0) neg = e == 2 || (e == 1 && !s) || (e == 3 && s);
  else neg = e == 3 || (e == 0 && s) || (e == 2 && !s);
  return (e & 1) | neg << 1;
}

// the per-CTA op tables of a class symmetry: op_in[k], op_out[k] for real entries k < R
QBX_D void m2l_sym_tables(int sym, int R, uint8_t* op_in, uint8_t* op_out, int tid, int nt)
{
  for (int k = tid; k < R; k += nt) {
    const int key = m2l_sym_key(k >> 1);
    op_in[k] = (uint8_t)m2l_sym_op(key, sym, false, k & 1);
    op_out[k] = (uint8_t)m2l_sym_op(key, sym, true, k & 1);
  }
}

// entry k of a mapped vector x (interleaved re, im) by its op
QBX_D double m2l_sym_apply(const double* x, int k, int op)
{
  const double v = __ldg(x + (k ^ (op & 1)));
  return (op & 2) ? -v : v;
}

// }}}

// {{{ 3D single entries by recurrence along n (used where a thread owns one coefficient)

QBX_D double2 sh3_R_nm(int n, int m, double x, double y, double z)
{
  int am = m < 0 ? -m : m;
  if (n < 0 || am > n) return c2(0.0);
  double r2 = x * x + y * y + z * z;
  double2 a = c2(1.0);
  for (int j = 1; j <= am; ++j) a = cscale(0.5 * rcp(j), cmul(a, c2(x, y)));
  double2 prev = c2(0.0);
  for (int k = am + 1; k <= n; ++k) {
    double2 b = cscale(rcp(k + am) * rcp(k - am),
                       csub(cscale((2.0 * k - 1) * z, a), cscale(r2, prev)));
    prev = a;
    a = b;
  }
  if (m < 0) {
    a = cconj(a);
    if (am & 1) a = c2(-a.x, -a.y);
  }
  return a;
}

QBX_D double2 sh3_S_nm(int n, int m, double x, double y, double z)
{
  int am = m < 0 ? -m : m;
  if (n < 0 || am > n) return c2(0.0);
  double r2 = x * x + y * y + z * z;
  double rinv2 = 1.0 / r2;
  double2 a = c2(sqrt(rinv2));
  for (int j = 1; j <= am; ++j) a = cscale((2.0 * j - 1) * rinv2, cmul(a, c2(x, y)));
  double2 prev = c2(0.0);
  for (int k = am + 1; k <= n; ++k) {
    double2 b = cscale(rinv2, csub(cscale((2.0 * k - 1) * z, a),
                                   cscale((double)(k + am - 1) * (k - am - 1), prev)));
    prev = a;
    a = b;
  }
  if (m < 0) {
    a = cconj(a);
    if (am & 1) a = c2(-a.x, -a.y);
  }
  return a;
}

// }}}

// {{{ 3D tables built cooperatively (threads split the m columns)

QBX_D void sh3_R_table(int p, double x, double y, double z, double2* tab, int tid, int nt)
{
  double r2 = x * x + y * y + z * z;
  for (int m = tid; m <= p; m += nt) {
    double2 a = c2(1.0);
    for (int j = 1; j <= m; ++j) a = cscale(0.5 * rcp(j), cmul(a, c2(x, y)));
    tab[idx3(m, m)] = a;
    double2 prev = c2(0.0);
    for (int n = m + 1; n <= p; ++n) {
      double2 b = cscale(rcp(n + m) * rcp(n - m),
                         csub(cscale((2.0 * n - 1) * z, a), cscale(r2, prev)));
      tab[idx3(n, m)] = b;
      prev = a;
      a = b;
    }
  }
}

QBX_D void sh3_S_table(int p, double x, double y, double z, double2* tab, int tid, int nt)
{
  double r2 = x * x + y * y + z * z;
  double rinv2 = 1.0 / r2;
  for (int m = tid; m <= p; m += nt) {
    double2 a = c2(sqrt(rinv2));
    for (int j = 1; j <= m; ++j) a = cscale((2.0 * j - 1) * rinv2, cmul(a, c2(x, y)));
    tab[idx3(m, m)] = a;
    double2 prev = c2(0.0);
    for (int n = m + 1; n <= p; ++n) {
      double2 b = cscale(rinv2, csub(cscale((2.0 * n - 1) * z, a),
                                     cscale((double)(n + m - 1) * (n - m - 1), prev)));
      tab[idx3(n, m)] = b;
      prev = a;
      a = b;
    }
  }
}

// entry (n, m) of a table with symmetry for m < 0; zero outside the table's range
QBX_D double2 sh3_get(const double2* tab, int n, int m)
{
  if (n < 0) return c2(0.0);
  if (m >= 0) return (m <= n) ? tab[idx3(n, m)] : c2(0.0);
  int am = -m;
  if (am > n) return c2(0.0);
  double2 v = tab[idx3(n, am)];
  return (am & 1) ? c2(-v.x, v.y) : c2(v.x, -v.y);
}

// }}}

// {{{ 3D compile-time S table (registers) for the QBX near field

template <int NMAX>
struct SRegs {
  static constexpr int N = (NMAX + 1) * (NMAX + 2) / 2;
  double2 v[N];

  QBX_D void build(double x, double y, double z, double rinv, double rinv2)
  {
    double2 mm = c2(rinv);
#pragma unroll
    for (int m = 0; m <= NMAX; ++m) {
      if (m > 0) mm = cscale((2.0 * m - 1) * rinv2, cmul(mm, c2(x, y)));
      v[idx3(m, m)] = mm;
      if (m + 1 <= NMAX) v[idx3(m + 1, m)] = cscale((2.0 * m + 1) * z * rinv2, mm);
#pragma unroll
      for (int n = m + 2; n <= NMAX; ++n)
        v[idx3(n, m)] = cscale(rinv2, csub(cscale((2.0 * n - 1) * z, v[idx3(n - 1, m)]),
                                           cscale((double)(n + m - 1) * (n - m - 1),
                                                  v[idx3(n - 2, m)])));
    }
  }

  QBX_D double2 get(int n, int m) const
  {
    if (m >= 0) return (m <= n) ? v[idx3(n, m)] : c2(0.0);
    int am = -m;
    if (am > n) return c2(0.0);
    double2 t = v[idx3(n, am)];
    return (am & 1) ? c2(-t.x, t.y) : c2(t.x, -t.y);
  }
};

template <int NMAX>
struct RRegs {
  static constexpr int N = (NMAX + 1) * (NMAX + 2) / 2;
  double2 v[N];

  QBX_D void build(double x, double y, double z)
  {
    double r2 = x * x + y * y + z * z;
    double2 mm = c2(1.0);
#pragma unroll
    for (int m = 0; m <= NMAX; ++m) {
      if (m > 0) mm = cscale(1.0 / (2 * m), cmul(mm, c2(x, y)));
      v[idx3(m, m)] = mm;
      if (m + 1 <= NMAX) v[idx3(m + 1, m)] = cscale(z, mm);
#pragma unroll
      for (int n = m + 2; n <= NMAX; ++n)
        v[idx3(n, m)] = cscale(1.0 / ((double)(n + m) * (n - m)),
                               csub(cscale((2.0 * n - 1) * z, v[idx3(n - 1, m)]),
                                    cscale(r2, v[idx3(n - 2, m)])));
    }
  }
};

// }}}

// {{{ 2D helpers

QBX_D double2 cinv(double2 a)
{
  double d = 1.0 / (a.x * a.x + a.y * a.y);
  return c2(a.x * d, -a.y * d);
}

QBX_D double2 cpow_int(double2 a, int k)
{
  double2 r = c2(1.0);
  for (int i = 0; i < k; ++i) r = cmul(r, a);
  return r;
}

QBX_D double binom(int n, int k)
{
  if (k < 0 || k > n) return 0.0;
  double r = 1.0;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

QBX_D double2 clog_(double2 a)
{
  return c2(0.5 * log(a.x * a.x + a.y * a.y), atan2(a.y, a.x));
}

// }}}

}  // namespace qbx
