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
