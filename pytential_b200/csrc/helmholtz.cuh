// 2D Helmholtz (H2D) expansion arithmetic, float64.
//
// G = (i/4) H_0^(1)(k|x - y|).  With Z_m(u) = Z_m(k|u|) e^{i m arg u} (Z = J or
// H = J + iY), Graf's addition theorem gives the translations
//   M2M: M'_m = sum_n M_n J_{n-m}(c' - c)      L2L: L'_m = sum_n L_n J_{n-m}(c' - c)
//   M2L: L_m  = sum_n M_n H_{n-m}(c' - c)
// and the expansions M_m = sum q conj(J_m(y - c)), L_m = sum q Hb_m(y - c) with
// Hb_m(u) = H_m(k|u|) e^{-i m arg u} = (-1)^m H_{-m}(u).  Source-normal
// derivatives use (d_x + i d_y) Z_m = -k Z_{m+1}, (d_x - i d_y) Z_m = k Z_{m-1}.
// Coefficients are scaled by rscale^|m| (multipoles divided, locals multiplied).
//
// Bessel functions: J_0..J_N by Miller's backward recurrence normalized with
// J_0 + 2 sum_k J_2k = 1; Y_0, Y_1 from the CUDA math library (y0, y1) and
// Y_{n+1} = (2n/x) Y_n - Y_{n-1} (stable upward).
#pragma once

#include "common.cuh"

namespace qbx {

// J[0..N], Y[0..N] (Y only if want_y) at x > 0.
QBX_D void bessel_jy(int N, double x, double* J, double* Y, bool want_y)
{
  double xinv = 1.0 / x;
  int nmax = N > (int)x ? N : (int)x;
  int start = 2 * ((nmax + 16 + (int)sqrt(40.0 * nmax)) / 2);
  double fp1 = 0.0, f = 1e-200, sum = 0.0;
  for (int j = 0; j <= N; ++j) J[j] = 0.0;
  for (int k = start; k > 0; --k) {
    // f = f_k, fp1 = f_{k+1}; f_{k-1} = (2k/x) f_k - f_{k+1}
    double fm1 = 2.0 * k * xinv * f - fp1;
    fp1 = f;
    f = fm1;
    if (k - 1 <= N) J[k - 1] = f;
    if (((k - 1) & 1) == 0 && k - 1 > 0) sum += 2.0 * f;
    if (fabs(f) > 1e200) {
      f *= 1e-200;
      fp1 *= 1e-200;
      sum *= 1e-200;
      for (int j = k - 1; j <= N; ++j) J[j] *= 1e-200;
    }
  }
  sum += f;   // f = f_0
  double norm = 1.0 / sum;
  for (int j = 0; j <= N; ++j) J[j] *= norm;
  if (want_y) {
    Y[0] = y0(x);
    if (N >= 1) Y[1] = y1(x);
    for (int j = 1; j < N; ++j) Y[j + 1] = 2.0 * j * xinv * Y[j] - Y[j - 1];
  }
}

// Z[N + m] = Z_m(u) for m in [-N, N]; Z = J (want_h false) or H (want_h true).
QBX_D void h2_zfun(int N, double k, double ux, double uy, double* Jb, double* Yb, double2* Z,
                   bool want_h)
{
  double r = sqrt(ux * ux + uy * uy);
  if (r == 0.0) {
    // J_0(0) = 1, J_m(0) = 0; the Hankel functions are singular there
    for (int m = -N; m <= N; ++m) Z[N + m] = c2(m == 0 && !want_h ? 1.0 : 0.0);
    return;
  }
  bessel_jy(N, k * r, Jb, Yb, want_h);
  double2 e1 = c2(ux / r, uy / r);
  double2 e = c2(1.0);
  for (int m = 0; m <= N; ++m) {
    double2 z = want_h ? c2(Jb[m], Yb[m]) : c2(Jb[m]);
    double2 v = cmul(z, e);
    Z[N + m] = v;
    double2 w = cmul(z, cconj(e));     // Z_m(kr) e^{-i m th}
    Z[N - m] = (m & 1) ? c2(-w.x, -w.y) : w;
    e = cmul(e, e1);
  }
}

}  // namespace qbx
