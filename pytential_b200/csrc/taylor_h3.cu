// The reference's default truncation of the 3D Helmholtz box and QBX expansions
// (sumpy's PDE-compressed Cartesian Taylor expansions, chosen by pytential's
// QBXDefaultExpansionFactory, pytential/qbx/__init__.py:98-112), kept in the
// library's spherical-wave coefficients.
//
// In wave units v = k x, a degree-p local about a center is the polynomial
// sum_nm b_nm f_nm(v) with f_nm(v) = j_n^[p](|v|) Y_n^m(v) (j_n cut to its power
// series of total degree p; b_nm = L_nm / s^n in the library's scaled coefficients).
// sumpy stores the Taylor coefficients whose exponent of z is <= 1 (the PDE
// eliminates u_zz) and rebuilds the others from the PDE, which is exactly what the
// basis f_nm spans; so
//   L2L (and L2QBXL, to order q): b' = Ginv * (stored coefficients of the local
//     polynomial re-centered at the new center),
//   M2M: the transpose of that map with m -> -m (sumpy translates a child's stored
//     moments with the others taken as zero; in these coefficients that is
//     (Ginv G(d))^T),
// where G(d)[s][nm] = [v^(stored s)] f_nm(v + k d) and Ginv = G(0)^-1.  The host part
// below builds the monomial tables, G(0)^-1 and the per-(level, child position) M2M /
// L2L matrices; the device part is the L2QBXL kernel, which expands each box local
// to its monomials once and re-centers it at each QBX center.
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <thread>
#include <vector>

#include "../../include/qbxfmm_api.h"
#include "kernels.h"
#include "taylor_h3.h"

namespace qbx {

// {{{ host tables

namespace {

using lcd = std::complex<long double>;

int cube(int a, int b, int c, int D1) { return (a * D1 + b) * D1 + c; }

// dense polynomial product in the cube layout, truncated at total degree D1 - 1
void poly_mul(const std::vector<lcd>& A, const std::vector<lcd>& B, std::vector<lcd>& C, int D1)
{
  const int D = D1 - 1;
  std::fill(C.begin(), C.end(), lcd(0));
  for (int a = 0; a <= D; ++a)
    for (int b = 0; a + b <= D; ++b)
      for (int c = 0; a + b + c <= D; ++c) {
        lcd x = A[cube(a, b, c, D1)];
        if (x == lcd(0)) continue;
        for (int a2 = 0; a + a2 <= D; ++a2)
          for (int b2 = 0; a + a2 + b + b2 <= D; ++b2)
            for (int c2_ = 0; a + a2 + b + b2 + c + c2_ <= D; ++c2_) {
              lcd y = B[cube(a2, b2, c2_, D1)];
              if (y != lcd(0)) C[cube(a + a2, b + b2, c + c2_, D1)] += x * y;
            }
      }
}

// Gauss-Jordan inverse with partial pivoting, long double
bool invert(std::vector<lcd>& A, std::vector<lcd>& Ai, int n)
{
  Ai.assign((size_t)n * n, lcd(0));
  for (int i = 0; i < n; ++i) Ai[(size_t)i * n + i] = 1;
  for (int col = 0; col < n; ++col) {
    int piv = col;
    for (int r = col + 1; r < n; ++r)
      if (std::abs(A[(size_t)r * n + col]) > std::abs(A[(size_t)piv * n + col])) piv = r;
    if (std::abs(A[(size_t)piv * n + col]) == 0) return false;
    if (piv != col)
      for (int j = 0; j < n; ++j) {
        std::swap(A[(size_t)piv * n + j], A[(size_t)col * n + j]);
        std::swap(Ai[(size_t)piv * n + j], Ai[(size_t)col * n + j]);
      }
    lcd d = lcd(1) / A[(size_t)col * n + col];
    for (int j = 0; j < n; ++j) {
      A[(size_t)col * n + j] *= d;
      Ai[(size_t)col * n + j] *= d;
    }
    for (int r = 0; r < n; ++r) {
      if (r == col) continue;
      lcd f = A[(size_t)r * n + col];
      if (f == lcd(0)) continue;
      for (int j = 0; j < n; ++j) {
        A[(size_t)r * n + j] -= f * A[(size_t)col * n + j];
        Ai[(size_t)r * n + j] -= f * Ai[(size_t)col * n + j];
      }
    }
  }
  return true;
}

int hq_index(int n, int m) { return n * n + n + m; }

}  // namespace

int h3t_mono_index(int p, int a, int b, int c)
{
  int off = 0;
  for (int a2 = 0; a2 < a; ++a2) off += (p - a2 + 1) * (p - a2 + 2) / 2;
  return off + b * (p - a + 1) - b * (b - 1) / 2 + c;
}

H3TaylorHost h3_taylor_host(int p)
{
  H3TaylorHost t;
  t.p = p;
  t.ncf = (p + 1) * (p + 1);
  t.nmono = (p + 1) * (p + 2) * (p + 3) / 6;
  const int D1 = p + 1, NC = D1 * D1 * D1;
  // (x^2 + y^2 + z^2)^i
  const int nr = p / 2 + 1;
  std::vector<std::vector<lcd>> r2(nr, std::vector<lcd>(NC, lcd(0)));
  r2[0][cube(0, 0, 0, D1)] = 1;
  std::vector<lcd> base(NC, lcd(0));
  if (p >= 2) {
    base[cube(2, 0, 0, D1)] = base[cube(0, 2, 0, D1)] = base[cube(0, 0, 2, D1)] = 1;
    for (int i = 1; i < nr; ++i) poly_mul(r2[i - 1], base, r2[i], D1);
  }
  // normalized Legendre parts p_n^m(t) = sum_i A[n][m][i] t^i (Y_n^m = p_n^m sin^m e^{im phi},
  // orthonormal, no Condon-Shortley phase)
  std::vector<long double> A((size_t)D1 * D1 * D1, 0.0L);
  auto PA = [&](int n, int m, int i) -> long double& { return A[((size_t)n * D1 + m) * D1 + i]; };
  long double pmm = 0.5L / std::sqrt(3.14159265358979323846264338327950288L);
  for (int m = 0; m <= p; ++m) {
    if (m > 0) pmm *= std::sqrt((2.0L * m + 1.0L) / (2.0L * m));
    PA(m, m, 0) = pmm;
    if (m + 1 <= p)
      for (int i = 0; i < p; ++i) PA(m + 1, m, i + 1) = std::sqrt(2.0L * m + 3.0L) * PA(m, m, i);
    for (int n = m + 2; n <= p; ++n) {
      long double a = std::sqrt((4.0L * n * n - 1.0L) / ((long double)n * n - (long double)m * m));
      long double b = std::sqrt(((n - 1.0L) * (n - 1.0L) - (long double)m * m) /
                                (4.0L * (n - 1.0L) * (n - 1.0L) - 1.0L));
      for (int i = 0; i <= p; ++i)
        PA(n, m, i) = a * ((i > 0 ? PA(n - 1, m, i - 1) : 0.0L) - b * PA(n - 2, m, i));
    }
  }
  t.F.assign((size_t)t.ncf * t.nmono, std::complex<double>(0.0));
  std::vector<lcd> Q(NC), W(NC), R(NC), T(NC);
  const lcd I(0.0L, 1.0L);
  for (int n = 0; n <= p; ++n)
    for (int m = 0; m <= n; ++m) {
      // |v|^(n-m) p_n^m(z / |v|) = sum_i A_{n-m-2i} z^(n-m-2i) |v|^(2i)
      std::fill(Q.begin(), Q.end(), lcd(0));
      for (int i = 0; 2 * i <= n - m; ++i) {
        long double coef = PA(n, m, n - m - 2 * i);
        if (coef == 0.0L) continue;
        int ez = n - m - 2 * i;
        for (int a = 0; a <= p; ++a)
          for (int b = 0; a + b <= p; ++b)
            for (int c = 0; a + b + c + ez <= p; ++c) {
              lcd v = r2[i][cube(a, b, c, D1)];
              if (v != lcd(0)) Q[cube(a, b, c + ez, D1)] += coef * v;
            }
      }
      // (x + i y)^m
      std::fill(W.begin(), W.end(), lcd(0));
      long double bin = 1;
      lcd ip = 1;
      for (int j = 0; j <= m; ++j) {
        W[cube(m - j, j, 0, D1)] = bin * ip;
        bin = bin * (m - j) / (j + 1);
        ip *= I;
      }
      poly_mul(Q, W, R, D1);   // |v|^n Y_n^m
      // f_nm = sum_j c_nj |v|^(2j) |v|^n Y_n^m, c_nj = (-1)^j / (2^j j! (2n + 2j + 1)!!)
      long double dfac = 1;
      for (int i = 1; i <= n; ++i) dfac *= 2 * i + 1;
      long double cj = 1 / dfac;
      for (int j = 0; n + 2 * j <= p; ++j) {
        poly_mul(r2[j], R, T, D1);
        for (int a = 0; a <= p; ++a)
          for (int b = 0; a + b <= p; ++b)
            for (int c = 0; a + b + c <= p; ++c) {
              lcd v = cj * T[cube(a, b, c, D1)];
              if (v == lcd(0)) continue;
              int mi = h3t_mono_index(p, a, b, c);
              t.F[(size_t)hq_index(n, m) * t.nmono + mi] += std::complex<double>((double)v.real(), (double)v.imag());
              if (m > 0)
                t.F[(size_t)hq_index(n, -m) * t.nmono + mi] +=
                    std::complex<double>((double)v.real(), -(double)v.imag());
            }
        cj *= -1.0L / (2.0L * (j + 1) * (2.0L * n + 2.0L * j + 3.0L));
      }
    }
  // stored multi-indices (c <= 1) and G0 = F[nm][stored], its inverse
  for (int c = 0; c <= std::min(1, p); ++c)
    for (int a = 0; a + c <= p; ++a)
      for (int b = 0; a + b + c <= p; ++b) t.st.push_back({a, b, c});
  const int nst = (int)t.st.size();
  std::vector<lcd> G((size_t)nst * t.ncf), Gi;
  t.G0.resize((size_t)nst * t.ncf);
  for (int s = 0; s < nst; ++s)
    for (int c = 0; c < t.ncf; ++c) {
      std::complex<double> v =
          t.F[(size_t)c * t.nmono + h3t_mono_index(p, t.st[s][0], t.st[s][1], t.st[s][2])];
      t.G0[(size_t)s * t.ncf + c] = v;
      G[(size_t)s * t.ncf + c] = lcd(v.real(), v.imag());
    }
  if (!invert(G, Gi, nst)) {
    t.p = -1;
    return t;
  }
  t.Ginv.resize((size_t)t.ncf * nst);
  for (size_t i = 0; i < Gi.size(); ++i)
    t.Ginv[i] = std::complex<double>((double)Gi[i].real(), (double)Gi[i].imag());
  return t;
}

// C = Ginv * G(vd), G(vd)[s][nm] = [v^(stored s)] f_nm(v + vd): the L2L map of the
// basis coefficients (ncf x ncf, row-major [nm_out][nm_in]).
void h3_taylor_translation(const H3TaylorHost& t, const double vd[3], std::complex<double>* C)
{
  const int p = t.p, ncf = t.ncf, nst = (int)t.st.size();
  std::vector<std::complex<double>> Gd((size_t)nst * ncf);
  std::vector<double> bx((size_t)(p + 1) * (p + 1)), by_(bx.size());
  // binom(B, b) v^(B - b)
  auto table = [&](double v, std::vector<double>& out) {
    for (int B = 0; B <= p; ++B) {
      double bin = 1.0;
      for (int b = 0; b <= B; ++b) {
        out[(size_t)B * (p + 1) + b] = bin * std::pow(v, B - b);
        bin = bin * (B - b) / (b + 1);
      }
    }
  };
  table(vd[0], bx);
  table(vd[1], by_);
  std::vector<std::complex<double>> Z((size_t)(p + 1) * (p + 1) * 2), Y(Z.size());
  for (int nm = 0; nm < ncf; ++nm) {
    const std::complex<double>* F = t.F.data() + (size_t)nm * t.nmono;
    // z: value and first derivative at vd[2]
    for (int a = 0; a <= p; ++a)
      for (int b = 0; a + b <= p; ++b) {
        std::complex<double> z0 = 0.0, z1 = 0.0;
        int base = h3t_mono_index(p, a, b, 0);
        for (int c = p - a - b; c >= 0; --c) {
          z1 = z1 * vd[2] + z0;
          z0 = z0 * vd[2] + F[base + c];
        }
        Z[((size_t)a * (p + 1) + b) * 2] = z0;
        Z[((size_t)a * (p + 1) + b) * 2 + 1] = z1;
      }
    // y
    for (int a = 0; a <= p; ++a)
      for (int b = 0; a + b <= p; ++b)
        for (int cz = 0; cz <= 1; ++cz) {
          std::complex<double> acc = 0.0;
          for (int B = b; a + B <= p; ++B)
            acc += Z[((size_t)a * (p + 1) + B) * 2 + cz] * by_[(size_t)B * (p + 1) + b];
          Y[((size_t)a * (p + 1) + b) * 2 + cz] = acc;
        }
    // x, at the stored multi-indices
    for (int s = 0; s < nst; ++s) {
      int ax = t.st[s][0], b = t.st[s][1], cz = t.st[s][2];
      std::complex<double> acc = 0.0;
      for (int A = ax; A + b + cz <= p; ++A)
        acc += Y[((size_t)A * (p + 1) + b) * 2 + cz] * bx[(size_t)A * (p + 1) + ax];
      Gd[(size_t)s * ncf + nm] = acc;
    }
  }
  for (int o = 0; o < ncf; ++o) {
    std::complex<double>* Cr = C + (size_t)o * ncf;
    std::fill(Cr, Cr + ncf, std::complex<double>(0.0));
    for (int s = 0; s < nst; ++s) {
      std::complex<double> g = t.Ginv[(size_t)o * nst + s];
      if (g == 0.0) continue;
      const std::complex<double>* Gs = Gd.data() + (size_t)s * ncf;
      for (int i = 0; i < ncf; ++i) Cr[i] += g * Gs[i];
    }
  }
}

// The M2M (parent levels 0 .. nlevels-2) and L2L (child levels 1 .. nlevels-1)
// matrices of every child position, in the layout of k_h3_trans_build (real rp x kp,
// row = output (nu, mu), column = input (n, m), complex entry v as [[Re, -Im],
// [Im, Re]], with the coefficient scalings of the multipoles (M s^n) and locals
// (L s^-n) folded in), written into T at the M2M and L2L bases of tc.
cudaError_t h3_taylor_translations(const H3TaylorHost& t, const TransCfg& tc, double k,
                                   double root_extent, int nlevels, double* T, cudaStream_t st)
{
  if (nlevels < 2) return cudaSuccess;
  const int p = t.p, ncf = t.ncf;
  const int npairs = nlevels - 1;          // (parent level, child level) pairs
  const size_t stride = (size_t)tc.rp * tc.kp;
  std::vector<std::complex<double>> C((size_t)npairs * 8 * ncf * ncf);
  unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (unsigned w = 0; w < nth; ++w)
    pool.emplace_back([&, w]() {
      for (int job = (int)w; job < npairs * 8; job += (int)nth) {
        int lev = job / 8, ci = job % 8;          // parent level, child position
        double wp = std::ldexp(root_extent, -lev);
        double vd[3];
        for (int d = 0; d < 3; ++d) vd[d] = k * (((ci >> d) & 1) ? 0.25 : -0.25) * wp;
        h3_taylor_translation(t, vd, C.data() + (size_t)job * ncf * ncf);
      }
    });
  for (auto& th : pool) th.join();
  std::vector<double> M(stride);
  auto put = [&](int o, int i, std::complex<double> v) {
    size_t r0 = (size_t)(2 * o) * tc.kp + 2 * i;
    M[r0] = v.real();
    M[r0 + 1] = -v.imag();
    M[r0 + tc.kp] = v.imag();
    M[r0 + tc.kp + 1] = v.real();
  };
  for (int lev = 0; lev < npairs; ++lev) {
    double sp = std::min(1.0, k * std::ldexp(root_extent, -lev));
    double sc = std::min(1.0, k * std::ldexp(root_extent, -(lev + 1)));
    for (int ci = 0; ci < 8; ++ci) {
      const std::complex<double>* Cj = C.data() + (size_t)(lev * 8 + ci) * ncf * ncf;
      for (int kind = 0; kind < 2; ++kind) {   // 0: M2M (parent lev), 1: L2L (child lev + 1)
        std::fill(M.begin(), M.end(), 0.0);
        for (int nu = 0; nu <= p; ++nu)
          for (int mu = -nu; mu <= nu; ++mu)
            for (int n = 0; n <= p; ++n)
              for (int m = -n; m <= n; ++m) {
                std::complex<double> v;
                if (kind == 0)   // M_par[nu mu] = sp^-nu sum C[(n,-m)][(nu,-mu)] sc^n M_child[n m]
                  v = Cj[(size_t)hq_index(n, -m) * ncf + hq_index(nu, -mu)] *
                      (std::pow(sc, n) / std::pow(sp, nu));
                else             // L_child[nu mu] = sc^nu sum C[(nu,mu)][(n,m)] sp^-n L_par[n m]
                  v = Cj[(size_t)hq_index(nu, mu) * ncf + hq_index(n, m)] *
                      (std::pow(sc, nu) / std::pow(sp, n));
                put(hq_index(nu, mu), hq_index(n, m), v);
              }
        size_t mi = kind == 0 ? tc.m2m_base + (size_t)lev * 8 + ci
                              : tc.l2l_base + (size_t)(lev + 1) * 8 + ci;
        cudaError_t e = cudaMemcpyAsync(T + mi * stride, M.data(), stride * sizeof(double),
                                        cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
      }
    }
  }
  return cudaSuccess;
}

// }}}

// {{{ L2QBXL

namespace {

constexpr int TNT = 128;

// CTA = one chunk of <= 32 QBX centers of one target box x RB densities.  The box's
// local (order p) becomes its monomials in wave units once (the stored ones from the
// coefficients through G0, the others from the PDE); each (center, density) item
// re-centers the polynomial at its center (z, then y, then x, keeping the exponents
// the order-q QBX local stores) and converts with Ginv_q.
template <int Q, int RB>
__global__ void __launch_bounds__(TNT)
k_h3_l2qbxl_taylor(qbxfmm_geometry g, HelmCoeffs hc, int p, int nrhs,
                   const double2* __restrict__ locals, const double2* __restrict__ G0,
                   const double2* __restrict__ Gq, double2* __restrict__ qbx_exps, int32_t* err)
{
  constexpr int NCQ = (Q + 1) * (Q + 1);
  constexpr int NS0 = (Q + 1) * (Q + 2) / 2;   // stored exponents with c = 0 (then c = 1)
  extern __shared__ double2 smem2[];
  const int ncf = (p + 1) * (p + 1);
  const int nmono = (p + 1) * (p + 2) * (p + 3) / 6;
  double2* P = smem2;                          // [nmono][RB]
  double2* bsh = P + (size_t)nmono * RB;       // [ncf][RB]
  double2* Gs = bsh + (size_t)ncf * RB;        // [NCQ][NCQ]
  __shared__ int offA[H3T_MAXP + 2];
  __shared__ int s_st[H3T_MAXP2 * 3];          // stored exponents of the box local

  const int chunk = blockIdx.x, r0 = blockIdx.y * RB;
  const int itb = g.qbx_chunk_target_box[chunk];
  const int nctr = g.qbx_chunk_count[chunk];
  if ((unsigned)itb >= (unsigned)g.ntarget_boxes) {
    if (threadIdx.x == 0) report(err, QBX_DEVERR_BAD_BOX);
    return;
  }
  const int tb = g.target_boxes[itb];
  if ((unsigned)tb >= (unsigned)g.nboxes) {
    if (threadIdx.x == 0) report(err, QBX_DEVERR_BAD_BOX);
    return;
  }
  const double k = hc.k;
  const double sb = fmin(1.0, k * level_width(g, g.box_levels[tb]));
  if (threadIdx.x <= p + 1) {
    int off = 0;
    for (int a2 = 0; a2 < (int)threadIdx.x; ++a2) off += (p - a2 + 1) * (p - a2 + 2) / 2;
    offA[threadIdx.x] = off;
  }
  if (threadIdx.x == 0) {
    int s = 0;
    for (int c = 0; c <= 1 && c <= p; ++c)
      for (int a = 0; a + c <= p; ++a)
        for (int b = 0; a + b + c <= p; ++b) {
          s_st[3 * s] = a;
          s_st[3 * s + 1] = b;
          s_st[3 * s + 2] = c;
          ++s;
        }
  }
  for (int e = threadIdx.x; e < ncf * RB; e += TNT) {
    int c = e / RB, rr = e - c * RB;
    int n = (int)sqrt((double)c);
    while (n * n > c) --n;
    while ((n + 1) * (n + 1) <= c) ++n;
    double2 v = c2(0.0);
    if (r0 + rr < nrhs)
      v = cscale(pow(sb, -(double)n), locals[((size_t)tb * nrhs + r0 + rr) * ncf + c]);
    bsh[e] = v;
  }
  for (int e = threadIdx.x; e < NCQ * NCQ; e += TNT) Gs[e] = Gq[e];
  __syncthreads();
  auto mono = [&](int a, int b, int c) { return offA[a] + b * (p - a + 1) - b * (b - 1) / 2 + c; };
  // stored monomials: P[st_s] = sum_nm G0[s][nm] b[nm], over the (n, m) that can have a
  // term x^a y^b z^c: n <= a+b+c of its parity, |m| <= a+b of the parity of a+b
  for (int e = threadIdx.x; e < ncf * RB; e += TNT) {
    int s = e / RB, rr = e - s * RB;
    int a = s_st[3 * s], b = s_st[3 * s + 1], c = s_st[3 * s + 2];
    int D = a + b + c, ab = a + b;
    double2 acc = c2(0.0);
    for (int n = D & 1; n <= D; n += 2) {
      int mm = min(n, ab);
      for (int m = -mm; m <= mm; ++m) {
        if (((m + ab) & 1) != 0) continue;
        int col = n * n + n + m;
        acc = cfma(G0[(size_t)s * ncf + col], bsh[col * RB + rr], acc);
      }
    }
    P[(size_t)mono(a, b, c) * RB + rr] = acc;
  }
  __syncthreads();
  // the others from the PDE in wave units (Delta u + u = 0), by increasing exponent of z
  for (int c = 2; c <= p; ++c) {
    const int nab = (p - c + 1) * (p - c + 2) / 2;
    for (int e = threadIdx.x; e < nab * RB; e += TNT) {
      int w = e / RB, rr = e - w * RB;
      int a = 0, rem = w;
      while (rem >= p - c - a + 1) {
        rem -= p - c - a + 1;
        ++a;
      }
      int b = rem;
      double2 v = cscale((a + 1.0) * (a + 2.0), P[(size_t)mono(a + 2, b, c - 2) * RB + rr]);
      v = caxpy((b + 1.0) * (b + 2.0), P[(size_t)mono(a, b + 2, c - 2) * RB + rr], v);
      v = cadd(v, P[(size_t)mono(a, b, c - 2) * RB + rr]);
      P[(size_t)mono(a, b, c) * RB + rr] = cscale(-1.0 / (c * (c - 1.0)), v);
    }
    __syncthreads();
  }
  // items: (center, density)
  const int item = threadIdx.x, ci = item / RB, rr = item - ci * RB;
  if (ci >= nctr || ci >= TNT / RB || r0 + rr >= nrhs) return;
  const int ctr = g.centers_by_target_box[g.qbx_chunk_start[chunk] + ci];
  if ((unsigned)ctr >= (unsigned)g.ncenters) {
    report(err, QBX_DEVERR_BAD_CENTER);
    return;
  }
  double cc[3], cb[3];
  load_point<3>(g.centers, g.ncenters, ctr, cc);
  load_point<3>(g.box_centers, g.nboxes, tb, cb);
  const double vx = k * (cc[0] - cb[0]), vy = k * (cc[1] - cb[1]), vz = k * (cc[2] - cb[2]);
  double2 O[NCQ];
#pragma unroll
  for (int i = 0; i < NCQ; ++i) O[i] = c2(0.0);
  double px[Q + 1];   // binom(A, ax) vx^(A - ax)
#pragma unroll
  for (int i = 0; i <= Q; ++i) px[i] = i == 0 ? 1.0 : 0.0;
  for (int A = 0; A <= p; ++A) {
    double2 Y0[Q + 1], Y1[Q + 1];
#pragma unroll
    for (int i = 0; i <= Q; ++i) Y0[i] = Y1[i] = c2(0.0);
    double py[Q + 1];
#pragma unroll
    for (int i = 0; i <= Q; ++i) py[i] = i == 0 ? 1.0 : 0.0;
    for (int B = 0; A + B <= p; ++B) {
      const double2* col = P + (size_t)mono(A, B, 0) * RB + rr;
      const int nC = p - A - B;
      double2 z0 = col[(size_t)nC * RB], z1 = c2(0.0);
      for (int C = nC - 1; C >= 0; --C) {
        z1 = caxpy(vz, z1, z0);
        z0 = caxpy(vz, z0, col[(size_t)C * RB]);
      }
#pragma unroll
      for (int b = 0; b <= Q; ++b) {
        Y0[b] = caxpy(py[b], z0, Y0[b]);
        Y1[b] = caxpy(py[b], z1, Y1[b]);
      }
#pragma unroll
      for (int b = Q; b >= 1; --b) py[b] = fma(vy, py[b], py[b - 1]);
      py[0] *= vy;
    }
    // O[(ax, by, cz)] += binom(A, ax) vx^(A - ax) Y_cz[by]
    {
      int s = 0;
#pragma unroll
      for (int ax = 0; ax <= Q; ++ax)
#pragma unroll
        for (int b = 0; ax + b <= Q; ++b, ++s) O[s] = caxpy(px[ax], Y0[b], O[s]);
#pragma unroll
      for (int ax = 0; ax < Q; ++ax)
#pragma unroll
        for (int b = 0; ax + b < Q; ++b, ++s) O[s] = caxpy(px[ax], Y1[b], O[s]);
    }
#pragma unroll
    for (int a = Q; a >= 1; --a) px[a] = fma(vx, px[a], px[a - 1]);
    px[0] *= vx;
  }
  (void)NS0;
  // b_qbx = Ginv_q O, scaled by s_c^n into the QBX coefficients
  const double sc = fmin(1.0, k * g.expansion_radii[ctr]);
  double2* out = qbx_exps + ((size_t)ctr * nrhs + r0 + rr) * NCQ;
  double f = 1.0;
#pragma unroll
  for (int n = 0; n <= Q; ++n) {
#pragma unroll
    for (int m = -n; m <= n; ++m) {
      const int o = n * n + n + m;
      double2 acc = c2(0.0);
#pragma unroll
      for (int s = 0; s < NCQ; ++s) acc = cfma(Gs[o * NCQ + s], O[s], acc);
      out[o] = caxpy(f, acc, out[o]);
    }
    f *= sc;
  }
}

template <int Q, int RB>
cudaError_t l2qbxl_taylor_launch(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                                 const double2* lo, const double2* G0, const double2* Gq,
                                 double2* qe, int32_t* err, cudaStream_t st)
{
  constexpr int NCQ = (Q + 1) * (Q + 1);
  const int ncf = (p + 1) * (p + 1), nmono = (p + 1) * (p + 2) * (p + 3) / 6;
  size_t sh = ((size_t)nmono * RB + (size_t)ncf * RB + (size_t)NCQ * NCQ) * sizeof(double2);
  cudaError_t e = cudaFuncSetAttribute(k_h3_l2qbxl_taylor<Q, RB>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return e;
  dim3 grid(g.nqbx_chunks, (nrhs + RB - 1) / RB);
  k_h3_l2qbxl_taylor<Q, RB><<<grid, TNT, sh, st>>>(g, hc, p, nrhs, lo, G0, Gq, qe, err);
  return cudaGetLastError();
}

template <int Q>
cudaError_t l2qbxl_taylor_q(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                            const double2* lo, const double2* G0, const double2* Gq, double2* qe,
                            int32_t* err, cudaStream_t st)
{
  if (hc.rb_l2q == 4 || (hc.rb_l2q == 0 && nrhs >= 4))   // the plan's tuning, else by nrhs
    return l2qbxl_taylor_launch<Q, 4>(g, hc, p, nrhs, lo, G0, Gq, qe, err, st);
  return l2qbxl_taylor_launch<Q, 1>(g, hc, p, nrhs, lo, G0, Gq, qe, err, st);
}

}  // namespace

cudaError_t h3_launch_l2qbxl_taylor(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int q,
                                    int nrhs, const double2* lo, const double2* G0,
                                    const double2* Gq, double2* qe, int32_t* err, cudaStream_t st)
{
  if (g.nqbx_chunks == 0) return cudaSuccess;
  if (p > H3T_MAXP) return cudaErrorInvalidValue;
  switch (q) {
    case 0: return l2qbxl_taylor_q<0>(g, hc, p, nrhs, lo, G0, Gq, qe, err, st);
    case 1: return l2qbxl_taylor_q<1>(g, hc, p, nrhs, lo, G0, Gq, qe, err, st);
    case 2: return l2qbxl_taylor_q<2>(g, hc, p, nrhs, lo, G0, Gq, qe, err, st);
    case 3: return l2qbxl_taylor_q<3>(g, hc, p, nrhs, lo, G0, Gq, qe, err, st);
    case 4: return l2qbxl_taylor_q<4>(g, hc, p, nrhs, lo, G0, Gq, qe, err, st);
    case 5: return l2qbxl_taylor_q<5>(g, hc, p, nrhs, lo, G0, Gq, qe, err, st);
    default: return cudaErrorInvalidValue;
  }
}

// }}}

}  // namespace qbx
