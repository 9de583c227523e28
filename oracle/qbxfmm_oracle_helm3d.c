/*
 * 3D Helmholtz part of the CPU checker (TEST INFRASTRUCTURE ONLY), included by
 * qbxfmm_oracle.c.
 *
 * Kernel G(x, y) = e^{ik|x-y|} / |x-y| (k real, > 0); the double layer is the
 * source-normal derivative; the scaling 1/(4 pi) is applied at assembly.
 *
 * Expansions are spherical-wave expansions, the basis of the reference's fmmlib
 * backend (pytential/qbx/fmmlib.py) and of its target-specific module
 * (pytential/qbx/target_specific/impl.pyx:363-563), which pins the near field:
 *   Y_n^m(v) = p_n^|m|(cos t) sin^|m| t e^{i m phi}, orthonormal, no Condon-Shortley
 *              phase (Y_n^-m = conj(Y_n^m)),
 *   R_n^m(v) = j_n(k|v|) Y_n^m(v),   S_n^m(v) = h_n(k|v|) Y_n^m(v)   (h = h^(1)),
 *   G(x, y) = 4 pi i k sum_{n,m} S_n^m(x - c) conj(R_n^m(y - c))      (|y-c| < |x-c|)
 *           = ik sum_n (2n+1) j_n(k|y-c|) h_n(k|x-c|) P_n(cos gamma).
 * Multipole about c: phi(x) = sum M_nm S_n^m(x - c), M_nm = 4 pi i k q R_n^-m(y - c);
 * local about c:     phi(x) = sum L_nm R_n^m(x - c), L_nm = 4 pi i k q S_n^-m(y - c).
 * Translations (addition theorem through the plane-wave representation
 * j_n Y_n^m(x) = i^-n / (4 pi) int e^{ik s.x} Y_n^m(s) ds):
 *   F_n^m(r + b) = sum_{nu,mu} c_{nu mu; n m}(b) R_nu^mu(r),
 *   c_{nu mu; n m}(b) = 4 pi sum_l i^{nu + l - n} f_l(k|b|) Y_l^{m-mu}(b) G(n,m; nu,mu; l),
 * with F = S, f = h for multipole-to-local (|r| < |b|), F = R, f = j for
 * local-to-local; multipole-to-multipole (|r| > |b|) uses f = j and S_nu^mu(r) on the
 * right.  G(n,m; nu,mu; l) = int Y_n^m conj(Y_nu^mu) conj(Y_l^{m-mu}) (Gaunt integral),
 * computed here by Gauss-Legendre quadrature in cos t (exact: the integrand is a
 * polynomial of degree <= n + nu + l).
 * Gradients (source-normal derivatives) by the ladder relations
 *   d_z F_n^m           = k (a_{n-1}^m F_{n-1}^m - a_n^m F_{n+1}^m),
 *   (d_x + i d_y) F_n^m = k (-c1 F_{n+1}^{m+1} + c2 F_{n-1}^{m+1}),
 *   (d_x - i d_y) F_n^m = k (-c3 F_{n+1}^{m-1} + c4 F_{n-1}^{m-1}),
 * a_n^m = sqrt((n+1-m)(n+1+m) / ((2n+1)(2n+3))), c1 = sg(m) A(m), c2 = -sg(m) B(m),
 * c3 = sg(-m) A(-m), c4 = -sg(-m) B(-m), A(m) = sqrt((n+m+1)(n+m+2)/((2n+1)(2n+3))),
 * B(m) = sqrt((n-m)(n-m-1)/((2n-1)(2n+1))), sg(m) = +1 for m >= 0, -1 for m < 0.
 * Coefficients are scaled with s = min(1, k rho) (rho = box width or expansion
 * radius), multipoles divided by s^n and locals multiplied by s^n, as fmmlib does.
 * j_n by Miller's backward recurrence (normalized by j_0 or j_1), h_n by the upward
 * recurrence from h_0, h_1.
 *
 * Two truncations are restated (qbxfmm_kernel.fmm_backend):
 *  - fmmlib (the reference's fmm_backend="fmmlib", pytential/qbx/fmmlib.py): the
 *    spherical-wave expansions above, translated by the addition theorem;
 *  - sumpy (the reference's default, pytential/qbx/__init__.py:98-112): sumpy's
 *    PDE-compressed Cartesian Taylor expansions of degree p (box) and q (QBX).  They
 *    are kept here in the same coefficients: a degree-p Taylor polynomial of a
 *    Helmholtz field sum L_nm j_n Y_n^m keeps the terms |v|^(n+2j) Y_n^m with
 *    n + 2j <= p, i.e. j_n replaced by its power series truncated at total degree p,
 *    j_n^[p]; a multipole formed from source moments of degree <= p has the moments
 *    j_n^[p] Y_n^-m(y - c) (j_n^[p-1] in the normal derivative of a dipole).  The
 *    stages sumpy defines through the compressed coefficients themselves are
 *    restated step by step in the monomial basis (v = k x): M2M converts the child's
 *    coefficients to its stored moments (those with exponent of z <= 1), shifts them
 *    with the other moments taken as zero, and converts the parent's full moments
 *    back; L2L and L2QBXL expand the local to its monomials, shift them to the new
 *    center, keep the coefficients with exponent of z <= 1 up to the new order and
 *    convert them back (sumpy rebuilds the others from the PDE, which is what the
 *    order-(p or q) basis j_n^[.] Y_n^m spans).
 */

#define H3Q(n, m) ((n) * (n) + (n) + (m))
#define H3_NMAX 48

/* {{{ special functions */

static void h3_sph_j(int N, double x, double* jv)
{
  for (int n = 0; n <= N; ++n) jv[n] = 0.0;
  if (x == 0.0) {
    jv[0] = 1.0;
    return;
  }
  int nmax = N > (int)x ? N : (int)x;
  int start = nmax + 16 + (int)sqrt(40.0 * (nmax + 1));
  double fp1 = 0.0, f = 1e-200, f0 = 0.0, f1 = 0.0;
  for (int n = start; n >= 1; --n) {
    double fm1 = (2.0 * n + 1.0) / x * f - fp1;   /* f_{n-1} */
    fp1 = f;
    f = fm1;
    if (n - 1 <= N) jv[n - 1] = f;
    if (n - 1 == 1) f1 = f;
    if (fabs(f) > 1e200) {
      f *= 1e-200;
      fp1 *= 1e-200;
      f1 *= 1e-200;
      for (int j = n - 1; j <= N; ++j) jv[j] *= 1e-200;
    }
  }
  f0 = f;
  double scale;
  if (x < 1.0 || fabs(sin(x)) >= 0.5) scale = (sin(x) / x) / f0;
  else scale = ((sin(x) / x - cos(x)) / x) / f1;
  for (int n = 0; n <= N; ++n) jv[n] *= scale;
}

static void h3_sph_h(int N, double x, cplx* hv)
{
  cplx e = cexp(I * x);
  hv[0] = -I * e / x;
  if (N >= 1) hv[1] = -e * (x + I) / (x * x);
  for (int n = 1; n < N; ++n) hv[n + 1] = (2.0 * n + 1.0) / x * hv[n] - hv[n - 1];
}

/* Y_n^m(v) for n <= N, all m, at Y[H3Q(n, m)] */
static void h3_ylm(int N, const double* v, cplx* Y)
{
  double r = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  double t = 1.0;
  cplx w = 0.0;
  if (r > 0.0) {
    t = v[2] / r;
    w = (v[0] + I * v[1]) / r;
  }
  double pmm = 0.5 / sqrt(M_PI);   /* p_0^0 */
  cplx wm = 1.0;
  for (int m = 0; m <= N; ++m) {
    if (m > 0) {
      pmm *= sqrt((2.0 * m + 1.0) / (2.0 * m));
      wm *= w;
    }
    double pm2 = 0.0, pm1 = pmm;
    Y[H3Q(m, m)] = pm1 * wm;
    if (m > 0) Y[H3Q(m, -m)] = conj(Y[H3Q(m, m)]);
    for (int n = m + 1; n <= N; ++n) {
      double pn;
      if (n == m + 1) {
        pn = sqrt(2.0 * m + 3.0) * t * pm1;
      } else {
        double a = sqrt((4.0 * n * n - 1.0) / ((double)n * n - (double)m * m));
        double b = sqrt(((n - 1.0) * (n - 1.0) - (double)m * m) / (4.0 * (n - 1.0) * (n - 1.0) - 1.0));
        pn = a * (t * pm1 - b * pm2);
      }
      pm2 = pm1;
      pm1 = pn;
      Y[H3Q(n, m)] = pn * wm;
      if (m > 0) Y[H3Q(n, -m)] = conj(Y[H3Q(n, m)]);
    }
  }
}

/* F_n^m(v) = f_n(k|v|) Y_n^m(v), f = j (singular = 0) or h (singular = 1), n <= N */
static void h3_waves(int N, double k, const double* v, int singular, cplx* F)
{
  double jv[H3_NMAX + 2];
  cplx hv[H3_NMAX + 2];
  double r = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  h3_ylm(N, v, F);
  if (singular) h3_sph_h(N, k * r, hv);
  else h3_sph_j(N, k * r, jv);
  for (int n = 0; n <= N; ++n)
    for (int m = -n; m <= n; ++m) F[H3Q(n, m)] *= singular ? hv[n] : jv[n];
}

static inline cplx h3_get(const cplx* F, int N, int n, int m)
{
  if (n < 0 || n > N || m > n || -m > n) return 0.0;
  return F[H3Q(n, m)];
}

/* nu . grad F_n^m from a wave table of order N >= n + 1 */
static cplx h3_dgrad(const cplx* F, int N, int n, int m, double k, const double* nu)
{
  double an = sqrt((double)(n + 1 - m) * (n + 1 + m) / ((2.0 * n + 1) * (2.0 * n + 3)));
  double anm1 = (n >= 1) ? sqrt((double)(n - m) * (n + m) / ((2.0 * n - 1) * (2.0 * n + 1))) : 0.0;
  cplx dz = k * (anm1 * h3_get(F, N, n - 1, m) - an * h3_get(F, N, n + 1, m));
  double sgp = m >= 0 ? 1.0 : -1.0, sgm = -m >= 0 ? 1.0 : -1.0;
  double Ap = sqrt((double)(n + m + 1) * (n + m + 2) / ((2.0 * n + 1) * (2.0 * n + 3)));
  double Bp = (n >= 1 && n - m - 1 >= 0)
                  ? sqrt((double)(n - m) * (n - m - 1) / ((2.0 * n - 1) * (2.0 * n + 1))) : 0.0;
  double Am = sqrt((double)(n - m + 1) * (n - m + 2) / ((2.0 * n + 1) * (2.0 * n + 3)));
  double Bm = (n >= 1 && n + m - 1 >= 0)
                  ? sqrt((double)(n + m) * (n + m - 1) / ((2.0 * n - 1) * (2.0 * n + 1))) : 0.0;
  cplx dplus = k * (-sgp * Ap * h3_get(F, N, n + 1, m + 1) - sgp * Bp * h3_get(F, N, n - 1, m + 1));
  cplx dminus = k * (-sgm * Am * h3_get(F, N, n + 1, m - 1) - sgm * Bm * h3_get(F, N, n - 1, m - 1));
  return 0.5 * (nu[0] - I * nu[1]) * dplus + 0.5 * (nu[0] + I * nu[1]) * dminus + nu[2] * dz;
}

/* }}} */

/* {{{ Gaunt table */

/* j_n^[T](x) = sum_{j: n + 2j <= T} (-x^2/2)^j x^n / (j! (2n + 2j + 1)!!), n <= N
 * (zero for n > T): the power series of j_n truncated at total degree T */
static void h3_sph_j_trunc(int N, double x, int T, double* jv)
{
  double xn = 1.0, dfac = 1.0;   /* x^n, (2n+1)!! */
  for (int n = 0; n <= N; ++n) {
    if (n > 0) {
      xn *= x;
      dfac *= 2.0 * n + 1.0;
    }
    double term = xn / dfac, acc = 0.0;
    for (int j = 0; n + 2 * j <= T; ++j) {
      acc += term;
      term *= -x * x / (2.0 * (j + 1) * (2.0 * n + 2.0 * j + 3.0));
    }
    jv[n] = acc;
  }
}

/* regular waves j_n^[T](k|v|) Y_n^m(v), n <= N */
static void h3_waves_trunc(int N, double k, const double* v, int T, cplx* F)
{
  double jv[H3_NMAX + 2];
  double r = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  h3_ylm(N, v, F);
  h3_sph_j_trunc(N, k * r, T, jv);
  for (int n = 0; n <= N; ++n)
    for (int m = -n; m <= n; ++m) F[H3Q(n, m)] *= jv[n];
}

/* Gauss-Legendre nodes/weights on [-1, 1] (Newton on P_n) */
static void h3_gauss_legendre(int n, double* x, double* w)
{
  for (int i = 0; i < n; ++i) {
    double z = cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; ++j) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      double z1 = z;
      z = z1 - p1 / pp;
      if (fabs(z - z1) < 1e-16) break;
    }
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

typedef struct {
  int p;          /* table covers n, nu <= p */
  int nl;         /* l slots: l = |n - nu| + 2 j, j < nl */
  double* G;      /* [(p+1)^2][(p+1)^2][nl] */
} h3gaunt_t;

static h3gaunt_t g_h3gaunt = {-1, 0, NULL};

static const h3gaunt_t* h3_gaunt(int p)
{
  if (g_h3gaunt.p == p) return &g_h3gaunt;
  free(g_h3gaunt.G);
  int C = (p + 1) * (p + 1), nl = p + 1, L = 2 * p;
  int ng = 2 * p + 2;
  double* x = malloc(sizeof(double) * ng);
  double* w = malloc(sizeof(double) * ng);
  h3_gauss_legendre(ng, x, w);
  /* polynomial parts p_n^m(t) (Y_n^m = p_n^m sin^m e^{im phi}) at the nodes, n <= L */
  int NP = (L + 1) * (L + 1);
  double* P = malloc(sizeof(double) * NP * ng);
  for (int i = 0; i < ng; ++i) {
    double v[3] = {sqrt(1.0 - x[i] * x[i]), 0.0, x[i]};   /* phi = 0 */
    cplx* Y = malloc(sizeof(cplx) * NP);
    h3_ylm(L, v, Y);
    double st = v[0];
    for (int n = 0; n <= L; ++n)
      for (int m = 0; m <= n; ++m) P[(size_t)(n * n + n + m) * ng + i] = creal(Y[H3Q(n, m)]) / pow(st, m);
    free(Y);
  }
  double* G = calloc((size_t)C * C * nl, sizeof(double));
  for (int n = 0; n <= p; ++n)
    for (int m = -n; m <= n; ++m)
      for (int nu = 0; nu <= p; ++nu)
        for (int mu = -nu; mu <= nu; ++mu) {
          int lam = m - mu;
          int am = abs(m), amu = abs(mu), alam = abs(lam);
          int e = (am + amu + alam) / 2;
          for (int j = 0; j < nl; ++j) {
            int l = abs(n - nu) + 2 * j;
            if (l > n + nu || alam > l) continue;
            double s = 0.0;
            for (int i = 0; i < ng; ++i) {
              double om = 1.0;
              for (int u = 0; u < e; ++u) om *= 1.0 - x[i] * x[i];
              s += w[i] * P[(size_t)(n * n + n + am) * ng + i] * P[(size_t)(nu * nu + nu + amu) * ng + i] *
                   P[(size_t)(l * l + l + alam) * ng + i] * om;
            }
            G[((size_t)H3Q(n, m) * C + H3Q(nu, mu)) * nl + j] = 2.0 * M_PI * s;
          }
        }
  free(P);
  free(x);
  free(w);
  g_h3gaunt.p = p;
  g_h3gaunt.nl = nl;
  g_h3gaunt.G = G;
  return &g_h3gaunt;
}

/* Eout (order pout) += translation of Ein (order pin) through wave table Fb of
 * order pin + pout at the translation vector (f = h or j):
 *   Eout_{nu mu} += s_out^{e_out nu} sum_{n m} c_{nu mu; n m} s_in^{e_in n} Ein_{n m} */
static void h3_translate(const h3gaunt_t* gt, int pin, int pout, const cplx* Ein, cplx* Eout,
                         const cplx* Fb, double s_in, int e_in, double s_out, int e_out)
{
  int C = (gt->p + 1) * (gt->p + 1);
  static const cplx ipow4[4] = {1.0, I, -1.0, -I};
  for (int nu = 0; nu <= pout; ++nu) {
    double fo = pow(s_out, e_out * nu);
    for (int mu = -nu; mu <= nu; ++mu) {
      cplx acc = 0.0;
      for (int n = 0; n <= pin; ++n) {
        double fi = pow(s_in, e_in * n);
        for (int m = -n; m <= n; ++m) {
          cplx ein = Ein[H3Q(n, m)];
          if (ein == 0.0) continue;
          int lam = m - mu;
          cplx t = 0.0;
          const double* g = gt->G + ((size_t)H3Q(n, m) * C + H3Q(nu, mu)) * gt->nl;
          for (int j = 0; j <= (n < nu ? n : nu); ++j) {
            int l = abs(n - nu) + 2 * j;
            if (abs(lam) > l) continue;
            int e = ((nu + l - n) % 4 + 4) % 4;
            t += ipow4[e] * Fb[H3Q(l, lam)] * g[j];
          }
          acc += 4.0 * M_PI * t * fi * ein;
        }
      }
      Eout[H3Q(nu, mu)] += fo * acc;
    }
  }
}

/* }}} */

/* {{{ sumpy's compressed Taylor truncation: the monomial basis */

typedef long double complex lcplx;

/* Monomial coefficients, in wave units v = k x, of the order-p local basis
 * f_nm(v) = j_n^[p](|v|) Y_n^m(v) (n <= p): F[H3Q(n,m)][cube(a,b,c)], a + b + c <= p,
 * cube(a,b,c) = (a (p+1) + b)(p+1) + c.  The multipole basis of the moments is
 * e_nm = f_{n,-m}.  The stored multi-indices are the (p+1)^2 with c <= 1 (sumpy
 * eliminates u_zz through the PDE); G[s][nm] = F[nm][stored s] is square and
 * Ginv = G^-1 ([nm][s]) converts stored Taylor coefficients to basis coefficients. */
typedef struct {
  int p, D1, nst;
  cplx* F;
  int* st;          /* cube index of each stored multi-index */
  int* sa;          /* [nst][3] its exponents */
  cplx* Ginv;
  double* fact;     /* 0! .. (2p+1)! */
} h3tay_t;

#define H3T_SLOTS 4
static h3tay_t g_h3tay[H3T_SLOTS] = {{-1}, {-1}, {-1}, {-1}};
static long g_h3tay_used[H3T_SLOTS], g_h3tay_clock = 0;

static int h3t_cube(int a, int b, int c, int D1) { return (a * D1 + b) * D1 + c; }

/* dense polynomial product, truncated at total degree D1 - 1 */
static void h3t_mul(const lcplx* A, const lcplx* B, lcplx* C, int D1)
{
  int D = D1 - 1;
  for (int i = 0; i < D1 * D1 * D1; ++i) C[i] = 0;
  for (int a = 0; a <= D; ++a)
    for (int b = 0; a + b <= D; ++b)
      for (int c = 0; a + b + c <= D; ++c) {
        lcplx x = A[h3t_cube(a, b, c, D1)];
        if (x == 0) continue;
        for (int a2 = 0; a + a2 <= D; ++a2)
          for (int b2 = 0; a + a2 + b + b2 <= D; ++b2)
            for (int c2 = 0; a + a2 + b + b2 + c + c2 <= D; ++c2) {
              lcplx y = B[h3t_cube(a2, b2, c2, D1)];
              if (y != 0) C[h3t_cube(a + a2, b + b2, c + c2, D1)] += x * y;
            }
      }
}

/* Gauss-Jordan inverse with partial pivoting (n x n, row-major), long double */
static int h3t_invert(lcplx* A, lcplx* Ainv, int n)
{
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) Ainv[(size_t)i * n + j] = (i == j) ? 1 : 0;
  for (int col = 0; col < n; ++col) {
    int piv = col;
    for (int r = col + 1; r < n; ++r)
      if (cabsl(A[(size_t)r * n + col]) > cabsl(A[(size_t)piv * n + col])) piv = r;
    if (cabsl(A[(size_t)piv * n + col]) == 0) return -1;
    if (piv != col)
      for (int j = 0; j < n; ++j) {
        lcplx t = A[(size_t)piv * n + j];
        A[(size_t)piv * n + j] = A[(size_t)col * n + j];
        A[(size_t)col * n + j] = t;
        t = Ainv[(size_t)piv * n + j];
        Ainv[(size_t)piv * n + j] = Ainv[(size_t)col * n + j];
        Ainv[(size_t)col * n + j] = t;
      }
    lcplx d = 1 / A[(size_t)col * n + col];
    for (int j = 0; j < n; ++j) {
      A[(size_t)col * n + j] *= d;
      Ainv[(size_t)col * n + j] *= d;
    }
    for (int r = 0; r < n; ++r) {
      if (r == col) continue;
      lcplx f = A[(size_t)r * n + col];
      if (f == 0) continue;
      for (int j = 0; j < n; ++j) {
        A[(size_t)r * n + j] -= f * A[(size_t)col * n + j];
        Ainv[(size_t)r * n + j] -= f * Ainv[(size_t)col * n + j];
      }
    }
  }
  return 0;
}

/* the table of order p (cached; least recently used slot replaced; not thread-safe:
 * call outside parallel regions) */
static const h3tay_t* h3_taylor(int p)
{
  for (int i = 0; i < H3T_SLOTS; ++i)
    if (g_h3tay[i].p == p) {
      g_h3tay_used[i] = ++g_h3tay_clock;
      return &g_h3tay[i];
    }
  int victim = 0;
  for (int i = 1; i < H3T_SLOTS; ++i)
    if (g_h3tay_used[i] < g_h3tay_used[victim]) victim = i;
  g_h3tay_used[victim] = ++g_h3tay_clock;
  h3tay_t* t = &g_h3tay[victim];
  if (t->p >= 0) {
    free(t->F);
    free(t->st);
    free(t->sa);
    free(t->Ginv);
    free(t->fact);
  }
  const int D1 = p + 1, NC = D1 * D1 * D1, ncf = (p + 1) * (p + 1);
  t->p = p;
  t->D1 = D1;
  t->nst = ncf;
  t->F = calloc((size_t)ncf * NC, sizeof(cplx));
  t->st = malloc(sizeof(int) * ncf);
  t->sa = malloc(sizeof(int) * 3 * ncf);
  t->Ginv = malloc(sizeof(cplx) * (size_t)ncf * ncf);
  t->fact = malloc(sizeof(double) * (2 * p + 2));
  t->fact[0] = 1.0;
  for (int i = 1; i <= 2 * p + 1; ++i) t->fact[i] = t->fact[i - 1] * i;
  /* (x^2 + y^2 + z^2)^i, i <= p/2 */
  int nr = p / 2 + 1;
  lcplx* r2 = calloc((size_t)nr * NC, sizeof(lcplx));
  lcplx* base = calloc(NC, sizeof(lcplx));
  r2[h3t_cube(0, 0, 0, D1)] = 1;
  if (p >= 2) {
    base[h3t_cube(2, 0, 0, D1)] = base[h3t_cube(0, 2, 0, D1)] = base[h3t_cube(0, 0, 2, D1)] = 1;
    for (int i = 1; i < nr; ++i) h3t_mul(r2 + (size_t)(i - 1) * NC, base, r2 + (size_t)i * NC, D1);
  }
  /* normalized Legendre parts p_n^m(t) = sum_i A[n][m][i] t^i (the recurrence of h3_ylm) */
  double* A = calloc((size_t)(p + 1) * (p + 1) * (p + 1), sizeof(double));
#define PA(n, m, i) A[(((size_t)(n) * (p + 1)) + (m)) * (p + 1) + (i)]
  double pmm = 0.5 / sqrt(M_PI);
  for (int m = 0; m <= p; ++m) {
    if (m > 0) pmm *= sqrt((2.0 * m + 1.0) / (2.0 * m));
    PA(m, m, 0) = pmm;
    if (m + 1 <= p)
      for (int i = 0; i <= p - 1; ++i) PA(m + 1, m, i + 1) = sqrt(2.0 * m + 3.0) * PA(m, m, i);
    for (int n = m + 2; n <= p; ++n) {
      double a = sqrt((4.0 * n * n - 1.0) / ((double)n * n - (double)m * m));
      double b = sqrt(((n - 1.0) * (n - 1.0) - (double)m * m) / (4.0 * (n - 1.0) * (n - 1.0) - 1.0));
      for (int i = 0; i <= p; ++i)
        PA(n, m, i) = a * ((i > 0 ? PA(n - 1, m, i - 1) : 0.0) - b * PA(n - 2, m, i));
    }
  }
  lcplx* Q = calloc(NC, sizeof(lcplx));
  lcplx* W = calloc(NC, sizeof(lcplx));
  lcplx* R = calloc(NC, sizeof(lcplx));
  lcplx* T = calloc(NC, sizeof(lcplx));
  for (int n = 0; n <= p; ++n)
    for (int m = 0; m <= n; ++m) {
      /* |v|^(n-m) p_n^m(z/|v|) = sum_i A_{n-m-2i} z^(n-m-2i) |v|^(2i) */
      for (int i = 0; i < NC; ++i) Q[i] = 0;
      for (int i = 0; 2 * i <= n - m; ++i) {
        double coef = PA(n, m, n - m - 2 * i);
        if (coef == 0.0) continue;
        for (int a = 0; a <= p; ++a)
          for (int b = 0; a + b <= p; ++b)
            for (int c = 0; a + b + c + (n - m - 2 * i) <= p; ++c) {
              lcplx v = r2[(size_t)i * NC + h3t_cube(a, b, c, D1)];
              if (v != 0) Q[h3t_cube(a, b, c + n - m - 2 * i, D1)] += coef * v;
            }
      }
      /* (x + i y)^m */
      for (int i = 0; i < NC; ++i) W[i] = 0;
      {
        long double bin = 1;
        lcplx ip = 1;
        for (int j = 0; j <= m; ++j) {
          W[h3t_cube(m - j, j, 0, D1)] = bin * ip;
          bin = bin * (m - j) / (j + 1);
          ip *= I;
        }
      }
      h3t_mul(Q, W, R, D1);   /* solid harmonic |v|^n Y_n^m */
      /* f_nm = sum_j c_nj |v|^(2j) R, c_nj = (-1)^j / (2^j j! (2n+2j+1)!!) */
      long double dfac = 1;
      for (int i = 1; i <= n; ++i) dfac *= 2 * i + 1;
      long double cj = 1 / dfac;
      for (int j = 0; n + 2 * j <= p; ++j) {
        h3t_mul(r2 + (size_t)j * NC, R, T, D1);
        for (int i = 0; i < NC; ++i) {
          if (T[i] == 0) continue;
          lcplx v = cj * T[i];
          t->F[(size_t)H3Q(n, m) * NC + i] += (cplx)v;
          if (m > 0) t->F[(size_t)H3Q(n, -m) * NC + i] += (cplx)conjl(v);
        }
        cj *= -1.0L / (2.0L * (j + 1) * (2.0L * n + 2.0L * j + 3.0L));
      }
    }
#undef PA
  /* stored multi-indices and the inverse of G */
  int s_ = 0;
  for (int c = 0; c <= 1 && c <= p; ++c)
    for (int a = 0; a + c <= p; ++a)
      for (int b = 0; a + b + c <= p; ++b) {
        t->st[s_] = h3t_cube(a, b, c, D1);
        t->sa[3 * s_] = a;
        t->sa[3 * s_ + 1] = b;
        t->sa[3 * s_ + 2] = c;
        ++s_;
      }
  lcplx* G = malloc(sizeof(lcplx) * (size_t)ncf * ncf);
  lcplx* Gi = malloc(sizeof(lcplx) * (size_t)ncf * ncf);
  for (int si = 0; si < ncf; ++si)
    for (int c = 0; c < ncf; ++c) G[(size_t)si * ncf + c] = t->F[(size_t)c * NC + t->st[si]];
  h3t_invert(G, Gi, ncf);
  for (size_t i = 0; i < (size_t)ncf * ncf; ++i) t->Ginv[i] = (cplx)Gi[i];
  free(G);
  free(Gi);
  free(r2);
  free(base);
  free(A);
  free(Q);
  free(W);
  free(R);
  free(T);
  return t;
}

/* v^e / e! for e = (a, b, c), a + b + c <= D (cube of side D + 1) */
static void h3t_powers(const double* v, int D, const double* fact, cplx* out)
{
  int D1 = D + 1;
  for (int a = 0; a <= D; ++a)
    for (int b = 0; a + b <= D; ++b)
      for (int c = 0; a + b + c <= D; ++c)
        out[h3t_cube(a, b, c, D1)] = pow(v[0], a) * pow(v[1], b) * pow(v[2], c) /
                                     (fact[a] * fact[b] * fact[c]);
}

/* sumpy M2M of one density: child multipole ac (order p, field 4 pi i k sum
 * ac_nm S_n^m, i.e. ac = M s^n without the 4 pi i k) about cc -> ap about the parent
 * (added), vd = k (cc - cp), the translation of the stored moments with the others
 * taken as zero. */
static void h3t_m2m(const h3tay_t* t, const double* vd, const cplx* ac, cplx* ap, cplx* work)
{
  const int p = t->p, D1 = t->D1, NC = D1 * D1 * D1, ncf = t->nst;
  cplx* mu = work;          /* moments, wave units, by cube index */
  cplx* dpow = work + NC;   /* vd^e / e! */
  for (int i = 0; i < NC; ++i) mu[i] = 0;
  /* stored moments: mu_s = (1/s!) sum_nm Ginv[nm][s] ac_{n,-m} */
  for (int si = 0; si < ncf; ++si) {
    cplx acc = 0;
    for (int n = 0; n <= p; ++n)
      for (int m = -n; m <= n; ++m) acc += t->Ginv[(size_t)H3Q(n, m) * ncf + si] * ac[H3Q(n, -m)];
    const int* e = t->sa + 3 * si;
    mu[t->st[si]] = acc / (t->fact[e[0]] * t->fact[e[1]] * t->fact[e[2]]);
  }
  h3t_powers(vd, p, t->fact, dpow);
  /* parent moments nu_b = sum_{a <= b} mu_a vd^(b-a) / (b-a)!, then
   * ap_nm += sum_b b! [v^b] e_nm nu_b (e_nm = f_{n,-m}) */
  for (int a = 0; a <= p; ++a)
    for (int b = 0; a + b <= p; ++b)
      for (int c = 0; a + b + c <= p; ++c) {
        cplx nu = 0;
        for (int a1 = 0; a1 <= a; ++a1)
          for (int b1 = 0; b1 <= b; ++b1)
            for (int c1 = 0; c1 <= c && c1 <= 1; ++c1) {
              cplx m_ = mu[h3t_cube(a1, b1, c1, D1)];
              if (m_ != 0) nu += m_ * dpow[h3t_cube(a - a1, b - b1, c - c1, D1)];
            }
        if (nu == 0) continue;
        int cb = h3t_cube(a, b, c, D1);
        double bf = t->fact[a] * t->fact[b] * t->fact[c];
        for (int n = 0; n <= p; ++n)
          for (int m = -n; m <= n; ++m) {
            cplx f = t->F[(size_t)H3Q(n, -m) * NC + cb];
            if (f != 0) ap[H3Q(n, m)] += bf * f * nu;
          }
      }
  (void)ncf;
}

/* the monomial coefficients (wave units, about the box center) of the local
 * sum_nm b_nm f_nm: P[cube] */
static void h3t_local_monomials(const h3tay_t* t, const cplx* b, cplx* P)
{
  const int p = t->p, D1 = t->D1, NC = D1 * D1 * D1;
  for (int i = 0; i < NC; ++i) P[i] = 0;
  for (int n = 0; n <= p; ++n)
    for (int m = -n; m <= n; ++m) {
      cplx bv = b[H3Q(n, m)];
      if (bv == 0) continue;
      const cplx* F = t->F + (size_t)H3Q(n, m) * NC;
      for (int i = 0; i < NC; ++i)
        if (F[i] != 0) P[i] += bv * F[i];
    }
}

/* sumpy L2L / L2QBXL of one density: the local polynomial P (monomials of the input
 * order about the old center, wave units) shifted by vd = k (c_new - c_old), its
 * coefficients with exponent of z <= 1 up to order to->p kept and converted to the
 * order-to->p basis: bo_nm += sum_s Ginv[nm][s] P'_s. */
static void h3t_l2l(const h3tay_t* from, const h3tay_t* to, const double* vd, const cplx* P,
                    cplx* bo, cplx* work)
{
  const int pin = from->p, D1 = from->D1, q = to->p, ncq = to->nst;
  cplx* dpow = work;   /* vd^e / e!, cube of the input order */
  h3t_powers(vd, pin, from->fact, dpow);
  for (int si = 0; si < ncq; ++si) {
    const int* e = to->sa + 3 * si;
    /* P'_e = sum_{b >= e} P_b binom(b, e) vd^(b-e) = sum_b P_b b!/e! vd^(b-e)/(b-e)! */
    cplx acc = 0;
    for (int a = e[0]; a <= pin; ++a)
      for (int b = e[1]; a + b <= pin; ++b)
        for (int c = e[2]; a + b + c <= pin; ++c) {
          cplx pv = P[h3t_cube(a, b, c, D1)];
          if (pv == 0) continue;
          double ratio = from->fact[a] * from->fact[b] * from->fact[c] /
                         (from->fact[e[0]] * from->fact[e[1]] * from->fact[e[2]]);
          acc += pv * ratio * dpow[h3t_cube(a - e[0], b - e[1], c - e[2], D1)];
        }
    for (int n = 0; n <= q; ++n)
      for (int m = -n; m <= n; ++m) bo[H3Q(n, m)] += to->Ginv[(size_t)H3Q(n, m) * ncq + si] * acc;
  }
}

/* }}} */

typedef struct {
  int pf, pq, nrhs, ncf, ncq;
  double k;
  cplx cq, cd;
  int sumpy;      /* the reference's default (compressed Taylor) truncation */
} h3ctx_t;

static int h3_ctx(const qbxfmm_kernel* kern, h3ctx_t* c)
{
  if (kern->dim != 3 || kern->k_im != 0.0 || !(kern->k_re > 0.0)) return QBXFMM_ERR_UNSUPPORTED;
  if (kern->fmm_order > 22 || kern->qbx_order > kern->fmm_order) return QBXFMM_ERR_UNSUPPORTED;
  c->pf = kern->fmm_order;
  c->pq = kern->qbx_order;
  c->nrhs = kern->nrhs;
  c->ncf = (c->pf + 1) * (c->pf + 1);
  c->ncq = (c->pq + 1) * (c->pq + 1);
  c->k = kern->k_re;
  c->cq = kern->charge_coeff_re + I * kern->charge_coeff_im;
  c->cd = kern->dipole_coeff_re + I * kern->dipole_coeff_im;
  c->sumpy = kern->fmm_backend == QBXFMM_BACKEND_SUMPY;
  return 0;
}

static double h3_scale(double k, double rho) { return k * rho < 1.0 ? k * rho : 1.0; }

/* P2M (local = 0) / P2L (local = 1) of one source into E (order p, scale s) */
static void h3_p2e(const h3ctx_t* c, int p, double s, const double* ctr, const double* y,
                   cplx q, cplx sigma, const double* nv, cplx* E, int local, cplx* F)
{
  double u[3] = {y[0] - ctr[0], y[1] - ctr[1], y[2] - ctr[2]};
  int N = p + 1;
  /* sumpy multipoles: moments of degree <= p, j_n^[p] (charge) and the normal
   * derivative of the degree-<=p moments, i.e. j_n^[p-1] in the ladder (dipole) */
  int trunc = !local && c->sumpy;
  cplx* Fd = F + (size_t)(N + 1) * (N + 1);
  if (trunc) {
    h3_waves_trunc(N, c->k, u, p, F);
    h3_waves_trunc(N, c->k, u, p - 1, Fd);
  } else {
    h3_waves(N, c->k, u, local, F);
    Fd = F;
  }
  cplx pre = 4.0 * M_PI * I * c->k;
  for (int n = 0; n <= p; ++n) {
    double f = local ? pow(s, n) : pow(s, -n);
    for (int m = -n; m <= n; ++m) {
      cplx v = q * F[H3Q(n, -m)];
      if (sigma != 0.0) v += sigma * h3_dgrad(Fd, N, n, -m, c->k, nv);
      E[H3Q(n, m)] += pre * f * v;
    }
  }
}

/* evaluate E (order p, scale s) at x: multipole (local = 0) or local (local = 1) */
static cplx h3_e2p(const h3ctx_t* c, int p, double s, const double* ctr, const double* x,
                   const cplx* E, int local, cplx* F)
{
  double u[3] = {x[0] - ctr[0], x[1] - ctr[1], x[2] - ctr[2]};
  /* sumpy locals: the degree-p Taylor polynomial, j_n^[p] */
  if (local && c->sumpy) h3_waves_trunc(p, c->k, u, p, F);
  else h3_waves(p, c->k, u, !local, F);
  cplx acc = 0.0;
  for (int n = 0; n <= p; ++n) {
    double f = local ? pow(s, -n) : pow(s, n);
    for (int m = -n; m <= n; ++m) acc += f * E[H3Q(n, m)] * F[H3Q(n, m)];
  }
  return acc;
}

static cplx h3_p2p(double k, const double* x, const double* y, cplx q, cplx sigma,
                   const double* nv)
{
  double d[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
  double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (r == 0) return 0;
  cplx e = cexp(I * k * r);
  cplx v = q * e / r;
  /* d/dn_y e^{ikr}/r = (n . (x - y)) / r * e^{ikr} (1 - ikr) / r^2 */
  if (sigma != 0.0)
    v += sigma * (nv[0] * d[0] + nv[1] * d[1] + nv[2] * d[2]) * e * (1.0 - I * k * r) / (r * r * r);
  return v;
}

#define H3_WORK (size_t)((2 * H3_NMAX + 2) * (2 * H3_NMAX + 2))

static int h3_form_multipoles(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                              const cplx* strengths, cplx* mpoles)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* F = malloc(sizeof(cplx) * H3_WORK);
#pragma omp for schedule(dynamic, 4)
    for (int isb = 0; isb < g->nsource_boxes; ++isb) {
      int b = g->source_boxes[isb];
      double s = h3_scale(c.k, level_width(g, g->box_levels[b]));
      double ctr[3], y[3], nv[3] = {0, 0, 0};
      load(g->box_centers, g->nboxes, b, 3, ctr);
      int s0 = g->box_source_starts[b], s1 = s0 + g->box_source_counts_nonchild[b];
      for (int r = 0; r < c.nrhs; ++r) {
        cplx* M = mpoles + ((size_t)b * c.nrhs + r) * c.ncf;
        for (int si = s0; si < s1; ++si) {
          load(g->sources, g->nsources, si, 3, y);
          if (c.cd != 0.0) load(g->source_normals, g->nsources, si, 3, nv);
          cplx st = strengths[(size_t)r * g->nsources + si];
          h3_p2e(&c, c.pf, s, ctr, y, c.cq * st, c.cd * st, nv, M, 0, F);
        }
      }
    }
    free(F);
  }
  return 0;
}

static int h3_coarsen_multipoles(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                                 cplx* mpoles)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
  if (c.sumpy) {
    const h3tay_t* t = h3_taylor(c.pf);
    const size_t NC = (size_t)t->D1 * t->D1 * t->D1;
    for (int lev = g->nlevels - 2; lev >= 0; --lev) {
      int i0 = g->level_start_source_parent_box_nrs[lev];
      int i1 = g->level_start_source_parent_box_nrs[lev + 1];
      double sp = h3_scale(c.k, level_width(g, lev)), sc = h3_scale(c.k, level_width(g, lev + 1));
#pragma omp parallel
      {
        cplx* work = malloc(sizeof(cplx) * (2 * NC + 2 * c.ncf));
        cplx* ac = work + 2 * NC;
        cplx* ap = ac + c.ncf;
#pragma omp for schedule(dynamic, 1)
        for (int i = i0; i < i1; ++i) {
          int b = g->source_parent_boxes[i];
          double cp[3], cc[3];
          load(g->box_centers, g->nboxes, b, 3, cp);
          for (int ci = 0; ci < 8; ++ci) {
            int ch = g->box_child_ids[(size_t)ci * g->nboxes + b];
            if (ch == 0 || g->box_source_counts_cumul[ch] == 0) continue;
            load(g->box_centers, g->nboxes, ch, 3, cc);
            double vd[3] = {c.k * (cc[0] - cp[0]), c.k * (cc[1] - cp[1]), c.k * (cc[2] - cp[2])};
            for (int r = 0; r < c.nrhs; ++r) {
              const cplx* Min = mpoles + ((size_t)ch * c.nrhs + r) * c.ncf;
              cplx* Mout = mpoles + ((size_t)b * c.nrhs + r) * c.ncf;
              for (int n = 0; n <= c.pf; ++n)
                for (int m = -n; m <= n; ++m) {
                  ac[H3Q(n, m)] = Min[H3Q(n, m)] * pow(sc, n);
                  ap[H3Q(n, m)] = 0;
                }
              h3t_m2m(t, vd, ac, ap, work);
              for (int n = 0; n <= c.pf; ++n)
                for (int m = -n; m <= n; ++m) Mout[H3Q(n, m)] += ap[H3Q(n, m)] * pow(sp, -n);
            }
          }
        }
        free(work);
      }
    }
    return 0;
  }
  const h3gaunt_t* gt = h3_gaunt(c.pf);
  for (int lev = g->nlevels - 2; lev >= 0; --lev) {
    int i0 = g->level_start_source_parent_box_nrs[lev];
    int i1 = g->level_start_source_parent_box_nrs[lev + 1];
#pragma omp parallel
    {
      cplx* F = malloc(sizeof(cplx) * H3_WORK);
#pragma omp for schedule(dynamic, 1)
      for (int i = i0; i < i1; ++i) {
        int b = g->source_parent_boxes[i];
        double sp = h3_scale(c.k, level_width(g, lev)), sc = h3_scale(c.k, level_width(g, lev + 1));
        double cp[3], cc[3];
        load(g->box_centers, g->nboxes, b, 3, cp);
        for (int ci = 0; ci < 8; ++ci) {
          int ch = g->box_child_ids[(size_t)ci * g->nboxes + b];
          if (ch == 0 || g->box_source_counts_cumul[ch] == 0) continue;
          load(g->box_centers, g->nboxes, ch, 3, cc);
          double bv[3] = {cp[0] - cc[0], cp[1] - cc[1], cp[2] - cc[2]};
          h3_waves(2 * c.pf, c.k, bv, 0, F);
          for (int r = 0; r < c.nrhs; ++r)
            h3_translate(gt, c.pf, c.pf, mpoles + ((size_t)ch * c.nrhs + r) * c.ncf,
                         mpoles + ((size_t)b * c.nrhs + r) * c.ncf, F, sc, 1, sp, -1);
        }
      }
      free(F);
    }
  }
  return 0;
}

static int h3_eval_direct(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                          const cplx* strengths, cplx* pot)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel for schedule(dynamic, 1)
  for (int itb = 0; itb < g->ntarget_boxes; ++itb) {
    int tb = g->target_boxes[itb];
    int t0 = g->nonqbx_box_target_starts[tb];
    int t1 = t0 + g->nonqbx_box_target_counts_nonchild[tb];
    for (int t = t0; t < t1; ++t) {
      double x[3], y[3], nv[3] = {0, 0, 0};
      load(g->nonqbx_targets, g->nfiltered_targets, t, 3, x);
      for (int r = 0; r < c.nrhs; ++r) {
        cplx acc = 0;
        for (int li = g->list1_starts[itb]; li < g->list1_starts[itb + 1]; ++li) {
          int sb = g->list1_lists[li];
          int s0 = g->box_source_starts[sb], s1 = s0 + g->box_source_counts_nonchild[sb];
          for (int si = s0; si < s1; ++si) {
            load(g->sources, g->nsources, si, 3, y);
            if (c.cd != 0.0) load(g->source_normals, g->nsources, si, 3, nv);
            cplx st = strengths[(size_t)r * g->nsources + si];
            acc += h3_p2p(c.k, x, y, c.cq * st, c.cd * st, nv);
          }
        }
        pot[(size_t)r * g->nfiltered_targets + t] += acc;
      }
    }
  }
  return 0;
}

static int h3_multipole_to_local(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                                 const cplx* mpoles, cplx* locals)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
  const h3gaunt_t* gt = h3_gaunt(c.pf);
#pragma omp parallel
  {
    cplx* F = malloc(sizeof(cplx) * H3_WORK);
#pragma omp for schedule(dynamic, 1)
    for (int i = 0; i < g->nttp_boxes; ++i) {
      int tb = g->target_or_target_parent_boxes[i];
      double s = h3_scale(c.k, level_width(g, g->box_levels[tb]));
      double ct[3], cs[3];
      load(g->box_centers, g->nboxes, tb, 3, ct);
      for (int li = g->list2_starts[i]; li < g->list2_starts[i + 1]; ++li) {
        int sb = g->list2_lists[li];
        load(g->box_centers, g->nboxes, sb, 3, cs);
        double bv[3] = {ct[0] - cs[0], ct[1] - cs[1], ct[2] - cs[2]};
        h3_waves(2 * c.pf, c.k, bv, 1, F);
        for (int r = 0; r < c.nrhs; ++r)
          h3_translate(gt, c.pf, c.pf, mpoles + ((size_t)sb * c.nrhs + r) * c.ncf,
                       locals + ((size_t)tb * c.nrhs + r) * c.ncf, F, s, 1, s, 1);
      }
    }
    free(F);
  }
  return 0;
}

static int h3_eval_multipoles(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                              const cplx* mpoles, cplx* pot)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* F = malloc(sizeof(cplx) * H3_WORK);
#pragma omp for schedule(dynamic, 1)
    for (int itb = 0; itb < g->ntarget_boxes; ++itb) {
      int tb = g->target_boxes[itb];
      int t0 = g->nonqbx_box_target_starts[tb];
      int t1 = t0 + g->nonqbx_box_target_counts_nonchild[tb];
      for (int t = t0; t < t1; ++t) {
        double x[3], cs[3];
        load(g->nonqbx_targets, g->nfiltered_targets, t, 3, x);
        for (int li = g->list3_starts[itb]; li < g->list3_starts[itb + 1]; ++li) {
          int sb = g->list3_lists[li];
          double s = h3_scale(c.k, level_width(g, g->box_levels[sb]));
          load(g->box_centers, g->nboxes, sb, 3, cs);
          for (int r = 0; r < c.nrhs; ++r)
            pot[(size_t)r * g->nfiltered_targets + t] +=
                h3_e2p(&c, c.pf, s, cs, x, mpoles + ((size_t)sb * c.nrhs + r) * c.ncf, 0, F);
        }
      }
    }
    free(F);
  }
  return 0;
}

static int h3_form_locals(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                          const cplx* strengths, cplx* locals)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* F = malloc(sizeof(cplx) * H3_WORK);
#pragma omp for schedule(dynamic, 1)
    for (int i = 0; i < g->nttp_boxes; ++i) {
      int tb = g->target_or_target_parent_boxes[i];
      double s = h3_scale(c.k, level_width(g, g->box_levels[tb]));
      double ct[3], y[3], nv[3] = {0, 0, 0};
      load(g->box_centers, g->nboxes, tb, 3, ct);
      for (int li = g->list4_starts[i]; li < g->list4_starts[i + 1]; ++li) {
        int sb = g->list4_lists[li];
        int s0 = g->box_source_starts[sb], s1 = s0 + g->box_source_counts_nonchild[sb];
        for (int si = s0; si < s1; ++si) {
          load(g->sources, g->nsources, si, 3, y);
          if (c.cd != 0.0) load(g->source_normals, g->nsources, si, 3, nv);
          for (int r = 0; r < c.nrhs; ++r) {
            cplx st = strengths[(size_t)r * g->nsources + si];
            h3_p2e(&c, c.pf, s, ct, y, c.cq * st, c.cd * st, nv,
                   locals + ((size_t)tb * c.nrhs + r) * c.ncf, 1, F);
          }
        }
      }
    }
    free(F);
  }
  return 0;
}

static int h3_refine_locals(const qbxfmm_kernel* kern, const qbxfmm_geometry* g, cplx* locals)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
  if (c.sumpy) {
    const h3tay_t* t = h3_taylor(c.pf);
    const size_t NC = (size_t)t->D1 * t->D1 * t->D1;
    for (int lev = 1; lev < g->nlevels; ++lev) {
      int i0 = g->level_start_ttp_box_nrs[lev], i1 = g->level_start_ttp_box_nrs[lev + 1];
      double sp = h3_scale(c.k, level_width(g, lev - 1)), sc = h3_scale(c.k, level_width(g, lev));
#pragma omp parallel
      {
        cplx* work = malloc(sizeof(cplx) * (2 * NC + 2 * c.ncf));
        cplx* P = work + NC;
        cplx* bp = P + NC;
        cplx* bc = bp + c.ncf;
#pragma omp for schedule(dynamic, 4)
        for (int i = i0; i < i1; ++i) {
          int b = g->target_or_target_parent_boxes[i];
          int par = g->box_parent_ids[b];
          double cp[3], cc[3];
          load(g->box_centers, g->nboxes, par, 3, cp);
          load(g->box_centers, g->nboxes, b, 3, cc);
          double vd[3] = {c.k * (cc[0] - cp[0]), c.k * (cc[1] - cp[1]), c.k * (cc[2] - cp[2])};
          for (int r = 0; r < c.nrhs; ++r) {
            const cplx* Lin = locals + ((size_t)par * c.nrhs + r) * c.ncf;
            cplx* Lout = locals + ((size_t)b * c.nrhs + r) * c.ncf;
            for (int n = 0; n <= c.pf; ++n)
              for (int m = -n; m <= n; ++m) {
                bp[H3Q(n, m)] = Lin[H3Q(n, m)] * pow(sp, -n);
                bc[H3Q(n, m)] = 0;
              }
            h3t_local_monomials(t, bp, P);
            h3t_l2l(t, t, vd, P, bc, work);
            for (int n = 0; n <= c.pf; ++n)
              for (int m = -n; m <= n; ++m) Lout[H3Q(n, m)] += bc[H3Q(n, m)] * pow(sc, n);
          }
        }
        free(work);
      }
    }
    return 0;
  }
  const h3gaunt_t* gt = h3_gaunt(c.pf);
  for (int lev = 1; lev < g->nlevels; ++lev) {
    int i0 = g->level_start_ttp_box_nrs[lev], i1 = g->level_start_ttp_box_nrs[lev + 1];
#pragma omp parallel
    {
      cplx* F = malloc(sizeof(cplx) * H3_WORK);
#pragma omp for schedule(dynamic, 4)
      for (int i = i0; i < i1; ++i) {
        int b = g->target_or_target_parent_boxes[i];
        int par = g->box_parent_ids[b];
        double sp = h3_scale(c.k, level_width(g, lev - 1)), sc = h3_scale(c.k, level_width(g, lev));
        double cp[3], cc[3];
        load(g->box_centers, g->nboxes, par, 3, cp);
        load(g->box_centers, g->nboxes, b, 3, cc);
        double bv[3] = {cc[0] - cp[0], cc[1] - cp[1], cc[2] - cp[2]};
        h3_waves(2 * c.pf, c.k, bv, 0, F);
        for (int r = 0; r < c.nrhs; ++r)
          h3_translate(gt, c.pf, c.pf, locals + ((size_t)par * c.nrhs + r) * c.ncf,
                       locals + ((size_t)b * c.nrhs + r) * c.ncf, F, sp, -1, sc, 1);
      }
      free(F);
    }
  }
  return 0;
}

static int h3_eval_locals(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                          const cplx* locals, cplx* pot)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* F = malloc(sizeof(cplx) * H3_WORK);
#pragma omp for schedule(dynamic, 4)
    for (int itb = 0; itb < g->ntarget_boxes; ++itb) {
      int tb = g->target_boxes[itb];
      int t0 = g->nonqbx_box_target_starts[tb];
      int t1 = t0 + g->nonqbx_box_target_counts_nonchild[tb];
      double s = h3_scale(c.k, level_width(g, g->box_levels[tb]));
      double ct[3], x[3];
      load(g->box_centers, g->nboxes, tb, 3, ct);
      for (int t = t0; t < t1; ++t) {
        load(g->nonqbx_targets, g->nfiltered_targets, t, 3, x);
        for (int r = 0; r < c.nrhs; ++r)
          pot[(size_t)r * g->nfiltered_targets + t] +=
              h3_e2p(&c, c.pf, s, ct, x, locals + ((size_t)tb * c.nrhs + r) * c.ncf, 1, F);
      }
    }
    free(F);
  }
  return 0;
}

static int h3_p2qbxl(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                     const cplx* strengths, cplx* qbx_exps, int all_sources)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* F = malloc(sizeof(cplx) * H3_WORK);
#pragma omp for schedule(dynamic, 16)
    for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
      int ctr = g->global_qbx_centers[ig];
      double cc[3], y[3], nv[3] = {0, 0, 0};
      load(g->centers, g->ncenters, ctr, 3, cc);
      double s = h3_scale(c.k, g->expansion_radii[ctr]);
      int itb = g->qbx_center_to_target_box[ctr];
      int l0 = all_sources ? 0 : g->list1_starts[itb];
      int l1 = all_sources ? 1 : g->list1_starts[itb + 1];
      for (int li = l0; li < l1; ++li) {
        int s0, s1;
        if (all_sources) {
          s0 = 0;
          s1 = g->nsources;
        } else {
          int sb = g->list1_lists[li];
          s0 = g->box_source_starts[sb];
          s1 = s0 + g->box_source_counts_nonchild[sb];
        }
        for (int si = s0; si < s1; ++si) {
          load(g->sources, g->nsources, si, 3, y);
          if (c.cd != 0.0) load(g->source_normals, g->nsources, si, 3, nv);
          for (int r = 0; r < c.nrhs; ++r) {
            cplx st = strengths[(size_t)r * g->nsources + si];
            h3_p2e(&c, c.pq, s, cc, y, c.cq * st, c.cd * st, nv,
                   qbx_exps + ((size_t)ctr * c.nrhs + r) * c.ncq, 1, F);
          }
        }
      }
    }
    free(F);
  }
  return 0;
}

static int h3_m2qbxl(const qbxfmm_kernel* kern, const qbxfmm_geometry* g, const cplx* mpoles,
                     cplx* qbx_exps)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
  const h3gaunt_t* gt = h3_gaunt(c.pf);
#pragma omp parallel
  {
    cplx* F = malloc(sizeof(cplx) * H3_WORK);
#pragma omp for schedule(dynamic, 16)
    for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
      int ctr = g->global_qbx_centers[ig];
      double cc[3], cs[3];
      load(g->centers, g->ncenters, ctr, 3, cc);
      double st = h3_scale(c.k, g->expansion_radii[ctr]);
      int itb = g->qbx_center_to_target_box[ctr];
      for (int li = g->list3_starts[itb]; li < g->list3_starts[itb + 1]; ++li) {
        int sb = g->list3_lists[li];
        double ss = h3_scale(c.k, level_width(g, g->box_levels[sb]));
        load(g->box_centers, g->nboxes, sb, 3, cs);
        double bv[3] = {cc[0] - cs[0], cc[1] - cs[1], cc[2] - cs[2]};
        h3_waves(c.pf + c.pq, c.k, bv, 1, F);
        for (int r = 0; r < c.nrhs; ++r)
          h3_translate(gt, c.pf, c.pq, mpoles + ((size_t)sb * c.nrhs + r) * c.ncf,
                       qbx_exps + ((size_t)ctr * c.nrhs + r) * c.ncq, F, ss, 1, st, 1);
      }
    }
    free(F);
  }
  return 0;
}

static int h3_l2qbxl(const qbxfmm_kernel* kern, const qbxfmm_geometry* g, const cplx* locals,
                     cplx* qbx_exps)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
  if (c.sumpy) {
    const h3tay_t* tp = h3_taylor(c.pf);
    const h3tay_t* tq = h3_taylor(c.pq);
    const size_t NC = (size_t)tp->D1 * tp->D1 * tp->D1;
    /* the monomials of every target box's local that holds a QBX center */
    cplx* Pall = calloc((size_t)g->ntarget_boxes * c.nrhs * NC, sizeof(cplx));
    char* need = calloc((size_t)g->ntarget_boxes, 1);
    for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig)
      need[g->qbx_center_to_target_box[g->global_qbx_centers[ig]]] = 1;
#pragma omp parallel
    {
      cplx* b = malloc(sizeof(cplx) * c.ncf);
#pragma omp for schedule(dynamic, 4)
      for (int itb = 0; itb < g->ntarget_boxes; ++itb) {
        if (!need[itb]) continue;
        int tb = g->target_boxes[itb];
        double sb_ = h3_scale(c.k, level_width(g, g->box_levels[tb]));
        for (int r = 0; r < c.nrhs; ++r) {
          const cplx* Lin = locals + ((size_t)tb * c.nrhs + r) * c.ncf;
          for (int n = 0; n <= c.pf; ++n)
            for (int m = -n; m <= n; ++m) b[H3Q(n, m)] = Lin[H3Q(n, m)] * pow(sb_, -n);
          h3t_local_monomials(tp, b, Pall + ((size_t)itb * c.nrhs + r) * NC);
        }
      }
      free(b);
    }
#pragma omp parallel
    {
      cplx* work = malloc(sizeof(cplx) * (NC + c.ncq));
      cplx* bq = work + NC;
#pragma omp for schedule(dynamic, 16)
      for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
        int ctr = g->global_qbx_centers[ig];
        int itb = g->qbx_center_to_target_box[ctr];
        int tb = g->target_boxes[itb];
        double cc[3], cb[3];
        load(g->centers, g->ncenters, ctr, 3, cc);
        load(g->box_centers, g->nboxes, tb, 3, cb);
        double sc = h3_scale(c.k, g->expansion_radii[ctr]);
        double vd[3] = {c.k * (cc[0] - cb[0]), c.k * (cc[1] - cb[1]), c.k * (cc[2] - cb[2])};
        for (int r = 0; r < c.nrhs; ++r) {
          for (int i = 0; i < c.ncq; ++i) bq[i] = 0;
          h3t_l2l(tp, tq, vd, Pall + ((size_t)itb * c.nrhs + r) * NC, bq, work);
          cplx* L = qbx_exps + ((size_t)ctr * c.nrhs + r) * c.ncq;
          for (int n = 0; n <= c.pq; ++n)
            for (int m = -n; m <= n; ++m) L[H3Q(n, m)] += bq[H3Q(n, m)] * pow(sc, n);
        }
      }
      free(work);
    }
    free(Pall);
    free(need);
    return 0;
  }
  const h3gaunt_t* gt = h3_gaunt(c.pf);
#pragma omp parallel
  {
    cplx* F = malloc(sizeof(cplx) * H3_WORK);
#pragma omp for schedule(dynamic, 16)
    for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
      int ctr = g->global_qbx_centers[ig];
      int tb = g->target_boxes[g->qbx_center_to_target_box[ctr]];
      double cc[3], cb[3];
      load(g->centers, g->ncenters, ctr, 3, cc);
      load(g->box_centers, g->nboxes, tb, 3, cb);
      double sb_ = h3_scale(c.k, level_width(g, g->box_levels[tb]));
      double sc = h3_scale(c.k, g->expansion_radii[ctr]);
      double bv[3] = {cc[0] - cb[0], cc[1] - cb[1], cc[2] - cb[2]};
      h3_waves(c.pf + c.pq, c.k, bv, 0, F);
      for (int r = 0; r < c.nrhs; ++r)
        h3_translate(gt, c.pf, c.pq, locals + ((size_t)tb * c.nrhs + r) * c.ncf,
                     qbx_exps + ((size_t)ctr * c.nrhs + r) * c.ncq, F, sb_, -1, sc, 1);
    }
    free(F);
  }
  return 0;
}

static int h3_eval_qbx_expansions(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                                  const cplx* qbx_exps, cplx* pot_tree)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* F = malloc(sizeof(cplx) * H3_WORK);
#pragma omp for schedule(dynamic, 16)
    for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
      int ctr = g->global_qbx_centers[ig];
      double cc[3], x[3];
      load(g->centers, g->ncenters, ctr, 3, cc);
      double s = h3_scale(c.k, g->expansion_radii[ctr]);
      for (int it = g->center_to_targets_starts[ctr]; it < g->center_to_targets_starts[ctr + 1];
           ++it) {
        int t = g->center_to_targets_lists[it];
        load(g->targets, g->ntargets, t, 3, x);
        for (int r = 0; r < c.nrhs; ++r)
          pot_tree[(size_t)r * g->ntargets + t] =
              h3_e2p(&c, c.pq, s, cc, x, qbx_exps + ((size_t)ctr * c.nrhs + r) * c.ncq, 1, F);
      }
    }
    free(F);
  }
  return 0;
}

static int h3_assemble(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                       const cplx* pot_nonqbx, const cplx* pot_tree, cplx* out)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
  double scale = 0.25 / M_PI;
  cplx* full = malloc(sizeof(cplx) * (g->ntargets + 1));
  for (int r = 0; r < c.nrhs; ++r) {
    memcpy(full, pot_tree + (size_t)r * g->ntargets, sizeof(cplx) * g->ntargets);
    for (int f = 0; f < g->nfiltered_targets; ++f)
      full[g->unfiltered_from_filtered_target_indices[f]] +=
          pot_nonqbx[(size_t)r * g->nfiltered_targets + f];
    for (int t = 0; t < g->ntargets; ++t) {
      int u = g->sorted_target_ids[t] - g->ncenters;
      if (u >= 0) out[(size_t)r * g->nuser_targets + u] = scale * full[t];
    }
  }
  free(full);
  return 0;
}

static int h3_apply(const qbxfmm_kernel* kern, const qbxfmm_geometry* g, const cplx* strengths,
                    cplx* out, int direct)
{
  h3ctx_t c;
  int rc = h3_ctx(kern, &c);
  if (rc) return rc;
  size_t nexp = (size_t)g->nboxes * c.nrhs * c.ncf;
  cplx* mpoles = calloc(nexp, sizeof(cplx));
  cplx* locals = calloc(nexp, sizeof(cplx));
  cplx* qexp = calloc((size_t)g->ncenters * c.nrhs * c.ncq, sizeof(cplx));
  cplx* pnq = calloc((size_t)c.nrhs * g->nfiltered_targets + 1, sizeof(cplx));
  cplx* ptree = calloc((size_t)c.nrhs * g->ntargets + 1, sizeof(cplx));
  if (!direct) {
    h3_form_multipoles(kern, g, strengths, mpoles);
    h3_coarsen_multipoles(kern, g, mpoles);
    h3_eval_direct(kern, g, strengths, pnq);
    h3_multipole_to_local(kern, g, mpoles, locals);
    h3_eval_multipoles(kern, g, mpoles, pnq);
    h3_form_locals(kern, g, strengths, locals);
    h3_refine_locals(kern, g, locals);
    h3_eval_locals(kern, g, locals, pnq);
    h3_p2qbxl(kern, g, strengths, qexp, 0);
    h3_m2qbxl(kern, g, mpoles, qexp);
    h3_l2qbxl(kern, g, locals, qexp);
  } else {
    h3_p2qbxl(kern, g, strengths, qexp, 1);
#pragma omp parallel for schedule(dynamic, 16)
    for (int t = 0; t < g->nfiltered_targets; ++t) {
      double x[3], y[3], nv[3] = {0, 0, 0};
      load(g->nonqbx_targets, g->nfiltered_targets, t, 3, x);
      for (int r = 0; r < c.nrhs; ++r) {
        cplx acc = 0;
        for (int si = 0; si < g->nsources; ++si) {
          load(g->sources, g->nsources, si, 3, y);
          if (c.cd != 0.0) load(g->source_normals, g->nsources, si, 3, nv);
          cplx st = strengths[(size_t)r * g->nsources + si];
          acc += h3_p2p(c.k, x, y, c.cq * st, c.cd * st, nv);
        }
        pnq[(size_t)r * g->nfiltered_targets + t] = acc;
      }
    }
  }
  h3_eval_qbx_expansions(kern, g, qexp, ptree);
  h3_assemble(kern, g, pnq, ptree, out);
  free(mpoles);
  free(locals);
  free(qexp);
  free(pnq);
  free(ptree);
  return 0;
}

/* The same recurrences at a complex argument (Miller's backward recurrence for j_n,
 * normalized with j_0 = sin z / z or j_1; h_n upward from h_0, h_1), for the
 * reference's own golden values of its spherical Bessel / Hankel routines. */
static void h3_sph_j_complex(int N, cplx z, cplx* jv)
{
  for (int n = 0; n <= N; ++n) jv[n] = 0.0;
  double az = cabs(z);
  if (az == 0.0) {
    jv[0] = 1.0;
    return;
  }
  int nmax = N > (int)az ? N : (int)az;
  int start = nmax + 16 + (int)sqrt(40.0 * (nmax + 1));
  cplx fp1 = 0.0, f = 1e-200, f1 = 0.0;
  for (int n = start; n >= 1; --n) {
    cplx fm1 = (2.0 * n + 1.0) / z * f - fp1;
    fp1 = f;
    f = fm1;
    if (n - 1 <= N) jv[n - 1] = f;
    if (n - 1 == 1) f1 = f;
    if (cabs(f) > 1e200) {
      f *= 1e-200;
      fp1 *= 1e-200;
      f1 *= 1e-200;
      for (int j = n - 1; j <= N; ++j) jv[j] *= 1e-200;
    }
  }
  cplx sz = csin(z), cz = ccos(z);
  cplx scale = (az < 1.0 || cabs(sz) >= 0.5) ? (sz / z) / f : ((sz / z - cz) / z) / f1;
  for (int n = 0; n <= N; ++n) jv[n] *= scale;
}

static void h3_sph_h_complex(int N, cplx z, cplx* hv)
{
  cplx e = cexp(I * z);
  hv[0] = -I * e / z;
  if (N >= 1) hv[1] = -e * (z + I) / (z * z);
  for (int n = 1; n < N; ++n) hv[n + 1] = (2.0 * n + 1.0) / z * hv[n] - hv[n - 1];
}

void orc_h3_sph_j_complex(int N, double zr, double zi, cplx* out)
{
  h3_sph_j_complex(N, zr + I * zi, out);
}
void orc_h3_sph_h_complex(int N, double zr, double zi, cplx* out)
{
  h3_sph_h_complex(N, zr + I * zi, out);
}

/* test hooks: special functions and wave tables */
void orc_h3_sph_j(int N, double x, double* out) { h3_sph_j(N, x, out); }
void orc_h3_sph_h(int N, double x, cplx* out) { h3_sph_h(N, x, out); }
void orc_h3_ylm(int N, const double* v, cplx* out) { h3_ylm(N, v, out); }
void orc_h3_waves(int N, double k, const double* v, int singular, cplx* out)
{
  h3_waves(N, k, v, singular, out);
}
cplx orc_h3_dgrad(const cplx* F, int N, int n, int m, double k, const double* nu)
{
  return h3_dgrad(F, N, n, m, k, nu);
}
void orc_h3_gaunt(int p, double* out)
{
  const h3gaunt_t* gt = h3_gaunt(p);
  int C = (p + 1) * (p + 1);
  memcpy(out, gt->G, sizeof(double) * (size_t)C * C * gt->nl);
}
