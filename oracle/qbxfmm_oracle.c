/*
 * qbxfmm_oracle.c -- CPU (C99 + OpenMP, float64/complex128) restatement of the
 * QBX-FMM apply.  TEST INFRASTRUCTURE ONLY: the checker for the CUDA library and
 * the timed CPU baseline; the product never links or calls it.
 *
 * Stage order and semantics follow pytential's FMM driver and QBX wrangler:
 *   drive_fmm                         pytential/qbx/fmm.py:414-594
 *   form_global_qbx_locals  (P2QBXL)  pytential/qbx/fmm.py:231-265, interactions.py:84-124
 *   translate_box_multipoles_to_qbx_local (M2QBXL)
 *                                     pytential/qbx/fmm.py:267-312, interactions.py:196-235
 *   translate_box_local_to_qbx_local (L2QBXL)
 *                                     pytential/qbx/fmm.py:314-356, interactions.py:318-356
 *   eval_qbx_expansions (QBXL2P)      pytential/qbx/fmm.py:358-389, interactions.py:442-479
 *   potential assembly / reorder      pytential/qbx/fmm.py:569-588
 * The point-FMM stages (P2M, M2M, P2P, M2L, M2P, P2L, L2L, L2P) are sumpy's, which
 * is not part of the reference tree; they are restated from the published
 * expansions:
 *   3D Laplace: regular/singular solid harmonics
 *       R_n^m(v) = r^n P_n^m(cos t) e^{i m p} / (n+m)!,
 *       S_n^m(v) = (n-m)! P_n^m(cos t) e^{i m p} / r^{n+1}   (no Condon-Shortley phase),
 *     with 1/|x-y| = sum conj(R_n^m(y)) S_n^m(x) and the addition theorems
 *       R_n^m(a+b) = sum R_k^l(a) R_{n-k}^{m-l}(b),
 *       S_n^m(x-y) = sum conj(R_k^l(y)) S_{n+k}^{m+l}(x).
 *     For a harmonic kernel the degree-p solid-harmonic truncation equals sumpy's
 *     default compressed Cartesian Taylor truncation (both are the degree-p Taylor
 *     polynomial), so the arithmetic is the same in exact arithmetic.
 *   2D Laplace: complex-analytic multipole/local expansions of log|z - w|
 *     (Greengard-Rokhlin), equal to the degree-p Taylor truncation for the same
 *     reason.
 * Coefficients are scaled by rscale^n (multipoles divided, locals multiplied) with
 * rscale = box width for box expansions and the expansion radius for QBX
 * expansions, as sumpy's level_to_rscale / QBX rscale do
 * (pytential/qbx/fmm.py:304, 348; interactions.py:90).
 *
 * Kernel scaling: G = 1/(4 pi |x-y|) (3D) and G = -log|x-y| / (2 pi) (2D); the
 * double layer is the source-normal derivative of G.  Scaling is applied once, at
 * assembly.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../include/qbxfmm.h"

typedef double complex cplx;

#define IDX3(n, m) ((n) * ((n) + 1) / 2 + (m))

int orc_ncoeff(const qbxfmm_kernel* k, int order)
{
  if (k->family == QBXFMM_LAPLACE) {
    if (k->dim == 3) return (order + 1) * (order + 2) / 2;
    return order + 1;
  }
  if (k->dim == 2) return 2 * order + 1;
  return (order + 1) * (order + 1);
}

static double level_width(const qbxfmm_geometry* g, int level)
{
  return g->root_extent / (double)(1 << level);
}

/* {{{ 3D Laplace solid harmonics */

static void sh3_R(int p, double x, double y, double z, cplx* R)
{
  double r2 = x * x + y * y + z * z;
  cplx xi = x + I * y;
  cplx rmm = 1.0;
  for (int m = 0; m <= p; ++m) {
    if (m > 0) rmm *= xi / (2.0 * m);
    R[IDX3(m, m)] = rmm;
    if (m + 1 <= p) R[IDX3(m + 1, m)] = z * rmm;
    for (int n = m + 2; n <= p; ++n)
      R[IDX3(n, m)] = ((2.0 * n - 1) * z * R[IDX3(n - 1, m)] - r2 * R[IDX3(n - 2, m)])
                      / ((double)(n + m) * (n - m));
  }
}

static void sh3_S(int p, double x, double y, double z, cplx* S)
{
  double r2 = x * x + y * y + z * z;
  double rinv2 = 1.0 / r2;
  cplx xi = x + I * y;
  cplx smm = 1.0 / sqrt(r2);
  for (int m = 0; m <= p; ++m) {
    if (m > 0) smm *= (2.0 * m - 1) * xi * rinv2;
    S[IDX3(m, m)] = smm;
    if (m + 1 <= p) S[IDX3(m + 1, m)] = (2.0 * m + 1) * z * smm * rinv2;
    for (int n = m + 2; n <= p; ++n)
      S[IDX3(n, m)] = ((2.0 * n - 1) * z * S[IDX3(n - 1, m)]
                       - (double)(n + m - 1) * (n - m - 1) * S[IDX3(n - 2, m)]) * rinv2;
  }
}

/* value at (n, m) for any sign of m; zero outside |m| <= n, n >= 0 */
static inline cplx sh3_get(const cplx* A, int n, int m)
{
  if (n < 0) return 0;
  if (m >= 0) return (m <= n) ? A[IDX3(n, m)] : 0;
  m = -m;
  if (m > n) return 0;
  return (m & 1) ? -conj(A[IDX3(n, m)]) : conj(A[IDX3(n, m)]);
}

/* P2M: charge q and dipole sigma*dvec at y into multipole about c (rscale rho) */
static void lap3_p2m(int p, double rho, const double* c, const double* y, double q,
                     double sigma, const double* dvec, cplx* M, cplx* work)
{
  double u[3] = {(y[0] - c[0]) / rho, (y[1] - c[1]) / rho, (y[2] - c[2]) / rho};
  sh3_R(p, u[0], u[1], u[2], work);
  for (int n = 0; n <= p; ++n)
    for (int m = 0; m <= n; ++m) {
      cplx v = q * conj(work[IDX3(n, m)]);
      if (sigma != 0 && n >= 1) {
        cplx dp = dvec[0] + I * dvec[1], dm = dvec[0] - I * dvec[1];
        cplx dr = dvec[2] * sh3_get(work, n - 1, m) + 0.5 * dp * sh3_get(work, n - 1, m - 1)
                  - 0.5 * dm * sh3_get(work, n - 1, m + 1);
        v += (sigma / rho) * conj(dr);
      }
      M[IDX3(n, m)] += v;
    }
}

/* P2L: charge/dipole at y into local about c (rscale rho) */
static void lap3_p2l(int p, double rho, const double* c, const double* y, double q,
                     double sigma, const double* dvec, cplx* L, cplx* work)
{
  double u[3] = {(y[0] - c[0]) / rho, (y[1] - c[1]) / rho, (y[2] - c[2]) / rho};
  sh3_S(p + 1, u[0], u[1], u[2], work);
  for (int n = 0; n <= p; ++n)
    for (int m = 0; m <= n; ++m) {
      cplx v = (q / rho) * work[IDX3(n, m)];
      if (sigma != 0) {
        cplx dp = dvec[0] + I * dvec[1], dm = dvec[0] - I * dvec[1];
        v += (sigma / (rho * rho))
             * (-dvec[2] * sh3_get(work, n + 1, m) + 0.5 * dp * sh3_get(work, n + 1, m - 1)
                - 0.5 * dm * sh3_get(work, n + 1, m + 1));
      }
      L[IDX3(n, m)] += v;
    }
}

static void lap3_m2m(int p, double rho_c, double rho_p, const double* d_over_rhop,
                     const cplx* Min, cplx* Mout, cplx* work)
{
  sh3_R(p, d_over_rhop[0], d_over_rhop[1], d_over_rhop[2], work);
  double ratio = rho_c / rho_p;
  for (int n = 0; n <= p; ++n)
    for (int m = 0; m <= n; ++m) {
      cplx acc = 0;
      double rk = 1.0;
      for (int k = 0; k <= n; ++k, rk *= ratio)
        for (int l = -k; l <= k; ++l) {
          if (abs(m - l) > n - k) continue;
          acc += rk * sh3_get(Min, k, l) * conj(sh3_get(work, n - k, m - l));
        }
      Mout[IDX3(n, m)] += acc;
    }
}

static void lap3_m2l(int pin, int pout, double rho_s, double rho_t,
                     const double* d_over_rhos, const cplx* Min, cplx* Lout, cplx* work)
{
  sh3_S(pin + pout, d_over_rhos[0], d_over_rhos[1], d_over_rhos[2], work);
  double ratio = rho_t / rho_s;
  double rj = 1.0 / rho_s;
  for (int j = 0; j <= pout; ++j, rj *= ratio)
    for (int i = 0; i <= j; ++i) {
      cplx acc = 0;
      for (int k = 0; k <= pin; ++k)
        for (int l = -k; l <= k; ++l)
          acc += sh3_get(Min, k, l) * sh3_get(work, k + j, l + i);
      Lout[IDX3(j, i)] += ((j & 1) ? -rj : rj) * acc;
    }
}

static void lap3_l2l(int pin, int pout, double rho_p, double rho_c,
                     const double* d_over_rhop, const cplx* Lin, cplx* Lout, cplx* work)
{
  sh3_R(pin, d_over_rhop[0], d_over_rhop[1], d_over_rhop[2], work);
  double ratio = rho_c / rho_p;
  double rk = 1.0;
  for (int k = 0; k <= pout; ++k, rk *= ratio)
    for (int l = 0; l <= k; ++l) {
      cplx acc = 0;
      for (int n = k; n <= pin; ++n)
        for (int m = -n; m <= n; ++m) {
          if (abs(m - l) > n - k) continue;
          acc += sh3_get(Lin, n, m) * conj(sh3_get(work, n - k, m - l));
        }
      Lout[IDX3(k, l)] += rk * acc;
    }
}

static double lap3_l2p(int p, double rho, const double* c, const double* x,
                       const cplx* L, cplx* work)
{
  sh3_R(p, (x[0] - c[0]) / rho, (x[1] - c[1]) / rho, (x[2] - c[2]) / rho, work);
  double acc = 0;
  for (int n = 0; n <= p; ++n) {
    acc += creal(L[IDX3(n, 0)] * conj(work[IDX3(n, 0)]));
    for (int m = 1; m <= n; ++m) acc += 2 * creal(L[IDX3(n, m)] * conj(work[IDX3(n, m)]));
  }
  return acc;
}

static double lap3_m2p(int p, double rho, const double* c, const double* x,
                       const cplx* M, cplx* work)
{
  sh3_S(p, (x[0] - c[0]) / rho, (x[1] - c[1]) / rho, (x[2] - c[2]) / rho, work);
  double acc = 0;
  for (int n = 0; n <= p; ++n) {
    acc += creal(M[IDX3(n, 0)] * work[IDX3(n, 0)]);
    for (int m = 1; m <= n; ++m) acc += 2 * creal(M[IDX3(n, m)] * work[IDX3(n, m)]);
  }
  return acc / rho;
}

static double lap3_p2p(const double* x, const double* y, double q, double sigma,
                       const double* dvec)
{
  double d0 = x[0] - y[0], d1 = x[1] - y[1], d2 = x[2] - y[2];
  double r2 = d0 * d0 + d1 * d1 + d2 * d2;
  if (r2 == 0) return 0;
  double rinv = 1.0 / sqrt(r2);
  double v = q * rinv;
  if (sigma != 0) v += sigma * (dvec[0] * d0 + dvec[1] * d1 + dvec[2] * d2) * rinv * rinv * rinv;
  return v;
}

/* }}} */

/* {{{ 2D Laplace (complex analytic) */

static double binom(int n, int k)
{
  if (k < 0 || k > n) return 0;
  double r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

static void lap2_p2m(int p, double rho, const double* c, const double* y, double q,
                     double sigma, const double* dvec, cplx* M)
{
  cplx u = ((y[0] - c[0]) + I * (y[1] - c[1])) / rho;
  cplx nu = dvec ? dvec[0] + I * dvec[1] : 0;
  M[0] += q;
  cplx uk = 1.0; /* u^(k-1) */
  for (int k = 1; k <= p; ++k) {
    cplx v = -q * uk * u / k;
    if (sigma != 0) v += -sigma * nu * uk / rho;
    M[k] += v;
    uk *= u;
  }
}

static void lap2_p2l(int p, double rho, const double* c, const double* y, double q,
                     double sigma, const double* dvec, cplx* L)
{
  cplx t = (y[0] - c[0]) + I * (y[1] - c[1]);
  cplx tau = t / rho;
  cplx nu = dvec ? dvec[0] + I * dvec[1] : 0;
  cplx tinv = 1.0 / tau;
  L[0] += q * log(cabs(t)) + (sigma != 0 ? sigma * nu / rho * tinv : 0);
  cplx tl = tinv; /* tau^-l */
  for (int l = 1; l <= p; ++l) {
    cplx v = -q * tl / l;
    if (sigma != 0) v += sigma * nu / rho * tl * tinv;
    L[l] += v;
    tl *= tinv;
  }
}

static void lap2_m2m(int p, double rho_c, double rho_p, const double* d_over_rhop,
                     const cplx* Min, cplx* Mout)
{
  cplx t = d_over_rhop[0] + I * d_over_rhop[1];
  double ratio = rho_c / rho_p;
  Mout[0] += Min[0];
  for (int l = 1; l <= p; ++l) {
    cplx acc = -Min[0] * cpow(t, l) / l;
    double rk = ratio;
    for (int k = 1; k <= l; ++k, rk *= ratio)
      acc += Min[k] * rk * binom(l - 1, k - 1) * cpow(t, l - k);
    Mout[l] += acc;
  }
}

static void lap2_m2l(int pin, int pout, double rho_s, double rho_t,
                     const double* d_over_rhos, const cplx* Min, cplx* Lout)
{
  cplx tau = d_over_rhos[0] + I * d_over_rhos[1];
  cplx t = tau * rho_s;
  cplx tinv = 1.0 / tau;
  double ratio = rho_t / rho_s;
  cplx acc0 = Min[0] * clog(t);
  for (int k = 1; k <= pin; ++k) acc0 += Min[k] * cpow(tinv, k);
  Lout[0] += acc0;
  double rl = ratio;
  for (int l = 1; l <= pout; ++l, rl *= ratio) {
    cplx tl = cpow(tinv, l);
    cplx acc = Min[0] * ((l & 1) ? 1.0 : -1.0) / l * tl;
    cplx s = 0;
    for (int k = 1; k <= pin; ++k) s += Min[k] * binom(k + l - 1, l) * cpow(tinv, k);
    acc += ((l & 1) ? -1.0 : 1.0) * tl * s;
    Lout[l] += rl * acc;
  }
}

static void lap2_l2l(int pin, int pout, double rho_p, double rho_c,
                     const double* d_over_rhop, const cplx* Lin, cplx* Lout)
{
  cplx s = d_over_rhop[0] + I * d_over_rhop[1];
  double ratio = rho_c / rho_p;
  double rl = 1.0;
  for (int l = 0; l <= pout; ++l, rl *= ratio) {
    cplx acc = 0;
    for (int k = l; k <= pin; ++k) acc += Lin[k] * binom(k, l) * cpow(s, k - l);
    Lout[l] += rl * acc;
  }
}

static double lap2_l2p(int p, double rho, const double* c, const double* x, const cplx* L)
{
  cplx u = ((x[0] - c[0]) + I * (x[1] - c[1])) / rho;
  cplx acc = 0, uk = 1.0;
  for (int k = 0; k <= p; ++k) {
    acc += L[k] * uk;
    uk *= u;
  }
  return creal(acc);
}

static double lap2_m2p(int p, double rho, const double* c, const double* x, const cplx* M)
{
  cplx zc = (x[0] - c[0]) + I * (x[1] - c[1]);
  cplx uinv = rho / zc;
  cplx acc = M[0] * clog(zc), uk = uinv;
  for (int k = 1; k <= p; ++k) {
    acc += M[k] * uk;
    uk *= uinv;
  }
  return creal(acc);
}

static double lap2_p2p(const double* x, const double* y, double q, double sigma,
                       const double* dvec)
{
  double d0 = x[0] - y[0], d1 = x[1] - y[1];
  double r2 = d0 * d0 + d1 * d1;
  if (r2 == 0) return 0;
  double v = 0.5 * q * log(r2);
  if (sigma != 0) v += -sigma * (dvec[0] * d0 + dvec[1] * d1) / r2;
  return v;
}

/* }}} */

/* {{{ dispatch helpers */

typedef struct {
  int dim, pf, pq, nrhs, ncf, ncq;
  double cq, cd;
} ctx_t;

/* Per-level FMM orders of the Laplace stages (the reference's fmm_level_to_order,
   pytential/qbx/__init__.py:276-285, read per level as the wrangler's level_orders,
   pytential/qbx/fmm.py:280-283, 327-330): each box expansion has its level's order and
   every translation runs between the orders of its two ends (expansions are stored at
   fmm_order with zeros above the box's order).  Empty: fmm_order everywhere. */
static int g_lorders[64];
static int g_nlorders = 0;

int orc_set_level_orders(const int* orders, int nlevels)
{
  if (!orders || nlevels <= 0) {
    g_nlorders = 0;
    return 0;
  }
  if (nlevels > 64) return QBXFMM_ERR_ARG;
  for (int l = 0; l < nlevels; ++l) g_lorders[l] = orders[l];
  g_nlorders = nlevels;
  return 0;
}

static int lp(const ctx_t* c, int level)
{
  return (g_nlorders && level >= 0 && level < g_nlorders) ? g_lorders[level] : c->pf;
}

static int make_ctx(const qbxfmm_kernel* k, ctx_t* c)
{
  if (k->family != QBXFMM_LAPLACE) return QBXFMM_ERR_UNSUPPORTED;
  if (k->dim != 2 && k->dim != 3) return QBXFMM_ERR_ARG;
  c->dim = k->dim;
  c->pf = k->fmm_order;
  c->pq = k->qbx_order;
  c->nrhs = k->nrhs;
  c->ncf = orc_ncoeff(k, k->fmm_order);
  c->ncq = orc_ncoeff(k, k->qbx_order);
  c->cq = k->charge_coeff_re;
  c->cd = k->dipole_coeff_re;
  return 0;
}

static void load(const double* soa, int n, int i, int dim, double* out)
{
  for (int d = 0; d < dim; ++d) out[d] = soa[(size_t)d * n + i];
}

static int work_size(int p) { return (p + 3) * (p + 4) / 2 * 4 + 64; }

/* }}} */


/* {{{ 2D Helmholtz forward declarations (qbxfmm_oracle_helm2d.c) */
static int h2_form_multipoles(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h2_coarsen_multipoles(const qbxfmm_kernel*, const qbxfmm_geometry*, cplx*);
static int h2_eval_direct(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h2_multipole_to_local(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h2_eval_multipoles(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h2_form_locals(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h2_refine_locals(const qbxfmm_kernel*, const qbxfmm_geometry*, cplx*);
static int h2_eval_locals(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h2_p2qbxl(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*, int);
static int h2_m2qbxl(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h2_l2qbxl(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h2_eval_qbx_expansions(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h2_assemble(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, const cplx*, cplx*);
static int h2_apply(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*, int);
/* }}} */

/* {{{ 3D Helmholtz forward declarations (qbxfmm_oracle_helm3d.c) */
static int h3_form_multipoles(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h3_coarsen_multipoles(const qbxfmm_kernel*, const qbxfmm_geometry*, cplx*);
static int h3_eval_direct(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h3_multipole_to_local(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h3_eval_multipoles(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h3_form_locals(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h3_refine_locals(const qbxfmm_kernel*, const qbxfmm_geometry*, cplx*);
static int h3_eval_locals(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h3_p2qbxl(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*, int);
static int h3_m2qbxl(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h3_l2qbxl(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h3_eval_qbx_expansions(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*);
static int h3_assemble(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, const cplx*, cplx*);
static int h3_apply(const qbxfmm_kernel*, const qbxfmm_geometry*, const cplx*, cplx*, int);
/* }}} */

#define IS_HELM(k) ((k)->family == QBXFMM_HELMHOLTZ)

/* {{{ stages */

int orc_form_multipoles(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                        const double* strengths, cplx* mpoles)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_form_multipoles(kern, g, (const cplx*)strengths, mpoles) : h2_form_multipoles(kern, g, (const cplx*)strengths, mpoles);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* work = malloc(sizeof(cplx) * work_size(c.pf));
#pragma omp for schedule(dynamic, 4)
    for (int isb = 0; isb < g->nsource_boxes; ++isb) {
      int b = g->source_boxes[isb];
      double rho = level_width(g, g->box_levels[b]);
      double ctr[3], y[3], nv[3] = {0, 0, 0};
      load(g->box_centers, g->nboxes, b, c.dim, ctr);
      int s0 = g->box_source_starts[b], s1 = s0 + g->box_source_counts_nonchild[b];
      for (int r = 0; r < c.nrhs; ++r) {
        cplx* M = mpoles + ((size_t)b * c.nrhs + r) * c.ncf;
        for (int s = s0; s < s1; ++s) {
          load(g->sources, g->nsources, s, c.dim, y);
          if (c.cd != 0) load(g->source_normals, g->nsources, s, c.dim, nv);
          double st = strengths[(size_t)r * g->nsources + s];
          if (c.dim == 3)
            lap3_p2m(lp(&c, g->box_levels[b]), rho, ctr, y, c.cq * st, c.cd * st, nv, M, work);
          else
            lap2_p2m(lp(&c, g->box_levels[b]), rho, ctr, y, c.cq * st, c.cd * st, nv, M);
        }
      }
    }
    free(work);
  }
  return 0;
}

int orc_coarsen_multipoles(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                           cplx* mpoles)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_coarsen_multipoles(kern, g, mpoles) : h2_coarsen_multipoles(kern, g, mpoles);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
  int nch = 1 << c.dim;
  for (int lev = g->nlevels - 2; lev >= 0; --lev) {
    int i0 = g->level_start_source_parent_box_nrs[lev];
    int i1 = g->level_start_source_parent_box_nrs[lev + 1];
#pragma omp parallel
    {
      cplx* work = malloc(sizeof(cplx) * work_size(c.pf));
#pragma omp for schedule(dynamic, 1)
      for (int i = i0; i < i1; ++i) {
        int b = g->source_parent_boxes[i];
        double rho_p = level_width(g, lev), rho_c = level_width(g, lev + 1);
        double cp[3], cc[3], d[3];
        load(g->box_centers, g->nboxes, b, c.dim, cp);
        for (int ci = 0; ci < nch; ++ci) {
          int ch = g->box_child_ids[(size_t)ci * g->nboxes + b];
          if (ch == 0 || g->box_source_counts_cumul[ch] == 0) continue;
          load(g->box_centers, g->nboxes, ch, c.dim, cc);
          for (int dd = 0; dd < c.dim; ++dd) d[dd] = (cc[dd] - cp[dd]) / rho_p;
          for (int r = 0; r < c.nrhs; ++r) {
            const cplx* Min = mpoles + ((size_t)ch * c.nrhs + r) * c.ncf;
            cplx* Mout = mpoles + ((size_t)b * c.nrhs + r) * c.ncf;
            if (c.dim == 3) lap3_m2m(lp(&c, lev), rho_c, rho_p, d, Min, Mout, work);
            else lap2_m2m(lp(&c, lev), rho_c, rho_p, d, Min, Mout);
          }
        }
      }
      free(work);
    }
  }
  return 0;
}

/* list 1 direct evaluation at non-QBX targets (adds into pot[nrhs][nfiltered]) */
int orc_eval_direct(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                    const double* strengths, double* pot)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_eval_direct(kern, g, (const cplx*)strengths, (cplx*)pot) : h2_eval_direct(kern, g, (const cplx*)strengths, (cplx*)pot);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel for schedule(dynamic, 1)
  for (int itb = 0; itb < g->ntarget_boxes; ++itb) {
    int tb = g->target_boxes[itb];
    int t0 = g->nonqbx_box_target_starts[tb];
    int t1 = t0 + g->nonqbx_box_target_counts_nonchild[tb];
    if (t1 == t0) continue;
    for (int t = t0; t < t1; ++t) {
      double x[3], y[3], nv[3] = {0, 0, 0};
      load(g->nonqbx_targets, g->nfiltered_targets, t, c.dim, x);
      for (int r = 0; r < c.nrhs; ++r) {
        double acc = 0;
        for (int li = g->list1_starts[itb]; li < g->list1_starts[itb + 1]; ++li) {
          int sb = g->list1_lists[li];
          int s0 = g->box_source_starts[sb], s1 = s0 + g->box_source_counts_nonchild[sb];
          for (int s = s0; s < s1; ++s) {
            load(g->sources, g->nsources, s, c.dim, y);
            if (c.cd != 0) load(g->source_normals, g->nsources, s, c.dim, nv);
            double st = strengths[(size_t)r * g->nsources + s];
            acc += (c.dim == 3) ? lap3_p2p(x, y, c.cq * st, c.cd * st, nv)
                                : lap2_p2p(x, y, c.cq * st, c.cd * st, nv);
          }
        }
        pot[(size_t)r * g->nfiltered_targets + t] += acc;
      }
    }
  }
  return 0;
}

int orc_multipole_to_local(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                           const cplx* mpoles, cplx* locals)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_multipole_to_local(kern, g, mpoles, locals) : h2_multipole_to_local(kern, g, mpoles, locals);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* work = malloc(sizeof(cplx) * work_size(2 * c.pf));
#pragma omp for schedule(dynamic, 1)
    for (int i = 0; i < g->nttp_boxes; ++i) {
      int tb = g->target_or_target_parent_boxes[i];
      double rho = level_width(g, g->box_levels[tb]);
      double ct[3], cs[3], d[3];
      load(g->box_centers, g->nboxes, tb, c.dim, ct);
      for (int li = g->list2_starts[i]; li < g->list2_starts[i + 1]; ++li) {
        int sb = g->list2_lists[li];
        load(g->box_centers, g->nboxes, sb, c.dim, cs);
        for (int dd = 0; dd < c.dim; ++dd) d[dd] = (ct[dd] - cs[dd]) / rho;
        for (int r = 0; r < c.nrhs; ++r) {
          const cplx* Min = mpoles + ((size_t)sb * c.nrhs + r) * c.ncf;
          cplx* Lout = locals + ((size_t)tb * c.nrhs + r) * c.ncf;
          const int ps = lp(&c, g->box_levels[sb]), pt = lp(&c, g->box_levels[tb]);
          if (c.dim == 3) lap3_m2l(ps, pt, rho, rho, d, Min, Lout, work);
          else lap2_m2l(ps, pt, rho, rho, d, Min, Lout);
        }
      }
    }
    free(work);
  }
  return 0;
}

/* list 3 multipoles evaluated at non-QBX targets */
int orc_eval_multipoles(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                        const cplx* mpoles, double* pot)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_eval_multipoles(kern, g, mpoles, (cplx*)pot) : h2_eval_multipoles(kern, g, mpoles, (cplx*)pot);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* work = malloc(sizeof(cplx) * work_size(c.pf));
#pragma omp for schedule(dynamic, 1)
    for (int itb = 0; itb < g->ntarget_boxes; ++itb) {
      int tb = g->target_boxes[itb];
      int t0 = g->nonqbx_box_target_starts[tb];
      int t1 = t0 + g->nonqbx_box_target_counts_nonchild[tb];
      for (int t = t0; t < t1; ++t) {
        double x[3], cs[3];
        load(g->nonqbx_targets, g->nfiltered_targets, t, c.dim, x);
        for (int li = g->list3_starts[itb]; li < g->list3_starts[itb + 1]; ++li) {
          int sb = g->list3_lists[li];
          double rho = level_width(g, g->box_levels[sb]);
          load(g->box_centers, g->nboxes, sb, c.dim, cs);
          for (int r = 0; r < c.nrhs; ++r) {
            const cplx* M = mpoles + ((size_t)sb * c.nrhs + r) * c.ncf;
            pot[(size_t)r * g->nfiltered_targets + t] +=
                (c.dim == 3) ? lap3_m2p(lp(&c, g->box_levels[sb]), rho, cs, x, M, work)
                             : lap2_m2p(lp(&c, g->box_levels[sb]), rho, cs, x, M);
          }
        }
      }
    }
    free(work);
  }
  return 0;
}

/* list 4 sources into box locals */
int orc_form_locals(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                    const double* strengths, cplx* locals)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_form_locals(kern, g, (const cplx*)strengths, locals) : h2_form_locals(kern, g, (const cplx*)strengths, locals);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* work = malloc(sizeof(cplx) * work_size(c.pf + 1));
#pragma omp for schedule(dynamic, 1)
    for (int i = 0; i < g->nttp_boxes; ++i) {
      int tb = g->target_or_target_parent_boxes[i];
      double rho = level_width(g, g->box_levels[tb]);
      double ct[3], y[3], nv[3] = {0, 0, 0};
      load(g->box_centers, g->nboxes, tb, c.dim, ct);
      for (int li = g->list4_starts[i]; li < g->list4_starts[i + 1]; ++li) {
        int sb = g->list4_lists[li];
        int s0 = g->box_source_starts[sb], s1 = s0 + g->box_source_counts_nonchild[sb];
        for (int s = s0; s < s1; ++s) {
          load(g->sources, g->nsources, s, c.dim, y);
          if (c.cd != 0) load(g->source_normals, g->nsources, s, c.dim, nv);
          for (int r = 0; r < c.nrhs; ++r) {
            double st = strengths[(size_t)r * g->nsources + s];
            cplx* L = locals + ((size_t)tb * c.nrhs + r) * c.ncf;
            if (c.dim == 3) lap3_p2l(lp(&c, g->box_levels[tb]), rho, ct, y, c.cq * st, c.cd * st, nv, L, work);
            else lap2_p2l(lp(&c, g->box_levels[tb]), rho, ct, y, c.cq * st, c.cd * st, nv, L);
          }
        }
      }
    }
    free(work);
  }
  return 0;
}

int orc_refine_locals(const qbxfmm_kernel* kern, const qbxfmm_geometry* g, cplx* locals)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_refine_locals(kern, g, locals) : h2_refine_locals(kern, g, locals);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
  for (int lev = 1; lev < g->nlevels; ++lev) {
    int i0 = g->level_start_ttp_box_nrs[lev], i1 = g->level_start_ttp_box_nrs[lev + 1];
#pragma omp parallel
    {
      cplx* work = malloc(sizeof(cplx) * work_size(c.pf));
#pragma omp for schedule(dynamic, 4)
      for (int i = i0; i < i1; ++i) {
        int b = g->target_or_target_parent_boxes[i];
        int par = g->box_parent_ids[b];
        double rho_p = level_width(g, lev - 1), rho_c = level_width(g, lev);
        double cp[3], cc[3], d[3];
        load(g->box_centers, g->nboxes, par, c.dim, cp);
        load(g->box_centers, g->nboxes, b, c.dim, cc);
        for (int dd = 0; dd < c.dim; ++dd) d[dd] = (cc[dd] - cp[dd]) / rho_p;
        for (int r = 0; r < c.nrhs; ++r) {
          const cplx* Lin = locals + ((size_t)par * c.nrhs + r) * c.ncf;
          cplx* Lout = locals + ((size_t)b * c.nrhs + r) * c.ncf;
          if (c.dim == 3) lap3_l2l(lp(&c, lev - 1), lp(&c, lev), rho_p, rho_c, d, Lin, Lout, work);
          else lap2_l2l(lp(&c, lev - 1), lp(&c, lev), rho_p, rho_c, d, Lin, Lout);
        }
      }
      free(work);
    }
  }
  return 0;
}

int orc_eval_locals(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                    const cplx* locals, double* pot)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_eval_locals(kern, g, locals, (cplx*)pot) : h2_eval_locals(kern, g, locals, (cplx*)pot);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* work = malloc(sizeof(cplx) * work_size(c.pf));
#pragma omp for schedule(dynamic, 4)
    for (int itb = 0; itb < g->ntarget_boxes; ++itb) {
      int tb = g->target_boxes[itb];
      int t0 = g->nonqbx_box_target_starts[tb];
      int t1 = t0 + g->nonqbx_box_target_counts_nonchild[tb];
      double rho = level_width(g, g->box_levels[tb]);
      double ct[3], x[3];
      load(g->box_centers, g->nboxes, tb, c.dim, ct);
      for (int t = t0; t < t1; ++t) {
        load(g->nonqbx_targets, g->nfiltered_targets, t, c.dim, x);
        for (int r = 0; r < c.nrhs; ++r) {
          const cplx* L = locals + ((size_t)tb * c.nrhs + r) * c.ncf;
          pot[(size_t)r * g->nfiltered_targets + t] +=
              (c.dim == 3) ? lap3_l2p(lp(&c, g->box_levels[tb]), rho, ct, x, L, work)
                           : lap2_l2p(lp(&c, g->box_levels[tb]), rho, ct, x, L);
        }
      }
    }
    free(work);
  }
  return 0;
}

/* P2QBXL over list 1 (fmm.py:231-265; interactions.py:84-124).  If all_sources,
 * every source contributes (direct, non-FMM QBX). */
static int p2qbxl_impl(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                       const double* strengths, cplx* qbx_exps, int all_sources)
{
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* work = malloc(sizeof(cplx) * work_size(c.pq + 1));
#pragma omp for schedule(dynamic, 16)
    for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
      int ctr = g->global_qbx_centers[ig];
      double cc[3], y[3], nv[3] = {0, 0, 0};
      load(g->centers, g->ncenters, ctr, c.dim, cc);
      double rho = g->expansion_radii[ctr];
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
        for (int s = s0; s < s1; ++s) {
          load(g->sources, g->nsources, s, c.dim, y);
          if (c.cd != 0) load(g->source_normals, g->nsources, s, c.dim, nv);
          for (int r = 0; r < c.nrhs; ++r) {
            double st = strengths[(size_t)r * g->nsources + s];
            cplx* L = qbx_exps + ((size_t)ctr * c.nrhs + r) * c.ncq;
            if (c.dim == 3) lap3_p2l(c.pq, rho, cc, y, c.cq * st, c.cd * st, nv, L, work);
            else lap2_p2l(c.pq, rho, cc, y, c.cq * st, c.cd * st, nv, L);
          }
        }
      }
    }
    free(work);
  }
  return 0;
}

int orc_form_global_qbx_locals(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                               const double* strengths, cplx* qbx_exps)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_p2qbxl(kern, g, (const cplx*)strengths, qbx_exps, 0) : h2_p2qbxl(kern, g, (const cplx*)strengths, qbx_exps, 0);
  return p2qbxl_impl(kern, g, strengths, qbx_exps, 0);
}

/* M2QBXL (fmm.py:267-312; interactions.py:196-235), for the used centers */
int orc_translate_box_multipoles_to_qbx_local(const qbxfmm_kernel* kern,
                                              const qbxfmm_geometry* g,
                                              const cplx* mpoles, cplx* qbx_exps)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_m2qbxl(kern, g, mpoles, qbx_exps) : h2_m2qbxl(kern, g, mpoles, qbx_exps);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* work = malloc(sizeof(cplx) * work_size(c.pf + c.pq));
#pragma omp for schedule(dynamic, 16)
    for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
      int ctr = g->global_qbx_centers[ig];
      double cc[3], cs[3], d[3];
      load(g->centers, g->ncenters, ctr, c.dim, cc);
      double rho_t = g->expansion_radii[ctr];
      int itb = g->qbx_center_to_target_box[ctr];
      for (int li = g->list3_starts[itb]; li < g->list3_starts[itb + 1]; ++li) {
        int sb = g->list3_lists[li];
        double rho_s = level_width(g, g->box_levels[sb]);
        load(g->box_centers, g->nboxes, sb, c.dim, cs);
        for (int dd = 0; dd < c.dim; ++dd) d[dd] = (cc[dd] - cs[dd]) / rho_s;
        for (int r = 0; r < c.nrhs; ++r) {
          const cplx* M = mpoles + ((size_t)sb * c.nrhs + r) * c.ncf;
          cplx* L = qbx_exps + ((size_t)ctr * c.nrhs + r) * c.ncq;
          if (c.dim == 3) lap3_m2l(lp(&c, g->box_levels[sb]), c.pq, rho_s, rho_t, d, M, L, work);
          else lap2_m2l(lp(&c, g->box_levels[sb]), c.pq, rho_s, rho_t, d, M, L);
        }
      }
    }
    free(work);
  }
  return 0;
}

/* L2QBXL (fmm.py:314-356; interactions.py:318-356), for the used centers */
int orc_translate_box_local_to_qbx_local(const qbxfmm_kernel* kern,
                                         const qbxfmm_geometry* g,
                                         const cplx* locals, cplx* qbx_exps)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_l2qbxl(kern, g, locals, qbx_exps) : h2_l2qbxl(kern, g, locals, qbx_exps);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* work = malloc(sizeof(cplx) * work_size(c.pf));
#pragma omp for schedule(dynamic, 16)
    for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
      int ctr = g->global_qbx_centers[ig];
      int tb = g->target_boxes[g->qbx_center_to_target_box[ctr]];
      double cc[3], cb[3], d[3];
      load(g->centers, g->ncenters, ctr, c.dim, cc);
      load(g->box_centers, g->nboxes, tb, c.dim, cb);
      double rho_b = level_width(g, g->box_levels[tb]);
      double rho_c = g->expansion_radii[ctr];
      for (int dd = 0; dd < c.dim; ++dd) d[dd] = (cc[dd] - cb[dd]) / rho_b;
      for (int r = 0; r < c.nrhs; ++r) {
        const cplx* Lin = locals + ((size_t)tb * c.nrhs + r) * c.ncf;
        cplx* L = qbx_exps + ((size_t)ctr * c.nrhs + r) * c.ncq;
        if (c.dim == 3) lap3_l2l(lp(&c, g->box_levels[tb]), c.pq, rho_b, rho_c, d, Lin, L, work);
        else lap2_l2l(lp(&c, g->box_levels[tb]), c.pq, rho_b, rho_c, d, Lin, L);
      }
    }
    free(work);
  }
  return 0;
}

/* QBXL2P (fmm.py:358-389; interactions.py:442-479): writes pot_tree[nrhs][ntargets] */
int orc_eval_qbx_expansions(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                            const cplx* qbx_exps, double* pot_tree)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_eval_qbx_expansions(kern, g, qbx_exps, (cplx*)pot_tree) : h2_eval_qbx_expansions(kern, g, qbx_exps, (cplx*)pot_tree);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx* work = malloc(sizeof(cplx) * work_size(c.pq));
#pragma omp for schedule(dynamic, 16)
    for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
      int ctr = g->global_qbx_centers[ig];
      double cc[3], x[3];
      load(g->centers, g->ncenters, ctr, c.dim, cc);
      double rho = g->expansion_radii[ctr];
      for (int it = g->center_to_targets_starts[ctr]; it < g->center_to_targets_starts[ctr + 1];
           ++it) {
        int t = g->center_to_targets_lists[it];
        load(g->targets, g->ntargets, t, c.dim, x);
        for (int r = 0; r < c.nrhs; ++r) {
          const cplx* L = qbx_exps + ((size_t)ctr * c.nrhs + r) * c.ncq;
          pot_tree[(size_t)r * g->ntargets + t] =
              (c.dim == 3) ? lap3_l2p(c.pq, rho, cc, x, L, work) : lap2_l2p(c.pq, rho, cc, x, L);
        }
      }
    }
    free(work);
  }
  return 0;
}

static double kernel_scaling(int dim) { return dim == 3 ? 0.25 / M_PI : -0.5 / M_PI; }

/* fmm.py:569-588 + qbx/__init__.py:775-793: non-QBX part scattered into tree
 * order, QBX part added, reorder to user targets, kernel scaling.
 * out: [nrhs][nuser_targets] */
int orc_assemble(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                 const double* pot_nonqbx, const double* pot_tree, double* out)
{
  if (IS_HELM(kern))
    return kern->dim == 3
               ? h3_assemble(kern, g, (const cplx*)pot_nonqbx, (const cplx*)pot_tree, (cplx*)out)
               : h2_assemble(kern, g, (const cplx*)pot_nonqbx, (const cplx*)pot_tree, (cplx*)out);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
  double scale = kernel_scaling(c.dim);
  double* full = malloc(sizeof(double) * g->ntargets);
  for (int r = 0; r < c.nrhs; ++r) {
    memcpy(full, pot_tree + (size_t)r * g->ntargets, sizeof(double) * g->ntargets);
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

/* The whole apply, in drive_fmm's order (fmm.py:436-588).  strengths are in tree
 * order; out is [nrhs][nuser_targets] in user order. */
int orc_apply(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
              const double* strengths, double* out)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_apply(kern, g, (const cplx*)strengths, (cplx*)out, 0) : h2_apply(kern, g, (const cplx*)strengths, (cplx*)out, 0);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
  size_t nexp = (size_t)g->nboxes * c.nrhs * c.ncf;
  cplx* mpoles = calloc(nexp, sizeof(cplx));
  cplx* locals = calloc(nexp, sizeof(cplx));
  cplx* qexp = calloc((size_t)g->ncenters * c.nrhs * c.ncq, sizeof(cplx));
  double* pnq = calloc((size_t)c.nrhs * g->nfiltered_targets + 1, sizeof(double));
  double* ptree = calloc((size_t)c.nrhs * g->ntargets + 1, sizeof(double));
  orc_form_multipoles(kern, g, strengths, mpoles);
  orc_coarsen_multipoles(kern, g, mpoles);
  orc_eval_direct(kern, g, strengths, pnq);
  orc_multipole_to_local(kern, g, mpoles, locals);
  orc_eval_multipoles(kern, g, mpoles, pnq);
  orc_form_locals(kern, g, strengths, locals);
  orc_refine_locals(kern, g, locals);
  orc_eval_locals(kern, g, locals, pnq);
  orc_form_global_qbx_locals(kern, g, strengths, qexp);
  orc_translate_box_multipoles_to_qbx_local(kern, g, mpoles, qexp);
  orc_translate_box_local_to_qbx_local(kern, g, locals, qexp);
  orc_eval_qbx_expansions(kern, g, qexp, ptree);
  orc_assemble(kern, g, pnq, ptree, out);
  free(mpoles);
  free(locals);
  free(qexp);
  free(pnq);
  free(ptree);
  return 0;
}

/* Direct (non-FMM) QBX: QBX targets get the QBX local formed from all sources,
 * non-QBX targets the direct sum over all sources (the reference's direct path,
 * pytential/qbx/__init__.py:797-1068, with the same truncation). */
int orc_apply_direct(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                     const double* strengths, double* out)
{
  if (IS_HELM(kern)) return kern->dim == 3 ? h3_apply(kern, g, (const cplx*)strengths, (cplx*)out, 1) : h2_apply(kern, g, (const cplx*)strengths, (cplx*)out, 1);
  ctx_t c;
  int rc = make_ctx(kern, &c);
  if (rc) return rc;
  cplx* qexp = calloc((size_t)g->ncenters * c.nrhs * c.ncq, sizeof(cplx));
  double* pnq = calloc((size_t)c.nrhs * g->nfiltered_targets + 1, sizeof(double));
  double* ptree = calloc((size_t)c.nrhs * g->ntargets + 1, sizeof(double));
  p2qbxl_impl(kern, g, strengths, qexp, 1);
  orc_eval_qbx_expansions(kern, g, qexp, ptree);
#pragma omp parallel for schedule(dynamic, 16)
  for (int t = 0; t < g->nfiltered_targets; ++t) {
    double x[3], y[3], nv[3] = {0, 0, 0};
    load(g->nonqbx_targets, g->nfiltered_targets, t, c.dim, x);
    for (int r = 0; r < c.nrhs; ++r) {
      double acc = 0;
      for (int s = 0; s < g->nsources; ++s) {
        load(g->sources, g->nsources, s, c.dim, y);
        if (c.cd != 0) load(g->source_normals, g->nsources, s, c.dim, nv);
        double st = strengths[(size_t)r * g->nsources + s];
        acc += (c.dim == 3) ? lap3_p2p(x, y, c.cq * st, c.cd * st, nv)
                            : lap2_p2p(x, y, c.cq * st, c.cd * st, nv);
      }
      pnq[(size_t)r * g->nfiltered_targets + t] = acc;
    }
  }
  orc_assemble(kern, g, pnq, ptree, out);
  free(qexp);
  free(pnq);
  free(ptree);
  return 0;
}

/* }}} */

/* {{{ transposed QBX stages (Laplace single layer, 2D and 3D)
 *
 * The transposes of QBXL2P, L2QBXL, M2QBXL and P2QBXL (fmm.py:231-389) in the
 * exchanged-role form: each global center carries the order-q multipole of its
 * targets' values times the charge coefficient (P2M about the center, its expansion
 * radius as rscale; the coefficient multiplies every path that starts there); it is
 * shifted into the multipole of its target box (M2M from the center, the reciprocal
 * of the box-to-center L2L), converted into the local of every box of the target
 * box's list 3 (M2L from the center, the reciprocal of M2QBXL), and evaluated at
 * the sources of every box of the target box's list 1 (M2P, the reciprocal of
 * P2QBXL).  Each loop runs over the centers and scatters into boxes and sources,
 * one thread. */

static int transpose_ctx(const qbxfmm_kernel* kern, ctx_t* c)
{
  int rc = make_ctx(kern, c);
  if (rc) return rc;
  if (c->cd != 0) return QBXFMM_ERR_UNSUPPORTED;
  return 0;
}

/* tree_vals: [nrhs][ntargets] (tree target order); center_mpoles: [ncenters][nrhs][ncq] */
int orc_transpose_eval_qbx_expansions(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                                      const double* tree_vals, cplx* center_mpoles)
{
  ctx_t c;
  int rc = transpose_ctx(kern, &c);
  if (rc) return rc;
  cplx* work = malloc(sizeof(cplx) * work_size(c.pq));
  double zero[3] = {0, 0, 0};
  for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
    int ctr = g->global_qbx_centers[ig];
    double cc[3], x[3];
    load(g->centers, g->ncenters, ctr, c.dim, cc);
    double rho = g->expansion_radii[ctr];
    for (int it = g->center_to_targets_starts[ctr]; it < g->center_to_targets_starts[ctr + 1];
         ++it) {
      int t = g->center_to_targets_lists[it];
      load(g->targets, g->ntargets, t, c.dim, x);
      for (int r = 0; r < c.nrhs; ++r) {
        double q = c.cq * tree_vals[(size_t)r * g->ntargets + t];
        cplx* M = center_mpoles + ((size_t)ctr * c.nrhs + r) * c.ncq;
        if (c.dim == 3) lap3_p2m(c.pq, rho, cc, x, q, 0, zero, M, work);
        else lap2_p2m(c.pq, rho, cc, x, q, 0, NULL, M);
      }
    }
  }
  free(work);
  return 0;
}

int orc_transpose_translate_box_local_to_qbx_local(const qbxfmm_kernel* kern,
                                                   const qbxfmm_geometry* g,
                                                   const cplx* center_mpoles, cplx* mpoles)
{
  ctx_t c;
  int rc = transpose_ctx(kern, &c);
  if (rc) return rc;
  cplx* work = malloc(sizeof(cplx) * work_size(c.pf));
  cplx* pad = malloc(sizeof(cplx) * c.ncf);
  for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
    int ctr = g->global_qbx_centers[ig];
    int tb = g->target_boxes[g->qbx_center_to_target_box[ctr]];
    double cc[3], cb[3], d[3];
    load(g->centers, g->ncenters, ctr, c.dim, cc);
    load(g->box_centers, g->nboxes, tb, c.dim, cb);
    double rho_b = level_width(g, g->box_levels[tb]);
    double rho_c = g->expansion_radii[ctr];
    for (int dd = 0; dd < c.dim; ++dd) d[dd] = (cc[dd] - cb[dd]) / rho_b;
    for (int r = 0; r < c.nrhs; ++r) {
      /* the center multipole zero-padded to the box order */
      for (int i = 0; i < c.ncf; ++i) pad[i] = 0;
      memcpy(pad, center_mpoles + ((size_t)ctr * c.nrhs + r) * c.ncq, sizeof(cplx) * c.ncq);
      cplx* M = mpoles + ((size_t)tb * c.nrhs + r) * c.ncf;
      if (c.dim == 3) lap3_m2m(c.pf, rho_c, rho_b, d, pad, M, work);
      else lap2_m2m(c.pf, rho_c, rho_b, d, pad, M);
    }
  }
  free(pad);
  free(work);
  return 0;
}

int orc_transpose_translate_box_multipoles_to_qbx_local(const qbxfmm_kernel* kern,
                                                        const qbxfmm_geometry* g,
                                                        const cplx* center_mpoles, cplx* locals)
{
  ctx_t c;
  int rc = transpose_ctx(kern, &c);
  if (rc) return rc;
  cplx* work = malloc(sizeof(cplx) * work_size(c.pf + c.pq));
  for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
    int ctr = g->global_qbx_centers[ig];
    double cc[3], cs[3], d[3];
    load(g->centers, g->ncenters, ctr, c.dim, cc);
    double rho_c = g->expansion_radii[ctr];
    int itb = g->qbx_center_to_target_box[ctr];
    for (int li = g->list3_starts[itb]; li < g->list3_starts[itb + 1]; ++li) {
      int sb = g->list3_lists[li];
      double rho_s = level_width(g, g->box_levels[sb]);
      load(g->box_centers, g->nboxes, sb, c.dim, cs);
      for (int dd = 0; dd < c.dim; ++dd) d[dd] = (cs[dd] - cc[dd]) / rho_c;
      for (int r = 0; r < c.nrhs; ++r) {
        const cplx* M = center_mpoles + ((size_t)ctr * c.nrhs + r) * c.ncq;
        cplx* L = locals + ((size_t)sb * c.nrhs + r) * c.ncf;
        if (c.dim == 3) lap3_m2l(c.pq, lp(&c, g->box_levels[sb]), rho_c, rho_s, d, M, L, work);
        else lap2_m2l(c.pq, lp(&c, g->box_levels[sb]), rho_c, rho_s, d, M, L);
      }
    }
  }
  free(work);
  return 0;
}

/* source_vals: [nrhs][nsources] (tree source order), added to */
int orc_transpose_form_global_qbx_locals(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                                         const cplx* center_mpoles, double* source_vals)
{
  ctx_t c;
  int rc = transpose_ctx(kern, &c);
  if (rc) return rc;
  cplx* work = malloc(sizeof(cplx) * work_size(c.pq));
  for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
    int ctr = g->global_qbx_centers[ig];
    double cc[3], y[3];
    load(g->centers, g->ncenters, ctr, c.dim, cc);
    double rho = g->expansion_radii[ctr];
    int itb = g->qbx_center_to_target_box[ctr];
    for (int li = g->list1_starts[itb]; li < g->list1_starts[itb + 1]; ++li) {
      int sb = g->list1_lists[li];
      int s0 = g->box_source_starts[sb], s1 = s0 + g->box_source_counts_nonchild[sb];
      for (int s = s0; s < s1; ++s) {
        load(g->sources, g->nsources, s, c.dim, y);
        for (int r = 0; r < c.nrhs; ++r) {
          const cplx* M = center_mpoles + ((size_t)ctr * c.nrhs + r) * c.ncq;
          source_vals[(size_t)r * g->nsources + s] +=
              (c.dim == 3) ? lap3_m2p(c.pq, rho, cc, y, M, work) : lap2_m2p(c.pq, rho, cc, y, M);
        }
      }
    }
  }
  free(work);
  return 0;
}

/* }}} */

#include "qbxfmm_oracle_helm2d.c"
#include "qbxfmm_oracle_helm3d.c"
