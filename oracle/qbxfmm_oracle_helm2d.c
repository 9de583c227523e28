/*
 * 2D Helmholtz part of the CPU checker (TEST INFRASTRUCTURE ONLY), included by
 * qbxfmm_oracle.c.
 *
 * Expansions follow sumpy's default for the 2D Helmholtz kernel, the H2D
 * (Bessel/Hankel) local and multipole expansions of order p (|m| <= p), with the
 * kernel G = (i/4) H_0^(1)(k |x - y|).  Writing Z_m(u) = Z_m(k|u|) e^{i m arg u}
 * (Z = J or H = H^(1)), Graf's addition theorem gives
 *   J_n(a + b) = sum_m J_m(a) J_{n-m}(b),  H_n(a + b) = sum_m H_m(a) J_{n-m}(b) (|b| < |a|),
 *   H_0(k|x - y|) = sum_m H_m(x - c) conj(J_m(y - c))       (|y - c| < |x - c|)
 *                 = sum_m J_m(x - c) Hb_m(y - c)             (|x - c| < |y - c|),
 * with Hb_m(u) = H_m(k|u|) e^{-i m arg u}, and the gradients
 *   (d_x + i d_y) Z_m = -k Z_{m+1},  (d_x - i d_y) Z_m = k Z_{m-1}.
 * Coefficients are scaled by rscale^|m| (multipoles divided, locals multiplied).
 */

/* J_0..J_N by Miller's backward recurrence (normalized with J_0 + 2 sum J_2k = 1),
 * Y_0, Y_1 from the C library and Y_{n+1} = (2n/x) Y_n - Y_{n-1}: the same published
 * algorithms the device code uses, so the comparison tests the FMM, not two
 * different Bessel implementations. */
static void h2_bessel(int N, double x, double* Jv, double* Yv, int needY)
{
  double xinv = 1.0 / x;
  int nmax = N > (int)x ? N : (int)x;
  int start = 2 * ((nmax + 16 + (int)sqrt(40.0 * nmax)) / 2);
  double fp1 = 0.0, f = 1e-200, sum = 0.0;
  for (int j = 0; j <= N; ++j) Jv[j] = 0.0;
  for (int k = start; k > 0; --k) {
    double fm1 = 2.0 * k * xinv * f - fp1;
    fp1 = f;
    f = fm1;
    if (k - 1 <= N) Jv[k - 1] = f;
    if (((k - 1) & 1) == 0 && k - 1 > 0) sum += 2.0 * f;
    if (fabs(f) > 1e200) {
      f *= 1e-200;
      fp1 *= 1e-200;
      sum *= 1e-200;
      for (int j = k - 1; j <= N; ++j) Jv[j] *= 1e-200;
    }
  }
  sum += f;
  for (int j = 0; j <= N; ++j) Jv[j] /= sum;
  if (needY) {
    Yv[0] = y0(x);
    if (N >= 1) Yv[1] = y1(x);
    for (int j = 1; j < N; ++j) Yv[j + 1] = 2.0 * j * xinv * Yv[j] - Yv[j - 1];
  }
}

static void h2_zfun(int N, double k, double ux, double uy, cplx* J, cplx* H, int needH)
{
  double r = sqrt(ux * ux + uy * uy);
  double th = atan2(uy, ux);
  double x = k * r;
  double Jv[160], Yv[160];
  h2_bessel(N, x, Jv, Yv, needH);
  for (int m = 0; m <= N; ++m) {
    double jm = Jv[m];
    double ym = needH ? Yv[m] : 0.0;
    cplx e = cexp(I * m * th);
    double sg = (m & 1) ? -1.0 : 1.0;
    J[N + m] = jm * e;
    J[N - m] = sg * jm * conj(e);
    if (needH) {
      H[N + m] = (jm + I * ym) * e;
      H[N - m] = sg * (jm + I * ym) * conj(e);
    }
  }
}

static double ipow(double x, int n)
{
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

typedef struct {
  int pf, pq, nrhs, ncf, ncq;
  double k;
  cplx cq, cd;
} h2ctx_t;

static int h2_ctx(const qbxfmm_kernel* kern, h2ctx_t* c)
{
  if (kern->dim != 2) return QBXFMM_ERR_UNSUPPORTED;
  if (kern->k_im != 0.0) return QBXFMM_ERR_UNSUPPORTED;
  c->pf = kern->fmm_order;
  c->pq = kern->qbx_order;
  c->nrhs = kern->nrhs;
  c->ncf = 2 * c->pf + 1;
  c->ncq = 2 * c->pq + 1;
  c->k = kern->k_re;
  c->cq = kern->charge_coeff_re + I * kern->charge_coeff_im;
  c->cd = kern->dipole_coeff_re + I * kern->dipole_coeff_im;
  return 0;
}

/* P2M / P2L accumulation of one source into expansion E (order p, rscale rho) */
static void h2_p2e(const h2ctx_t* c, int p, double rho, const double* ctr, const double* y,
                   cplx q, cplx sigma, const double* nv, cplx* E, int local, cplx* J, cplx* H)
{
  int N = p + 1;
  h2_zfun(N, c->k, y[0] - ctr[0], y[1] - ctr[1], J, H, local);
  cplx nu = nv[0] + I * nv[1];
  for (int m = -p; m <= p; ++m) {
    cplx v;
    if (!local) {
      /* conj(J_m(u)) and its source-normal derivative */
      v = q * conj(J[N + m]);
      if (sigma != 0)
        v += sigma * 0.5 * c->k * (conj(nu) * conj(J[N + m - 1]) - nu * conj(J[N + m + 1]));
      E[m + p] += v / ipow(rho, abs(m));
    } else {
      /* Hb_m(u) = (-1)^m H_{-m}(u) */
#define HB(mm) ((((mm) & 1) ? -1.0 : 1.0) * H[N - (mm)])
      v = q * HB(m);
      if (sigma != 0) v += sigma * 0.5 * c->k * (conj(nu) * HB(m - 1) - nu * HB(m + 1));
#undef HB
      E[m + p] += v * ipow(rho, abs(m));
    }
  }
}

static int h2_form_multipoles(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                              const cplx* strengths, cplx* mpoles)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx J[2 * 64 + 3], H[2 * 64 + 3];
#pragma omp for schedule(dynamic, 4)
    for (int isb = 0; isb < g->nsource_boxes; ++isb) {
      int b = g->source_boxes[isb];
      double rho = level_width(g, g->box_levels[b]);
      double ctr[2], y[2], nv[2] = {0, 0};
      load(g->box_centers, g->nboxes, b, 2, ctr);
      int s0 = g->box_source_starts[b], s1 = s0 + g->box_source_counts_nonchild[b];
      for (int r = 0; r < c.nrhs; ++r) {
        cplx* M = mpoles + ((size_t)b * c.nrhs + r) * c.ncf;
        for (int s = s0; s < s1; ++s) {
          load(g->sources, g->nsources, s, 2, y);
          if (c.cd != 0) load(g->source_normals, g->nsources, s, 2, nv);
          cplx st = strengths[(size_t)r * g->nsources + s];
          h2_p2e(&c, c.pf, rho, ctr, y, c.cq * st, c.cd * st, nv, M, 0, J, H);
        }
      }
    }
  }
  return 0;
}

/* generic translation E_out[m] += f_out(m) sum_n E_in[n] f_in(n) Z_{n-m}(d) */
static void h2_translate(int pin, int pout, const cplx* Ein, cplx* Eout, const cplx* Z, int NZ,
                         double s_in, int in_div, double s_out, int out_div)
{
  for (int m = -pout; m <= pout; ++m) {
    cplx acc = 0;
    for (int n = -pin; n <= pin; ++n) {
      double fin = in_div ? 1.0 / ipow(s_in, abs(n)) : ipow(s_in, abs(n));
      acc += Ein[n + pin] * fin * Z[NZ + n - m];
    }
    double fout = out_div ? 1.0 / ipow(s_out, abs(m)) : ipow(s_out, abs(m));
    Eout[m + pout] += fout * acc;
  }
}

static int h2_coarsen_multipoles(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                                 cplx* mpoles)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
  for (int lev = g->nlevels - 2; lev >= 0; --lev) {
    int i0 = g->level_start_source_parent_box_nrs[lev];
    int i1 = g->level_start_source_parent_box_nrs[lev + 1];
#pragma omp parallel
    {
      cplx J[4 * 64 + 3], H[4 * 64 + 3];
#pragma omp for schedule(dynamic, 1)
      for (int i = i0; i < i1; ++i) {
        int b = g->source_parent_boxes[i];
        double rho_p = level_width(g, lev), rho_c = level_width(g, lev + 1);
        double cp[2], cc[2];
        load(g->box_centers, g->nboxes, b, 2, cp);
        for (int ci = 0; ci < 4; ++ci) {
          int ch = g->box_child_ids[(size_t)ci * g->nboxes + b];
          if (ch == 0 || g->box_source_counts_cumul[ch] == 0) continue;
          load(g->box_centers, g->nboxes, ch, 2, cc);
          /* M'_m = sum_n M_n J_{n-m}(c' - c) */
          h2_zfun(2 * c.pf, c.k, cp[0] - cc[0], cp[1] - cc[1], J, H, 0);
          for (int r = 0; r < c.nrhs; ++r)
            h2_translate(c.pf, c.pf, mpoles + ((size_t)ch * c.nrhs + r) * c.ncf,
                         mpoles + ((size_t)b * c.nrhs + r) * c.ncf, J, 2 * c.pf, rho_c, 0,
                         rho_p, 1);
        }
      }
    }
  }
  return 0;
}

static cplx h2_p2p(double k, const double* x, const double* y, cplx q, cplx sigma,
                   const double* nv)
{
  double d0 = x[0] - y[0], d1 = x[1] - y[1];
  double r = sqrt(d0 * d0 + d1 * d1);
  if (r == 0) return 0;
  cplx v = q * (j0(k * r) + I * y0(k * r));
  if (sigma != 0) v += sigma * k * (j1(k * r) + I * y1(k * r)) * (nv[0] * d0 + nv[1] * d1) / r;
  return v;
}

static int h2_eval_direct(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                          const cplx* strengths, cplx* pot)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel for schedule(dynamic, 1)
  for (int itb = 0; itb < g->ntarget_boxes; ++itb) {
    int tb = g->target_boxes[itb];
    int t0 = g->nonqbx_box_target_starts[tb];
    int t1 = t0 + g->nonqbx_box_target_counts_nonchild[tb];
    for (int t = t0; t < t1; ++t) {
      double x[2], y[2], nv[2] = {0, 0};
      load(g->nonqbx_targets, g->nfiltered_targets, t, 2, x);
      for (int r = 0; r < c.nrhs; ++r) {
        cplx acc = 0;
        for (int li = g->list1_starts[itb]; li < g->list1_starts[itb + 1]; ++li) {
          int sb = g->list1_lists[li];
          int s0 = g->box_source_starts[sb], s1 = s0 + g->box_source_counts_nonchild[sb];
          for (int s = s0; s < s1; ++s) {
            load(g->sources, g->nsources, s, 2, y);
            if (c.cd != 0) load(g->source_normals, g->nsources, s, 2, nv);
            cplx st = strengths[(size_t)r * g->nsources + s];
            acc += h2_p2p(c.k, x, y, c.cq * st, c.cd * st, nv);
          }
        }
        pot[(size_t)r * g->nfiltered_targets + t] += acc;
      }
    }
  }
  return 0;
}

static int h2_multipole_to_local(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                                 const cplx* mpoles, cplx* locals)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx J[4 * 64 + 3], H[4 * 64 + 3];
#pragma omp for schedule(dynamic, 1)
    for (int i = 0; i < g->nttp_boxes; ++i) {
      int tb = g->target_or_target_parent_boxes[i];
      double rho = level_width(g, g->box_levels[tb]);
      double ct[2], cs[2];
      load(g->box_centers, g->nboxes, tb, 2, ct);
      for (int li = g->list2_starts[i]; li < g->list2_starts[i + 1]; ++li) {
        int sb = g->list2_lists[li];
        load(g->box_centers, g->nboxes, sb, 2, cs);
        /* L_m = sum_n M_n H_{n-m}(c' - c) */
        h2_zfun(2 * c.pf, c.k, ct[0] - cs[0], ct[1] - cs[1], J, H, 1);
        for (int r = 0; r < c.nrhs; ++r)
          h2_translate(c.pf, c.pf, mpoles + ((size_t)sb * c.nrhs + r) * c.ncf,
                       locals + ((size_t)tb * c.nrhs + r) * c.ncf, H, 2 * c.pf, rho, 0, rho, 0);
      }
    }
  }
  return 0;
}

static cplx h2_m2p(const h2ctx_t* c, int p, double rho, const double* ctr, const double* x,
                   const cplx* M, cplx* J, cplx* H)
{
  h2_zfun(p, c->k, x[0] - ctr[0], x[1] - ctr[1], J, H, 1);
  cplx acc = 0;
  for (int m = -p; m <= p; ++m) acc += M[m + p] * ipow(rho, abs(m)) * H[p + m];
  return acc;
}

static cplx h2_l2p(const h2ctx_t* c, int p, double rho, const double* ctr, const double* x,
                   const cplx* L, cplx* J, cplx* H)
{
  h2_zfun(p, c->k, x[0] - ctr[0], x[1] - ctr[1], J, H, 0);
  cplx acc = 0;
  for (int m = -p; m <= p; ++m) acc += L[m + p] / ipow(rho, abs(m)) * J[p + m];
  return acc;
}

static int h2_eval_multipoles(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                              const cplx* mpoles, cplx* pot)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx J[2 * 64 + 3], H[2 * 64 + 3];
#pragma omp for schedule(dynamic, 1)
    for (int itb = 0; itb < g->ntarget_boxes; ++itb) {
      int tb = g->target_boxes[itb];
      int t0 = g->nonqbx_box_target_starts[tb];
      int t1 = t0 + g->nonqbx_box_target_counts_nonchild[tb];
      for (int t = t0; t < t1; ++t) {
        double x[2], cs[2];
        load(g->nonqbx_targets, g->nfiltered_targets, t, 2, x);
        for (int li = g->list3_starts[itb]; li < g->list3_starts[itb + 1]; ++li) {
          int sb = g->list3_lists[li];
          double rho = level_width(g, g->box_levels[sb]);
          load(g->box_centers, g->nboxes, sb, 2, cs);
          for (int r = 0; r < c.nrhs; ++r)
            pot[(size_t)r * g->nfiltered_targets + t] +=
                h2_m2p(&c, c.pf, rho, cs, x, mpoles + ((size_t)sb * c.nrhs + r) * c.ncf, J, H);
        }
      }
    }
  }
  return 0;
}

static int h2_form_locals(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                          const cplx* strengths, cplx* locals)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx J[2 * 64 + 3], H[2 * 64 + 3];
#pragma omp for schedule(dynamic, 1)
    for (int i = 0; i < g->nttp_boxes; ++i) {
      int tb = g->target_or_target_parent_boxes[i];
      double rho = level_width(g, g->box_levels[tb]);
      double ct[2], y[2], nv[2] = {0, 0};
      load(g->box_centers, g->nboxes, tb, 2, ct);
      for (int li = g->list4_starts[i]; li < g->list4_starts[i + 1]; ++li) {
        int sb = g->list4_lists[li];
        int s0 = g->box_source_starts[sb], s1 = s0 + g->box_source_counts_nonchild[sb];
        for (int s = s0; s < s1; ++s) {
          load(g->sources, g->nsources, s, 2, y);
          if (c.cd != 0) load(g->source_normals, g->nsources, s, 2, nv);
          for (int r = 0; r < c.nrhs; ++r) {
            cplx st = strengths[(size_t)r * g->nsources + s];
            h2_p2e(&c, c.pf, rho, ct, y, c.cq * st, c.cd * st, nv,
                   locals + ((size_t)tb * c.nrhs + r) * c.ncf, 1, J, H);
          }
        }
      }
    }
  }
  return 0;
}

static int h2_refine_locals(const qbxfmm_kernel* kern, const qbxfmm_geometry* g, cplx* locals)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
  for (int lev = 1; lev < g->nlevels; ++lev) {
    int i0 = g->level_start_ttp_box_nrs[lev], i1 = g->level_start_ttp_box_nrs[lev + 1];
#pragma omp parallel
    {
      cplx J[4 * 64 + 3], H[4 * 64 + 3];
#pragma omp for schedule(dynamic, 4)
      for (int i = i0; i < i1; ++i) {
        int b = g->target_or_target_parent_boxes[i];
        int par = g->box_parent_ids[b];
        double rho_p = level_width(g, lev - 1), rho_c = level_width(g, lev);
        double cp[2], cc[2];
        load(g->box_centers, g->nboxes, par, 2, cp);
        load(g->box_centers, g->nboxes, b, 2, cc);
        /* L''_m = sum_n L_n J_{n-m}(c'' - c) */
        h2_zfun(2 * c.pf, c.k, cc[0] - cp[0], cc[1] - cp[1], J, H, 0);
        for (int r = 0; r < c.nrhs; ++r)
          h2_translate(c.pf, c.pf, locals + ((size_t)par * c.nrhs + r) * c.ncf,
                       locals + ((size_t)b * c.nrhs + r) * c.ncf, J, 2 * c.pf, rho_p, 1, rho_c,
                       0);
      }
    }
  }
  return 0;
}

static int h2_eval_locals(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                          const cplx* locals, cplx* pot)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx J[2 * 64 + 3], H[2 * 64 + 3];
#pragma omp for schedule(dynamic, 4)
    for (int itb = 0; itb < g->ntarget_boxes; ++itb) {
      int tb = g->target_boxes[itb];
      int t0 = g->nonqbx_box_target_starts[tb];
      int t1 = t0 + g->nonqbx_box_target_counts_nonchild[tb];
      double rho = level_width(g, g->box_levels[tb]);
      double ct[2], x[2];
      load(g->box_centers, g->nboxes, tb, 2, ct);
      for (int t = t0; t < t1; ++t) {
        load(g->nonqbx_targets, g->nfiltered_targets, t, 2, x);
        for (int r = 0; r < c.nrhs; ++r)
          pot[(size_t)r * g->nfiltered_targets + t] +=
              h2_l2p(&c, c.pf, rho, ct, x, locals + ((size_t)tb * c.nrhs + r) * c.ncf, J, H);
      }
    }
  }
  return 0;
}

static int h2_p2qbxl(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                     const cplx* strengths, cplx* qbx_exps, int all_sources)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx J[2 * 64 + 3], H[2 * 64 + 3];
#pragma omp for schedule(dynamic, 16)
    for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
      int ctr = g->global_qbx_centers[ig];
      double cc[2], y[2], nv[2] = {0, 0};
      load(g->centers, g->ncenters, ctr, 2, cc);
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
          load(g->sources, g->nsources, s, 2, y);
          if (c.cd != 0) load(g->source_normals, g->nsources, s, 2, nv);
          for (int r = 0; r < c.nrhs; ++r) {
            cplx st = strengths[(size_t)r * g->nsources + s];
            h2_p2e(&c, c.pq, rho, cc, y, c.cq * st, c.cd * st, nv,
                   qbx_exps + ((size_t)ctr * c.nrhs + r) * c.ncq, 1, J, H);
          }
        }
      }
    }
  }
  return 0;
}

static int h2_m2qbxl(const qbxfmm_kernel* kern, const qbxfmm_geometry* g, const cplx* mpoles,
                     cplx* qbx_exps)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx J[4 * 64 + 3], H[4 * 64 + 3];
#pragma omp for schedule(dynamic, 16)
    for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
      int ctr = g->global_qbx_centers[ig];
      double cc[2], cs[2];
      load(g->centers, g->ncenters, ctr, 2, cc);
      double rho_t = g->expansion_radii[ctr];
      int itb = g->qbx_center_to_target_box[ctr];
      for (int li = g->list3_starts[itb]; li < g->list3_starts[itb + 1]; ++li) {
        int sb = g->list3_lists[li];
        double rho_s = level_width(g, g->box_levels[sb]);
        load(g->box_centers, g->nboxes, sb, 2, cs);
        int NZ = c.pf + c.pq;
        h2_zfun(NZ, c.k, cc[0] - cs[0], cc[1] - cs[1], J, H, 1);
        for (int r = 0; r < c.nrhs; ++r)
          h2_translate(c.pf, c.pq, mpoles + ((size_t)sb * c.nrhs + r) * c.ncf,
                       qbx_exps + ((size_t)ctr * c.nrhs + r) * c.ncq, H, NZ, rho_s, 0, rho_t, 0);
      }
    }
  }
  return 0;
}

static int h2_l2qbxl(const qbxfmm_kernel* kern, const qbxfmm_geometry* g, const cplx* locals,
                     cplx* qbx_exps)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx J[4 * 64 + 3], H[4 * 64 + 3];
#pragma omp for schedule(dynamic, 16)
    for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
      int ctr = g->global_qbx_centers[ig];
      int tb = g->target_boxes[g->qbx_center_to_target_box[ctr]];
      double cc[2], cb[2];
      load(g->centers, g->ncenters, ctr, 2, cc);
      load(g->box_centers, g->nboxes, tb, 2, cb);
      double rho_b = level_width(g, g->box_levels[tb]);
      double rho_c = g->expansion_radii[ctr];
      int NZ = c.pf + c.pq;
      h2_zfun(NZ, c.k, cc[0] - cb[0], cc[1] - cb[1], J, H, 0);
      for (int r = 0; r < c.nrhs; ++r)
        h2_translate(c.pf, c.pq, locals + ((size_t)tb * c.nrhs + r) * c.ncf,
                     qbx_exps + ((size_t)ctr * c.nrhs + r) * c.ncq, J, NZ, rho_b, 1, rho_c, 0);
    }
  }
  return 0;
}

static int h2_eval_qbx_expansions(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                                  const cplx* qbx_exps, cplx* pot_tree)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
#pragma omp parallel
  {
    cplx J[2 * 64 + 3], H[2 * 64 + 3];
#pragma omp for schedule(dynamic, 16)
    for (int ig = 0; ig < g->nglobal_qbx_centers; ++ig) {
      int ctr = g->global_qbx_centers[ig];
      double cc[2], x[2];
      load(g->centers, g->ncenters, ctr, 2, cc);
      double rho = g->expansion_radii[ctr];
      for (int it = g->center_to_targets_starts[ctr]; it < g->center_to_targets_starts[ctr + 1];
           ++it) {
        int t = g->center_to_targets_lists[it];
        load(g->targets, g->ntargets, t, 2, x);
        for (int r = 0; r < c.nrhs; ++r)
          pot_tree[(size_t)r * g->ntargets + t] =
              h2_l2p(&c, c.pq, rho, cc, x, qbx_exps + ((size_t)ctr * c.nrhs + r) * c.ncq, J, H);
      }
    }
  }
  return 0;
}

static int h2_assemble(const qbxfmm_kernel* kern, const qbxfmm_geometry* g,
                       const cplx* pot_nonqbx, const cplx* pot_tree, cplx* out)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
  cplx scale = 0.25 * I;
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

static int h2_apply(const qbxfmm_kernel* kern, const qbxfmm_geometry* g, const cplx* strengths,
                    cplx* out, int direct)
{
  h2ctx_t c;
  int rc = h2_ctx(kern, &c);
  if (rc) return rc;
  size_t nexp = (size_t)g->nboxes * c.nrhs * c.ncf;
  cplx* mpoles = calloc(nexp, sizeof(cplx));
  cplx* locals = calloc(nexp, sizeof(cplx));
  cplx* qexp = calloc((size_t)g->ncenters * c.nrhs * c.ncq, sizeof(cplx));
  cplx* pnq = calloc((size_t)c.nrhs * g->nfiltered_targets + 1, sizeof(cplx));
  cplx* ptree = calloc((size_t)c.nrhs * g->ntargets + 1, sizeof(cplx));
  if (!direct) {
    h2_form_multipoles(kern, g, strengths, mpoles);
    h2_coarsen_multipoles(kern, g, mpoles);
    h2_eval_direct(kern, g, strengths, pnq);
    h2_multipole_to_local(kern, g, mpoles, locals);
    h2_eval_multipoles(kern, g, mpoles, pnq);
    h2_form_locals(kern, g, strengths, locals);
    h2_refine_locals(kern, g, locals);
    h2_eval_locals(kern, g, locals, pnq);
    h2_p2qbxl(kern, g, strengths, qexp, 0);
    h2_m2qbxl(kern, g, mpoles, qexp);
    h2_l2qbxl(kern, g, locals, qexp);
  } else {
    h2_p2qbxl(kern, g, strengths, qexp, 1);
#pragma omp parallel for schedule(dynamic, 16)
    for (int t = 0; t < g->nfiltered_targets; ++t) {
      double x[2], y[2], nv[2] = {0, 0};
      load(g->nonqbx_targets, g->nfiltered_targets, t, 2, x);
      for (int r = 0; r < c.nrhs; ++r) {
        cplx acc = 0;
        for (int s = 0; s < g->nsources; ++s) {
          load(g->sources, g->nsources, s, 2, y);
          if (c.cd != 0) load(g->source_normals, g->nsources, s, 2, nv);
          cplx st = strengths[(size_t)r * g->nsources + s];
          acc += h2_p2p(c.k, x, y, c.cq * st, c.cd * st, nv);
        }
        pnq[(size_t)r * g->nfiltered_targets + t] = acc;
      }
    }
  }
  h2_eval_qbx_expansions(kern, g, qexp, ptree);
  h2_assemble(kern, g, pnq, ptree, out);
  free(mpoles);
  free(locals);
  free(qexp);
  free(pnq);
  free(ptree);
  return 0;
}
