// 3D Helmholtz QBX-FMM stage kernels, complex128, sm_100a.
//
// Kernel G(x, y) = e^{ik|x-y|} / |x-y| (k real), scaled by 1/(4 pi) at assembly.
// Spherical-wave expansions (the basis of pytential's fmmlib backend,
// pytential/qbx/fmmlib.py, and of its target-specific module,
// pytential/qbx/target_specific/impl.pyx:363-563):
//   Y_n^m = p_n^|m|(cos t) sin^|m| t e^{i m phi} (orthonormal, no Condon-Shortley phase),
//   R_n^m(v) = j_n(k|v|) Y_n^m(v),  S_n^m(v) = h_n(k|v|) Y_n^m(v),
//   multipole about c: sum M_nm S_n^m(x - c), M_nm = 4 pi i k q R_n^-m(y - c) / s^n,
//   local about c:     sum L_nm R_n^m(x - c), L_nm = 4 pi i k q S_n^-m(y - c) s^n,
// with s = min(1, k rho) (rho = box width or expansion radius) and coefficient index
// n^2 + n + m.  Translations use the addition theorem
//   F_n^m(r + b) = sum c_{nu mu; n m}(b) R_nu^mu(r),
//   c_{nu mu; n m}(b) = 4 pi sum_l i^{nu + l - n} f_l(k|b|) Y_l^{m - mu}(b) G(n,m; nu,mu; l)
// (G: Gaunt integrals, a host-computed table, layout [(nu,mu)][j][(n,m)]), applied as per-level, per-class
// complex matrices on the FP64 tensor cores for M2M / M2L / L2L and directly for the
// point-to-box translations into QBX centers.  Source-normal derivatives use the
// ladder relations of R and S.
#include <cooperative_groups.h>

#include <algorithm>
#include <string>
#include <type_traits>

#include "../../include/qbxfmm_api.h"
#include "laplace.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace qbx {

namespace {

constexpr int NT = 128;
constexpr int NW = NT / 32;
constexpr int MAXB = 128;
constexpr int H3_LMAX = 44;        // largest order of a radial / harmonic table
constexpr int H3_MAXP = 17;        // largest FMM order
constexpr double FOUR_PI = 12.566370614359172953850573533118;

QBX_HD int hq(int n, int m) { return n * n + n + m; }

QBX_HD void hq_decode(int c, int& n, int& m)
{
  n = (int)sqrt((double)c);
  while ((n + 1) * (n + 1) <= c) ++n;
  while (n * n > c) --n;
  m = c - n * n - n;
}

// Recurrence table for the normalized associated Legendre polynomial parts, n <= N:
// rec[idx3(n, m)] = (p_m^m, 0) at n = m, (sqrt(2m + 3), 0) at n = m + 1, else
// (a_nm, b_nm) with p_n^m = a_nm (t p_{n-1}^m - b_nm p_{n-2}^m).
QBX_D void h3_rec_table(int N, double2* rec, int tid, int nt)
{
  int tot = (N + 1) * (N + 2) / 2;
  for (int e = tid; e < tot; e += nt) {
    int n, m;
    decode3(e, n, m);
    double a, b = 0.0;
    if (n == m) {
      a = 0.28209479177387814347;   // 1 / sqrt(4 pi)
      for (int i = 1; i <= m; ++i) a *= sqrt((2.0 * i + 1.0) / (2.0 * i));
    } else if (n == m + 1) {
      a = sqrt(2.0 * m + 3.0);
    } else {
      a = sqrt((4.0 * n * n - 1.0) / ((double)n * n - (double)m * m));
      b = sqrt(((n - 1.0) * (n - 1.0) - (double)m * m) / (4.0 * (n - 1.0) * (n - 1.0) - 1.0));
    }
    rec[e] = c2(a, b);
  }
}

// t = cos(theta), w = sin(theta) e^{i phi} of v (v = 0: t = 1, w = 0)
QBX_D double h3_dir(const double* v, double2& w, double& r)
{
  r = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if (r == 0.0) {
    w = c2(0.0);
    return 1.0;
  }
  double ri = 1.0 / r;
  w = c2(v[0] * ri, v[1] * ri);
  return v[2] * ri;
}

// j_n(x), n <= N, by Miller's backward recurrence normalized with j_0 or j_1
QBX_D void h3_sph_j(int N, double x, double* jv)
{
  for (int n = 0; n <= N; ++n) jv[n] = 0.0;
  if (x == 0.0) {
    jv[0] = 1.0;
    return;
  }
  int nmax = max(N, (int)x);
  int start = nmax + 16 + (int)sqrt(40.0 * (nmax + 1));
  double xi = 1.0 / x;
  double fp1 = 0.0, f = 1e-200, f1 = 0.0;
  for (int n = start; n >= 1; --n) {
    double fm1 = (2.0 * n + 1.0) * xi * f - fp1;
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
  double s, c;
  sincos(x, &s, &c);
  double scale = (x < 1.0 || fabs(s) >= 0.5) ? (s * xi) / f : ((s * xi - c) * xi) / f1;
  for (int n = 0; n <= N; ++n) jv[n] *= scale;
}

// j_n^[T](x) = sum_{j: n + 2j <= T} (-x^2/2)^j x^n / (j! (2n+2j+1)!!), n <= N: the
// power series of j_n cut at total degree T (zero for n > T); T < 0: j_n itself.  The
// degree-T Taylor polynomial of sum L_nm j_n(k|v|) Y_n^m(v) is sum L_nm j_n^[T] Y_n^m.
QBX_D void h3_sph_j_cut(int N, double x, int T, double* jv)
{
  if (T < 0) {
    h3_sph_j(N, x, jv);
    return;
  }
  double xn = 1.0, dfac = 1.0, mx2 = -0.5 * x * x;
  for (int n = 0; n <= N; ++n) {
    if (n > 0) {
      xn *= x;
      dfac *= 2.0 * n + 1.0;
    }
    double term = xn / dfac, acc = 0.0;
    for (int j = 0; n + 2 * j <= T; ++j) {
      acc += term;
      term *= mx2 * rcp(j + 1) * rcp(2 * n + 2 * j + 3);
    }
    jv[n] = acc;
  }
}

// h_n(x) = j_n(x) + i y_n(x), n <= N, by the upward recurrence
QBX_D void h3_sph_h(int N, double x, double2* hv)
{
  double s, c;
  sincos(x, &s, &c);
  double xi = 1.0 / x;
  hv[0] = c2(s * xi, -c * xi);
  if (N >= 1) hv[1] = c2((s - c * x) * xi * xi, -(s * x + c) * xi * xi);
  for (int n = 1; n < N; ++n) {
    double f = (2.0 * n + 1.0) * xi;
    hv[n + 1] = c2(f * hv[n].x - hv[n - 1].x, f * hv[n].y - hv[n - 1].y);
  }
}

// Ladder terms of nu . grad F_n^mm (mm = -m for the source coefficient (n, m)):
// six table entries with real weights (0 where the entry is outside the table).
// Order: z-, z+ (times nu_z), p+, p- (times (nu_x - i nu_y) / 2), m+, m- (times
// (nu_x + i nu_y) / 2); entry offsets are hq() indices.
struct Ladder {
  int o[6];
  double w[6];
};

QBX_HD Ladder h3_ladder(int n, int mm, double k)
{
  Ladder L;
  for (int i = 0; i < 6; ++i) {
    L.o[i] = 0;
    L.w[i] = 0.0;
  }
  double an = sqrt((double)(n + 1 - mm) * (n + 1 + mm) / ((2.0 * n + 1) * (2.0 * n + 3)));
  if (n >= 1 && abs(mm) <= n - 1) {
    L.o[0] = hq(n - 1, mm);
    L.w[0] = k * sqrt((double)(n - mm) * (n + mm) / ((2.0 * n - 1) * (2.0 * n + 1)));
  }
  L.o[1] = hq(n + 1, mm);
  L.w[1] = -k * an;
  double sgp = mm >= 0 ? 1.0 : -1.0, sgm = -mm >= 0 ? 1.0 : -1.0;
  L.o[2] = hq(n + 1, mm + 1);
  L.w[2] = -k * sgp * sqrt((double)(n + mm + 1) * (n + mm + 2) / ((2.0 * n + 1) * (2.0 * n + 3)));
  if (n >= 1 && abs(mm + 1) <= n - 1) {
    L.o[3] = hq(n - 1, mm + 1);
    L.w[3] = -k * sgp * sqrt((double)(n - mm) * (n - mm - 1) / ((2.0 * n - 1) * (2.0 * n + 1)));
  }
  L.o[4] = hq(n + 1, mm - 1);
  L.w[4] = -k * sgm * sqrt((double)(n - mm + 1) * (n - mm + 2) / ((2.0 * n + 1) * (2.0 * n + 3)));
  if (n >= 1 && abs(mm - 1) <= n - 1) {
    L.o[5] = hq(n - 1, mm - 1);
    L.w[5] = -k * sgm * sqrt((double)(n + mm) * (n + mm - 1) / ((2.0 * n - 1) * (2.0 * n + 1)));
  }
  return L;
}

// Fill column m (n = m..N) of a wave table: T[hq(n, +-m) * ts] = f_n Y_n^{+-m}
// (f = radial values, complex), given t, w and the recurrence table.
QBX_D void h3_wave_column(int m, int N, double t, double2 w, const double2* rec, const double2* rad,
                          double2* T, int ts)
{
  double2 wm = c2(1.0);
  for (int i = 0; i < m; ++i) wm = cmul(wm, w);
  double pm1 = rec[idx3(m, m)].x, pm2 = 0.0;
  for (int n = m; n <= N; ++n) {
    double pn;
    if (n == m) {
      pn = pm1;
    } else if (n == m + 1) {
      pn = rec[idx3(n, m)].x * t * pm1;
      pm2 = pm1;
      pm1 = pn;
    } else {
      double2 ab = rec[idx3(n, m)];
      pn = ab.x * (t * pm1 - ab.y * pm2);
      pm2 = pm1;
      pm1 = pn;
    }
    double2 y = cscale(pn, wm);
    T[hq(n, m) * ts] = cmul(rad[n], y);
    if (m > 0) T[hq(n, -m) * ts] = cmul(rad[n], cconj(y));
  }
}

QBX_D double h3_scale(double k, double rho) { return fmin(1.0, k * rho); }

// i^e for integer e
QBX_D double2 ipow(int e)
{
  switch (e & 3) {
    case 0: return c2(1.0, 0.0);
    case 1: return c2(0.0, 1.0);
    case 2: return c2(-1.0, 0.0);
    default: return c2(0.0, -1.0);
  }
}

// list helpers (as in the Laplace kernels)
QBX_D void h3_list_prefix(const qbxfmm_geometry& g, const int32_t* __restrict__ lists, int gb,
                          int nb, int* s_pref, int* s_start, int32_t* err)
{
  if (threadIdx.x >= 32) return;
  int lane = threadIdx.x;
  int cnt[4], loc = 0;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    int k = lane * 4 + u;
    cnt[u] = 0;
    if (k < nb) {
      int sb = lists[gb + k];
      int s0 = 0;
      if ((unsigned)sb < (unsigned)g.nboxes) {
        s0 = g.box_source_starts[sb];
        cnt[u] = g.box_source_counts_nonchild[sb];
      } else {
        report(err, QBX_DEVERR_BAD_BOX);
      }
      s_start[k] = s0;
    }
    loc += cnt[u];
  }
  int incl = loc;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    int v = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += v;
  }
  int run = incl - loc;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    int k = lane * 4 + u;
    if (k < nb) s_pref[k] = run;
    run += cnt[u];
  }
  if (lane == 31) s_pref[nb] = incl;
}

QBX_D int h3_stream_source(int v, int nb, const int* s_pref, const int* s_start)
{
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (s_pref[mid] <= v) lo = mid;
    else hi = mid - 1;
  }
  return s_start[lo] + (v - s_pref[lo]);
}

}  // namespace

// {{{ P2M / P2L

// One CTA per box (P2M: source boxes, own sources; P2L: target-or-parent boxes, list-4
// sources) and group of RB densities.  Sources in sub-tiles of SUB: one thread per
// source computes the radial values (j_n for P2M, h_n for P2L, n <= p + 1), one thread
// per (column, source) fills the wave table (entry-major, padded stride), then one
// thread per coefficient forms the source's kernel row cq F_n^-m + cd nu . grad F_n^-m
// (precomputed ladder offsets) once and adds density x row for each of the RB
// densities, so the table and the row serve all densities of the group.
constexpr int H3_SUB = 16;
constexpr int H3_TS = H3_SUB + 1;
constexpr int H3_NH = 3;          // coefficients per thread: (p+1)^2 <= 3 * 128

// TH threads per CTA, NH coefficients per thread ((p+1)^2 <= NH x TH): 128 x 3 with up
// to 8 densities, or 256 x 1 with 16 (the wave tables of a source serve all 16)
template <bool LOCAL, int RB, int TH = NT, int NH = H3_NH>
__global__ void __launch_bounds__(TH, TH == NT ? 1 : 2)
k_h3_p2e(qbxfmm_geometry g, HelmCoeffs hc, int p, int nrhs, const double2* __restrict__ strengths,
         double2* __restrict__ exps, int32_t* err)
{
  constexpr int SUB = H3_SUB, TS = H3_TS;
  extern __shared__ double2 smem2[];
  const int N = p + 1;
  const int ncf = (p + 1) * (p + 1);
  double2* tab = smem2;                              // [(N+1)^2][TS]
  double2* rec = smem2 + (size_t)(N + 1) * (N + 1) * TS;   // [(N+1)(N+2)/2]
  __shared__ double2 s_rad[SUB][H3_LMAX + 2];
  __shared__ double s_t[SUB];
  __shared__ double2 s_w[SUB], s_sig[SUB][RB], s_np[SUB], s_nm[SUB];
  __shared__ double s_nz[SUB];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];

  int b, l0 = 0, l1 = 0;
  if (LOCAL) {
    int i = blockIdx.x;
    b = g.target_or_target_parent_boxes[i];
    l0 = g.list4_starts[i];
    l1 = g.list4_starts[i + 1];
    if (l1 <= l0) return;
  } else {
    b = g.source_boxes[blockIdx.x];
  }
  int r0 = blockIdx.y * RB;
  double rho = level_width(g, g.box_levels[b]);
  double sc = h3_scale(hc.k, rho);
  double c[3];
  load_point<3>(g.box_centers, g.nboxes, b, c);
  const bool dip = hc.cd.x != 0.0 || hc.cd.y != 0.0;
  // the reference's default multipoles (moments of degree <= p): the charge row from
  // j_n^[p], the normal derivative from j_n^[p-1] (a second table)
  const bool two = !LOCAL && hc.taylor && dip;
  double2* tab2 = two ? rec + (size_t)(N + 1) * (N + 2) / 2 : tab;   // [(N+1)^2][TS]
  double2* rad2 = two ? tab2 + (size_t)(N + 1) * (N + 1) * TS : nullptr;   // [SUB][N+2]
  h3_rec_table(N, rec, threadIdx.x, TH);

  int o_c[NH];
  Ladder lad[NH];
  bool valid[NH];
#pragma unroll
  for (int h = 0; h < NH; ++h) {
    int ci = threadIdx.x + h * TH;
    valid[h] = ci < ncf;
    int n = 0, m = 0;
    if (valid[h]) hq_decode(ci, n, m);
    o_c[h] = hq(n, -m) * TS;
    lad[h] = h3_ladder(n, -m, hc.k);
#pragma unroll
    for (int u = 0; u < 6; ++u) lad[h].o[u] *= TS;
  }
  double2 acc[NH][RB];
#pragma unroll
  for (int h = 0; h < NH; ++h)
#pragma unroll
    for (int rr = 0; rr < RB; ++rr) acc[h][rr] = c2(0.0);

  // one stream over the box's own sources (P2M) or the list-4 boxes' sources (P2L)
  for (int gb = l0; gb < (LOCAL ? l1 : 1); gb += MAXB) {
    int nb = 0, total;
    __syncthreads();
    if (LOCAL) {
      nb = min(MAXB, l1 - gb);
      h3_list_prefix(g, g.list4_lists, gb, nb, s_pref, s_start, err);
      __syncthreads();
      total = s_pref[nb];
    } else {
      total = g.box_source_counts_nonchild[b];
    }
    int s0 = LOCAL ? 0 : g.box_source_starts[b];
    for (int base = 0; base < total; base += SUB) {
      int cnt = min(SUB, total - base);
      __syncthreads();
      if (threadIdx.x < cnt) {
        int j = threadIdx.x;
        int s = LOCAL ? h3_stream_source(base + j, nb, s_pref, s_start) : s0 + base + j;
        double y[3], u[3], rr;
        load_point<3>(g.sources, g.nsources, s, y);
#pragma unroll
        for (int d = 0; d < 3; ++d) u[d] = y[d] - c[d];
        double2 w;
        s_t[j] = h3_dir(u, w, rr);
        s_w[j] = w;
        double x = hc.k * rr;
        if (LOCAL) {
          h3_sph_h(N, x, s_rad[j]);
        } else {
          double jv[H3_LMAX + 2];
          h3_sph_j_cut(N, x, hc.taylor ? p : -1, jv);
          for (int n = 0; n <= N; ++n) s_rad[j][n] = c2(jv[n]);
          if (two) {
            h3_sph_j_cut(N, x, p - 1, jv);
            for (int n = 0; n <= N; ++n) rad2[j * (N + 2) + n] = c2(jv[n]);
          }
        }
#pragma unroll
        for (int rr = 0; rr < RB; ++rr)
          s_sig[j][rr] = r0 + rr < nrhs ? strengths[(size_t)(r0 + rr) * g.nsources + s] : c2(0.0);
        if (dip) {
          double nv[3];
          load_point<3>(g.source_normals, g.nsources, s, nv);
          s_np[j] = c2(0.5 * nv[0], -0.5 * nv[1]);
          s_nm[j] = c2(0.5 * nv[0], 0.5 * nv[1]);
          s_nz[j] = nv[2];
        }
      }
      __syncthreads();
      for (int wk = threadIdx.x; wk < cnt * (N + 1); wk += TH) {
        int m = wk / cnt, j = wk - m * cnt;
        h3_wave_column(m, N, s_t[j], s_w[j], rec, s_rad[j], tab + j, TS);
        if (two) h3_wave_column(m, N, s_t[j], s_w[j], rec, rad2 + j * (N + 2), tab2 + j, TS);
      }
      __syncthreads();
#pragma unroll
      for (int h = 0; h < NH; ++h) {
        if (!valid[h]) continue;
        for (int j = 0; j < cnt; ++j) {
          const double2* T = tab + j;
          double2 kr = cmul(hc.cq, T[o_c[h]]);
          if (dip) {
            T = tab2 + j;
            const Ladder& L = lad[h];
            double2 vz = caxpy(L.w[0], T[L.o[0]], cscale(L.w[1], T[L.o[1]]));
            double2 vp = caxpy(L.w[2], T[L.o[2]], cscale(L.w[3], T[L.o[3]]));
            double2 vm = caxpy(L.w[4], T[L.o[4]], cscale(L.w[5], T[L.o[5]]));
            double2 v = cfma(s_np[j], vp, cfma(s_nm[j], vm, cscale(s_nz[j], vz)));
            kr = cfma(hc.cd, v, kr);
          }
#pragma unroll
          for (int rr = 0; rr < RB; ++rr) acc[h][rr] = cfma(s_sig[j][rr], kr, acc[h][rr]);
        }
      }
    }
  }
#pragma unroll
  for (int h = 0; h < NH; ++h) {
    if (!valid[h]) continue;
    int ci = threadIdx.x + h * TH;
    int n, m;
    hq_decode(ci, n, m);
    double f = FOUR_PI * hc.k * (LOCAL ? pow(sc, (double)n) : pow(sc, -(double)n));
#pragma unroll
    for (int rr = 0; rr < RB; ++rr) {
      if (r0 + rr >= nrhs) break;
      // 4 pi i k f acc
      double2* E = exps + ((size_t)b * nrhs + r0 + rr) * ncf + ci;
      *E = cadd(*E, c2(-f * acc[h][rr].y, f * acc[h][rr].x));
    }
  }
}

// }}}

// {{{ point evaluations at non-QBX targets

constexpr int H3_PSPLIT = 8;

QBX_D double2 h3_cluster_lane_sum(double2 acc, double2 (*s_red)[32], double2* s_part)
{
  cg::cluster_group cl = cg::this_cluster();
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (warp > 0) s_red[warp - 1][lane] = acc;
  __syncthreads();
  if (warp == 0) {
    for (int w = 1; w < NW; ++w) acc = cadd(acc, s_red[w - 1][lane]);
    s_part[lane] = acc;
  }
  cl.sync();
  if (cl.block_rank() == 0 && warp == 0) {
    for (unsigned q = 1; q < cl.num_blocks(); ++q) acc = cadd(acc, *cl.map_shared_rank(s_part + lane, q));
  }
  cl.sync();
  return acc;
}

// P2P over list 1: a cluster of H3_PSPLIT CTAs per chunk of <= 32 non-QBX targets,
// source tiles dealt round-robin to the CTAs, fixed-order reduction over DSMEM.
__global__ void __cluster_dims__(H3_PSPLIT, 1, 1) __launch_bounds__(NT)
k_h3_eval_direct(qbxfmm_geometry g, HelmCoeffs hc, int nrhs, const double2* __restrict__ strengths,
                 double2* __restrict__ pot, int32_t* err)
{
  __shared__ double s_y[3][NT], s_n[3][NT];
  __shared__ double2 s_q[NT], s_d[NT];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];
  __shared__ double2 s_red[NW - 1][32];
  __shared__ double2 s_part[32];
  int chunk = blockIdx.x / H3_PSPLIT;
  int part = blockIdx.x - chunk * H3_PSPLIT;
  int r = blockIdx.y;
  int itb = g.nonqbx_chunk_target_box[chunk];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bool active = lane < g.nonqbx_chunk_count[chunk];
  int t = g.nonqbx_chunk_start[chunk] + lane;
  double x[3] = {0, 0, 0};
  if (active) load_point<3>(g.nonqbx_targets, g.nfiltered_targets, t, x);
  const double2* st = strengths + (size_t)r * g.nsources;
  const bool dip = hc.cd.x != 0.0 || hc.cd.y != 0.0;
  double2 acc = c2(0.0);
  int l0 = g.list1_starts[itb], l1 = g.list1_starts[itb + 1];
  int tile = 0;
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    h3_list_prefix(g, g.list1_lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += NT, ++tile) {
      if (tile % H3_PSPLIT != part) continue;
      int v = base + threadIdx.x;
      if (v < total) {
        int s = h3_stream_source(v, nb, s_pref, s_start);
        double y[3], nv[3] = {0, 0, 0};
        load_point<3>(g.sources, g.nsources, s, y);
        if (dip) load_point<3>(g.source_normals, g.nsources, s, nv);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          s_y[d][threadIdx.x] = y[d];
          s_n[d][threadIdx.x] = nv[d];
        }
        double2 sv = st[s];
        s_q[threadIdx.x] = cmul(hc.cq, sv);
        s_d[threadIdx.x] = cmul(hc.cd, sv);
      }
      __syncthreads();
      int jbeg = warp * 32, jend = min(jbeg + 32, total - base);
      if (active) {
        for (int j = jbeg; j < jend; ++j) {
          double dx = x[0] - s_y[0][j], dy = x[1] - s_y[1][j], dz = x[2] - s_y[2][j];
          double r2 = dx * dx + dy * dy + dz * dz;
          if (r2 == 0.0) continue;
          double rinv = rsqrt(r2);
          double rr = r2 * rinv;
          double sn, cs;
          sincos(hc.k * rr, &sn, &cs);
          double2 e = c2(cs * rinv, sn * rinv);   // e^{ikr} / r
          acc = cfma(s_q[j], e, acc);
          if (dip) {
            // n . (x - y) e^{ikr} (1 - ikr) / r^3
            double f = (s_n[0][j] * dx + s_n[1][j] * dy + s_n[2][j] * dz) * rinv * rinv;
            double2 v = cmul(e, c2(f, -f * hc.k * rr));
            acc = cfma(s_d[j], v, acc);
          }
        }
      }
      __syncthreads();
    }
  }
  acc = h3_cluster_lane_sum(acc, s_red, s_part);
  if (part == 0 && warp == 0 && active) {
    double2* P = pot + (size_t)r * g.nfiltered_targets + t;
    *P = cadd(*P, acc);
  }
}

// Evaluate an expansion (order p, scale s) of box b at point x: multipole (singular
// waves, coefficient * s^n) or local (regular waves, coefficient / s^n).
// (local: jcut >= 0 cuts j_n at total degree jcut, the reference's default truncation)
QBX_D double2 h3_e2p(const double2* E, int p, bool local, double k, double s, const double* cb,
                     const double* x, const double2* rec, int jcut = -1)
{
  double u[3] = {x[0] - cb[0], x[1] - cb[1], x[2] - cb[2]};
  double2 w;
  double rr;
  double t = h3_dir(u, w, rr);
  double2 rad[H3_LMAX + 2];
  if (local) {
    double jv[H3_LMAX + 2];
    h3_sph_j_cut(p, k * rr, jcut, jv);
    double f = 1.0, si = 1.0 / s;
    for (int n = 0; n <= p; ++n, f *= si) rad[n] = c2(jv[n] * f);
  } else {
    h3_sph_h(p, k * rr, rad);
    double f = 1.0;
    for (int n = 0; n <= p; ++n, f *= s) rad[n] = cscale(f, rad[n]);
  }
  double2 acc = c2(0.0);
  double2 wm = c2(1.0);
  for (int m = 0; m <= p; ++m) {
    if (m > 0) wm = cmul(wm, w);
    double pm1 = rec[idx3(m, m)].x, pm2 = 0.0;
    for (int n = m; n <= p; ++n) {
      double pn;
      if (n == m) {
        pn = pm1;
      } else if (n == m + 1) {
        pn = rec[idx3(n, m)].x * t * pm1;
        pm2 = pm1;
        pm1 = pn;
      } else {
        double2 ab = rec[idx3(n, m)];
        pn = ab.x * (t * pm1 - ab.y * pm2);
        pm2 = pm1;
        pm1 = pn;
      }
      double2 y = cscale(pn, wm);
      double2 v = cmul(E[hq(n, m)], y);
      if (m > 0) v = cadd(v, cmul(E[hq(n, -m)], cconj(y)));
      acc = cfma(rad[n], v, acc);
    }
  }
  return acc;
}

// M2P over list 3: CTA per chunk of <= 32 non-QBX targets (lane = target), the warps
// split the list-3 boxes and stage each multipole in their own shared slice.
__global__ void __launch_bounds__(NT)
k_h3_eval_multipoles(qbxfmm_geometry g, HelmCoeffs hc, int p, int nrhs,
                     const double2* __restrict__ mpoles, double2* __restrict__ pot, int32_t* err)
{
  extern __shared__ double2 smem2[];
  const int ncf = (p + 1) * (p + 1);
  double2* rec = smem2;                                  // [(p+1)(p+2)/2]
  int nrec = (p + 1) * (p + 2) / 2;
  __shared__ double2 s_red[NW - 1][32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double2* M = smem2 + nrec + (size_t)warp * ncf;
  h3_rec_table(p, rec, threadIdx.x, NT);
  __syncthreads();
  int chunk = blockIdx.x;
  int r = blockIdx.y;
  int itb = g.nonqbx_chunk_target_box[chunk];
  int t = g.nonqbx_chunk_start[chunk] + lane;
  bool active = lane < g.nonqbx_chunk_count[chunk];
  double x[3] = {0, 0, 0};
  if (active) load_point<3>(g.nonqbx_targets, g.nfiltered_targets, t, x);
  double2 acc = c2(0.0);
  for (int li = g.list3_starts[itb] + warp; li < g.list3_starts[itb + 1]; li += NW) {
    int sb = g.list3_lists[li];
    if ((unsigned)sb >= (unsigned)g.nboxes) {
      report(err, QBX_DEVERR_BAD_BOX);
      continue;
    }
    __syncwarp();
    const double2* src = mpoles + ((size_t)sb * nrhs + r) * ncf;
    for (int q = lane; q < ncf; q += 32) M[q] = src[q];
    __syncwarp();
    if (!active) continue;
    double cs[3];
    load_point<3>(g.box_centers, g.nboxes, sb, cs);
    double s = h3_scale(hc.k, level_width(g, g.box_levels[sb]));
    acc = cadd(acc, h3_e2p(M, p, false, hc.k, s, cs, x, rec));
  }
  __syncthreads();
  if (warp > 0) s_red[warp - 1][lane] = acc;
  __syncthreads();
  if (warp == 0 && active) {
    for (int w = 1; w < NW; ++w) acc = cadd(acc, s_red[w - 1][lane]);
    double2* P = pot + (size_t)r * g.nfiltered_targets + t;
    *P = cadd(*P, acc);
  }
}

// L2P: one thread per non-QBX target, its own box's local expansion
__global__ void __launch_bounds__(NT)
k_h3_eval_locals(qbxfmm_geometry g, HelmCoeffs hc, int p, int nrhs,
                 const double2* __restrict__ locals, double2* __restrict__ pot)
{
  extern __shared__ double2 smem2[];
  double2* rec = smem2;
  h3_rec_table(p, rec, threadIdx.x, NT);
  __syncthreads();
  int chunk = blockIdx.x;
  int r = blockIdx.y;
  int lane = threadIdx.x;
  if (lane >= 32 || lane >= g.nonqbx_chunk_count[chunk]) return;
  int itb = g.nonqbx_chunk_target_box[chunk];
  int tb = g.target_boxes[itb];
  int t = g.nonqbx_chunk_start[chunk] + lane;
  double x[3], cb[3];
  load_point<3>(g.nonqbx_targets, g.nfiltered_targets, t, x);
  load_point<3>(g.box_centers, g.nboxes, tb, cb);
  double s = h3_scale(hc.k, level_width(g, g.box_levels[tb]));
  const int ncf = (p + 1) * (p + 1);
  double2 v = h3_e2p(locals + ((size_t)tb * nrhs + r) * ncf, p, true, hc.k, s, cb, x, rec,
                     hc.taylor ? p : -1);
  double2* P = pot + (size_t)r * g.nfiltered_targets + t;
  *P = cadd(*P, v);
}

// }}}

// {{{ QBX: P2QBXL, M2QBXL / L2QBXL, QBXL2P

// P2QBXL over list 1: CTA per chunk of <= 32 centers of one target box (lane =
// center, coefficients in registers); the list-1 sources stream through shared memory
// in tiles of 128, each warp taking 32; per (center, source) pair the lane builds its
// singular-wave table (order Q + 1) in its own column of a lane-minor shared array.
template <int Q>
__global__ void __launch_bounds__(NT)
k_h3_p2qbxl(qbxfmm_geometry g, HelmCoeffs hc, int nrhs, const double2* __restrict__ strengths,
            double2* __restrict__ qbx_exps, int32_t* err)
{
  constexpr int N = Q + 1;
  constexpr int NE = (N + 1) * (N + 1);    // wave-table entries
  constexpr int NC = (Q + 1) * (Q + 1);
  extern __shared__ double2 smem2[];
  double2* tabs = smem2;                          // [NW][NE][32]
  __shared__ double2 rec[(N + 1) * (N + 2) / 2];
  __shared__ Ladder s_lad[NC];
  __shared__ double s_y[3][NT], s_n[3][NT];
  __shared__ double2 s_q[NT], s_d[NT];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];
  h3_rec_table(N, rec, threadIdx.x, NT);
  for (int ci = threadIdx.x; ci < NC; ci += NT) {
    int n, m;
    hq_decode(ci, n, m);
    s_lad[ci] = h3_ladder(n, -m, hc.k);
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double2* T = tabs + (size_t)warp * NE * 32 + lane;
  int chunk = blockIdx.x;
  int r = blockIdx.y;
  int itb = g.qbx_chunk_target_box[chunk];
  bool has_center = lane < g.qbx_chunk_count[chunk];
  int ctr = has_center ? g.centers_by_target_box[g.qbx_chunk_start[chunk] + lane] : 0;
  if ((unsigned)ctr >= (unsigned)g.ncenters) {
    report(err, QBX_DEVERR_BAD_CENTER);
    has_center = false;
    ctr = 0;
  }
  double cc[3];
  load_point<3>(g.centers, g.ncenters, ctr, cc);
  const double2* st = strengths + (size_t)r * g.nsources;
  const bool dip = hc.cd.x != 0.0 || hc.cd.y != 0.0;
  double2 acc[NC];
#pragma unroll
  for (int i = 0; i < NC; ++i) acc[i] = c2(0.0);
  int l0 = g.list1_starts[itb], l1 = g.list1_starts[itb + 1];
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    h3_list_prefix(g, g.list1_lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += NT) {
      int v = base + threadIdx.x;
      if (v < total) {
        int s = h3_stream_source(v, nb, s_pref, s_start);
        double y[3], nv[3] = {0, 0, 0};
        load_point<3>(g.sources, g.nsources, s, y);
        if (dip) load_point<3>(g.source_normals, g.nsources, s, nv);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          s_y[d][threadIdx.x] = y[d];
          s_n[d][threadIdx.x] = nv[d];
        }
        double2 sv = st[s];
        s_q[threadIdx.x] = cmul(hc.cq, sv);
        s_d[threadIdx.x] = cmul(hc.cd, sv);
      }
      __syncthreads();
      int jbeg = warp * 32, jend = min(jbeg + 32, total - base);
      if (has_center) {
        for (int j = jbeg; j < jend; ++j) {
          double u[3] = {s_y[0][j] - cc[0], s_y[1][j] - cc[1], s_y[2][j] - cc[2]};
          double2 w;
          double rr;
          double t = h3_dir(u, w, rr);
          if (rr == 0.0) continue;
          double2 rad[N + 1];
          h3_sph_h(N, hc.k * rr, rad);
#pragma unroll
          for (int m = 0; m <= N; ++m) h3_wave_column(m, N, t, w, rec, rad, T, 32);
          double2 q = s_q[j];
#pragma unroll
          for (int n = 0; n <= Q; ++n)
#pragma unroll
            for (int m = -n; m <= n; ++m) acc[hq(n, m)] = cfma(q, T[hq(n, -m) * 32], acc[hq(n, m)]);
          if (dip) {
            double2 np = c2(0.5 * s_n[0][j], -0.5 * s_n[1][j]);
            double2 nm = c2(0.5 * s_n[0][j], 0.5 * s_n[1][j]);
            double nz = s_n[2][j];
            double2 d = s_d[j];
#pragma unroll
            for (int ci = 0; ci < NC; ++ci) {
              const Ladder& L = s_lad[ci];
              double2 vz = caxpy(L.w[0], T[L.o[0] * 32], cscale(L.w[1], T[L.o[1] * 32]));
              double2 vp = caxpy(L.w[2], T[L.o[2] * 32], cscale(L.w[3], T[L.o[3] * 32]));
              double2 vm = caxpy(L.w[4], T[L.o[4] * 32], cscale(L.w[5], T[L.o[5] * 32]));
              double2 vv = cfma(np, vp, cfma(nm, vm, cscale(nz, vz)));
              acc[ci] = cfma(d, vv, acc[ci]);
            }
          }
        }
      }
      __syncthreads();
    }
  }
  // reduce the warps' partial sums through the (now free) table space
  __syncthreads();
  double2* red = tabs;   // [NW-1][32][NC]
  if (warp > 0) {
#pragma unroll
    for (int i = 0; i < NC; ++i) red[((warp - 1) * 32 + lane) * NC + i] = acc[i];
  }
  __syncthreads();
  if (warp == 0 && has_center) {
    double s = h3_scale(hc.k, g.expansion_radii[ctr]);
    double2* out = qbx_exps + ((size_t)ctr * nrhs + r) * NC;
    double fs = FOUR_PI * hc.k;
#pragma unroll
    for (int i = 0; i < NC; ++i) {
      double2 a = acc[i];
      for (int w = 1; w < NW; ++w) a = cadd(a, red[((w - 1) * 32 + lane) * NC + i]);
      int n, m;
      hq_decode(i, n, m);
      double f = fs * pow(s, (double)n);
      out[i] = cadd(out[i], c2(-f * a.y, f * a.x));
    }
  }
}

// M2QBXL (list-3 multipoles) and L2QBXL (own box's local) into the QBX local of order
// Q at a center, by rotation: rotate the frame so that the translation vector b lies
// on the z axis, translate coaxially, rotate back,
//   c(b) = R_back(-beta, alpha) . coax(|b|) . R(beta, alpha),
// with, for the orthonormal harmonics without the Condon-Shortley phase,
//   rotated coefficients  M'_{n mu} = sum_m e^{i m alpha} eps_m eps_mu d^n_{m mu}(beta) M_{n m},
//   coaxial coefficients  c^mu_{nu n} = 4 pi sum_l i^{nu + l - n} f_l(k|b|) Y_l^0(z) G(n,mu; nu,mu; l),
//   back rotation         L_{nu mu''} = e^{-i mu'' alpha} sum_mu eps_mu eps_mu'' d^nu_{mu mu''}(-beta) L'_{nu mu},
// (d: Wigner's small-d matrices, eps_m = (-1)^m for m > 0, else 1; beta, alpha the
// polar and azimuthal angles of b).  Equal in exact arithmetic to the Gaunt sum
// c_{nu mu; n m}(b) of the file comment; only |mu| <= Q of the rotated source
// coefficients are needed, so the work per (center, box) pair is O(pf^2 Q) per
// density instead of O(pf^2 Q^2).
// The pass runs over the source order n: d^n_{m mu} for fixed (m, mu >= 0) follows
// the three-term recurrence in n (Jacobi polynomials),
//   n s_{n+1} d^{n+1} = (2n+1)(n(n+1) cos(beta) - m mu) d^n - (n+1) s_n d^{n-1},
//   s_n = sqrt((n^2 - m^2)(n^2 - mu^2)),
// started at n0 = max(|m|, mu) from the single surviving term of Wigner's formula;
// each lane advances its (m, mu) recurrences in registers, the slice of order n
// (with d^n_{m,-mu} = (-1)^{m+mu} d^n_{-m,mu} and the phases) goes through shared
// memory to the lanes that rotate and translate, and the coaxial coefficients of
// order n are formed on the fly, so no table of all orders is stored.  The slices of
// orders n <= Q are also the back-rotation matrices (d^nu_{mu mu''}(-beta) =
// d^nu_{mu'' mu}(beta)).
// One warp per center (H3_ROT_ZS CTAs x 4 warps per chunk of <= 32 centers), RB
// densities per CTA staged in shared memory per box; lane tasks are (m, mu)
// recurrences, (mu, density) for the rotation + coaxial step and (output, density)
// for the back rotation, whose results stay in registers across the boxes.
// D (8x8, two per lane: row lane/4, columns 2 (lane%4) + {0,1}) += A (8x4, row major,
// element (lane/4, lane%4)) B (4x8, column major, element (lane%4, lane/4)), FP64
QBX_D void h3_dmma(double& d0, double& d1, double a, double b)
{
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

constexpr int H3_ROT_ZS = 8;
constexpr int H3_ROT_SLOTS = 7;   // recurrence tasks per lane: (2 pf + 1)(Q + 1) <= 7 x 32

template <typename R, bool FROM_LOCAL, int Q, int RB>
__global__ void __launch_bounds__(NT)
k_h3_e2qbxl_rot(qbxfmm_geometry g, HelmCoeffs hc, int pf, int nrhs,
                const double2* __restrict__ exps, const double* __restrict__ rot,
                double2* __restrict__ qbx_exps, int32_t* err)
{
  // R: the arithmetic (double, or float in the mixed-precision form; expansions are
  // read and added in float64 either way)
  using V = cplx_t<R>;
  constexpr bool F64 = std::is_same<R, double>::value;
  constexpr int NCQ = (Q + 1) * (Q + 1);
  constexpr int NMU = 2 * Q + 1;
  constexpr int NOUT = (NCQ * RB + 31) / 32;
  constexpr int TPL = (NMU * RB + 31) / 32;
  constexpr int RSL = H3_ROT_SLOTS;
  extern __shared__ double2 smem2[];
  const int ncf = (pf + 1) * (pf + 1);
  const int L = pf + Q;
  const int nl = pf + 1;
  const int nm = 2 * pf + 1;
  const int ntask = nm * (Q + 1);
  const int nisq = (pf + 2) * (pf + 1), nrt = (pf + 1) * (pf + 1);
  const double* rstart = rot;                                   // [nm][Q+1][4]
  const double* g_isq = rstart + (size_t)nm * (Q + 1) * 4;      // [pf+2][pf+1]
  const double* g_rt = g_isq + nisq;                            // [pf+1][pf+1]
  const double* g0c = g_rt + nrt;                               // [NCQ][nl][Q+1]
  // CTA-wide
  V* Es = reinterpret_cast<V*>(smem2);                          // [ncf][RB]
  R* s_isq = reinterpret_cast<R*>(Es + (size_t)ncf * RB);
  R* s_rt = s_isq + nisq;
  R* spow = s_rt + nrt;                                         // [nl]: s_box^{+-n}
  const size_t ctad = ((size_t)nisq + nrt + nl + 1) & ~(size_t)1;
  V* wbase = reinterpret_cast<V*>(s_isq + ctad);
  // per warp
  const size_t perd = ((size_t)NMU * NCQ + 2 * (size_t)nm + 1) / 2;
  const size_t per = (size_t)nm * NMU + NCQ + (size_t)NCQ * RB + (L + 2) + nm + perd;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  V* Dph = wbase + (size_t)warp * per;                          // [nm][NMU] slice x phase
  V* coaxn = Dph + (size_t)nm * NMU;                            // [NCQ] coaxial column n
  V* Lp = coaxn + NCQ;                                          // [NCQ][RB]
  V* rad = Lp + (size_t)NCQ * RB;                               // [L + 2]
  V* ph = rad + (L + 2);                                        // [nm]: e^{i m alpha}
  R* Tb = reinterpret_cast<R*>(ph + nm);                        // [NMU][NCQ]
  R* chp = Tb + (size_t)NMU * NCQ;                              // [nm] cos(beta/2)^k
  R* shp = chp + nm;                                            // [nm] sin(beta/2)^k

  __shared__ unsigned char s_nof[(H3_MAXP + 1) * (H3_MAXP + 1)];   // order n of coefficient (n, m)
  for (int x = threadIdx.x; x < nisq + nrt; x += NT) s_isq[x] = (R)__ldg(g_isq + x);
  for (int n = 0; n <= pf; ++n)
    for (int x = n * n + threadIdx.x; x < (n + 1) * (n + 1); x += NT) s_nof[x] = (unsigned char)n;
  __syncthreads();
  int chunk = blockIdx.x;
  int r0 = blockIdx.y * RB;
  int itb = g.qbx_chunk_target_box[chunk];
  int nctr = g.qbx_chunk_count[chunk];
  if (blockIdx.z * NW >= nctr) return;     // the whole CTA is idle
  int ci = blockIdx.z * NW + warp;
  bool has = ci < nctr;
  int ctr = has ? g.centers_by_target_box[g.qbx_chunk_start[chunk] + ci] : 0;
  if ((unsigned)ctr >= (unsigned)g.ncenters) {
    report(err, QBX_DEVERR_BAD_CENTER);
    has = false;
    ctr = 0;
  }
  double cc[3];
  load_point<3>(g.centers, g.ncenters, ctr, cc);
  V acc[NOUT];
#pragma unroll
  for (int i = 0; i < NOUT; ++i) acc[i] = cmake<R>(0);

  int nbox = FROM_LOCAL ? 1 : g.list3_starts[itb + 1] - g.list3_starts[itb];
  for (int bi = 0; bi < nbox; ++bi) {
    int sbx = FROM_LOCAL ? g.target_boxes[itb] : g.list3_lists[g.list3_starts[itb] + bi];
    if ((unsigned)sbx >= (unsigned)g.nboxes) {
      report(err, QBX_DEVERR_BAD_BOX);
      continue;
    }
    double cb[3];
    load_point<3>(g.box_centers, g.nboxes, sbx, cb);
    double sb = h3_scale(hc.k, level_width(g, g.box_levels[sbx]));
    __syncthreads();
    if (threadIdx.x == 0) {
      double f = 1.0, fs = FROM_LOCAL ? 1.0 / sb : sb;
      for (int n = 0; n < nl; ++n, f *= fs) spow[n] = (R)f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < ncf * RB; e += NT) {
      int ei = e / RB, ri = e - ei * RB;
      int n = s_nof[ei];
      V v = cmake<R>(0);
      if (r0 + ri < nrhs) v = cscale(spow[n], cto(exps[((size_t)sbx * nrhs + r0 + ri) * ncf + ei], V()));
      Es[e] = v;
    }
    __syncthreads();
    if (!has) continue;
    // translation vector and its angles
    double bv[3] = {cc[0] - cb[0], cc[1] - cb[1], cc[2] - cb[2]};
    double bl = sqrt(bv[0] * bv[0] + bv[1] * bv[1] + bv[2] * bv[2]);
    double cbeta = bl > 0.0 ? fmin(1.0, fmax(-1.0, bv[2] / bl)) : 1.0;
    double alpha = (bv[0] == 0.0 && bv[1] == 0.0) ? 0.0 : atan2(bv[1], bv[0]);
    double beta = acos(cbeta);
    double ch = cos(0.5 * beta), sh = sin(0.5 * beta);
    if (lane == 0) {
      if (FROM_LOCAL) {
        double jv[H3_LMAX + 2];
        h3_sph_j(L, hc.k * bl, jv);
        for (int l = 0; l <= L; ++l) rad[l] = cmake<R>((R)jv[l]);
      } else if constexpr (F64) {
        h3_sph_h(L, hc.k * bl, reinterpret_cast<double2*>(rad));
      } else {
        double2 hv[H3_LMAX + 2];
        h3_sph_h(L, hc.k * bl, hv);
        for (int l = 0; l <= L; ++l) rad[l] = cto(hv[l], V());
      }
    }
    for (int m = lane; m < nm; m += 32) {
      double sn, cs;
      sincos((m - pf) * alpha, &sn, &cs);
      ph[m] = cmake<R>((R)cs, (R)sn);
      double a = 1.0, b = 1.0;
      for (int u = 0; u < m; ++u) {
        a *= ch;
        b *= sh;
      }
      chp[m] = (R)a;
      shp[m] = (R)b;
    }
    __syncwarp();
    // 4 pi Y_l^0(z) i^l f_l, Y_l^0(z) = sqrt((2l+1)/(4 pi)), one lane per order
    for (int l = lane; l <= L; l += 32)
      rad[l] = cmul(cto(cscale(sqrt(FOUR_PI * (2.0 * l + 1.0)), ipow(l)), V()), rad[l]);
    __syncwarp();
    // recurrence tasks t = (m + pf) (Q + 1) + mu, mu >= 0: start values
    R cur[RSL], prev[RSL], v0[RSL];
    int n0[RSL];
#pragma unroll
    for (int sl = 0; sl < RSL; ++sl) {
      int t = lane + 32 * sl;
      cur[sl] = prev[sl] = v0[sl] = R(0);
      n0[sl] = 1 << 20;
      if (t < ntask) {
        int m = t / (Q + 1) - pf, mu = t % (Q + 1);
        n0[sl] = max(abs(m), mu);
        v0[sl] = (R)__ldg(rstart + 4 * t) * chp[(int)__ldg(rstart + 4 * t + 1)] *
                 shp[(int)__ldg(rstart + 4 * t + 2)];
      }
    }
    // per-lane (mu, density) slots of the coaxially translated coefficients: the TPL
    // lane tasks, or with 8 densities the 4 entries of the tensor-core output tiles
    // this lane holds
    constexpr bool DMMA = F64 && RB == 8;
    constexpr int LSL = DMMA ? 4 : TPL;
    V lacc[LSL][Q + 1];
#pragma unroll
    for (int ts = 0; ts < LSL; ++ts)
#pragma unroll
      for (int nu = 0; nu <= Q; ++nu) lacc[ts][nu] = cmake<R>(0);

    for (int n = 0; n <= pf; ++n) {
      // (1) the slice of order n, written by the recurrence lanes themselves: the
      // task (m, mu >= 0) holds d = d^n_{m mu} and stores the signed, phased entries
      // (m, mu) and, with d^n_{-m,-mu} = (-1)^{m+mu} d^n_{m mu}, (-m, -mu); orders
      // n <= Q also give the back-rotation matrices (without the phase).  Rows
      // |m| > n are not read at this order (tasks below their start order hold 0,
      // which zero-fills the columns |mu| > n); then the step to n + 1
      const R rn = n > 0 ? R(1) / R(n) : R(0);
      const R h1 = (R)((2.0 * n + 1.0) * n * (n + 1.0) * cbeta);
      const int tbase = n * n + n;
#pragma unroll
      for (int sl = 0; sl < RSL; ++sl) {
        int t = lane + 32 * sl;
        if (t >= ntask) continue;
        if (n == n0[sl]) cur[sl] = v0[sl];
        {
          const int m = t / (Q + 1) - pf, mu = t - (t / (Q + 1)) * (Q + 1);
          if (abs(m) <= n) {
            const R d = n >= n0[sl] ? cur[sl] : R(0);
            const R v1 = (((m > 0) && (m & 1)) != ((mu & 1) != 0)) ? -d : d;
            Dph[(m + pf) * NMU + mu + Q] = cscale(v1, ph[m + pf]);
            if (n <= Q) Tb[(mu + Q) * NCQ + tbase + m] = v1;
            if (mu > 0) {
              // sign (-1)^{m+mu} eps_{-m}, eps_{-m} = (-1)^m for m < 0
              const bool neg = (((m + mu) & 1) != 0) != ((m < 0) && (m & 1));
              const R v2 = neg ? -d : d;
              Dph[(pf - m) * NMU + Q - mu] = cscale(v2, ph[pf - m]);
              if (n <= Q) Tb[(Q - mu) * NCQ + tbase - m] = v2;
            }
          }
        }
        if (n >= n0[sl] && n < pf) {
          R nxt;
          if (n == 0) {
            nxt = (R)cbeta * cur[sl];
          } else {
            int m = t / (Q + 1) - pf, mu = t % (Q + 1);
            int am = abs(m);
            R w = rn * s_isq[(n + 1) * (pf + 1) + am] * s_isq[(n + 1) * (pf + 1) + mu];
            R A = (h1 - R((2 * n + 1) * m * mu)) * w;
            R C = R(n + 1) * rn * s_rt[n * (pf + 1) + am] * s_rt[n * (pf + 1) + mu];
            nxt = fma(A, cur[sl], -C * prev[sl]);
          }
          prev[sl] = cur[sl];
          cur[sl] = nxt;
        }
      }
      // (2) coaxial column n: coaxn[(nu,mu)] = i^{nu-n} sum_j G(nu,mu; j; n,mu) rad[|n-nu|+2j]
      // for mu >= 0 only (G(n,-mu; nu,-mu; l) = G(n,mu; nu,mu; l): the column of -mu is
      // that of mu), one lane per (nu, mu >= 0), its table reads issued before the sum
      static_assert((Q + 1) * (Q + 2) / 2 <= 32, "one lane per coaxial entry");
      if (lane < (Q + 1) * (Q + 2) / 2) {
        int nu = (int)((sqrtf(8.0f * lane + 1.0f) - 1.0f) * 0.5f);
        if ((nu + 1) * (nu + 2) / 2 <= lane) ++nu;
        if (nu * (nu + 1) / 2 > lane) --nu;
        const int mu = lane - nu * (nu + 1) / 2;
        const int o = nu * nu + nu + mu;
        V tt = cmake<R>(0);
        if (n >= mu) {
          const double* G = g0c + ((size_t)o * nl + n) * (Q + 1);
          int lbase = abs(n - nu), jmax = min(n, nu);
          R gj[Q + 1];
#pragma unroll
          for (int j = 0; j <= Q; ++j) gj[j] = j <= jmax ? (R)__ldg(G + j) : R(0);
#pragma unroll
          for (int j = 0; j <= Q; ++j)
            if (j <= jmax) tt = caxpy(gj[j], rad[lbase + 2 * j], tt);
          tt = cmul(cto(ipow(nu - n + 4 * pf), V()), tt);
        }
        coaxn[o] = tt;
      }
      __syncwarp();
      // (3) rotate and translate coaxially
      const int base = n * n + n;
      if constexpr (DMMA) {
        // the rotation of order n as a real product on the FP64 tensor cores:
        // rows (mu, re / im) of the rotated coefficients, k = (m, re / im), columns the
        // 8 densities; tiles 0/1 hold re/im of mu index 0..7, tiles 2/3 of 8..15,
        // A[(mu, re)][(m, re)] = Re z, [(mu, re)][(m, im)] = -Im z, [(mu, im)][(m, re)] =
        // Im z, [(mu, im)][(m, im)] = Re z with z = Dph[m][mu]; K = 2 (2n+1) padded to 4
        constexpr int NTILE = (NMU > 8) ? 4 : 2;
        const int rho = lane >> 2, kq = lane & 3;
        double c[NTILE][2];
#pragma unroll
        for (int t = 0; t < NTILE; ++t) c[t][0] = c[t][1] = 0.0;
        const double2* Eb = Es + (base - n) * RB + rho;
        const double2* Db = Dph + (pf - n) * NMU;
        for (int sk = 0; sk <= n; ++sk) {
          const int kap = 4 * sk + kq, mi = kap >> 1, pin = kap & 1;
          const bool vk = mi <= 2 * n;
          double2 e = vk ? Eb[mi * RB] : c2(0.0);
          double b = pin ? e.y : e.x;
          double2 z0 = (vk && rho < NMU) ? Db[mi * NMU + rho] : c2(0.0);
          h3_dmma(c[0][0], c[0][1], pin ? -z0.y : z0.x, b);
          h3_dmma(c[1][0], c[1][1], pin ? z0.x : z0.y, b);
          if (NTILE == 4) {
            double2 z1 = (vk && 8 + rho < NMU) ? Db[mi * NMU + 8 + rho] : c2(0.0);
            h3_dmma(c[NTILE - 2][0], c[NTILE - 2][1], pin ? -z1.y : z1.x, b);
            h3_dmma(c[NTILE - 1][0], c[NTILE - 1][1], pin ? z1.x : z1.y, b);
          }
        }
#pragma unroll
        for (int sl = 0; sl < 4; ++sl) {
          const int grp = sl >> 1, v = sl & 1;
          const int mu = (grp ? 8 + rho : rho) - Q;
          if (grp * 8 + rho >= NMU || abs(mu) > n || (grp && NTILE < 4)) continue;
          double2 mr = c2(c[2 * grp][v], c[2 * grp + 1][v]);
          const int amu = abs(mu);
#pragma unroll
          for (int nu = 0; nu <= Q; ++nu)
            if (nu >= amu) lacc[sl][nu] = cfma(coaxn[nu * nu + nu + amu], mr, lacc[sl][nu]);
        }
      } else {
        // lane tasks (mu, density), all of a lane's tasks in one pass over m so that
        // their multiply-adds interleave
        V mr[TPL];
        int toff[TPL], eoff[TPL];
        bool act[TPL];
#pragma unroll
        for (int ts = 0; ts < TPL; ++ts) {
          int task = lane + 32 * ts;
          int mu = task / RB - Q, r = task - (task / RB) * RB;
          act[ts] = task < NMU * RB && abs(mu) <= n;
          toff[ts] = act[ts] ? (pf - n) * NMU + mu + Q : 0;
          eoff[ts] = act[ts] ? (base - n) * RB + r : 0;
          mr[ts] = cmake<R>(0);
        }
        for (int m = 0; m < 2 * n + 1; ++m) {
#pragma unroll
          for (int ts = 0; ts < TPL; ++ts)
            if (act[ts]) mr[ts] = cfma(Dph[toff[ts] + m * NMU], Es[eoff[ts] + m * RB], mr[ts]);
        }
#pragma unroll
        for (int ts = 0; ts < TPL; ++ts) {
          if (!act[ts]) continue;
          int task = lane + 32 * ts;
          int mu = task / RB - Q;
          int amu = abs(mu);
#pragma unroll
          for (int nu = 0; nu <= Q; ++nu)
            if (nu >= amu) lacc[ts][nu] = cfma(coaxn[nu * nu + nu + amu], mr[ts], lacc[ts][nu]);
        }
      }
      __syncwarp();
    }
    if constexpr (DMMA) {
      const int rho = lane >> 2;
#pragma unroll
      for (int sl = 0; sl < 4; ++sl) {
        const int grp = sl >> 1, r = 2 * (lane & 3) + (sl & 1);
        const int mu = (grp ? 8 + rho : rho) - Q;
        if (grp * 8 + rho >= NMU) continue;
#pragma unroll
        for (int nu = 0; nu <= Q; ++nu)
          if (nu >= abs(mu)) Lp[(nu * nu + nu + mu) * RB + r] = lacc[sl][nu];
      }
    } else {
#pragma unroll
      for (int ts = 0; ts < TPL; ++ts) {
        int task = lane + 32 * ts;
        if (task >= NMU * RB) continue;
        int mu = task / RB - Q, r = task - (task / RB) * RB;
#pragma unroll
        for (int nu = 0; nu <= Q; ++nu)
          if (nu >= abs(mu)) Lp[(nu * nu + nu + mu) * RB + r] = lacc[ts][nu];
      }
    }
    __syncwarp();
    // rotate back into the register outputs: lane task (o = (nu, mu2), density)
#pragma unroll
    for (int i = 0; i < NOUT; ++i) {
      int task = lane + 32 * i;
      if (task >= NCQ * RB) break;
      int o = task / RB, r = task - o * RB;
      int nu = s_nof[o];
      int mu2 = o - nu * nu - nu;
      V a = cmake<R>(0);
      for (int mu = -nu; mu <= nu; ++mu) a = caxpy(Tb[(mu + Q) * NCQ + o], Lp[(nu * nu + nu + mu) * RB + r], a);
      acc[i] = cfma(cconj(ph[mu2 + pf]), a, acc[i]);
    }
    __syncwarp();
  }
  if (!has) return;
  double st = h3_scale(hc.k, g.expansion_radii[ctr]);
#pragma unroll
  for (int i = 0; i < NOUT; ++i) {
    int task = lane + 32 * i;
    if (task >= NCQ * RB) break;
    int o = task / RB, r = task - o * RB;
    if (r0 + r >= nrhs) continue;
    int nu = s_nof[o];
    double2* out = qbx_exps + ((size_t)ctr * nrhs + r0 + r) * NCQ + o;
    *out = caxpy(pow(st, (double)nu), c2d(acc[i]), *out);
  }
}

// M2QBXL in FP64 with the per-pair tables shared by 16 densities: the same rotation,
// coaxial translation and back rotation as k_h3_e2qbxl_rot, but two warps per center
// (CTA: 2 centers x 2 warps), each warp applying the tables to 8 of the 16 densities
// on the FP64 tensor cores.  The pair of warps splits the table work of a (center,
// box) pair: the Wigner-d recurrence tasks are interleaved between them (blocks of 32
// tasks), warp 1 forms the coaxial column, warp 0 the radial factors and warp 1 the
// phases; the (real) slice and the column of order n are double-buffered, so one
// named barrier per order (64 threads, one per center) separates writing order n + 1
// from reading order n.  The phases e^{i m alpha} are applied to the source
// coefficients as they enter the tensor-core product, so the rotation is a real
// matrix times the real and imaginary parts: half the products of a complex one.  Shared memory per CTA stays at two CTAs per SM (the box's 16-density
// multipole block is staged once for both centers).
constexpr int H3P_SLOTS = 4;   // recurrence tasks per lane: (2 pf + 1)(Q + 1) <= 2 x 4 x 32

// named barrier of the two warps of center cp (barrier 0 is __syncthreads)
QBX_D void h3_pair_bar(int cp)
{
  if (cp == 0) asm volatile("bar.sync 1, 64;\n" ::: "memory");
  else asm volatile("bar.sync 2, 64;\n" ::: "memory");
}

template <int Q>
__global__ void __launch_bounds__(NT)
k_h3_m2qbxl_pair(qbxfmm_geometry g, HelmCoeffs hc, int pf, int nrhs,
                 const double2* __restrict__ exps, const double* __restrict__ rot,
                 double2* __restrict__ qbx_exps, int32_t* err)
{
  constexpr int NCQ = (Q + 1) * (Q + 1);
  constexpr int NMU = 2 * Q + 1;
  constexpr int RB = 16, HB = 8;                 // densities per CTA / per warp
  constexpr int NOUT = (NCQ * HB + 31) / 32;
  constexpr int RSL = H3P_SLOTS;
  constexpr int NTILE = (NMU > 8) ? 4 : 2;
  extern __shared__ double2 smem2[];
  const int ncf = (pf + 1) * (pf + 1);
  const int L = pf + Q;
  const int nl = pf + 1;
  const int nm = 2 * pf + 1;
  const int ntask = nm * (Q + 1);
  const int nisq = (pf + 2) * (pf + 1), nrt = (pf + 1) * (pf + 1);
  const double* rstart = rot;                                   // [nm][Q+1][4]
  const double* g_isq = rstart + (size_t)nm * (Q + 1) * 4;      // [pf+2][pf+1]
  const double* g_rt = g_isq + nisq;                            // [pf+1][pf+1]
  const double* g0c = g_rt + nrt;                               // [NCQ][nl][Q+1]
  // CTA-wide
  double2* Es = smem2;                                          // [ncf][RB]
  double* s_isq = reinterpret_cast<double*>(Es + (size_t)ncf * RB);
  double* s_rt = s_isq + nisq;
  double* spow = s_rt + nrt;                                    // [nl]: s_box^n
  double2* cbase = reinterpret_cast<double2*>(s_isq + (((size_t)nisq + nrt + nl + 1) & ~(size_t)1));
  // per center: real slices eps_m eps_mu d^n_{m mu} (two buffers of [nm][NMU]; after
  // the order loop the two warps' [NCQ][HB] blocks of translated coefficients),
  // coaxial columns (two buffers), radial factors, phases, back-rotation matrices,
  // half-angle powers
  const size_t nsl = max((size_t)nm * NMU, (size_t)2 * NCQ * HB);
  const size_t per = nsl + 2 * NCQ + (L + 2) + nm + ((size_t)NMU * NCQ + 2 * (size_t)nm + 1) / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int cp = warp >> 1, half = warp & 1;
  double2* Dsl = cbase + (size_t)cp * per;                      // (double) [2][nm][NMU]
  double2* Lp = Dsl + (size_t)half * NCQ * HB;                  // [NCQ][HB] (after the loop)
  double2* coax = Dsl + nsl;                                    // [2][NCQ]
  double2* rad = coax + 2 * NCQ;                                // [L + 2]
  double2* ph = rad + (L + 2);                                  // [nm]: e^{i m alpha}
  double* Tb = reinterpret_cast<double*>(ph + nm);              // [NMU][NCQ]
  double* chp = Tb + (size_t)NMU * NCQ;                         // [nm] cos(beta/2)^k
  double* shp = chp + nm;                                       // [nm] sin(beta/2)^k

  __shared__ unsigned char s_nof[(H3_MAXP + 1) * (H3_MAXP + 1)];
  for (int x = threadIdx.x; x < nisq + nrt; x += NT) s_isq[x] = __ldg(g_isq + x);
  for (int n = 0; n <= pf; ++n)
    for (int x = n * n + threadIdx.x; x < (n + 1) * (n + 1); x += NT) s_nof[x] = (unsigned char)n;
  __syncthreads();
  const int chunk = blockIdx.x;
  const int r0 = blockIdx.y * RB;
  const int itb = g.qbx_chunk_target_box[chunk];
  const int nctr = g.qbx_chunk_count[chunk];
  if (blockIdx.z * 2 >= nctr) return;      // the whole CTA is idle
  const int ci = blockIdx.z * 2 + cp;
  bool has = ci < nctr;                    // the same for both warps of a center
  int ctr = has ? g.centers_by_target_box[g.qbx_chunk_start[chunk] + ci] : 0;
  if ((unsigned)ctr >= (unsigned)g.ncenters) {
    report(err, QBX_DEVERR_BAD_CENTER);
    has = false;
    ctr = 0;
  }
  double cc[3];
  load_point<3>(g.centers, g.ncenters, ctr, cc);
  double2 acc[NOUT];
#pragma unroll
  for (int i = 0; i < NOUT; ++i) acc[i] = c2(0.0);

  const int nbox = g.list3_starts[itb + 1] - g.list3_starts[itb];
  for (int bi = 0; bi < nbox; ++bi) {
    const int sbx = g.list3_lists[g.list3_starts[itb] + bi];
    if ((unsigned)sbx >= (unsigned)g.nboxes) {
      report(err, QBX_DEVERR_BAD_BOX);
      continue;                            // uniform over the CTA: the list is shared
    }
    double cb[3];
    load_point<3>(g.box_centers, g.nboxes, sbx, cb);
    const double sb = h3_scale(hc.k, level_width(g, g.box_levels[sbx]));
    __syncthreads();
    if (threadIdx.x == 0) {
      double f = 1.0;
      for (int n = 0; n < nl; ++n, f *= sb) spow[n] = f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < ncf * RB; e += NT) {
      const int ei = e / RB, ri = e - ei * RB;
      double2 v = c2(0.0);
      if (r0 + ri < nrhs) v = cscale(spow[s_nof[ei]], exps[((size_t)sbx * nrhs + r0 + ri) * ncf + ei]);
      Es[e] = v;
    }
    __syncthreads();
    if (!has) continue;
    const double bv[3] = {cc[0] - cb[0], cc[1] - cb[1], cc[2] - cb[2]};
    const double bl = sqrt(bv[0] * bv[0] + bv[1] * bv[1] + bv[2] * bv[2]);
    const double cbeta = bl > 0.0 ? fmin(1.0, fmax(-1.0, bv[2] / bl)) : 1.0;
    const double alpha = (bv[0] == 0.0 && bv[1] == 0.0) ? 0.0 : atan2(bv[1], bv[0]);
    const double beta = acos(cbeta);
    if (half == 0) {
      // radial factors 4 pi Y_l^0(z) i^l h_l(k |b|), Y_l^0(z) = sqrt((2l+1)/(4 pi))
      if (lane == 0) h3_sph_h(L, hc.k * bl, rad);
      __syncwarp();
      for (int l = lane; l <= L; l += 32)
        rad[l] = cmul(cscale(sqrt(FOUR_PI * (2.0 * l + 1.0)), ipow(l)), rad[l]);
    } else {
      const double ch = cos(0.5 * beta), sh = sin(0.5 * beta);
      for (int m = lane; m < nm; m += 32) {
        double sn, cs;
        sincos((m - pf) * alpha, &sn, &cs);
        ph[m] = c2(cs, sn);
        double a = 1.0, b = 1.0;
        for (int u = 0; u < m; ++u) {
          a *= ch;
          b *= sh;
        }
        chp[m] = a;
        shp[m] = b;
      }
    }
    h3_pair_bar(cp);
    // this warp's recurrence tasks t = (2 sl + half) 32 + lane, t = (m + pf)(Q + 1) + mu
    double cur[RSL], prev[RSL], v0[RSL];
    int n0[RSL];
#pragma unroll
    for (int sl = 0; sl < RSL; ++sl) {
      const int t = (2 * sl + half) * 32 + lane;
      cur[sl] = prev[sl] = v0[sl] = 0.0;
      n0[sl] = 1 << 20;
      if (t < ntask) {
        const int m = t / (Q + 1) - pf, mu = t % (Q + 1);
        n0[sl] = max(abs(m), mu);
        v0[sl] = __ldg(rstart + 4 * t) * chp[(int)__ldg(rstart + 4 * t + 1)] *
                 shp[(int)__ldg(rstart + 4 * t + 2)];
      }
    }
    double2 lacc[4][Q + 1];
#pragma unroll
    for (int ts = 0; ts < 4; ++ts)
#pragma unroll
      for (int nu = 0; nu <= Q; ++nu) lacc[ts][nu] = c2(0.0);

    for (int n = 0; n <= pf; ++n) {
      double* Dre = reinterpret_cast<double*>(Dsl) + (size_t)(n & 1) * nm * NMU;
      double2* coaxn = coax + (n & 1) * NCQ;
      // (1) slice of order n from this warp's recurrence tasks (as in k_h3_e2qbxl_rot)
      const double rn = n > 0 ? 1.0 / n : 0.0;
      const double h1 = (2.0 * n + 1.0) * n * (n + 1.0) * cbeta;
      const int tbase = n * n + n;
#pragma unroll
      for (int sl = 0; sl < RSL; ++sl) {
        const int t = (2 * sl + half) * 32 + lane;
        if (t >= ntask) continue;
        if (n == n0[sl]) cur[sl] = v0[sl];
        const int m = t / (Q + 1) - pf, mu = t - (t / (Q + 1)) * (Q + 1);
        if (abs(m) <= n) {
          const double d = n >= n0[sl] ? cur[sl] : 0.0;
          const double v1 = (((m > 0) && (m & 1)) != ((mu & 1) != 0)) ? -d : d;
          Dre[(m + pf) * NMU + mu + Q] = v1;
          if (n <= Q) Tb[(mu + Q) * NCQ + tbase + m] = v1;
          if (mu > 0) {
            const bool neg = (((m + mu) & 1) != 0) != ((m < 0) && (m & 1));
            const double v2 = neg ? -d : d;
            Dre[(pf - m) * NMU + Q - mu] = v2;
            if (n <= Q) Tb[(Q - mu) * NCQ + tbase - m] = v2;
          }
        }
        if (n >= n0[sl] && n < pf) {
          double nxt;
          if (n == 0) {
            nxt = cbeta * cur[sl];
          } else {
            const int am = abs(m);
            const double w = rn * s_isq[(n + 1) * (pf + 1) + am] * s_isq[(n + 1) * (pf + 1) + mu];
            const double A = (h1 - (double)((2 * n + 1) * m * mu)) * w;
            const double C = (n + 1) * rn * s_rt[n * (pf + 1) + am] * s_rt[n * (pf + 1) + mu];
            nxt = fma(A, cur[sl], -C * prev[sl]);
          }
          prev[sl] = cur[sl];
          cur[sl] = nxt;
        }
      }
      // (2) warp 1: the coaxial column of order n for mu >= 0 (the column of -mu is
      // the same), one lane per (nu, mu)
      if (half == 1 && lane < (Q + 1) * (Q + 2) / 2) {
        int nu = (int)((sqrtf(8.0f * lane + 1.0f) - 1.0f) * 0.5f);
        if ((nu + 1) * (nu + 2) / 2 <= lane) ++nu;
        if (nu * (nu + 1) / 2 > lane) --nu;
        const int mu = lane - nu * (nu + 1) / 2;
        const int o = nu * nu + nu + mu;
        double2 tt = c2(0.0);
        if (n >= mu) {
          const double* G = g0c + ((size_t)o * nl + n) * (Q + 1);
          const int lbase = abs(n - nu), jmax = min(n, nu);
          double gj[Q + 1];
#pragma unroll
          for (int j = 0; j <= Q; ++j) gj[j] = j <= jmax ? __ldg(G + j) : 0.0;
#pragma unroll
          for (int j = 0; j <= Q; ++j)
            if (j <= jmax) tt = caxpy(gj[j], rad[lbase + 2 * j], tt);
          tt = cmul(ipow(nu - n + 4 * pf), tt);
        }
        coaxn[o] = tt;
      }
      h3_pair_bar(cp);     // slice and column of order n complete
      // (3) rotate this warp's 8 densities on the FP64 tensor cores and translate:
      // M'(mu, r) = sum_m A[mu][m] B[m][r] with the real A = eps_m eps_mu d^n_{m mu} and
      // B = e^{i m alpha} M(n, m, r), whose real and imaginary parts are two column
      // tiles (K = 2n + 1 padded to 4; row tiles mu index 0..7 and 8..15)
      const int base = n * n + n;
      const int rho = lane >> 2, kq = lane & 3;
      double c[2][2][2];
#pragma unroll
      for (int t = 0; t < 2; ++t) c[t][0][0] = c[t][0][1] = c[t][1][0] = c[t][1][1] = 0.0;
      const double2* Eb = Es + (base - n) * RB + half * HB + rho;
      const double* Dr = Dre + (pf - n) * NMU;
      const double2* phn = ph + (pf - n);
      for (int sk = 0; 4 * sk <= 2 * n; ++sk) {
        const int kap = 4 * sk + kq;
        const bool vk = kap <= 2 * n;
        const double2 b = vk ? cmul(Eb[kap * RB], phn[kap]) : c2(0.0);
        const double a0 = (vk && rho < NMU) ? Dr[kap * NMU + rho] : 0.0;
        h3_dmma(c[0][0][0], c[0][0][1], a0, b.x);
        h3_dmma(c[0][1][0], c[0][1][1], a0, b.y);
        if (NTILE == 4) {
          const double a1 = (vk && 8 + rho < NMU) ? Dr[kap * NMU + 8 + rho] : 0.0;
          h3_dmma(c[1][0][0], c[1][0][1], a1, b.x);
          h3_dmma(c[1][1][0], c[1][1][1], a1, b.y);
        }
      }
#pragma unroll
      for (int sl = 0; sl < 4; ++sl) {
        const int grp = sl >> 1, v = sl & 1;
        const int mu = (grp ? 8 + rho : rho) - Q;
        if (grp * 8 + rho >= NMU || abs(mu) > n || (grp && NTILE < 4)) continue;
        const double2 mr = c2(c[grp][0][v], c[grp][1][v]);
        const int amu = abs(mu);
#pragma unroll
        for (int nu = 0; nu <= Q; ++nu)
          if (nu >= amu) lacc[sl][nu] = cfma(coaxn[nu * nu + nu + amu], mr, lacc[sl][nu]);
      }
    }
    h3_pair_bar(cp);       // both warps done with the slices; back-rotation matrices complete
    {
      const int rho = lane >> 2;
#pragma unroll
      for (int sl = 0; sl < 4; ++sl) {
        const int grp = sl >> 1, r = 2 * (lane & 3) + (sl & 1);
        const int mu = (grp ? 8 + rho : rho) - Q;
        if (grp * 8 + rho >= NMU) continue;
#pragma unroll
        for (int nu = 0; nu <= Q; ++nu)
          if (nu >= abs(mu)) Lp[(nu * nu + nu + mu) * HB + r] = lacc[sl][nu];
      }
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < NOUT; ++i) {
      const int task = lane + 32 * i;
      if (task >= NCQ * HB) break;
      const int o = task / HB, r = task - o * HB;
      const int nu = s_nof[o];
      const int mu2 = o - nu * nu - nu;
      double2 a = c2(0.0);
      for (int mu = -nu; mu <= nu; ++mu) a = caxpy(Tb[(mu + Q) * NCQ + o], Lp[(nu * nu + nu + mu) * HB + r], a);
      acc[i] = cfma(cconj(ph[mu2 + pf]), a, acc[i]);
    }
  }
  if (!has) return;
  const double st = h3_scale(hc.k, g.expansion_radii[ctr]);
#pragma unroll
  for (int i = 0; i < NOUT; ++i) {
    const int task = lane + 32 * i;
    if (task >= NCQ * HB) break;
    const int o = task / HB, r = task - o * HB;
    const int rr = r0 + half * HB + r;
    if (rr >= nrhs) continue;
    const int nu = s_nof[o];
    double2* out = qbx_exps + ((size_t)ctr * nrhs + rr) * NCQ + o;
    *out = caxpy(pow(st, (double)nu), acc[i], *out);
  }
}

// QBXL2P: one thread per used center, over its targets
__global__ void __launch_bounds__(NT)
k_h3_qbxl2p(qbxfmm_geometry g, HelmCoeffs hc, int q, int nrhs, const double2* __restrict__ qbx_exps,
            double2* __restrict__ pot_tree)
{
  extern __shared__ double2 smem2[];
  double2* rec = smem2;
  h3_rec_table(q, rec, threadIdx.x, NT);
  __syncthreads();
  int ig = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (ig >= g.nglobal_qbx_centers) return;
  int ctr = g.global_qbx_centers[ig];
  double cc[3];
  load_point<3>(g.centers, g.ncenters, ctr, cc);
  double s = h3_scale(hc.k, g.expansion_radii[ctr]);
  int ncq = (q + 1) * (q + 1);
  const double2* Lc = qbx_exps + ((size_t)ctr * nrhs + r) * ncq;
  for (int it = g.center_to_targets_starts[ctr]; it < g.center_to_targets_starts[ctr + 1]; ++it) {
    int t = g.center_to_targets_lists[it];
    double x[3];
    load_point<3>(g.targets, g.ntargets, t, x);
    double2* P = pot_tree + (size_t)r * g.ntargets + t;
    *P = cadd(*P, h3_e2p(Lc, q, true, hc.k, s, cc, x, rec, hc.taylor ? q : -1));
  }
}

// Target-specific near field (eval_target_specific_qbx_locals, pytential/qbx/fmm.py:391-394;
// the reference's native module pytential/qbx/target_specific/impl.pyx:363-563):
// per (target t, its center c, list-1 source y), with a = t - c, b = y - c,
//   K_S = ik sum_{n<=Q} (2n+1) j_n(k|a|) h_n(k|b|) P_n(cos g),
//   K_D = ik sum (2n+1) j_n(k|a|) (k h_n'(k|b|) P_n nu.bh + h_n P_n' (nu.ah - cos g nu.bh) / |b|),
// the order-Q spherical-wave QBX expansion evaluated without forming it.  The kernel
// value K = cq K_S + cd K_D is computed once per pair and applied to RB densities at
// a time (lane = target; 4 warps split each 128-source tile; strengths of the tile's
// sources for the RB densities staged in shared memory).
template <int Q, int RB>
__global__ void __launch_bounds__(NT)
k_h3_tsqbx(qbxfmm_geometry g, HelmCoeffs hc, int nrhs, const double2* __restrict__ strengths,
           double2* __restrict__ pot_tree, int32_t* err)
{
  __shared__ double s_y[3][NT], s_n[3][NT];
  __shared__ double2 s_q[RB][NT];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];
  extern __shared__ double2 smem2[];
  double2* s_red = smem2;   // [NW-1][32][RB]
  int chunk = blockIdx.x;
  int r0 = blockIdx.y * RB;
  int itb = g.tsqbx_chunk_target_box[chunk];
  int i0 = g.tsqbx_chunk_start[chunk];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bool active = lane < g.tsqbx_chunk_count[chunk];
  int t = active ? g.tsqbx_targets[i0 + lane] : 0;
  int ctr = active ? g.tsqbx_centers[i0 + lane] : 0;
  if ((unsigned)ctr >= (unsigned)g.ncenters || (unsigned)t >= (unsigned)g.ntargets) {
    report(err, QBX_DEVERR_BAD_CENTER);
    active = false;
    t = ctr = 0;
  }
  double cc[3], x[3];
  load_point<3>(g.centers, g.ncenters, ctr, cc);
  load_point<3>(g.targets, g.ntargets, t, x);
  double a[3] = {x[0] - cc[0], x[1] - cc[1], x[2] - cc[2]};
  double alen = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  double ainv = alen > 0.0 ? 1.0 / alen : 0.0;
  double ah[3] = {a[0] * ainv, a[1] * ainv, a[2] * ainv};
  double jn[Q + 1];
  {
    double jv[H3_LMAX + 2];
    h3_sph_j_cut(Q, hc.k * alen, hc.taylor ? Q : -1, jv);
#pragma unroll
    for (int n = 0; n <= Q; ++n) jn[n] = (2.0 * n + 1.0) * jv[n];
  }
  const bool chg = hc.cq.x != 0.0 || hc.cq.y != 0.0;
  const bool dip = hc.cd.x != 0.0 || hc.cd.y != 0.0;
  // ik cq, ik cd
  const double2 kq = c2(-hc.k * hc.cq.y, hc.k * hc.cq.x), kd = c2(-hc.k * hc.cd.y, hc.k * hc.cd.x);
  double2 acc[RB];
#pragma unroll
  for (int i = 0; i < RB; ++i) acc[i] = c2(0.0);
  int l0 = g.list1_starts[itb], l1 = g.list1_starts[itb + 1];
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    h3_list_prefix(g, g.list1_lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += NT) {
      int v = base + threadIdx.x;
      if (v < total) {
        int s = h3_stream_source(v, nb, s_pref, s_start);
        double y[3], nv[3] = {0, 0, 0};
        load_point<3>(g.sources, g.nsources, s, y);
        if (dip) load_point<3>(g.source_normals, g.nsources, s, nv);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          s_y[d][threadIdx.x] = y[d];
          s_n[d][threadIdx.x] = nv[d];
        }
#pragma unroll
        for (int i = 0; i < RB; ++i)
          s_q[i][threadIdx.x] = (r0 + i < nrhs) ? strengths[(size_t)(r0 + i) * g.nsources + s] : c2(0.0);
      }
      __syncthreads();
      int jbeg = warp * 32, jend = min(jbeg + 32, total - base);
      if (active) {
        for (int j = jbeg; j < jend; ++j) {
          double b0 = s_y[0][j] - cc[0], b1 = s_y[1][j] - cc[1], b2 = s_y[2][j] - cc[2];
          double b2s = b0 * b0 + b1 * b1 + b2 * b2;
          if (b2s == 0.0) continue;
          double binv = rsqrt(b2s);
          double blen = b2s * binv;
          double cg = (ah[0] * b0 + ah[1] * b1 + ah[2] * b2) * binv;
          double2 h[Q + 2];
          h3_sph_h(Q + 1, hc.k * blen, h);
          double xinv = 1.0 / (hc.k * blen);
          double pm1 = 1.0, pm2 = 0.0, dm1 = 0.0;
          double2 sS = c2(0.0), sA = c2(0.0), sB = c2(0.0);
#pragma unroll
          for (int n = 0; n <= Q; ++n) {
            double pn, dn;
            if (n == 0) {
              pn = 1.0;
              dn = 0.0;
            } else if (n == 1) {
              pn = cg;
              dn = 1.0;
            } else {
              pn = ((2.0 * n - 1) * cg * pm1 - (n - 1.0) * pm2) * (1.0 / n);
              dn = n * pm1 + cg * dm1;
            }
            if (chg) sS = caxpy(jn[n] * pn, h[n], sS);
            if (dip) {
              // h_n'(x) = h_{n-1} - (n+1)/x h_n  (n >= 1), h_0' = -h_1
              double2 hd = (n == 0) ? c2(-h[1].x, -h[1].y)
                                    : caxpy(-(n + 1.0) * xinv, h[n], h[n - 1]);
              sA = caxpy(jn[n] * pn * hc.k, hd, sA);
              sB = caxpy(jn[n] * dn, h[n], sB);
            }
            pm2 = pm1;
            pm1 = pn;
            dm1 = dn;
          }
          double2 K = c2(0.0);
          if (chg) K = cmul(kq, sS);
          if (dip) {
            double db = (s_n[0][j] * b0 + s_n[1][j] * b1 + s_n[2][j] * b2) * binv;
            double da = s_n[0][j] * ah[0] + s_n[1][j] * ah[1] + s_n[2][j] * ah[2];
            double2 vd = caxpy(db, sA, cscale((da - cg * db) * binv, sB));
            K = cfma(kd, vd, K);
          }
#pragma unroll
          for (int i = 0; i < RB; ++i) acc[i] = cfma(K, s_q[i][j], acc[i]);
        }
      }
      __syncthreads();
    }
  }
  if (warp > 0) {
#pragma unroll
    for (int i = 0; i < RB; ++i) s_red[((warp - 1) * 32 + lane) * RB + i] = acc[i];
  }
  __syncthreads();
  if (warp == 0 && active) {
#pragma unroll
    for (int i = 0; i < RB; ++i) {
      if (r0 + i >= nrhs) continue;
      double2 v = acc[i];
      for (int w = 1; w < NW; ++w) v = cadd(v, s_red[((w - 1) * 32 + lane) * RB + i]);
      double2* P = pot_tree + (size_t)(r0 + i) * g.ntargets + t;
      *P = cadd(*P, v);
    }
  }
}

// }}}

// {{{ translation matrices

// One CTA per matrix.  kind 1: M2M (parent level lev, child position ci; b = c_parent -
// c_child), kind 2: L2L (child level lev, child position ci; b = c_child - c_parent).
// T is the real (rp x kp) form of the complex (ncf x ncf) matrix acting on
// interleaved (re, im) coefficient vectors; entries outside 2 ncf are zero.
__global__ void __launch_bounds__(NT)
k_h3_trans_build(int kind, int p, int rp, int kp, double k, double root_extent, int lev0,
                 const double* __restrict__ gaunt, double* __restrict__ T)
{
  extern __shared__ double2 smem2[];
  const int L = 2 * p;
  const int ncf = (p + 1) * (p + 1);
  const int nl = p + 1;
  double2* rec = smem2;                                  // [(L+1)(L+2)/2]
  double2* Wt = rec + (L + 1) * (L + 2) / 2;              // [(L+1)^2]
  double2* rad = Wt + (L + 1) * (L + 1);                 // [L+2]
  double* pw = reinterpret_cast<double*>(rad + L + 2);   // [2][p+1]: s_in^{e n}, s_out^{e nu}
  int mi = blockIdx.x;
  double b[3];
  double s_in, s_out;
  int e_in, e_out;
  {
    int lev = lev0 + mi / 8, ci = mi % 8;
    int plev = (kind == 1) ? lev : lev - 1;        // parent level
    double wp = ldexp(root_extent, -plev);
    double sgn = (kind == 1) ? -1.0 : 1.0;         // M2M: c_p - c_c; L2L: c_c - c_p
    for (int d = 0; d < 3; ++d) b[d] = sgn * (((ci >> d) & 1) ? 0.25 : -0.25) * wp;
    double sp = fmin(1.0, k * wp), sc = fmin(1.0, k * 0.5 * wp);
    if (kind == 1) {
      s_in = sc; e_in = 1; s_out = sp; e_out = -1;
    } else {
      s_in = sp; e_in = -1; s_out = sc; e_out = 1;
    }
  }
  h3_rec_table(L, rec, threadIdx.x, NT);
  double2 w;
  double rr;
  double t = h3_dir(b, w, rr);
  if (threadIdx.x == 0) {
    double jv[H3_LMAX + 2];
    h3_sph_j(L, k * rr, jv);
    for (int l = 0; l <= L; ++l) rad[l] = cmul(cscale(FOUR_PI, ipow(l)), c2(jv[l]));
  }
  for (int n = threadIdx.x; n <= p; n += NT) {
    pw[n] = pow(s_in, (double)(e_in * n));
    pw[p + 1 + n] = pow(s_out, (double)(e_out * n));
  }
  __syncthreads();
  for (int m = threadIdx.x; m <= L; m += NT) h3_wave_column(m, L, t, w, rec, rad, Wt, 1);
  __syncthreads();
  double* Tm = T + (size_t)mi * rp * kp;
  for (int e = threadIdx.x; e < ncf * ncf; e += NT) {
    int o = e / ncf, i = e - o * ncf;      // row (nu, mu), column (n, m)
    int nu, mu, n, m;
    hq_decode(o, nu, mu);
    hq_decode(i, n, m);
    const double* Gc = gaunt + (size_t)o * nl * ncf + i;
    int lam = m - mu, lbase = abs(n - nu), jmax = min(n, nu);
    double2 tt = c2(0.0);
    for (int j = 0; j <= jmax; ++j) {
      int l = lbase + 2 * j;
      if (abs(lam) > l) continue;
      tt = caxpy(Gc[(size_t)j * ncf], Wt[hq(l, lam)], tt);
    }
    // c = i^{nu - n} tt, scaled
    double2 v = cscale(pw[n] * pw[p + 1 + nu], cmul(ipow(nu - n + 4 * p), tt));
    size_t r0 = (size_t)(2 * o) * kp + 2 * i;
    Tm[r0] = v.x;
    Tm[r0 + 1] = -v.y;
    Tm[r0 + kp] = v.y;
    Tm[r0 + kp + 1] = v.x;
  }
  // zero padding
  for (size_t e = threadIdx.x; e < (size_t)rp * kp; e += NT) {
    int row = (int)(e / kp), col = (int)(e % kp);
    if (row >= 2 * ncf || col >= 2 * ncf) Tm[e] = 0.0;
  }
}

// }}}

// {{{ assembly

__global__ void k_h3_assemble_tree(qbxfmm_geometry g, int nrhs, const double2* __restrict__ pot_tree,
                                   double2* __restrict__ out)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (t >= g.ntargets) return;
  int u = g.sorted_target_ids[t] - g.ncenters;
  if (u >= 0) out[(size_t)r * g.nuser_targets + u] = cscale(1.0 / FOUR_PI, pot_tree[(size_t)r * g.ntargets + t]);
}

__global__ void k_h3_assemble_nonqbx(qbxfmm_geometry g, int nrhs,
                                     const double2* __restrict__ pot_nonqbx, double2* __restrict__ out)
{
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (f >= g.nfiltered_targets) return;
  int t = g.unfiltered_from_filtered_target_indices[f];
  int u = g.sorted_target_ids[t] - g.ncenters;
  if (u >= 0) {
    double2* o = out + (size_t)r * g.nuser_targets + u;
    *o = caxpy(1.0 / FOUR_PI, pot_nonqbx[(size_t)r * g.nfiltered_targets + f], *o);
  }
}

// }}}

// {{{ M2L by rotation (3D Helmholtz)

// Multipole -> local translation between boxes of one level by rotation, coaxial
// translation and back rotation (the same factorization as the QBX translations
// above, with output order pf and all |mu| <= pf).  The rotation depends only on the
// direction of the box offset and the coaxial part only on its length and the level,
// so both are tabulated once per plan: per direction the phases e^{i m alpha} and the
// blocks T^n[m][mu] = eps_m eps_mu d^n_{m mu}(beta), |mu| <= n <= pf, for m >= 0 only
// (with these signs T^n[-m][-mu] = T^n[m][mu]); per (length, level) the coaxial
// blocks for mu >= 0 (C^{-mu} = C^mu, the Gaunt coefficients of +-mu being equal),
// C^mu[n][nu] = s^nu s^n i^{nu-n} sum_j G(n,mu; nu,mu; |n-nu|+2j) sqrt(4 pi (2l+1))
// i^l h_l(k|b|) (l = |n-nu|+2j), s = min(1, k width).

// start of order n's block: sum_{k<n} (k+1)(2k+1)
QBX_D int h3_dblock(int n) { return n * (n - 1) * (2 * n - 1) / 3 + 3 * n * (n - 1) / 2 + n; }

// start of the coaxial block of |mu| = mu: sum_{u<mu} (pf+1-u)^2
QBX_D int h3_cblock(int pf, int mu)
{
  int o = 0;
  for (int u = 0; u < mu; ++u) o += (pf + 1 - u) * (pf + 1 - u);
  return o;
}

__host__ __device__ size_t h3_m2l_dsize(int pf)
{
  size_t nm = 2 * pf + 1, v = 2 * nm;
  for (int n = 0; n <= pf; ++n) v += (size_t)(n + 1) * (2 * n + 1);
  return (v + 1) & ~(size_t)1;
}

__host__ __device__ size_t h3_m2l_csize(int pf)
{
  size_t s = 0;
  for (int u = 0; u <= pf; ++u) s += (size_t)(pf + 1 - u) * (pf + 1 - u);
  return s;
}

// Tables: CTAs [0, ndir) one direction each, [ndir, ndir + ncoax) one (length, level)
// each.  dirs[4 d] = unit offset; coaxp[2 c] = (k |b|, s); start: [nm][nm][4] start
// values of d^n_{m mu} (coefficient, exponents of cos and sin of beta/2); isq / rt: the
// recurrence factors of the rotation tables; gaunt: [(nu,mu)][j][(n,m)].
__global__ void __launch_bounds__(NT)
k_h3_m2l_tables(int pf, int ndir, int ncoax, const double* __restrict__ dirs,
                const double* __restrict__ coaxp, const double* __restrict__ start,
                const double* __restrict__ isq, const double* __restrict__ rt,
                const double* __restrict__ gaunt, double* __restrict__ Dtab,
                double2* __restrict__ Ctab)
{
  __shared__ double2 s_rad[2 * H3_MAXP + 4];
  __shared__ double s_pw[H3_MAXP + 1];
  const int nm = 2 * pf + 1, nl = pf + 1, ncf = (pf + 1) * (pf + 1);
  if ((int)blockIdx.x < ndir) {
    const double* u = dirs + 4 * blockIdx.x;
    double cbeta = fmin(1.0, fmax(-1.0, u[2]));
    double alpha = (u[0] == 0.0 && u[1] == 0.0) ? 0.0 : atan2(u[1], u[0]);
    double beta = acos(cbeta);
    double ch = cos(0.5 * beta), sh = sin(0.5 * beta);
    double* D = Dtab + blockIdx.x * h3_m2l_dsize(pf);
    double2* ph = reinterpret_cast<double2*>(D);
    double* blocks = D + 2 * nm;
    for (int m = threadIdx.x; m < nm; m += NT) {
      double sn, cs;
      sincos((m - pf) * alpha, &sn, &cs);
      ph[m] = c2(cs, sn);
    }
    for (int t = threadIdx.x; t < (pf + 1) * nm; t += NT) {
      int m = t / nm, mu = t % nm - pf;   // rows m >= 0 (T^n[-m][-mu] = T^n[m][mu])
      int am = abs(m), amu = abs(mu);
      int n0 = max(am, amu);
      const int ts = (m + pf) * nm + (mu + pf);   // index of the start table
      double v = start[4 * ts];
      int ec = (int)start[4 * ts + 1], es = (int)start[4 * ts + 2];
      for (int k = 0; k < ec; ++k) v *= ch;
      for (int k = 0; k < es; ++k) v *= sh;
      double eps = ((m > 0 && (m & 1)) ? -1.0 : 1.0) * ((mu > 0 && (mu & 1)) ? -1.0 : 1.0);
      double prev = 0.0, cur = v;
      for (int n = n0; n <= pf; ++n) {
        blocks[h3_dblock(n) + m * (2 * n + 1) + (mu + n)] = eps * cur;
        if (n == pf) break;
        double nxt;
        if (n == 0) {
          nxt = cbeta * cur;
        } else {
          double rn = 1.0 / n;
          double w = rn * isq[(n + 1) * (pf + 1) + am] * isq[(n + 1) * (pf + 1) + amu];
          double A = (2.0 * n + 1.0) * (n * (n + 1.0) * cbeta - (double)m * mu) * w;
          double C = (n + 1.0) * rn * rt[n * (pf + 1) + am] * rt[n * (pf + 1) + amu];
          nxt = fma(A, cur, -C * prev);
        }
        prev = cur;
        cur = nxt;
      }
    }
    return;
  }
  int c = blockIdx.x - ndir;
  if (c >= ncoax) return;
  double kb = coaxp[2 * c], s = coaxp[2 * c + 1];
  const int L = 2 * pf;
  if (threadIdx.x == 0) {
    h3_sph_h(L, kb, s_rad);
    for (int l = 0; l <= L; ++l) s_rad[l] = cmul(cscale(sqrt(FOUR_PI * (2.0 * l + 1.0)), ipow(l)), s_rad[l]);
  }
  for (int n = threadIdx.x; n <= pf; n += NT) s_pw[n] = pow(s, (double)n);
  __syncthreads();
  double2* C = Ctab + (size_t)c * h3_m2l_csize(pf);
  int total = (int)h3_m2l_csize(pf);
  for (int e = threadIdx.x; e < total; e += NT) {
    // decode (mu >= 0, n, nu)
    int mu = 0, off = 0;
    for (;;) {
      int w = pf + 1 - mu;
      if (e < off + w * w) break;
      off += w * w;
      ++mu;
    }
    int am = mu, w = pf + 1 - am;
    int n = am + (e - off) / w, nu = am + (e - off) % w;
    int o = nu * nu + nu + mu;
    int lbase = abs(n - nu), jmax = min(n, nu);
    double2 tt = c2(0.0);
    for (int j = 0; j <= jmax; ++j)
      tt = caxpy(__ldg(gaunt + ((size_t)o * nl + j) * ncf + n * n + n + mu), s_rad[lbase + 2 * j], tt);
    tt = cmul(ipow(nu - n + 4 * pf), tt);
    C[e] = cscale(s_pw[nu] * s_pw[n], tt);
  }
}

constexpr int H3M2L_NT = 256;
// task groups of 4 outputs: sum_n ceil((2n+1)/4) <= 99 and sum_mu ceil((pf+1-|mu|)/4)
// <= 116 for pf <= H3_MAXP
constexpr int H3M2L_NG = 100;
constexpr int H3M2L_NCG = 120;

// One CTA per target-or-parent box (blockIdx.x) and group of RB densities; its
// list-2 sources in turn: X = e^{i m alpha} M (shared), A = rotated (all n, |mu| <= n),
// B = coaxially translated (into X), then the back rotation adds into register
// accumulators owned by fixed (order, 4 consecutive m, density) tasks; the sum is
// added into the box's local once.  Each task keeps four outputs, so one shared
// load of the input feeds eight FMAs.  The pair's rotation table, then its coaxial
// table, then the rotation table again are copied into one shared buffer by all
// threads (16-byte loads, all in flight together) before the step that reads them,
// so the inner loops read shared memory only.
template <typename R, int RB>
__global__ void __launch_bounds__(H3M2L_NT)
k_h3_m2l_rot(qbxfmm_geometry g, int pf, int nrhs, const double2* __restrict__ mp,
             double2* __restrict__ lo, const double* __restrict__ Dtab,
             const double2* __restrict__ Ctab, const double* __restrict__ clsmap,
             int32_t* err)
{
  // R: the arithmetic (double, or float in the mixed-precision form; expansions are
  // read and added in float64 either way)
  using V = cplx_t<R>;
  extern __shared__ double2 smem2[];
  __shared__ int s_gn[H3M2L_NG], s_gm0[H3M2L_NG];        // rotation task groups
  __shared__ int s_cmu[H3M2L_NCG], s_cnu0[H3M2L_NCG];    // coaxial task groups
  __shared__ int s_ng, s_ncg;
  __shared__ unsigned char s_nof[(H3_MAXP + 1) * (H3_MAXP + 1)];   // order n of coefficient (n, m)
  constexpr int NTHR = H3M2L_NT;
  constexpr int KMAX = (H3M2L_NG * RB + NTHR - 1) / NTHR;
  const int ncf = (pf + 1) * (pf + 1), XS = ncf + 1, nm = 2 * pf + 1;
  V* X = reinterpret_cast<V*>(smem2);      // [RB][ncf + 1]
  V* A = X + (size_t)RB * XS;               // [RB][ncf + 1]
  V* Tbuf = A + (size_t)RB * XS;            // rotation or coaxial table of the pair
  if (threadIdx.x == 0) {
    int ng = 0;
    for (int n = 0; n <= pf; ++n)
      for (int m0 = -n; m0 <= n; m0 += 4) {
        s_gn[ng] = n;
        s_gm0[ng] = m0;
        ++ng;
      }
    s_ng = ng;
    int ncg = 0;
    for (int mu = -pf; mu <= pf; ++mu)
      for (int nu0 = abs(mu); nu0 <= pf; nu0 += 4) {
        s_cmu[ncg] = mu;
        s_cnu0[ncg] = nu0;
        ++ncg;
      }
    s_ncg = ncg;
  }
  for (int n = 0; n <= pf; ++n)
    for (int x = n * n + threadIdx.x; x < (n + 1) * (n + 1); x += NTHR) s_nof[x] = (unsigned char)n;
  __syncthreads();
  const int i = blockIdx.x;
  const int r0 = blockIdx.y * RB;
  const int q0 = g.m2l_tgt_pair_starts[i], q1 = g.m2l_tgt_pair_starts[i + 1];
  if (q1 <= q0) return;
  const int ng = s_ng, ncg = s_ncg;
  const size_t dsz = h3_m2l_dsize(pf), csz = h3_m2l_csize(pf);
  V acc[KMAX][4];
#pragma unroll
  for (int k = 0; k < KMAX; ++k)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[k][j] = cmake<R>(0);

  for (int q = q0; q < q1; ++q) {
    int pr = g.m2l_tgt_pairs[q];
    int src = g.m2l_pair_src[pr];
    // class of the pair: m2l_class_starts[c] <= pr < m2l_class_starts[c + 1]
    int lo_c = 0, hi_c = g.m2l_nclasses - 1;
    while (lo_c < hi_c) {
      int mid = (lo_c + hi_c + 1) >> 1;
      if (g.m2l_class_starts[mid] <= pr) lo_c = mid;
      else hi_c = mid - 1;
    }
    if ((unsigned)src >= (unsigned)g.nboxes) {
      if (threadIdx.x == 0) report(err, QBX_DEVERR_BAD_BOX);
      continue;   // uniform across the CTA
    }
    const double2* Dg = reinterpret_cast<const double2*>(Dtab + (size_t)clsmap[2 * lo_c] * dsz);
    const double2* Cg = Ctab + (size_t)clsmap[2 * lo_c + 1] * csz;
    // the rotation table into Tbuf (phases, then the d blocks)
    for (int x = threadIdx.x; x < (int)(dsz / 2); x += NTHR) Tbuf[x] = cto(__ldg(Dg + x), V());
    const V* ph = Tbuf;
    const R* blocks = reinterpret_cast<const R*>(Tbuf) + 2 * nm;
    const V* C = Tbuf;
    // X = e^{i m alpha} M
    for (int e = threadIdx.x; e < RB * ncf; e += NTHR) {
      int r = e / ncf, ci = e - r * ncf;
      int n = s_nof[ci];
      V v = cmake<R>(0);
      if (r0 + r < nrhs)
        v = cto(cmul(__ldg(Dg + ci - n * n - n + pf), mp[((size_t)src * nrhs + r0 + r) * ncf + ci]), V());
      X[r * XS + ci] = v;
    }
    __syncthreads();
    // A[(n, mu)] = sum_m T^n[m][mu] X[(n, m)]
    for (int t = threadIdx.x; t < ng * RB; t += NTHR) {
      int grp = t / RB, r = t - grp * RB;
      int n = s_gn[grp], mu0 = s_gm0[grp];
      const R* Tn = blocks + h3_dblock(n);
      const int w = 2 * n + 1, nv = min(4, n - mu0 + 1);
      V o[4] = {cmake<R>(0), cmake<R>(0), cmake<R>(0), cmake<R>(0)};
      const V* Xr = X + r * XS + n * n;
      for (int m = 0; m < w; ++m) {
        V x = Xr[m];
        // T^n[m - n][mu0 + j]: row m - n >= 0 directly, else row n - m at -mu (reversed)
        const int ma = m - n;
        const R* row = ma >= 0 ? Tn + ma * w + (mu0 + n) : Tn + (-ma) * w + (n - mu0);
        const int step = ma >= 0 ? 1 : -1;
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (j < nv) o[j] = caxpy(row[step * j], x, o[j]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (j < nv) A[r * XS + n * n + n + mu0 + j] = o[j];
    }
    __syncthreads();
    for (int x = threadIdx.x; x < (int)csz; x += NTHR) Tbuf[x] = cto(__ldg(Cg + x), V());
    __syncthreads();
    // B[(nu, mu)] = sum_{n >= |mu|} C^mu[n][nu] A[(n, mu)]   (into X)
    for (int t = threadIdx.x; t < ncg * RB; t += NTHR) {
      int grp = t / RB, r = t - grp * RB;
      int mu = s_cmu[grp], nu0 = s_cnu0[grp];
      int am = abs(mu), w = pf + 1 - am, nv = min(4, pf - nu0 + 1);
      const V* Cb = C + h3_cblock(pf, am) + (nu0 - am);
      V o[4] = {cmake<R>(0), cmake<R>(0), cmake<R>(0), cmake<R>(0)};
      const V* Ar = A + r * XS;
      for (int n = am; n <= pf; ++n) {
        V a = Ar[n * n + n + mu];
        const V* row = Cb + (n - am) * w;
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (j < nv) o[j] = cfma(row[j], a, o[j]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int nu = nu0 + j;
        if (j < nv) X[r * XS + nu * nu + nu + mu] = o[j];
      }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < (int)(dsz / 2); x += NTHR) Tbuf[x] = cto(__ldg(Dg + x), V());
    __syncthreads();
    // L[(nu, m2)] += e^{-i m2 alpha} sum_mu T^nu[m2][mu] B[(nu, mu)]
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
      int t = threadIdx.x + k * NTHR;
      if (t >= ng * RB) break;
      int grp = t / RB, r = t - grp * RB;
      int nu = s_gn[grp], m20 = s_gm0[grp];
      const int w = 2 * nu + 1, nv = min(4, nu - m20 + 1);
      const R* Tn = blocks + h3_dblock(nu);
      // T^nu[m2][mu] for m2 = m20 + j: row m2 >= 0 directly, else row -m2 at -mu
      const R* pj[4];
      int sj[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int m2 = m20 + j;
        pj[j] = m2 >= 0 ? Tn + m2 * w : Tn + (-m2) * w + 2 * nu;
        sj[j] = m2 >= 0 ? 1 : -1;
      }
      V o[4] = {cmake<R>(0), cmake<R>(0), cmake<R>(0), cmake<R>(0)};
      const V* Br = X + r * XS + nu * nu;
      for (int mu = 0; mu < w; ++mu) {
        V b = Br[mu];
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (j < nv) o[j] = caxpy(pj[j][sj[j] * mu], b, o[j]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (j < nv) acc[k][j] = cfma(cconj(ph[m20 + j + pf]), o[j], acc[k][j]);
    }
    __syncthreads();
  }
  int tb = g.target_or_target_parent_boxes[i];
  if ((unsigned)tb >= (unsigned)g.nboxes) {
    if (threadIdx.x == 0) report(err, QBX_DEVERR_BAD_BOX);
    return;
  }
#pragma unroll
  for (int k = 0; k < KMAX; ++k) {
    int t = threadIdx.x + k * NTHR;
    if (t >= ng * RB) break;
    int grp = t / RB, r = t - grp * RB;
    if (r0 + r >= nrhs) continue;
    int nu = s_gn[grp], m20 = s_gm0[grp];
    int nv = min(4, nu - m20 + 1);
    double2* out = lo + ((size_t)tb * nrhs + r0 + r) * ncf + nu * nu + nu + m20;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (j < nv) out[j] = cadd(out[j], c2d(acc[k][j]));
  }
}

// {{{ M2L with the pair tables brought in by bulk copies

QBX_D unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

QBX_D void mbar_init(uint64_t* mb)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(mb)) : "memory");
}

// one arrival that also expects `bytes` of copy completion on the barrier
QBX_D void mbar_expect(uint64_t* mb, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n"
               ::"r"(smem_addr(mb)), "r"(bytes) : "memory");
}

// global -> this CTA's shared memory, completion counted on mb (16-byte aligned
// addresses, size a multiple of 16)
QBX_D void bulk_copy(void* dst, const void* src, unsigned bytes, uint64_t* mb)
{
  asm volatile("fence.proxy.async.shared::cta;\n"
               "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
               ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(mb)) : "memory");
}

// bounded wait for the phase of the given parity; false if it did not complete
QBX_D bool mbar_wait(uint64_t* mb, unsigned parity)
{
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done) : "r"(smem_addr(mb)), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}

// The FP64 M2L of k_h3_m2l_rot with its pair tables brought in by bulk copies
// (cp.async.bulk, completion on an mbarrier) into buffers of their own: the rotation
// table once per pair (the register-staged form copies it twice, before the rotation
// and again before the back rotation, because it shares one buffer with the coaxial
// table) and the coaxial table of pair q + 1 while pair q's back rotation runs.  One
// thread issues the copies; waits are bounded: a copy that does not arrive sets the
// error word, the CTA waits (bounded) for the copies it issued and stops.  With ND = 2
// the rotation table has two buffers: pair q + 1's is requested as soon as pair q's
// has arrived (into the buffer pair q - 1 used), so its copy runs under all of pair
// q's work instead of between the pairs.
template <int RB, int NTHR = H3M2L_NT, int ND = 1>
__global__ void __launch_bounds__(NTHR, NTHR == H3M2L_NT ? 2 : 1)
k_h3_m2l_bulk(qbxfmm_geometry g, int pf, int nrhs, const double2* __restrict__ mp,
              double2* __restrict__ lo, const double* __restrict__ Dtab,
              const double2* __restrict__ Ctab, const double* __restrict__ clsmap,
              int32_t* err)
{
  static_assert(ND == 1 || ND == 2, "one or two rotation-table buffers");
  extern __shared__ double2 smem2[];
  __shared__ uint64_t mbD[ND], mbC;
  __shared__ int s_gn[H3M2L_NG], s_gm0[H3M2L_NG];
  __shared__ int s_cmu[H3M2L_NCG], s_cnu0[H3M2L_NCG];
  __shared__ int s_ng, s_ncg;
  __shared__ unsigned char s_nof[(H3_MAXP + 1) * (H3_MAXP + 1)];
  constexpr int KMAX = (H3M2L_NG * RB + NTHR - 1) / NTHR;
  const int ncf = (pf + 1) * (pf + 1), XS = ncf + 1, nm = 2 * pf + 1;
  const size_t dsz = h3_m2l_dsize(pf), csz = h3_m2l_csize(pf);
  double2* X = smem2;                                              // [RB][ncf + 1]
  double2* A = X + (size_t)RB * XS;                                // [RB][ncf + 1]
  double* Db0 = reinterpret_cast<double*>(A + (size_t)RB * XS);    // [ND][dsz]
  double2* Cb = reinterpret_cast<double2*>(Db0 + ND * dsz);         // [csz]
  if (threadIdx.x == 0) {
    int ng = 0;
    for (int n = 0; n <= pf; ++n)
      for (int m0 = -n; m0 <= n; m0 += 4) {
        s_gn[ng] = n;
        s_gm0[ng] = m0;
        ++ng;
      }
    s_ng = ng;
    int ncg = 0;
    for (int mu = -pf; mu <= pf; ++mu)
      for (int nu0 = abs(mu); nu0 <= pf; nu0 += 4) {
        s_cmu[ncg] = mu;
        s_cnu0[ncg] = nu0;
        ++ncg;
      }
    s_ncg = ncg;
    for (int b = 0; b < ND; ++b) mbar_init(&mbD[b]);
    mbar_init(&mbC);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  for (int n = 0; n <= pf; ++n)
    for (int x = n * n + threadIdx.x; x < (n + 1) * (n + 1); x += NTHR) s_nof[x] = (unsigned char)n;
  __syncthreads();
  const int i = blockIdx.x;
  const int r0 = blockIdx.y * RB;
  const int q0 = g.m2l_tgt_pair_starts[i], q1 = g.m2l_tgt_pair_starts[i + 1];
  if (q1 <= q0) return;                    // before any copy is issued
  const int ng = s_ng, ncg = s_ncg;
  const unsigned dbytes = (unsigned)(dsz * sizeof(double)), cbytes = (unsigned)(csz * sizeof(double2));
  auto cls_of = [&](int q) {
    const int pr = g.m2l_tgt_pairs[q];
    int lo_c = 0, hi_c = g.m2l_nclasses - 1;
    while (lo_c < hi_c) {
      const int mid = (lo_c + hi_c + 1) >> 1;
      if (g.m2l_class_starts[mid] <= pr) lo_c = mid;
      else hi_c = mid - 1;
    }
    return lo_c;
  };
  // copies issued / completed-and-waited per barrier (the phase parity of the next
  // wait is the completed count's)
  int nd_issued[ND], nd_done[ND], nc_issued = 0, nc_done = 0;
#pragma unroll
  for (int b = 0; b < ND; ++b) nd_issued[b] = nd_done[b] = 0;
  auto issue_D = [&](int q, int b) {
    if (threadIdx.x == 0) {
      const int c = cls_of(q);
      mbar_expect(&mbD[b], dbytes);
      bulk_copy(Db0 + b * dsz, Dtab + (size_t)clsmap[2 * c] * dsz, dbytes, &mbD[b]);
    }
    ++nd_issued[b];
  };
  auto issue_C = [&](int q) {
    if (threadIdx.x == 0) {
      const int c = cls_of(q);
      mbar_expect(&mbC, cbytes);
      bulk_copy(Cb, Ctab + (size_t)clsmap[2 * c + 1] * csz, cbytes, &mbC);
    }
    ++nc_issued;
  };
  auto wait_D = [&](int b) {
    if (!mbar_wait(&mbD[b], nd_done[b] & 1)) return 1;
    ++nd_done[b];
    return 0;
  };
  auto wait_C = [&]() {
    if (!mbar_wait(&mbC, nc_done & 1)) return 1;
    ++nc_done;
    return 0;
  };
  // after a copy that did not arrive: report, then wait (bounded) for the copies
  // still in flight so that none outlives the CTA
  auto drain = [&]() {
    if (threadIdx.x == 0) report(err, QBX_DEVERR_COPY_TIMEOUT);
#pragma unroll
    for (int b = 0; b < ND; ++b)
      for (; nd_done[b] < nd_issued[b]; ++nd_done[b]) mbar_wait(&mbD[b], nd_done[b] & 1);
    for (; nc_done < nc_issued; ++nc_done) mbar_wait(&mbC, nc_done & 1);
  };

  double2 acc[KMAX][4];
#pragma unroll
  for (int k = 0; k < KMAX; ++k)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[k][j] = c2(0.0);

  issue_D(q0, 0);
  issue_C(q0);
  for (int q = q0; q < q1; ++q) {
    const int buf = ND == 2 ? ((q - q0) & 1) : 0;
    const double* Db = Db0 + buf * dsz;
    const int src = g.m2l_pair_src[g.m2l_tgt_pairs[q]];
    const bool bad = (unsigned)src >= (unsigned)g.nboxes;
    if (bad && threadIdx.x == 0) report(err, QBX_DEVERR_BAD_BOX);
    int fail = wait_D(buf);
    // the other buffer was last read by pair q - 1, before the barrier that ended it
    if (ND == 2 && q + 1 < q1) issue_D(q + 1, buf ^ 1);
    const double2* ph = reinterpret_cast<const double2*>(Db);
    const double* blocks = Db + 2 * nm;
    // X = e^{i m alpha} M
    for (int e = threadIdx.x; e < RB * ncf; e += NTHR) {
      const int r = e / ncf, ci = e - r * ncf;
      const int n = s_nof[ci];
      double2 v = c2(0.0);
      if (!fail && !bad && r0 + r < nrhs)
        v = cmul(ph[ci - n * n - n + pf], mp[((size_t)src * nrhs + r0 + r) * ncf + ci]);
      X[r * XS + ci] = v;
    }
    if (__syncthreads_or(fail)) {
      drain();
      return;
    }
    // A[(n, mu)] = sum_m T^n[m][mu] X[(n, m)]
    for (int t = threadIdx.x; t < ng * RB; t += NTHR) {
      const int grp = t / RB, r = t - grp * RB;
      const int n = s_gn[grp], mu0 = s_gm0[grp];
      const double* Tn = blocks + h3_dblock(n);
      const int w = 2 * n + 1, nv = min(4, n - mu0 + 1);
      double2 o[4] = {c2(0.0), c2(0.0), c2(0.0), c2(0.0)};
      const double2* Xr = X + r * XS + n * n;
      for (int m = 0; m < w; ++m) {
        const double2 x = Xr[m];
        const int ma = m - n;
        const double* row = ma >= 0 ? Tn + ma * w + (mu0 + n) : Tn + (-ma) * w + (n - mu0);
        const int step = ma >= 0 ? 1 : -1;
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (j < nv) o[j] = caxpy(row[step * j], x, o[j]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (j < nv) A[r * XS + n * n + n + mu0 + j] = o[j];
    }
    fail = wait_C();
    if (__syncthreads_or(fail)) {
      drain();
      return;
    }
    // B[(nu, mu)] = sum_{n >= |mu|} C^mu[n][nu] A[(n, mu)]   (into X)
    for (int t = threadIdx.x; t < ncg * RB; t += NTHR) {
      const int grp = t / RB, r = t - grp * RB;
      const int mu = s_cmu[grp], nu0 = s_cnu0[grp];
      const int am = abs(mu), w = pf + 1 - am, nv = min(4, pf - nu0 + 1);
      const double2* Cq = Cb + h3_cblock(pf, am) + (nu0 - am);
      double2 o[4] = {c2(0.0), c2(0.0), c2(0.0), c2(0.0)};
      const double2* Ar = A + r * XS;
      for (int n = am; n <= pf; ++n) {
        const double2 a = Ar[n * n + n + mu];
        const double2* row = Cq + (n - am) * w;
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (j < nv) o[j] = cfma(row[j], a, o[j]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int nu = nu0 + j;
        if (j < nv) X[r * XS + nu * nu + nu + mu] = o[j];
      }
    }
    __syncthreads();
    // the coaxial buffer is free: the next pair's table lands during the back rotation
    if (q + 1 < q1) issue_C(q + 1);
    // L[(nu, m2)] += e^{-i m2 alpha} sum_mu T^nu[m2][mu] B[(nu, mu)]
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
      const int t = threadIdx.x + k * NTHR;
      if (t >= ng * RB) break;
      const int grp = t / RB, r = t - grp * RB;
      const int nu = s_gn[grp], m20 = s_gm0[grp];
      const int w = 2 * nu + 1, nv = min(4, nu - m20 + 1);
      const double* Tn = blocks + h3_dblock(nu);
      const double* pj[4];
      int sj[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int m2 = m20 + j;
        pj[j] = m2 >= 0 ? Tn + m2 * w : Tn + (-m2) * w + 2 * nu;
        sj[j] = m2 >= 0 ? 1 : -1;
      }
      double2 o[4] = {c2(0.0), c2(0.0), c2(0.0), c2(0.0)};
      const double2* Br = X + r * XS + nu * nu;
      for (int mu = 0; mu < w; ++mu) {
        const double2 bb = Br[mu];
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (j < nv) o[j] = caxpy(pj[j][sj[j] * mu], bb, o[j]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (j < nv) acc[k][j] = cfma(cconj(ph[m20 + j + pf]), o[j], acc[k][j]);
    }
    __syncthreads();
    // the rotation buffer is free
    if (ND == 1 && q + 1 < q1) issue_D(q + 1, 0);
  }
  const int tb = g.target_or_target_parent_boxes[i];
  if ((unsigned)tb >= (unsigned)g.nboxes) {
    if (threadIdx.x == 0) report(err, QBX_DEVERR_BAD_BOX);
    return;
  }
#pragma unroll
  for (int k = 0; k < KMAX; ++k) {
    const int t = threadIdx.x + k * NTHR;
    if (t >= ng * RB) break;
    const int grp = t / RB, r = t - grp * RB;
    if (r0 + r >= nrhs) continue;
    const int nu = s_gn[grp], m20 = s_gm0[grp];
    const int nv = min(4, nu - m20 + 1);
    double2* out = lo + ((size_t)tb * nrhs + r0 + r) * ncf + nu * nu + nu + m20;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (j < nv) out[j] = cadd(out[j], acc[k][j]);
  }
}

// }}}

// dynamic shared memory of k_h3_m2l_bulk: the X and A blocks, nd rotation tables,
// the coaxial table
static size_t h3_m2l_bulk_smem(int rb, int pf, int nd)
{
  return 2 * (size_t)rb * ((pf + 1) * (pf + 1) + 1) * sizeof(double2) +
         nd * h3_m2l_dsize(pf) * sizeof(double) + h3_m2l_csize(pf) * sizeof(double2);
}

// dynamic shared memory a CTA may use beside the kernels' static arrays (227 KB less
// a margin for them)
constexpr size_t H3M2L_SMEM_MAX = 227 * 1024 - 4 * 1024;

template <int RB, int NTHR = H3M2L_NT, int ND = 1>
static cudaError_t h3_m2l_bulk_launch(const qbxfmm_geometry& g, int pf, int nrhs, const double2* mp,
                                      double2* lo, const double* Dtab, const double2* Ctab,
                                      const double* clsmap, int32_t* err, cudaStream_t st)
{
  // bulk copies need 16-byte aligned tables
  if ((reinterpret_cast<uintptr_t>(Dtab) | reinterpret_cast<uintptr_t>(Ctab)) & 15)
    return cudaErrorInvalidValue;
  const size_t sh = h3_m2l_bulk_smem(RB, pf, ND);
  if (sh > H3M2L_SMEM_MAX) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_h3_m2l_bulk<RB, NTHR, ND>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return e;
  dim3 grid(g.nttp_boxes, (nrhs + RB - 1) / RB);
  k_h3_m2l_bulk<RB, NTHR, ND><<<grid, NTHR, sh, st>>>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err);
  return cudaGetLastError();
}

// 16 densities per CTA (512 threads, one CTA per SM): two rotation-table buffers where
// they fit, else one, else 8 densities per CTA
static cudaError_t h3_m2l_bulk16(const qbxfmm_geometry& g, int pf, int nrhs, const double2* mp,
                                 double2* lo, const double* Dtab, const double2* Ctab,
                                 const double* clsmap, int32_t* err, cudaStream_t st)
{
  if (h3_m2l_bulk_smem(16, pf, 2) <= H3M2L_SMEM_MAX)
    return h3_m2l_bulk_launch<16, 2 * H3M2L_NT, 2>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
  if (h3_m2l_bulk_smem(16, pf, 1) <= H3M2L_SMEM_MAX)
    return h3_m2l_bulk_launch<16, 2 * H3M2L_NT, 1>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
  return h3_m2l_bulk_launch<8>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
}

template <typename R, int RB>
static cudaError_t h3_m2l_rot_launch(const qbxfmm_geometry& g, int pf, int nrhs, const double2* mp,
                                     double2* lo, const double* Dtab, const double2* Ctab,
                                     const double* clsmap, int32_t* err, cudaStream_t st)
{
  using V = cplx_t<R>;
  size_t sh = (2 * (size_t)RB * ((pf + 1) * (pf + 1) + 1) +
               std::max(h3_m2l_dsize(pf) / 2, h3_m2l_csize(pf))) * sizeof(V);
  cudaFuncSetAttribute(k_h3_m2l_rot<R, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  dim3 grid(g.nttp_boxes, (nrhs + RB - 1) / RB);
  k_h3_m2l_rot<R, RB><<<grid, H3M2L_NT, sh, st>>>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err);
  return cudaGetLastError();
}

cudaError_t h3_launch_m2l_rot(const qbxfmm_geometry& g, int pf, int nrhs, const double2* mp,
                              double2* lo, const double* Dtab, const double2* Ctab,
                              const double* clsmap, int32_t* err, cudaStream_t st, bool fp32,
                              int rb)
{
  if (g.nttp_boxes == 0 || g.m2l_nclasses == 0) return cudaSuccess;
  if (pf > H3_MAXP) return cudaErrorInvalidValue;
  switch (rb) {   // the plan's tuning
    case 1:
      return fp32 ? h3_m2l_rot_launch<float, 1>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st)
                  : h3_m2l_rot_launch<double, 1>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
    case 4:
      return fp32 ? h3_m2l_rot_launch<float, 4>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st)
                  : h3_m2l_rot_launch<double, 4>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
    case 8:
      return fp32 ? h3_m2l_rot_launch<float, 8>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st)
                  : h3_m2l_bulk_launch<8>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
    case 16:
      if (fp32) return h3_m2l_rot_launch<float, 16>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
      return h3_m2l_bulk16(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
    default: break;
  }
  if (fp32) {   // mixed form: FP32 arithmetic, all 16 densities of a pair's tables at once
    if (nrhs >= 16) return h3_m2l_rot_launch<float, 16>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
    if (nrhs >= 8) return h3_m2l_rot_launch<float, 8>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
    return h3_m2l_rot_launch<float, 4>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
  }
  // 16 densities per CTA (512 threads) when there are as many: at the 3D Helmholtz
  // benchmark size the autotuner measured 158 ms against 162 ms for 8
  if (nrhs >= 16) return h3_m2l_bulk16(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
  if (nrhs >= 8) return h3_m2l_bulk_launch<8>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
  if (nrhs >= 2) return h3_m2l_rot_launch<double, 4>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
  return h3_m2l_rot_launch<double, 1>(g, pf, nrhs, mp, lo, Dtab, Ctab, clsmap, err, st);
}

cudaError_t h3_launch_m2l_tables(int pf, int ndir, int ncoax, const double* dirs,
                                 const double* coaxp, const double* start, const double* isq,
                                 const double* rt, const double* gaunt, double* Dtab,
                                 double2* Ctab, cudaStream_t st)
{
  if (ndir + ncoax == 0) return cudaSuccess;
  if (pf > H3_MAXP) return cudaErrorInvalidValue;
  k_h3_m2l_tables<<<ndir + ncoax, NT, 0, st>>>(pf, ndir, ncoax, dirs, coaxp, start, isq, rt, gaunt,
                                               Dtab, Ctab);
  return cudaGetLastError();
}

// }}}

// {{{ launchers

static int gridy(int nrhs) { return nrhs; }

// densities per CTA: 8, 4 or 1
template <bool LOCAL>
static cudaError_t h3_p2e_launch(int nbox, size_t sh, const qbxfmm_geometry& g, HelmCoeffs hc, int p,
                                 int nrhs, const double2* s, double2* e, int32_t* err,
                                 cudaStream_t st)
{
#define QBX_H3_P2E(RB)                                                                          \
  {                                                                                             \
    cudaFuncSetAttribute(k_h3_p2e<LOCAL, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize,      \
                         (int)sh);                                                              \
    k_h3_p2e<LOCAL, RB><<<dim3(nbox, (nrhs + RB - 1) / RB), NT, sh, st>>>(g, hc, p, nrhs, s, e, \
                                                                          err);                 \
    return cudaGetLastError();                                                                  \
  }
  // 16 densities: 256 threads, one coefficient each
  const bool wide = (p + 1) * (p + 1) <= 2 * NT;
  if (hc.rb_p2e == 16 || (hc.rb_p2e == 0 && nrhs > 8 && wide)) {
    if (!wide) return cudaErrorInvalidValue;
    cudaFuncSetAttribute(k_h3_p2e<LOCAL, 16, 2 * NT, 1>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    k_h3_p2e<LOCAL, 16, 2 * NT, 1><<<dim3(nbox, (nrhs + 15) / 16), 2 * NT, sh, st>>>(
        g, hc, p, nrhs, s, e, err);
    return cudaGetLastError();
  }
  if (hc.rb_p2e == 8) QBX_H3_P2E(8)   // the plan's tuning
  if (hc.rb_p2e == 4) QBX_H3_P2E(4)
  if (hc.rb_p2e == 1) QBX_H3_P2E(1)
  if (nrhs >= 8) QBX_H3_P2E(8)
  if (nrhs >= 3) QBX_H3_P2E(4)
  QBX_H3_P2E(1)
#undef QBX_H3_P2E
}

cudaError_t h3_launch_p2m(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                          const double2* s, double2* mp, cudaStream_t st)
{
  if (g.nsource_boxes == 0) return cudaSuccess;
  int N = p + 1;
  size_t sh = ((size_t)(N + 1) * (N + 1) * H3_TS + (size_t)(N + 1) * (N + 2) / 2) * sizeof(double2);
  if (hc.taylor && (hc.cd.x != 0.0 || hc.cd.y != 0.0))   // second (dipole) table
    sh += ((size_t)(N + 1) * (N + 1) * H3_TS + (size_t)H3_SUB * (N + 2)) * sizeof(double2);
  return h3_p2e_launch<false>(g.nsource_boxes, sh, g, hc, p, nrhs, s, mp, nullptr, st);
}

cudaError_t h3_launch_p2l(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                          const double2* s, double2* lo, int32_t* err, cudaStream_t st)
{
  if (g.nttp_boxes == 0) return cudaSuccess;
  int N = p + 1;
  size_t sh = ((size_t)(N + 1) * (N + 1) * H3_TS + (size_t)(N + 1) * (N + 2) / 2) * sizeof(double2);
  return h3_p2e_launch<true>(g.nttp_boxes, sh, g, hc, p, nrhs, s, lo, err, st);
}

cudaError_t h3_launch_eval_direct(const qbxfmm_geometry& g, HelmCoeffs hc, int nrhs,
                                  const double2* s, double2* pot, int32_t* err, cudaStream_t st)
{
  if (g.nnonqbx_chunks == 0) return cudaSuccess;
  k_h3_eval_direct<<<dim3(g.nnonqbx_chunks * H3_PSPLIT, gridy(nrhs)), NT, 0, st>>>(g, hc, nrhs, s,
                                                                                  pot, err);
  return cudaGetLastError();
}

cudaError_t h3_launch_eval_multipoles(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                                      const double2* mp, double2* pot, int32_t* err, cudaStream_t st)
{
  if (g.nnonqbx_chunks == 0) return cudaSuccess;
  size_t sh = ((size_t)(p + 1) * (p + 2) / 2 + (size_t)NW * (p + 1) * (p + 1)) * sizeof(double2);
  cudaFuncSetAttribute(k_h3_eval_multipoles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  k_h3_eval_multipoles<<<dim3(g.nnonqbx_chunks, gridy(nrhs)), NT, sh, st>>>(g, hc, p, nrhs, mp, pot,
                                                                            err);
  return cudaGetLastError();
}

cudaError_t h3_launch_eval_locals(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                                  const double2* lo, double2* pot, cudaStream_t st)
{
  if (g.nnonqbx_chunks == 0) return cudaSuccess;
  size_t sh = (size_t)(p + 1) * (p + 2) / 2 * sizeof(double2);
  k_h3_eval_locals<<<dim3(g.nnonqbx_chunks, gridy(nrhs)), NT, sh, st>>>(g, hc, p, nrhs, lo, pot);
  return cudaGetLastError();
}

template <int Q>
static cudaError_t h3_p2qbxl_q(const qbxfmm_geometry& g, HelmCoeffs hc, int nrhs, const double2* s,
                               double2* qe, int32_t* err, cudaStream_t st)
{
  constexpr int N = Q + 1;
  size_t sh = (size_t)NW * (N + 1) * (N + 1) * 32 * sizeof(double2);
  size_t red = (size_t)(NW - 1) * 32 * (Q + 1) * (Q + 1) * sizeof(double2);
  sh = std::max(sh, red);
  cudaFuncSetAttribute(k_h3_p2qbxl<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  k_h3_p2qbxl<Q><<<dim3(g.nqbx_chunks, gridy(nrhs)), NT, sh, st>>>(g, hc, nrhs, s, qe, err);
  return cudaGetLastError();
}

cudaError_t h3_launch_p2qbxl(const qbxfmm_geometry& g, HelmCoeffs hc, int q, int nrhs,
                             const double2* s, double2* qe, int32_t* err, cudaStream_t st)
{
  if (g.nqbx_chunks == 0) return cudaSuccess;
  switch (q) {
    case 0: return h3_p2qbxl_q<0>(g, hc, nrhs, s, qe, err, st);
    case 1: return h3_p2qbxl_q<1>(g, hc, nrhs, s, qe, err, st);
    case 2: return h3_p2qbxl_q<2>(g, hc, nrhs, s, qe, err, st);
    case 3: return h3_p2qbxl_q<3>(g, hc, nrhs, s, qe, err, st);
    case 4: return h3_p2qbxl_q<4>(g, hc, nrhs, s, qe, err, st);
    case 5: return h3_p2qbxl_q<5>(g, hc, nrhs, s, qe, err, st);
    default: return cudaErrorInvalidValue;
  }
}

template <int Q, int RB>
static cudaError_t h3_tsqbx_qr(const qbxfmm_geometry& g, HelmCoeffs hc, int nrhs, const double2* s,
                               double2* pt, int32_t* err, cudaStream_t st)
{
  size_t sh = (size_t)(NW - 1) * 32 * RB * sizeof(double2);
  dim3 grid(g.ntsqbx_chunks, (nrhs + RB - 1) / RB);
  cudaFuncSetAttribute(k_h3_tsqbx<Q, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  k_h3_tsqbx<Q, RB><<<grid, NT, sh, st>>>(g, hc, nrhs, s, pt, err);
  return cudaGetLastError();
}

template <int Q>
static cudaError_t h3_tsqbx_q(const qbxfmm_geometry& g, HelmCoeffs hc, int nrhs, const double2* s,
                              double2* pt, int32_t* err, cudaStream_t st)
{
  switch (hc.rb_ts) {   // the plan's tuning
    case 1: return h3_tsqbx_qr<Q, 1>(g, hc, nrhs, s, pt, err, st);
    case 4: return h3_tsqbx_qr<Q, 4>(g, hc, nrhs, s, pt, err, st);
    case 16: return h3_tsqbx_qr<Q, 16>(g, hc, nrhs, s, pt, err, st);
    default: break;
  }
  if (nrhs == 1) return h3_tsqbx_qr<Q, 1>(g, hc, nrhs, s, pt, err, st);
  if (nrhs <= 4) return h3_tsqbx_qr<Q, 4>(g, hc, nrhs, s, pt, err, st);
  return h3_tsqbx_qr<Q, 16>(g, hc, nrhs, s, pt, err, st);
}

cudaError_t h3_launch_tsqbx(const qbxfmm_geometry& g, HelmCoeffs hc, int q, int nrhs,
                            const double2* s, double2* pt, int32_t* err, cudaStream_t st)
{
  if (g.ntsqbx_chunks == 0) return cudaSuccess;
  switch (q) {
    case 0: return h3_tsqbx_q<0>(g, hc, nrhs, s, pt, err, st);
    case 1: return h3_tsqbx_q<1>(g, hc, nrhs, s, pt, err, st);
    case 2: return h3_tsqbx_q<2>(g, hc, nrhs, s, pt, err, st);
    case 3: return h3_tsqbx_q<3>(g, hc, nrhs, s, pt, err, st);
    case 4: return h3_tsqbx_q<4>(g, hc, nrhs, s, pt, err, st);
    case 5: return h3_tsqbx_q<5>(g, hc, nrhs, s, pt, err, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename R, bool FROM_LOCAL, int Q, int RB>
static size_t h3_rot_smem(int pf)
{
  constexpr int NCQ = (Q + 1) * (Q + 1), NMU = 2 * Q + 1;
  int ncf = (pf + 1) * (pf + 1), L = pf + Q, nl = pf + 1, nm = 2 * pf + 1;
  size_t nisq = (size_t)(pf + 2) * (pf + 1), nrt = (size_t)(pf + 1) * (pf + 1);
  size_t ctad = (nisq + nrt + nl + 1) & ~(size_t)1;
  size_t perd = ((size_t)NMU * NCQ + 2 * (size_t)nm + 1) / 2;
  size_t per = (size_t)nm * NMU + NCQ + (size_t)NCQ * RB + (L + 2) + nm + perd;
  return ((size_t)ncf * RB + NW * per) * sizeof(cplx_t<R>) + ctad * sizeof(R);
}

template <int Q>
static size_t h3_pair_smem(int pf)
{
  constexpr int NCQ = (Q + 1) * (Q + 1), NMU = 2 * Q + 1;
  const size_t ncf = (size_t)(pf + 1) * (pf + 1), L = pf + Q, nl = pf + 1, nm = 2 * pf + 1;
  const size_t nisq = (size_t)(pf + 2) * (pf + 1), nrt = (size_t)(pf + 1) * (pf + 1);
  const size_t ctad = (nisq + nrt + nl + 1) & ~(size_t)1;
  const size_t nsl = std::max((size_t)nm * NMU, (size_t)2 * NCQ * 8);
  const size_t per = nsl + 2 * NCQ + (L + 2) + nm + ((size_t)NMU * NCQ + 2 * nm + 1) / 2;
  return (ncf * 16 + 2 * per) * sizeof(double2) + ctad * sizeof(double);
}

template <int Q>
static cudaError_t h3_pair_launch(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int nrhs,
                                  const double2* e, const double* rot, double2* qe, int32_t* err,
                                  cudaStream_t st)
{
  if ((2 * pf + 1) * (Q + 1) > 2 * H3P_SLOTS * 32) return cudaErrorInvalidValue;
  size_t sh = h3_pair_smem<Q>(pf);
  cudaFuncSetAttribute(k_h3_m2qbxl_pair<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  dim3 grid(g.nqbx_chunks, (nrhs + 15) / 16, (H3_ROT_ZS * NW) / 2);
  k_h3_m2qbxl_pair<Q><<<grid, NT, sh, st>>>(g, hc, pf, nrhs, e, rot, qe, err);
  return cudaGetLastError();
}

template <typename R, bool FROM_LOCAL, int Q, int RB>
static cudaError_t h3_rot_launch(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int nrhs,
                                 const double2* e, const double* rot, double2* qe, int32_t* err,
                                 cudaStream_t st)
{
  size_t sh = h3_rot_smem<R, FROM_LOCAL, Q, RB>(pf);
  cudaFuncSetAttribute(k_h3_e2qbxl_rot<R, FROM_LOCAL, Q, RB>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  dim3 grid(g.nqbx_chunks, (nrhs + RB - 1) / RB, H3_ROT_ZS);
  k_h3_e2qbxl_rot<R, FROM_LOCAL, Q, RB><<<grid, NT, sh, st>>>(g, hc, pf, nrhs, e, rot, qe, err);
  return cudaGetLastError();
}

// densities per CTA: FP64 M2QBXL with more than 8 densities, the two-warps-per-center
// kernel (16 densities share each pair's tables); otherwise FP64, 8 when two CTAs
// still fit an SM's shared memory, else 4, else 1; FP32 (the mixed form), all 16 of a
// 16-density job in one CTA so that the per-pair rotation tables serve every density
template <typename R, bool FROM_LOCAL, int Q>
static cudaError_t h3_rot_q(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int nrhs,
                            const double2* e, const double* rot, double2* qe, int32_t* err,
                            cudaStream_t st)
{
  constexpr bool PAIR = std::is_same<R, double>::value && !FROM_LOCAL;
  switch (hc.rb_rot) {   // the plan's tuning
    case 1: return h3_rot_launch<R, FROM_LOCAL, Q, 1>(g, hc, pf, nrhs, e, rot, qe, err, st);
    case 4: return h3_rot_launch<R, FROM_LOCAL, Q, 4>(g, hc, pf, nrhs, e, rot, qe, err, st);
    case 8: return h3_rot_launch<R, FROM_LOCAL, Q, 8>(g, hc, pf, nrhs, e, rot, qe, err, st);
    case 16:
      if constexpr (!std::is_same<R, double>::value)
        return h3_rot_launch<R, FROM_LOCAL, Q, 16>(g, hc, pf, nrhs, e, rot, qe, err, st);
      else if constexpr (PAIR)
        return h3_pair_launch<Q>(g, hc, pf, nrhs, e, rot, qe, err, st);
      return cudaErrorInvalidValue;
    default: break;
  }
  const size_t two_per_sm = 112 * 1024;
  if constexpr (!std::is_same<R, double>::value)
    if (nrhs >= 16 && h3_rot_smem<R, FROM_LOCAL, Q, 16>(pf) <= two_per_sm)
      return h3_rot_launch<R, FROM_LOCAL, Q, 16>(g, hc, pf, nrhs, e, rot, qe, err, st);
  if constexpr (PAIR)
    if (nrhs > 8 && h3_pair_smem<Q>(pf) <= two_per_sm &&
        (2 * pf + 1) * (Q + 1) <= 2 * H3P_SLOTS * 32)
      return h3_pair_launch<Q>(g, hc, pf, nrhs, e, rot, qe, err, st);
  if (nrhs >= 8 && h3_rot_smem<R, FROM_LOCAL, Q, 8>(pf) <= two_per_sm)
    return h3_rot_launch<R, FROM_LOCAL, Q, 8>(g, hc, pf, nrhs, e, rot, qe, err, st);
  if (nrhs >= 4)
    return h3_rot_launch<R, FROM_LOCAL, Q, 4>(g, hc, pf, nrhs, e, rot, qe, err, st);
  return h3_rot_launch<R, FROM_LOCAL, Q, 1>(g, hc, pf, nrhs, e, rot, qe, err, st);
}

template <typename R, bool FROM_LOCAL>
static cudaError_t h3_e2qbxl(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int q, int nrhs,
                             const double2* e, const double* rot, double2* qe, int32_t* err,
                             cudaStream_t st)
{
  if (g.nqbx_chunks == 0) return cudaSuccess;
  if (2 * pf + 1 > 35) return cudaErrorInvalidValue;   // recurrence slots per lane
  switch (q) {
    case 0: return h3_rot_q<R, FROM_LOCAL, 0>(g, hc, pf, nrhs, e, rot, qe, err, st);
    case 1: return h3_rot_q<R, FROM_LOCAL, 1>(g, hc, pf, nrhs, e, rot, qe, err, st);
    case 2: return h3_rot_q<R, FROM_LOCAL, 2>(g, hc, pf, nrhs, e, rot, qe, err, st);
    case 3: return h3_rot_q<R, FROM_LOCAL, 3>(g, hc, pf, nrhs, e, rot, qe, err, st);
    case 4: return h3_rot_q<R, FROM_LOCAL, 4>(g, hc, pf, nrhs, e, rot, qe, err, st);
    case 5: return h3_rot_q<R, FROM_LOCAL, 5>(g, hc, pf, nrhs, e, rot, qe, err, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t h3_launch_m2qbxl(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int q, int nrhs,
                             const double2* mp, const double* rot, double2* qe, int32_t* err,
                             cudaStream_t st, bool fp32)
{
  if (fp32) return h3_e2qbxl<float, false>(g, hc, pf, q, nrhs, mp, rot, qe, err, st);
  return h3_e2qbxl<double, false>(g, hc, pf, q, nrhs, mp, rot, qe, err, st);
}

cudaError_t h3_launch_l2qbxl(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int q, int nrhs,
                             const double2* lo, const double* rot, double2* qe, int32_t* err,
                             cudaStream_t st)
{
  return h3_e2qbxl<double, true>(g, hc, pf, q, nrhs, lo, rot, qe, err, st);
}

cudaError_t h3_launch_qbxl2p(const qbxfmm_geometry& g, HelmCoeffs hc, int q, int nrhs,
                             const double2* qe, double2* pt, cudaStream_t st)
{
  if (g.nglobal_qbx_centers == 0) return cudaSuccess;
  size_t sh = (size_t)(q + 1) * (q + 2) / 2 * sizeof(double2);
  k_h3_qbxl2p<<<dim3((g.nglobal_qbx_centers + NT - 1) / NT, gridy(nrhs)), NT, sh, st>>>(g, hc, q, nrhs,
                                                                                       qe, pt);
  return cudaGetLastError();
}

cudaError_t h3_launch_assemble(const qbxfmm_geometry& g, int nrhs, const double2* pot_nonqbx,
                               const double2* pot_tree, double2* out, cudaStream_t st)
{
  if (g.ntargets > 0) {
    k_h3_assemble_tree<<<dim3((g.ntargets + 255) / 256, nrhs), 256, 0, st>>>(g, nrhs, pot_tree, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (g.nfiltered_targets > 0)
    k_h3_assemble_nonqbx<<<dim3((g.nfiltered_targets + 255) / 256, nrhs), 256, 0, st>>>(
        g, nrhs, pot_nonqbx, out);
  return cudaGetLastError();
}

cudaError_t h3_launch_trans_build(const qbxfmm_geometry& g, const TransCfg& tc, double k,
                                  const double* gaunt, double* T, cudaStream_t st)
{
  int p = tc.p, L = 2 * p;
  size_t sh = ((size_t)(L + 1) * (L + 2) / 2 + (size_t)(L + 1) * (L + 1) + (L + 2)) * sizeof(double2) +
              2 * (size_t)(p + 1) * sizeof(double);
  cudaFuncSetAttribute(k_h3_trans_build, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  size_t stride = (size_t)tc.rp * tc.kp;
  // M2M: parent levels 0 .. nlevels-2; L2L: child levels 1 .. nlevels-1 (8 per level)
  if (g.nlevels > 1) {
    k_h3_trans_build<<<8 * (g.nlevels - 1), NT, sh, st>>>(1, p, tc.rp, tc.kp, k, g.root_extent, 0,
                                                          gaunt, T + tc.m2m_base * stride);
    k_h3_trans_build<<<8 * (g.nlevels - 1), NT, sh, st>>>(2, p, tc.rp, tc.kp, k, g.root_extent, 1,
                                                          gaunt, T + (tc.l2l_base + 8) * stride);
  }
  return cudaGetLastError();
}

// }}}

}  // namespace qbx

// {{{ dense QBX matrix

namespace qbx {
int set_last_error(int code, const std::string& msg);

namespace {

// Entry (t, s) of the 3D Helmholtz layer potential with charge / dipole weights:
//   QBX targets (center c): the target-specific series of k_h3_tsqbx,
//     ik sum_{n<=Q} (2n+1) j_n(k|a|) [cq h_n(k|b|) P_n(cos g) + cd (dipole terms)]
//     (j_n cut to its degree-Q power series in the reference's default truncation),
//   other targets: cq e^{ikr}/r + cd nu.(t - s) e^{ikr} (1 - ikr) / r^3;
// times 1/(4 pi).  CTA = 128 sources (thread = source) x 32 targets.
constexpr int H3D_DS = 128;
constexpr int H3D_DTG = 32;

template <int Q>
__global__ void __launch_bounds__(H3D_DS)
k_h3_qbx_matrix(int nsrc, const double* __restrict__ src, const double* __restrict__ nrm,
                HelmCoeffs hc, int ntgt, const double* __restrict__ tgt,
                const int32_t* __restrict__ tcenter, int ncenters,
                const double* __restrict__ centers, double2* __restrict__ K)
{
  __shared__ double s_x[3][H3D_DTG], s_c[3][H3D_DTG], s_ah[3][H3D_DTG];
  __shared__ double s_jn[H3D_DTG][Q + 1];
  __shared__ int s_qbx[H3D_DTG];
  const int t0 = blockIdx.y * H3D_DTG;
  if (threadIdx.x < H3D_DTG) {
    const int i = threadIdx.x, t = t0 + i;
    int c = t < ntgt ? tcenter[t] : -1;
    if (c >= ncenters) c = -1;
    double x[3] = {0, 0, 0}, cc[3] = {0, 0, 0};
    if (t < ntgt)
      for (int d = 0; d < 3; ++d) x[d] = tgt[(size_t)d * ntgt + t];
    if (c >= 0)
      for (int d = 0; d < 3; ++d) cc[d] = centers[(size_t)d * ncenters + c];
    double a[3] = {x[0] - cc[0], x[1] - cc[1], x[2] - cc[2]};
    double alen = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    double ainv = alen > 0.0 ? 1.0 / alen : 0.0;
    for (int d = 0; d < 3; ++d) {
      s_x[d][i] = x[d];
      s_c[d][i] = cc[d];
      s_ah[d][i] = a[d] * ainv;
    }
    s_qbx[i] = c >= 0;
    double jv[H3_LMAX + 2];
    h3_sph_j_cut(Q, hc.k * alen, hc.taylor ? Q : -1, jv);
#pragma unroll
    for (int n = 0; n <= Q; ++n) s_jn[i][n] = (2.0 * n + 1.0) * jv[n];
  }
  __syncthreads();
  const int s = blockIdx.x * H3D_DS + threadIdx.x;
  if (s >= nsrc) return;
  const double y[3] = {src[s], src[(size_t)nsrc + s], src[2 * (size_t)nsrc + s]};
  const bool chg = hc.cq.x != 0.0 || hc.cq.y != 0.0;
  const bool dip = hc.cd.x != 0.0 || hc.cd.y != 0.0;
  double nv[3] = {0, 0, 0};
  if (dip)
    for (int d = 0; d < 3; ++d) nv[d] = nrm[(size_t)d * nsrc + s];
  const double2 kq = c2(-hc.k * hc.cq.y, hc.k * hc.cq.x), kd = c2(-hc.k * hc.cd.y, hc.k * hc.cd.x);
  const int tend = min(H3D_DTG, ntgt - t0);
  for (int i = 0; i < tend; ++i) {
    double2 v = c2(0.0);
    if (s_qbx[i]) {
      double b0 = y[0] - s_c[0][i], b1 = y[1] - s_c[1][i], b2 = y[2] - s_c[2][i];
      double b2s = b0 * b0 + b1 * b1 + b2 * b2;
      if (b2s != 0.0) {
        double binv = rsqrt(b2s);
        double blen = b2s * binv;
        double cg = (s_ah[0][i] * b0 + s_ah[1][i] * b1 + s_ah[2][i] * b2) * binv;
        double2 h[Q + 2];
        h3_sph_h(Q + 1, hc.k * blen, h);
        double xinv = 1.0 / (hc.k * blen);
        double pm1 = 1.0, pm2 = 0.0, dm1 = 0.0;
        double2 sS = c2(0.0), sA = c2(0.0), sB = c2(0.0);
        const double* jn = s_jn[i];
#pragma unroll
        for (int n = 0; n <= Q; ++n) {
          double pn, dn;
          if (n == 0) {
            pn = 1.0;
            dn = 0.0;
          } else if (n == 1) {
            pn = cg;
            dn = 1.0;
          } else {
            pn = ((2.0 * n - 1) * cg * pm1 - (n - 1.0) * pm2) * (1.0 / n);
            dn = n * pm1 + cg * dm1;
          }
          if (chg) sS = caxpy(jn[n] * pn, h[n], sS);
          if (dip) {
            double2 hd = (n == 0) ? c2(-h[1].x, -h[1].y) : caxpy(-(n + 1.0) * xinv, h[n], h[n - 1]);
            sA = caxpy(jn[n] * pn * hc.k, hd, sA);
            sB = caxpy(jn[n] * dn, h[n], sB);
          }
          pm2 = pm1;
          pm1 = pn;
          dm1 = dn;
        }
        if (chg) v = cmul(kq, sS);
        if (dip) {
          double db = (nv[0] * b0 + nv[1] * b1 + nv[2] * b2) * binv;
          double da = nv[0] * s_ah[0][i] + nv[1] * s_ah[1][i] + nv[2] * s_ah[2][i];
          double2 vd = caxpy(db, sA, cscale((da - cg * db) * binv, sB));
          v = cfma(kd, vd, v);
        }
      }
    } else {
      double dx = s_x[0][i] - y[0], dy = s_x[1][i] - y[1], dz = s_x[2][i] - y[2];
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > 0.0) {
        double rinv = rsqrt(r2);
        double rr = r2 * rinv;
        double sn, cs;
        sincos(hc.k * rr, &sn, &cs);
        double2 e = c2(cs * rinv, sn * rinv);     // e^{ikr} / r
        v = cmul(hc.cq, e);
        if (dip) {
          double f = (nv[0] * dx + nv[1] * dy + nv[2] * dz) * rinv * rinv;
          v = cfma(hc.cd, cmul(e, c2(f, -f * hc.k * rr)), v);
        }
      }
    }
    K[(size_t)(t0 + i) * nsrc + s] = cscale(1.0 / FOUR_PI, v);
  }
}

template <int Q>
cudaError_t launch_h3_matrix(dim3 grid, cudaStream_t st, int nsrc, const double* src,
                             const double* nrm, HelmCoeffs hc, int ntgt, const double* tgt,
                             const int32_t* tc, int ncen, const double* cen, double2* K)
{
  k_h3_qbx_matrix<Q><<<grid, H3D_DS, 0, st>>>(nsrc, src, nrm, hc, ntgt, tgt, tc, ncen, cen, K);
  return cudaGetLastError();
}

}  // namespace
}  // namespace qbx

extern "C" int qbxfmm_helmholtz3d_qbx_matrix(int nsources, const double* sources,
                                             const double* normals, double k, double charge_re,
                                             double charge_im, double dipole_re,
                                             double dipole_im, int ntargets,
                                             const double* targets, const int32_t* target_center,
                                             int ncenters, const double* centers, int qbx_order,
                                             int fmm_backend, void* K, void* stream)
{
  using namespace qbx;
  if (nsources < 0 || ntargets < 0 || ncenters < 0)
    return set_last_error(QBXFMM_ERR_ARG, "negative size");
  if (fmm_backend != QBXFMM_BACKEND_SUMPY && fmm_backend != QBXFMM_BACKEND_FMMLIB)
    return set_last_error(QBXFMM_ERR_ARG, "fmm_backend must be QBXFMM_BACKEND_SUMPY or _FMMLIB");
  if (qbx_order < 0 || qbx_order > 8)
    return set_last_error(QBXFMM_ERR_UNSUPPORTED, "qbx_order must be in [0, 8]");
  if (!(k > 0.0)) return set_last_error(QBXFMM_ERR_ARG, "wave number must be positive");
  if (nsources == 0 || ntargets == 0) return QBXFMM_OK;
  const bool dip = dipole_re != 0.0 || dipole_im != 0.0;
  if (!sources || !targets || !target_center || !K || (ncenters > 0 && !centers) ||
      (dip && !normals))
    return set_last_error(QBXFMM_ERR_ARG, "null argument");
  dim3 grid((nsources + H3D_DS - 1) / H3D_DS, (ntargets + H3D_DTG - 1) / H3D_DTG);
  if (grid.y > 65535) return set_last_error(QBXFMM_ERR_UNSUPPORTED, "too many targets");
  HelmCoeffs hc;
  hc.k = k;
  hc.cq = c2(charge_re, charge_im);
  hc.cd = c2(dipole_re, dipole_im);
  hc.taylor = fmm_backend == QBXFMM_BACKEND_SUMPY;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  double2* Kd = static_cast<double2*>(K);
  cudaError_t e;
  switch (qbx_order) {
#define QBX_H3M_CASE(QQ) \
  case QQ: e = launch_h3_matrix<QQ>(grid, st, nsources, sources, normals, hc, ntargets, targets, \
                                     target_center, ncenters, centers, Kd); break;
    QBX_H3M_CASE(0) QBX_H3M_CASE(1) QBX_H3M_CASE(2) QBX_H3M_CASE(3) QBX_H3M_CASE(4)
    QBX_H3M_CASE(5) QBX_H3M_CASE(6) QBX_H3M_CASE(7) QBX_H3M_CASE(8)
#undef QBX_H3M_CASE
    default: return set_last_error(QBXFMM_ERR_UNSUPPORTED, "qbx_order");
  }
  if (e != cudaSuccess)
    return set_last_error(QBXFMM_ERR_CUDA, std::string("helmholtz3d_qbx_matrix: ") + cudaGetErrorString(e));
  return QBXFMM_OK;
}

// }}}
