// extern "C" entry points of libqbxfmm.so (declared in include/qbxfmm_api.h).
//
// Each stage entry mirrors one method of pytential's QBX expansion wrangler as
// called by the FMM driver (pytential/qbx/fmm.py:414-594); qbxfmm_apply runs them
// all in the driver's order.  Stage outputs are accumulated (+=) into caller-owned
// device buffers; the library allocates no device memory.
#include <algorithm>
#include <array>
#include <initializer_list>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <numeric>
#include <string>
#include <utility>
#include <vector>

#include "../../include/qbxfmm_api.h"
#include "kernels.h"
#include "taylor_h3.h"

using namespace qbx;

struct qbxfmm_plan {
  qbxfmm_kernel kern;
  qbxfmm_geometry geo;
  std::vector<int32_t> lvl_source_parent;  // host copy of level_start_source_parent_box_nrs
  std::vector<int32_t> lvl_ttp;            // host copy of level_start_ttp_box_nrs
  SourceCoeffs sc;
  HelmCoeffs hc;
  bool helm;
  int ncf, ncq;
  bool trans_ok;                           // matrix form of M2L / M2M / L2L available
  TransHost th;
  TransCfg tc;
  int device = -1;                         // CUDA device current at plan creation
  // per-level FMM orders (empty: fmm_order at every level); level_box_start: the
  // boxes of level l are [level_box_start[l], level_box_start[l + 1])
  std::vector<int32_t> lorders, level_box_start;
  int32_t* lorders_dev = nullptr;
  bool h3;                                 // 3D Helmholtz
  bool mixed;                              // FP32 far field (3D Laplace)
  bool tf32_ok;                            // split-TF32 translation matrices in use
  std::vector<double> h3gaunt;             // Gaunt table, [(nu,mu)][j][(n,m)]
  std::vector<double> h3rot;               // rotation tables, after the Gaunt table
  // host part of the rotation-based M2L tables (h3_m2l_host_tables), after the
  // rotation tables; then the device-built direction and coaxial tables
  std::vector<double> h3m2l;
  int h3_ndir = 0, h3_ncoax = 0;
  // 3D Helmholtz in the reference's default truncation (hc.taylor): monomial tables
  // of the box (order p) and QBX (order q) expansions
  H3TaylorHost h3tp, h3tq;
  // 3D Helmholtz: translation buffer and pair scratch registered by
  // qbxfmm_precompute_translations, used by the translation stage entries
  mutable const double* trans_dev = nullptr;
  mutable double* scratch_dev = nullptr;
  // 3D Laplace: M2L classes merged by offset symmetry; their index arrays (canonical
  // offsets, then at m2l_aux_cls the class codes) are uploaded into the translations
  // buffer at m2l_aux_off
  M2LSymClasses m2l_sym;
  std::vector<uint8_t> m2l_aux;
  size_t m2l_aux_off = 0, m2l_aux_cls = 0;
  // qbxfmm_apply runs the independent branches of the stage graph on three side
  // streams joined back into the caller's stream by events (fork/join, also
  // under stream capture): near field + M2P; P2L; P2QBXL + M2QBXL (the longest
  // branch, on a high-priority stream)
  cudaStream_t side[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr, ev_mpoles = nullptr, ev_near = nullptr, ev_p2l = nullptr,
              ev_qbx = nullptr;
  ~qbxfmm_plan()
  {
    for (cudaStream_t s : side)
      if (s) cudaStreamDestroy(s);
    for (cudaEvent_t e : {ev_fork, ev_mpoles, ev_near, ev_p2l, ev_qbx})
      if (e) cudaEventDestroy(e);
    if (lorders_dev) cudaFree(lorders_dev);
  }
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg)
{
  g_last_error = msg;
  return code;
}

int cuda_check(cudaError_t e, const char* where)
{
  if (e == cudaSuccess) return QBXFMM_OK;
  return fail(QBXFMM_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

cudaStream_t S(void* stream) { return reinterpret_cast<cudaStream_t>(stream); }

int check_plan(const qbxfmm_plan* p)
{
  if (!p) return fail(QBXFMM_ERR_ARG, "null plan");
  return QBXFMM_OK;
}

// the M2L class maps of a 3D Laplace plan in its translations buffer (empty otherwise)
TransAux trans_aux(const qbxfmm_plan* p, const void* translations)
{
  TransAux a;
  if (!translations || p->m2l_aux.empty()) return a;
  const char* b = static_cast<const char*>(translations) + p->m2l_aux_off;
  a.canon_off = reinterpret_cast<const int32_t*>(b);
  a.cls_code = reinterpret_cast<const int32_t*>(b + p->m2l_aux_cls);
  return a;
}

size_t h3_rot_offset(const qbxfmm_plan* p);

// Offsets in doubles of the 3D Helmholtz sections of the translation buffer, after
// the M2M / L2L matrices: [0] Gaunt table, [1] rotation tables, [2] host M2L tables,
// [3] M2L direction tables, [4] M2L coaxial tables (complex), [5] G0 of the order-p
// monomial tables and [6] Ginv of the order-q ones (complex; the reference's default
// truncation only, else empty), [7] end.
void h3_layout(const qbxfmm_plan* p, size_t o[8])
{
  o[0] = p->tc.nmatrices * p->tc.rp * p->tc.kp;
  o[1] = o[0] + p->h3gaunt.size();
  o[2] = (o[1] + p->h3rot.size() + 1) & ~(size_t)1;
  o[3] = (o[2] + p->h3m2l.size() + 1) & ~(size_t)1;    // 16-byte aligned for bulk copies
  o[4] = o[3] + (size_t)p->h3_ndir * h3_m2l_dsize(p->kern.fmm_order);
  o[5] = (o[4] + 2 * (size_t)p->h3_ncoax * h3_m2l_csize(p->kern.fmm_order) + 1) & ~(size_t)1;
  o[6] = o[5] + 2 * p->h3tp.G0.size();
  o[7] = o[6] + 2 * p->h3tq.Ginv.size();
}

size_t h3_rot_offset(const qbxfmm_plan* p)
{
  size_t o[8];
  h3_layout(p, o);
  return o[1];
}

// Gaunt integrals G(n,m; nu,mu; l) = int Y_n^m conj(Y_nu^mu) conj(Y_l^{m-mu}) for
// n, nu <= p (orthonormal spherical harmonics without the Condon-Shortley phase),
// l = |n - nu| + 2 j, j <= min(n, nu); layout [(nu,mu)][j][(n,m)], j < p + 1.  Exact
// Gauss-Legendre quadrature in cos(theta) of the polynomial integrand.
std::vector<double> h3_gaunt_table(int p)
{
  const int C = (p + 1) * (p + 1), nl = p + 1, L = 2 * p, ng = 2 * p + 2;
  std::vector<double> x(ng), w(ng);
  for (int i = 0; i < ng; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (ng + 0.5)), pp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= ng; ++j) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = ng * (z * p1 - p2) / (z * z - 1.0);
      double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) < 1e-16) break;
    }
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
  // polynomial parts p_n^m(t) (normalized; Y_n^m = p_n^m sin^m e^{i m phi}), n <= L
  auto pidx = [](int n, int m) { return n * (n + 1) / 2 + m; };
  std::vector<double> P((size_t)(L + 1) * (L + 2) / 2 * ng);
  for (int i = 0; i < ng; ++i) {
    double t = x[i], pmm = 0.28209479177387814347;
    for (int m = 0; m <= L; ++m) {
      if (m > 0) pmm *= std::sqrt((2.0 * m + 1.0) / (2.0 * m));
      double pm2 = 0.0, pm1 = pmm;
      P[(size_t)pidx(m, m) * ng + i] = pmm;
      for (int n = m + 1; n <= L; ++n) {
        double pn;
        if (n == m + 1) {
          pn = std::sqrt(2.0 * m + 3.0) * t * pm1;
        } else {
          double a = std::sqrt((4.0 * n * n - 1.0) / ((double)n * n - (double)m * m));
          double b = std::sqrt(((n - 1.0) * (n - 1.0) - (double)m * m) / (4.0 * (n - 1.0) * (n - 1.0) - 1.0));
          pn = a * (t * pm1 - b * pm2);
        }
        pm2 = pm1;
        pm1 = pn;
        P[(size_t)pidx(n, m) * ng + i] = pn;
      }
    }
  }
  std::vector<double> G((size_t)C * C * nl, 0.0);
  for (int nu = 0; nu <= p; ++nu)
    for (int mu = -nu; mu <= nu; ++mu)
      for (int n = 0; n <= p; ++n)
        for (int m = -n; m <= n; ++m) {
          int lam = m - mu, am = std::abs(m), amu = std::abs(mu), alam = std::abs(lam);
          int e = (am + amu + alam) / 2;
          size_t orow = nu * nu + nu + mu, icol = n * n + n + m;
          for (int j = 0; j <= std::min(n, nu); ++j) {
            int l = std::abs(n - nu) + 2 * j;
            if (alam > l) continue;
            double acc = 0.0;
            for (int i = 0; i < ng; ++i) {
              double om = 1.0;
              for (int u = 0; u < e; ++u) om *= 1.0 - x[i] * x[i];
              acc += w[i] * P[(size_t)pidx(n, am) * ng + i] * P[(size_t)pidx(nu, amu) * ng + i] *
                     P[(size_t)pidx(l, alam) * ng + i] * om;
            }
            G[(orow * nl + j) * C + icol] = 2.0 * M_PI * acc;
          }
        }
  return G;
}

// Tables of the rotation-based M2QBXL / L2QBXL (p = fmm order, q = QBX order):
//   start values of d^n_{m mu}(beta) at n0 = max(|m|, mu), mu >= 0: [2p+1][q+1][4] =
//     (coefficient, exponent of cos(beta/2), exponent of sin(beta/2), unused), from
//     the single surviving term of Wigner's formula;
//   isq[N][k] = 1 / sqrt(N^2 - k^2) (N > k, else 0), N <= p + 1, k <= p;
//   rt[n][k] = sqrt(n^2 - k^2) / sqrt((n+1)^2 - k^2) (n >= k, else 0), n, k <= p;
//   the lambda = 0 Gaunt slice g0[(nu,mu)][n][j] = G(n,mu; nu,mu; |n - nu| + 2 j),
//     nu <= q, n <= p, j <= q (zero outside n >= |mu|, j <= min(n, nu)),
//     read from the Gaunt table (layout [(nu,mu)][j][(n,m)]).
std::vector<double> h3_rotation_tables(int p, int q, const std::vector<double>& gaunt)
{
  const int nm = 2 * p + 1, ncf = (p + 1) * (p + 1), nl = p + 1, ncq = (q + 1) * (q + 1);
  const size_t nstart = (size_t)nm * (q + 1) * 4, nisq = (size_t)(p + 2) * (p + 1),
               nrt = (size_t)(p + 1) * (p + 1), ng0 = (size_t)ncq * nl * (q + 1);
  std::vector<double> t(nstart + nisq + nrt + ng0, 0.0);
  double* start = t.data();
  double* isq = start + nstart;
  double* rt = isq + nisq;
  double* g0 = rt + nrt;
  for (int m = -p; m <= p; ++m)
    for (int mu = 0; mu <= q; ++mu) {
      size_t idx = (size_t)(m + p) * (q + 1) + mu;
      int j = std::max(std::abs(m), mu);
      int kk = std::max(0, mu - m);
      int a1 = j + mu - kk, a3 = j - kk - m, a4 = kk - mu + m;
      double lf = 0.5 * (std::lgamma(j + m + 1.0) + std::lgamma(j - m + 1.0) +
                         std::lgamma(j + mu + 1.0) + std::lgamma(j - mu + 1.0)) -
                  (std::lgamma(a1 + 1.0) + std::lgamma(kk + 1.0) + std::lgamma(a3 + 1.0) +
                   std::lgamma(a4 + 1.0));
      start[4 * idx] = (((kk - mu + m) & 1) ? -1.0 : 1.0) * std::exp(lf);
      start[4 * idx + 1] = 2 * j + mu - m - 2 * kk;
      start[4 * idx + 2] = 2 * kk - mu + m;
    }
  for (int N = 0; N <= p + 1; ++N)
    for (int k = 0; k <= p; ++k)
      isq[(size_t)N * (p + 1) + k] = N > k ? 1.0 / std::sqrt((double)N * N - (double)k * k) : 0.0;
  for (int n = 0; n <= p; ++n)
    for (int k = 0; k <= p; ++k)
      rt[(size_t)n * (p + 1) + k] =
          n >= k ? std::sqrt(((double)n * n - (double)k * k) / ((n + 1.0) * (n + 1.0) - (double)k * k))
                 : 0.0;
  for (int nu = 0; nu <= q; ++nu)
    for (int mu = -nu; mu <= nu; ++mu) {
      int o = nu * nu + nu + mu;
      for (int n = std::abs(mu); n <= p; ++n)
        for (int j = 0; j <= std::min(n, nu); ++j)
          g0[((size_t)o * nl + n) * (q + 1) + j] = gaunt[((size_t)o * nl + j) * ncf + n * n + n + mu];
    }
  return t;
}

// Host part of the 3D Helmholtz M2L tables (p = fmm order), laid out as
//   start[(m + p)(2p + 1) + mu + p][4]: d^n_{m mu}(beta) at n0 = max(|m|, |mu|) for all
//     |m|, |mu| <= p (coefficient, exponents of cos(beta/2) and sin(beta/2), unused);
//   dirs[ndir][4]: the distinct directions of the M2L class offsets (unit vectors);
//   coaxp[ncoax][2]: (k |b|, min(1, k width)) for the distinct (|offset|^2, level);
//   clsmap[nclasses][2]: direction and coaxial table of each class;
// padded to an even length.  offs: [3][nclasses] integer offsets in box widths.
std::vector<double> h3_m2l_host_tables(int p, double k, double root_extent, int nclasses,
                                       const std::vector<int32_t>& offs,
                                       const std::vector<int32_t>& levels, int* ndir_out,
                                       int* ncoax_out)
{
  const int nm = 2 * p + 1;
  std::vector<double> start((size_t)nm * nm * 4, 0.0);
  for (int m = -p; m <= p; ++m)
    for (int mu = -p; mu <= p; ++mu) {
      size_t idx = (size_t)(m + p) * nm + (mu + p);
      int j = std::max(std::abs(m), std::abs(mu));
      int kk = std::max(0, mu - m);
      int a1 = j + mu - kk, a3 = j - kk - m, a4 = kk - mu + m;
      double lf = 0.5 * (std::lgamma(j + m + 1.0) + std::lgamma(j - m + 1.0) +
                         std::lgamma(j + mu + 1.0) + std::lgamma(j - mu + 1.0)) -
                  (std::lgamma(a1 + 1.0) + std::lgamma(kk + 1.0) + std::lgamma(a3 + 1.0) +
                   std::lgamma(a4 + 1.0));
      start[4 * idx] = (((kk - mu + m) & 1) ? -1.0 : 1.0) * std::exp(lf);
      start[4 * idx + 1] = 2 * j + mu - m - 2 * kk;
      start[4 * idx + 2] = 2 * kk - mu + m;
    }
  std::map<std::array<int, 3>, int> dir_id;
  std::map<std::pair<int, int>, int> coax_id;
  std::vector<double> dirs, coaxp, clsmap(2 * (size_t)nclasses);
  for (int c = 0; c < nclasses; ++c) {
    int o[3] = {offs[c], offs[(size_t)nclasses + c], offs[2 * (size_t)nclasses + c]};
    int gd = std::gcd(std::gcd(std::abs(o[0]), std::abs(o[1])), std::abs(o[2]));
    if (gd == 0) gd = 1;
    std::array<int, 3> key = {o[0] / gd, o[1] / gd, o[2] / gd};
    auto it = dir_id.find(key);
    if (it == dir_id.end()) {
      double len = std::sqrt((double)key[0] * key[0] + (double)key[1] * key[1] + (double)key[2] * key[2]);
      it = dir_id.emplace(key, (int)dir_id.size()).first;
      dirs.insert(dirs.end(), {key[0] / len, key[1] / len, key[2] / len, 0.0});
    }
    int n2 = o[0] * o[0] + o[1] * o[1] + o[2] * o[2];
    auto ck = std::make_pair(n2, levels[c]);
    auto jt = coax_id.find(ck);
    if (jt == coax_id.end()) {
      double w = std::ldexp(root_extent, -levels[c]);
      jt = coax_id.emplace(ck, (int)coax_id.size()).first;
      coaxp.insert(coaxp.end(), {k * std::sqrt((double)n2) * w, std::min(1.0, k * w)});
    }
    clsmap[2 * (size_t)c] = it->second;
    clsmap[2 * (size_t)c + 1] = jt->second;
  }
  *ndir_out = (int)dir_id.size();
  *ncoax_out = (int)coax_id.size();
  std::vector<double> t;
  t.reserve(start.size() + dirs.size() + coaxp.size() + clsmap.size() + 1);
  t.insert(t.end(), start.begin(), start.end());
  t.insert(t.end(), dirs.begin(), dirs.end());
  t.insert(t.end(), coaxp.begin(), coaxp.end());
  t.insert(t.end(), clsmap.begin(), clsmap.end());
  if (t.size() & 1) t.push_back(0.0);
  return t;
}

#define QBX_TRY(expr, where)                         \
  do {                                               \
    int _rc = cuda_check((expr), where);             \
    if (_rc != QBXFMM_OK) return _rc;                \
  } while (0)

// Per-level FMM orders: box expansions live at fmm_order (the largest level order);
// after every stage that writes them, the coefficients above a box's level order are
// zeroed, M2M and L2L level by level (a level's translations read the level written
// before it).
bool level_orders_on(const qbxfmm_plan* p) { return !p->lorders.empty(); }

int mask_levels(const qbxfmm_plan* p, void* exps, int lev0, int lev1, cudaStream_t st)
{
  int b0 = p->level_box_start[lev0], b1 = p->level_box_start[lev1 + 1];
  QBX_TRY(launch_level_mask(p->geo, b0, b1, p->lorders_dev, p->kern.family, p->ncf, p->kern.nrhs,
                            (double2*)exps, st),
          "per-level orders");
  return QBXFMM_OK;
}

int mask_all_levels(const qbxfmm_plan* p, void* exps, cudaStream_t st)
{
  return level_orders_on(p) ? mask_levels(p, exps, 0, p->geo.nlevels - 1, st) : QBXFMM_OK;
}

// the host level-start array restricted to level lev (every other level empty)
std::vector<int32_t> one_level(const std::vector<int32_t>& starts, int lev)
{
  std::vector<int32_t> r(starts.size());
  for (size_t i = 0; i < r.size(); ++i) r[i] = (int)i <= lev ? starts[lev] : starts[lev + 1];
  return r;
}

// the translation host table restricted to the M2M groups of parent level lev or
// the L2L groups of child level lev
TransHost one_level(const TransHost& th, int lev, bool m2m)
{
  TransHost r = th;
  for (int l = 0; l < 64; ++l)
    if (l != lev) {
      if (m2m) r.m2m_level_max_group[l] = 0;
      else {
        r.l2l_level_max_group[l] = 0;
        r.l2l_level_pairs[l] = 0;
      }
    }
  return r;
}

}  // namespace

namespace qbx {

// Byte sizes of the first six workspace buffers (no device access), for the
// allocation-free entry point.
int plan_base_workspace_sizes(const qbxfmm_plan* p, size_t* sizes6)
{
  if (int rc = check_plan(p)) return rc;
  const qbxfmm_geometry& g = p->geo;
  size_t nr = (size_t)p->kern.nrhs;
  size_t scal = (p->kern.family == QBXFMM_LAPLACE) ? sizeof(double) : 2 * sizeof(double);
  sizes6[0] = nr * g.nsources * scal;
  sizes6[1] = (size_t)g.nboxes * nr * p->ncf * 2 * sizeof(double);
  sizes6[2] = sizes6[1];
  sizes6[3] = (size_t)g.ncenters * nr * p->ncq * 2 * sizeof(double);
  sizes6[4] = nr * (size_t)(g.nfiltered_targets > 0 ? g.nfiltered_targets : 1) * scal;
  sizes6[5] = nr * (size_t)g.ntargets * scal;
  return QBXFMM_OK;
}

int set_last_error(int code, const std::string& msg) { return fail(code, msg); }

int plan_device(const qbxfmm_plan* p) { return p ? p->device : -1; }

bool plan_needs_translation_tables(const qbxfmm_plan* p) { return p && p->h3; }

}  // namespace qbx

extern "C" {

int qbxfmm_version(void) { return 1; }

const char* qbxfmm_last_error(void) { return g_last_error.c_str(); }

int qbxfmm_plan_create(const qbxfmm_kernel* kernel, const qbxfmm_geometry* geometry,
                       qbxfmm_plan** out)
{
  if (!kernel || !geometry || !out) return fail(QBXFMM_ERR_ARG, "null argument");
  *out = nullptr;
  const qbxfmm_kernel& k = *kernel;
  const qbxfmm_geometry& g = *geometry;
  if (k.family != QBXFMM_LAPLACE && k.family != QBXFMM_HELMHOLTZ)
    return fail(QBXFMM_ERR_UNSUPPORTED, "kernel family must be Laplace or Helmholtz");
  if (k.dim != 2 && k.dim != 3) return fail(QBXFMM_ERR_ARG, "dim must be 2 or 3");
  if (k.family == QBXFMM_HELMHOLTZ && (k.k_im != 0.0 || !(k.k_re > 0.0)))
    return fail(QBXFMM_ERR_UNSUPPORTED, "Helmholtz wave number must be real and positive");
  if (g.dim != k.dim) return fail(QBXFMM_ERR_ARG, "kernel and geometry dimensions differ");
  if (k.qbx_order < 0 || k.qbx_order > 8)
    return fail(QBXFMM_ERR_UNSUPPORTED, "qbx_order must be in [0, 8]");
  if (k.fmm_order < 1 || k.fmm_order > 20 || (k.family == QBXFMM_HELMHOLTZ && k.qbx_order + k.fmm_order > 28))
    return fail(QBXFMM_ERR_UNSUPPORTED, "fmm_order must be in [1, 20]");
  if (k.nrhs < 1) return fail(QBXFMM_ERR_ARG, "nrhs must be >= 1");
  if (k.precision != 0 && k.precision != 1)
    return fail(QBXFMM_ERR_ARG, "precision must be 0 (FP64) or 1 (mixed)");
  if (k.fmm_backend != QBXFMM_BACKEND_SUMPY && k.fmm_backend != QBXFMM_BACKEND_FMMLIB)
    return fail(QBXFMM_ERR_ARG, "fmm_backend must be QBXFMM_BACKEND_SUMPY or QBXFMM_BACKEND_FMMLIB");
  if (k.precision == 1 && k.dim != 3)
    return fail(QBXFMM_ERR_UNSUPPORTED, "the mixed-precision form is built for 3D Laplace and 3D Helmholtz");
  if (k.family == QBXFMM_HELMHOLTZ && k.dim == 3) {
    if (k.qbx_order > 5 || k.qbx_order > k.fmm_order)
      return fail(QBXFMM_ERR_UNSUPPORTED, "3D Helmholtz: qbx_order must be <= min(5, fmm_order)");
    if (k.fmm_order > 17)
      return fail(QBXFMM_ERR_UNSUPPORTED, "3D Helmholtz: fmm_order must be <= 17");
    if (g.m2l_nclasses > 0 && !g.m2l_class_levels)
      return fail(QBXFMM_ERR_ARG, "3D Helmholtz needs per-level M2L classes (m2l_class_levels)");
  }
  if (k.family == QBXFMM_LAPLACE && (k.charge_coeff_im != 0.0 || k.dipole_coeff_im != 0.0))
    return fail(QBXFMM_ERR_ARG, "Laplace source coefficients must be real");
  if (g.nlevels < 1 || g.nboxes < 1 || g.nlevels > 40) return fail(QBXFMM_ERR_ARG, "bad tree sizes");
  if (k.dipole_coeff_re != 0.0 && !g.source_normals)
    return fail(QBXFMM_ERR_ARG, "double layer requested without source normals");

  qbxfmm_plan* p = new (std::nothrow) qbxfmm_plan;
  if (!p) return fail(QBXFMM_ERR_ARG, "out of host memory");
  p->kern = k;
  p->geo = g;
  p->sc.cq = k.charge_coeff_re;
  p->sc.cd = k.dipole_coeff_re;
  p->helm = k.family == QBXFMM_HELMHOLTZ;
  p->hc.cq = make_double2(k.charge_coeff_re, k.charge_coeff_im);
  p->hc.cd = make_double2(k.dipole_coeff_re, k.dipole_coeff_im);
  p->hc.k = k.k_re;
  p->ncf = ncoeff(k.family, k.dim, k.fmm_order);
  p->ncq = ncoeff(k.family, k.dim, k.qbx_order);
  p->lvl_source_parent.resize(g.nlevels + 1);
  p->lvl_ttp.resize(g.nlevels + 1);
  cudaError_t e = cudaMemcpy(p->lvl_source_parent.data(), g.level_start_source_parent_box_nrs,
                             sizeof(int32_t) * (g.nlevels + 1), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    e = cudaMemcpy(p->lvl_ttp.data(), g.level_start_ttp_box_nrs, sizeof(int32_t) * (g.nlevels + 1),
                   cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaGetDevice(&p->device);
  p->h3 = p->helm && k.dim == 3;
  p->mixed = k.precision == 1;
  if (k.dim == 3 && !p->h3 && g.m2l_nclasses > 0 && e == cudaSuccess) {
    std::vector<int32_t> off(3 * (size_t)g.m2l_nclasses);
    e = cudaMemcpy(off.data(), g.m2l_class_offsets, sizeof(int32_t) * off.size(),
                   cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) p->m2l_sym = m2l_symmetry_classes(g.m2l_nclasses, off);
    if (p->m2l_sym.ncanon < 0) {
      delete p;
      return fail(QBXFMM_ERR_ARG, "M2L class offsets are not integer lattice offsets");
    }
  }
  if (k.dim == 3)
    p->tc = p->h3 ? trans_cfg_helm3(k.fmm_order, 0, g.nlevels)   // M2L by rotation, no class matrices
                  : trans_cfg_laplace3(k.fmm_order, p->m2l_sym.ncanon);
  p->trans_ok = k.dim == 3 && trans_supported(p->tc) && g.nlevels <= 64;
  p->tf32_ok = p->mixed && p->trans_ok && tf32_supported(p->tc);
  if (k.dim == 3 && !p->h3) {
    // the index arrays after the matrices (and their TF32 planes), 16-byte aligned
    auto al = [](size_t b) { return (b + 15) / 16 * 16; };
    const M2LSymClasses& ms = p->m2l_sym;
    p->m2l_aux_off = al(trans_matrix_bytes(p->tc) + (p->tf32_ok ? tf32_matrix_bytes(p->tc) : 0));
    p->m2l_aux_cls = al(ms.canon_off.size() * sizeof(int32_t));
    p->m2l_aux.assign(al(p->m2l_aux_cls + ms.cls_code.size() * sizeof(int32_t)), 0);
    std::memcpy(p->m2l_aux.data(), ms.canon_off.data(), ms.canon_off.size() * sizeof(int32_t));
    std::memcpy(p->m2l_aux.data() + p->m2l_aux_cls, ms.cls_code.data(),
                ms.cls_code.size() * sizeof(int32_t));
  }
  if (p->h3 && !p->trans_ok) {
    delete p;
    return fail(QBXFMM_ERR_UNSUPPORTED, "3D Helmholtz: translation matrices unsupported for this order");
  }
  p->hc.taylor = p->h3 && k.fmm_backend == QBXFMM_BACKEND_SUMPY;
  if (p->hc.taylor) {
    p->h3tp = h3_taylor_host(k.fmm_order);
    p->h3tq = h3_taylor_host(k.qbx_order);
    if (p->h3tp.p < 0 || p->h3tq.p < 0) {
      delete p;
      return fail(QBXFMM_ERR_UNSUPPORTED, "3D Helmholtz: singular Taylor basis table");
    }
  }
  if (p->h3) {
    p->h3gaunt = h3_gaunt_table(k.fmm_order);
    p->h3rot = h3_rotation_tables(k.fmm_order, k.qbx_order, p->h3gaunt);
    std::vector<int32_t> off(3 * (size_t)g.m2l_nclasses), lev(g.m2l_nclasses);
    if (g.m2l_nclasses > 0 && e == cudaSuccess)
      e = cudaMemcpy(off.data(), g.m2l_class_offsets, sizeof(int32_t) * off.size(),
                     cudaMemcpyDeviceToHost);
    if (g.m2l_nclasses > 0 && e == cudaSuccess)
      e = cudaMemcpy(lev.data(), g.m2l_class_levels, sizeof(int32_t) * lev.size(),
                     cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
      p->h3m2l = h3_m2l_host_tables(k.fmm_order, k.k_re, g.root_extent, g.m2l_nclasses, off, lev,
                                    &p->h3_ndir, &p->h3_ncoax);
  }
  if (e == cudaSuccess && p->trans_ok) {
    const int nch = 8;
    std::vector<int32_t> cs(g.m2l_nclasses + 1), ms(g.nlevels * nch + 1), ls(g.nlevels * nch + 1);
    e = cudaMemcpy(cs.data(), g.m2l_class_starts, sizeof(int32_t) * cs.size(), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
      e = cudaMemcpy(ms.data(), g.m2m_group_starts, sizeof(int32_t) * ms.size(), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
      e = cudaMemcpy(ls.data(), g.l2l_group_starts, sizeof(int32_t) * ls.size(), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) {
      for (int c = 0; c < g.m2l_nclasses; ++c)
        p->th.m2l_max_pairs = std::max(p->th.m2l_max_pairs, cs[c + 1] - cs[c]);
      p->th.m2l_npairs = cs[g.m2l_nclasses];
      for (int lev = 0; lev < g.nlevels; ++lev)
        for (int ci = 0; ci < nch; ++ci) {
          int gi = lev * nch + ci;
          p->th.m2m_level_max_group[lev] = std::max(p->th.m2m_level_max_group[lev], ms[gi + 1] - ms[gi]);
          p->th.l2l_level_max_group[lev] = std::max(p->th.l2l_level_max_group[lev], ls[gi + 1] - ls[gi]);
        }
      for (int lev = 0; lev < g.nlevels; ++lev)
        p->th.l2l_level_pairs[lev] = ls[(lev + 1) * nch] - ls[lev * nch];
      p->th.lvl_source_parent = p->lvl_source_parent.data();
    }
  }
  int prio_least = 0, prio_greatest = 0;
  if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
  for (int i = 0; i < 3 && e == cudaSuccess; ++i)
    e = cudaStreamCreateWithPriority(&p->side[i], cudaStreamNonBlocking,
                                     i == 2 ? prio_greatest : prio_least);
  for (cudaEvent_t* ev : {&p->ev_fork, &p->ev_mpoles, &p->ev_near, &p->ev_p2l, &p->ev_qbx})
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    delete p;
    return cuda_check(e, "qbxfmm_plan_create");
  }
  *out = p;
  return QBXFMM_OK;
}

int qbxfmm_plan_destroy(qbxfmm_plan* plan)
{
  delete plan;
  return QBXFMM_OK;
}

int qbxfmm_form_strengths(const qbxfmm_plan* p, const qbxfmm_upsample* up, const void* density,
                          void* strengths, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (!up || !density || !strengths) return fail(QBXFMM_ERR_ARG, "null argument");
  if (up->quad_nodes_per_element * up->nelements != p->geo.nsources)
    return fail(QBXFMM_ERR_ARG, "upsampler does not match the number of sources");
  if (p->helm)
    QBX_TRY(h2_launch_form_strengths(p->geo, *up, p->kern.nrhs, (const double2*)density,
                                     (double2*)strengths, S(stream)),
            "form_strengths");
  else
    QBX_TRY(launch_form_strengths(p->geo, *up, p->kern.nrhs, (const double*)density,
                                  (double*)strengths, S(stream)),
            "form_strengths");
  return QBXFMM_OK;
}

int qbxfmm_form_multipoles(const qbxfmm_plan* p, const void* strengths, void* mpoles, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3) {
    QBX_TRY(h3_launch_p2m(p->geo, p->hc, p->kern.fmm_order, p->kern.nrhs, (const double2*)strengths,
                          (double2*)mpoles, S(stream)),
            "form_multipoles");
    return mask_all_levels(p, mpoles, S(stream));
  }
  if (p->helm)
    QBX_TRY(h2_launch_p2m(p->geo, p->hc, p->kern.fmm_order, p->kern.nrhs,
                          (const double2*)strengths, (double2*)mpoles, nullptr, S(stream)),
            "form_multipoles");
  else if (p->mixed)
    QBX_TRY(launch_p2m_mixed(p->geo, p->sc, p->kern.fmm_order, p->kern.nrhs,
                             (const double*)strengths, (double2*)mpoles, S(stream)),
            "form_multipoles");
  else
    QBX_TRY(launch_p2m(p->geo, p->sc, p->kern.fmm_order, p->kern.nrhs, (const double*)strengths,
                       (double2*)mpoles, S(stream)),
            "form_multipoles");
  return mask_all_levels(p, mpoles, S(stream));
}

int qbxfmm_coarsen_multipoles(const qbxfmm_plan* p, void* mpoles, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3 && !p->trans_dev)
    return fail(QBXFMM_ERR_ARG, "3D Helmholtz: call qbxfmm_precompute_translations first");
  if (level_orders_on(p)) {
    // parents of level lev from children of level lev + 1, then truncated
    for (int lev = p->geo.nlevels - 2; lev >= 0; --lev) {
      if (p->h3) {
        QBX_TRY(launch_m2m_direct(p->geo, one_level(p->th, lev, true), p->tc, p->kern.nrhs,
                                  p->trans_dev, (double2*)mpoles, nullptr, S(stream)),
                "coarsen_multipoles");
      } else {
        std::vector<int32_t> lv = one_level(p->lvl_source_parent, lev);
        if (p->helm)
          QBX_TRY(h2_launch_m2m(p->geo, lv.data(), p->hc, p->kern.fmm_order, p->kern.nrhs,
                                (double2*)mpoles, nullptr, S(stream)),
                  "coarsen_multipoles");
        else
          QBX_TRY(launch_m2m(p->geo, lv.data(), p->kern.fmm_order, p->kern.nrhs, (double2*)mpoles,
                             S(stream)),
                  "coarsen_multipoles");
      }
      if (int rc = mask_levels(p, mpoles, lev, lev, S(stream))) return rc;
    }
    return QBXFMM_OK;
  }
  if (p->h3) {
    QBX_TRY(launch_m2m_direct(p->geo, p->th, p->tc, p->kern.nrhs, p->trans_dev, (double2*)mpoles,
                              nullptr, S(stream)),
            "coarsen_multipoles");
    return QBXFMM_OK;
  }
  if (p->helm)
    QBX_TRY(h2_launch_m2m(p->geo, p->lvl_source_parent.data(), p->hc, p->kern.fmm_order,
                          p->kern.nrhs, (double2*)mpoles, nullptr, S(stream)),
            "coarsen_multipoles");
  else
    QBX_TRY(launch_m2m(p->geo, p->lvl_source_parent.data(), p->kern.fmm_order, p->kern.nrhs,
                       (double2*)mpoles, S(stream)),
            "coarsen_multipoles");
  return QBXFMM_OK;
}

int qbxfmm_eval_direct(const qbxfmm_plan* p, const void* strengths, void* pot_nonqbx,
                       int32_t* error_word, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3) {
    QBX_TRY(h3_launch_eval_direct(p->geo, p->hc, p->kern.nrhs, (const double2*)strengths,
                                  (double2*)pot_nonqbx, error_word, S(stream)),
            "eval_direct");
    return QBXFMM_OK;
  }
  if (p->helm)
    QBX_TRY(h2_launch_eval_direct(p->geo, p->hc, p->kern.nrhs, (const double2*)strengths,
                                  (double2*)pot_nonqbx, error_word, S(stream)),
            "eval_direct");
  else
    QBX_TRY(launch_eval_direct(p->geo, p->sc, p->kern.nrhs, (const double*)strengths,
                               (double*)pot_nonqbx, error_word, S(stream)),
            "eval_direct");
  return QBXFMM_OK;
}

int qbxfmm_multipole_to_local(const qbxfmm_plan* p, const void* mpoles, void* locals,
                              int32_t* error_word, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3) {
    if (!p->trans_dev)
      return fail(QBXFMM_ERR_ARG, "3D Helmholtz: call qbxfmm_precompute_translations first");
    size_t o[8];
    h3_layout(p, o);
    const int nm = 2 * p->kern.fmm_order + 1;
    const double* clsmap = p->trans_dev + o[2] + (size_t)nm * nm * 4 + 4 * (size_t)p->h3_ndir +
                           2 * (size_t)p->h3_ncoax;
    QBX_TRY(h3_launch_m2l_rot(p->geo, p->kern.fmm_order, p->kern.nrhs, (const double2*)mpoles,
                              (double2*)locals, p->trans_dev + o[3],
                              reinterpret_cast<const double2*>(p->trans_dev + o[4]), clsmap,
                              error_word, S(stream), p->mixed, p->hc.rb_m2l),
            "multipole_to_local");
    return mask_all_levels(p, locals, S(stream));
  }
  if (p->helm)
    QBX_TRY(h2_launch_m2l(p->geo, p->hc, p->kern.fmm_order, p->kern.nrhs, (const double2*)mpoles,
                          (double2*)locals, error_word, S(stream)),
            "multipole_to_local");
  else
    QBX_TRY(launch_m2l(p->geo, p->kern.fmm_order, p->kern.nrhs, (const double2*)mpoles,
                       (double2*)locals, error_word, S(stream)),
            "multipole_to_local");
  return mask_all_levels(p, locals, S(stream));
}

int qbxfmm_eval_multipoles(const qbxfmm_plan* p, const void* mpoles, void* pot_nonqbx,
                           int32_t* error_word, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3) {
    QBX_TRY(h3_launch_eval_multipoles(p->geo, p->hc, p->kern.fmm_order, p->kern.nrhs,
                                      (const double2*)mpoles, (double2*)pot_nonqbx, error_word,
                                      S(stream)),
            "eval_multipoles");
    return QBXFMM_OK;
  }
  if (p->helm)
    QBX_TRY(h2_launch_eval_multipoles(p->geo, p->hc, p->kern.fmm_order, p->kern.nrhs,
                                      (const double2*)mpoles, (double2*)pot_nonqbx, error_word,
                                      S(stream)),
            "eval_multipoles");
  else
    QBX_TRY(launch_eval_multipoles(p->geo, p->kern.fmm_order, p->kern.nrhs, (const double2*)mpoles,
                                   (double*)pot_nonqbx, error_word, S(stream)),
            "eval_multipoles");
  return QBXFMM_OK;
}

int qbxfmm_form_locals(const qbxfmm_plan* p, const void* strengths, void* locals,
                       int32_t* error_word, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3) {
    QBX_TRY(h3_launch_p2l(p->geo, p->hc, p->kern.fmm_order, p->kern.nrhs, (const double2*)strengths,
                          (double2*)locals, error_word, S(stream)),
            "form_locals");
    return mask_all_levels(p, locals, S(stream));
  }
  if (p->helm)
    QBX_TRY(h2_launch_p2l(p->geo, p->hc, p->kern.fmm_order, p->kern.nrhs,
                          (const double2*)strengths, (double2*)locals, error_word, S(stream)),
            "form_locals");
  else if (p->mixed)
    QBX_TRY(launch_p2l_mixed(p->geo, p->sc, p->kern.fmm_order, p->kern.nrhs,
                             (const double*)strengths, (double2*)locals, error_word, S(stream)),
            "form_locals");
  else
    QBX_TRY(launch_p2l(p->geo, p->sc, p->kern.fmm_order, p->kern.nrhs, (const double*)strengths,
                       (double2*)locals, error_word, S(stream)),
            "form_locals");
  return mask_all_levels(p, locals, S(stream));
}

int qbxfmm_refine_locals(const qbxfmm_plan* p, void* locals, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3 && !p->trans_dev)
    return fail(QBXFMM_ERR_ARG, "3D Helmholtz: call qbxfmm_precompute_translations first");
  if (level_orders_on(p)) {
    // children of level lev from parents of level lev - 1, then truncated
    for (int lev = 1; lev < p->geo.nlevels; ++lev) {
      if (p->h3) {
        QBX_TRY(launch_l2l_direct(p->geo, one_level(p->th, lev, false), p->tc, p->kern.nrhs,
                                  p->trans_dev, (double2*)locals, nullptr, S(stream)),
                "refine_locals");
      } else {
        std::vector<int32_t> lv = one_level(p->lvl_ttp, lev);
        if (p->helm)
          QBX_TRY(h2_launch_l2l(p->geo, lv.data(), p->hc, p->kern.fmm_order, p->kern.nrhs,
                                (double2*)locals, nullptr, S(stream)),
                  "refine_locals");
        else
          QBX_TRY(launch_l2l(p->geo, lv.data(), p->kern.fmm_order, p->kern.nrhs, (double2*)locals,
                             S(stream)),
                  "refine_locals");
      }
      if (int rc = mask_levels(p, locals, lev, lev, S(stream))) return rc;
    }
    return QBXFMM_OK;
  }
  if (p->h3) {
    QBX_TRY(launch_l2l_direct(p->geo, p->th, p->tc, p->kern.nrhs, p->trans_dev, (double2*)locals,
                              nullptr, S(stream)),
            "refine_locals");
    return QBXFMM_OK;
  }
  if (p->helm)
    QBX_TRY(h2_launch_l2l(p->geo, p->lvl_ttp.data(), p->hc, p->kern.fmm_order, p->kern.nrhs,
                          (double2*)locals, nullptr, S(stream)),
            "refine_locals");
  else
    QBX_TRY(launch_l2l(p->geo, p->lvl_ttp.data(), p->kern.fmm_order, p->kern.nrhs,
                       (double2*)locals, S(stream)),
            "refine_locals");
  return QBXFMM_OK;
}

int qbxfmm_eval_locals(const qbxfmm_plan* p, const void* locals, void* pot_nonqbx, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3) {
    QBX_TRY(h3_launch_eval_locals(p->geo, p->hc, p->kern.fmm_order, p->kern.nrhs,
                                  (const double2*)locals, (double2*)pot_nonqbx, S(stream)),
            "eval_locals");
    return QBXFMM_OK;
  }
  if (p->helm)
    QBX_TRY(h2_launch_eval_locals(p->geo, p->hc, p->kern.fmm_order, p->kern.nrhs,
                                  (const double2*)locals, (double2*)pot_nonqbx, nullptr, S(stream)),
            "eval_locals");
  else
    QBX_TRY(launch_eval_locals(p->geo, p->kern.fmm_order, p->kern.nrhs, (const double2*)locals,
                               (double*)pot_nonqbx, S(stream)),
            "eval_locals");
  return QBXFMM_OK;
}

int qbxfmm_form_global_qbx_locals(const qbxfmm_plan* p, const void* strengths, void* qbx_exps,
                                  int32_t* error_word, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3) {
    QBX_TRY(h3_launch_p2qbxl(p->geo, p->hc, p->kern.qbx_order, p->kern.nrhs,
                             (const double2*)strengths, (double2*)qbx_exps, error_word, S(stream)),
            "form_global_qbx_locals");
    return QBXFMM_OK;
  }
  if (p->helm)
    QBX_TRY(h2_launch_p2qbxl(p->geo, p->hc, p->kern.qbx_order, p->kern.nrhs,
                             (const double2*)strengths, (double2*)qbx_exps, error_word, S(stream)),
            "form_global_qbx_locals");
  else
    QBX_TRY(launch_p2qbxl(p->geo, p->sc, p->kern.qbx_order, p->kern.nrhs, (const double*)strengths,
                          (double2*)qbx_exps, error_word, S(stream)),
            "form_global_qbx_locals");
  return QBXFMM_OK;
}

int qbxfmm_translate_box_multipoles_to_qbx_local(const qbxfmm_plan* p, const void* mpoles,
                                                 void* qbx_exps, int32_t* error_word, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3) {
    if (!p->trans_dev)
      return fail(QBXFMM_ERR_ARG, "3D Helmholtz: call qbxfmm_precompute_translations first");
    QBX_TRY(h3_launch_m2qbxl(p->geo, p->hc, p->kern.fmm_order, p->kern.qbx_order, p->kern.nrhs,
                             (const double2*)mpoles,
                             p->trans_dev + h3_rot_offset(p),
                             (double2*)qbx_exps, error_word, S(stream), p->mixed),
            "translate_box_multipoles_to_qbx_local");
    return QBXFMM_OK;
  }
  if (p->helm)
    QBX_TRY(h2_launch_m2qbxl(p->geo, p->hc, p->kern.fmm_order, p->kern.qbx_order, p->kern.nrhs,
                             (const double2*)mpoles, (double2*)qbx_exps, error_word, S(stream)),
            "translate_box_multipoles_to_qbx_local");
  else if (p->mixed)
    QBX_TRY(launch_m2qbxl_mixed(p->geo, p->kern.fmm_order, p->kern.qbx_order, p->kern.nrhs,
                                (const double2*)mpoles, (double2*)qbx_exps, error_word, S(stream)),
            "translate_box_multipoles_to_qbx_local");
  else
    QBX_TRY(launch_m2qbxl(p->geo, p->kern.fmm_order, p->kern.qbx_order, p->kern.nrhs,
                          (const double2*)mpoles, (double2*)qbx_exps, error_word, S(stream)),
            "translate_box_multipoles_to_qbx_local");
  return QBXFMM_OK;
}

int qbxfmm_translate_box_local_to_qbx_local(const qbxfmm_plan* p, const void* locals,
                                            void* qbx_exps, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3) {
    if (!p->trans_dev)
      return fail(QBXFMM_ERR_ARG, "3D Helmholtz: call qbxfmm_precompute_translations first");
    if (p->hc.taylor) {
      size_t o[8];
      h3_layout(p, o);
      QBX_TRY(h3_launch_l2qbxl_taylor(p->geo, p->hc, p->kern.fmm_order, p->kern.qbx_order,
                                      p->kern.nrhs, (const double2*)locals,
                                      reinterpret_cast<const double2*>(p->trans_dev + o[5]),
                                      reinterpret_cast<const double2*>(p->trans_dev + o[6]),
                                      (double2*)qbx_exps, nullptr, S(stream)),
              "translate_box_local_to_qbx_local");
      return QBXFMM_OK;
    }
    QBX_TRY(h3_launch_l2qbxl(p->geo, p->hc, p->kern.fmm_order, p->kern.qbx_order, p->kern.nrhs,
                             (const double2*)locals,
                             p->trans_dev + h3_rot_offset(p),
                             (double2*)qbx_exps, nullptr, S(stream)),
            "translate_box_local_to_qbx_local");
    return QBXFMM_OK;
  }
  if (p->helm)
    QBX_TRY(h2_launch_l2qbxl(p->geo, p->hc, p->kern.fmm_order, p->kern.qbx_order, p->kern.nrhs,
                             (const double2*)locals, (double2*)qbx_exps, nullptr, S(stream)),
            "translate_box_local_to_qbx_local");
  else
    QBX_TRY(launch_l2qbxl(p->geo, p->kern.fmm_order, p->kern.qbx_order, p->kern.nrhs,
                          (const double2*)locals, (double2*)qbx_exps, S(stream)),
            "translate_box_local_to_qbx_local");
  return QBXFMM_OK;
}

int qbxfmm_eval_qbx_expansions(const qbxfmm_plan* p, const void* qbx_exps, void* pot_tree,
                               void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3) {
    QBX_TRY(h3_launch_qbxl2p(p->geo, p->hc, p->kern.qbx_order, p->kern.nrhs,
                             (const double2*)qbx_exps, (double2*)pot_tree, S(stream)),
            "eval_qbx_expansions");
    return QBXFMM_OK;
  }
  if (p->helm)
    QBX_TRY(h2_launch_qbxl2p(p->geo, p->hc, p->kern.qbx_order, p->kern.nrhs,
                             (const double2*)qbx_exps, (double2*)pot_tree, S(stream)),
            "eval_qbx_expansions");
  else
    QBX_TRY(launch_qbxl2p(p->geo, p->kern.qbx_order, p->kern.nrhs, (const double2*)qbx_exps,
                          (double*)pot_tree, S(stream)),
            "eval_qbx_expansions");
  return QBXFMM_OK;
}

int qbxfmm_eval_target_specific_qbx_locals(const qbxfmm_plan* p, const void* strengths,
                                           void* pot_tree, int32_t* error_word, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3) {
    QBX_TRY(h3_launch_tsqbx(p->geo, p->hc, p->kern.qbx_order, p->kern.nrhs, (const double2*)strengths,
                            (double2*)pot_tree, error_word, S(stream)),
            "eval_target_specific_qbx_locals");
    return QBXFMM_OK;
  }
  if (p->helm) {
    QBX_TRY(h2_launch_tsqbx(p->geo, p->hc, p->kern.qbx_order, p->kern.nrhs, (const double2*)strengths,
                            (double2*)pot_tree, error_word, S(stream)),
            "eval_target_specific_qbx_locals");
    return QBXFMM_OK;
  }
  QBX_TRY(launch_tsqbx(p->geo, p->sc, p->kern.qbx_order, p->kern.nrhs, (const double*)strengths,
                       (double*)pot_tree, error_word, S(stream)),
          "eval_target_specific_qbx_locals");
  return QBXFMM_OK;
}

int qbxfmm_assemble(const qbxfmm_plan* p, const void* pot_nonqbx, const void* pot_tree, void* out,
                    void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->h3) {
    QBX_TRY(h3_launch_assemble(p->geo, p->kern.nrhs, (const double2*)pot_nonqbx,
                               (const double2*)pot_tree, (double2*)out, S(stream)),
            "assemble");
    return QBXFMM_OK;
  }
  if (p->helm)
    QBX_TRY(h2_launch_assemble(p->geo, p->kern.nrhs, (const double2*)pot_nonqbx,
                               (const double2*)pot_tree, (double2*)out, S(stream)),
            "assemble");
  else
    QBX_TRY(launch_assemble(p->geo, p->kern.nrhs, (const double*)pot_nonqbx,
                            (const double*)pot_tree, (double*)out, S(stream)),
            "assemble");
  return QBXFMM_OK;
}

int qbxfmm_plan_set_tuning(qbxfmm_plan* p, const qbxfmm_tuning* t)
{
  if (int rc = check_plan(p)) return rc;
  if (!t) return fail(QBXFMM_ERR_ARG, "null tuning");
  auto ok = [](int v, std::initializer_list<int> allowed) {
    if (v == 0) return true;
    for (int a : allowed)
      if (v == a) return true;
    return false;
  };
  if (!ok(t->m2qbxl_densities, {1, 4, 8, 16}) || !ok(t->m2l_densities, {1, 4, 8, 16}) ||
      !ok(t->p2e_densities, {1, 4, 8, 16}) || !ok(t->l2qbxl_densities, {1, 4}) ||
      !ok(t->tsqbx_densities, {1, 4, 16}))
    return fail(QBXFMM_ERR_ARG, "tuning: unsupported densities-per-CTA value");
  p->hc.rb_rot = t->m2qbxl_densities;
  p->hc.rb_m2l = t->m2l_densities;
  p->hc.rb_p2e = t->p2e_densities;
  p->hc.rb_l2q = t->l2qbxl_densities;
  p->hc.rb_ts = t->tsqbx_densities;
  return QBXFMM_OK;
}

int qbxfmm_plan_get_tuning(const qbxfmm_plan* p, qbxfmm_tuning* t)
{
  if (int rc = check_plan(p)) return rc;
  if (!t) return fail(QBXFMM_ERR_ARG, "null tuning");
  t->m2qbxl_densities = p->hc.rb_rot;
  t->m2l_densities = p->hc.rb_m2l;
  t->p2e_densities = p->hc.rb_p2e;
  t->l2qbxl_densities = p->hc.rb_l2q;
  t->tsqbx_densities = p->hc.rb_ts;
  return QBXFMM_OK;
}

int qbxfmm_plan_set_level_orders(qbxfmm_plan* p, const int32_t* orders, int32_t nlevels)
{
  if (int rc = check_plan(p)) return rc;
  if (!orders) {
    p->lorders.clear();
    return QBXFMM_OK;
  }
  if (nlevels != p->geo.nlevels)
    return fail(QBXFMM_ERR_ARG, "level orders: one order per tree level expected");
  bool all_max = true;
  for (int l = 0; l < nlevels; ++l) {
    if (orders[l] < 0 || orders[l] > p->kern.fmm_order)
      return fail(QBXFMM_ERR_ARG, "level orders: each order must be in [0, fmm_order]");
    all_max &= orders[l] == p->kern.fmm_order;
  }
  if (p->hc.taylor)
    return fail(QBXFMM_ERR_UNSUPPORTED,
                "level orders: not built for the compressed-Taylor 3D Helmholtz truncation "
                "(fmm_backend QBXFMM_BACKEND_FMMLIB supports them)");
  if (all_max) {
    p->lorders.clear();
    return QBXFMM_OK;
  }
  // boxes are numbered by level: find each level's range
  std::vector<int32_t> lv(p->geo.nboxes);
  cudaError_t e = cudaMemcpy(lv.data(), p->geo.box_levels, sizeof(int32_t) * lv.size(),
                             cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_check(e, "qbxfmm_plan_set_level_orders");
  std::vector<int32_t> starts(nlevels + 1, 0);
  for (int b = 0; b < p->geo.nboxes; ++b) {
    if (lv[b] < 0 || lv[b] >= nlevels || (b > 0 && lv[b] < lv[b - 1]))
      return fail(QBXFMM_ERR_ARG, "level orders: boxes must be numbered by level");
  }
  for (int l = 0; l <= nlevels; ++l)
    starts[l] = (int32_t)(std::lower_bound(lv.begin(), lv.end(), l) - lv.begin());
  if (!p->lorders_dev) {
    e = cudaMalloc(&p->lorders_dev, sizeof(int32_t) * 64);
    if (e != cudaSuccess) return cuda_check(e, "qbxfmm_plan_set_level_orders");
  }
  e = cudaMemcpy(p->lorders_dev, orders, sizeof(int32_t) * nlevels, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_check(e, "qbxfmm_plan_set_level_orders");
  p->lorders.assign(orders, orders + nlevels);
  p->level_box_start = starts;
  return QBXFMM_OK;
}

int qbxfmm_plan_get_level_orders(const qbxfmm_plan* p, int32_t* orders, int32_t nlevels)
{
  if (int rc = check_plan(p)) return rc;
  if (!orders || nlevels != p->geo.nlevels)
    return fail(QBXFMM_ERR_ARG, "level orders: one order per tree level expected");
  for (int l = 0; l < nlevels; ++l)
    orders[l] = p->lorders.empty() ? p->kern.fmm_order : p->lorders[l];
  return QBXFMM_OK;
}

int qbxfmm_workspace_sizes(const qbxfmm_plan* p, size_t* sizes6 /* 8 entries */)
{
  if (int rc = check_plan(p)) return rc;
  if (!sizes6) return fail(QBXFMM_ERR_ARG, "null sizes");
  const qbxfmm_geometry& g = p->geo;
  // entries 0-5 come from the one formula the allocation-free apply lays out its
  // array with
  if (int rc = qbx::plan_base_workspace_sizes(p, sizes6)) return rc;
  if (p->trans_ok) {
    int npairs = std::max(p->th.m2l_npairs, g.m2m_npairs);
    size_t o[8];
    h3_layout(p, o);
    sizes6[6] = p->h3 ? o[7] * sizeof(double) : p->m2l_aux_off + p->m2l_aux.size();
    sizes6[7] = p->h3 ? 0 : trans_scratch_bytes(p->tc, npairs, p->kern.nrhs);
  } else {
    sizes6[6] = sizes6[7] = 0;
  }
  return QBXFMM_OK;
}

int qbxfmm_precompute_translations(const qbxfmm_plan* p, const qbxfmm_workspace* ws, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (!ws) return fail(QBXFMM_ERR_ARG, "null workspace");
  if (p->h3) {
    if (!ws->translations)
      return fail(QBXFMM_ERR_ARG, "3D Helmholtz needs the translations buffer");
    double* T = (double*)ws->translations;
    size_t o[8];
    h3_layout(p, o);
    const int pf = p->kern.fmm_order, q = p->kern.qbx_order, nm = 2 * pf + 1;
    double* G = T + o[0];
    double* R = T + o[1];
    double* H = T + o[2];
    QBX_TRY(cudaMemcpyAsync(G, p->h3gaunt.data(), p->h3gaunt.size() * sizeof(double),
                            cudaMemcpyHostToDevice, S(stream)),
            "precompute_translations: Gaunt table");
    QBX_TRY(cudaMemcpyAsync(R, p->h3rot.data(), p->h3rot.size() * sizeof(double),
                            cudaMemcpyHostToDevice, S(stream)),
            "precompute_translations: rotation tables");
    QBX_TRY(cudaMemcpyAsync(H, p->h3m2l.data(), p->h3m2l.size() * sizeof(double),
                            cudaMemcpyHostToDevice, S(stream)),
            "precompute_translations: M2L tables");
    if (p->hc.taylor) {
      // M2M / L2L of the reference's default truncation, built on the host; the monomial
      // tables the L2QBXL kernel reads
      QBX_TRY(h3_taylor_translations(p->h3tp, p->tc, p->kern.k_re, p->geo.root_extent,
                                     p->geo.nlevels, T, S(stream)),
              "precompute_translations: Taylor M2M / L2L");
      QBX_TRY(cudaMemcpyAsync(T + o[5], p->h3tp.G0.data(), p->h3tp.G0.size() * sizeof(double2),
                              cudaMemcpyHostToDevice, S(stream)),
              "precompute_translations: Taylor tables");
      QBX_TRY(cudaMemcpyAsync(T + o[6], p->h3tq.Ginv.data(),
                              p->h3tq.Ginv.size() * sizeof(double2), cudaMemcpyHostToDevice,
                              S(stream)),
              "precompute_translations: Taylor tables");
      QBX_TRY(cudaStreamSynchronize(S(stream)), "precompute_translations");
    } else {
      QBX_TRY(h3_launch_trans_build(p->geo, p->tc, p->kern.k_re, G, T, S(stream)),
              "precompute_translations");
    }
    // rotation-table layout (h3_rotation_tables): start values, then isq, then rt
    const double* isq = R + (size_t)nm * (q + 1) * 4;
    const double* rt = isq + (size_t)(pf + 2) * (pf + 1);
    const double* dirs = H + (size_t)nm * nm * 4;
    const double* coaxp = dirs + 4 * (size_t)p->h3_ndir;
    QBX_TRY(h3_launch_m2l_tables(pf, p->h3_ndir, p->h3_ncoax, dirs, coaxp, H, isq, rt, G, T + o[3],
                                 reinterpret_cast<double2*>(T + o[4]), S(stream)),
            "precompute_translations: M2L tables");
    p->trans_dev = T;
    p->scratch_dev = (double*)ws->pair_scratch;
    return QBXFMM_OK;
  }
  if (!p->trans_ok || !ws->translations) return QBXFMM_OK;
  const TransAux aux = trans_aux(p, ws->translations);
  if (!p->m2l_aux.empty())
    QBX_TRY(cudaMemcpyAsync((char*)ws->translations + p->m2l_aux_off, p->m2l_aux.data(),
                            p->m2l_aux.size(), cudaMemcpyHostToDevice, S(stream)),
            "precompute_translations: M2L class maps");
  QBX_TRY(launch_trans_build(p->tc, p->m2l_sym.ncanon, aux.canon_off, (double*)ws->translations,
                             S(stream)),
          "precompute_translations");
  if (p->tf32_ok)
    QBX_TRY(launch_trans_split_tf32(p->tc, (const double*)ws->translations,
                                    reinterpret_cast<uint32_t*>((double*)ws->translations +
                                                                trans_matrix_bytes(p->tc) / sizeof(double)),
                                    S(stream)),
            "precompute_translations (TF32 planes)");
  return QBXFMM_OK;
}

}  // extern "C"

namespace {

// M2M / L2L: the FP64 matrix-vector kernels whenever the matrices are small (both
// precisions: they are latency-bound, a TF32 form would not be faster); M2L: split
// TF32 in the mixed form.  `gemm`: the translation matrices of ws are built; T32:
// their split-TF32 planes (mixed form), or NULL.
int run_m2m(const qbxfmm_plan* p, const qbxfmm_workspace* ws, const uint32_t* T32, bool gemm,
            void* stream)
{
  cudaStream_t st = S(stream);
  if (gemm && trans_mv_supported(p->tc))
    QBX_TRY(launch_m2m_mv(p->geo, p->th, p->tc, p->kern.nrhs, (const double*)ws->translations,
                          (double2*)ws->mpoles, ws->error_word, st),
            "coarsen_multipoles (matrix form)");
  else if (T32)
    QBX_TRY(launch_m2m_gemm_mixed(p->geo, p->th, p->tc, p->kern.nrhs, T32, (double2*)ws->mpoles,
                                  (double*)ws->pair_scratch, ws->error_word, st),
            "coarsen_multipoles (split TF32)");
  else if (gemm)
    QBX_TRY(launch_m2m_gemm(p->geo, p->th, p->tc, p->kern.nrhs, (const double*)ws->translations,
                            (double2*)ws->mpoles, (double*)ws->pair_scratch, ws->error_word, st),
            "coarsen_multipoles (matrix form)");
  else
    return qbxfmm_coarsen_multipoles(p, ws->mpoles, stream);
  return QBXFMM_OK;
}

int run_m2l(const qbxfmm_plan* p, const qbxfmm_workspace* ws, const uint32_t* T32, bool gemm,
            void* stream)
{
  cudaStream_t st = S(stream);
  if (T32)
    QBX_TRY(launch_m2l_gemm_mixed(p->geo, p->th, p->tc, p->kern.nrhs, T32,
                                  trans_aux(p, ws->translations), (const double2*)ws->mpoles, (double2*)ws->locals,
                                  (double*)ws->pair_scratch, ws->error_word, st),
            "multipole_to_local (split TF32)");
  else if (gemm)
    QBX_TRY(launch_m2l_gemm(p->geo, p->th, p->tc, p->kern.nrhs, (const double*)ws->translations,
                            trans_aux(p, ws->translations), (const double2*)ws->mpoles, (double2*)ws->locals,
                            (double*)ws->pair_scratch, ws->error_word, st),
            "multipole_to_local (matrix form)");
  else
    return qbxfmm_multipole_to_local(p, ws->mpoles, ws->locals, ws->error_word, stream);
  return QBXFMM_OK;
}

int run_l2l(const qbxfmm_plan* p, const qbxfmm_workspace* ws, const uint32_t* T32, bool gemm,
            void* stream)
{
  cudaStream_t st = S(stream);
  if (gemm && trans_mv_supported(p->tc))
    QBX_TRY(launch_l2l_mv(p->geo, p->th, p->tc, p->kern.nrhs, (const double*)ws->translations,
                          (double2*)ws->locals, ws->error_word, st),
            "refine_locals (matrix form)");
  else if (T32)
    QBX_TRY(launch_l2l_gemm_mixed(p->geo, p->th, p->tc, p->kern.nrhs, T32, (double2*)ws->locals,
                                  ws->error_word, st),
            "refine_locals (split TF32)");
  else if (gemm)
    QBX_TRY(launch_l2l_gemm(p->geo, p->th, p->tc, p->kern.nrhs, (const double*)ws->translations,
                            (double2*)ws->locals, ws->error_word, st),
            "refine_locals (matrix form)");
  else
    return qbxfmm_refine_locals(p, ws->locals, stream);
  return QBXFMM_OK;
}

}  // namespace

extern "C" {

int qbxfmm_apply(const qbxfmm_plan* p, const qbxfmm_upsample* up, const qbxfmm_workspace* ws,
                 const void* density, void* out, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (!up || !ws || !density || !out) return fail(QBXFMM_ERR_ARG, "null argument");
  if (!ws->strengths || !ws->mpoles || !ws->locals || !ws->qbx_exps || !ws->pot_nonqbx ||
      !ws->pot_tree)
    return fail(QBXFMM_ERR_ARG, "incomplete workspace");
  size_t sz[8];
  if (int rc = qbxfmm_workspace_sizes(p, sz)) return rc;
  // (per-level orders run the stage entries, which truncate level by level)
  const bool gemm = !p->h3 && p->trans_ok && ws->translations && ws->pair_scratch &&
                    !level_orders_on(p);
  if (p->h3) {
    if (!ws->translations)
      return fail(QBXFMM_ERR_ARG, "3D Helmholtz needs the translations buffer");
    p->trans_dev = (const double*)ws->translations;
    p->scratch_dev = (double*)ws->pair_scratch;
  }
  cudaStream_t st = S(stream);
  QBX_TRY(cudaMemsetAsync(ws->mpoles, 0, sz[1], st), "apply: clear");
  QBX_TRY(cudaMemsetAsync(ws->locals, 0, sz[2], st), "apply: clear");
  QBX_TRY(cudaMemsetAsync(ws->qbx_exps, 0, sz[3], st), "apply: clear");
  QBX_TRY(cudaMemsetAsync(ws->pot_nonqbx, 0, sz[4], st), "apply: clear");
  QBX_TRY(cudaMemsetAsync(ws->pot_tree, 0, sz[5], st), "apply: clear");
  if (ws->error_word) QBX_TRY(cudaMemsetAsync(ws->error_word, 0, sizeof(int32_t), st), "apply: clear");
  int rc;
  const uint32_t* T32 = (gemm && p->tf32_ok)
                            ? reinterpret_cast<const uint32_t*>((const double*)ws->translations +
                                                                trans_matrix_bytes(p->tc) / sizeof(double))
                            : nullptr;
  auto m2m = [&]() -> int { return run_m2m(p, ws, T32, gemm, stream); };
  auto m2l = [&]() -> int { return run_m2l(p, ws, T32, gemm, stream); };
  auto l2l = [&]() -> int { return run_l2l(p, ws, T32, gemm, stream); };
  // The stage graph of drive_fmm (fmm.py:436-588) on four streams.  Every buffer
  // that several stages add into is written by one stream at a time:
  //   caller's stream: strengths, P2M, M2M | M2L, L2L | L2P | L2QBXL, QBXL2P, assembly
  //   side[0]:         P2P, target-specific near field | M2P
  //   side[1]:         P2L
  //   side[2]:         P2QBXL | M2QBXL
  // with events: fork after the strengths; M2P and M2QBXL wait for M2M; M2L waits
  // for P2L (both add into the locals); L2P and QBXL2P wait for side[0]
  // (pot_nonqbx, pot_tree); L2QBXL waits for side[2] (the QBX expansions).  Every
  // stage adds into its outputs, so the order of the writers of one buffer does not
  // matter, only that they do not overlap.
  void* s1 = p->side[0];
  void* s2 = p->side[1];
  void* s3 = p->side[2];
  cudaStream_t side1 = p->side[0], side2 = p->side[1], side3 = p->side[2];
  const bool tsqbx = p->kern.target_specific_qbx != 0;
  bool forked = false;
  // on an error, join the side streams before returning, so that a stream capture
  // of the caller's stream stays well formed
  auto join = [&](int code) -> int {
    if (forked) {
      cudaEventRecord(p->ev_near, side1);
      cudaEventRecord(p->ev_p2l, side2);
      cudaEventRecord(p->ev_qbx, side3);
      cudaStreamWaitEvent(st, p->ev_near, 0);
      cudaStreamWaitEvent(st, p->ev_p2l, 0);
      cudaStreamWaitEvent(st, p->ev_qbx, 0);
    }
    return code;
  };
#define QBX_STEP(call)                  \
  do {                                  \
    if ((rc = (call))) return join(rc); \
  } while (0)
#define QBX_CUDA_STEP(call, what)                            \
  do {                                                       \
    if ((rc = cuda_check((call), what))) return join(rc);   \
  } while (0)
  if ((rc = qbxfmm_form_strengths(p, up, density, ws->strengths, stream))) return rc;
  QBX_CUDA_STEP(cudaEventRecord(p->ev_fork, st), "apply: fork");
  for (cudaStream_t s : {side1, side2, side3})
    QBX_CUDA_STEP(cudaStreamWaitEvent(s, p->ev_fork, 0), "apply: fork");
  forked = true;
  QBX_STEP(qbxfmm_form_locals(p, ws->strengths, ws->locals, ws->error_word, s2));
  QBX_CUDA_STEP(cudaEventRecord(p->ev_p2l, side2), "apply: P2L event");
  QBX_STEP(qbxfmm_eval_direct(p, ws->strengths, ws->pot_nonqbx, ws->error_word, s1));
  if (tsqbx) {
    QBX_STEP(qbxfmm_eval_target_specific_qbx_locals(p, ws->strengths, ws->pot_tree, ws->error_word, s1));
  } else {
    QBX_STEP(qbxfmm_form_global_qbx_locals(p, ws->strengths, ws->qbx_exps, ws->error_word, s3));
  }
  QBX_STEP(qbxfmm_form_multipoles(p, ws->strengths, ws->mpoles, stream));
  QBX_STEP(m2m());
  QBX_CUDA_STEP(cudaEventRecord(p->ev_mpoles, st), "apply: multipole event");
  QBX_CUDA_STEP(cudaStreamWaitEvent(side3, p->ev_mpoles, 0), "apply: multipole event");
  QBX_STEP(qbxfmm_translate_box_multipoles_to_qbx_local(p, ws->mpoles, ws->qbx_exps,
                                                        ws->error_word, s3));
  QBX_CUDA_STEP(cudaEventRecord(p->ev_qbx, side3), "apply: QBX-expansion event");
  QBX_CUDA_STEP(cudaStreamWaitEvent(side1, p->ev_mpoles, 0), "apply: multipole event");
  QBX_STEP(qbxfmm_eval_multipoles(p, ws->mpoles, ws->pot_nonqbx, ws->error_word, s1));
  QBX_CUDA_STEP(cudaEventRecord(p->ev_near, side1), "apply: near-field event");
  QBX_CUDA_STEP(cudaStreamWaitEvent(st, p->ev_p2l, 0), "apply: join P2L");
  QBX_STEP(m2l());
  QBX_STEP(l2l());
  QBX_CUDA_STEP(cudaStreamWaitEvent(st, p->ev_near, 0), "apply: join near field");
  QBX_STEP(qbxfmm_eval_locals(p, ws->locals, ws->pot_nonqbx, stream));
  QBX_CUDA_STEP(cudaStreamWaitEvent(st, p->ev_qbx, 0), "apply: join QBX expansions");
  forked = false;
#undef QBX_STEP
#undef QBX_CUDA_STEP
  if ((rc = qbxfmm_translate_box_local_to_qbx_local(p, ws->locals, ws->qbx_exps, stream))) return rc;
  if ((rc = qbxfmm_eval_qbx_expansions(p, ws->qbx_exps, ws->pot_tree, stream))) return rc;
  return qbxfmm_assemble(p, ws->pot_nonqbx, ws->pot_tree, out, stream);
}

int qbxfmm_eval_target_gradients(const qbxfmm_plan* p, const void* strengths, const void* mpoles,
                                  const void* locals, void* grad, int32_t* err, void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->helm || p->sc.cd != 0.0)
    return fail(QBXFMM_ERR_UNSUPPORTED, "target gradients cover the Laplace single layer");
  if (level_orders_on(p))
    return fail(QBXFMM_ERR_UNSUPPORTED, "target gradients take one FMM order");
  if (!strengths || !mpoles || !locals || !grad) return fail(QBXFMM_ERR_ARG, "null argument");
  const int dim = p->kern.dim;
  size_t bytes = (size_t)p->kern.nrhs * dim * p->geo.nfiltered_targets * sizeof(double);
  if (bytes) QBX_TRY(cudaMemsetAsync(grad, 0, bytes, S(stream)), "eval_target_gradients: clear");
  if (dim == 2)
    QBX_TRY(launch_grad2_targets(p->geo, p->sc.cq, -0.5 / M_PI, p->kern.fmm_order, p->kern.nrhs,
                                 (const double*)strengths, (const double2*)mpoles,
                                 (const double2*)locals, (double*)grad, err, S(stream)),
            "eval_target_gradients");
  else
    QBX_TRY(launch_grad_targets(p->geo, p->sc.cq, 0.25 / M_PI, p->kern.fmm_order, p->kern.nrhs,
                                (const double*)strengths, (const double2*)mpoles,
                                (const double2*)locals, (double*)grad, err, S(stream)),
            "eval_target_gradients");
  return QBXFMM_OK;
}

int qbxfmm_eval_qbx_target_gradients(const qbxfmm_plan* p, const void* strengths,
                                      const void* qbx_exps, void* grad, int32_t* err,
                                      void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (p->helm || p->sc.cd != 0.0)
    return fail(QBXFMM_ERR_UNSUPPORTED, "target gradients cover the Laplace single layer");
  if (p->kern.qbx_order > 8) return fail(QBXFMM_ERR_UNSUPPORTED, "qbx_order > 8");
  if (!strengths || !qbx_exps || !grad) return fail(QBXFMM_ERR_ARG, "null argument");
  const int dim = p->kern.dim;
  size_t bytes = (size_t)p->kern.nrhs * dim * p->geo.ntargets * sizeof(double);
  if (bytes) QBX_TRY(cudaMemsetAsync(grad, 0, bytes, S(stream)), "eval_qbx_target_gradients: clear");
  if (dim == 2)
    QBX_TRY(launch_grad2_qbx_targets(p->geo, p->sc.cq, -0.5 / M_PI, p->kern.qbx_order,
                                     p->kern.nrhs, p->kern.target_specific_qbx != 0,
                                     (const double*)strengths, (const double2*)qbx_exps,
                                     (double*)grad, err, S(stream)),
            "eval_qbx_target_gradients");
  else
    QBX_TRY(launch_grad_qbx_targets(p->geo, p->sc.cq, 0.25 / M_PI, p->kern.qbx_order,
                                    p->kern.nrhs, p->kern.target_specific_qbx != 0,
                                    (const double*)strengths, (const double2*)qbx_exps,
                                    (double*)grad, err, S(stream)),
            "eval_qbx_target_gradients");
  return QBXFMM_OK;
}

// {{{ transposed QBX stages

namespace {

int transpose_ok(const qbxfmm_plan* p, bool allow_dipole = false)
{
  if (int rc = check_plan(p)) return rc;
  if (p->helm)
    return fail(QBXFMM_ERR_UNSUPPORTED, "the transposed apply covers Laplace");
  if (p->kern.dim == 2 && p->sc.cd != 0.0)
    return fail(QBXFMM_ERR_UNSUPPORTED, "the 2D transposed apply covers the single layer");
  if (p->kern.dim == 2 && p->kern.fmm_order > 20)
    return fail(QBXFMM_ERR_UNSUPPORTED, "the 2D transposed apply takes fmm_order <= 20");
  if (p->sc.cd != 0.0 && !allow_dipole)
    return fail(QBXFMM_ERR_UNSUPPORTED,
                "the transposed stage entries cover the single layer; the double layer "
                "runs through qbxfmm_apply_transpose");
  if (p->mixed || level_orders_on(p))
    return fail(QBXFMM_ERR_UNSUPPORTED,
                "the transposed apply runs in FP64 with one FMM order");
  if (p->kern.qbx_order > 8 || p->kern.fmm_order > 21)
    return fail(QBXFMM_ERR_UNSUPPORTED, "the transposed apply takes qbx_order <= 8, fmm_order <= 21");
  return QBXFMM_OK;
}

}  // namespace

int qbxfmm_transpose_eval_qbx_expansions(const qbxfmm_plan* p, const void* target_values,
                                         void* center_mpoles, int32_t* err, void* stream)
{
  if (int rc = transpose_ok(p)) return rc;
  if (!target_values || !center_mpoles) return fail(QBXFMM_ERR_ARG, "null argument");
  size_t bytes = (size_t)p->geo.ncenters * p->kern.nrhs * p->ncq * 2 * sizeof(double);
  if (bytes) QBX_TRY(cudaMemsetAsync(center_mpoles, 0, bytes, S(stream)), "transpose: clear");
  if (p->kern.dim == 2)
    QBX_TRY(launch_tr2_stages(0, p->geo, nullptr, p->kern.fmm_order, p->kern.qbx_order,
                              p->kern.nrhs, p->sc.cq, (const double*)target_values,
                              (double2*)center_mpoles, nullptr, nullptr, err, S(stream)),
            "transpose_eval_qbx_expansions");
  else
    QBX_TRY(launch_tr_qbxl2p(p->geo, p->kern.qbx_order, p->kern.nrhs, p->sc.cq,
                             (const double*)target_values, (double2*)center_mpoles, err,
                             S(stream)),
            "transpose_eval_qbx_expansions");
  return QBXFMM_OK;
}

int qbxfmm_transpose_translate_box_local_to_qbx_local(const qbxfmm_plan* p,
                                                      const qbxfmm_transpose_index* ix,
                                                      const void* center_mpoles, void* mpoles,
                                                      int32_t* err, void* stream)
{
  if (int rc = transpose_ok(p)) return rc;
  if (!ix || !center_mpoles || !mpoles) return fail(QBXFMM_ERR_ARG, "null argument");
  if (p->kern.dim == 2)
    QBX_TRY(launch_tr2_stages(1, p->geo, ix, p->kern.fmm_order, p->kern.qbx_order, p->kern.nrhs,
                              1.0, nullptr, (double2*)center_mpoles, (double2*)mpoles, nullptr,
                              err, S(stream)),
            "transpose_translate_box_local_to_qbx_local");
  else
    QBX_TRY(launch_tr_l2qbxl(p->geo, *ix, p->kern.fmm_order, p->kern.qbx_order, p->kern.nrhs,
                             (const double2*)center_mpoles, (double2*)mpoles, err, S(stream)),
            "transpose_translate_box_local_to_qbx_local");
  return QBXFMM_OK;
}

int qbxfmm_transpose_translate_box_multipoles_to_qbx_local(const qbxfmm_plan* p,
                                                           const qbxfmm_transpose_index* ix,
                                                           const void* center_mpoles,
                                                           void* locals, int32_t* err,
                                                           void* stream)
{
  if (int rc = transpose_ok(p)) return rc;
  if (!ix || !center_mpoles || !locals) return fail(QBXFMM_ERR_ARG, "null argument");
  if (p->kern.dim == 2)
    QBX_TRY(launch_tr2_stages(2, p->geo, ix, p->kern.fmm_order, p->kern.qbx_order, p->kern.nrhs,
                              1.0, nullptr, (double2*)center_mpoles, (double2*)locals, nullptr,
                              err, S(stream)),
            "transpose_translate_box_multipoles_to_qbx_local");
  else
    QBX_TRY(launch_tr_m2qbxl(p->geo, *ix, p->kern.fmm_order, p->kern.qbx_order, p->kern.nrhs,
                             (const double2*)center_mpoles, (double2*)locals, err, S(stream)),
            "transpose_translate_box_multipoles_to_qbx_local");
  return QBXFMM_OK;
}

int qbxfmm_transpose_form_global_qbx_locals(const qbxfmm_plan* p, const qbxfmm_transpose_index* ix,
                                            const void* target_values, void* source_values,
                                            int32_t* err, void* stream)
{
  if (int rc = transpose_ok(p)) return rc;
  if (!ix || !target_values || !source_values) return fail(QBXFMM_ERR_ARG, "null argument");
  if (p->kern.dim == 2)
    QBX_TRY(launch_tr2_stages(3, p->geo, ix, p->kern.fmm_order, p->kern.qbx_order, p->kern.nrhs,
                              p->sc.cq, (const double*)target_values, nullptr, nullptr,
                              (double*)source_values, err, S(stream)),
            "transpose_form_global_qbx_locals");
  else
    QBX_TRY(launch_tr_p2qbxl(p->geo, *ix, p->kern.qbx_order, p->kern.nrhs, p->sc.cq,
                             (const double*)target_values, (double*)source_values, nullptr, err,
                             S(stream)),
            "transpose_form_global_qbx_locals");
  return QBXFMM_OK;
}

int qbxfmm_apply_transpose(const qbxfmm_plan* p, const qbxfmm_plan* d,
                           const qbxfmm_transpose_index* ix, const qbxfmm_workspace* ws,
                           const void* target_values, const void* strengths,
                           void* center_mpoles, void* grad_scratch, void* out, void* stream)
{
  if (int rc = transpose_ok(p, true)) return rc;
  if (int rc = check_plan(d)) return rc;
  if (d->helm || d->kern.dim != p->kern.dim || d->mixed || level_orders_on(d) || d->geo.ncenters != 0 ||
      d->kern.fmm_order != p->kern.fmm_order || d->kern.nrhs != p->kern.nrhs ||
      d->geo.nboxes != p->geo.nboxes || d->geo.nsources != p->geo.nfiltered_targets ||
      d->geo.ntargets != p->geo.nsources || d->sc.cq != 1.0 || d->sc.cd != 0.0)
    return fail(QBXFMM_ERR_ARG, "the second plan is not the exchanged-role plan of the first");
  const bool dip = p->sc.cd != 0.0, d2 = p->kern.dim == 2;
  if (!ix || !ws || !target_values || !strengths || !center_mpoles || !out ||
      (dip && !grad_scratch))
    return fail(QBXFMM_ERR_ARG, "null argument");
  if (!ws->mpoles || !ws->locals || !ws->pot_nonqbx || !ws->pot_tree)
    return fail(QBXFMM_ERR_ARG, "incomplete workspace");
  size_t sz[8];
  if (int rc = qbxfmm_workspace_sizes(d, sz)) return rc;
  const bool gemm = d->trans_ok && ws->translations && ws->pair_scratch;
  cudaStream_t st = S(stream);
  const int nrhs = p->kern.nrhs, q = p->kern.qbx_order;
  QBX_TRY(cudaMemsetAsync(ws->mpoles, 0, sz[1], st), "apply_transpose: clear");
  QBX_TRY(cudaMemsetAsync(ws->locals, 0, sz[2], st), "apply_transpose: clear");
  QBX_TRY(cudaMemsetAsync(ws->pot_nonqbx, 0, sz[4], st), "apply_transpose: clear");
  if (dip)
    QBX_TRY(cudaMemsetAsync(grad_scratch, 0, (size_t)nrhs * 3 * p->geo.nsources * sizeof(double),
                            st),
            "apply_transpose: clear");
  if (ws->error_word)
    QBX_TRY(cudaMemsetAsync(ws->error_word, 0, sizeof(int32_t), st), "apply_transpose: clear");
  // every value below is of the unit-charge exchanged-role potential; the layer's
  // coefficients enter once, at the sources (k_tr_combine)
  size_t cbytes = (size_t)p->geo.ncenters * nrhs * p->ncq * 2 * sizeof(double);
  if (cbytes) QBX_TRY(cudaMemsetAsync(center_mpoles, 0, cbytes, st), "apply_transpose: clear");
  if (d2)
    QBX_TRY(launch_tr2_stages(0, p->geo, nullptr, p->kern.fmm_order, q, nrhs, 1.0,
                              (const double*)target_values, (double2*)center_mpoles, nullptr,
                              nullptr, ws->error_word, st),
            "apply_transpose: center multipoles");
  else
    QBX_TRY(launch_tr_qbxl2p(p->geo, q, nrhs, 1.0, (const double*)target_values,
                             (double2*)center_mpoles, ws->error_word, st),
            "apply_transpose: center multipoles");
  // The exchanged-role stage graph on the second plan's four streams, as in
  // qbxfmm_apply, with the transposed QBX stages where their outputs are consumed:
  //   caller's stream: P2M, L2QBXL^T, M2M | M2L, L2L | L2P, gradients, combination
  //   side[0]:         P2P, P2QBXL^T | M2P
  //   side[1]:         P2L, M2QBXL^T
  // (every stage adds into its outputs; the writers of one buffer never overlap)
  cudaStream_t side1 = d->side[0], side2 = d->side[1], side3 = d->side[2];
  void* s1 = d->side[0];
  void* s2 = d->side[1];
  bool forked = false;
  int rc;
  auto join = [&](int code) -> int {
    if (forked) {
      cudaEventRecord(d->ev_near, side1);
      cudaEventRecord(d->ev_p2l, side2);
      cudaEventRecord(d->ev_qbx, side3);
      cudaStreamWaitEvent(st, d->ev_near, 0);
      cudaStreamWaitEvent(st, d->ev_p2l, 0);
      cudaStreamWaitEvent(st, d->ev_qbx, 0);
    }
    return code;
  };
#define QBX_STEP(call)                  \
  do {                                  \
    if ((rc = (call))) return join(rc); \
  } while (0)
#define QBX_CUDA_STEP(call, what)                            \
  do {                                                       \
    if ((rc = cuda_check((call), what))) return join(rc);   \
  } while (0)
  QBX_CUDA_STEP(cudaEventRecord(d->ev_fork, st), "apply_transpose: fork");
  for (cudaStream_t sx : {side1, side2, side3})
    QBX_CUDA_STEP(cudaStreamWaitEvent(sx, d->ev_fork, 0), "apply_transpose: fork");
  forked = true;
  QBX_STEP(qbxfmm_form_locals(d, strengths, ws->locals, ws->error_word, s2));
  QBX_CUDA_STEP(d2 ? launch_tr2_stages(2, p->geo, ix, p->kern.fmm_order, q, nrhs, 1.0, nullptr,
                                      (double2*)center_mpoles, (double2*)ws->locals, nullptr,
                                      ws->error_word, side2)
                   : launch_tr_m2qbxl(p->geo, *ix, p->kern.fmm_order, q, nrhs,
                                      (const double2*)center_mpoles, (double2*)ws->locals,
                                      ws->error_word, side2),
                "apply_transpose: M2QBXL^T");
  QBX_CUDA_STEP(cudaEventRecord(d->ev_p2l, side2), "apply_transpose: P2L event");
  QBX_STEP(qbxfmm_eval_direct(d, strengths, ws->pot_nonqbx, ws->error_word, s1));
  QBX_CUDA_STEP(d2 ? launch_tr2_stages(3, p->geo, ix, p->kern.fmm_order, q, nrhs, 1.0,
                                      (const double*)target_values, nullptr, nullptr,
                                      (double*)ws->pot_nonqbx, ws->error_word, side1)
                   : launch_tr_p2qbxl(p->geo, *ix, q, nrhs, 1.0, (const double*)target_values,
                                      (double*)ws->pot_nonqbx,
                                      dip ? (double*)grad_scratch : nullptr, ws->error_word,
                                      side1),
                "apply_transpose: P2QBXL^T");
  QBX_STEP(qbxfmm_form_multipoles(d, strengths, ws->mpoles, stream));
  QBX_CUDA_STEP(d2 ? launch_tr2_stages(1, p->geo, ix, p->kern.fmm_order, q, nrhs, 1.0, nullptr,
                                      (double2*)center_mpoles, (double2*)ws->mpoles, nullptr,
                                      ws->error_word, st)
                   : launch_tr_l2qbxl(p->geo, *ix, p->kern.fmm_order, q, nrhs,
                                      (const double2*)center_mpoles, (double2*)ws->mpoles,
                                      ws->error_word, st),
                "apply_transpose: L2QBXL^T");
  QBX_STEP(run_m2m(d, ws, nullptr, gemm, stream));
  QBX_CUDA_STEP(cudaEventRecord(d->ev_mpoles, st), "apply_transpose: multipole event");
  QBX_CUDA_STEP(cudaStreamWaitEvent(side1, d->ev_mpoles, 0), "apply_transpose: multipole event");
  QBX_STEP(qbxfmm_eval_multipoles(d, ws->mpoles, ws->pot_nonqbx, ws->error_word, s1));
  QBX_CUDA_STEP(cudaEventRecord(d->ev_near, side1), "apply_transpose: near-field event");
  QBX_CUDA_STEP(cudaEventRecord(d->ev_qbx, side3), "apply_transpose: idle stream");
  QBX_CUDA_STEP(cudaStreamWaitEvent(st, d->ev_p2l, 0), "apply_transpose: join P2L");
  QBX_STEP(run_m2l(d, ws, nullptr, gemm, stream));
  QBX_STEP(run_l2l(d, ws, nullptr, gemm, stream));
  QBX_CUDA_STEP(cudaStreamWaitEvent(st, d->ev_near, 0), "apply_transpose: join near field");
  QBX_CUDA_STEP(cudaStreamWaitEvent(st, d->ev_qbx, 0), "apply_transpose: join");
  QBX_STEP(qbxfmm_eval_locals(d, ws->locals, ws->pot_nonqbx, stream));
  forked = false;
#undef QBX_STEP
#undef QBX_CUDA_STEP
  // the dipole part: the gradient of the exchanged-role potential at the sources
  // (P2P, M2P, L2P differentiated there), the near-field part already added
  if (dip)
    QBX_TRY(launch_grad_targets(d->geo, 1.0, 1.0, d->kern.fmm_order, nrhs,
                                (const double*)strengths, (const double2*)ws->mpoles,
                                (const double2*)ws->locals, (double*)grad_scratch, ws->error_word,
                                st),
            "apply_transpose: gradients");
  QBX_TRY(launch_tr_combine(p->geo, nrhs, d2 ? -0.5 / M_PI : 0.25 / M_PI, p->sc.cq, p->sc.cd,
                            (const double*)ws->pot_nonqbx, dip ? (const double*)grad_scratch : nullptr,
                            (double*)out, st),
          "apply_transpose: combination");
  return QBXFMM_OK;
}

// }}}

int qbxfmm_apply_host(const qbxfmm_plan* p, const qbxfmm_upsample* up, const qbxfmm_workspace* ws,
                      const void* density_host, void* out_host, void* density_dev, void* out_dev,
                      void* stream)
{
  if (int rc = check_plan(p)) return rc;
  if (!density_host || !out_host || !density_dev || !out_dev)
    return fail(QBXFMM_ERR_ARG, "null argument");
  size_t scal = (p->kern.family == QBXFMM_LAPLACE) ? sizeof(double) : 2 * sizeof(double);
  size_t nin = (size_t)p->kern.nrhs * up->nelements * up->nodes_per_element * scal;
  size_t nout = (size_t)p->kern.nrhs * p->geo.nuser_targets * scal;
  cudaStream_t st = S(stream);
  QBX_TRY(cudaMemcpyAsync(density_dev, density_host, nin, cudaMemcpyHostToDevice, st), "apply_host: h2d");
  int rc = qbxfmm_apply(p, up, ws, density_dev, out_dev, stream);
  if (rc) return rc;
  QBX_TRY(cudaMemcpyAsync(out_host, out_dev, nout, cudaMemcpyDeviceToHost, st), "apply_host: d2h");
  QBX_TRY(cudaStreamSynchronize(st), "apply_host: sync");
  if (ws->error_word) {
    int32_t w = 0;
    QBX_TRY(cudaMemcpy(&w, ws->error_word, sizeof(int32_t), cudaMemcpyDeviceToHost), "apply_host: error word");
    if (w != 0) return fail(QBXFMM_ERR_DEVICE, "a kernel met an out-of-range index (code " + std::to_string(w) + ")");
  }
  return QBXFMM_OK;
}

}  // extern "C"
