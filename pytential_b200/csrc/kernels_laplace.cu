// Laplace QBX-FMM stage kernels (2D and 3D), float64, sm_100a.
//
// One kernel per wrangler stage of pytential's FMM driver
// (pytential/qbx/fmm.py:414-594).  Box kernels assign one CTA per box of the
// relevant traversal list and stage sources / expansions / translation tables in
// shared memory; the QBX near-field kernel assigns one CTA per chunk of centers
// that share a target box, holds each center's coefficients in registers and
// streams that box's list-1 sources through shared memory in tiles of 128.
#include <algorithm>

#include <cooperative_groups.h>

#include "laplace.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace qbx {

constexpr int NT = 128;

// {{{ strengths: upsample + weight + reorder to tree order

// get_flat_strengths_from_densities (pytential/qbx/__init__.py:1075-1096) and
// reorder_sources (pytential/qbx/fmm.py:199-200), one thread per tree source.
__global__ void __launch_bounds__(256)
k_form_strengths(int nsources, int ndofs, int npe, int nqpe,
                 const double* __restrict__ U, const double* __restrict__ qw,
                 const int32_t* __restrict__ user_source_ids,
                 const double* __restrict__ density, double* __restrict__ out)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (t >= nsources) return;
  int j = __ldg(user_source_ids + t);
  int e = j / nqpe;
  int jj = j - e * nqpe;
  const double* u = U + (size_t)jj * npe;
  const double* d = density + (size_t)r * ndofs + (size_t)e * npe;
  double acc = 0.0;
  for (int i = 0; i < npe; ++i) acc = fma(__ldg(u + i), __ldg(d + i), acc);
  out[(size_t)r * nsources + t] = acc * __ldg(qw + j);
}

// }}}

// {{{ helpers

constexpr int NW = NT / 32;     // warps per CTA
constexpr int MAXB = 128;       // list boxes staged per pass

// Warp 0 writes the running source counts of list boxes [gb, gb + nb) (nb <= 128)
// into s_pref[0..nb] and their first source into s_start; caller syncs.
QBX_D void list_prefix(const qbxfmm_geometry& g, const int32_t* __restrict__ lists, int gb,
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

// tree source index of virtual stream position v (0 <= v < s_pref[nb])
QBX_D int stream_source(int v, int nb, const int* s_pref, const int* s_start)
{
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (s_pref[mid] <= v) lo = mid;
    else hi = mid - 1;
  }
  return s_start[lo] + (v - s_pref[lo]);
}

// Stage sources [base, base + NT) of the stream into shared memory.
template <int DIM, bool NORMALS>
QBX_D void load_stream_tile(const qbxfmm_geometry& g, const double* __restrict__ st, int total,
                            int nb, int base, const int* s_pref, const int* s_start,
                            double (*s_y)[NT], double (*s_n)[NT], double* s_q)
{
  int v = base + threadIdx.x;
  if (v < total) {
    int s = stream_source(v, nb, s_pref, s_start);
    double y[3];
    load_point<DIM>(g.sources, g.nsources, s, y);
#pragma unroll
    for (int d = 0; d < DIM; ++d) s_y[d][threadIdx.x] = y[d];
    if (NORMALS) {
      double nv[3];
      load_point<DIM>(g.source_normals, g.nsources, s, nv);
#pragma unroll
      for (int d = 0; d < DIM; ++d) s_n[d][threadIdx.x] = nv[d];
    }
    s_q[threadIdx.x] = __ldg(st + s);
  }
}

// }}}

// {{{ P2M (form_multipoles, fmm.py:441-445)

// tables of R_n^m((y - c)/rho) for SUB sources at a time, one thread per column
// The per-source tables are stored entry-major, tab[entry * P2M_TS + source]: the lanes
// building one column write consecutive words, and the padded stride spreads the
// lanes that read different entries of one source over the banks.
constexpr int P2M_SUB = 16;
constexpr int P2M_TS = P2M_SUB + 1;

template <int DIM>
__global__ void __launch_bounds__(NT)
k_p2m(qbxfmm_geometry g, SourceCoeffs sc, int p, int ncf, int nrhs,
      const double* __restrict__ strengths, double2* __restrict__ mpoles)
{
  constexpr int SUB = P2M_SUB;
  constexpr int TS = P2M_TS;
  extern __shared__ double2 smem2[];
  double2* tab = smem2;                                  // [ncf][TS]
  __shared__ double s_u[SUB][3], s_n[SUB][3], s_q[SUB];

  int b = g.source_boxes[blockIdx.x];
  int r = blockIdx.y;
  double rho = level_width(g, g.box_levels[b]);
  double rinv = 1.0 / rho;
  double c[3];
  load_point<DIM>(g.box_centers, g.nboxes, b, c);
  int s0 = g.box_source_starts[b];
  int ns = g.box_source_counts_nonchild[b];
  const double* st = strengths + (size_t)r * g.nsources;
  const bool dip = sc.cd != 0.0;

  // per-thread coefficient bookkeeping (3D): table offsets of R_n^m and of the dipole
  // neighbours R_{n-1}^m, R_{n-1}^{m-1}, R_{n-1}^{m+1} (weight 0 where outside the
  // table; R_{n-1}^{-1} = -conj(R_{n-1}^1))
  int o_nm[2], o_a[2], o_b[2], o_c[2];
  double w_a[2], w_b[2], w_c[2];
  bool valid[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int ci = threadIdx.x + h * NT;
    valid[h] = ci < ncf;
    o_nm[h] = o_a[h] = o_b[h] = o_c[h] = 0;
    w_a[h] = w_b[h] = w_c[h] = 0.0;
    if (DIM == 3 && valid[h]) {
      int n, m;
      decode3(ci, n, m);
      o_nm[h] = idx3(n, m) * TS;
      if (n >= 1) {
        if (m <= n - 1) { o_a[h] = idx3(n - 1, m) * TS; w_a[h] = 1.0; }
        if (m >= 1) { o_b[h] = idx3(n - 1, m - 1) * TS; w_b[h] = 1.0; }
        else if (n - 1 >= 1) { o_b[h] = idx3(n - 1, 1) * TS; w_b[h] = -1.0; }
        if (m + 1 <= n - 1) { o_c[h] = idx3(n - 1, m + 1) * TS; w_c[h] = 1.0; }
      }
    }
  }

  double2 acc[2] = {c2(0.0), c2(0.0)};
  for (int base = 0; base < ns; base += SUB) {
    int cnt = min(SUB, ns - base);
    if (threadIdx.x < cnt) {
      int s = s0 + base + threadIdx.x;
      double y[3];
      load_point<DIM>(g.sources, g.nsources, s, y);
#pragma unroll
      for (int d = 0; d < DIM; ++d) s_u[threadIdx.x][d] = (y[d] - c[d]) * rinv;
      if (dip) {
        double nv[3];
        load_point<DIM>(g.source_normals, g.nsources, s, nv);
#pragma unroll
        for (int d = 0; d < DIM; ++d) s_n[threadIdx.x][d] = nv[d];
      }
      s_q[threadIdx.x] = __ldg(st + s);
    }
    __syncthreads();
    if (DIM == 3) {
      for (int w = threadIdx.x; w < cnt * (p + 1); w += NT) {
        int m = w / cnt, j = w - m * cnt;
        // column m of R for source j
        double x = s_u[j][0], y = s_u[j][1], z = s_u[j][2];
        double r2 = x * x + y * y + z * z;
        double2 a = c2(1.0);
        for (int k = 1; k <= m; ++k) a = cscale(0.5 * rcp(k), cmul(a, c2(x, y)));
        double2* T = tab + j;
        T[idx3(m, m) * TS] = a;
        double2 prev = c2(0.0);
        for (int n = m + 1; n <= p; ++n) {
          double2 bb = cscale(rcp(n + m) * rcp(n - m),
                              csub(cscale((2.0 * n - 1) * z, a), cscale(r2, prev)));
          T[idx3(n, m) * TS] = bb;
          prev = a;
          a = bb;
        }
      }
    } else {
      for (int j = threadIdx.x; j < cnt; j += NT) {
        double2 u = c2(s_u[j][0], s_u[j][1]);
        double2* T = tab + j;
        double2 a = c2(1.0);
        for (int k = 0; k <= p; ++k) {
          T[k * TS] = a;  // u^k
          a = cmul(a, u);
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (!valid[h]) continue;
      int ci = threadIdx.x + h * NT;
      double2 a = acc[h];
      if (DIM == 3) {
        for (int j = 0; j < cnt; ++j) {
          const double2* T = tab + j;
          double q = s_q[j];
          a = caxpy(sc.cq * q, cconj(T[o_nm[h]]), a);
          if (dip) {
            double f = sc.cd * q * rinv;
            double dx = s_n[j][0], dy = s_n[j][1], dz = s_n[j][2];
            // conj(dz R_{n-1}^m + (dx+idy)/2 R_{n-1}^{m-1} - (dx-idy)/2 R_{n-1}^{m+1})
            double2 tb_ = T[o_b[h]];
            if (w_b[h] < 0) tb_ = c2(-tb_.x, tb_.y);
            else tb_ = cscale(w_b[h], tb_);
            double2 v = cscale(dz * w_a[h], T[o_a[h]]);
            v = cfma(c2(0.5 * dx, 0.5 * dy), tb_, v);
            v = cfma(c2(-0.5 * dx * w_c[h], 0.5 * dy * w_c[h]), T[o_c[h]], v);
            a = caxpy(f, cconj(v), a);
          }
        }
      } else {
        int k = ci;
        for (int j = 0; j < cnt; ++j) {
          const double2* T = tab + j;
          double q = s_q[j];
          if (k == 0) {
            a.x += sc.cq * q;
          } else {
            a = caxpy(-sc.cq * q * rcp(k), T[k * TS], a);
            if (dip) {
              double2 nu = c2(s_n[j][0], s_n[j][1]);
              a = cfma(cscale(-sc.cd * q * rinv, nu), T[(k - 1) * TS], a);
            }
          }
        }
      }
      acc[h] = a;
    }
    __syncthreads();
  }
  double2* M = mpoles + ((size_t)b * nrhs + r) * ncf;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int ci = threadIdx.x + h * NT;
    if (ci < ncf) M[ci] = cadd(M[ci], acc[h]);
  }
}

// }}}

// {{{ M2M (coarsen_multipoles, fmm.py:451-455), one launch per parent level

template <int DIM>
__global__ void __launch_bounds__(NT)
k_m2m(qbxfmm_geometry g, int p, int ncf, int nrhs, int i0, double2* __restrict__ mpoles)
{
  extern __shared__ double2 smem2[];
  double2* tab = smem2;          // [ncf] R table / powers
  double2* Min = smem2 + ncf;    // [ncf]
  int b = g.source_parent_boxes[i0 + blockIdx.x];
  int r = blockIdx.y;
  int lev = g.box_levels[b];
  double rho_p = level_width(g, lev), rho_c = level_width(g, lev + 1);
  double ratio = rho_c / rho_p;
  double cp[3];
  load_point<DIM>(g.box_centers, g.nboxes, b, cp);
  double2 acc[2] = {c2(0.0), c2(0.0)};
  const int nch = 1 << DIM;
  for (int ci = 0; ci < nch; ++ci) {
    int ch = g.box_child_ids[(size_t)ci * g.nboxes + b];
    if (ch == 0 || g.box_source_counts_cumul[ch] == 0) continue;
    double cc[3], d[3];
    load_point<DIM>(g.box_centers, g.nboxes, ch, cc);
#pragma unroll
    for (int k = 0; k < DIM; ++k) d[k] = (cc[k] - cp[k]) / rho_p;
    const double2* src = mpoles + ((size_t)ch * nrhs + r) * ncf;
    for (int i = threadIdx.x; i < ncf; i += NT) Min[i] = src[i];
    if (DIM == 3) {
      sh3_R_table(p, d[0], d[1], d[2], tab, threadIdx.x, NT);
    } else if (threadIdx.x == 0) {
      double2 t = c2(d[0], d[1]), a = c2(1.0);
      for (int k = 0; k <= p; ++k) {
        tab[k] = a;
        a = cmul(a, t);
      }
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      int o = threadIdx.x + h * NT;
      if (o >= ncf) break;
      double2 a = acc[h];
      if (DIM == 3) {
        int n, m;
        decode3(o, n, m);
        double rk = 1.0;
        for (int k = 0; k <= n; ++k, rk *= ratio)
          for (int l = -k; l <= k; ++l) {
            int dm = m - l;
            if (dm > n - k || -dm > n - k) continue;
            a = cfmac(cscale(rk, sh3_get(Min, k, l)), sh3_get(tab, n - k, dm), a);
          }
      } else {
        int l = o;
        if (l == 0) {
          a = cadd(a, Min[0]);
        } else {
          a = cfma(cscale(-rcp(l), Min[0]), tab[l], a);
          double rk = ratio, bin = 1.0;  // C(l-1, k-1)
          for (int k = 1; k <= l; ++k) {
            a = cfma(cscale(rk * bin, Min[k]), tab[l - k], a);
            rk *= ratio;
            bin = bin * (l - k) * rcp(k);
          }
        }
      }
      acc[h] = a;
    }
    __syncthreads();
  }
  double2* M = mpoles + ((size_t)b * nrhs + r) * ncf;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int o = threadIdx.x + h * NT;
    if (o < ncf) M[o] = cadd(M[o], acc[h]);
  }
}

// }}}

// {{{ M2L (multipole_to_local, fmm.py:472-478), one CTA per target-or-parent box

// 3D: L_j^i = (-1)^j / rho sum_{k<=p, |l|<=k} M_k^l S_{k+j}^{l+i}(d).  Batches of PB
// list-2 pairs: the singular-harmonic tables (rows 0..2p, columns -p..2p) and the
// multipoles (rows 0..p, columns -p..p) are expanded into zero-padded dense arrays
// in shared memory, so the inner product is branch-free.  Each output's sum is
// split over two threads (k ranges with about equal term counts).
__global__ void __launch_bounds__(NT)
k_m2l3(qbxfmm_geometry g, int p, int ncf, int nrhs, int pb_max, const double2* __restrict__ mpoles,
       double2* __restrict__ locals, int32_t* err)
{
  extern __shared__ double2 smem2[];
  const int SW = 3 * p + 1, SR = 2 * p + 1, SS = SR * SW;   // S table
  const int MW = 2 * p + 1, MS = (p + 1) * MW;              // M table
  double2* Spad = smem2;                                    // [pb_max][SS]
  double2* Mpad = Spad + (size_t)pb_max * SS;               // [pb_max][MS]
  double2* red = Mpad + (size_t)pb_max * MS;                // [ncf]
  __shared__ int s_sb[8];
  __shared__ double s_d[8][3];

  int i = blockIdx.x;
  int tb = g.target_or_target_parent_boxes[i];
  int r = blockIdx.y;
  double rho = level_width(g, g.box_levels[tb]);
  double ct[3];
  load_point<3>(g.box_centers, g.nboxes, tb, ct);

  for (int q = threadIdx.x; q < pb_max * (SS + MS); q += NT) smem2[q] = c2(0.0);

  // k split point: first half takes rows 0..ksplit-1
  int ksplit = 0;
  {
    int half = (p + 1) * (p + 1) / 2, cum = 0;
    while (ksplit <= p && cum + ksplit <= half) cum += 2 * ksplit + 1, ++ksplit;
  }
  double2 acc[2] = {c2(0.0), c2(0.0)};
  int l0 = g.list2_starts[i], l1 = g.list2_starts[i + 1];
  for (int lb = l0; lb < l1; lb += pb_max) {
    int nbat = min(pb_max, l1 - lb);
    __syncthreads();
    if (threadIdx.x < nbat) {
      int sb = g.list2_lists[lb + threadIdx.x];
      if ((unsigned)sb >= (unsigned)g.nboxes) {
        report(err, QBX_DEVERR_BAD_BOX);
        sb = -1;
      }
      s_sb[threadIdx.x] = sb;
      if (sb >= 0) {
        double cs[3];
        load_point<3>(g.box_centers, g.nboxes, sb, cs);
        for (int d = 0; d < 3; ++d) s_d[threadIdx.x][d] = (ct[d] - cs[d]) / rho;
      }
    }
    __syncthreads();
    // S tables: one thread per (pair, column m in 0..2p); negative columns by symmetry
    for (int w = threadIdx.x; w < nbat * (2 * p + 1); w += NT) {
      int b = w / (2 * p + 1), m = w - b * (2 * p + 1);
      double2* S = Spad + (size_t)b * SS;
      if (s_sb[b] < 0) {
        for (int n = m; n <= 2 * p; ++n) {
          S[n * SW + p + m] = c2(0.0);
          if (m >= 1 && m <= p) S[n * SW + p - m] = c2(0.0);
        }
        continue;
      }
      double x = s_d[b][0], y = s_d[b][1], z = s_d[b][2];
      double rinv2 = 1.0 / (x * x + y * y + z * z);
      double2 a = c2(sqrt(rinv2));
      for (int k = 1; k <= m; ++k) a = cscale((2.0 * k - 1) * rinv2, cmul(a, c2(x, y)));
      double2 prev = c2(0.0);
      for (int n = m; n <= 2 * p; ++n) {
        if (n > m) {
          double2 bb = cscale(rinv2, csub(cscale((2.0 * n - 1) * z, a),
                                          cscale((double)(n + m - 1) * (n - m - 1), prev)));
          prev = a;
          a = bb;
        }
        S[n * SW + p + m] = a;
        if (m >= 1 && m <= p) S[n * SW + p - m] = (m & 1) ? c2(-a.x, a.y) : c2(a.x, -a.y);
      }
    }
    // M tables
    for (int w = threadIdx.x; w < nbat * ncf; w += NT) {
      int b = w / ncf, c = w - b * ncf;
      int k, l;
      decode3(c, k, l);
      double2 v = c2(0.0);
      if (s_sb[b] >= 0) v = mpoles[((size_t)s_sb[b] * nrhs + r) * ncf + c];
      double2* M = Mpad + (size_t)b * MS;
      M[k * MW + p + l] = v;
      if (l > 0) M[k * MW + p - l] = (l & 1) ? c2(-v.x, v.y) : c2(v.x, -v.y);
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      int job = threadIdx.x + h * NT;
      if (job >= 2 * ncf) break;
      int o = job >> 1, half = job & 1;
      int j, ii;
      decode3(o, j, ii);
      int k0 = half ? ksplit : 0, k1 = half ? p + 1 : ksplit;
      double2 a = acc[h];
      for (int b = 0; b < nbat; ++b) {
        const double2* M = Mpad + (size_t)b * MS;
        const double2* S = Spad + (size_t)b * SS;
        for (int k = k0; k < k1; ++k) {
          const double2* mrow = M + k * MW + p - k;
          const double2* srow = S + (k + j) * SW + p + ii - k;
          for (int l = 0; l <= 2 * k; ++l) a = cfma(mrow[l], srow[l], a);
        }
      }
      acc[h] = a;
    }
  }
  // combine the two halves of each output
  __syncthreads();
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int job = threadIdx.x + h * NT;
    if (job < 2 * ncf && (job & 1)) red[job >> 1] = acc[h];
  }
  __syncthreads();
  double2* L = locals + ((size_t)tb * nrhs + r) * ncf;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int job = threadIdx.x + h * NT;
    if (job < 2 * ncf && !(job & 1)) {
      int o = job >> 1;
      int j, ii;
      decode3(o, j, ii);
      double2 v = cadd(acc[h], red[o]);
      L[o] = caxpy((j & 1) ? -1.0 / rho : 1.0 / rho, v, L[o]);
    }
  }
}

// 2D: L_0 = M_0 log t + sum_k M_k tau^-k,
//     L_l = (-1)^(l+1) M_0 / (l tau^l) + (-1)^l tau^-l sum_k M_k C(k+l-1, l) tau^-k.
__global__ void __launch_bounds__(NT)
k_m2l2(qbxfmm_geometry g, int p, int ncf, int nrhs, const double2* __restrict__ mpoles,
       double2* __restrict__ locals, int32_t* err)
{
  extern __shared__ double2 smem2[];
  double2* Min = smem2;             // [ncf]
  double2* tab = smem2 + ncf;       // [2p+2]
  int i = blockIdx.x;
  int tb = g.target_or_target_parent_boxes[i];
  int r = blockIdx.y;
  double rho = level_width(g, g.box_levels[tb]);
  double ct[3];
  load_point<2>(g.box_centers, g.nboxes, tb, ct);
  double2 acc = c2(0.0);
  int l0 = g.list2_starts[i], l1 = g.list2_starts[i + 1];
  for (int li = l0; li < l1; ++li) {
    int sb = g.list2_lists[li];
    if ((unsigned)sb >= (unsigned)g.nboxes) {
      report(err, QBX_DEVERR_BAD_BOX);
      continue;
    }
    double cs[3];
    load_point<2>(g.box_centers, g.nboxes, sb, cs);
    double d0 = (ct[0] - cs[0]) / rho, d1 = (ct[1] - cs[1]) / rho;
    const double2* src = mpoles + ((size_t)sb * nrhs + r) * ncf;
    for (int q = threadIdx.x; q < ncf; q += NT) Min[q] = src[q];
    if (threadIdx.x == 0) {
      double2 tinv = cinv(c2(d0, d1)), a = tinv;
      tab[0] = clog_(c2(d0 * rho, d1 * rho));
      for (int k = 1; k <= 2 * p + 1; ++k) {
        tab[k] = a;  // tau^-k
        a = cmul(a, tinv);
      }
    }
    __syncthreads();
    int l = threadIdx.x;
    if (l < ncf) {
      if (l == 0) {
        double2 s = cmul(Min[0], tab[0]);
        for (int k = 1; k <= p; ++k) s = cfma(Min[k], tab[k], s);
        acc = cadd(acc, s);
      } else {
        double2 s = c2(0.0);
        double bin = 1.0;  // C(k+l-1, l) at k = 1
        for (int k = 1; k <= p; ++k) {
          s = cfma(cscale(bin, Min[k]), tab[k], s);
          bin = bin * (k + l) * rcp(k);
        }
        double2 v = cscale(((l & 1) ? 1.0 : -1.0) * rcp(l), Min[0]);
        v = cadd(v, cscale((l & 1) ? -1.0 : 1.0, s));
        acc = cfma(v, tab[l], acc);
      }
    }
    __syncthreads();
  }
  if (threadIdx.x < ncf) {
    double2* L = locals + ((size_t)tb * nrhs + r) * ncf;
    L[threadIdx.x] = cadd(L[threadIdx.x], acc);
  }
}

// }}}

// {{{ P2L (form_locals, list 4, fmm.py:502-510)

// One CTA per target-or-parent box; its list-4 sources stream through shared memory
// in sub-tiles of SUB; per sub-tile each source's singular-harmonic table (orders
// 0..p+1) is built by one thread per (source, column), then each thread accumulates
// its coefficient(s) with precomputed table offsets.  The tables are stored
// entry-major, tab[entry * P2L_TS + source], so the lanes of a warp building one
// column write consecutive words, and the lanes reading different entries of one
// source are spread over the banks by the padded stride.
constexpr int P2L_SUB = 32;
constexpr int P2L_TS = P2L_SUB + 1;

template <int DIM>
__global__ void __launch_bounds__(NT)
k_p2l(qbxfmm_geometry g, SourceCoeffs sc, int p, int ncf, int nrhs,
      const double* __restrict__ strengths, double2* __restrict__ locals, int32_t* err)
{
  constexpr int SUB = P2L_SUB;
  constexpr int TS = P2L_TS;
  extern __shared__ double2 smem2[];
  double2* tab = smem2;   // [nct][TS]
  __shared__ double s_u[SUB][3], s_n[SUB][3], s_q[SUB];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];
  int i = blockIdx.x;
  int tb = g.target_or_target_parent_boxes[i];
  int r = blockIdx.y;
  double rho = level_width(g, g.box_levels[tb]);
  double rinv = 1.0 / rho;
  double c[3];
  load_point<DIM>(g.box_centers, g.nboxes, tb, c);
  const double* st = strengths + (size_t)r * g.nsources;
  const bool dip = sc.cd != 0.0;

  // per-thread coefficient bookkeeping (3D): table offsets of S_n^m and the
  // dipole neighbours S_{n+1}^{m-1}, S_{n+1}^m, S_{n+1}^{m+1}
  int o_nm[2], o_a[2], o_b[2], o_c[2];
  double sb_sign[2];
  bool valid[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int ci = threadIdx.x + h * NT;
    valid[h] = ci < ncf;
    o_nm[h] = o_a[h] = o_b[h] = o_c[h] = 0;
    sb_sign[h] = 1.0;
    if (DIM == 3 && valid[h]) {
      int n, m;
      decode3(ci, n, m);
      o_nm[h] = idx3(n, m) * TS;
      o_a[h] = idx3(n + 1, m) * TS;
      o_b[h] = idx3(n + 1, m > 0 ? m - 1 : 1) * TS;   // m = 0: S_{n+1}^{-1} = -conj(S_{n+1}^1)
      sb_sign[h] = m > 0 ? 1.0 : -1.0;
      o_c[h] = idx3(n + 1, m + 1) * TS;
    }
  }

  double2 acc[2] = {c2(0.0), c2(0.0)};
  int l0 = g.list4_starts[i], l1 = g.list4_starts[i + 1];
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    list_prefix(g, g.list4_lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += SUB) {
      int cnt = min(SUB, total - base);
      if (threadIdx.x < cnt) {
        int s = stream_source(base + threadIdx.x, nb, s_pref, s_start);
        double y[3];
        load_point<DIM>(g.sources, g.nsources, s, y);
#pragma unroll
        for (int d = 0; d < DIM; ++d) s_u[threadIdx.x][d] = (y[d] - c[d]) * rinv;
        if (dip) {
          double nv[3];
          load_point<DIM>(g.source_normals, g.nsources, s, nv);
#pragma unroll
          for (int d = 0; d < DIM; ++d) s_n[threadIdx.x][d] = nv[d];
        }
        s_q[threadIdx.x] = __ldg(st + s);
      }
      __syncthreads();
      if (DIM == 3) {
        for (int w = threadIdx.x; w < cnt * (p + 2); w += NT) {
          int m = w / cnt, j = w - m * cnt;
          double x = s_u[j][0], y = s_u[j][1], z = s_u[j][2];
          double rinv2 = 1.0 / (x * x + y * y + z * z);
          double2 a = c2(sqrt(rinv2));
          for (int k = 1; k <= m; ++k) a = cscale((2.0 * k - 1) * rinv2, cmul(a, c2(x, y)));
          double2* T = tab + j;
          T[idx3(m, m) * TS] = a;
          double2 prev = c2(0.0);
          for (int n = m + 1; n <= p + 1; ++n) {
            double2 bb = cscale(rinv2, csub(cscale((2.0 * n - 1) * z, a),
                                            cscale((double)(n + m - 1) * (n - m - 1), prev)));
            T[idx3(n, m) * TS] = bb;
            prev = a;
            a = bb;
          }
        }
      } else {
        for (int j = threadIdx.x; j < cnt; j += NT) {
          double2 tinv = cinv(c2(s_u[j][0], s_u[j][1]));
          double2* T = tab + j;
          double2 a = c2(1.0);
          for (int k = 0; k <= p + 1; ++k) {
            T[k * TS] = a;   // tau^-k
            a = cmul(a, tinv);
          }
          T[(p + 2) * TS] =
              c2(0.5 * log((s_u[j][0] * s_u[j][0] + s_u[j][1] * s_u[j][1]) * rho * rho));
        }
      }
      __syncthreads();
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (!valid[h]) continue;
        int ci = threadIdx.x + h * NT;
        double2 a = acc[h];
        for (int j = 0; j < cnt; ++j) {
          const double2* T = tab + j;
          double q = s_q[j];
          if (DIM == 3) {
            a = caxpy(sc.cq * q * rinv, T[o_nm[h]], a);
            if (dip) {
              double f = sc.cd * q * rinv * rinv;
              double dx = s_n[j][0], dy = s_n[j][1], dz = s_n[j][2];
              double2 tb_ = T[o_b[h]];
              if (sb_sign[h] < 0) tb_ = c2(-tb_.x, tb_.y);
              double2 v = cscale(-dz, T[o_a[h]]);
              v = cfma(c2(0.5 * dx, 0.5 * dy), tb_, v);
              v = cfma(c2(-0.5 * dx, 0.5 * dy), T[o_c[h]], v);
              a = caxpy(f, v, a);
            }
          } else {
            int l = ci;
            if (l == 0) a.x += sc.cq * q * T[(p + 2) * TS].x;
            else a = caxpy(-sc.cq * q * rcp(l), T[l * TS], a);
            if (dip) {
              double2 nu = c2(s_n[j][0], s_n[j][1]);
              a = cfma(cscale(sc.cd * q * rinv, nu), T[(l + 1) * TS], a);
            }
          }
        }
        acc[h] = a;
      }
      __syncthreads();
    }
  }
  double2* L = locals + ((size_t)tb * nrhs + r) * ncf;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int o = threadIdx.x + h * NT;
    if (o < ncf) L[o] = cadd(L[o], acc[h]);
  }
}

// }}}

// 3D P2L with every coefficient split over two threads: a block of
// P2L3_SPLIT x ncf threads (rounded up to whole warps) takes, per 32-source tile, the
// sources [0, 16) in the first half of the threads and [16, 32) in the second, so no
// thread waits idle through the accumulation (with one thread per coefficient, 62 of
// 128 threads had nothing to accumulate at p = 10).  All threads build the tile's
// harmonic tables; the halves are added in shared memory at the end.
constexpr int P2L3_SPLIT = 2;
constexpr int P2L3_MAXT = 256;

__global__ void __launch_bounds__(P2L3_MAXT)
k_p2l3s(qbxfmm_geometry g, SourceCoeffs sc, int p, int ncf, int nrhs,
        const double* __restrict__ strengths, double2* __restrict__ locals, int32_t* err)
{
  constexpr int SUB = P2L_SUB;
  constexpr int TS = P2L_TS;
  constexpr int HALF = SUB / P2L3_SPLIT;
  extern __shared__ double2 smem2[];
  double2* tab = smem2;   // [nct][TS]
  __shared__ double s_u[SUB][3], s_n[SUB][3], s_q[SUB];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];
  const int nthr = blockDim.x;
  int i = blockIdx.x;
  int tb = g.target_or_target_parent_boxes[i];
  int r = blockIdx.y;
  double rho = level_width(g, g.box_levels[tb]);
  double rinv = 1.0 / rho;
  double c[3];
  load_point<3>(g.box_centers, g.nboxes, tb, c);
  const double* st = strengths + (size_t)r * g.nsources;
  const bool dip = sc.cd != 0.0;

  // this thread's coefficient (n, m) and source half; table offsets of S_n^m and of
  // the dipole neighbours S_{n+1}^{m-1}, S_{n+1}^m, S_{n+1}^{m+1}
  const bool active = (int)threadIdx.x < P2L3_SPLIT * ncf;
  const int ci = active ? (int)threadIdx.x % ncf : 0;
  const int half = active ? (int)threadIdx.x / ncf : 0;
  int n, m;
  decode3(ci, n, m);
  const int o_nm = idx3(n, m) * TS;
  const int o_a = idx3(n + 1, m) * TS;
  const int o_b = idx3(n + 1, m > 0 ? m - 1 : 1) * TS;   // m = 0: S_{n+1}^{-1} = -conj(S_{n+1}^1)
  const double sb_sign = m > 0 ? 1.0 : -1.0;
  const int o_c = idx3(n + 1, m + 1) * TS;

  double2 acc = c2(0.0);
  int l0 = g.list4_starts[i], l1 = g.list4_starts[i + 1];
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    list_prefix(g, g.list4_lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += SUB) {
      int cnt = min(SUB, total - base);
      if ((int)threadIdx.x < cnt) {
        int s = stream_source(base + threadIdx.x, nb, s_pref, s_start);
        double y[3];
        load_point<3>(g.sources, g.nsources, s, y);
#pragma unroll
        for (int d = 0; d < 3; ++d) s_u[threadIdx.x][d] = (y[d] - c[d]) * rinv;
        if (dip) {
          double nv[3];
          load_point<3>(g.source_normals, g.nsources, s, nv);
#pragma unroll
          for (int d = 0; d < 3; ++d) s_n[threadIdx.x][d] = nv[d];
        }
        s_q[threadIdx.x] = __ldg(st + s);
      }
      __syncthreads();
      for (int w = threadIdx.x; w < cnt * (p + 2); w += nthr) {
        int mm = w / cnt, j = w - mm * cnt;
        double x = s_u[j][0], yy = s_u[j][1], z = s_u[j][2];
        double rinv2 = 1.0 / (x * x + yy * yy + z * z);
        double2 a = c2(sqrt(rinv2));
        for (int k = 1; k <= mm; ++k) a = cscale((2.0 * k - 1) * rinv2, cmul(a, c2(x, yy)));
        double2* T = tab + j;
        T[idx3(mm, mm) * TS] = a;
        double2 prev = c2(0.0);
        for (int nn = mm + 1; nn <= p + 1; ++nn) {
          double2 bb = cscale(rinv2, csub(cscale((2.0 * nn - 1) * z, a),
                                          cscale((double)(nn + mm - 1) * (nn - mm - 1), prev)));
          T[idx3(nn, mm) * TS] = bb;
          prev = a;
          a = bb;
        }
      }
      __syncthreads();
      if (active) {
        int jend = min(cnt, (half + 1) * HALF);
        for (int j = half * HALF; j < jend; ++j) {
          const double2* T = tab + j;
          double q = s_q[j];
          acc = caxpy(sc.cq * q * rinv, T[o_nm], acc);
          if (dip) {
            double f = sc.cd * q * rinv * rinv;
            double dx = s_n[j][0], dy = s_n[j][1], dz = s_n[j][2];
            double2 tb_ = T[o_b];
            if (sb_sign < 0) tb_ = c2(-tb_.x, tb_.y);
            double2 v = cscale(-dz, T[o_a]);
            v = cfma(c2(0.5 * dx, 0.5 * dy), tb_, v);
            v = cfma(c2(-0.5 * dx, 0.5 * dy), T[o_c], v);
            acc = caxpy(f, v, acc);
          }
        }
      }
      __syncthreads();
    }
  }
  // the second half's sums through the (now free) table space
  if (active && half == 1) tab[ci] = acc;
  __syncthreads();
  if (active && half == 0) {
    double2* L = locals + ((size_t)tb * nrhs + r) * ncf;
    L[ci] = cadd(L[ci], cadd(acc, tab[ci]));
  }
}

// {{{ L2L (refine_locals, fmm.py:519-523), one launch per child level

template <int DIM>
__global__ void __launch_bounds__(NT)
k_l2l(qbxfmm_geometry g, int p, int ncf, int nrhs, int i0, double2* __restrict__ locals)
{
  extern __shared__ double2 smem2[];
  double2* tab = smem2;
  double2* Lin = smem2 + ncf;
  int b = g.target_or_target_parent_boxes[i0 + blockIdx.x];
  int r = blockIdx.y;
  int par = g.box_parent_ids[b];
  int lev = g.box_levels[b];
  double rho_p = level_width(g, lev - 1), rho_c = level_width(g, lev);
  double ratio = rho_c / rho_p;
  double cp[3], cc[3], d[3];
  load_point<DIM>(g.box_centers, g.nboxes, par, cp);
  load_point<DIM>(g.box_centers, g.nboxes, b, cc);
#pragma unroll
  for (int k = 0; k < DIM; ++k) d[k] = (cc[k] - cp[k]) / rho_p;
  const double2* src = locals + ((size_t)par * nrhs + r) * ncf;
  for (int q = threadIdx.x; q < ncf; q += NT) Lin[q] = src[q];
  if (DIM == 3) {
    sh3_R_table(p, d[0], d[1], d[2], tab, threadIdx.x, NT);
  } else if (threadIdx.x == 0) {
    double2 s = c2(d[0], d[1]), a = c2(1.0);
    for (int k = 0; k <= p; ++k) {
      tab[k] = a;
      a = cmul(a, s);
    }
  }
  __syncthreads();
  double2* L = locals + ((size_t)b * nrhs + r) * ncf;
  for (int o = threadIdx.x; o < ncf; o += NT) {
    double2 a = c2(0.0);
    if (DIM == 3) {
      int k, l;
      decode3(o, k, l);
      for (int n = k; n <= p; ++n)
        for (int m = -n; m <= n; ++m) {
          int dm = m - l;
          if (dm > n - k || -dm > n - k) continue;
          a = cfmac(sh3_get(Lin, n, m), sh3_get(tab, n - k, dm), a);
        }
      a = cscale(pow(ratio, (double)k), a);
    } else {
      int l = o;
      double bin = 1.0;  // C(k, l)
      for (int k = l; k <= p; ++k) {
        a = cfma(cscale(bin, Lin[k]), tab[k - l], a);
        bin = bin * (k + 1) * rcp(k + 1 - l);
      }
      a = cscale(pow(ratio, (double)l), a);
    }
    L[o] = cadd(L[o], a);
  }
}

// }}}

// {{{ point evaluations at non-QBX targets: P2P (list 1), M2P (list 3), L2P

// P2P over list 1 (eval_direct, fmm.py:461-466).  A cluster of PSPLIT CTAs serves one
// chunk of <= 32 non-QBX targets of a target box (lane = target): the list-1 sources
// stream through shared memory in tiles of 128, tile t going to CTA t % PSPLIT of the
// cluster and, within it, 32 sources to each warp.  The partial sums are combined in
// a fixed order through distributed shared memory by CTA 0 of the cluster.
constexpr int PSPLIT = 8;

// Sum of acc over the CTA's warps and then over the cluster's CTAs, in a fixed order;
// returns the total in lane t of warp 0 of CTA 0 (other threads: unspecified).
QBX_D double cluster_lane_sum(double acc, double (*s_red)[32], double* s_part)
{
  cg::cluster_group cl = cg::this_cluster();
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (warp > 0) s_red[warp - 1][lane] = acc;
  __syncthreads();
  if (warp == 0) {
    for (int w = 1; w < NW; ++w) acc += s_red[w - 1][lane];
    s_part[lane] = acc;
  }
  cl.sync();
  if (cl.block_rank() == 0 && warp == 0) {
    for (unsigned q = 1; q < cl.num_blocks(); ++q) acc += *cl.map_shared_rank(s_part + lane, q);
  }
  cl.sync();
  return acc;
}

template <int DIM>
__global__ void __cluster_dims__(PSPLIT, 1, 1) __launch_bounds__(NT)
k_eval_direct(qbxfmm_geometry g, SourceCoeffs sc, int nrhs, const double* __restrict__ strengths,
              double* __restrict__ pot, int32_t* err)
{
  __shared__ double s_y[3][NT], s_n[3][NT], s_q[NT];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];
  __shared__ double s_red[NW - 1][32];
  __shared__ double s_part[32];
  int chunk = blockIdx.x / PSPLIT;
  int part = blockIdx.x - chunk * PSPLIT;
  int r = blockIdx.y;
  int itb = g.nonqbx_chunk_target_box[chunk];
  int t0 = g.nonqbx_chunk_start[chunk];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bool active = lane < g.nonqbx_chunk_count[chunk];
  int t = t0 + lane;
  double x[3] = {0, 0, 0};
  if (active) load_point<DIM>(g.nonqbx_targets, g.nfiltered_targets, t, x);
  const double* st = strengths + (size_t)r * g.nsources;
  const bool dip = sc.cd != 0.0;
  double acc = 0.0;
  int l0 = g.list1_starts[itb], l1 = g.list1_starts[itb + 1];
  int tile = 0;
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    list_prefix(g, g.list1_lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += NT, ++tile) {
      if (tile % PSPLIT != part) continue;
      if (dip) load_stream_tile<DIM, true>(g, st, total, nb, base, s_pref, s_start, s_y, s_n, s_q);
      else load_stream_tile<DIM, false>(g, st, total, nb, base, s_pref, s_start, s_y, s_n, s_q);
      __syncthreads();
      int jbeg = warp * 32, jend = min(jbeg + 32, total - base);
      if (active) {
        for (int j = jbeg; j < jend; ++j) {
          double dx = x[0] - s_y[0][j], dy = x[1] - s_y[1][j];
          double dz = (DIM == 3) ? x[2] - s_y[2][j] : 0.0;
          double r2 = dx * dx + dy * dy + dz * dz;
          if (r2 == 0.0) continue;
          double q = s_q[j];
          if (DIM == 3) {
            double rinv = rsqrt(r2);
            double v = sc.cq * rinv;
            if (dip)
              v += sc.cd * (s_n[0][j] * dx + s_n[1][j] * dy + s_n[2][j] * dz) * rinv * rinv * rinv;
            acc = fma(q, v, acc);
          } else {
            double v = 0.5 * sc.cq * log(r2);
            if (dip) {
              double ri = rsqrt(r2);
              v -= sc.cd * (s_n[0][j] * dx + s_n[1][j] * dy) * ri * ri;
            }
            acc = fma(q, v, acc);
          }
        }
      }
      __syncthreads();
    }
  }
  acc = cluster_lane_sum(acc, s_red, s_part);
  if (part == 0 && warp == 0 && active) pot[(size_t)r * g.nfiltered_targets + t] += acc;
}

// M2P over list 3 (eval_multipoles, fmm.py:487-493).  Same clusters; the list-3 boxes
// are dealt round-robin to the PSPLIT x 4 warps, each staging its multipole in its own
// shared slice.
template <int DIM>
__global__ void __cluster_dims__(PSPLIT, 1, 1) __launch_bounds__(NT)
k_eval_multipoles(qbxfmm_geometry g, int p, int ncf, int nrhs,
                  const double2* __restrict__ mpoles, double* __restrict__ pot, int32_t* err)
{
  extern __shared__ double2 smem2[];
  __shared__ double s_red[NW - 1][32];
  __shared__ double s_part[32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double2* M = smem2 + (size_t)warp * ncf;
  int chunk = blockIdx.x / PSPLIT;
  int part = blockIdx.x - chunk * PSPLIT;
  int r = blockIdx.y;
  int itb = g.nonqbx_chunk_target_box[chunk];
  int t = g.nonqbx_chunk_start[chunk] + lane;
  bool active = lane < g.nonqbx_chunk_count[chunk];
  double x[3] = {0, 0, 0};
  if (active) load_point<DIM>(g.nonqbx_targets, g.nfiltered_targets, t, x);
  double acc = 0.0;
  for (int li = g.list3_starts[itb] + part * NW + warp; li < g.list3_starts[itb + 1];
       li += NW * PSPLIT) {
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
    double rho = level_width(g, g.box_levels[sb]);
    double cs[3];
    load_point<DIM>(g.box_centers, g.nboxes, sb, cs);
    double u0 = (x[0] - cs[0]) / rho, u1 = (x[1] - cs[1]) / rho;
    if (DIM == 3) {
      double u2 = (x[2] - cs[2]) / rho;
      double rinv2 = 1.0 / (u0 * u0 + u1 * u1 + u2 * u2);
      double2 mm = c2(sqrt(rinv2));
      double s = 0.0;
      for (int m = 0; m <= p; ++m) {
        if (m > 0) mm = cscale((2.0 * m - 1) * rinv2, cmul(mm, c2(u0, u1)));
        double w = (m == 0) ? 1.0 : 2.0;
        double2 a = mm, prev = c2(0.0);
        const double2* mc = M + idx3(m, m);
        for (int n = m; n <= p; ++n) {
          if (n > m) {
            double2 bb = cscale(rinv2, csub(cscale((2.0 * n - 1) * u2, a),
                                            cscale((double)(n + m - 1) * (n - m - 1), prev)));
            prev = a;
            a = bb;
          }
          double2 cm = *mc;
          mc += n + 1;   // idx3(n+1, m) - idx3(n, m)
          s += w * (cm.x * a.x - cm.y * a.y);
        }
      }
      acc += s / rho;
    } else {
      double2 zc = c2(x[0] - cs[0], x[1] - cs[1]);
      double2 uinv = cinv(c2(u0, u1));
      double2 sum = cmul(M[0], clog_(zc));
      double2 pw = uinv;
      for (int k = 1; k <= p; ++k) {
        sum = cfma(M[k], pw, sum);
        pw = cmul(pw, uinv);
      }
      acc += sum.x;
    }
  }
  acc = cluster_lane_sum(acc, s_red, s_part);
  if (part == 0 && warp == 0 && active) pot[(size_t)r * g.nfiltered_targets + t] += acc;
}

template <int DIM>
__global__ void __launch_bounds__(NT)
k_eval_locals(qbxfmm_geometry g, int p, int ncf, int nrhs, const double2* __restrict__ locals,
              double* __restrict__ pot)
{
  extern __shared__ double2 smem2[];
  double2* L = smem2;
  int itb = blockIdx.x;
  int tb = g.target_boxes[itb];
  int r = blockIdx.y;
  int t0 = g.nonqbx_box_target_starts[tb];
  int nt = g.nonqbx_box_target_counts_nonchild[tb];
  if (nt == 0) return;
  const double2* src = locals + ((size_t)tb * nrhs + r) * ncf;
  for (int q = threadIdx.x; q < ncf; q += NT) L[q] = src[q];
  __syncthreads();
  double rho = level_width(g, g.box_levels[tb]);
  double cb[3];
  load_point<DIM>(g.box_centers, g.nboxes, tb, cb);
  for (int t = threadIdx.x; t < nt; t += NT) {
    double x[3];
    load_point<DIM>(g.nonqbx_targets, g.nfiltered_targets, t0 + t, x);
    double u0 = (x[0] - cb[0]) / rho, u1 = (x[1] - cb[1]) / rho;
    double acc = 0.0;
    if (DIM == 3) {
      double u2 = (x[2] - cb[2]) / rho;
      double r2 = u0 * u0 + u1 * u1 + u2 * u2;
      double2 mm = c2(1.0);
      for (int m = 0; m <= p; ++m) {
        if (m > 0) mm = cscale(0.5 * rcp(m), cmul(mm, c2(u0, u1)));
        double w = (m == 0) ? 1.0 : 2.0;
        double2 a = mm, prev = c2(0.0);
        for (int n = m; n <= p; ++n) {
          if (n > m) {
            double2 bb = cscale(rcp(n + m) * rcp(n - m),
                                csub(cscale((2.0 * n - 1) * u2, a), cscale(r2, prev)));
            prev = a;
            a = bb;
          }
          double2 cl = L[idx3(n, m)];
          acc += w * (cl.x * a.x + cl.y * a.y);   // Re(L conj(R))
        }
      }
    } else {
      double2 u = c2(u0, u1), pw = c2(1.0), sum = c2(0.0);
      for (int k = 0; k <= p; ++k) {
        sum = cfma(L[k], pw, sum);
        pw = cmul(pw, u);
      }
      acc = sum.x;
    }
    pot[(size_t)r * g.nfiltered_targets + t0 + t] += acc;
  }
}

// }}}

// {{{ QBX stages

// P2QBXL (form_global_qbx_locals, fmm.py:231-265; interactions.py:84-124).
// CTA = 4 warps over one chunk of <= 32 centers of a target box (lane = center);
// the list-1 sources stream through shared memory in tiles of 128, each warp
// taking 32 of them; the warps' partial expansions are summed at the end.
template <int DIM, int Q, bool CHG, bool DIP>
__global__ void __launch_bounds__(NT)
k_p2qbxl(qbxfmm_geometry g, SourceCoeffs sc, int nrhs, const double* __restrict__ strengths,
         double2* __restrict__ qbx_exps, int32_t* err)
{
  constexpr int NC = (DIM == 3) ? (Q + 1) * (Q + 2) / 2 : Q + 1;
  __shared__ double s_y[3][NT];
  __shared__ double s_n[3][NT];
  __shared__ double s_q[NT];
  __shared__ int s_pref[MAXB + 1];
  __shared__ int s_start[MAXB];
  extern __shared__ double2 s_red[];   // [NW-1][32][NC]

  int chunk = blockIdx.x;
  int r = blockIdx.y;
  int itb = g.qbx_chunk_target_box[chunk];
  int cstart = g.qbx_chunk_start[chunk];
  int ccount = g.qbx_chunk_count[chunk];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bool has_center = lane < ccount;
  int ctr = has_center ? g.centers_by_target_box[cstart + lane] : 0;
  if ((unsigned)ctr >= (unsigned)g.ncenters) {
    report(err, QBX_DEVERR_BAD_CENTER);
    has_center = false;
    ctr = 0;
  }
  double cc[3] = {0, 0, 0};
  load_point<DIM>(g.centers, g.ncenters, ctr, cc);
  double rho = g.expansion_radii[ctr];
  double rinv = 1.0 / rho;
  const double* st = strengths + (size_t)r * g.nsources;

  double2 acc[NC];
#pragma unroll
  for (int i = 0; i < NC; ++i) acc[i] = c2(0.0);

  int l0 = g.list1_starts[itb], l1 = g.list1_starts[itb + 1];
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    list_prefix(g, g.list1_lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += NT) {
      load_stream_tile<DIM, DIP>(g, st, total, nb, base, s_pref, s_start, s_y, s_n, s_q);
      __syncthreads();
      int jbeg = warp * 32;
      int jend = min(jbeg + 32, total - base);
      if (has_center) {
        for (int j = jbeg; j < jend; ++j) {
          double q = s_q[j];
          if (DIM == 3) {
            double ux = (s_y[0][j] - cc[0]) * rinv;
            double uy = (s_y[1][j] - cc[1]) * rinv;
            double uz = (s_y[2][j] - cc[2]) * rinv;
            double r2 = ux * ux + uy * uy + uz * uz;
            double ri = rsqrt(r2);
            double ri2 = ri * ri;
            SRegs<DIP ? Q + 1 : Q> S;
            S.build(ux, uy, uz, ri, ri2);
            double fq = sc.cq * q * rinv;
            double fd = sc.cd * q * rinv * rinv;
            double dz = fd * s_n[2][j];
            double2 dp = c2(0.5 * fd * s_n[0][j], 0.5 * fd * s_n[1][j]);
            double2 dm = c2(0.5 * fd * s_n[0][j], -0.5 * fd * s_n[1][j]);
#pragma unroll
            for (int n = 0; n <= Q; ++n)
#pragma unroll
              for (int m = 0; m <= n; ++m) {
                double2 a = acc[idx3(n, m)];
                if (CHG) a = caxpy(fq, S.v[idx3(n, m)], a);
                if (DIP) {
                  a = caxpy(-dz, S.v[idx3(n + 1, m)], a);
                  a = cfma(dp, S.get(n + 1, m - 1), a);
                  a = cfma(c2(-dm.x, -dm.y), S.v[idx3(n + 1, m + 1)], a);
                }
                acc[idx3(n, m)] = a;
              }
          } else {
            double tx = s_y[0][j] - cc[0], ty = s_y[1][j] - cc[1];
            double2 tinv = cinv(c2(tx * rinv, ty * rinv));
            double2 pw = tinv;   // tau^-l
            if (CHG) acc[0].x += sc.cq * q * 0.5 * log(tx * tx + ty * ty);
            double2 fnu = c2(sc.cd * q * rinv * s_n[0][j], sc.cd * q * rinv * s_n[1][j]);
#pragma unroll
            for (int l = 0; l <= Q; ++l) {
              if (l > 0) {
                if (CHG) acc[l] = caxpy(-sc.cq * q * rcp(l), pw, acc[l]);
                pw = cmul(pw, tinv);
              }
              if (DIP) acc[l] = cfma(fnu, pw, acc[l]);   // pw = tau^-(l+1)
            }
          }
        }
      }
      __syncthreads();
    }
  }
  // reduce the warps' partial sums
  if (warp > 0) {
#pragma unroll
    for (int i = 0; i < NC; ++i) s_red[((warp - 1) * 32 + lane) * NC + i] = acc[i];
  }
  __syncthreads();
  if (warp == 0 && has_center) {
    double2* out = qbx_exps + ((size_t)ctr * nrhs + r) * NC;
#pragma unroll
    for (int i = 0; i < NC; ++i) {
      double2 a = acc[i];
      for (int w = 1; w < NW; ++w) a = cadd(a, s_red[((w - 1) * 32 + lane) * NC + i]);
      out[i] = cadd(out[i], a);
    }
  }
}

// M2QBXL (translate_box_multipoles_to_qbx_local, fmm.py:267-312;
// interactions.py:196-235), all source levels in one launch.  A cluster of MZ CTAs
// x 4 warps per chunk of <= 32 centers (lane = center); the MZ * 4 warps split the
// list-3 boxes, and the partial sums meet in CTA 0 of the cluster in a fixed order
// (warps through shared memory, CTAs through distributed shared memory), so the
// result does not depend on scheduling.  Splitting a chunk over MZ CTAs evens out
// chunks with long list-3 runs.
// 3D: each warp expands the source multipole into a zero-padded dense table
// Mpad[k][l] (rows k in [-Q, pf+Q], columns l in [-(pf+2Q), pf+Q]); each lane runs the
// singular-harmonic recurrence for its center column by column and scatters every
// S_{n'}^{m'} into its register-resident coefficients (j, i) through
// Mpad[n'-j][m'-i]: one broadcast shared load and one complex FMA per term, no
// branches.
template <int DIM, int Q, int MZ>
__global__ void __launch_bounds__(NT)
k_m2qbxl(qbxfmm_geometry g, int pf, int ncf, int nrhs, const double2* __restrict__ mpoles,
         double2* __restrict__ qbx_exps, int32_t* err)
{
  constexpr int NC = (DIM == 3) ? (Q + 1) * (Q + 2) / 2 : Q + 1;
  extern __shared__ double2 smem2[];
  const int MW = 2 * pf + 3 * Q + 1;      // columns l + (pf + 2Q)
  const int MR = pf + 2 * Q + 1;          // rows k + Q
  const int MSZ = (DIM == 3) ? MR * MW : ncf;
  const int loff = pf + 2 * Q;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double2* Mw = smem2 + (size_t)warp * MSZ;
  double2* red = smem2 + (size_t)NW * MSZ;   // [NW-1][32][NC]
  double2* cpart = red + (NW - 1) * 32 * NC;  // [32][NC]: this CTA's sum (MZ > 1)

  int chunk = blockIdx.x / MZ;
  int zpart = blockIdx.x - chunk * MZ;
  int r = blockIdx.y;
  int itb = g.qbx_chunk_target_box[chunk];
  bool has_center = lane < g.qbx_chunk_count[chunk];
  int ctr = has_center ? g.centers_by_target_box[g.qbx_chunk_start[chunk] + lane] : 0;
  if ((unsigned)ctr >= (unsigned)g.ncenters) {
    report(err, QBX_DEVERR_BAD_CENTER);
    has_center = false;
    ctr = 0;
  }
  double cc[3] = {0, 0, 0};
  load_point<DIM>(g.centers, g.ncenters, ctr, cc);
  double rho_t = g.expansion_radii[ctr];
  if (DIM == 3)
    for (int q = lane; q < MSZ; q += 32) Mw[q] = c2(0.0);
  double2 acc[NC];
#pragma unroll
  for (int i = 0; i < NC; ++i) acc[i] = c2(0.0);

  int l0 = g.list3_starts[itb], l1 = g.list3_starts[itb + 1];
  for (int li = l0 + zpart * NW + warp; li < l1; li += MZ * NW) {
    int sb = g.list3_lists[li];
    if ((unsigned)sb >= (unsigned)g.nboxes) {
      report(err, QBX_DEVERR_BAD_BOX);
      continue;
    }
    __syncwarp();
    const double2* src = mpoles + ((size_t)sb * nrhs + r) * ncf;
    double rho_s = level_width(g, g.box_levels[sb]);
    if (DIM == 3) {
      // rows scaled by rho_s^k: with the harmonics taken at the unscaled offset
      // c - c_s, the per-box factor rho_s^-(j+1) of the scaled form moves into the
      // table and the boxes' terms add into acc directly
      for (int q = lane; q < ncf; q += 32) {
        int k, l;
        decode3(q, k, l);
        double sc = 1.0;
        for (int u = 0; u < k; ++u) sc *= rho_s;
        double2 v = cscale(sc, src[q]);
        Mw[(k + Q) * MW + loff + l] = v;
        if (l > 0) Mw[(k + Q) * MW + loff - l] = (l & 1) ? c2(-v.x, v.y) : c2(v.x, -v.y);
      }
    } else {
      for (int q = lane; q < ncf; q += 32) Mw[q] = src[q];
    }
    __syncwarp();
    if (!has_center) continue;
    double cs[3];
    load_point<DIM>(g.box_centers, g.nboxes, sb, cs);
    double ratio = rho_t / rho_s;
    if (DIM == 3) {
      double d0 = cc[0] - cs[0], d1 = cc[1] - cs[1], d2 = cc[2] - cs[2];
      double rinv2 = 1.0 / (d0 * d0 + d1 * d1 + d2 * d2);
      int nmax = pf + Q;
      double2* part = acc;
      double2 mm = c2(sqrt(rinv2));
      for (int mp = 0; mp <= nmax; ++mp) {
        if (mp > 0) mm = cscale((2.0 * mp - 1) * rinv2, cmul(mm, c2(d0, d1)));
        double2 a = mm, prev = c2(0.0);
        const double2* bpos = Mw + (mp + Q) * MW + loff + mp;   // row n'=mp, column m'
        const double2* bneg = Mw + (mp + Q) * MW + loff - mp;   // column -m'
        for (int np = mp; np <= nmax; ++np) {
          if (np > mp) {
            double2 bb = cscale(rinv2, csub(cscale((2.0 * np - 1) * d2, a),
                                            cscale((double)(np + mp - 1) * (np - mp - 1), prev)));
            prev = a;
            a = bb;
          }
#pragma unroll
          for (int j = 0; j <= Q; ++j)
#pragma unroll
            for (int ii = 0; ii <= j; ++ii)
              part[idx3(j, ii)] = cfma(bpos[-j * MW - ii], a, part[idx3(j, ii)]);
          if (mp > 0) {
            double2 aneg = (mp & 1) ? c2(-a.x, a.y) : c2(a.x, -a.y);
#pragma unroll
            for (int j = 0; j <= Q; ++j)
#pragma unroll
              for (int ii = 0; ii <= j; ++ii)
                part[idx3(j, ii)] = cfma(bneg[-j * MW - ii], aneg, part[idx3(j, ii)]);
          }
          bpos += MW;
          bneg += MW;
        }
      }
    } else {
      const double2* M = Mw;
      double2 tau = c2((cc[0] - cs[0]) / rho_s, (cc[1] - cs[1]) / rho_s);
      double2 tinv = cinv(tau);
      double2 t = c2(cc[0] - cs[0], cc[1] - cs[1]);
      double2 s0 = cmul(M[0], clog_(t));
      double2 sl[Q + 1];
      double bin[Q + 1];
#pragma unroll
      for (int l = 0; l <= Q; ++l) {
        sl[l] = c2(0.0);
        bin[l] = 1.0;
      }
      double2 pw = tinv;
      for (int k = 1; k <= pf; ++k) {
        double2 mk = cmul(M[k], pw);
        s0 = cadd(s0, mk);
#pragma unroll
        for (int l = 1; l <= Q; ++l) {
          sl[l] = caxpy(bin[l], mk, sl[l]);
          bin[l] = bin[l] * (k + l) * rcp(k);
        }
        pw = cmul(pw, tinv);
      }
      acc[0] = cadd(acc[0], s0);
      double2 tl = tinv;
      double rl = ratio;
#pragma unroll
      for (int l = 1; l <= Q; ++l) {
        double2 v = cscale(((l & 1) ? 1.0 : -1.0) * rcp(l), M[0]);
        v = cadd(v, cscale((l & 1) ? -1.0 : 1.0, sl[l]));
        acc[l] = cadd(acc[l], cscale(rl, cmul(v, tl)));
        tl = cmul(tl, tinv);
        rl *= ratio;
      }
    }
  }
  __syncthreads();
  if (warp > 0) {
#pragma unroll
    for (int i = 0; i < NC; ++i) red[((warp - 1) * 32 + lane) * NC + i] = acc[i];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NC; ++i)
      for (int w = 1; w < NW; ++w) acc[i] = cadd(acc[i], red[((w - 1) * 32 + lane) * NC + i]);
  }
  if (MZ > 1) {
    cg::cluster_group cl = cg::this_cluster();
    if (warp == 0) {
#pragma unroll
      for (int i = 0; i < NC; ++i) cpart[lane * NC + i] = acc[i];
    }
    cl.sync();
    if (zpart == 0 && warp == 0) {
      for (unsigned q = 1; q < MZ; ++q) {
        const double2* rp = cl.map_shared_rank(cpart, q) + lane * NC;
#pragma unroll
        for (int i = 0; i < NC; ++i) acc[i] = cadd(acc[i], rp[i]);
      }
    }
    cl.sync();
  }
  if (zpart == 0 && warp == 0 && has_center) {
    double2* out = qbx_exps + ((size_t)ctr * nrhs + r) * NC;
    if (DIM == 3) {
      // (-1)^j rho_t^j of the local coefficient of order j
      double f = 1.0;
#pragma unroll
      for (int j = 0; j <= Q; ++j) {
#pragma unroll
        for (int ii = 0; ii <= j; ++ii) acc[idx3(j, ii)] = cscale(f, acc[idx3(j, ii)]);
        f *= -rho_t;
      }
    }
#pragma unroll
    for (int i = 0; i < NC; ++i) out[i] = cadd(out[i], acc[i]);
  }
}

// Target-specific near field (eval_target_specific_qbx_locals, fmm.py:391-394;
// reference native code pytential/qbx/target_specific/impl.pyx:222-362, 566-785).
// For a QBX target t with center c and a list-1 source s, a = t - c, b = s - c:
//   3D: 1/|t-s| ~ sum_{n<=Q} |a|^n / |b|^{n+1} P_n(cos g),  cos g = a.b / (|a||b|),
//       double layer d.grad_s = sum_n |a|^n/|b|^{n+2} [-(n+1)(d.b^) P_n + (d.a^ - cos g d.b^) P_n']
//   2D: log|t-s| ~ log|b| - Re sum_{n=1..Q} (a/b)^n / n,
//       double layer Re(nu / b sum_{n=0..Q} (a/b)^n)      (nu = n_x + i n_y)
// the same truncation as forming the order-Q QBX local from the list-1 sources and
// evaluating it at t.  CTA = 4 warps over a chunk of <= 32 (target, center) pairs of
// one target box (lane = pair); warps split the list-1 source tiles.
template <int DIM, int Q, bool CHG, bool DIP>
__global__ void __launch_bounds__(NT)
k_tsqbx(qbxfmm_geometry g, SourceCoeffs sc, int nrhs, const double* __restrict__ strengths,
        double* __restrict__ pot_tree, int32_t* err)
{
  __shared__ double s_y[3][NT];
  __shared__ double s_n[3][NT];
  __shared__ double s_q[NT];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];
  __shared__ double s_red[NW - 1][32];
  int chunk = blockIdx.x;
  int r = blockIdx.y;
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
  double cc[3] = {0, 0, 0}, x[3] = {0, 0, 0};
  load_point<DIM>(g.centers, g.ncenters, ctr, cc);
  load_point<DIM>(g.targets, g.ntargets, t, x);
  double a[3] = {x[0] - cc[0], x[1] - cc[1], DIM == 3 ? x[2] - cc[2] : 0.0};
  double alen = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  double ainv = alen > 0.0 ? 1.0 / alen : 0.0;
  double ah[3] = {a[0] * ainv, a[1] * ainv, a[2] * ainv};
  const double* st = strengths + (size_t)r * g.nsources;
  double acc = 0.0;
  int l0 = g.list1_starts[itb], l1 = g.list1_starts[itb + 1];
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    list_prefix(g, g.list1_lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += NT) {
      load_stream_tile<DIM, DIP>(g, st, total, nb, base, s_pref, s_start, s_y, s_n, s_q);
      __syncthreads();
      int jbeg = warp * 32, jend = min(jbeg + 32, total - base);
      if (active) {
        for (int j = jbeg; j < jend; ++j) {
          double q = s_q[j];
          if (DIM == 3) {
            double b0 = s_y[0][j] - cc[0], b1 = s_y[1][j] - cc[1], b2 = s_y[2][j] - cc[2];
            double b2s = b0 * b0 + b1 * b1 + b2 * b2;
            double binv = rsqrt(b2s);
            double cg = (ah[0] * b0 + ah[1] * b1 + ah[2] * b2) * binv;   // cos g
            double ratio = alen * binv;                                  // |a| / |b|
            // Legendre P_n, P_n' by recurrence; R_n = ratio^n / |b|
            double pm1 = 1.0, pm2 = 0.0, dm1 = 0.0, dm2 = 0.0;
            double rn = binv;
            double sS = 0.0, sA = 0.0, sB = 0.0;
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
              if (CHG) sS = fma(rn, pn, sS);
              if (DIP) {
                sA = fma(-(n + 1.0) * rn, pn, sA);
                sB = fma(rn, dn, sB);
              }
              pm2 = pm1;
              pm1 = pn;
              dm2 = dm1;
              dm1 = dn;
              rn *= ratio;
            }
            double v = 0.0;
            if (CHG) v = sc.cq * sS;
            if (DIP) {
              double db = (s_n[0][j] * b0 + s_n[1][j] * b1 + s_n[2][j] * b2) * binv;
              double da = s_n[0][j] * ah[0] + s_n[1][j] * ah[1] + s_n[2][j] * ah[2];
              v += sc.cd * binv * (sA * db + sB * (da - cg * db));
            }
            acc = fma(q, v, acc);
            (void)dm2;
          } else {
            double2 bb = c2(s_y[0][j] - cc[0], s_y[1][j] - cc[1]);
            double2 binv = cinv(bb);
            double2 w = cmul(c2(a[0], a[1]), binv);   // a / b
            double2 pw = w;
            double2 sl = c2(0.0);   // sum_{n>=1} w^n / n
            double2 sd = c2(1.0);   // sum_{n>=0} w^n
#pragma unroll
            for (int n = 1; n <= Q; ++n) {
              if (CHG) sl = caxpy(1.0 / n, pw, sl);
              if (DIP) sd = cadd(sd, pw);
              pw = cmul(pw, w);
            }
            double v = 0.0;
            if (CHG) v = sc.cq * (0.5 * log(bb.x * bb.x + bb.y * bb.y) - sl.x);
            if (DIP) {
              double2 f = cmul(cmul(c2(s_n[0][j], s_n[1][j]), binv), sd);
              v += sc.cd * f.x;
            }
            acc = fma(q, v, acc);
          }
        }
      }
      __syncthreads();
    }
  }
  if (warp > 0) s_red[warp - 1][lane] = acc;
  __syncthreads();
  if (warp == 0 && active) {
    for (int w = 1; w < NW; ++w) acc += s_red[w - 1][lane];
    pot_tree[(size_t)r * g.ntargets + t] += acc;
  }
}

// L2QBXL (translate_box_local_to_qbx_local, fmm.py:314-356; interactions.py:318-356)
// 3D: L2Q_SPLIT adjacent lanes per center split the columns b of the regular-harmonic
// table (b = lane part, + L2Q_SPLIT, ...) and meet by shuffles; 2D: one lane per center.
constexpr int L2Q_SPLIT = 4;

template <int DIM, int Q>
__global__ void __launch_bounds__(NT)
k_l2qbxl(qbxfmm_geometry g, int pf, int ncf, int nrhs, const double2* __restrict__ locals,
         double2* __restrict__ qbx_exps)
{
  constexpr int NC = (DIM == 3) ? (Q + 1) * (Q + 2) / 2 : Q + 1;
  constexpr int SPLIT = (DIM == 3) ? L2Q_SPLIT : 1;
  int gt = blockIdx.x * blockDim.x + threadIdx.x;
  int ig = gt / SPLIT, part = gt - ig * SPLIT;
  int r = blockIdx.y;
  if (ig >= g.nglobal_qbx_centers) return;   // whole groups of SPLIT lanes leave together
  int ctr = g.global_qbx_centers[ig];
  int tb = g.target_boxes[g.qbx_center_to_target_box[ctr]];
  double cc[3], cb[3];
  load_point<DIM>(g.centers, g.ncenters, ctr, cc);
  load_point<DIM>(g.box_centers, g.nboxes, tb, cb);
  double rho_b = level_width(g, g.box_levels[tb]);
  double rho_c = g.expansion_radii[ctr];
  double ratio = rho_c / rho_b;
  const double2* Lin = locals + ((size_t)tb * nrhs + r) * ncf;
  double2 acc[NC];
#pragma unroll
  for (int i = 0; i < NC; ++i) acc[i] = c2(0.0);
  if (DIM == 3) {
    double d0 = (cc[0] - cb[0]) / rho_b, d1 = (cc[1] - cb[1]) / rho_b, d2 = (cc[2] - cb[2]) / rho_b;
    double r2 = d0 * d0 + d1 * d1 + d2 * d2;
    // R_a^b(d): output (k,l) += L_{a+k}^{b+l} conj(R_a^b); the lanes of a center
    // take the columns b = part, part + SPLIT, ... in lockstep
    double2 mm = c2(1.0);
    for (int b = 1; b <= part; ++b) mm = cscale(0.5 * rcp(b), cmul(mm, c2(d0, d1)));
    for (int bm = part; bm <= pf; bm += SPLIT) {
      double2 a = mm, prev = c2(0.0);
      for (int b = bm + 1; b <= bm + SPLIT; ++b) mm = cscale(0.5 * rcp(b), cmul(mm, c2(d0, d1)));
      for (int an = bm; an <= pf; ++an) {
        if (an > bm) {
          double2 bb = cscale(rcp(an + bm) * rcp(an - bm),
                              csub(cscale((2.0 * an - 1) * d2, a), cscale(r2, prev)));
          prev = a;
          a = bb;
        }
        double2 aneg = (bm & 1) ? c2(-a.x, a.y) : c2(a.x, -a.y);  // R_an^{-bm}
#pragma unroll
        for (int k = 0; k <= Q; ++k)
#pragma unroll
          for (int l = 0; l <= k; ++l) {
            int n = an + k;
            if (n > pf) continue;
            int m = bm + l;
            if (m <= n) acc[idx3(k, l)] = cfmac(sh3_get(Lin, n, m), a, acc[idx3(k, l)]);
            if (bm > 0) {
              int m2 = -bm + l;
              if (-m2 <= n && m2 <= n)
                acc[idx3(k, l)] = cfmac(sh3_get(Lin, n, m2), aneg, acc[idx3(k, l)]);
            }
          }
      }
    }
    // the SPLIT lanes of a center are adjacent and all present (SPLIT divides 32)
    const unsigned gmask = ((1u << SPLIT) - 1u) << ((threadIdx.x & 31) & ~(SPLIT - 1));
#pragma unroll
    for (int off = 1; off < SPLIT; off <<= 1)
#pragma unroll
      for (int i = 0; i < NC; ++i) {
        acc[i].x += __shfl_xor_sync(gmask, acc[i].x, off, SPLIT);
        acc[i].y += __shfl_xor_sync(gmask, acc[i].y, off, SPLIT);
      }
    if (part != 0) return;
    double rk = 1.0;
#pragma unroll
    for (int k = 0; k <= Q; ++k) {
#pragma unroll
      for (int l = 0; l <= k; ++l) acc[idx3(k, l)] = cscale(rk, acc[idx3(k, l)]);
      rk *= ratio;
    }
  } else {
    double2 s = c2((cc[0] - cb[0]) / rho_b, (cc[1] - cb[1]) / rho_b);
    double rl = 1.0;
#pragma unroll
    for (int l = 0; l <= Q; ++l) {
      double2 a = c2(0.0), sp = c2(1.0);
      double bin = 1.0;
      for (int k = l; k <= pf; ++k) {
        a = cfma(cscale(bin, Lin[k]), sp, a);
        sp = cmul(sp, s);
        bin = bin * (k + 1) / (k + 1 - l);
      }
      acc[l] = cscale(rl, a);
      rl *= ratio;
    }
  }
  double2* out = qbx_exps + ((size_t)ctr * nrhs + r) * NC;
#pragma unroll
  for (int i = 0; i < NC; ++i) out[i] = cadd(out[i], acc[i]);
}

// QBXL2P (eval_qbx_expansions, fmm.py:358-389; interactions.py:442-479)
template <int DIM, int Q>
__global__ void __launch_bounds__(NT)
k_qbxl2p(qbxfmm_geometry g, int nrhs, const double2* __restrict__ qbx_exps,
         double* __restrict__ pot_tree)
{
  constexpr int NC = (DIM == 3) ? (Q + 1) * (Q + 2) / 2 : Q + 1;
  int ig = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (ig >= g.nglobal_qbx_centers) return;
  int ctr = g.global_qbx_centers[ig];
  double cc[3];
  load_point<DIM>(g.centers, g.ncenters, ctr, cc);
  double rinv = 1.0 / g.expansion_radii[ctr];
  double2 L[NC];
  const double2* src = qbx_exps + ((size_t)ctr * nrhs + r) * NC;
#pragma unroll
  for (int i = 0; i < NC; ++i) L[i] = src[i];
  for (int it = g.center_to_targets_starts[ctr]; it < g.center_to_targets_starts[ctr + 1]; ++it) {
    int t = g.center_to_targets_lists[it];
    double x[3];
    load_point<DIM>(g.targets, g.ntargets, t, x);
    double acc = 0.0;
    if (DIM == 3) {
      RRegs<Q> R;
      R.build((x[0] - cc[0]) * rinv, (x[1] - cc[1]) * rinv, (x[2] - cc[2]) * rinv);
#pragma unroll
      for (int n = 0; n <= Q; ++n)
#pragma unroll
        for (int m = 0; m <= n; ++m) {
          double2 a = L[idx3(n, m)], b = R.v[idx3(n, m)];
          acc += (m == 0 ? 1.0 : 2.0) * (a.x * b.x + a.y * b.y);
        }
    } else {
      double2 u = c2((x[0] - cc[0]) * rinv, (x[1] - cc[1]) * rinv), pw = c2(1.0), s = c2(0.0);
#pragma unroll
      for (int k = 0; k <= Q; ++k) {
        s = cfma(L[k], pw, s);
        pw = cmul(pw, u);
      }
      acc = s.x;
    }
    pot_tree[(size_t)r * g.ntargets + t] += acc;
  }
}

// }}}

// {{{ assembly (fmm.py:569-588; qbx/__init__.py:775-793)

__global__ void k_assemble_tree(qbxfmm_geometry g, double scale, int nrhs,
                                const double* __restrict__ pot_tree, double* __restrict__ out)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (t >= g.ntargets) return;
  int u = g.sorted_target_ids[t] - g.ncenters;
  if (u >= 0) out[(size_t)r * g.nuser_targets + u] = scale * pot_tree[(size_t)r * g.ntargets + t];
}

__global__ void k_assemble_nonqbx(qbxfmm_geometry g, double scale, int nrhs,
                                  const double* __restrict__ pot_nonqbx, double* __restrict__ out)
{
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (f >= g.nfiltered_targets) return;
  int t = g.unfiltered_from_filtered_target_indices[f];
  int u = g.sorted_target_ids[t] - g.ncenters;
  if (u >= 0) out[(size_t)r * g.nuser_targets + u] += scale * pot_nonqbx[(size_t)r * g.nfiltered_targets + f];
}

// }}}

// {{{ launchers

static int grid_y(int nrhs) { return nrhs; }

static size_t ncoef_dim(int dim, int p) { return dim == 3 ? (size_t)(p + 1) * (p + 2) / 2 : (size_t)p + 1; }

cudaError_t launch_form_strengths(const qbxfmm_geometry& g, const qbxfmm_upsample& up, int nrhs,
                                  const double* density, double* strengths, cudaStream_t st)
{
  dim3 grid((g.nsources + 255) / 256, nrhs);
  k_form_strengths<<<grid, 256, 0, st>>>(g.nsources, up.nelements * up.nodes_per_element,
                                         up.nodes_per_element, up.quad_nodes_per_element,
                                         up.matrix, up.quad_weights, g.user_source_ids, density,
                                         strengths);
  return cudaGetLastError();
}

template <int DIM>
static cudaError_t p2m_(const qbxfmm_geometry& g, SourceCoeffs sc, int p, int nrhs,
                        const double* s, double2* mp, cudaStream_t st)
{
  int ncf = (int)ncoef_dim(DIM, p);
  size_t sh = (size_t)P2M_TS * ncf * sizeof(double2);
  if (g.nsource_boxes == 0) return cudaSuccess;
  cudaFuncSetAttribute(k_p2m<DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  k_p2m<DIM><<<dim3(g.nsource_boxes, grid_y(nrhs)), NT, sh, st>>>(g, sc, p, ncf, nrhs, s, mp);
  return cudaGetLastError();
}

cudaError_t launch_p2m(const qbxfmm_geometry& g, SourceCoeffs sc, int p, int nrhs,
                       const double* s, double2* mp, cudaStream_t st)
{
  return g.dim == 3 ? p2m_<3>(g, sc, p, nrhs, s, mp, st) : p2m_<2>(g, sc, p, nrhs, s, mp, st);
}

template <int DIM>
static cudaError_t m2m_(const qbxfmm_geometry& g, const int32_t* lvl_host, int p, int nrhs,
                        double2* mp, cudaStream_t st)
{
  int ncf = (int)ncoef_dim(DIM, p);
  size_t sh = 2 * (size_t)ncf * sizeof(double2);
  for (int lev = g.nlevels - 2; lev >= 0; --lev) {
    int i0 = lvl_host[lev], i1 = lvl_host[lev + 1];
    if (i1 <= i0) continue;
    k_m2m<DIM><<<dim3(i1 - i0, grid_y(nrhs)), NT, sh, st>>>(g, p, ncf, nrhs, i0, mp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_m2m(const qbxfmm_geometry& g, const int32_t* lvl_host, int p, int nrhs,
                       double2* mp, cudaStream_t st)
{
  return g.dim == 3 ? m2m_<3>(g, lvl_host, p, nrhs, mp, st) : m2m_<2>(g, lvl_host, p, nrhs, mp, st);
}

cudaError_t launch_m2l(const qbxfmm_geometry& g, int p, int nrhs, const double2* mp, double2* lo,
                       int32_t* err, cudaStream_t st)
{
  if (g.nttp_boxes == 0) return cudaSuccess;
  int ncf = (int)ncoef_dim(g.dim, p);
  if (g.dim == 3) {
    size_t per = ((size_t)(2 * p + 1) * (3 * p + 1) + (size_t)(p + 1) * (2 * p + 1)) * sizeof(double2);
    int pb = (int)std::min<size_t>(4, std::max<size_t>(1, (160 * 1024 - ncf * sizeof(double2)) / per));
    size_t sh = pb * per + ncf * sizeof(double2);
    cudaFuncSetAttribute(k_m2l3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    k_m2l3<<<dim3(g.nttp_boxes, grid_y(nrhs)), NT, sh, st>>>(g, p, ncf, nrhs, pb, mp, lo, err);
  } else {
    size_t sh = ((size_t)ncf + 2 * p + 2) * sizeof(double2);
    k_m2l2<<<dim3(g.nttp_boxes, grid_y(nrhs)), NT, sh, st>>>(g, p, ncf, nrhs, mp, lo, err);
  }
  return cudaGetLastError();
}

template <int DIM>
static cudaError_t p2l_(const qbxfmm_geometry& g, SourceCoeffs sc, int p, int nrhs,
                        const double* s, double2* lo, int32_t* err, cudaStream_t st)
{
  if (g.nttp_boxes == 0) return cudaSuccess;
  int ncf = (int)ncoef_dim(DIM, p);
  int nct = DIM == 3 ? (p + 2) * (p + 3) / 2 : p + 3;
  size_t sh = (size_t)P2L_TS * nct * sizeof(double2);
  int nthr = (P2L3_SPLIT * ncf + 31) / 32 * 32;
  if (DIM == 3 && nthr <= P2L3_MAXT) {
    cudaFuncSetAttribute(k_p2l3s, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    k_p2l3s<<<dim3(g.nttp_boxes, grid_y(nrhs)), nthr, sh, st>>>(g, sc, p, ncf, nrhs, s, lo, err);
    return cudaGetLastError();
  }
  cudaFuncSetAttribute(k_p2l<DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  k_p2l<DIM><<<dim3(g.nttp_boxes, grid_y(nrhs)), NT, sh, st>>>(g, sc, p, ncf, nrhs, s, lo, err);
  return cudaGetLastError();
}

cudaError_t launch_p2l(const qbxfmm_geometry& g, SourceCoeffs sc, int p, int nrhs,
                       const double* s, double2* lo, int32_t* err, cudaStream_t st)
{
  return g.dim == 3 ? p2l_<3>(g, sc, p, nrhs, s, lo, err, st) : p2l_<2>(g, sc, p, nrhs, s, lo, err, st);
}

template <int DIM>
static cudaError_t l2l_(const qbxfmm_geometry& g, const int32_t* lvl_host, int p, int nrhs,
                        double2* lo, cudaStream_t st)
{
  int ncf = (int)ncoef_dim(DIM, p);
  size_t sh = 2 * (size_t)ncf * sizeof(double2);
  for (int lev = 1; lev < g.nlevels; ++lev) {
    int i0 = lvl_host[lev], i1 = lvl_host[lev + 1];
    if (i1 <= i0) continue;
    k_l2l<DIM><<<dim3(i1 - i0, grid_y(nrhs)), NT, sh, st>>>(g, p, ncf, nrhs, i0, lo);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_l2l(const qbxfmm_geometry& g, const int32_t* lvl_host, int p, int nrhs,
                       double2* lo, cudaStream_t st)
{
  return g.dim == 3 ? l2l_<3>(g, lvl_host, p, nrhs, lo, st) : l2l_<2>(g, lvl_host, p, nrhs, lo, st);
}

cudaError_t launch_eval_direct(const qbxfmm_geometry& g, SourceCoeffs sc, int nrhs,
                               const double* s, double* pot, int32_t* err, cudaStream_t st)
{
  if (g.nnonqbx_chunks == 0) return cudaSuccess;
  dim3 grid(g.nnonqbx_chunks * PSPLIT, grid_y(nrhs));   // one cluster per chunk
  if (g.dim == 3) k_eval_direct<3><<<grid, NT, 0, st>>>(g, sc, nrhs, s, pot, err);
  else k_eval_direct<2><<<grid, NT, 0, st>>>(g, sc, nrhs, s, pot, err);
  return cudaGetLastError();
}

cudaError_t launch_eval_multipoles(const qbxfmm_geometry& g, int p, int nrhs, const double2* mp,
                                   double* pot, int32_t* err, cudaStream_t st)
{
  if (g.nnonqbx_chunks == 0) return cudaSuccess;
  int ncf = (int)ncoef_dim(g.dim, p);
  size_t sh = (size_t)NW * ncf * sizeof(double2);
  dim3 grid(g.nnonqbx_chunks * PSPLIT, grid_y(nrhs));   // one cluster per chunk
  if (g.dim == 3) k_eval_multipoles<3><<<grid, NT, sh, st>>>(g, p, ncf, nrhs, mp, pot, err);
  else k_eval_multipoles<2><<<grid, NT, sh, st>>>(g, p, ncf, nrhs, mp, pot, err);
  return cudaGetLastError();
}

cudaError_t launch_eval_locals(const qbxfmm_geometry& g, int p, int nrhs, const double2* lo,
                               double* pot, cudaStream_t st)
{
  if (g.ntarget_boxes == 0 || g.nfiltered_targets == 0) return cudaSuccess;
  int ncf = (int)ncoef_dim(g.dim, p);
  size_t sh = (size_t)ncf * sizeof(double2);
  dim3 grid(g.ntarget_boxes, grid_y(nrhs));
  if (g.dim == 3) k_eval_locals<3><<<grid, NT, sh, st>>>(g, p, ncf, nrhs, lo, pot);
  else k_eval_locals<2><<<grid, NT, sh, st>>>(g, p, ncf, nrhs, lo, pot);
  return cudaGetLastError();
}

template <int DIM, int Q>
static cudaError_t p2qbxl_q(const qbxfmm_geometry& g, SourceCoeffs sc, int nrhs, const double* s,
                            double2* qe, int32_t* err, cudaStream_t st)
{
  constexpr int NC = (DIM == 3) ? (Q + 1) * (Q + 2) / 2 : Q + 1;
  size_t sh = (size_t)(NT / 32 - 1) * 32 * NC * sizeof(double2);
  dim3 grid(g.nqbx_chunks, grid_y(nrhs));
  if (sc.cq != 0.0 && sc.cd != 0.0) {
    cudaFuncSetAttribute(k_p2qbxl<DIM, Q, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    k_p2qbxl<DIM, Q, true, true><<<grid, NT, sh, st>>>(g, sc, nrhs, s, qe, err);
  } else if (sc.cd != 0.0) {
    cudaFuncSetAttribute(k_p2qbxl<DIM, Q, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    k_p2qbxl<DIM, Q, false, true><<<grid, NT, sh, st>>>(g, sc, nrhs, s, qe, err);
  } else {
    cudaFuncSetAttribute(k_p2qbxl<DIM, Q, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    k_p2qbxl<DIM, Q, true, false><<<grid, NT, sh, st>>>(g, sc, nrhs, s, qe, err);
  }
  return cudaGetLastError();
}

// CTAs per chunk in the 3D M2QBXL cluster launch
constexpr int M2QBXL_Z = 4;

template <int DIM, int Q>
static cudaError_t m2qbxl_q(const qbxfmm_geometry& g, int pf, int nrhs, const double2* mp,
                            double2* qe, int32_t* err, cudaStream_t st)
{
  int ncf = (int)ncoef_dim(DIM, pf);
  constexpr int NC = (DIM == 3) ? (Q + 1) * (Q + 2) / 2 : Q + 1;
  size_t msz = DIM == 3 ? (size_t)(pf + 2 * Q + 1) * (2 * pf + 3 * Q + 1) : (size_t)ncf;
  size_t sh = (NW * msz + (size_t)NW * 32 * NC) * sizeof(double2);
  if constexpr (DIM == 2) {
    cudaFuncSetAttribute(k_m2qbxl<DIM, Q, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    k_m2qbxl<DIM, Q, 1><<<dim3(g.nqbx_chunks, grid_y(nrhs)), NT, sh, st>>>(g, pf, ncf, nrhs, mp, qe,
                                                                          err);
    return cudaGetLastError();
  } else {
  // 3D: clusters of M2QBXL_Z CTAs per chunk
  constexpr int MZ = M2QBXL_Z;
  cudaFuncSetAttribute(k_m2qbxl<DIM, Q, MZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(g.nqbx_chunks * MZ, grid_y(nrhs));
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = sh;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = MZ;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_m2qbxl<DIM, Q, MZ>, g, pf, ncf, nrhs, mp, qe, err);
  }
}

template <int DIM, int Q>
static cudaError_t l2qbxl_q(const qbxfmm_geometry& g, int pf, int nrhs, const double2* lo,
                            double2* qe, cudaStream_t st)
{
  int ncf = (int)ncoef_dim(DIM, pf);
  size_t lanes = (size_t)g.nglobal_qbx_centers * (DIM == 3 ? L2Q_SPLIT : 1);
  dim3 grid((unsigned)((lanes + NT - 1) / NT), grid_y(nrhs));
  k_l2qbxl<DIM, Q><<<grid, NT, 0, st>>>(g, pf, ncf, nrhs, lo, qe);
  return cudaGetLastError();
}

template <int DIM, int Q>
static cudaError_t qbxl2p_q(const qbxfmm_geometry& g, int nrhs, const double2* qe, double* pt,
                            cudaStream_t st)
{
  dim3 grid((g.nglobal_qbx_centers + NT - 1) / NT, grid_y(nrhs));
  k_qbxl2p<DIM, Q><<<grid, NT, 0, st>>>(g, nrhs, qe, pt);
  return cudaGetLastError();
}

#define QBX_DISPATCH_Q(FN, DIM, Q, ...)                               \
  switch (Q) {                                                        \
    case 0: return FN<DIM, 0>(__VA_ARGS__);                            \
    case 1: return FN<DIM, 1>(__VA_ARGS__);                            \
    case 2: return FN<DIM, 2>(__VA_ARGS__);                            \
    case 3: return FN<DIM, 3>(__VA_ARGS__);                            \
    case 4: return FN<DIM, 4>(__VA_ARGS__);                            \
    case 5: return FN<DIM, 5>(__VA_ARGS__);                            \
    case 6: return FN<DIM, 6>(__VA_ARGS__);                            \
    case 7: return FN<DIM, 7>(__VA_ARGS__);                            \
    case 8: return FN<DIM, 8>(__VA_ARGS__);                            \
    default: return cudaErrorInvalidValue;                            \
  }

cudaError_t launch_p2qbxl(const qbxfmm_geometry& g, SourceCoeffs sc, int q, int nrhs,
                          const double* s, double2* qe, int32_t* err, cudaStream_t st)
{
  if (g.nqbx_chunks == 0) return cudaSuccess;
  if (g.dim == 3) { QBX_DISPATCH_Q(p2qbxl_q, 3, q, g, sc, nrhs, s, qe, err, st) }
  QBX_DISPATCH_Q(p2qbxl_q, 2, q, g, sc, nrhs, s, qe, err, st)
}

cudaError_t launch_m2qbxl(const qbxfmm_geometry& g, int pf, int q, int nrhs, const double2* mp,
                          double2* qe, int32_t* err, cudaStream_t st)
{
  if (g.nqbx_chunks == 0) return cudaSuccess;
  if (g.dim == 3) { QBX_DISPATCH_Q(m2qbxl_q, 3, q, g, pf, nrhs, mp, qe, err, st) }
  QBX_DISPATCH_Q(m2qbxl_q, 2, q, g, pf, nrhs, mp, qe, err, st)
}

cudaError_t launch_l2qbxl(const qbxfmm_geometry& g, int pf, int q, int nrhs, const double2* lo,
                          double2* qe, cudaStream_t st)
{
  if (g.nglobal_qbx_centers == 0) return cudaSuccess;
  if (g.dim == 3) { QBX_DISPATCH_Q(l2qbxl_q, 3, q, g, pf, nrhs, lo, qe, st) }
  QBX_DISPATCH_Q(l2qbxl_q, 2, q, g, pf, nrhs, lo, qe, st)
}

cudaError_t launch_qbxl2p(const qbxfmm_geometry& g, int q, int nrhs, const double2* qe,
                          double* pt, cudaStream_t st)
{
  if (g.nglobal_qbx_centers == 0) return cudaSuccess;
  if (g.dim == 3) { QBX_DISPATCH_Q(qbxl2p_q, 3, q, g, nrhs, qe, pt, st) }
  QBX_DISPATCH_Q(qbxl2p_q, 2, q, g, nrhs, qe, pt, st)
}

template <int DIM, int Q>
static cudaError_t tsqbx_q(const qbxfmm_geometry& g, SourceCoeffs sc, int nrhs, const double* s,
                           double* pt, int32_t* err, cudaStream_t st)
{
  dim3 grid(g.ntsqbx_chunks, grid_y(nrhs));
  if (sc.cq != 0.0 && sc.cd != 0.0) k_tsqbx<DIM, Q, true, true><<<grid, NT, 0, st>>>(g, sc, nrhs, s, pt, err);
  else if (sc.cd != 0.0) k_tsqbx<DIM, Q, false, true><<<grid, NT, 0, st>>>(g, sc, nrhs, s, pt, err);
  else k_tsqbx<DIM, Q, true, false><<<grid, NT, 0, st>>>(g, sc, nrhs, s, pt, err);
  return cudaGetLastError();
}

cudaError_t launch_tsqbx(const qbxfmm_geometry& g, SourceCoeffs sc, int q, int nrhs,
                         const double* s, double* pt, int32_t* err, cudaStream_t st)
{
  if (g.ntsqbx_chunks == 0) return cudaSuccess;
  if (g.dim == 3) { QBX_DISPATCH_Q(tsqbx_q, 3, q, g, sc, nrhs, s, pt, err, st) }
  QBX_DISPATCH_Q(tsqbx_q, 2, q, g, sc, nrhs, s, pt, err, st)
}

cudaError_t launch_assemble(const qbxfmm_geometry& g, int nrhs, const double* pot_nonqbx,
                            const double* pot_tree, double* out, cudaStream_t st)
{
  double scale = g.dim == 3 ? 0.25 / M_PI : -0.5 / M_PI;
  if (g.ntargets > 0) {
    k_assemble_tree<<<dim3((g.ntargets + 255) / 256, nrhs), 256, 0, st>>>(g, scale, nrhs, pot_tree, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (g.nfiltered_targets > 0) {
    k_assemble_nonqbx<<<dim3((g.nfiltered_targets + 255) / 256, nrhs), 256, 0, st>>>(
        g, scale, nrhs, pot_nonqbx, out);
  }
  return cudaGetLastError();
}

// }}}

}  // namespace qbx
