// 2D Helmholtz QBX-FMM stage kernels (H2D expansions), complex128, sm_100a.
//
// Same stage set and work decomposition as the Laplace kernels
// (pytential/qbx/fmm.py:414-594): box kernels one CTA per box, point evaluations
// and the QBX near field over the chunked schedules, with complex densities and
// Bessel/Hankel bases (helmholtz.cuh).  Per source the single- and double-layer
// weights are folded into three complex factors
//   q = cq s,  a = (k/2) cd s conj(nu),  b = (k/2) cd s nu      (nu = n_x + i n_y)
// so that a multipole coefficient gets q conj(J_m) + a conj(J_{m-1}) - b conj(J_{m+1})
// and a local coefficient q Hb_m + a Hb_{m-1} - b Hb_{m+1}.
#include "helmholtz.cuh"
#include "kernels.h"

namespace qbx {

namespace {

constexpr int NT = 128;
constexpr int NW = NT / 32;
constexpr int MAXB = 128;
constexpr int ZMAX = 2 * 20 + 2;   // Bessel scratch: orders 0..2 * max fmm_order + 1

QBX_D void h_list_prefix(const qbxfmm_geometry& g, const int32_t* __restrict__ lists, int gb,
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

QBX_D int h_stream_source(int v, int nb, const int* s_pref, const int* s_start)
{
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (s_pref[mid] <= v) lo = mid;
    else hi = mid - 1;
  }
  return s_start[lo] + (v - s_pref[lo]);
}

// the three per-source factors (see the file comment)
QBX_D void source_factors(const HelmCoeffs& hc, double2 s, double nx, double ny, bool dip,
                          double2& q, double2& a, double2& b)
{
  q = cmul(hc.cq, s);
  if (dip) {
    double2 sig = cscale(0.5 * hc.k, cmul(hc.cd, s));
    a = cmul(sig, c2(nx, -ny));
    b = cmul(sig, c2(nx, ny));
  } else {
    a = b = c2(0.0);
  }
}

QBX_D double2 cneg(double2 a) { return c2(-a.x, -a.y); }

// Hb_m(u) = (-1)^m H_{-m}(u) from a Z table centred at index N
QBX_D double2 hbar(const double2* Z, int N, int m)
{
  double2 v = Z[N - m];
  return (m & 1) ? cneg(v) : v;
}

}  // namespace

// {{{ strengths (complex density)

__global__ void __launch_bounds__(256)
k_h2_form_strengths(int nsources, int ndofs, int npe, int nqpe, const double* __restrict__ U,
                    const double* __restrict__ qw, const int32_t* __restrict__ user_source_ids,
                    const double2* __restrict__ density, double2* __restrict__ out)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (t >= nsources) return;
  int j = __ldg(user_source_ids + t);
  int e = j / nqpe;
  int jj = j - e * nqpe;
  const double* u = U + (size_t)jj * npe;
  const double2* d = density + (size_t)r * ndofs + (size_t)e * npe;
  double2 acc = c2(0.0);
  for (int i = 0; i < npe; ++i) acc = caxpy(__ldg(u + i), d[i], acc);
  out[(size_t)r * nsources + t] = cscale(__ldg(qw + j), acc);
}

// }}}

// {{{ P2M (source boxes) and P2L (list 4)

// E_m[r] += f(m) sum_s W_s(m) str_s[r]: per source the weights
//   P2M: W(m) = cq conj(Z_m) + kd (conj(nu) conj(Z_{m-1}) - nu conj(Z_{m+1})),  Z = J
//   P2L: W(m) = cq Hb_m + kd (conj(nu) Hb_{m-1} - nu Hb_{m+1})
// (kd = (k/2) cd) do not depend on the density, so a box is a (2p+1) x nsrc times
// nsrc x rhs complex product.  One CTA per (box, tile of RW * TR right-hand sides),
// thread layout as in k_h2_translate; SUB sources per stage: Bessel tables one per
// thread, then W and the strengths tile in shared memory.
template <bool LOCAL, int RW, int TR>
__global__ void __launch_bounds__(NT)
k_h2_p2e(qbxfmm_geometry g, HelmCoeffs hc, int p, int nrhs, const double2* __restrict__ strengths,
         double2* __restrict__ exps, int32_t* err)
{
  constexpr int SUB = 32;
  constexpr int G = NT / RW;
  constexpr int TM = (2 * 20 + 1 + G - 1) / G;
  constexpr int RC = RW * TR;
  extern __shared__ double2 smem2[];
  const int N = p + 1, ZW = 2 * N + 1, NC = 2 * p + 1;
  double2* Z = smem2;                        // [SUB][ZW]
  double2* W = Z + (size_t)SUB * ZW;         // [SUB][NC]
  double2* S = W + (size_t)SUB * NC;         // [SUB][RC + 1] (padded rows)
  __shared__ double2 s_nu[SUB];
  __shared__ int s_src[SUB];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];
  int i = blockIdx.x;
  int r0 = blockIdx.y * RC;
  int nr = min(RC, nrhs - r0);
  int b, l0, l1;
  const int32_t* lists;
  if (LOCAL) {
    b = g.target_or_target_parent_boxes[i];
    lists = g.list4_lists;
    l0 = g.list4_starts[i];
    l1 = g.list4_starts[i + 1];
  } else {
    b = g.source_boxes[i];
    lists = g.source_boxes;   // the box's own sources
    l0 = i;
    l1 = i + 1;
  }
  double c[2];
  load_point<2>(g.box_centers, g.nboxes, b, c);
  const bool dip = hc.cd.x != 0.0 || hc.cd.y != 0.0;
  const double2 kd = cscale(0.5 * hc.k, hc.cd);
  double Jb[ZMAX], Yb[ZMAX];
  const int rl = threadIdx.x % RW, mg = threadIdx.x / RW;
  double2 acc[TM][TR];
#pragma unroll
  for (int a = 0; a < TM; ++a)
#pragma unroll
    for (int j = 0; j < TR; ++j) acc[a][j] = c2(0.0);
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    h_list_prefix(g, lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += SUB) {
      int cnt = min(SUB, total - base);
      if (threadIdx.x < cnt) {
        int s = h_stream_source(base + threadIdx.x, nb, s_pref, s_start);
        double y[2], nv[2] = {0, 0};
        load_point<2>(g.sources, g.nsources, s, y);
        if (dip) load_point<2>(g.source_normals, g.nsources, s, nv);
        s_src[threadIdx.x] = s;
        s_nu[threadIdx.x] = c2(nv[0], nv[1]);
        h2_zfun(N, hc.k, y[0] - c[0], y[1] - c[1], Jb, Yb, Z + (size_t)threadIdx.x * ZW, LOCAL);
      }
      __syncthreads();
      for (int w = threadIdx.x; w < cnt * NC; w += NT) {
        int j = w / NC, m = w - j * NC - p;
        const double2* Zt = Z + (size_t)j * ZW;
        double2 v;
        if (!LOCAL) {
          v = cmulc(hc.cq, Zt[N + m]);
          if (dip) {
            double2 nu = s_nu[j];
            v = cfma(kd, csub(cmulc(cconj(nu), Zt[N + m - 1]), cmulc(nu, Zt[N + m + 1])), v);
          }
        } else {
          v = cmul(hc.cq, hbar(Zt, N, m));
          if (dip) {
            double2 nu = s_nu[j];
            v = cfma(kd, csub(cmul(cconj(nu), hbar(Zt, N, m - 1)), cmul(nu, hbar(Zt, N, m + 1))), v);
          }
        }
        W[w] = v;
      }
      for (int w = threadIdx.x; w < cnt * RC; w += NT) {
        int r = w / cnt, j = w - r * cnt;
        S[j * (RC + 1) + r] = r < nr ? strengths[(size_t)(r0 + r) * g.nsources + s_src[j]] : c2(0.0);
      }
      __syncthreads();
      for (int j = 0; j < cnt; ++j) {
        double2 e[TR];
#pragma unroll
        for (int jj = 0; jj < TR; ++jj) e[jj] = S[j * (RC + 1) + rl + RW * jj];
#pragma unroll
        for (int a = 0; a < TM; ++a) {
          int m = min(mg + G * a, NC - 1);
          double2 wv = W[j * NC + m];
#pragma unroll
          for (int jj = 0; jj < TR; ++jj) acc[a][jj] = cfma(wv, e[jj], acc[a][jj]);
        }
      }
      __syncthreads();
    }
  }
  double rho = level_width(g, g.box_levels[b]);
  double2* E = exps + ((size_t)b * nrhs + r0) * NC;
#pragma unroll
  for (int a = 0; a < TM; ++a) {
    int m = mg + G * a;
    if (m >= NC) continue;
    int am = m - p < 0 ? p - m : m - p;
    double sc = LOCAL ? pow(rho, (double)am) : pow(rho, -(double)am);
#pragma unroll
    for (int jj = 0; jj < TR; ++jj) {
      int r = rl + RW * jj;
      if (r < nr) E[(size_t)r * NC + m] = caxpy(sc, acc[a][jj], E[(size_t)r * NC + m]);
    }
  }
}

// }}}

// {{{ translations: M2M, L2L (per level), M2L (list 2)

// Eout_m[r] += fout(m) sum_n Z_{n-m}(d) fin(n) Ein_n[r] with Z = J (M2M, L2L) or H (M2L):
// per source box a Toeplitz (2p+1) x (2p+1) matrix applied to a tile of right-hand
// sides.  One CTA per (output box, tile of RW * TR right-hand sides); thread t takes
// the right-hand sides rl + RW j (rl = t % RW, j < TR) and the coefficients
// mg + G i (mg = t / RW, G = NT / RW, i < TM), all in registers.  The Z tables (order
// 2p) of up to PB source boxes are built one per thread into shared memory, once for
// the whole tile; each source box's coefficient block ([rhs][coef], contiguous in
// global memory) is staged scaled by fin(n) into shared memory with coalesced loads.
template <int KIND, int RW, int TR>   // KIND 0 = M2M, 1 = M2L, 2 = L2L
__global__ void __launch_bounds__(NT)
k_h2_translate(qbxfmm_geometry g, HelmCoeffs hc, int p, int nrhs, int i0,
               const double2* __restrict__ ein, double2* __restrict__ eout, int32_t* err)
{
  constexpr int PB = 16;
  constexpr int G = NT / RW;
  constexpr int TM = (2 * 20 + 1 + G - 1) / G;
  constexpr int RC = RW * TR;
  extern __shared__ double2 smem2[];
  const int NZ = 2 * p, ZW = 2 * NZ + 1, NC = 2 * p + 1;
  double2* Z = smem2;                       // [PB][ZW]
  double2* E = Z + (size_t)PB * ZW;         // [RC][NC]
  __shared__ int s_src[PB];
  __shared__ double s_fin[PB][2 * 20 + 1];
  double Jb[ZMAX], Yb[ZMAX];
  int ib = i0 + blockIdx.x;
  int r0 = blockIdx.y * RC;
  int nr = min(RC, nrhs - r0);
  int tb;
  int l0, l1;
  if (KIND == 0) {
    tb = g.source_parent_boxes[ib];
    l0 = 0;
    l1 = 4;     // children
  } else if (KIND == 1) {
    tb = g.target_or_target_parent_boxes[ib];
    l0 = g.list2_starts[ib];
    l1 = g.list2_starts[ib + 1];
  } else {
    tb = g.target_or_target_parent_boxes[ib];
    l0 = 0;
    l1 = 1;     // parent
  }
  double ct[2];
  load_point<2>(g.box_centers, g.nboxes, tb, ct);
  const int rl = threadIdx.x % RW, mg = threadIdx.x / RW;
  double2 acc[TM][TR];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TR; ++j) acc[i][j] = c2(0.0);
  for (int lb = l0; lb < l1; lb += PB) {
    int nbat = min(PB, l1 - lb);
    __syncthreads();
    if (threadIdx.x < nbat) {
      int sb;
      if (KIND == 0) {
        sb = g.box_child_ids[(size_t)(lb + threadIdx.x) * g.nboxes + tb];
        if (sb == 0 || g.box_source_counts_cumul[sb] == 0) sb = -1;
      } else if (KIND == 1) {
        sb = g.list2_lists[lb + threadIdx.x];
        if ((unsigned)sb >= (unsigned)g.nboxes) {
          report(err, QBX_DEVERR_BAD_BOX);
          sb = -1;
        }
      } else {
        sb = g.box_parent_ids[tb];
      }
      s_src[threadIdx.x] = sb;
      if (sb >= 0) {
        double cs[2];
        load_point<2>(g.box_centers, g.nboxes, sb, cs);
        // d = c_out - c_in
        h2_zfun(NZ, hc.k, ct[0] - cs[0], ct[1] - cs[1], Jb, Yb, Z + (size_t)threadIdx.x * ZW,
                KIND == 1);
      }
    }
    __syncthreads();
    for (int w = threadIdx.x; w < nbat * NC; w += NT) {
      int bb = w / NC, n = w - bb * NC - p;
      int sb = s_src[bb];
      if (sb >= 0) {
        double rin = level_width(g, g.box_levels[sb]);
        int an = n < 0 ? -n : n;
        s_fin[bb][n + p] = (KIND == 2) ? pow(rin, -(double)an) : pow(rin, (double)an);
      }
    }
    for (int bb = 0; bb < nbat; ++bb) {
      int sb = s_src[bb];
      if (sb < 0) continue;      // uniform over the CTA
      __syncthreads();           // E free, s_fin written
      const double2* src = ein + ((size_t)sb * nrhs + r0) * NC;
      for (int w = threadIdx.x; w < nr * NC; w += NT) {
        int n = w % NC;
        E[w] = cscale(s_fin[bb][n], src[w]);
      }
      __syncthreads();
      // Z_{n-m} for coefficient indices n, m in [0, 2p] at Zt[n - m]
      const double2* Zt = Z + (size_t)bb * ZW + NZ;
      for (int n = 0; n < NC; ++n) {
        double2 e[TR];
#pragma unroll
        for (int j = 0; j < TR; ++j) e[j] = E[(rl + RW * j) * NC + n];
#pragma unroll
        for (int i = 0; i < TM; ++i) {
          int m = min(mg + G * i, NC - 1);
          double2 z = Zt[n - m];
#pragma unroll
          for (int j = 0; j < TR; ++j) acc[i][j] = cfma(z, e[j], acc[i][j]);
        }
      }
    }
  }
  // the tile through shared memory, then one coalesced read-modify-write
  double rho_t = level_width(g, g.box_levels[tb]);
  __syncthreads();
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    int m = mg + G * i;
    if (m >= NC) continue;
    int am = m - p < 0 ? p - m : m - p;
    double f = (KIND == 0) ? pow(rho_t, -(double)am) : pow(rho_t, (double)am);
#pragma unroll
    for (int j = 0; j < TR; ++j) {
      int r = rl + RW * j;
      if (r < nr) E[r * NC + m] = cscale(f, acc[i][j]);
    }
  }
  __syncthreads();
  double2* dst = eout + ((size_t)tb * nrhs + r0) * NC;
  for (int w = threadIdx.x; w < nr * NC; w += NT) dst[w] = cadd(dst[w], E[w]);
}

// }}}

// {{{ point evaluations at non-QBX targets

__global__ void __launch_bounds__(NT)
k_h2_eval_direct(qbxfmm_geometry g, HelmCoeffs hc, int nrhs, const double2* __restrict__ strengths,
                 double2* __restrict__ pot, int32_t* err)
{
  __shared__ double s_y[2][NT], s_n[2][NT];
  __shared__ double2 s_q[NT], s_d[NT];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];
  __shared__ double2 s_red[NW - 1][32];
  int chunk = blockIdx.x;
  int r = blockIdx.y;
  int itb = g.nonqbx_chunk_target_box[chunk];
  int t = g.nonqbx_chunk_start[chunk] + (threadIdx.x & 31);
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bool active = lane < g.nonqbx_chunk_count[chunk];
  double x[2] = {0, 0};
  if (active) load_point<2>(g.nonqbx_targets, g.nfiltered_targets, t, x);
  const double2* st = strengths + (size_t)r * g.nsources;
  const bool dip = hc.cd.x != 0.0 || hc.cd.y != 0.0;
  double2 acc = c2(0.0);
  int l0 = g.list1_starts[itb], l1 = g.list1_starts[itb + 1];
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    h_list_prefix(g, g.list1_lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += NT) {
      int v = base + threadIdx.x;
      if (v < total) {
        int s = h_stream_source(v, nb, s_pref, s_start);
        double y[2], nv[2] = {0, 0};
        load_point<2>(g.sources, g.nsources, s, y);
        if (dip) load_point<2>(g.source_normals, g.nsources, s, nv);
        s_y[0][threadIdx.x] = y[0];
        s_y[1][threadIdx.x] = y[1];
        s_n[0][threadIdx.x] = nv[0];
        s_n[1][threadIdx.x] = nv[1];
        s_q[threadIdx.x] = cmul(hc.cq, st[s]);
        s_d[threadIdx.x] = cscale(hc.k, cmul(hc.cd, st[s]));
      }
      __syncthreads();
      int jbeg = warp * 32, jend = min(jbeg + 32, total - base);
      if (active) {
        for (int j = jbeg; j < jend; ++j) {
          double dx = x[0] - s_y[0][j], dy = x[1] - s_y[1][j];
          double r2 = dx * dx + dy * dy;
          if (r2 == 0.0) continue;
          double rr = sqrt(r2), kr = hc.k * rr;
          acc = cfma(s_q[j], c2(j0(kr), y0(kr)), acc);
          if (dip) {
            double cn = (s_n[0][j] * dx + s_n[1][j] * dy) / rr;
            acc = cfma(cscale(cn, s_d[j]), c2(j1(kr), y1(kr)), acc);
          }
        }
      }
      __syncthreads();
    }
  }
  if (warp > 0) s_red[warp - 1][lane] = acc;
  __syncthreads();
  if (warp == 0 && active) {
    for (int w = 1; w < NW; ++w) acc = cadd(acc, s_red[w - 1][lane]);
    double2* P = pot + (size_t)r * g.nfiltered_targets + t;
    *P = cadd(*P, acc);
  }
}

// M2P over list 3 (lanes = targets, warps split the boxes) and L2P (own box)
template <bool LOCAL>
__global__ void __launch_bounds__(NT)
k_h2_eval_exp(qbxfmm_geometry g, HelmCoeffs hc, int p, int nrhs, const double2* __restrict__ exps,
              double2* __restrict__ pot, int32_t* err)
{
  __shared__ double2 s_red[NW - 1][32];
  double Jb[ZMAX], Yb[ZMAX];
  double2 Zt[2 * 21 + 1];
  int chunk = blockIdx.x;
  int r = blockIdx.y;
  int itb = g.nonqbx_chunk_target_box[chunk];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int t = g.nonqbx_chunk_start[chunk] + lane;
  bool active = lane < g.nonqbx_chunk_count[chunk];
  double x[2] = {0, 0};
  if (active) load_point<2>(g.nonqbx_targets, g.nfiltered_targets, t, x);
  double2 acc = c2(0.0);
  int l0, l1;
  if (LOCAL) {
    l0 = 0;
    l1 = 1;
  } else {
    l0 = g.list3_starts[itb];
    l1 = g.list3_starts[itb + 1];
  }
  for (int li = l0 + warp; li < l1 && active; li += NW) {
    int sb = LOCAL ? g.target_boxes[itb] : g.list3_lists[li];
    if ((unsigned)sb >= (unsigned)g.nboxes) {
      report(err, QBX_DEVERR_BAD_BOX);
      continue;
    }
    double rho = level_width(g, g.box_levels[sb]);
    double cs[2];
    load_point<2>(g.box_centers, g.nboxes, sb, cs);
    h2_zfun(p, hc.k, x[0] - cs[0], x[1] - cs[1], Jb, Yb, Zt, !LOCAL);
    const double2* E = exps + ((size_t)sb * nrhs + r) * (2 * p + 1);
    double f = 1.0, finv = 1.0, rinv = 1.0 / rho;
    for (int am = 0; am <= p; ++am) {
      double sc = LOCAL ? finv : f;
      acc = cfma(cscale(sc, E[p + am]), Zt[p + am], acc);
      if (am > 0) acc = cfma(cscale(sc, E[p - am]), Zt[p - am], acc);
      f *= rho;
      finv *= rinv;
    }
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

// }}}

// {{{ QBX stages

// P2QBXL: lanes = centers of a chunk, warps split the list-1 source tiles; the
// Hankel table of each (center, source) pair is built in registers (orders
// 0..Q+1 by Miller's recurrence, downward part unrolled).
template <int Q>
__global__ void __launch_bounds__(NT)
k_h2_p2qbxl(qbxfmm_geometry g, HelmCoeffs hc, int nrhs, const double2* __restrict__ strengths,
            double2* __restrict__ qbx_exps, int32_t* err)
{
  constexpr int NC = 2 * Q + 1;
  constexpr int N = Q + 1;
  __shared__ double s_y[2][NT];
  __shared__ double2 s_q[NT], s_a[NT], s_b[NT];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];
  extern __shared__ double2 s_red[];   // [NW-1][32][NC]
  int chunk = blockIdx.x;
  int r = blockIdx.y;
  int itb = g.qbx_chunk_target_box[chunk];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bool has_center = lane < g.qbx_chunk_count[chunk];
  int ctr = has_center ? g.centers_by_target_box[g.qbx_chunk_start[chunk] + lane] : 0;
  if ((unsigned)ctr >= (unsigned)g.ncenters) {
    report(err, QBX_DEVERR_BAD_CENTER);
    has_center = false;
    ctr = 0;
  }
  double cc[2];
  load_point<2>(g.centers, g.ncenters, ctr, cc);
  double rho = g.expansion_radii[ctr];
  const double2* st = strengths + (size_t)r * g.nsources;
  const bool dip = hc.cd.x != 0.0 || hc.cd.y != 0.0;
  double2 acc[NC];
#pragma unroll
  for (int i = 0; i < NC; ++i) acc[i] = c2(0.0);
  int l0 = g.list1_starts[itb], l1 = g.list1_starts[itb + 1];
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    h_list_prefix(g, g.list1_lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += NT) {
      int v = base + threadIdx.x;
      if (v < total) {
        int s = h_stream_source(v, nb, s_pref, s_start);
        double y[2], nv[2] = {0, 0};
        load_point<2>(g.sources, g.nsources, s, y);
        if (dip) load_point<2>(g.source_normals, g.nsources, s, nv);
        s_y[0][threadIdx.x] = y[0];
        s_y[1][threadIdx.x] = y[1];
        double2 q, a, b;
        source_factors(hc, st[s], nv[0], nv[1], dip, q, a, b);
        s_q[threadIdx.x] = q;
        s_a[threadIdx.x] = a;
        s_b[threadIdx.x] = b;
      }
      __syncthreads();
      int jbeg = warp * 32, jend = min(jbeg + 32, total - base);
      if (has_center) {
        for (int j = jbeg; j < jend; ++j) {
          double ux = s_y[0][j] - cc[0], uy = s_y[1][j] - cc[1];
          double r2 = ux * ux + uy * uy;
          double rr = sqrt(r2);
          double x = hc.k * rr, xinv = 1.0 / x;
          // Miller: downward from an even start to N+1 (runtime), then unrolled to 0
          int nmax = N > (int)x ? N : (int)x;
          int start = 2 * ((nmax + 16 + (int)sqrt(40.0 * nmax)) / 2);
          double fp1 = 0.0, f = 1e-200, sum = 0.0;
          for (int k = start; k > N + 1; --k) {
            double fm1 = 2.0 * k * xinv * f - fp1;
            fp1 = f;
            f = fm1;
            if (((k - 1) & 1) == 0) sum += 2.0 * f;
            if (fabs(f) > 1e200) {
              f *= 1e-200;
              fp1 *= 1e-200;
              sum *= 1e-200;
            }
          }
          double J[N + 1];
          // f = f_{N+1}, fp1 = f_{N+2}
#pragma unroll
          for (int k = N + 1; k > 0; --k) {
            double fm1 = 2.0 * k * xinv * f - fp1;
            fp1 = f;
            f = fm1;
            J[k - 1] = f;
            if (((k - 1) & 1) == 0 && k - 1 > 0) sum += 2.0 * f;
          }
          sum += f;
          double norm = 1.0 / sum;
          double Y[N + 1];
          Y[0] = y0(x);
          Y[1] = y1(x);
#pragma unroll
          for (int k = 1; k < N; ++k) Y[k + 1] = 2.0 * k * xinv * Y[k] - Y[k - 1];
          // Hb_m = H_m(kr) e^{-i m th} for m >= 0; Hb_{-m} = (-1)^m H_m(kr) e^{i m th}
          double2 e1 = c2(ux / rr, -uy / rr);   // e^{-i th}
          double2 e = c2(1.0);
          double2 hp[N + 1], hm[N + 1];
#pragma unroll
          for (int m = 0; m <= N; ++m) {
            double2 h = c2(J[m] * norm, Y[m]);
            hp[m] = cmul(h, e);                       // Hb_m
            double2 w = cmul(h, cconj(e));
            hm[m] = (m & 1) ? cneg(w) : w;            // Hb_{-m}
            e = cmul(e, e1);
          }
          double2 q = s_q[j], a = s_a[j], b = s_b[j];
#pragma unroll
          for (int m = -Q; m <= Q; ++m) {
            double2 h0 = m >= 0 ? hp[m] : hm[-m];
            double2 hl = (m - 1) >= 0 ? hp[m - 1] : hm[1 - m];
            double2 hr = (m + 1) >= 0 ? hp[m + 1] : hm[-m - 1];
            double2 v = cmul(q, h0);
            if (dip) {
              v = cfma(a, hl, v);
              v = cfma(cneg(b), hr, v);
            }
            acc[m + Q] = cadd(acc[m + Q], v);
          }
        }
      }
      __syncthreads();
    }
  }
  if (warp > 0) {
#pragma unroll
    for (int i = 0; i < NC; ++i) s_red[((warp - 1) * 32 + lane) * NC + i] = acc[i];
  }
  __syncthreads();
  if (warp == 0 && has_center) {
    double2* out = qbx_exps + ((size_t)ctr * nrhs + r) * NC;
    double f = 1.0;
#pragma unroll
    for (int am = 0; am <= Q; ++am) {
      double2 ap = acc[Q + am], an = acc[Q - am];
      for (int w = 1; w < NW; ++w) {
        ap = cadd(ap, s_red[((w - 1) * 32 + lane) * NC + Q + am]);
        if (am > 0) an = cadd(an, s_red[((w - 1) * 32 + lane) * NC + Q - am]);
      }
      out[Q + am] = caxpy(f, ap, out[Q + am]);
      if (am > 0) out[Q - am] = caxpy(f, an, out[Q - am]);
      f *= rho;
    }
  }
}

// Target-specific near field (eval_target_specific_qbx_locals, pytential/qbx/fmm.py:391-394)
// for the H2D expansion: per (target t, its center c, list-1 source y) the order-Q
// QBX expansion is evaluated without forming it,
//   K = sum_{|m|<=Q} Z_m(t - c) (cq Hb_m(y - c) + (k/2) cd (conj(nu) Hb_{m-1} - nu Hb_{m+1})),
// Z_m = J_m e^{i m th}, the same series as P2QBXL followed by QBXL2P.  H_m(k|y - c|)
// by the upward recurrence from H_0, H_1 (dominant solution).  K is computed once per
// pair and applied to RB densities (lane = target; warps split each source tile).
template <int Q, int RB>
__global__ void __launch_bounds__(NT)
k_h2_tsqbx(qbxfmm_geometry g, HelmCoeffs hc, int nrhs, const double2* __restrict__ strengths,
           double2* __restrict__ pot_tree, int32_t* err)
{
  __shared__ double s_y[2][NT], s_n[2][NT];
  __shared__ double2 s_q[RB][NT];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];
  extern __shared__ double2 s_red[];   // [NW-1][32][RB]
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
  double cc[2], x[2];
  load_point<2>(g.centers, g.ncenters, ctr, cc);
  load_point<2>(g.targets, g.ntargets, t, x);
  // Z_m(t - c), m in [-Q, Q], at Zt[Q + m]
  double2 Zt[2 * Q + 1];
  {
    double ax = x[0] - cc[0], ay = x[1] - cc[1];
    double alen = sqrt(ax * ax + ay * ay);
    double J[Q + 1];
    if (alen > 0.0) {
      double Yd[1];
      bessel_jy(Q, hc.k * alen, J, Yd, false);
    } else {
#pragma unroll
      for (int m = 0; m <= Q; ++m) J[m] = (m == 0) ? 1.0 : 0.0;
    }
    double2 e1 = alen > 0.0 ? c2(ax / alen, ay / alen) : c2(1.0);
    double2 e = c2(1.0);
#pragma unroll
    for (int m = 0; m <= Q; ++m) {
      Zt[Q + m] = cscale(J[m], e);
      double2 w = cscale(J[m], cconj(e));
      Zt[Q - m] = (m & 1) ? cneg(w) : w;
      e = cmul(e, e1);
    }
  }
  const bool chg = hc.cq.x != 0.0 || hc.cq.y != 0.0;
  const bool dip = hc.cd.x != 0.0 || hc.cd.y != 0.0;
  const double2 kd = cscale(0.5 * hc.k, hc.cd);
  double2 acc[RB];
#pragma unroll
  for (int i = 0; i < RB; ++i) acc[i] = c2(0.0);
  int l0 = g.list1_starts[itb], l1 = g.list1_starts[itb + 1];
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    h_list_prefix(g, g.list1_lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += NT) {
      int v = base + threadIdx.x;
      if (v < total) {
        int s = h_stream_source(v, nb, s_pref, s_start);
        double y[2], nv[2] = {0, 0};
        load_point<2>(g.sources, g.nsources, s, y);
        if (dip) load_point<2>(g.source_normals, g.nsources, s, nv);
        s_y[0][threadIdx.x] = y[0];
        s_y[1][threadIdx.x] = y[1];
        s_n[0][threadIdx.x] = nv[0];
        s_n[1][threadIdx.x] = nv[1];
#pragma unroll
        for (int i = 0; i < RB; ++i)
          s_q[i][threadIdx.x] = (r0 + i < nrhs) ? strengths[(size_t)(r0 + i) * g.nsources + s] : c2(0.0);
      }
      __syncthreads();
      int jbeg = warp * 32, jend = min(jbeg + 32, total - base);
      if (active) {
        for (int j = jbeg; j < jend; ++j) {
          double ux = s_y[0][j] - cc[0], uy = s_y[1][j] - cc[1];
          double b2 = ux * ux + uy * uy;
          if (b2 == 0.0) continue;
          double binv = rsqrt(b2);
          double xx = hc.k * b2 * binv, xinv = 1.0 / xx;
          double2 H[Q + 2];
          H[0] = c2(j0(xx), y0(xx));
          H[1] = c2(j1(xx), y1(xx));
#pragma unroll
          for (int m = 1; m <= Q; ++m)
            H[m + 1] = c2(2.0 * m * xinv * H[m].x - H[m - 1].x, 2.0 * m * xinv * H[m].y - H[m - 1].y);
          // Hb_m for m in [-(Q+1), Q+1] at Hb[Q + 1 + m]
          double2 Hb[2 * Q + 3];
          double2 e1 = c2(ux * binv, -uy * binv);     // e^{-i th}
          double2 e = c2(1.0);
#pragma unroll
          for (int m = 0; m <= Q + 1; ++m) {
            Hb[Q + 1 + m] = cmul(H[m], e);
            double2 w = cmul(H[m], cconj(e));
            Hb[Q + 1 - m] = (m & 1) ? cneg(w) : w;
            e = cmul(e, e1);
          }
          double2 K = c2(0.0);
          if (chg) {
            double2 s0 = c2(0.0);
#pragma unroll
            for (int m = -Q; m <= Q; ++m) s0 = cfma(Zt[Q + m], Hb[Q + 1 + m], s0);
            K = cmul(hc.cq, s0);
          }
          if (dip) {
            double2 sm = c2(0.0), sp = c2(0.0);
#pragma unroll
            for (int m = -Q; m <= Q; ++m) {
              sm = cfma(Zt[Q + m], Hb[Q + m], sm);
              sp = cfma(Zt[Q + m], Hb[Q + 2 + m], sp);
            }
            double2 nu = c2(s_n[0][j], s_n[1][j]);
            K = cfma(kd, csub(cmul(cconj(nu), sm), cmul(nu, sp)), K);
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
      double2 vv = acc[i];
      for (int w = 1; w < NW; ++w) vv = cadd(vv, s_red[((w - 1) * 32 + lane) * RB + i]);
      double2* P = pot_tree + (size_t)(r0 + i) * g.ntargets + t;
      *P = cadd(*P, vv);
    }
  }
}

// The same near field for many right-hand sides: per source tile of TS_ST sources the
// kernel values K(t, y) of all (target, source) pairs of the chunk are computed once,
// packed over all threads (a chunk holds the few targets of one box), into shared
// memory; then pot[t][r] += sum_y K(t, y) str_y[r] over a tile of 64 right-hand sides
// (thread: rhs tid % 64, targets tid / 64 + 2 i).
constexpr int TS_ST = 32;
constexpr int TS_RC = 64;

template <int Q>
__global__ void __launch_bounds__(NT)
k_h2_tsqbx_many(qbxfmm_geometry g, HelmCoeffs hc, int nrhs, const double2* __restrict__ strengths,
                double2* __restrict__ pot_tree, int32_t* err)
{
  constexpr int NQ = 2 * Q + 1;
  extern __shared__ double2 smem2[];
  double2* S = smem2;                         // [TS_ST][TS_RC + 1] (padded rows)
  double2* K = S + TS_ST * (TS_RC + 1);       // [TS_ST][32]
  __shared__ double2 s_zt[32][NQ];
  __shared__ double s_cc[2][32];
  __shared__ double s_y[2][TS_ST], s_n[2][TS_ST];
  __shared__ int s_src[TS_ST];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];
  int chunk = blockIdx.x;
  int r0 = blockIdx.y * TS_RC;
  int nr = min(TS_RC, nrhs - r0);
  int itb = g.tsqbx_chunk_target_box[chunk];
  int i0 = g.tsqbx_chunk_start[chunk];
  int cnt = min(g.tsqbx_chunk_count[chunk], 32);
  if (g.tsqbx_chunk_count[chunk] > 32 && blockIdx.y == 0 && threadIdx.x == 0)
    report(err, QBX_DEVERR_BAD_CENTER);
  // per target: its center and J_m(t - c) e^{i m th}
  if (threadIdx.x < cnt) {
    int t = g.tsqbx_targets[i0 + threadIdx.x];
    int ctr = g.tsqbx_centers[i0 + threadIdx.x];
    double cc[2] = {0, 0}, x[2] = {0, 0};
    if ((unsigned)ctr >= (unsigned)g.ncenters || (unsigned)t >= (unsigned)g.ntargets) {
      report(err, QBX_DEVERR_BAD_CENTER);
    } else {
      load_point<2>(g.centers, g.ncenters, ctr, cc);
      load_point<2>(g.targets, g.ntargets, t, x);
    }
    s_cc[0][threadIdx.x] = cc[0];
    s_cc[1][threadIdx.x] = cc[1];
    double ax = x[0] - cc[0], ay = x[1] - cc[1];
    double alen = sqrt(ax * ax + ay * ay);
    double J[Q + 1];
    if (alen > 0.0) {
      double Yd[1];
      bessel_jy(Q, hc.k * alen, J, Yd, false);
    } else {
#pragma unroll
      for (int m = 0; m <= Q; ++m) J[m] = (m == 0) ? 1.0 : 0.0;
    }
    double2 e1 = alen > 0.0 ? c2(ax / alen, ay / alen) : c2(1.0);
    double2 e = c2(1.0);
#pragma unroll
    for (int m = 0; m <= Q; ++m) {
      s_zt[threadIdx.x][Q + m] = cscale(J[m], e);
      double2 w = cscale(J[m], cconj(e));
      s_zt[threadIdx.x][Q - m] = (m & 1) ? cneg(w) : w;
      e = cmul(e, e1);
    }
  }
  const bool chg = hc.cq.x != 0.0 || hc.cq.y != 0.0;
  const bool dip = hc.cd.x != 0.0 || hc.cd.y != 0.0;
  const double2 kd = cscale(0.5 * hc.k, hc.cd);
  const int rr = threadIdx.x % TS_RC, th = threadIdx.x / TS_RC;
  const int nti = (cnt - th + 1) / 2;           // targets th + 2 i, i < nti
  double2 acc[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) acc[i] = c2(0.0);
  int l0 = g.list1_starts[itb], l1 = g.list1_starts[itb + 1];
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    h_list_prefix(g, g.list1_lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += TS_ST) {
      int ns = min(TS_ST, total - base);
      if (threadIdx.x < ns) {
        int s = h_stream_source(base + threadIdx.x, nb, s_pref, s_start);
        double y[2], nv[2] = {0, 0};
        load_point<2>(g.sources, g.nsources, s, y);
        if (dip) load_point<2>(g.source_normals, g.nsources, s, nv);
        s_src[threadIdx.x] = s;
        s_y[0][threadIdx.x] = y[0];
        s_y[1][threadIdx.x] = y[1];
        s_n[0][threadIdx.x] = nv[0];
        s_n[1][threadIdx.x] = nv[1];
      }
      __syncthreads();
      for (int w = threadIdx.x; w < ns * TS_RC; w += NT) {
        int r = w / ns, j = w - r * ns;       // sources fastest: coalesced rows
        S[j * (TS_RC + 1) + r] = r < nr ? strengths[(size_t)(r0 + r) * g.nsources + s_src[j]] : c2(0.0);
      }
      for (int pr = threadIdx.x; pr < ns * cnt; pr += NT) {
        int j = pr / cnt, t = pr - j * cnt;
        double ux = s_y[0][j] - s_cc[0][t], uy = s_y[1][j] - s_cc[1][t];
        double b2 = ux * ux + uy * uy;
        double2 Kv = c2(0.0);
        if (b2 != 0.0) {
          double binv = rsqrt(b2);
          double xx = hc.k * b2 * binv, xinv = 1.0 / xx;
          double2 H[Q + 2];
          H[0] = c2(j0(xx), y0(xx));
          H[1] = c2(j1(xx), y1(xx));
#pragma unroll
          for (int m = 1; m <= Q; ++m)
            H[m + 1] = c2(2.0 * m * xinv * H[m].x - H[m - 1].x, 2.0 * m * xinv * H[m].y - H[m - 1].y);
          // Hb_m for m in [-(Q+1), Q+1] at Hb[Q + 1 + m]
          double2 Hb[2 * Q + 3];
          double2 e1 = c2(ux * binv, -uy * binv);     // e^{-i th}
          double2 e = c2(1.0);
#pragma unroll
          for (int m = 0; m <= Q + 1; ++m) {
            Hb[Q + 1 + m] = cmul(H[m], e);
            double2 w = cmul(H[m], cconj(e));
            Hb[Q + 1 - m] = (m & 1) ? cneg(w) : w;
            e = cmul(e, e1);
          }
          const double2* Zt = s_zt[t];
          if (chg) {
            double2 s0 = c2(0.0);
#pragma unroll
            for (int m = -Q; m <= Q; ++m) s0 = cfma(Zt[Q + m], Hb[Q + 1 + m], s0);
            Kv = cmul(hc.cq, s0);
          }
          if (dip) {
            double2 sm = c2(0.0), sp = c2(0.0);
#pragma unroll
            for (int m = -Q; m <= Q; ++m) {
              sm = cfma(Zt[Q + m], Hb[Q + m], sm);
              sp = cfma(Zt[Q + m], Hb[Q + 2 + m], sp);
            }
            double2 nu = c2(s_n[0][j], s_n[1][j]);
            Kv = cfma(kd, csub(cmul(cconj(nu), sm), cmul(nu, sp)), Kv);
          }
        }
        K[j * 32 + t] = Kv;
      }
      __syncthreads();
      for (int j = 0; j < ns; ++j) {
        double2 sv = S[j * (TS_RC + 1) + rr];
        const double2* Kj = K + j * 32 + th;
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (i < nti) acc[i] = cfma(Kj[2 * i], sv, acc[i]);
      }
      __syncthreads();
    }
  }
  if (rr >= nr) return;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    if (i >= nti) break;
    int t = g.tsqbx_targets[i0 + th + 2 * i];
    if ((unsigned)t >= (unsigned)g.ntargets) continue;
    double2* P = pot_tree + (size_t)(r0 + rr) * g.ntargets + t;
    *P = cadd(*P, acc[i]);
  }
}

// M2QBXL (list 3) and L2QBXL (own target box):
//   Q_m[r] += rho_c^|m| sum_n Z_{n-m}(c - c_b) f(n) E_n[r],  f(n) = rho_b^{+-|n|},
// Z = H (from multipoles) or J (from locals), m in [-Q, Q], n in [-pf, pf].  One CTA
// per (CW centers of a QBX chunk, tile of RW * TR right-hand sides); all centers of a
// chunk share a target box and so its list 3.  Thread t: rhs lane rl = t % RW (rhs
// rl + RW j), center t / RW, all 2Q+1 coefficients in registers.  Source boxes go in
// batches of E2Q_LB: the Z tables (order pf + Q) of all (center, box) pairs of a batch
// are built in parallel, one per thread (CW * E2Q_LB = 32 for the 128-thread tiles); then per box the scaled coefficient block is
// staged once in shared memory for all centers.
constexpr int E2Q_LB = 8;

template <int Q, bool FROM_LOCAL, int RW, int TR, int CW>
__global__ void __launch_bounds__(RW * CW)
k_h2_e2qbxl(qbxfmm_geometry g, HelmCoeffs hc, int pf, int nrhs, const double2* __restrict__ exps,
            double2* __restrict__ qbx_exps, int32_t* err)
{
  constexpr int NQ = 2 * Q + 1;
  constexpr int NTH = RW * CW;
  constexpr int RC = RW * TR;
  constexpr int NSUB = 32 / CW;
  extern __shared__ double2 smem2[];
  const int NZ = pf + Q, ZW = 2 * NZ + 1, NC = 2 * pf + 1;
  double2* Zc = smem2;                                 // [E2Q_LB][CW][ZW]
  double2* E = Zc + (size_t)E2Q_LB * CW * ZW;          // [RC][NC]
  __shared__ double s_fn[E2Q_LB][2 * 20 + 1];
  __shared__ int s_sb[E2Q_LB];
  __shared__ double s_cc[2][CW];
  double Jb[ZMAX], Yb[ZMAX];
  // the sub-chunks of a chunk are adjacent in launch order: they read the same boxes
  int chunk = blockIdx.x / NSUB;
  int sub = blockIdx.x % NSUB;
  int r0 = blockIdx.y * RC;
  int nr = min(RC, nrhs - r0);
  int ncen = g.qbx_chunk_count[chunk];
  if (ncen > 32 && sub == 0 && threadIdx.x == 0) report(err, QBX_DEVERR_BAD_CENTER);
  ncen -= sub * CW;
  if (ncen <= 0) return;                       // uniform over the CTA
  ncen = min(ncen, CW);
  int itb = g.qbx_chunk_target_box[chunk];
  const int rl = threadIdx.x % RW, cw = threadIdx.x / RW;
  bool has_center = cw < ncen;
  int ctr = has_center ? g.centers_by_target_box[g.qbx_chunk_start[chunk] + sub * CW + cw] : 0;
  if ((unsigned)ctr >= (unsigned)g.ncenters) {
    report(err, QBX_DEVERR_BAD_CENTER);
    has_center = false;
    ctr = 0;
  }
  if (rl == 0) {
    double cc[2];
    load_point<2>(g.centers, g.ncenters, ctr, cc);
    s_cc[0][cw] = cc[0];
    s_cc[1][cw] = cc[1];
  }
  double2 acc[NQ][TR];
#pragma unroll
  for (int a = 0; a < NQ; ++a)
#pragma unroll
    for (int j = 0; j < TR; ++j) acc[a][j] = c2(0.0);
  int l0 = FROM_LOCAL ? 0 : g.list3_starts[itb];
  int l1 = FROM_LOCAL ? 1 : g.list3_starts[itb + 1];
  for (int lb = l0; lb < l1; lb += E2Q_LB) {
    int nbat = min(E2Q_LB, l1 - lb);
    __syncthreads();                           // Zc, s_sb, s_fn free; s_cc written
    if (threadIdx.x < nbat) {
      int sb = FROM_LOCAL ? g.target_boxes[itb] : g.list3_lists[lb + threadIdx.x];
      if ((unsigned)sb >= (unsigned)g.nboxes) {
        report(err, QBX_DEVERR_BAD_BOX);
        sb = -1;
      }
      s_sb[threadIdx.x] = sb;
    }
    __syncthreads();
    for (int pi = threadIdx.x; pi < nbat * CW; pi += NTH) {
      int bb = pi / CW, c = pi % CW;
      int sb = s_sb[bb];
      if (sb >= 0 && c < ncen) {
        double cs[2];
        load_point<2>(g.box_centers, g.nboxes, sb, cs);
        h2_zfun(NZ, hc.k, s_cc[0][c] - cs[0], s_cc[1][c] - cs[1], Jb, Yb,
                Zc + ((size_t)bb * CW + c) * ZW, !FROM_LOCAL);
      }
    }
    for (int w = threadIdx.x; w < nbat * NC; w += NTH) {
      int bb = w / NC, n = w - bb * NC;
      int sb = s_sb[bb];
      if (sb < 0) continue;
      double rho_s = level_width(g, g.box_levels[sb]);
      int an = n - pf < 0 ? pf - n : n - pf;
      s_fn[bb][n] = FROM_LOCAL ? pow(rho_s, -(double)an) : pow(rho_s, (double)an);
    }
    for (int bb = 0; bb < nbat; ++bb) {
      int sb = s_sb[bb];
      if (sb < 0) continue;                    // uniform over the CTA
      __syncthreads();                         // E free; Zc, s_fn written
      const double2* src = exps + ((size_t)sb * nrhs + r0) * NC;
      for (int w = threadIdx.x; w < nr * NC; w += NTH) E[w] = cscale(s_fn[bb][w % NC], src[w]);
      __syncthreads();
      if (has_center) {
        // Z_{n-m} for coefficient indices n in [0, 2pf], a = m + Q in [0, 2Q] at Zr[n - a]
        const double2* Zr = Zc + ((size_t)bb * CW + cw) * ZW + NZ - pf + Q;
        for (int n = 0; n < NC; ++n) {
          double2 e[TR];
#pragma unroll
          for (int j = 0; j < TR; ++j) e[j] = E[(rl + RW * j) * NC + n];
#pragma unroll
          for (int a = 0; a < NQ; ++a) {
            double2 z = Zr[n - a];
#pragma unroll
            for (int j = 0; j < TR; ++j) acc[a][j] = cfma(z, e[j], acc[a][j]);
          }
        }
      }
    }
  }
  if (!has_center) return;
  double rho_t = g.expansion_radii[ctr];
#pragma unroll
  for (int j = 0; j < TR; ++j) {
    int r = rl + RW * j;
    if (r >= nr) continue;
    double2* out = qbx_exps + ((size_t)ctr * nrhs + r0 + r) * NQ;
    double f = 1.0;
#pragma unroll
    for (int am = 0; am <= Q; ++am) {
      out[Q + am] = caxpy(f, acc[Q + am][j], out[Q + am]);
      if (am > 0) out[Q - am] = caxpy(f, acc[Q - am][j], out[Q - am]);
      f *= rho_t;
    }
  }
}

template <int Q>
__global__ void __launch_bounds__(NT)
k_h2_qbxl2p(qbxfmm_geometry g, HelmCoeffs hc, int nrhs, const double2* __restrict__ qbx_exps,
            double2* __restrict__ pot_tree)
{
  constexpr int NC = 2 * Q + 1;
  double Jb[Q + 2], Yb[Q + 2];
  double2 Z[2 * Q + 1];
  int ig = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (ig >= g.nglobal_qbx_centers) return;
  int ctr = g.global_qbx_centers[ig];
  double cc[2];
  load_point<2>(g.centers, g.ncenters, ctr, cc);
  double rinv = 1.0 / g.expansion_radii[ctr];
  const double2* L = qbx_exps + ((size_t)ctr * nrhs + r) * NC;
  for (int it = g.center_to_targets_starts[ctr]; it < g.center_to_targets_starts[ctr + 1]; ++it) {
    int t = g.center_to_targets_lists[it];
    double x[2];
    load_point<2>(g.targets, g.ntargets, t, x);
    double2 acc = c2(0.0);
    double ux = x[0] - cc[0], uy = x[1] - cc[1];
    if (ux * ux + uy * uy == 0.0) {
      acc = L[Q];   // J_0(0) = 1, J_m(0) = 0
    } else {
      h2_zfun(Q, hc.k, ux, uy, Jb, Yb, Z, false);
      double f = 1.0;
#pragma unroll
      for (int am = 0; am <= Q; ++am) {
        acc = cfma(cscale(f, L[Q + am]), Z[Q + am], acc);
        if (am > 0) acc = cfma(cscale(f, L[Q - am]), Z[Q - am], acc);
        f *= rinv;
      }
    }
    double2* P = pot_tree + (size_t)r * g.ntargets + t;
    *P = cadd(*P, acc);
  }
}

// }}}

// {{{ assembly

__global__ void k_h2_assemble_tree(qbxfmm_geometry g, int nrhs, const double2* __restrict__ pot_tree,
                                   double2* __restrict__ out)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (t >= g.ntargets) return;
  int u = g.sorted_target_ids[t] - g.ncenters;
  double2 v = pot_tree[(size_t)r * g.ntargets + t];
  if (u >= 0) out[(size_t)r * g.nuser_targets + u] = c2(-0.25 * v.y, 0.25 * v.x);   // (i/4) v
}

__global__ void k_h2_assemble_nonqbx(qbxfmm_geometry g, int nrhs,
                                     const double2* __restrict__ pot_nonqbx, double2* __restrict__ out)
{
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (f >= g.nfiltered_targets) return;
  int t = g.unfiltered_from_filtered_target_indices[f];
  int u = g.sorted_target_ids[t] - g.ncenters;
  double2 v = pot_nonqbx[(size_t)r * g.nfiltered_targets + f];
  if (u >= 0) {
    double2* o = out + (size_t)r * g.nuser_targets + u;
    *o = cadd(*o, c2(-0.25 * v.y, 0.25 * v.x));
  }
}

// }}}

// {{{ launchers

static size_t zsh(int p) { return (size_t)(2 * (p + 1) + 1); }

cudaError_t h2_launch_form_strengths(const qbxfmm_geometry& g, const qbxfmm_upsample& up, int nrhs,
                                     const double2* density, double2* strengths, cudaStream_t st)
{
  dim3 grid((g.nsources + 255) / 256, nrhs);
  k_h2_form_strengths<<<grid, 256, 0, st>>>(g.nsources, up.nelements * up.nodes_per_element,
                                            up.nodes_per_element, up.quad_nodes_per_element,
                                            up.matrix, up.quad_weights, g.user_source_ids, density,
                                            strengths);
  return cudaGetLastError();
}

template <bool LOCAL, int RW, int TR>
static cudaError_t h2_p2e_rt(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs, int nb,
                             const double2* s, double2* e, int32_t* err, cudaStream_t st)
{
  size_t sh = (size_t)32 * (zsh(p) + (2 * p + 1) + RW * TR + 1) * sizeof(double2);
  cudaError_t ce = cudaFuncSetAttribute(k_h2_p2e<LOCAL, RW, TR>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (ce != cudaSuccess) return ce;
  k_h2_p2e<LOCAL, RW, TR><<<dim3(nb, (nrhs + RW * TR - 1) / (RW * TR)), NT, sh, st>>>(
      g, hc, p, nrhs, s, e, err);
  return cudaGetLastError();
}

template <bool LOCAL>
static cudaError_t h2_p2e(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs, int nb,
                          const double2* s, double2* e, int32_t* err, cudaStream_t st)
{
  if (p > 20) return cudaErrorInvalidValue;
  if (nrhs == 1) return h2_p2e_rt<LOCAL, 1, 1>(g, hc, p, nrhs, nb, s, e, err, st);
  if (nrhs <= 4) return h2_p2e_rt<LOCAL, 4, 1>(g, hc, p, nrhs, nb, s, e, err, st);
  if (nrhs <= 16) return h2_p2e_rt<LOCAL, 16, 1>(g, hc, p, nrhs, nb, s, e, err, st);
  if (nrhs <= 32) return h2_p2e_rt<LOCAL, 32, 1>(g, hc, p, nrhs, nb, s, e, err, st);
  return h2_p2e_rt<LOCAL, 32, 2>(g, hc, p, nrhs, nb, s, e, err, st);
}

cudaError_t h2_launch_p2m(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                          const double2* s, double2* mp, int32_t* err, cudaStream_t st)
{
  if (g.nsource_boxes == 0) return cudaSuccess;
  return h2_p2e<false>(g, hc, p, nrhs, g.nsource_boxes, s, mp, err, st);
}

cudaError_t h2_launch_p2l(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                          const double2* s, double2* lo, int32_t* err, cudaStream_t st)
{
  if (g.nttp_boxes == 0) return cudaSuccess;
  return h2_p2e<true>(g, hc, p, nrhs, g.nttp_boxes, s, lo, err, st);
}

// right-hand-side tiling of the translation kernels: (lanes over rhs, rhs per lane)
template <int KIND, int RW, int TR>
static cudaError_t h2_translate_rt(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                                   int i0, int nb, const double2* ein, double2* eout, int32_t* err,
                                   cudaStream_t st)
{
  size_t sh = ((size_t)16 * (4 * p + 1) + (size_t)RW * TR * (2 * p + 1)) * sizeof(double2);
  cudaError_t e = cudaFuncSetAttribute(k_h2_translate<KIND, RW, TR>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return e;
  dim3 grid(nb, (nrhs + RW * TR - 1) / (RW * TR));
  k_h2_translate<KIND, RW, TR><<<grid, NT, sh, st>>>(g, hc, p, nrhs, i0, ein, eout, err);
  return cudaGetLastError();
}

template <int KIND>
static cudaError_t h2_translate(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs, int i0,
                                int nb, const double2* ein, double2* eout, int32_t* err,
                                cudaStream_t st)
{
  if (p > 20) return cudaErrorInvalidValue;
  if (nrhs == 1) return h2_translate_rt<KIND, 1, 1>(g, hc, p, nrhs, i0, nb, ein, eout, err, st);
  if (nrhs <= 4) return h2_translate_rt<KIND, 4, 1>(g, hc, p, nrhs, i0, nb, ein, eout, err, st);
  if (nrhs <= 16) return h2_translate_rt<KIND, 16, 1>(g, hc, p, nrhs, i0, nb, ein, eout, err, st);
  if (nrhs <= 32) return h2_translate_rt<KIND, 32, 1>(g, hc, p, nrhs, i0, nb, ein, eout, err, st);
  return h2_translate_rt<KIND, 32, 2>(g, hc, p, nrhs, i0, nb, ein, eout, err, st);
}

cudaError_t h2_launch_m2m(const qbxfmm_geometry& g, const int32_t* lvl_host, HelmCoeffs hc, int p,
                          int nrhs, double2* mp, int32_t* err, cudaStream_t st)
{
  for (int lev = g.nlevels - 2; lev >= 0; --lev) {
    int i0 = lvl_host[lev], i1 = lvl_host[lev + 1];
    if (i1 <= i0) continue;
    cudaError_t e = h2_translate<0>(g, hc, p, nrhs, i0, i1 - i0, mp, mp, err, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t h2_launch_m2l(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                          const double2* mp, double2* lo, int32_t* err, cudaStream_t st)
{
  if (g.nttp_boxes == 0) return cudaSuccess;
  return h2_translate<1>(g, hc, p, nrhs, 0, g.nttp_boxes, mp, lo, err, st);
}

cudaError_t h2_launch_l2l(const qbxfmm_geometry& g, const int32_t* lvl_host, HelmCoeffs hc, int p,
                          int nrhs, double2* lo, int32_t* err, cudaStream_t st)
{
  for (int lev = 1; lev < g.nlevels; ++lev) {
    int i0 = lvl_host[lev], i1 = lvl_host[lev + 1];
    if (i1 <= i0) continue;
    cudaError_t e = h2_translate<2>(g, hc, p, nrhs, i0, i1 - i0, lo, lo, err, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t h2_launch_eval_direct(const qbxfmm_geometry& g, HelmCoeffs hc, int nrhs,
                                  const double2* s, double2* pot, int32_t* err, cudaStream_t st)
{
  if (g.nnonqbx_chunks == 0) return cudaSuccess;
  k_h2_eval_direct<<<dim3(g.nnonqbx_chunks, nrhs), NT, 0, st>>>(g, hc, nrhs, s, pot, err);
  return cudaGetLastError();
}

cudaError_t h2_launch_eval_multipoles(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                                      const double2* mp, double2* pot, int32_t* err, cudaStream_t st)
{
  if (g.nnonqbx_chunks == 0) return cudaSuccess;
  k_h2_eval_exp<false><<<dim3(g.nnonqbx_chunks, nrhs), NT, 0, st>>>(g, hc, p, nrhs, mp, pot, err);
  return cudaGetLastError();
}

cudaError_t h2_launch_eval_locals(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int nrhs,
                                  const double2* lo, double2* pot, int32_t* err, cudaStream_t st)
{
  if (g.nnonqbx_chunks == 0) return cudaSuccess;
  k_h2_eval_exp<true><<<dim3(g.nnonqbx_chunks, nrhs), NT, 0, st>>>(g, hc, p, nrhs, lo, pot, err);
  return cudaGetLastError();
}

template <int Q>
static cudaError_t h2_p2qbxl_q(const qbxfmm_geometry& g, HelmCoeffs hc, int nrhs, const double2* s,
                               double2* qe, int32_t* err, cudaStream_t st)
{
  size_t sh = (size_t)(NW - 1) * 32 * (2 * Q + 1) * sizeof(double2);
  k_h2_p2qbxl<Q><<<dim3(g.nqbx_chunks, nrhs), NT, sh, st>>>(g, hc, nrhs, s, qe, err);
  return cudaGetLastError();
}

template <int Q, bool FROM_LOCAL, int RW, int TR, int CW>
static cudaError_t h2_e2qbxl_rt(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int nrhs,
                                const double2* e, double2* qe, int32_t* err, cudaStream_t st)
{
  size_t sh = ((size_t)E2Q_LB * CW * (2 * (pf + Q) + 1) + (size_t)RW * TR * (2 * pf + 1)) *
              sizeof(double2);
  cudaError_t ce = cudaFuncSetAttribute(k_h2_e2qbxl<Q, FROM_LOCAL, RW, TR, CW>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (ce != cudaSuccess) return ce;
  dim3 grid(g.nqbx_chunks * (32 / CW), (nrhs + RW * TR - 1) / (RW * TR));
  k_h2_e2qbxl<Q, FROM_LOCAL, RW, TR, CW><<<grid, RW * CW, sh, st>>>(g, hc, pf, nrhs, e, qe, err);
  return cudaGetLastError();
}

template <int Q, bool FROM_LOCAL>
static cudaError_t h2_e2qbxl_qf(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int nrhs,
                                const double2* e, double2* qe, int32_t* err, cudaStream_t st)
{
  if (nrhs == 1) return h2_e2qbxl_rt<Q, FROM_LOCAL, 1, 1, 32>(g, hc, pf, nrhs, e, qe, err, st);
  if (nrhs <= 4) return h2_e2qbxl_rt<Q, FROM_LOCAL, 4, 1, 32>(g, hc, pf, nrhs, e, qe, err, st);
  if (nrhs <= 32) return h2_e2qbxl_rt<Q, FROM_LOCAL, 32, 1, 4>(g, hc, pf, nrhs, e, qe, err, st);
  return h2_e2qbxl_rt<Q, FROM_LOCAL, 32, 2, 4>(g, hc, pf, nrhs, e, qe, err, st);
}

template <int Q>
static cudaError_t h2_e2qbxl_q(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int nrhs,
                               const double2* e, double2* qe, int32_t* err, bool from_local,
                               cudaStream_t st)
{
  if (pf > 20 || g.nqbx_chunks == 0) return pf > 20 ? cudaErrorInvalidValue : cudaSuccess;
  if (from_local) return h2_e2qbxl_qf<Q, true>(g, hc, pf, nrhs, e, qe, err, st);
  return h2_e2qbxl_qf<Q, false>(g, hc, pf, nrhs, e, qe, err, st);
}

template <int Q>
static cudaError_t h2_qbxl2p_q(const qbxfmm_geometry& g, HelmCoeffs hc, int nrhs, const double2* qe,
                               double2* pt, cudaStream_t st)
{
  dim3 grid((g.nglobal_qbx_centers + NT - 1) / NT, nrhs);
  k_h2_qbxl2p<Q><<<grid, NT, 0, st>>>(g, hc, nrhs, qe, pt);
  return cudaGetLastError();
}

#define QBX_H2_DISPATCH(FN, Q, ...)                                  \
  switch (Q) {                                                       \
    case 0: return FN<0>(__VA_ARGS__);                               \
    case 1: return FN<1>(__VA_ARGS__);                               \
    case 2: return FN<2>(__VA_ARGS__);                               \
    case 3: return FN<3>(__VA_ARGS__);                               \
    case 4: return FN<4>(__VA_ARGS__);                               \
    case 5: return FN<5>(__VA_ARGS__);                               \
    case 6: return FN<6>(__VA_ARGS__);                               \
    case 7: return FN<7>(__VA_ARGS__);                               \
    case 8: return FN<8>(__VA_ARGS__);                               \
    default: return cudaErrorInvalidValue;                           \
  }

cudaError_t h2_launch_p2qbxl(const qbxfmm_geometry& g, HelmCoeffs hc, int q, int nrhs,
                             const double2* s, double2* qe, int32_t* err, cudaStream_t st)
{
  if (g.nqbx_chunks == 0) return cudaSuccess;
  QBX_H2_DISPATCH(h2_p2qbxl_q, q, g, hc, nrhs, s, qe, err, st)
}

cudaError_t h2_launch_m2qbxl(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int q, int nrhs,
                             const double2* mp, double2* qe, int32_t* err, cudaStream_t st)
{
  if (g.nglobal_qbx_centers == 0) return cudaSuccess;
  QBX_H2_DISPATCH(h2_e2qbxl_q, q, g, hc, pf, nrhs, mp, qe, err, false, st)
}

cudaError_t h2_launch_l2qbxl(const qbxfmm_geometry& g, HelmCoeffs hc, int pf, int q, int nrhs,
                             const double2* lo, double2* qe, int32_t* err, cudaStream_t st)
{
  if (g.nglobal_qbx_centers == 0) return cudaSuccess;
  QBX_H2_DISPATCH(h2_e2qbxl_q, q, g, hc, pf, nrhs, lo, qe, err, true, st)
}

cudaError_t h2_launch_qbxl2p(const qbxfmm_geometry& g, HelmCoeffs hc, int q, int nrhs,
                             const double2* qe, double2* pt, cudaStream_t st)
{
  if (g.nglobal_qbx_centers == 0) return cudaSuccess;
  QBX_H2_DISPATCH(h2_qbxl2p_q, q, g, hc, nrhs, qe, pt, st)
}

template <int Q, int RB>
static cudaError_t h2_tsqbx_qr(const qbxfmm_geometry& g, HelmCoeffs hc, int nrhs, const double2* s,
                               double2* pt, int32_t* err, cudaStream_t st)
{
  size_t sh = (size_t)(NW - 1) * 32 * RB * sizeof(double2);
  cudaFuncSetAttribute(k_h2_tsqbx<Q, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  dim3 grid(g.ntsqbx_chunks, (nrhs + RB - 1) / RB);
  k_h2_tsqbx<Q, RB><<<grid, NT, sh, st>>>(g, hc, nrhs, s, pt, err);
  return cudaGetLastError();
}

template <int Q>
static cudaError_t h2_tsqbx_many_q(const qbxfmm_geometry& g, HelmCoeffs hc, int nrhs,
                                   const double2* s, double2* pt, int32_t* err, cudaStream_t st)
{
  size_t sh = (size_t)TS_ST * (TS_RC + 1 + 32) * sizeof(double2);
  cudaError_t ce = cudaFuncSetAttribute(k_h2_tsqbx_many<Q>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (ce != cudaSuccess) return ce;
  dim3 grid(g.ntsqbx_chunks, (nrhs + TS_RC - 1) / TS_RC);
  k_h2_tsqbx_many<Q><<<grid, NT, sh, st>>>(g, hc, nrhs, s, pt, err);
  return cudaGetLastError();
}

template <int Q>
static cudaError_t h2_tsqbx_q(const qbxfmm_geometry& g, HelmCoeffs hc, int nrhs, const double2* s,
                              double2* pt, int32_t* err, cudaStream_t st)
{
  if (nrhs > 16) return h2_tsqbx_many_q<Q>(g, hc, nrhs, s, pt, err, st);
  if (nrhs == 1) return h2_tsqbx_qr<Q, 1>(g, hc, nrhs, s, pt, err, st);
  if (nrhs <= 4) return h2_tsqbx_qr<Q, 4>(g, hc, nrhs, s, pt, err, st);
  return h2_tsqbx_qr<Q, 16>(g, hc, nrhs, s, pt, err, st);
}

cudaError_t h2_launch_tsqbx(const qbxfmm_geometry& g, HelmCoeffs hc, int q, int nrhs,
                            const double2* s, double2* pt, int32_t* err, cudaStream_t st)
{
  if (g.ntsqbx_chunks == 0) return cudaSuccess;
  QBX_H2_DISPATCH(h2_tsqbx_q, q, g, hc, nrhs, s, pt, err, st)
}

cudaError_t h2_launch_assemble(const qbxfmm_geometry& g, int nrhs, const double2* pot_nonqbx,
                               const double2* pot_tree, double2* out, cudaStream_t st)
{
  if (g.ntargets > 0) {
    k_h2_assemble_tree<<<dim3((g.ntargets + 255) / 256, nrhs), 256, 0, st>>>(g, nrhs, pot_tree, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (g.nfiltered_targets > 0)
    k_h2_assemble_nonqbx<<<dim3((g.nfiltered_targets + 255) / 256, nrhs), 256, 0, st>>>(
        g, nrhs, pot_nonqbx, out);
  return cudaGetLastError();
}

// }}}

}  // namespace qbx
