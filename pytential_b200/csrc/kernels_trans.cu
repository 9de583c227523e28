// Matrix form of the 3D Laplace box translations (M2L, M2M, L2L) on the FP64
// tensor cores (mma.sync m8n8k4 f64), sm_100a.
//
// With rscale-scaled coefficients a translation between boxes depends only on the
// translation vector in units of the box width: every list-2 pair with the same
// integer offset uses the same matrix (times 1/rho of the level, applied in the
// reduction), every M2M / L2L pair with the same child position uses the same
// matrix at every level.  A translation acts on the stored coefficients
// (m >= 0, the rest by conjugate symmetry) as a real-linear map, so each class is a
// real (2 ncoeff) x (2 ncoeff) matrix T acting on interleaved (re, im) vectors.
//
//   k_trans_build  : one CTA per class, T from the harmonic table of the class vector
//   k_trans_gemm   : one CTA per (class, 32 pairs x rhs): C = T X with X the gathered
//                    source expansions; T and X staged in shared memory
//   k_trans_reduce : deterministic sum of each output box's pair results (list order)
//
// M2L classes related by a lattice symmetry (quarter turns about z, y and z
// reflections) share the matrix of their canonical offset: the GEMM applies the
// class's input map to the gathered columns and its output map to the products
// (m2l_symmetry_classes, laplace.cuh).
#include "laplace.cuh"
#include "kernels.h"

#include <algorithm>
#include <array>
#include <cstdlib>
#include <map>
#include <vector>

#include <cooperative_groups.h>
namespace cg = cooperative_groups;

namespace qbx {

namespace {

constexpr int NT = 128;
constexpr int NTILE = 32;            // max columns (pair x rhs) per CTA
constexpr int XS = NTILE + 4;        // padded X row stride (conflict-free B fragments)

QBX_D void dmma_8x8x4(double& d0, double& d1, double a, double b)
{
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

}  // namespace

// {{{ T construction

// kind 0 = M2L (class vector d = offset, S table of order 2p; value (-1)^j S),
// kind 1 = M2M (d = (child - parent) / rho_parent, R table of order p),
// kind 2 = L2L (same d, R table).
__global__ void __launch_bounds__(NT)
k_trans_build(int kind, int p, int ncf, int rp, int kp, int nclasses, const int32_t* __restrict__ offs,
              double* __restrict__ T)
{
  extern __shared__ double2 tab[];
  int cls = blockIdx.x;
  double d[3];
  if (kind == 0) {
    for (int k = 0; k < 3; ++k) d[k] = (double)offs[k * nclasses + cls];
  } else {
    // child position bits -> +-1/4 per axis (child centre relative to the parent)
    for (int k = 0; k < 3; ++k) d[k] = ((cls >> k) & 1) ? 0.25 : -0.25;
  }
  if (kind == 0) sh3_S_table(2 * p, d[0], d[1], d[2], tab, threadIdx.x, NT);
  else sh3_R_table(p, d[0], d[1], d[2], tab, threadIdx.x, NT);
  __syncthreads();
  double* Tc = T + (size_t)cls * rp * kp;
  const int R = 2 * ncf;
  for (int e = threadIdx.x; e < rp * kp; e += NT) {
    int row = e / kp, col = e - row * kp;
    double v = 0.0;
    if (row < R && col < R) {
      int co = row >> 1, ci = col >> 1;
      int no, mo, ni, mi;
      decode3(co, no, mo);
      decode3(ci, ni, mi);
      // unit input u at stored (ni, mi); its symmetric partner at -mi is u' = (-1)^mi conj(u)
      double2 u = (col & 1) ? c2(0.0, 1.0) : c2(1.0, 0.0);
      double2 up = cconj(u);
      if (mi & 1) up = c2(-up.x, -up.y);
      double2 val = c2(0.0);
      if (kind == 0) {
        // L_j^i = (-1)^j sum M_k^l S_{k+j}^{l+i}
        val = cmul(u, sh3_get(tab, ni + no, mi + mo));
        if (mi > 0) val = cadd(val, cmul(up, sh3_get(tab, ni + no, -mi + mo)));
        if (no & 1) val = c2(-val.x, -val.y);
      } else if (kind == 1) {
        // M'_n^m = sum (1/2)^k M_k^l conj(R_{n-k}^{m-l})
        double rk = ldexp(1.0, -ni);
        val = cmulc(u, sh3_get(tab, no - ni, mo - mi));
        if (mi > 0) val = cadd(val, cmulc(up, sh3_get(tab, no - ni, mo + mi)));
        val = cscale(rk, val);
      } else {
        // L''_k^l = (1/2)^k sum L_n^m conj(R_{n-k}^{m-l})
        double rk = ldexp(1.0, -no);
        val = cmulc(u, sh3_get(tab, ni - no, mi - mo));
        if (mi > 0) val = cadd(val, cmulc(up, sh3_get(tab, ni - no, -mi - mo)));
        val = cscale(rk, val);
      }
      v = (row & 1) ? val.y : val.x;
    }
    Tc[e] = v;
  }
}

// }}}

// {{{ GEMM

constexpr int KC = 32;               // K chunk staged per step
constexpr int TSTR = KC + 4;         // padded T-chunk row stride (== 4 mod 16 doubles)

// C = T X for one group (class) and one tile of columns (pair x rhs).  Warps are
// arranged NWN (column tiles of 8) x NWM (row groups); each warp holds MTW m-tiles
// of 8 rows x one 8-column tile in registers.  T and X are streamed in K chunks of
// KC through shared memory.  If pair_dst is given the result is added (x scale)
// into the destination box's expansion (each destination occurs once per launch),
// else stored into cpair[pair * nrhs + r][0..rp).
template <int MTW>
__global__ void __launch_bounds__(NT)
k_trans_gemm(int ncf, int rp, int kp, int nrhs, int nwm, const double* __restrict__ T,
             int mat_base, int mat_mod, const int32_t* __restrict__ cls_code,
             const int32_t* __restrict__ group_starts, int g0,
             const int32_t* __restrict__ pair_src, const int32_t* __restrict__ pair_dst,
             const double2* __restrict__ ein, double2* __restrict__ eout, double scale,
             double* __restrict__ cpair, int32_t* err, int nboxes)
{
  extern __shared__ double sm[];
  const int nwn = 4 / nwm;
  const int ntile = 8 * nwn;
  double* Ts = sm;                          // [rp][TSTR]
  double* Xs = sm + (size_t)rp * TSTR;      // [KC][XS]
  __shared__ int s_src[NTILE];
  int grp = g0 + blockIdx.y;
  int p0 = group_starts[grp], p1 = group_starts[grp + 1];
  int ncol = (p1 - p0) * nrhs;
  int c0 = blockIdx.x * ntile;
  if (c0 >= ncol) return;
  int mat = mat_base + (mat_mod > 0 ? (grp % mat_mod) : grp), sym = 0;
  if (cls_code) {
    const int code = cls_code[grp];
    mat = mat_base + (code >> 4);
    sym = code & 15;
  }
  const double* Tg = T + (size_t)mat * rp * kp;
  const int R = 2 * ncf;
  __shared__ uint8_t s_opi[M2L_SYM_MAXR], s_opo[M2L_SYM_MAXR];
  if (sym) m2l_sym_tables(sym, R, s_opi, s_opo, threadIdx.x, NT);
  for (int j = threadIdx.x; j < ntile; j += NT) {
    int c = c0 + j;
    int src = -1;
    if (c < ncol) {
      src = pair_src[p0 + c / nrhs];
      if ((unsigned)src >= (unsigned)nboxes) {
        report(err, QBX_DEVERR_BAD_BOX);
        src = -1;
      }
    }
    s_src[j] = src;
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int g = lane >> 2, tq = lane & 3;
  int wn = warp % nwn, wm = warp / nwn;
  int mt = rp / 8;
  int mtw = (mt + nwm - 1) / nwm;
  int mbeg = wm * mtw;
  double acc[MTW][2];
#pragma unroll
  for (int i = 0; i < MTW; ++i) acc[i][0] = acc[i][1] = 0.0;
  for (int kc = 0; kc < kp; kc += KC) {
    int kw = min(KC, kp - kc);
    __syncthreads();
    // 16-byte loads and stores: kp, kc, kw, TSTR, R and every matrix offset are even
    constexpr int KH = KC / 2;
    for (int e = threadIdx.x; e < rp * KH; e += NT) {
      const int row = e / KH, col = 2 * (e - row * KH);
      const double2 v = col < kw
          ? __ldg(reinterpret_cast<const double2*>(Tg + (size_t)row * kp + kc + col)) : c2(0.0);
      *reinterpret_cast<double2*>(Ts + row * TSTR + col) = v;
    }
    for (int e = threadIdx.x; e < ntile * KH; e += NT) {
      const int j = e / KH, k = 2 * (e - j * KH);
      const int src = s_src[j];
      double v0 = 0.0, v1 = 0.0;
      if (src >= 0 && k < kw && kc + k < R) {
        const int r = (c0 + j) % nrhs, kg = kc + k;
        const double2 z = __ldg(ein + ((size_t)src * nrhs + r) * ncf + (kg >> 1));
        if (sym) {
          const int o0 = s_opi[kg], o1 = s_opi[kg + 1];
          v0 = (o0 & 1) ? z.y : z.x;
          v1 = (o1 & 1) ? z.x : z.y;
          if (o0 & 2) v0 = -v0;
          if (o1 & 2) v1 = -v1;
        } else {
          v0 = z.x;
          v1 = z.y;
        }
      }
      Xs[k * XS + j] = v0;
      Xs[(k + 1) * XS + j] = v1;
    }
    __syncthreads();
    for (int k0 = 0; k0 < kw; k0 += 4) {
      double b = Xs[(k0 + tq) * XS + wn * 8 + g];
#pragma unroll
      for (int i = 0; i < MTW; ++i) {
        int mi = mbeg + i;
        if (mi < mt) {
          double a = Ts[(mi * 8 + g) * TSTR + k0 + tq];
          dmma_8x8x4(acc[i][0], acc[i][1], a, b);
        }
      }
    }
  }
  // epilogue: acc[i][v] = C[row = (mbeg + i) * 8 + g][col = wn * 8 + 2 tq + v]; with a
  // class symmetry, its output map first (the other half of row's coefficient, row ^ 1,
  // is in lane ^ 4)
  if (sym) {
#pragma unroll
    for (int v = 0; v < 2; ++v)
#pragma unroll
      for (int i = 0; i < MTW; ++i) {
        const double other = __shfl_xor_sync(0xffffffffu, acc[i][v], 4);
        const int row = (mbeg + i) * 8 + g;
        if (mbeg + i < mt && row < R) {
          const int op = s_opo[row];
          const double w = (op & 1) ? other : acc[i][v];
          acc[i][v] = (op & 2) ? -w : w;
        }
      }
  }
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    int j = wn * 8 + 2 * tq + v;
    int c = c0 + j;
    if (c >= ncol) continue;
    int pr = p0 + c / nrhs, r = c % nrhs;
    if (pair_dst) {
      int dst = pair_dst[pr];
      if ((unsigned)dst >= (unsigned)nboxes) {
        report(err, QBX_DEVERR_BAD_BOX);
        continue;
      }
      double* y = reinterpret_cast<double*>(eout + ((size_t)dst * nrhs + r) * ncf);
#pragma unroll
      for (int i = 0; i < MTW; ++i) {
        int row = (mbeg + i) * 8 + g;
        if (mbeg + i < mt && row < R) y[row] += scale * acc[i][v];
      }
    } else {
      double* y = cpair + ((size_t)pr * nrhs + r) * rp;
#pragma unroll
      for (int i = 0; i < MTW; ++i) {
        int row = (mbeg + i) * 8 + g;
        if (mbeg + i < mt) y[row] = acc[i][v];
      }
    }
  }
}

// Tiled form for large matrices (rp >= 256): CTA tile of 64 rows x 64 columns
// (pair x rhs), K streamed in chunks of 32; warp (wm, wn) owns 32 x 32 of the tile
// as 4 x 4 m8n8 accumulators.  Groups g0 .. g0 + gridDim.z - 1 (blockIdx.z).  The
// result is added (x scale) into pair_dst's expansion when given (the caller
// guarantees each destination occurs once per launch), else stored per pair.
constexpr int GT_M = 64, GT_N = 64, GT_K = 32;
constexpr int GT_AS = GT_K + 4;      // A row stride (doubles)
constexpr int GT_BS = GT_N + 8;      // B row stride (doubles)

__global__ void __launch_bounds__(NT)
k_trans_gemm_tiled(int ncf, int rp, int kp, int nrhs, const double* __restrict__ T, int mat_mod,
                   const int32_t* __restrict__ group_starts, int g0,
                   const int32_t* __restrict__ pair_src, const int32_t* __restrict__ pair_dst,
                   const double2* __restrict__ ein, double2* __restrict__ eout, double scale,
                   double* __restrict__ cpair, int32_t* err, int nboxes)
{
  __shared__ __align__(16) double As[GT_M][GT_AS];
  __shared__ __align__(16) double Bs[GT_K][GT_BS];
  __shared__ int s_src[GT_N];
  int grp = g0 + blockIdx.z;
  int p0 = group_starts[grp], p1 = group_starts[grp + 1];
  int ncol = (p1 - p0) * nrhs;
  int c0 = blockIdx.x * GT_N;
  int m0 = blockIdx.y * GT_M;
  if (c0 >= ncol || m0 >= rp) return;
  int mat = mat_mod > 0 ? (grp % mat_mod) : grp;
  const double* Tg = T + (size_t)mat * rp * kp;
  const int R = 2 * ncf;
  for (int j = threadIdx.x; j < GT_N; j += NT) {
    int c = c0 + j;
    int src = -1;
    if (c < ncol) {
      src = pair_src[p0 + c / nrhs];
      if ((unsigned)src >= (unsigned)nboxes) {
        report(err, QBX_DEVERR_BAD_BOX);
        src = -1;
      }
    }
    s_src[j] = src;
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int g = lane >> 2, tq = lane & 3;
  int wm = warp & 1, wn = warp >> 1;
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  for (int kc = 0; kc < kp; kc += GT_K) {
    __syncthreads();
    // 16-byte loads and stores (kp, kc, GT_AS, R and the matrix offsets are even)
    constexpr int KH = GT_K / 2;
    for (int e = threadIdx.x; e < GT_M * KH; e += NT) {
      const int row = e / KH, k = 2 * (e - row * KH);
      const double2 v = (m0 + row < rp && kc + k < kp)
          ? __ldg(reinterpret_cast<const double2*>(Tg + (size_t)(m0 + row) * kp + kc + k)) : c2(0.0);
      *reinterpret_cast<double2*>(&As[row][k]) = v;
    }
    for (int e = threadIdx.x; e < GT_N * KH; e += NT) {
      const int j = e / KH, k = 2 * (e - j * KH);
      const int src = s_src[j];
      double2 v = c2(0.0);
      if (src >= 0 && kc + k < R)
        v = __ldg(ein + ((size_t)src * nrhs + (c0 + j) % nrhs) * ncf + ((kc + k) >> 1));
      Bs[k][j] = v.x;
      Bs[k + 1][j] = v.y;
    }
    __syncthreads();
#pragma unroll
    for (int k0 = 0; k0 < GT_K; k0 += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[wm * 32 + i * 8 + g][k0 + tq];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[k0 + tq][wn * 32 + j * 8 + g];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
  }
  // epilogue: acc[i][j][v] = C[row = m0 + wm*32 + i*8 + g][col = c0 + wn*32 + j*8 + 2 tq + v]
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      int c = c0 + wn * 32 + j * 8 + 2 * tq + v;
      if (c >= ncol) continue;
      int pr = p0 + c / nrhs, r = c % nrhs;
      if (pair_dst) {
        int dst = pair_dst[pr];
        if ((unsigned)dst >= (unsigned)nboxes) {
          report(err, QBX_DEVERR_BAD_BOX);
          continue;
        }
        double* y = reinterpret_cast<double*>(eout + ((size_t)dst * nrhs + r) * ncf);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          int row = m0 + wm * 32 + i * 8 + g;
          if (row < R) y[row] += scale * acc[i][j][v];
        }
      } else {
        double* y = cpair + ((size_t)pr * nrhs + r) * rp;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          int row = m0 + wm * 32 + i * 8 + g;
          if (row < rp) y[row] = acc[i][j][v];
        }
      }
    }
}

// out box o (o = boxes[obase + blockIdx.x]): eout[o][r] += scale(o) sum_{pairs} cpair[pair][r]
// scale(o) = 1 / width(level(o)) when div_by_width, else 1.
__global__ void __launch_bounds__(NT)
k_trans_reduce(int ncf, int rp, int nrhs, const int32_t* __restrict__ boxes, int obase,
               const int32_t* __restrict__ starts, const int32_t* __restrict__ pairs,
               const double* __restrict__ cpair, double2* __restrict__ eout, int div_by_width,
               const int32_t* __restrict__ box_levels, double root_extent)
{
  int i = obase + blockIdx.x;
  int o = boxes[i];
  int r = blockIdx.y;
  double sc = div_by_width ? ldexp(1.0, box_levels[o]) / root_extent : 1.0;
  int R = 2 * ncf;
  double* y = reinterpret_cast<double*>(eout + ((size_t)o * nrhs + r) * ncf);
  const int q0 = starts[i], q1 = starts[i + 1];
  // the box's pair rows, staged once per chunk so that the loads of successive pairs
  // are independent
  constexpr int QC = 256;
  __shared__ const double* s_row[QC];
  for (int row0 = 0; row0 < R; row0 += NT) {
    const int row = row0 + threadIdx.x;
    double acc = 0.0;
    for (int qc = q0; qc < q1; qc += QC) {
      const int nq = min(QC, q1 - qc);
      __syncthreads();
      for (int t = threadIdx.x; t < nq; t += NT)
        s_row[t] = cpair + ((size_t)pairs[qc + t] * nrhs + r) * rp;
      __syncthreads();
      if (row < R) {
#pragma unroll 4
        for (int t = 0; t < nq; ++t) acc += s_row[t][row];
      }
    }
    if (row < R) y[row] += sc * acc;
  }
}

// }}}

// {{{ M2M / L2L as matrix-vector products (small matrices)

// group g of a pair: group_starts[g] <= pr < group_starts[g + 1], g in [g0, g0 + 8)
QBX_D int pair_group(const int32_t* __restrict__ group_starts, int g0, int pr)
{
  int grp = g0;
  while (grp + 1 < g0 + 8 && group_starts[grp + 1] <= pr) ++grp;
  return grp;
}

// y[row] += sum_k T[row][k] x[k] over one matrix, rows row0 and row0 + NT; x in
// shared memory (kp doubles, zero-padded).  Eight row loads are issued before their
// products, so that a thread keeps 128 bytes of the (L2-resident) matrix in flight.
QBX_D void mv_rows(const double* __restrict__ Tm, int kp, int R, const double* x, double* acc2,
                   int row0)
{
  const int n2 = kp / 2;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int row = row0 + h * NT;
    if (row >= R) break;
    const double2* tr = reinterpret_cast<const double2*>(Tm + (size_t)row * kp);
    const double2* xv = reinterpret_cast<const double2*>(x);
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    int k2 = 0;
    for (; k2 + 8 <= n2; k2 += 8) {
      double2 t[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) t[u] = __ldg(tr + k2 + u);
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        double2 xx = xv[k2 + u];
        a[u & 3] = fma(t[u].x, xx.x, a[u & 3]);
        a[u & 3] = fma(t[u].y, xx.y, a[u & 3]);
      }
    }
    for (; k2 < n2; ++k2) {
      double2 t0 = __ldg(tr + k2), x0 = xv[k2];
      a[0] = fma(t0.x, x0.x, a[0]);
      a[1] = fma(t0.y, x0.y, a[1]);
    }
    acc2[h] += (a[0] + a[1]) + (a[2] + a[3]);
  }
}

// M2M of one level: a cluster of eight CTAs per source parent box (i = i0 +
// blockIdx.x / 8, density blockIdx.y); CTA c multiplies child slot c's multipole by
// its (child position) matrix, and CTA 0 adds the eight products into the parent in
// a fixed order through distributed shared memory.
__global__ void __cluster_dims__(8, 1, 1) __launch_bounds__(NT)
k_trans_m2m_mv(int ncf, int rp, int kp, int nrhs, const double* __restrict__ T, size_t mat_base,
               int mat_mod, const int32_t* __restrict__ group_starts, int g0,
               const int32_t* __restrict__ parents, int i0, const int32_t* __restrict__ par_starts,
               const int32_t* __restrict__ par_pairs, const int32_t* __restrict__ pair_src,
               double2* __restrict__ mp, int32_t* err, int nboxes)
{
  extern __shared__ double xs[];   // [kp] child multipole, then [2 NT] product rows
  double* res = xs + kp;
  cg::cluster_group cl = cg::this_cluster();
  int i = i0 + blockIdx.x / 8;
  int slot = blockIdx.x & 7;
  int r = blockIdx.y;
  int q0 = par_starts[i];
  int nch = min(par_starts[i + 1] - q0, 8);
  const int R = 2 * ncf;
  double acc[2] = {0.0, 0.0};
  if (slot < nch) {
    int pr = par_pairs[q0 + slot];
    int src = pair_src[pr];
    int grp = pair_group(group_starts, g0, pr);
    bool ok = (unsigned)src < (unsigned)nboxes;
    if (!ok && threadIdx.x == 0) report(err, QBX_DEVERR_BAD_BOX);
    const double* x = reinterpret_cast<const double*>(mp + ((size_t)(ok ? src : 0) * nrhs + r) * ncf);
    for (int k = threadIdx.x; k < kp; k += NT) xs[k] = (ok && k < R) ? x[k] : 0.0;
    __syncthreads();
    int mat = (int)mat_base + (mat_mod > 0 ? grp % mat_mod : grp);
    mv_rows(T + (size_t)mat * rp * kp, kp, R, xs, acc, threadIdx.x);
  }
  res[threadIdx.x] = acc[0];
  res[threadIdx.x + NT] = acc[1];
  cl.sync();
  if (slot == 0) {
    int parent = parents[i];
    if ((unsigned)parent >= (unsigned)nboxes) {
      if (threadIdx.x == 0) report(err, QBX_DEVERR_BAD_BOX);
    } else {
      double s0 = 0.0, s1 = 0.0;
      for (int q = 0; q < nch; ++q) {
        const double* rq = cl.map_shared_rank(res, q);
        s0 += rq[threadIdx.x];
        s1 += rq[threadIdx.x + NT];
      }
      double* y = reinterpret_cast<double*>(mp + ((size_t)parent * nrhs + r) * ncf);
      if (threadIdx.x < R) y[threadIdx.x] += s0;
      if (threadIdx.x + NT < R) y[threadIdx.x + NT] += s1;
    }
  }
  cl.sync();
}

// L2L of one level: CTA per (parent, child) pair p0 + blockIdx.x of the level's
// eight groups; child local += T_{child position} parent local.
__global__ void __launch_bounds__(NT)
k_trans_l2l_mv(int ncf, int rp, int kp, int nrhs, const double* __restrict__ T, size_t mat_base,
               int mat_mod, const int32_t* __restrict__ group_starts, int g0,
               const int32_t* __restrict__ pair_src, const int32_t* __restrict__ pair_dst,
               double2* __restrict__ lo, int32_t* err, int nboxes)
{
  extern __shared__ double xs[];   // [kp]
  int pr = group_starts[g0] + blockIdx.x;
  int r = blockIdx.y;
  int grp = pair_group(group_starts, g0, pr);
  int src = pair_src[pr], dst = pair_dst[pr];
  if ((unsigned)src >= (unsigned)nboxes || (unsigned)dst >= (unsigned)nboxes) {
    if (threadIdx.x == 0) report(err, QBX_DEVERR_BAD_BOX);
    return;
  }
  const int R = 2 * ncf;
  const double* x = reinterpret_cast<const double*>(lo + ((size_t)src * nrhs + r) * ncf);
  for (int k = threadIdx.x; k < kp; k += NT) xs[k] = k < R ? x[k] : 0.0;
  __syncthreads();
  double acc[2] = {0.0, 0.0};
  int mat = (int)mat_base + (mat_mod > 0 ? grp % mat_mod : grp);
  mv_rows(T + (size_t)mat * rp * kp, kp, R, xs, acc, threadIdx.x);
  double* y = reinterpret_cast<double*>(lo + ((size_t)dst * nrhs + r) * ncf);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int row = threadIdx.x + h * NT;
    if (row < R) y[row] += acc[h];
  }
}

// }}}

// {{{ launchers

static void dims_from_ncf(int ncf, int& rp, int& kp)
{
  rp = (2 * ncf + 7) / 8 * 8;
  kp = (2 * ncf + 3) / 4 * 4;
}

TransCfg trans_cfg_laplace3(int p, int nclasses)
{
  TransCfg c;
  c.p = p;
  c.ncf = (p + 1) * (p + 2) / 2;
  dims_from_ncf(c.ncf, c.rp, c.kp);
  c.m2m_mat_mod = 8;
  c.m2m_base = nclasses;
  c.l2l_base = nclasses + 8;
  c.m2l_div_by_width = 1;
  c.nmatrices = nclasses + 16;
  return c;
}

TransCfg trans_cfg_helm3(int p, int nclasses, int nlevels)
{
  TransCfg c;
  c.p = p;
  c.ncf = (p + 1) * (p + 1);
  dims_from_ncf(c.ncf, c.rp, c.kp);
  c.m2m_mat_mod = 0;
  c.m2m_base = nclasses;
  c.l2l_base = nclasses + 8 * (size_t)nlevels;
  c.m2l_div_by_width = 0;
  c.nmatrices = nclasses + 16 * (size_t)nlevels;
  return c;
}

size_t trans_matrix_bytes(const TransCfg& c) { return c.nmatrices * c.rp * c.kp * sizeof(double); }

size_t trans_scratch_bytes(const TransCfg& c, int npairs, int nrhs)
{
  return (size_t)(npairs > 0 ? npairs : 1) * nrhs * c.rp * sizeof(double);
}

static size_t gemm_smem(int rp) { return ((size_t)rp * TSTR + (size_t)KC * XS) * sizeof(double); }

// warp arrangement: nwm row groups so that each warp holds <= 24 m-tiles
static int gemm_nwm(int rp)
{
  int mt = rp / 8;
  return mt <= 24 ? 1 : (mt <= 48 ? 2 : 4);
}

bool trans_supported(const TransCfg& c) { return c.rp / 8 <= 96 && gemm_smem(c.rp) <= 200 * 1024; }

M2LSymClasses m2l_symmetry_classes(int nclasses, const std::vector<int32_t>& offs)
{
  M2LSymClasses r;
  r.cls_code.resize(nclasses);
  std::vector<std::array<int, 3>> canon;
  std::map<std::array<int, 3>, int> index;
  for (int c = 0; c < nclasses; ++c) {
    const int dx = offs[c], dy = offs[(size_t)nclasses + c], dz = offs[2 * (size_t)nclasses + c];
    const int a = std::max(std::abs(dx), std::abs(dy)), b = std::min(std::abs(dx), std::abs(dy));
    const std::array<int, 3> key = {a, b, std::abs(dz)};
    // (dx, dy) = R^q C^s (a, b)
    int code = -1;
    for (int q = 0; q < 4 && code < 0; ++q)
      for (int s = 0; s < 2 && code < 0; ++s) {
        int x = a, y = s ? -b : b;
        for (int i = 0; i < q; ++i) {
          const int t = x;
          x = -y;
          y = t;
        }
        if (x == dx && y == dy) code = q | s << 2 | (dz < 0 ? 8 : 0);
      }
    auto it = index.find(key);
    int ci;
    if (it == index.end()) {
      ci = (int)canon.size();
      index.emplace(key, ci);
      canon.push_back(key);
    } else {
      ci = it->second;
    }
    if (code < 0) {                      // not a lattice offset: no shared matrices
      r.ncanon = -1;
      return r;
    }
    r.cls_code[c] = ci << 4 | code;
  }
  r.ncanon = (int)canon.size();
  r.canon_off.resize(3 * (size_t)r.ncanon);
  for (int i = 0; i < r.ncanon; ++i)
    for (int k = 0; k < 3; ++k) r.canon_off[(size_t)k * r.ncanon + i] = canon[i][k];
  return r;
}

// T layout: [0, nm2l) M2L matrices (one per canonical offset), then M2M and L2L
// matrices (TransCfg bases); offs: [3][nm2l] on the device
cudaError_t launch_trans_build(const TransCfg& c, int nm2l, const int32_t* offs, double* T,
                               cudaStream_t st)
{
  int p = c.p;
  size_t sh = (size_t)(2 * p + 1) * (2 * p + 2) / 2 * sizeof(double2);
  size_t stride = (size_t)c.rp * c.kp;
  if (nm2l > 0)
    k_trans_build<<<nm2l, NT, sh, st>>>(0, p, c.ncf, c.rp, c.kp, nm2l, offs, T);
  k_trans_build<<<8, NT, sh, st>>>(1, p, c.ncf, c.rp, c.kp, 8, nullptr, T + c.m2m_base * stride);
  k_trans_build<<<8, NT, sh, st>>>(2, p, c.ncf, c.rp, c.kp, 8, nullptr, T + c.l2l_base * stride);
  return cudaGetLastError();
}

static cudaError_t gemm_launch(const qbxfmm_geometry& g, const TransCfg& c, int nrhs, const double* T,
                               size_t mat_base, int mat_mod, const int32_t* cls_code,
                               const int32_t* group_starts_dev,
                               int g0, int ngroups, int maxcols, const int32_t* pair_src,
                               const int32_t* pair_dst, const double2* ein, double2* eout,
                               double scale, double* cpair, int32_t* err, cudaStream_t st)
{
  if (ngroups <= 0 || maxcols <= 0) return cudaSuccess;
  int ncf = c.ncf, rp = c.rp, kp = c.kp;
  size_t sh = gemm_smem(rp);
  int nwm = gemm_nwm(rp);
  int ntile = 8 * (4 / nwm);
  int mtw = (rp / 8 + nwm - 1) / nwm;
  dim3 grid((maxcols + ntile - 1) / ntile, ngroups);
  const double* Tb = T + mat_base * (size_t)rp * kp;
#define QBX_GEMM_CASE(W)                                                                        \
  if (mtw <= W) {                                                                               \
    cudaFuncSetAttribute(k_trans_gemm<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh); \
    k_trans_gemm<W><<<grid, NT, sh, st>>>(ncf, rp, kp, nrhs, nwm, Tb, 0, mat_mod, cls_code,     \
                                          group_starts_dev, g0, pair_src, pair_dst, ein, eout,  \
                                          scale, cpair, err, g.nboxes);                         \
    return cudaGetLastError();                                                                  \
  }
  QBX_GEMM_CASE(8)
  QBX_GEMM_CASE(12)
  QBX_GEMM_CASE(16)
  QBX_GEMM_CASE(20)
  QBX_GEMM_CASE(24)
#undef QBX_GEMM_CASE
  return cudaErrorInvalidValue;
}

cudaError_t launch_m2l_gemm(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                            int nrhs, const double* T, const TransAux& aux, const double2* mp,
                            double2* lo, double* cpair, int32_t* err, cudaStream_t st)
{
  if (g.m2l_nclasses == 0) return cudaSuccess;
  cudaError_t e = gemm_launch(g, c, nrhs, T, 0, 0, aux.cls_code, g.m2l_class_starts, 0,
                              g.m2l_nclasses, th.m2l_max_pairs * nrhs, g.m2l_pair_src, nullptr, mp,
                              nullptr, 1.0, cpair, err, st);
  if (e != cudaSuccess) return e;
  return launch_trans_reduce_m2l(g, c, nrhs, cpair, lo, st);
}

cudaError_t launch_m2m_gemm(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                            int nrhs, const double* T, double2* mp, double* cpair, int32_t* err,
                            cudaStream_t st)
{
  const int nch = 8;
  for (int lev = g.nlevels - 2; lev >= 0; --lev) {
    int g0 = lev * nch;
    int maxp = th.m2m_level_max_group[lev];
    if (maxp == 0) continue;
    cudaError_t e = gemm_launch(g, c, nrhs, T, c.m2m_base, c.m2m_mat_mod, nullptr, g.m2m_group_starts, g0,
                                nch, maxp * nrhs, g.m2m_pair_src, nullptr, mp, nullptr, 1.0, cpair,
                                err, st);
    if (e != cudaSuccess) return e;
    int i0 = th.lvl_source_parent[lev], i1 = th.lvl_source_parent[lev + 1];
    if (i1 > i0)
      k_trans_reduce<<<dim3(i1 - i0, nrhs), NT, 0, st>>>(c.ncf, c.rp, nrhs, g.source_parent_boxes,
                                                         i0, g.m2m_par_pair_starts, g.m2m_par_pairs,
                                                         cpair, mp, 0, g.box_levels, g.root_extent);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_l2l_gemm(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                            int nrhs, const double* T, double2* lo, int32_t* err, cudaStream_t st)
{
  const int nch = 8;
  for (int lev = 1; lev < g.nlevels; ++lev) {
    int g0 = lev * nch;
    int maxp = th.l2l_level_max_group[lev];
    if (maxp == 0) continue;
    cudaError_t e = gemm_launch(g, c, nrhs, T, c.l2l_base, c.m2m_mat_mod, nullptr, g.l2l_group_starts, g0,
                                nch, maxp * nrhs, g.l2l_pair_src, g.l2l_pair_dst, lo, lo, 1.0,
                                nullptr, err, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_trans_reduce_m2l(const qbxfmm_geometry& g, const TransCfg& c, int nrhs,
                                    const double* cpair, double2* lo, cudaStream_t st)
{
  if (g.nttp_boxes == 0) return cudaSuccess;
  k_trans_reduce<<<dim3(g.nttp_boxes, nrhs), NT, 0, st>>>(
      c.ncf, c.rp, nrhs, g.target_or_target_parent_boxes, 0, g.m2l_tgt_pair_starts,
      g.m2l_tgt_pairs, cpair, lo, c.m2l_div_by_width, g.box_levels, g.root_extent);
  return cudaGetLastError();
}

cudaError_t launch_trans_reduce_m2m(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                                    int lev, int nrhs, const double* cpair, double2* mp,
                                    cudaStream_t st)
{
  int i0 = th.lvl_source_parent[lev], i1 = th.lvl_source_parent[lev + 1];
  if (i1 > i0)
    k_trans_reduce<<<dim3(i1 - i0, nrhs), NT, 0, st>>>(c.ncf, c.rp, nrhs, g.source_parent_boxes, i0,
                                                       g.m2m_par_pair_starts, g.m2m_par_pairs, cpair,
                                                       mp, 0, g.box_levels, g.root_extent);
  return cudaGetLastError();
}

static cudaError_t gemm_tiled_launch(const qbxfmm_geometry& g, const TransCfg& c, int nrhs,
                                     const double* T, size_t mat_base, int mat_mod,
                                     const int32_t* group_starts_dev, int g0, int ngroups,
                                     int maxcols, const int32_t* pair_src, const int32_t* pair_dst,
                                     const double2* ein, double2* eout, double scale,
                                     double* cpair, int32_t* err, cudaStream_t st)
{
  if (ngroups <= 0 || maxcols <= 0) return cudaSuccess;
  dim3 grid((maxcols + GT_N - 1) / GT_N, (c.rp + GT_M - 1) / GT_M, ngroups);
  k_trans_gemm_tiled<<<grid, NT, 0, st>>>(c.ncf, c.rp, c.kp, nrhs, T + mat_base * (size_t)c.rp * c.kp,
                                          mat_mod, group_starts_dev, g0, pair_src, pair_dst, ein,
                                          eout, scale, cpair, err, g.nboxes);
  return cudaGetLastError();
}

// M2M without pair scratch: one launch per (parent level, child position) group,
// whose parents are distinct.
cudaError_t launch_m2m_direct(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                              int nrhs, const double* T, double2* mp, int32_t* err, cudaStream_t st)
{
  const int nch = 8;
  for (int lev = g.nlevels - 2; lev >= 0; --lev) {
    int maxp = th.m2m_level_max_group[lev];
    if (maxp == 0) continue;
    for (int ci = 0; ci < nch; ++ci) {
      cudaError_t e = gemm_tiled_launch(g, c, nrhs, T, c.m2m_base, c.m2m_mat_mod, g.m2m_group_starts,
                                        lev * nch + ci, 1, maxp * nrhs, g.m2m_pair_src,
                                        g.m2m_pair_dst, mp, mp, 1.0, nullptr, err, st);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

// L2L on the tiled kernel (children are distinct across a level's eight groups)
cudaError_t launch_l2l_direct(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                              int nrhs, const double* T, double2* lo, int32_t* err, cudaStream_t st)
{
  const int nch = 8;
  for (int lev = 1; lev < g.nlevels; ++lev) {
    int maxp = th.l2l_level_max_group[lev];
    if (maxp == 0) continue;
    cudaError_t e = gemm_tiled_launch(g, c, nrhs, T, c.l2l_base, c.m2m_mat_mod, g.l2l_group_starts,
                                      lev * nch, nch, maxp * nrhs, g.l2l_pair_src, g.l2l_pair_dst,
                                      lo, lo, 1.0, nullptr, err, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}


bool trans_mv_supported(const TransCfg& c) { return 2 * c.ncf <= 2 * NT && c.kp % 2 == 0; }

// M2M level by level as matrix-vector products, eight CTAs per parent (small matrices)
cudaError_t launch_m2m_mv(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                          int nrhs, const double* T, double2* mp, int32_t* err, cudaStream_t st)
{
  size_t sh = ((size_t)c.kp + 2 * NT) * sizeof(double);
  for (int lev = g.nlevels - 2; lev >= 0; --lev) {
    int i0 = th.lvl_source_parent[lev], i1 = th.lvl_source_parent[lev + 1];
    if (i1 <= i0) continue;
    k_trans_m2m_mv<<<dim3(8 * (i1 - i0), nrhs), NT, sh, st>>>(
        c.ncf, c.rp, c.kp, nrhs, T, c.m2m_base, c.m2m_mat_mod, g.m2m_group_starts, lev * 8,
        g.source_parent_boxes, i0, g.m2m_par_pair_starts, g.m2m_par_pairs, g.m2m_pair_src, mp, err,
        g.nboxes);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// L2L level by level, CTA per (parent, child) pair
cudaError_t launch_l2l_mv(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                          int nrhs, const double* T, double2* lo, int32_t* err, cudaStream_t st)
{
  size_t sh = (size_t)c.kp * sizeof(double);
  for (int lev = 1; lev < g.nlevels; ++lev) {
    int n = th.l2l_level_pairs[lev];
    if (n == 0) continue;
    k_trans_l2l_mv<<<dim3(n, nrhs), NT, sh, st>>>(c.ncf, c.rp, c.kp, nrhs, T, c.l2l_base,
                                                  c.m2m_mat_mod, g.l2l_group_starts, lev * 8,
                                                  g.l2l_pair_src, g.l2l_pair_dst, lo, err, g.nboxes);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// }}}

}  // namespace qbx
