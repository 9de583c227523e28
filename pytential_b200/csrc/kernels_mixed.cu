// Mixed-precision far field of the 3D Laplace apply (qbxfmm_kernel.precision = 1).
//
// The far-field stages compute in FP32 while the expansions stay stored in FP64
// (each kernel loads FP64, computes in FP32, accumulates its result back into the
// FP64 array): P2M, P2L and M2QBXL on the FP32 pipe, and the matrix-form
// translations (M2M, M2L, L2L) on the tensor cores as split-TF32 products
// (a = a_hi + a_lo in TF32, a b ~ a_hi b_hi + a_hi b_lo + a_lo b_hi, FP32 accumulation):
// M2L on tcgen05 with the accumulator in tensor memory, the rest (and matrices of more
// than 256 rows) with mma.sync m16n8k8 tf32.  The QBX near field (P2QBXL / target-specific, QBXL2P), the
// non-QBX point evaluations and L2QBXL stay FP64.  Expansions, scalings and work
// decomposition are those of the FP64 kernels in kernels_laplace.cu / kernels_trans.cu.
#include <algorithm>

#include "laplace.cuh"
#include "kernels.h"

#include <cooperative_groups.h>
namespace cg = cooperative_groups;

namespace qbx {

namespace {

constexpr int NT = 128;
constexpr int NW = NT / 32;
constexpr int MAXB = 128;

QBX_D float frcp(int i) { return (float)rcp(i); }

QBX_D void mx_list_prefix(const qbxfmm_geometry& g, const int32_t* __restrict__ lists, int gb,
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

QBX_D int mx_stream_source(int v, int nb, const int* s_pref, const int* s_start)
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

// {{{ P2M (FP32)

constexpr int MX_SUB = 16;
constexpr int MX_TS = MX_SUB + 1;

__global__ void __launch_bounds__(NT)
k_p2m3_f32(qbxfmm_geometry g, SourceCoeffs sc, int p, int ncf, int nrhs,
           const double* __restrict__ strengths, double2* __restrict__ mpoles)
{
  constexpr int SUB = MX_SUB, TS = MX_TS;
  extern __shared__ float2 smf[];
  float2* tab = smf;                                   // [ncf][TS]
  __shared__ float s_u[SUB][3], s_n[SUB][3], s_q[SUB];
  int b = g.source_boxes[blockIdx.x];
  int r = blockIdx.y;
  double rho = level_width(g, g.box_levels[b]);
  double rinv = 1.0 / rho;
  double c[3];
  load_point<3>(g.box_centers, g.nboxes, b, c);
  int s0 = g.box_source_starts[b];
  int ns = g.box_source_counts_nonchild[b];
  const double* st = strengths + (size_t)r * g.nsources;
  const bool dip = sc.cd != 0.0;
  const float cq = (float)sc.cq, cdr = (float)(sc.cd * rinv);

  int o_nm[2], o_a[2], o_b[2], o_c[2];
  float w_a[2], w_b[2], w_c[2];
  bool valid[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int ci = threadIdx.x + h * NT;
    valid[h] = ci < ncf;
    o_nm[h] = o_a[h] = o_b[h] = o_c[h] = 0;
    w_a[h] = w_b[h] = w_c[h] = 0.0f;
    if (valid[h]) {
      int n, m;
      decode3(ci, n, m);
      o_nm[h] = idx3(n, m) * TS;
      if (n >= 1) {
        if (m <= n - 1) { o_a[h] = idx3(n - 1, m) * TS; w_a[h] = 1.0f; }
        if (m >= 1) { o_b[h] = idx3(n - 1, m - 1) * TS; w_b[h] = 1.0f; }
        else if (n - 1 >= 1) { o_b[h] = idx3(n - 1, 1) * TS; w_b[h] = -1.0f; }
        if (m + 1 <= n - 1) { o_c[h] = idx3(n - 1, m + 1) * TS; w_c[h] = 1.0f; }
      }
    }
  }
  float2 acc[2] = {f2(0.0f), f2(0.0f)};
  for (int base = 0; base < ns; base += SUB) {
    int cnt = min(SUB, ns - base);
    if (threadIdx.x < cnt) {
      int s = s0 + base + threadIdx.x;
      double y[3];
      load_point<3>(g.sources, g.nsources, s, y);
#pragma unroll
      for (int d = 0; d < 3; ++d) s_u[threadIdx.x][d] = (float)((y[d] - c[d]) * rinv);
      if (dip) {
        double nv[3];
        load_point<3>(g.source_normals, g.nsources, s, nv);
#pragma unroll
        for (int d = 0; d < 3; ++d) s_n[threadIdx.x][d] = (float)nv[d];
      }
      s_q[threadIdx.x] = (float)__ldg(st + s);
    }
    __syncthreads();
    for (int w = threadIdx.x; w < cnt * (p + 1); w += NT) {
      int m = w / cnt, j = w - m * cnt;
      float x = s_u[j][0], y = s_u[j][1], z = s_u[j][2];
      float r2 = x * x + y * y + z * z;
      float2 a = f2(1.0f);
      for (int k = 1; k <= m; ++k) a = fscale(0.5f * frcp(k), fmul(a, f2(x, y)));
      float2* T = tab + j;
      T[idx3(m, m) * TS] = a;
      float2 prev = f2(0.0f);
      for (int n = m + 1; n <= p; ++n) {
        float2 bb = fscale(frcp(n + m) * frcp(n - m), fsub(fscale((2.0f * n - 1) * z, a), fscale(r2, prev)));
        T[idx3(n, m) * TS] = bb;
        prev = a;
        a = bb;
      }
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (!valid[h]) continue;
      float2 a = acc[h];
      for (int j = 0; j < cnt; ++j) {
        const float2* T = tab + j;
        float q = s_q[j];
        a = faxpy(cq * q, fconj(T[o_nm[h]]), a);
        if (dip) {
          float f = cdr * q;
          float dx = s_n[j][0], dy = s_n[j][1], dz = s_n[j][2];
          float2 tb_ = T[o_b[h]];
          tb_ = (w_b[h] < 0.0f) ? f2(-tb_.x, tb_.y) : fscale(w_b[h], tb_);
          float2 v = fscale(dz * w_a[h], T[o_a[h]]);
          v = ffma(f2(0.5f * dx, 0.5f * dy), tb_, v);
          v = ffma(f2(-0.5f * dx * w_c[h], 0.5f * dy * w_c[h]), T[o_c[h]], v);
          a = faxpy(f, fconj(v), a);
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
    if (ci < ncf) M[ci] = cadd(M[ci], tod(acc[h]));
  }
}

// }}}

// {{{ P2L (FP32)

constexpr int MX_LSUB = 32;
constexpr int MX_LTS = MX_LSUB + 1;

__global__ void __launch_bounds__(NT)
k_p2l3_f32(qbxfmm_geometry g, SourceCoeffs sc, int p, int ncf, int nrhs,
           const double* __restrict__ strengths, double2* __restrict__ locals, int32_t* err)
{
  constexpr int SUB = MX_LSUB, TS = MX_LTS;
  extern __shared__ float2 smf[];
  float2* tab = smf;   // [nct][TS]
  __shared__ float s_u[SUB][3], s_n[SUB][3], s_q[SUB];
  __shared__ int s_pref[MAXB + 1], s_start[MAXB];
  int i = blockIdx.x;
  int tb = g.target_or_target_parent_boxes[i];
  int r = blockIdx.y;
  int l0 = g.list4_starts[i], l1 = g.list4_starts[i + 1];
  if (l1 <= l0) return;
  double rho = level_width(g, g.box_levels[tb]);
  double rinv = 1.0 / rho;
  double c[3];
  load_point<3>(g.box_centers, g.nboxes, tb, c);
  const double* st = strengths + (size_t)r * g.nsources;
  const bool dip = sc.cd != 0.0;
  const float cqr = (float)(sc.cq * rinv), cdr2 = (float)(sc.cd * rinv * rinv);
  int o_nm[2], o_a[2], o_b[2], o_c[2];
  float sb_sign[2];
  bool valid[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int ci = threadIdx.x + h * NT;
    valid[h] = ci < ncf;
    o_nm[h] = o_a[h] = o_b[h] = o_c[h] = 0;
    sb_sign[h] = 1.0f;
    if (valid[h]) {
      int n, m;
      decode3(ci, n, m);
      o_nm[h] = idx3(n, m) * TS;
      o_a[h] = idx3(n + 1, m) * TS;
      o_b[h] = idx3(n + 1, m > 0 ? m - 1 : 1) * TS;
      sb_sign[h] = m > 0 ? 1.0f : -1.0f;
      o_c[h] = idx3(n + 1, m + 1) * TS;
    }
  }
  float2 acc[2] = {f2(0.0f), f2(0.0f)};
  for (int gb = l0; gb < l1; gb += MAXB) {
    int nb = min(MAXB, l1 - gb);
    __syncthreads();
    mx_list_prefix(g, g.list4_lists, gb, nb, s_pref, s_start, err);
    __syncthreads();
    int total = s_pref[nb];
    for (int base = 0; base < total; base += SUB) {
      int cnt = min(SUB, total - base);
      if (threadIdx.x < cnt) {
        int s = mx_stream_source(base + threadIdx.x, nb, s_pref, s_start);
        double y[3];
        load_point<3>(g.sources, g.nsources, s, y);
#pragma unroll
        for (int d = 0; d < 3; ++d) s_u[threadIdx.x][d] = (float)((y[d] - c[d]) * rinv);
        if (dip) {
          double nv[3];
          load_point<3>(g.source_normals, g.nsources, s, nv);
#pragma unroll
          for (int d = 0; d < 3; ++d) s_n[threadIdx.x][d] = (float)nv[d];
        }
        s_q[threadIdx.x] = (float)__ldg(st + s);
      }
      __syncthreads();
      for (int w = threadIdx.x; w < cnt * (p + 2); w += NT) {
        int m = w / cnt, j = w - m * cnt;
        float x = s_u[j][0], y = s_u[j][1], z = s_u[j][2];
        float rinv2 = 1.0f / (x * x + y * y + z * z);
        float2 a = f2(sqrtf(rinv2));
        for (int k = 1; k <= m; ++k) a = fscale((2.0f * k - 1) * rinv2, fmul(a, f2(x, y)));
        float2* T = tab + j;
        T[idx3(m, m) * TS] = a;
        float2 prev = f2(0.0f);
        for (int n = m + 1; n <= p + 1; ++n) {
          float2 bb = fscale(rinv2, fsub(fscale((2.0f * n - 1) * z, a),
                                         fscale((float)((n + m - 1) * (n - m - 1)), prev)));
          T[idx3(n, m) * TS] = bb;
          prev = a;
          a = bb;
        }
      }
      __syncthreads();
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (!valid[h]) continue;
        float2 a = acc[h];
        for (int j = 0; j < cnt; ++j) {
          const float2* T = tab + j;
          float q = s_q[j];
          a = faxpy(cqr * q, T[o_nm[h]], a);
          if (dip) {
            float f = cdr2 * q;
            float dx = s_n[j][0], dy = s_n[j][1], dz = s_n[j][2];
            float2 tb_ = T[o_b[h]];
            if (sb_sign[h] < 0.0f) tb_ = f2(-tb_.x, tb_.y);
            float2 v = fscale(-dz, T[o_a[h]]);
            v = ffma(f2(0.5f * dx, 0.5f * dy), tb_, v);
            v = ffma(f2(-0.5f * dx, 0.5f * dy), T[o_c[h]], v);
            a = faxpy(f, v, a);
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
    if (o < ncf) L[o] = cadd(L[o], tod(acc[h]));
  }
}

// }}}

// {{{ M2QBXL (FP32)

// clusters of M2QBXL3_F32_Z CTAs per chunk split the list-3 boxes; partial sums meet
// in CTA 0 of the cluster in a fixed order through distributed shared memory
constexpr int M2QBXL3_F32_Z = 4;

template <int Q>
__global__ void __cluster_dims__(M2QBXL3_F32_Z, 1, 1) __launch_bounds__(NT)
k_m2qbxl3_f32(qbxfmm_geometry g, int pf, int ncf, int nrhs, const double2* __restrict__ mpoles,
              double2* __restrict__ qbx_exps, int32_t* err)
{
  constexpr int NC = (Q + 1) * (Q + 2) / 2;
  extern __shared__ float2 smf[];
  const int MW = 2 * pf + 3 * Q + 1;
  const int MR = pf + 2 * Q + 1;
  const int MSZ = MR * MW;
  const int loff = pf + 2 * Q;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int MZ = M2QBXL3_F32_Z;
  float2* Mw = smf + (size_t)warp * MSZ;
  float2* red = smf + (size_t)NW * MSZ;   // [NW-1][32][NC]
  float2* cpart = red + (NW - 1) * 32 * NC;  // [32][NC]: this CTA's sum
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
  double cc[3];
  load_point<3>(g.centers, g.ncenters, ctr, cc);
  double rho_t = g.expansion_radii[ctr];
  for (int q = lane; q < MSZ; q += 32) Mw[q] = f2(0.0f);
  float2 acc[NC];
#pragma unroll
  for (int i = 0; i < NC; ++i) acc[i] = f2(0.0f);
  int l0 = g.list3_starts[itb], l1 = g.list3_starts[itb + 1];
  for (int li = l0 + zpart * NW + warp; li < l1; li += MZ * NW) {
    int sb = g.list3_lists[li];
    if ((unsigned)sb >= (unsigned)g.nboxes) {
      report(err, QBX_DEVERR_BAD_BOX);
      continue;
    }
    __syncwarp();
    const double2* src = mpoles + ((size_t)sb * nrhs + r) * ncf;
    for (int q = lane; q < ncf; q += 32) {
      int k, l;
      decode3(q, k, l);
      float2 v = tof(src[q]);
      Mw[(k + Q) * MW + loff + l] = v;
      if (l > 0) Mw[(k + Q) * MW + loff - l] = (l & 1) ? f2(-v.x, v.y) : f2(v.x, -v.y);
    }
    __syncwarp();
    if (!has_center) continue;
    double rho_s = level_width(g, g.box_levels[sb]);
    double cs[3];
    load_point<3>(g.box_centers, g.nboxes, sb, cs);
    float ratio = (float)(rho_t / rho_s);
    float d0 = (float)((cc[0] - cs[0]) / rho_s), d1 = (float)((cc[1] - cs[1]) / rho_s),
          d2 = (float)((cc[2] - cs[2]) / rho_s);
    float rinv2 = 1.0f / (d0 * d0 + d1 * d1 + d2 * d2);
    int nmax = pf + Q;
    float2 part[NC];
#pragma unroll
    for (int i = 0; i < NC; ++i) part[i] = f2(0.0f);
    float2 mm = f2(sqrtf(rinv2));
    for (int mp = 0; mp <= nmax; ++mp) {
      if (mp > 0) mm = fscale((2.0f * mp - 1) * rinv2, fmul(mm, f2(d0, d1)));
      float2 a = mm, prev = f2(0.0f);
      const float2* bpos = Mw + (mp + Q) * MW + loff + mp;
      const float2* bneg = Mw + (mp + Q) * MW + loff - mp;
      for (int np = mp; np <= nmax; ++np) {
        if (np > mp) {
          float2 bb = fscale(rinv2, fsub(fscale((2.0f * np - 1) * d2, a),
                                         fscale((float)((np + mp - 1) * (np - mp - 1)), prev)));
          prev = a;
          a = bb;
        }
#pragma unroll
        for (int j = 0; j <= Q; ++j)
#pragma unroll
          for (int ii = 0; ii <= j; ++ii)
            part[idx3(j, ii)] = ffma(bpos[-j * MW - ii], a, part[idx3(j, ii)]);
        if (mp > 0) {
          float2 aneg = (mp & 1) ? f2(-a.x, a.y) : f2(a.x, -a.y);
#pragma unroll
          for (int j = 0; j <= Q; ++j)
#pragma unroll
            for (int ii = 0; ii <= j; ++ii)
              part[idx3(j, ii)] = ffma(bneg[-j * MW - ii], aneg, part[idx3(j, ii)]);
        }
        bpos += MW;
        bneg += MW;
      }
    }
    float rj = (float)(1.0 / rho_s);
#pragma unroll
    for (int j = 0; j <= Q; ++j) {
#pragma unroll
      for (int ii = 0; ii <= j; ++ii)
        acc[idx3(j, ii)] = faxpy((j & 1) ? -rj : rj, part[idx3(j, ii)], acc[idx3(j, ii)]);
      rj *= ratio;
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
    for (int i = 0; i < NC; ++i) {
      for (int w = 1; w < NW; ++w) acc[i] = fadd(acc[i], red[((w - 1) * 32 + lane) * NC + i]);
      cpart[lane * NC + i] = acc[i];
    }
  }
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();
  if (zpart == 0 && warp == 0) {
    for (unsigned q = 1; q < MZ; ++q) {
      const float2* rp = cl.map_shared_rank(cpart, q) + lane * NC;
#pragma unroll
      for (int i = 0; i < NC; ++i) acc[i] = fadd(acc[i], rp[i]);
    }
  }
  cl.sync();
  if (zpart == 0 && warp == 0 && has_center) {
    double2* out = qbx_exps + ((size_t)ctr * nrhs + r) * NC;
#pragma unroll
    for (int i = 0; i < NC; ++i) out[i] = cadd(out[i], tod(acc[i]));
  }
}

// }}}

// {{{ split-TF32 translation GEMM

QBX_D uint32_t to_tf32(float x)
{
  uint32_t u;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(x));
  return u;
}

QBX_D void mma_tf32(float* d, const uint32_t* a, const uint32_t* b)
{
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
      "{%8, %9}, {%0, %1, %2, %3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// FP64 matrices [nmat][rp][kp] -> TF32 hi / lo planes [nmat][rp16][kp8] (zero padded)
__global__ void k_trans_split_tf32(int nmat, int rp, int kp, int rp16, int kp8, int R,
                                   const double* __restrict__ T, uint32_t* __restrict__ Thi,
                                   uint32_t* __restrict__ Tlo)
{
  size_t n = (size_t)nmat * rp16 * kp8;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    size_t mat = e / ((size_t)rp16 * kp8);
    int rem = (int)(e - mat * rp16 * kp8);
    int row = rem / kp8, col = rem - row * kp8;
    float v = (row < R && col < R) ? (float)T[(mat * rp + row) * kp + col] : 0.0f;
    uint32_t hi = to_tf32(v);
    Thi[e] = hi;
    Tlo[e] = to_tf32(v - __uint_as_float(hi));
  }
}

constexpr int X3_KC = 32;      // K staged per step
constexpr int X3_AS = X3_KC + 4;
constexpr int X3_NW = 4;       // warps, one n8 column tile each
constexpr int X3_N = 8 * X3_NW;
constexpr int X3_MT = 16;      // max m16 tiles (rows <= 256)

// C = T X (split TF32, FP32 accumulation) for one group and 32 columns (pair x rhs);
// all row tiles in every warp.  Output as in k_trans_gemm: added (x scale) into
// pair_dst's expansion, or stored per pair into cpair (FP64, row stride rp).
__global__ void __launch_bounds__(NT)
k_trans_gemm_x3(int ncf, int rp, int rp16, int kp8, int nrhs, const uint32_t* __restrict__ Thi,
                const uint32_t* __restrict__ Tlo, int mat_mod, const int32_t* __restrict__ cls_code,
                const int32_t* __restrict__ group_starts,
                int g0, const int32_t* __restrict__ pair_src, const int32_t* __restrict__ pair_dst,
                const double2* __restrict__ ein, double2* __restrict__ eout, double scale,
                double* __restrict__ cpair, int32_t* err, int nboxes)
{
  extern __shared__ uint32_t smu[];
  uint32_t* Ah = smu;                                   // [rp16][X3_AS]
  uint32_t* Al = Ah + (size_t)rp16 * X3_AS;             // [rp16][X3_AS]
  uint32_t* Bh = Al + (size_t)rp16 * X3_AS;             // [X3_KC][X3_N + 4]
  uint32_t* Bl = Bh + (size_t)X3_KC * (X3_N + 4);
  __shared__ int s_src[X3_N];
  const int BS = X3_N + 4;
  int grp = g0 + blockIdx.y;
  int p0 = group_starts[grp], p1 = group_starts[grp + 1];
  int ncol = (p1 - p0) * nrhs;
  int c0 = blockIdx.x * X3_N;
  if (c0 >= ncol) return;
  int mat = mat_mod > 0 ? (grp % mat_mod) : grp, sym = 0;
  if (cls_code) {
    const int code = cls_code[grp];
    mat = code >> 4;
    sym = code & 15;
  }
  __shared__ uint8_t s_opi[M2L_SYM_MAXR], s_opo[M2L_SYM_MAXR];
  if (sym) m2l_sym_tables(sym, 2 * ncf, s_opi, s_opo, threadIdx.x, NT);
  const uint32_t* Th = Thi + (size_t)mat * rp16 * kp8;
  const uint32_t* Tl = Tlo + (size_t)mat * rp16 * kp8;
  const int R = 2 * ncf;
  for (int j = threadIdx.x; j < X3_N; j += NT) {
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
  int mt = rp16 / 16;
  float acc[X3_MT][4];
#pragma unroll
  for (int i = 0; i < X3_MT; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.0f;
  for (int kc = 0; kc < kp8; kc += X3_KC) {
    int kw = min(X3_KC, kp8 - kc);
    __syncthreads();
    for (int e = threadIdx.x; e < rp16 * X3_KC; e += NT) {
      int row = e / X3_KC, col = e - row * X3_KC;
      bool ok = col < kw;
      Ah[row * X3_AS + col] = ok ? __ldg(Th + (size_t)row * kp8 + kc + col) : 0u;
      Al[row * X3_AS + col] = ok ? __ldg(Tl + (size_t)row * kp8 + kc + col) : 0u;
    }
    for (int e = threadIdx.x; e < X3_N * X3_KC; e += NT) {
      int j = e / X3_KC, k = e - j * X3_KC;
      int src = s_src[j];
      float v = 0.0f;
      if (src >= 0 && k < kw && kc + k < R) {
        int r = (c0 + j) % nrhs;
        const double2* x2 = ein + ((size_t)src * nrhs + r) * ncf;
        const int kg = kc + k;
        const double* x = reinterpret_cast<const double*>(x2);
        v = (float)(sym ? m2l_sym_apply(x, kg, s_opi[kg]) : __ldg(x + kg));
      }
      uint32_t hi = to_tf32(v);
      Bh[k * BS + j] = hi;
      Bl[k * BS + j] = to_tf32(v - __uint_as_float(hi));
    }
    __syncthreads();
    for (int k0 = 0; k0 < kw; k0 += 8) {
      uint32_t bh[2], bl[2];
      int col = warp * 8 + g;
      bh[0] = Bh[(k0 + tq) * BS + col];
      bh[1] = Bh[(k0 + tq + 4) * BS + col];
      bl[0] = Bl[(k0 + tq) * BS + col];
      bl[1] = Bl[(k0 + tq + 4) * BS + col];
#pragma unroll
      for (int i = 0; i < X3_MT; ++i) {
        if (i >= mt) break;
        int r0 = i * 16 + g;
        uint32_t ah[4], al[4];
        ah[0] = Ah[r0 * X3_AS + k0 + tq];
        ah[1] = Ah[(r0 + 8) * X3_AS + k0 + tq];
        ah[2] = Ah[r0 * X3_AS + k0 + tq + 4];
        ah[3] = Ah[(r0 + 8) * X3_AS + k0 + tq + 4];
        al[0] = Al[r0 * X3_AS + k0 + tq];
        al[1] = Al[(r0 + 8) * X3_AS + k0 + tq];
        al[2] = Al[r0 * X3_AS + k0 + tq + 4];
        al[3] = Al[(r0 + 8) * X3_AS + k0 + tq + 4];
        mma_tf32(acc[i], al, bh);
        mma_tf32(acc[i], ah, bl);
        mma_tf32(acc[i], ah, bh);
      }
    }
  }
  // epilogue: acc[i][v] = C[row = i*16 + g + 8 (v >> 1)][col = warp*8 + 2 tq + (v & 1)];
  // with a class symmetry, its output map first (row ^ 1 is in lane ^ 4)
  if (sym) {
#pragma unroll
    for (int i = 0; i < X3_MT; ++i)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const float other = __shfl_xor_sync(0xffffffffu, acc[i][v], 4);
        const int row = i * 16 + g + 8 * (v >> 1);
        if (i < mt && row < R) {
          const int op = s_opo[row];
          const float w = (op & 1) ? other : acc[i][v];
          acc[i][v] = (op & 2) ? -w : w;
        }
      }
  }
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    int c = c0 + warp * 8 + 2 * tq + (v & 1);
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
      for (int i = 0; i < X3_MT; ++i) {
        if (i >= mt) break;
        int row = i * 16 + g + 8 * (v >> 1);
        if (row < R) y[row] += scale * (double)acc[i][v];
      }
    } else {
      double* y = cpair + ((size_t)pr * nrhs + r) * rp;
#pragma unroll
      for (int i = 0; i < X3_MT; ++i) {
        if (i >= mt) break;
        int row = i * 16 + g + 8 * (v >> 1);
        if (row < R) y[row] = (double)acc[i][v];
      }
    }
  }
}

// }}}

// {{{ split-TF32 M2L on the 5th-generation tensor cores (tcgen05, accumulator in TMEM)

// C^T = X^T T^T for one translation class and 128 columns (pair x density): M = 128
// columns, N = the matrix rows (rp16 <= 256), K = kp8 in chunks of 32, split TF32
// (three products lo.hi, hi.lo, hi.hi into one FP32 accumulator in tensor memory).
// Operands live in shared memory in the no-swizzle K-major layout (8-row x 16-byte
// core matrices, contiguous).  The class matrix's TF32 planes are stored at precompute
// in that layout chunk by chunk, so each chunk of B arrives with one bulk copy per
// plane (cp.async.bulk, completion on an mbarrier); the threads split the gathered
// source expansions (A) into TF32 hi / lo.  Two stages: while the tensor core works
// on chunk i (one thread issues its MMAs and commits them to the stage's mbarrier),
// the copy engine and the threads fill chunk i + 1.  The accumulator is read back with
// tcgen05.ld (warps w and w + 4 own TMEM lanes 32 (w mod 4) .. + 31, i.e. those
// columns, and split the rows) and stored per pair into the FP64 pair scratch.  Waits
// are bounded: a wait that runs out sets the error word; the CTA then waits (bounded)
// for its copies and MMAs, frees its tensor memory and stops.
constexpr int UM_M = 128;        // columns per CTA (MMA M)
constexpr int UM_KC = 32;        // K per chunk (four MMA K-steps of 8)
constexpr int UM_TCOLS = 256;    // tensor-memory columns allocated (>= N, power of two)
constexpr int UM_NT = 256;       // threads

QBX_D unsigned um_smem(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// no-swizzle K-major shared-memory descriptor: start address, leading byte offset
// (between the two 16-byte K halves of an MMA K-step), stride byte offset (between
// 8-row groups), version 1 (sm_100), layout type 0
QBX_D uint64_t um_desc(unsigned saddr, unsigned lbo, unsigned sbo)
{
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// offset (in 32-bit words) of element (row, k) of a [rows][UM_KC] operand chunk
QBX_HD int um_off(int row, int k)
{
  return (((row >> 3) * (UM_KC / 4) + (k >> 2)) << 5) + ((row & 7) << 2) + (k & 3);
}

QBX_D void um_mma(unsigned tmem, uint64_t da, uint64_t db, unsigned idesc, int acc)
{
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n"
      ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

QBX_D bool um_wait(uint64_t* mb, unsigned parity)
{
  const unsigned a = um_smem(mb);
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done) : "r"(a), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}

// FP64 matrices [nmat][rp][kp] -> TF32 hi / lo planes in the chunked core-matrix layout
// [nmat][kp8 / 32 chunks][rp16 x 32] (zero padded)
__global__ void k_trans_umma_planes(int nmat, int rp, int kp, int rp16, int nkc, int R,
                                    const double* __restrict__ T, uint32_t* __restrict__ Uhi,
                                    uint32_t* __restrict__ Ulo)
{
  const size_t per = (size_t)nkc * rp16 * UM_KC;
  const size_t n = (size_t)nmat * per;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t mat = e / per;
    const int rem = (int)(e - mat * per);
    const int kc = rem / (rp16 * UM_KC), w = rem - kc * (rp16 * UM_KC);
    const int row = w / UM_KC, kk = w - row * UM_KC, k = kc * UM_KC + kk;
    const float v = (row < R && k < R) ? (float)T[(mat * rp + row) * kp + k] : 0.0f;
    const uint32_t hi = to_tf32(v);
    const size_t o = mat * per + (size_t)kc * rp16 * UM_KC + um_off(row, kk);
    Uhi[o] = hi;
    Ulo[o] = to_tf32(v - __uint_as_float(hi));
  }
}

__global__ void __launch_bounds__(UM_NT)
k_trans_gemm_umma(int ncf, int rp, int rp16, int nkc, int nrhs, const uint32_t* __restrict__ Uhi,
                  const uint32_t* __restrict__ Ulo, const int32_t* __restrict__ cls_code,
                  const int32_t* __restrict__ group_starts,
                  const int32_t* __restrict__ pair_src, const double2* __restrict__ ein,
                  double* __restrict__ cpair, int32_t* err, int nboxes)
{
  extern __shared__ __align__(1024) uint32_t smu[];
  const int aw = UM_M * UM_KC, bw = rp16 * UM_KC;       // words per plane and stage
  // stage s: A hi, A lo, B hi, B lo
  auto Ah = [&](int st) { return smu + (size_t)st * 2 * (aw + bw); };
  auto Al = [&](int st) { return Ah(st) + aw; };
  auto Bh = [&](int st) { return Al(st) + aw; };
  auto Bl = [&](int st) { return Bh(st) + bw; };
  __shared__ uint64_t full[2], mdone[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_src[UM_M];
  const int grp = blockIdx.y;
  const int p0 = group_starts[grp], p1 = group_starts[grp + 1];
  const int ncol = (p1 - p0) * nrhs;
  const int c0 = blockIdx.x * UM_M;
  if (c0 >= ncol) return;                               // uniform, before any allocation
  const size_t mper = (size_t)nkc * bw;
  const int code = cls_code ? cls_code[grp] : grp << 4;
  const int mat = code >> 4, sym = code & 15;
  __shared__ uint8_t s_opi[M2L_SYM_MAXR], s_opo[M2L_SYM_MAXR];
  if (sym) m2l_sym_tables(sym, 2 * ncf, s_opi, s_opo, threadIdx.x, UM_NT);
  const uint32_t* Th = Uhi + (size_t)mat * mper;
  const uint32_t* Tl = Ulo + (size_t)mat * mper;
  const int R = 2 * ncf;
  const int warp = threadIdx.x >> 5;
  if (threadIdx.x < UM_M) {
    const int c = c0 + threadIdx.x;
    int src = -1;
    if (c < ncol) {
      src = pair_src[p0 + c / nrhs];
      if ((unsigned)src >= (unsigned)nboxes) {
        report(err, QBX_DEVERR_BAD_BOX);
        src = -1;
      }
    }
    s_src[threadIdx.x] = src;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                 ::"r"(um_smem(&s_tmem)), "r"(UM_TCOLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (threadIdx.x == 0) {
    for (int b = 0; b < 2; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(um_smem(&full[b])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(um_smem(&mdone[b])) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const unsigned tmem = s_tmem;
  // kind::tf32: D F32 (bit 4), A and B TF32 (bits 7, 10), both K-major, N >> 3 at bit
  // 17, M >> 4 at bit 24
  const unsigned idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(rp16 >> 3) << 17) |
                         ((unsigned)(UM_M >> 4) << 24);
  const unsigned LBO = 128, SBO = (UM_KC / 4) * 128;
  const unsigned bbytes = (unsigned)bw * sizeof(uint32_t);
  // this thread's part of A: column row, K half khalf
  const int row = threadIdx.x & (UM_M - 1), khalf = threadIdx.x / UM_M;
  const int src = s_src[row];
  const double* xin = src >= 0
      ? reinterpret_cast<const double*>(ein + ((size_t)src * nrhs + (c0 + row) % nrhs) * ncf)
      : nullptr;
  // issued / completed counts per barrier (the same in every thread)
  int f_iss[2] = {0, 0}, f_done[2] = {0, 0}, m_iss[2] = {0, 0}, m_done[2] = {0, 0};
  auto fill = [&](int kc, int st) {
    if (threadIdx.x == 0) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n"
                   ::"r"(um_smem(&full[st])), "r"(2 * bbytes) : "memory");
      const uint32_t* gh = Th + (size_t)kc * bw;
      const uint32_t* gl = Tl + (size_t)kc * bw;
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                   ::"r"(um_smem(Bh(st))), "l"(gh), "r"(bbytes), "r"(um_smem(&full[st])) : "memory");
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                   ::"r"(um_smem(Bl(st))), "l"(gl), "r"(bbytes), "r"(um_smem(&full[st])) : "memory");
    }
    ++f_iss[st];
    uint32_t* ah = Ah(st);
    uint32_t* al = Al(st);
    // one coefficient (two entries, kg even; R is even) per load
#pragma unroll 4
    for (int j = 0; j < UM_KC / 2; j += 2) {
      const int k = khalf * (UM_KC / 2) + j, kg = kc * UM_KC + k;
      double2 z = c2(0.0);
      if (xin && kg < R) z = __ldg(reinterpret_cast<const double2*>(xin) + (kg >> 1));
      float v[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int op = sym ? s_opi[kg + u] : 0;
        const double w = ((u ^ op) & 1) ? z.y : z.x;
        v[u] = (float)((op & 2) ? -w : w);
        const uint32_t hi = to_tf32(v[u]);
        ah[um_off(row, k + u)] = hi;
        al[um_off(row, k + u)] = to_tf32(v[u] - __uint_as_float(hi));
      }
    }
  };
  bool fail = false;
  fill(0, 0);
  for (int kc = 0; kc < nkc; ++kc) {
    const int st = kc & 1;
    // chunk kc: its B copies have landed, its A is written (made visible to the
    // tensor core through the proxy fence and the barrier)
    if (!um_wait(&full[st], f_done[st] & 1)) fail = true;
    else ++f_done[st];
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    if (__syncthreads_or(fail)) break;
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const unsigned sAh = um_smem(Ah(st)), sAl = um_smem(Al(st));
      const unsigned sBh = um_smem(Bh(st)), sBl = um_smem(Bl(st));
      for (int s = 0; s < UM_KC / 8; ++s) {
        const unsigned off = (unsigned)s * 2 * 128;   // two 16-byte K halves per K-step
        const uint64_t dAh = um_desc(sAh + off, LBO, SBO), dAl = um_desc(sAl + off, LBO, SBO);
        const uint64_t dBh = um_desc(sBh + off, LBO, SBO), dBl = um_desc(sBl + off, LBO, SBO);
        const int first = (kc == 0 && s == 0);
        um_mma(tmem, dAl, dBh, idesc, !first);
        um_mma(tmem, dAh, dBl, idesc, 1);
        um_mma(tmem, dAh, dBh, idesc, 1);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                   ::"r"(um_smem(&mdone[st])) : "memory");
    }
    ++m_iss[st];
    if (kc + 1 < nkc) {
      // the other stage is free once the MMAs of chunk kc - 1 have read it
      const int so = st ^ 1;
      if (m_iss[so] > m_done[so]) {
        if (!um_wait(&mdone[so], m_done[so] & 1)) fail = true;
        else ++m_done[so];
      }
      if (__syncthreads_or(fail)) break;
      fill(kc + 1, so);
    }
  }
  // the last chunk's MMAs complete the accumulator
  if (!fail) {
    const int sl = (nkc - 1) & 1;
    if (m_iss[sl] > m_done[sl]) {
      if (!um_wait(&mdone[sl], m_done[sl] & 1)) fail = true;
      else ++m_done[sl];
    }
  }
  if (__syncthreads_or(fail)) {
    // drain (bounded) whatever is still in flight before the tensor memory goes
    if (threadIdx.x == 0) report(err, QBX_DEVERR_COPY_TIMEOUT);
    for (int b = 0; b < 2; ++b) {
      for (; f_done[b] < f_iss[b]; ++f_done[b]) um_wait(&full[b], f_done[b] & 1);
      for (; m_done[b] < m_iss[b]; ++m_done[b]) um_wait(&mdone[b], m_done[b] & 1);
    }
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const int lane_base = 32 * (warp & 3), c = c0 + lane_base + (threadIdx.x & 31);
    double* y = (c < ncol) ? cpair + ((size_t)(p0 + c / nrhs) * nrhs + c % nrhs) * rp : nullptr;
    for (int nb = 16 * (warp >> 2); nb < rp16; nb += 32) {
      uint32_t v[16];
      const unsigned ta = tmem + ((unsigned)lane_base << 16) + (unsigned)nb;
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, "
                   "%9, %10, %11, %12, %13, %14, %15}, [%16];\n"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                     "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                     "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                   : "r"(ta));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      if (y) {
        if (sym) {
          // the class symmetry's output map (rows nb + 2u, nb + 2u + 1 are one coefficient)
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (nb + j < R) {
              const int op = s_opo[nb + j];
              const float w = __uint_as_float((op & 1) ? v[j ^ 1] : v[j]);
              y[nb + j] = (double)((op & 2) ? -w : w);
            }
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (nb + j < R) y[nb + j] = (double)__uint_as_float(v[j]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n"
                 ::"r"(tmem), "r"(UM_TCOLS) : "memory");
  }
}

// }}}

// {{{ launchers

cudaError_t launch_p2m_mixed(const qbxfmm_geometry& g, SourceCoeffs sc, int p, int nrhs,
                             const double* s, double2* mp, cudaStream_t st)
{
  if (g.nsource_boxes == 0) return cudaSuccess;
  int ncf = (p + 1) * (p + 2) / 2;
  size_t sh = (size_t)MX_TS * ncf * sizeof(float2);
  cudaFuncSetAttribute(k_p2m3_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  k_p2m3_f32<<<dim3(g.nsource_boxes, nrhs), NT, sh, st>>>(g, sc, p, ncf, nrhs, s, mp);
  return cudaGetLastError();
}

cudaError_t launch_p2l_mixed(const qbxfmm_geometry& g, SourceCoeffs sc, int p, int nrhs,
                             const double* s, double2* lo, int32_t* err, cudaStream_t st)
{
  if (g.nttp_boxes == 0) return cudaSuccess;
  int ncf = (p + 1) * (p + 2) / 2;
  int nct = (p + 2) * (p + 3) / 2;
  size_t sh = (size_t)MX_LTS * nct * sizeof(float2);
  cudaFuncSetAttribute(k_p2l3_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  k_p2l3_f32<<<dim3(g.nttp_boxes, nrhs), NT, sh, st>>>(g, sc, p, ncf, nrhs, s, lo, err);
  return cudaGetLastError();
}

template <int Q>
static cudaError_t m2qbxl_mixed_q(const qbxfmm_geometry& g, int pf, int nrhs, const double2* mp,
                                  double2* qe, int32_t* err, cudaStream_t st)
{
  constexpr int NC = (Q + 1) * (Q + 2) / 2;
  int ncf = (pf + 1) * (pf + 2) / 2;
  size_t msz = (size_t)(pf + 2 * Q + 1) * (2 * pf + 3 * Q + 1);
  size_t sh = (NW * msz + (size_t)NW * 32 * NC) * sizeof(float2);
  cudaFuncSetAttribute(k_m2qbxl3_f32<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  k_m2qbxl3_f32<Q><<<dim3(g.nqbx_chunks * M2QBXL3_F32_Z, nrhs), NT, sh, st>>>(g, pf, ncf, nrhs, mp,
                                                                               qe, err);
  return cudaGetLastError();
}

cudaError_t launch_m2qbxl_mixed(const qbxfmm_geometry& g, int pf, int q, int nrhs,
                                const double2* mp, double2* qe, int32_t* err, cudaStream_t st)
{
  if (g.nqbx_chunks == 0) return cudaSuccess;
  switch (q) {
    case 0: return m2qbxl_mixed_q<0>(g, pf, nrhs, mp, qe, err, st);
    case 1: return m2qbxl_mixed_q<1>(g, pf, nrhs, mp, qe, err, st);
    case 2: return m2qbxl_mixed_q<2>(g, pf, nrhs, mp, qe, err, st);
    case 3: return m2qbxl_mixed_q<3>(g, pf, nrhs, mp, qe, err, st);
    case 4: return m2qbxl_mixed_q<4>(g, pf, nrhs, mp, qe, err, st);
    case 5: return m2qbxl_mixed_q<5>(g, pf, nrhs, mp, qe, err, st);
    case 6: return m2qbxl_mixed_q<6>(g, pf, nrhs, mp, qe, err, st);
    case 7: return m2qbxl_mixed_q<7>(g, pf, nrhs, mp, qe, err, st);
    case 8: return m2qbxl_mixed_q<8>(g, pf, nrhs, mp, qe, err, st);
    default: return cudaErrorInvalidValue;
  }
}

void tf32_dims(const TransCfg& c, int& rp16, int& kp8)
{
  rp16 = (2 * c.ncf + 15) / 16 * 16;
  kp8 = (2 * c.ncf + 7) / 8 * 8;
}

bool tf32_supported(const TransCfg& c)
{
  int rp16, kp8;
  tf32_dims(c, rp16, kp8);
  return rp16 / 16 <= X3_MT;
}

static size_t umma_plane_words(const TransCfg& c);
static bool umma_shape_ok(const TransCfg& c);
static void umma_dims(const TransCfg& c, int& rp16, int& nkc);

// the mma.sync planes [nmat][rp16][kp8] (hi, lo), then for the tcgen05 form the
// chunked core-matrix planes (hi, lo)
size_t tf32_matrix_bytes(const TransCfg& c)
{
  int rp16, kp8;
  tf32_dims(c, rp16, kp8);
  return (2 * c.nmatrices * (size_t)rp16 * kp8 + (umma_shape_ok(c) ? 2 * umma_plane_words(c) : 0)) *
         sizeof(uint32_t);
}

cudaError_t launch_trans_split_tf32(const TransCfg& c, const double* T, uint32_t* T32,
                                    cudaStream_t st)
{
  int rp16, kp8;
  tf32_dims(c, rp16, kp8);
  size_t n = c.nmatrices * (size_t)rp16 * kp8;
  int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_trans_split_tf32<<<blocks, 256, 0, st>>>((int)c.nmatrices, c.rp, c.kp, rp16, kp8, 2 * c.ncf, T,
                                             T32, T32 + n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !umma_shape_ok(c)) return e;
  int nkc;
  umma_dims(c, rp16, nkc);
  const size_t nu = umma_plane_words(c);
  blocks = (int)std::min<size_t>((nu + 255) / 256, 148 * 16);
  k_trans_umma_planes<<<blocks, 256, 0, st>>>((int)c.nmatrices, c.rp, c.kp, rp16, nkc, 2 * c.ncf, T,
                                              T32 + 2 * n, T32 + 2 * n + nu);
  return cudaGetLastError();
}

static cudaError_t x3_launch(const qbxfmm_geometry& g, const TransCfg& c, int nrhs, const uint32_t* T32,
                             size_t mat_base, int mat_mod, const int32_t* cls_code,
                             const int32_t* group_starts, int g0,
                             int ngroups, int maxcols, const int32_t* pair_src,
                             const int32_t* pair_dst, const double2* ein, double2* eout,
                             double scale, double* cpair, int32_t* err, cudaStream_t st)
{
  if (ngroups <= 0 || maxcols <= 0) return cudaSuccess;
  int rp16, kp8;
  tf32_dims(c, rp16, kp8);
  size_t n = c.nmatrices * (size_t)rp16 * kp8;
  size_t plane = (size_t)rp16 * kp8;
  size_t sh = (2 * (size_t)rp16 * X3_AS + 2 * (size_t)X3_KC * (X3_N + 4)) * sizeof(uint32_t);
  cudaFuncSetAttribute(k_trans_gemm_x3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  dim3 grid((maxcols + X3_N - 1) / X3_N, ngroups);
  k_trans_gemm_x3<<<grid, NT, sh, st>>>(c.ncf, c.rp, rp16, kp8, nrhs, T32 + mat_base * plane,
                                        T32 + n + mat_base * plane, mat_mod, cls_code,
                                        group_starts, g0,
                                        pair_src, pair_dst, ein, eout, scale, cpair, err, g.nboxes);
  return cudaGetLastError();
}

// the tcgen05 form for matrices of at most 256 rows (one MMA N), else the mma.sync one
static void umma_dims(const TransCfg& c, int& rp16, int& nkc)
{
  int kp8;
  tf32_dims(c, rp16, kp8);
  nkc = (kp8 + UM_KC - 1) / UM_KC;
}

static bool umma_shape_ok(const TransCfg& c)
{
  int rp16, nkc;
  umma_dims(c, rp16, nkc);
  return rp16 % 16 == 0 && rp16 >= 16 && rp16 <= UM_TCOLS;
}

static size_t umma_plane_words(const TransCfg& c)
{
  int rp16, nkc;
  umma_dims(c, rp16, nkc);
  return c.nmatrices * (size_t)nkc * rp16 * UM_KC;
}

static cudaError_t umma_launch(const qbxfmm_geometry& g, const TransCfg& c, int nrhs,
                               const uint32_t* U, const int32_t* cls_code, int ngroups, int maxcols,
                               const int32_t* group_starts, const int32_t* pair_src,
                               const double2* ein, double* cpair, int32_t* err, cudaStream_t st)
{
  if (ngroups <= 0 || maxcols <= 0) return cudaSuccess;
  int rp16, nkc;
  umma_dims(c, rp16, nkc);
  const size_t sh = 2 * (2 * (size_t)UM_M + 2 * (size_t)rp16) * UM_KC * sizeof(uint32_t);
  cudaError_t e = cudaFuncSetAttribute(k_trans_gemm_umma,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  if (e != cudaSuccess) return e;
  dim3 grid((maxcols + UM_M - 1) / UM_M, ngroups);
  k_trans_gemm_umma<<<grid, UM_NT, sh, st>>>(c.ncf, c.rp, rp16, nkc, nrhs, U,
                                             U + umma_plane_words(c), cls_code, group_starts,
                                             pair_src, ein,
                                             cpair, err, g.nboxes);
  return cudaGetLastError();
}

cudaError_t launch_m2l_gemm_mixed(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                                  int nrhs, const uint32_t* T32, const TransAux& aux,
                                  const double2* mp, double2* lo, double* cpair, int32_t* err,
                                  cudaStream_t st)
{
  if (g.m2l_nclasses == 0) return cudaSuccess;
  int rp16, kp8;
  tf32_dims(c, rp16, kp8);
  const uint32_t* U = T32 + 2 * c.nmatrices * (size_t)rp16 * kp8;   // after the mma.sync planes
  // (bulk copies need 16-byte aligned planes)
  const bool umma = umma_shape_ok(c) && (reinterpret_cast<uintptr_t>(U) & 15) == 0;
  cudaError_t e = umma
      ? umma_launch(g, c, nrhs, U, aux.cls_code, g.m2l_nclasses, th.m2l_max_pairs * nrhs,
                    g.m2l_class_starts, g.m2l_pair_src, mp, cpair, err, st)
      : x3_launch(g, c, nrhs, T32, 0, 0, aux.cls_code, g.m2l_class_starts, 0, g.m2l_nclasses,
                  th.m2l_max_pairs * nrhs, g.m2l_pair_src, nullptr, mp, nullptr, 1.0, cpair, err,
                  st);
  if (e != cudaSuccess) return e;
  return launch_trans_reduce_m2l(g, c, nrhs, cpair, lo, st);
}

cudaError_t launch_m2m_gemm_mixed(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                                  int nrhs, const uint32_t* T32, double2* mp, double* cpair,
                                  int32_t* err, cudaStream_t st)
{
  const int nch = 8;
  for (int lev = g.nlevels - 2; lev >= 0; --lev) {
    int maxp = th.m2m_level_max_group[lev];
    if (maxp == 0) continue;
    cudaError_t e = x3_launch(g, c, nrhs, T32, c.m2m_base, c.m2m_mat_mod, nullptr, g.m2m_group_starts,
                              lev * nch, nch, maxp * nrhs, g.m2m_pair_src, nullptr, mp, nullptr,
                              1.0, cpair, err, st);
    if (e != cudaSuccess) return e;
    e = launch_trans_reduce_m2m(g, th, c, lev, nrhs, cpair, mp, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_l2l_gemm_mixed(const qbxfmm_geometry& g, const TransHost& th, const TransCfg& c,
                                  int nrhs, const uint32_t* T32, double2* lo, int32_t* err,
                                  cudaStream_t st)
{
  const int nch = 8;
  for (int lev = 1; lev < g.nlevels; ++lev) {
    int maxp = th.l2l_level_max_group[lev];
    if (maxp == 0) continue;
    cudaError_t e = x3_launch(g, c, nrhs, T32, c.l2l_base, c.m2m_mat_mod, nullptr, g.l2l_group_starts,
                              lev * nch, nch, maxp * nrhs, g.l2l_pair_src, g.l2l_pair_dst, lo, lo,
                              1.0, nullptr, err, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// }}}

}  // namespace qbx
