// The reference's default (sumpy, compressed Taylor) truncation of the 3D Helmholtz
// expansions in the library's spherical-wave coefficients: host tables, the M2M / L2L
// matrices and the L2QBXL launcher (taylor_h3.cu).
#pragma once

#include <array>
#include <complex>
#include <vector>

#include "kernels.h"

namespace qbx {

constexpr int H3T_MAXP = 17;                              // largest FMM order
constexpr int H3T_MAXP2 = (H3T_MAXP + 1) * (H3T_MAXP + 1);

// Monomial tables of the order-p local basis f_nm(v) = j_n^[p](|v|) Y_n^m(v) (wave
// units v = k x; monomials x^a y^b z^c, a + b + c <= p, compact index
// h3t_mono_index): F [ncf][nmono]; the stored exponents st (c <= 1, in the order
// c, a, b); G0[s][nm] = F[nm][st_s] and Ginv = G0^-1 ([nm][s]).  p = -1 on failure.
struct H3TaylorHost {
  int p = -1, ncf = 0, nmono = 0;
  std::vector<std::complex<double>> F;
  std::vector<std::array<int, 3>> st;
  std::vector<std::complex<double>> G0;
  std::vector<std::complex<double>> Ginv;
};

int h3t_mono_index(int p, int a, int b, int c);
H3TaylorHost h3_taylor_host(int p);
void h3_taylor_translation(const H3TaylorHost& t, const double vd[3], std::complex<double>* C);
cudaError_t h3_taylor_translations(const H3TaylorHost& t, const TransCfg& tc, double k,
                                   double root_extent, int nlevels, double* T, cudaStream_t st);
cudaError_t h3_launch_l2qbxl_taylor(const qbxfmm_geometry& g, HelmCoeffs hc, int p, int q,
                                    int nrhs, const double2* lo, const double2* G0,
                                    const double2* Gq, double2* qe, int32_t* err, cudaStream_t st);

}  // namespace qbx
