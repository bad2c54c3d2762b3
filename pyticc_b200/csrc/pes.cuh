// Analytic interaction PES on the atom-diatom tensor grid, evaluated on the device.
//
// The reference evaluates a user PES on the host, on the tensor grid of
// src/pyticc/pes/adiabatic.py:109-137 (get_Vgrid_atom_diatom: R x r x theta, meshgrid
// "ij" order, so V[a][i][k] with k fastest).  For PES given in the Legendre-expansion form
//     V(R, r, theta) = sum_t P_lam_t(cos theta) * f_t(R) * g_t(r - re),
//     f_t(R) = sum of radial primitives, g_t(d) = sum_q c_tq d^q,
// the grid is filled here directly in device memory, one thread per grid point, so the
// PotentialGrid needs no host evaluation and no host-to-device copy.  Radial primitives:
//     kPesPower  a R^-b                       kPesExp    a exp(-b (R - c))
//     kPesGauss  a exp(-((R - c) / b)^2)      kPesLJ     a ((b/R)^12 - 2 (b/R)^6)
#pragma once

#include "ticc_common.cuh"

namespace ticc {

constexpr int kPesMaxTerms = 16, kPesMaxPrim = 4, kPesMaxPoly = 4, kPesMaxLam = 32;
enum PesKind : int { kPesPower = 0, kPesExp = 1, kPesGauss = 2, kPesLJ = 3 };

struct PesTable {
  int n_terms;
  int lmax;
  double re;
  int lam[kPesMaxTerms];
  int n_prim[kPesMaxTerms];
  int kind[kPesMaxTerms][kPesMaxPrim];
  double a[kPesMaxTerms][kPesMaxPrim], b[kPesMaxTerms][kPesMaxPrim], c[kPesMaxTerms][kPesMaxPrim];
  int n_poly[kPesMaxTerms];
  double poly[kPesMaxTerms][kPesMaxPoly];
};

__device__ __forceinline__ double pes_primitive(int kind, double a, double b, double c, double R) {
  switch (kind) {
    case kPesPower:
      return a * pow(R, -b);
    case kPesExp:
      return a * exp(-b * (R - c));
    case kPesGauss: {
      const double z = (R - c) / b;
      return a * exp(-(z * z));
    }
    default: {
      const double s = b / R, s2 = s * s, s6 = s2 * s2 * s2;
      return a * (s6 * s6 - 2.0 * s6);
    }
  }
}

// V[a][i][k] for R[a], r[i], x[k] = cos(theta_k); one thread per point.
__global__ void __launch_bounds__(256) pes_legendre_kernel(const __grid_constant__ PesTable tab, const double* __restrict__ R, int n_R, const double* __restrict__ r, int n_r,
                                                            const double* __restrict__ x, int n_x, double* __restrict__ V) {
  const long long total = (long long)n_R * n_r * n_x;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(e % n_x);
    const int i = (int)((e / n_x) % n_r);
    const int a = (int)(e / ((long long)n_x * n_r));
    const double RR = R[a], d = r[i] - tab.re, xx = x[k];
    // Legendre polynomials by the three-term recurrence (l + 1) P_{l+1} = (2l + 1) x P_l - l P_{l-1}
    double P[kPesMaxLam + 1];
    P[0] = 1.0;
    if (tab.lmax >= 1) P[1] = xx;
    for (int l = 1; l < tab.lmax; ++l) P[l + 1] = ((2 * l + 1) * xx * P[l] - l * P[l - 1]) / (l + 1);
    double v = 0.0;
    for (int t = 0; t < tab.n_terms; ++t) {
      double f = 0.0;
      for (int p = 0; p < tab.n_prim[t]; ++p) f += pes_primitive(tab.kind[t][p], tab.a[t][p], tab.b[t][p], tab.c[t][p], RR);
      double g = 0.0;
      for (int q = tab.n_poly[t] - 1; q >= 0; --q) g = g * d + tab.poly[t][q];
      v += P[tab.lam[t]] * f * g;
    }
    V[e] = v;
  }
}

}  // namespace ticc
