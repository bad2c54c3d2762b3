// Asymptotic matching of SF log-derivatives to S matrices, per energy, on the device.
//
// With J, N, J', N' the energy-normalised Riccati-Bessel functions of the open channels
// and Gamma the decaying-solution log-derivative of the closed channels:
//   Z = Y - diag(gamma),  gamma_i = Gamma_i (closed) or 0 (open)
//   G = (Z^{-1})_oo = Y_eff^{-1},   Y_eff = Y_oo - Y_oc (Y_cc - Gamma)^{-1} Y_co
// The reference forms K = -(Y_eff N - N')^{-1}(Y_eff J - J') and S = (I + iK)^{-1}(I - iK).
// Multiplying through by G, the same S is a single complex solve:
//   S = A^{-1} B,  A = diag(N - iJ) - G diag(N' - iJ'),  B = diag(N + iJ) - G diag(N' + iJ').
// Z is inverted by the symmetric sweep; A (general complex) by the general sweep of the
// transpose of its real 2x2 embedding; A^{-1} B is one DMMA GEMM.
#pragma once

#include "bessel.cuh"
#include "gemm.cuh"
#include "ldmd.cuh"
#include "sweep.cuh"

namespace ticc {

enum MatchDeviceStatus : int { kDeviceOpenOverflow = 5 };

struct MatchLayout {
  int n, n_energy, is_complex, max_open;
  int npz;  // padded size of Z (real or complex embedding)
  int npa;  // padded size of the 2 * max_open real embedding of A
  double* Jv;
  double* Nv;
  double* Jp;
  double* Np;
  double* gamma;  // [n_energy][n]
  int* oidx;      // [n_energy][n] open channel indices, ascending
  double* Z;      // [n_energy][npz][npz]
  double* A;      // [n_energy][npa][npa]
  double* B;      // [n_energy][npa][npa]
  double* C;      // [n_energy][npa][npa]
  double* scratch;
};

// Reference functions for every (energy, channel).
__global__ void match_refs_kernel(MatchLayout L, double Rmatch, const double* energies, double mu, const double* E_int, const double* Lam, int* status) {
  const long long total = (long long)L.n_energy * L.n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(idx / L.n), i = (int)(idx % L.n);
    const double diff = energies[e] - E_int[i];
    double J = 0.0, N = 0.0, Jd = 0.0, Nd = 0.0, g = 0.0;
    if (diff == 0.0) {
      report_status(status, kDeviceThreshold, e, i);
    } else {
      const double k = sqrt(2.0 * mu * fabs(diff));
      const double x = k * Rmatch;
      if (diff > 0.0) {
        const BesselJY r = riccati_bessel(Lam[i], x);
        if (!r.ok) report_status(status, kDeviceBesselFailed, e, i);
        const double sk = sqrt(k);
        J = r.J / sk;
        N = r.Y / sk;
        Jd = sk * r.Jp;
        Nd = sk * r.Yp;
      } else {
        const double kl = bessel_k_logd(Lam[i] + 0.5, x);
        if (!isfinite(kl)) report_status(status, kDeviceBesselFailed, e, i);
        g = 0.5 / Rmatch + k * kl;
      }
    }
    L.Jv[idx] = J;
    L.Nv[idx] = N;
    L.Jp[idx] = Jd;
    L.Np[idx] = Nd;
    L.gamma[idx] = g;
  }
}

// Open-channel list per energy (one CTA per energy; n is at most a few thousand).
__global__ void match_open_kernel(MatchLayout L, const double* energies, const double* E_int, int* n_open, int* status) {
  const int e = blockIdx.x;
  if (threadIdx.x != 0) return;
  int count = 0;
  for (int i = 0; i < L.n; ++i)
    if (E_int[i] < energies[e]) L.oidx[(long long)e * L.n + count++] = i;
  n_open[e] = count;
  if (count > L.max_open) report_status(status, kDeviceOpenOverflow, e, count);
}

// Z = Y - diag(gamma) into the padded sweep buffer.
__global__ void match_build_z_kernel(MatchLayout L, const double* Y) {
  const int e = blockIdx.y;
  const int n = L.n, np = L.npz;
  const int nl = L.is_complex ? np / 2 : np;
  double* Zb = L.Z + (long long)e * np * np;
  const double* gam = L.gamma + (long long)e * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)nl * nl; idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / nl), j = (int)(idx % nl);
    if (i >= n || j >= n) {
      if (L.is_complex) {
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) put_padding(Zb, np, 2LL * i + a, 2LL * j + b);
      } else {
        put_padding(Zb, np, i, j);
      }
      continue;
    }
    double x, z = 0.0;
    if (L.is_complex) {
      const double* Yb = Y + (long long)e * n * n * 2;
      x = 0.5 * (Yb[2 * ((long long)i * n + j)] + Yb[2 * ((long long)j * n + i)]);
      z = 0.5 * (Yb[2 * ((long long)i * n + j) + 1] + Yb[2 * ((long long)j * n + i) + 1]);
    } else {
      const double* Yb = Y + (long long)e * n * n;
      x = 0.5 * (Yb[(long long)i * n + j] + Yb[(long long)j * n + i]);
    }
    if (i == j) x -= gam[i];
    put_element(Zb, np, i, j, x, z, L.is_complex);
  }
}

// A^T (real embedding, transposed) into L.A with identity padding; B (real embedding) into L.B.
__global__ void match_build_ab_kernel(MatchLayout L, const int* n_open) {
  const int e = blockIdx.y;
  const int no = n_open[e] < L.max_open ? n_open[e] : L.max_open;
  const int np = L.npa, npz = L.npz, n = L.n;
  double* Ab = L.A + (long long)e * np * np;
  double* Bb = L.B + (long long)e * np * np;
  const double* Zb = L.Z + (long long)e * npz * npz;
  const int* oi = L.oidx + (long long)e * n;
  const double* Jv = L.Jv + (long long)e * n;
  const double* Nv = L.Nv + (long long)e * n;
  const double* Jp = L.Jp + (long long)e * n;
  const double* Np = L.Np + (long long)e * n;
  const int nl = np / 2;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)nl * nl; idx += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(idx / nl), b = (int)(idx % nl);
    double ar, ai, br, bi;
    if (a < no && b < no) {
      double sr, si;
      get_swept(Zb, npz, oi[a], oi[b], L.is_complex, sr, si);
      const double gr = -sr, gi = -si;  // G = (Z^-1)_oo
      const double dr = (a == b) ? 1.0 : 0.0;
      const double Na = Nv[oi[a]], Ja = Jv[oi[a]];
      const double Npb = Np[oi[b]], Jpb = Jp[oi[b]];
      // A = diag(N - iJ) - G (N' - iJ');  B = diag(N + iJ) - G (N' + iJ')
      ar = dr * Na - (gr * Npb + gi * Jpb);
      ai = -dr * Ja - (gi * Npb - gr * Jpb);
      br = dr * Na - (gr * Npb - gi * Jpb);
      bi = dr * Ja - (gi * Npb + gr * Jpb);
    } else {
      ar = (a == b) ? 1.0 : 0.0;
      ai = 0.0;
      br = 0.0;
      bi = 0.0;
    }
    // E(A)[2a+p][2b+q] = [[ar, -ai], [ai, ar]]; store its transpose at [2b+q][2a+p]
    Ab[(long long)(2 * b) * np + 2 * a] = ar;
    Ab[(long long)(2 * b + 1) * np + 2 * a] = -ai;
    Ab[(long long)(2 * b) * np + 2 * a + 1] = ai;
    Ab[(long long)(2 * b + 1) * np + 2 * a + 1] = ar;
    Bb[(long long)(2 * a) * np + 2 * b] = br;
    Bb[(long long)(2 * a) * np + 2 * b + 1] = -bi;
    Bb[(long long)(2 * a + 1) * np + 2 * b] = bi;
    Bb[(long long)(2 * a + 1) * np + 2 * b + 1] = br;
  }
}

// S_ab from C = -E(S): S = -(C[2a][2b] + i C[2a+1][2b]); zero outside the open block.
__global__ void match_extract_kernel(MatchLayout L, const int* n_open, double* S, int* status) {
  const int e = blockIdx.y;
  const int no = n_open[e] < L.max_open ? n_open[e] : L.max_open;
  const int n = L.n, np = L.npa;
  const double* Cb = L.C + (long long)e * np * np;
  double* Sb = S + (long long)e * n * n * 2;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)n * n; idx += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(idx / n), b = (int)(idx % n);
    double re = 0.0, im = 0.0;
    if (a < no && b < no) {
      re = -Cb[(long long)(2 * a) * np + 2 * b];
      im = -Cb[(long long)(2 * a + 1) * np + 2 * b];
      if (!isfinite(re) || !isfinite(im)) report_status(status, kDeviceNonFinite, e, a);
    }
    Sb[2 * idx] = re;
    Sb[2 * idx + 1] = im;
  }
}

inline cudaError_t match_smatrix(const double* Y, double Rmatch, const double* energies, double mu, const double* E_int, const double* Lam, double* S, int* n_open, MatchLayout& L, int* status, cudaStream_t stream) {
  const long long ne = (long long)L.n_energy * L.n;
  match_refs_kernel<<<grid_for(ne, 128), 128, 0, stream>>>(L, Rmatch, energies, mu, E_int, Lam, status);
  note_launch();
  match_open_kernel<<<L.n_energy, 32, 0, stream>>>(L, energies, E_int, n_open, status);
  note_launch();
  const long long nlz = L.is_complex ? L.npz / 2 : L.npz;
  match_build_z_kernel<<<dim3(grid_for(nlz * nlz, 256, 8192), L.n_energy), 256, 0, stream>>>(L, Y);
  note_launch();
  cudaError_t err = sweep_sym(L.Z, (long long)L.npz * L.npz, L.npz, L.n_energy, L.scratch, status, stream, nullptr, L.is_complex ? 2 * L.n : L.n);
  if (err != cudaSuccess) return err;
  const long long nla = L.npa / 2;
  match_build_ab_kernel<<<dim3(grid_for(nla * nla, 256, 8192), L.n_energy), 256, 0, stream>>>(L, n_open);
  note_launch();
  err = sweep_general(L.A, (long long)L.npa * L.npa, L.npa, L.n_energy, L.scratch, status, stream);
  if (err != cudaSuccess) return err;
  GemmBatch g{L.A, L.npa, (long long)L.npa * L.npa, L.B, L.npa, (long long)L.npa * L.npa, L.C, L.npa, (long long)L.npa * L.npa, L.npa, 1.0, 0};
  err = gemm_tn(g, L.npa, L.npa, L.n_energy, stream);
  if (err != cudaSuccess) return err;
  match_extract_kernel<<<dim3(grid_for((long long)L.n * L.n, 256, 8192), L.n_energy), 256, 0, stream>>>(L, n_open, S, status);
  note_launch();
  return cudaGetLastError();
}

}  // namespace ticc
