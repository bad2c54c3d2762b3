// PotentialGrid -> V(R) contraction with the W_base assembly fused in.
//
// For one K group with weighted rows B (n_K x n_grid) and PES values v(R) on the
// quadrature grid, V_K(R)[a][b] = norm sum_q (Br[a][q] Br[b][q] + Bi[a][q] Bi[b][q]) v[q].
// Each CTA computes a 32x32 lower-triangular tile of one group at one R and writes both
// (a, b) and (b, a), so V is exactly symmetric (the reference symmetrises explicitly).
// The init kernel writes U/R^2 + 2 mu diag(E_int) (or zeros when only V is wanted) and
// the group kernels add 2 mu V (or V) at the rows' output channel positions.
#pragma once

#include "ticc_common.cuh"

namespace ticc {

constexpr int kCTile = 32;

__global__ void contract_init_kernel(double* out, int n, int n_R, const double* radial_points, const double* U, const double* E_int, double mu) {
  const long long total = (long long)n_R * n * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (U != nullptr) {
      const long long r = idx / ((long long)n * n);
      const long long ij = idx % ((long long)n * n);
      const int i = (int)(ij / n), j = (int)(ij % n);
      const double R = radial_points[r];
      v = U[ij] / (R * R);
      if (i == j) v += 2.0 * mu * E_int[i];
    }
    out[idx] = v;
  }
}

// grid: (lower tile pairs of the group, n_R); block 16 x 16 threads, 2 x 2 outputs each.
__global__ void __launch_bounds__(256) contract_group_kernel(const double* __restrict__ Br, const double* __restrict__ Bi, int row0, int n_rows, const int* __restrict__ row_out, int n_grid, double scale, const double* __restrict__ potential, long long pot_stride, int n, double* __restrict__ out) {
  __shared__ double As[kCTile][kCTile + 1];
  __shared__ double Bs[kCTile][kCTile + 1];
  __shared__ double Ai[kCTile][kCTile + 1];
  __shared__ double Bj[kCTile][kCTile + 1];
  __shared__ double vs[kCTile];
  int ta = (int)((sqrt(8.0 * blockIdx.x + 1.0) - 1.0) * 0.5);
  while ((ta + 1) * (ta + 2) / 2 <= (int)blockIdx.x) ++ta;
  while (ta * (ta + 1) / 2 > (int)blockIdx.x) --ta;
  const int tb = blockIdx.x - ta * (ta + 1) / 2;
  const int r = blockIdx.y;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const double* v = potential + (long long)r * pot_stride;
  const bool imag = (Bi != nullptr);
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (int q0 = 0; q0 < n_grid; q0 += kCTile) {
    for (int idx = threadIdx.x; idx < kCTile * kCTile; idx += 256) {
      const int rr = idx / kCTile, qq = idx % kCTile;
      const int q = q0 + qq;
      const int ra = ta * kCTile + rr, rb = tb * kCTile + rr;
      const bool qin = q < n_grid;
      As[qq][rr] = (qin && ra < n_rows) ? Br[(long long)(row0 + ra) * n_grid + q] : 0.0;
      Bs[qq][rr] = (qin && rb < n_rows) ? Br[(long long)(row0 + rb) * n_grid + q] : 0.0;
      if (imag) {
        Ai[qq][rr] = (qin && ra < n_rows) ? Bi[(long long)(row0 + ra) * n_grid + q] : 0.0;
        Bj[qq][rr] = (qin && rb < n_rows) ? Bi[(long long)(row0 + rb) * n_grid + q] : 0.0;
      }
    }
    if (threadIdx.x < kCTile) vs[threadIdx.x] = (q0 + threadIdx.x < n_grid) ? v[q0 + threadIdx.x] : 0.0;
    __syncthreads();
#pragma unroll 8
    for (int qq = 0; qq < kCTile; ++qq) {
      const double w = vs[qq];
      const double a0 = As[qq][ty] * w, a1 = As[qq][ty + 16] * w;
      const double b0 = Bs[qq][tx], b1 = Bs[qq][tx + 16];
      acc[0][0] += a0 * b0;
      acc[0][1] += a0 * b1;
      acc[1][0] += a1 * b0;
      acc[1][1] += a1 * b1;
      if (imag) {
        const double c0 = Ai[qq][ty] * w, c1 = Ai[qq][ty + 16] * w;
        const double d0 = Bj[qq][tx], d1 = Bj[qq][tx + 16];
        acc[0][0] += c0 * d0;
        acc[0][1] += c0 * d1;
        acc[1][0] += c1 * d0;
        acc[1][1] += c1 * d1;
      }
    }
    __syncthreads();
  }
  double* o = out + (long long)r * n * n;
  for (int u = 0; u < 2; ++u)
    for (int w = 0; w < 2; ++w) {
      const int a = ta * kCTile + ty + 16 * u;
      const int b = tb * kCTile + tx + 16 * w;
      if (a >= n_rows || b >= n_rows || b > a) continue;
      const int pa = row_out[row0 + a], pb = row_out[row0 + b];
      const double val = scale * acc[u][w];
      o[(long long)pa * n + pb] += val;
      if (a != b) o[(long long)pb * n + pa] += val;
    }
}

// One block of a state-resolved (diabatic) contraction at every R:
//     X(R)[i][j] = sum_q A[i][q] w(R)[q] B[j][q],   A: n_a x n_grid, B: n_b x n_grid (row strides n_grid)
// written to out(R)[pos_a[i]][pos_b[j]] and, with `mirror`, also to out(R)[pos_b[j]][pos_a[i]].
// A symmetric block (`symmetric`: B is A and pos_b is pos_a) computes only i >= j and writes
// both (i, j) and (j, i), so the block is exactly symmetric.  grid: (tiles of A, tiles of B,
// n_R); block 16 x 16 threads, 2 x 2 outputs each.
__global__ void __launch_bounds__(256) weighted_block_kernel(const double* __restrict__ A, int n_a, const double* __restrict__ B, int n_b, int n_grid, const double* __restrict__ w,
                                                             long long w_stride, const int* __restrict__ pos_a, const int* __restrict__ pos_b, int symmetric, int mirror, int n,
                                                             double* __restrict__ out) {
  const int ti = blockIdx.x, tj = blockIdx.y, R = blockIdx.z;
  if (symmetric && tj > ti) return;
  __shared__ double As[kCTile][kCTile + 1];
  __shared__ double Bs[kCTile][kCTile + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int i0 = ti * kCTile, j0 = tj * kCTile;
  const double* wr = w + (long long)R * w_stride;
  double acc[2][2] = {};
  for (int q0 = 0; q0 < n_grid; q0 += kCTile) {
    for (int e = threadIdx.x; e < kCTile * kCTile; e += 256) {
      const int rr = e / kCTile, qq = e % kCTile, q = q0 + qq;
      const bool inq = q < n_grid;
      As[rr][qq] = (inq && i0 + rr < n_a) ? A[(long long)(i0 + rr) * n_grid + q] * wr[q] : 0.0;
      Bs[rr][qq] = (inq && j0 + rr < n_b) ? B[(long long)(j0 + rr) * n_grid + q] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int qq = 0; qq < kCTile; ++qq) {
      const double a0 = As[ty][qq], a1 = As[ty + 16][qq];
      const double b0 = Bs[tx][qq], b1 = Bs[tx + 16][qq];
      acc[0][0] = fma(a0, b0, acc[0][0]);
      acc[0][1] = fma(a0, b1, acc[0][1]);
      acc[1][0] = fma(a1, b0, acc[1][0]);
      acc[1][1] = fma(a1, b1, acc[1][1]);
    }
    __syncthreads();
  }
  double* o = out + (long long)R * n * n;
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      const int i = i0 + ty + 16 * u, j = j0 + tx + 16 * v;
      if (i >= n_a || j >= n_b || (symmetric && j > i)) continue;
      const int pa = pos_a[i], pb = pos_b[j];
      o[(long long)pa * n + pb] = acc[u][v];
      if (mirror || (symmetric && i != j)) o[(long long)pb * n + pa] = acc[u][v];
    }
}


// Packed lower-triangle channel pairs of a fine-structure contraction into matrices: for every R
// and pair p = (i, j) = (pair_rows[p], pair_cols[p]), i >= j, with value v = src(R, p):
//   real (scalar FS):   out[i][j] = out[j][i] = v;
//   complex (spin FS):  v is conjugated where reversed[p]; out[i][j] = v, out[j][i] = conj(v),
//                       a diagonal element keeps the real part.
// src: n_R rows of src_stride elements (doubles, or interleaved complex doubles); out: n_R x n x n.
__global__ void __launch_bounds__(256) pairs_to_matrix_kernel(const double* __restrict__ src, int is_complex, long long src_stride, int n_pairs, const int* __restrict__ pair_rows,
                                                              const int* __restrict__ pair_cols, const unsigned char* __restrict__ reversed, int n, int n_R,
                                                              double* __restrict__ out) {
  const long long total = (long long)n_R * n_pairs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int R = (int)(e / n_pairs), p = (int)(e % n_pairs);
    const int i = pair_rows[p], j = pair_cols[p];
    if (is_complex) {
      const double re = src[(long long)R * src_stride + 2 * p];
      double im = src[(long long)R * src_stride + 2 * p + 1];
      if (reversed != nullptr && reversed[p]) im = -im;
      double* o = out + 2 * (long long)R * n * n;
      if (i == j) {
        o[2 * ((long long)i * n + i)] = re;
        o[2 * ((long long)i * n + i) + 1] = 0.0;
      } else {
        o[2 * ((long long)i * n + j)] = re;
        o[2 * ((long long)i * n + j) + 1] = im;
        o[2 * ((long long)j * n + i)] = re;
        o[2 * ((long long)j * n + i) + 1] = -im;
      }
    } else {
      const double v = src[(long long)R * src_stride + p];
      double* o = out + (long long)R * n * n;
      o[(long long)i * n + j] = v;
      o[(long long)j * n + i] = v;
    }
  }
}

}  // namespace ticc
