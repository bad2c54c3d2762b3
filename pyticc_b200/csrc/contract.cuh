// PotentialGrid -> V(R) contraction with the W_base assembly fused in.
//
// For one K group with weighted rows B (n_K x n_grid) and PES values v(R) on the
// quadrature grid, V_K(R)[a][b] = norm sum_q (Br[a][q] Br[b][q] + Bi[a][q] Bi[b][q]) v[q].
// One launch covers every group: each CTA computes a 64x64 lower-triangular tile of one group
// at one R on the FP64 tensor pipe and writes both (a, b) and (b, a), so V is exactly symmetric
// (the reference symmetrises explicitly).  The init kernel writes U/R^2 + 2 mu diag(E_int) (or
// zeros when only V is wanted) and the group kernel adds 2 mu V (or V) at the rows' output
// channel positions.
#pragma once

#include "dmma_tile.cuh"
#include "ticc_common.cuh"

namespace ticc {

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

// ---- the weighted-product tile on the FP64 tensor pipe ------------------------------------------
// A CTA of 8 warps computes one 64 x 64 tile X[i][j] = sum_q A[i][q] w[q] B[j][q] (plus the same
// over a second pair A2, B2: the imaginary rows of a complex basis) with mma.sync m8n8k4 f64
// (DMMA), FP64 accumulation.  The rows are read as stored (row-major, q contiguous, any n_grid
// and any row offset) in chunks of 32 grid points: each warp loads whole 256-byte row segments,
// the weight is applied to A on the way into shared memory, and rows past the operand's end read
// as zeros.  Shared tiles are [row][q] with a row stride of 36 doubles, so the fragment loads of a
// half-warp (rows mr = 0..3, k = 0..3) hit 16 distinct bank pairs.  Chunk c + 1 is fetched into
// registers while chunk c is multiplied from the other shared buffer (one barrier per chunk).
// Warp w owns rows (w / 4) * 32 .. +31 and columns (w % 4) * 16 .. +15 of the tile: 4 x 2 DMMA
// accumulators, element [mt][nt][h] at row (w/4)*32 + 8 mt + lane/4, column (w%4)*16 + 8 nt +
// 2 (lane%4) + h.
constexpr int kVTile = 64;
constexpr int kVChunk = 32;
constexpr int kVLd = kVChunk + 4;
constexpr int kVMaxGroups = 128;
constexpr size_t kVSmemBytes = size_t(2) * 2 * kVTile * kVLd * sizeof(double);  // 73728

struct VTileAcc {
  double v[4][2][2];
};

// A, B (and A2, B2) point at the tile's first row; rows at or beyond na (nb) read as zero.
__device__ inline void vtile_product(VTileAcc& acc, const double* __restrict__ A, int na, const double* __restrict__ B, int nb, const double* __restrict__ A2,
                                     const double* __restrict__ B2, int n_grid, const double* __restrict__ w, double* smem) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int qq = lane, rbase = warp;  // loader: grid point q0 + lane of rows warp + 8 i
  const int wm = (warp >> 2) * 32, wn = (warp & 3) * 16, kr = lane & 3, mr = lane >> 2;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) acc.v[mt][nt][0] = acc.v[mt][nt][1] = 0.0;
  const int nq = (n_grid + kVChunk - 1) / kVChunk;
  const int nc = A2 != nullptr ? 2 * nq : nq;
  double ra[8], rb[8];
  auto fetch = [&](int c) {
    const bool second = c >= nq;
    const double* sa = second ? A2 : A;
    const double* sb = second ? B2 : B;
    const int q = (second ? c - nq : c) * kVChunk + qq;
    const bool in = q < n_grid;
    const double wq = in ? w[q] : 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int row = rbase + 8 * i;
      ra[i] = (in && row < na) ? sa[(long long)row * n_grid + q] * wq : 0.0;
      rb[i] = (in && row < nb) ? sb[(long long)row * n_grid + q] : 0.0;
    }
  };
  auto put = [&](double* buf) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      buf[(rbase + 8 * i) * kVLd + qq] = ra[i];
      buf[kVTile * kVLd + (rbase + 8 * i) * kVLd + qq] = rb[i];
    }
  };
  fetch(0);
  put(smem);
  __syncthreads();
  for (int c = 0; c < nc; ++c) {
    if (c + 1 < nc) fetch(c + 1);
    const double* As = smem + (c & 1) * 2 * kVTile * kVLd;
    const double* Bs = As + kVTile * kVLd;
#pragma unroll
    for (int kk = 0; kk < kVChunk; kk += 4) {
      double a[4], b[2];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) a[mt] = As[(wm + mt * 8 + mr) * kVLd + kk + kr];
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) b[nt] = Bs[(wn + nt * 8 + mr) * kVLd + kk + kr];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) dmma_8x8x4(acc.v[mt][nt], a[mt], b[nt]);
    }
    if (c + 1 < nc) put(smem + ((c + 1) & 1) * 2 * kVTile * kVLd);
    __syncthreads();
  }
}

// Lower 64-tiles of every K group in one launch: tile t belongs to the group g with
// tile_start[g] <= t < tile_start[g + 1] (only groups with rows are listed).
struct ContractTiles {
  int n_groups;
  int tile_start[kVMaxGroups + 1];
  int row0[kVMaxGroups];
  int rows[kVMaxGroups];
};

// grid: (the table's tiles, radial points r_first ..); 256 threads; kVSmemBytes dynamic shared memory.
__global__ void __launch_bounds__(256) contract_group_kernel(const __grid_constant__ ContractTiles tiles, const double* __restrict__ Br, const double* __restrict__ Bi,
                                                             const int* __restrict__ row_out, int n_grid, double scale, const double* __restrict__ potential,
                                                             long long pot_stride, int r_first, int n, double* __restrict__ out) {
  extern __shared__ __align__(16) double vsmem[];
  const int t = blockIdx.x;
  int g = 0, hi = tiles.n_groups - 1;
  while (g < hi) {  // the last group whose first tile is at or before t
    const int mid = (g + hi + 1) >> 1;
    if (tiles.tile_start[mid] <= t) g = mid;
    else hi = mid - 1;
  }
  const int local = t - tiles.tile_start[g];
  int ta = (int)((sqrt(8.0 * local + 1.0) - 1.0) * 0.5);
  while ((ta + 1) * (ta + 2) / 2 <= local) ++ta;
  while (ta * (ta + 1) / 2 > local) --ta;
  const int tb = local - ta * (ta + 1) / 2;
  const int row0 = tiles.row0[g], rows = tiles.rows[g];
  const int r = r_first + blockIdx.y;
  const long long ia = (long long)(row0 + ta * kVTile) * n_grid, ib = (long long)(row0 + tb * kVTile) * n_grid;
  VTileAcc acc;
  vtile_product(acc, Br + ia, rows - ta * kVTile, Br + ib, rows - tb * kVTile, Bi != nullptr ? Bi + ia : nullptr, Bi != nullptr ? Bi + ib : nullptr, n_grid,
                potential + (long long)r * pot_stride, vsmem);
  double* o = out + (long long)r * n * n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp >> 2) * 32, wn = (warp & 3) * 16;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int a = ta * kVTile + wm + mt * 8 + (lane >> 2);
        const int b = tb * kVTile + wn + nt * 8 + 2 * (lane & 3) + h;
        if (a >= rows || b >= rows || b > a) continue;
        const int pa = row_out[row0 + a], pb = row_out[row0 + b];
        const double val = scale * acc.v[mt][nt][h];
        o[(long long)pa * n + pb] += val;
        if (a != b) o[(long long)pb * n + pa] += val;
      }
}

// One block of a state-resolved (diabatic) contraction at every R:
//     X(R)[i][j] = sum_q A[i][q] w(R)[q] B[j][q],   A: n_a x n_grid, B: n_b x n_grid (row strides n_grid)
// written to out(R)[pos_a[i]][pos_b[j]] and, with `mirror`, also to out(R)[pos_b[j]][pos_a[i]].
// A symmetric block (`symmetric`: B is A and pos_b is pos_a) computes only i >= j and writes
// both (i, j) and (j, i), so the block is exactly symmetric.  grid: (64-tiles of A, 64-tiles of B,
// radial points r_first ..); 256 threads; kVSmemBytes dynamic shared memory.
__global__ void __launch_bounds__(256) weighted_block_kernel(const double* __restrict__ A, int n_a, const double* __restrict__ B, int n_b, int n_grid, const double* __restrict__ w,
                                                             long long w_stride, int r_first, const int* __restrict__ pos_a, const int* __restrict__ pos_b, int symmetric,
                                                             int mirror, int n, double* __restrict__ out) {
  extern __shared__ __align__(16) double vsmem[];
  const int ti = blockIdx.x, tj = blockIdx.y, R = r_first + blockIdx.z;
  if (symmetric && tj > ti) return;
  const int i0 = ti * kVTile, j0 = tj * kVTile;
  VTileAcc acc;
  vtile_product(acc, A + (long long)i0 * n_grid, n_a - i0, B + (long long)j0 * n_grid, n_b - j0, nullptr, nullptr, n_grid, w + (long long)R * w_stride, vsmem);
  double* o = out + (long long)R * n * n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp >> 2) * 32, wn = (warp & 3) * 16;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = i0 + wm + mt * 8 + (lane >> 2), j = j0 + wn + nt * 8 + 2 * (lane & 3) + h;
        if (i >= n_a || j >= n_b || (symmetric && j > i)) continue;
        const int pa = pos_a[i], pb = pos_b[j];
        o[(long long)pa * n + pb] = acc.v[mt][nt][h];
        if (mirror || (symmetric && i != j)) o[(long long)pb * n + pa] = acc.v[mt][nt][h];
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
