// Batched blocked symmetric sweep: M <- -M^{-1} for a batch of padded symmetric
// matrices, in place.
//
// The sweep (principal pivot transform) over an index block K with P = M_KK:
//     M_KK <- -P^{-1},   M_KR <- P^{-1} M_KR,   M_RK <- M_RK P^{-1},
//     M_RR <- M_RR - M_RK P^{-1} M_KR,
// keeps M symmetric, and sweeping every block in turn yields -M^{-1}.  The symmetric sweep
// keeps only the lower and diagonal 128-tiles current (an upper tile is read as the
// transpose of its lower partner; get_swept does this for every reader).  Per block:
//   1. pivot: the 128x128 block P is inverted in shared memory by Gauss-Jordan exchange
//      with partial pivoting (local to the block); -P^{-1} goes into M_KK and P^{-1} into
//      a scratch slot;
//   2. row panel: per 128-column tile the old rows K (read from the lower partner for
//      tiles right of K) are kept in `cold` and U = P^{-1} cold is computed on the FP64
//      tensor pipe; U goes into the rows K (for tiles right of K that storage is otherwise
//      unused and serves as this step's update operand) and U^T into the lower tiles of the
//      columns K;
//   3. update: lower-triangular tiles M_RR -= cold^T U, so the update costs N^2 * 128 flops
//      instead of 2 N^2 * 128, and no tile is written twice.
// The symmetric sweep runs steps 2-3 and the next step's pivot as one persistent launch
// per step (sweep_step_kernel); the general sweep (matching) keeps separate row-panel,
// column-panel and update kernels over the full matrix.
// Total work for an N x N inverse: N^3 flops (vs 2 N^3 for a general inverse).
#pragma once

#include "dmma_tile.cuh"
#include "tc_update.cuh"
#include "ticc_common.cuh"

namespace ticc {

constexpr int kPivotLd = kStride;  // the pivot block lives in a [128][kStride] shared tile
constexpr int kSub = 64;           // Gauss-Jordan sub-block of the pivot block
constexpr size_t kGJAuxDoubles = 2 * kSub + 4;  // Gauss-Jordan bookkeeping: pivot row, pivot column, candidates
constexpr size_t kPivotAuxBytes = size_t(2) * kSub * kSub * sizeof(double) + kGJAuxDoubles * sizeof(double) + (4 + kSub) * sizeof(int);
constexpr size_t kPivotSmemBytes = size_t(kBlock) * kPivotLd * sizeof(double) + kPivotAuxBytes;
constexpr size_t kUpdateSmemBytes = kUpdTileSmemBytes + 16;  // + the broadcast slot of the tile queue  // stages + C tile; the pivot aux reuses the stages
static_assert(kPivotAuxBytes <= size_t(kUpdStageDoubles) * sizeof(double), "pivot scratch must fit in the update stages");

// Gauss-Jordan exchange of a 64x64 sub-block S (row stride Ld) with partial
// pivoting over its rows, by the kPivotThreads threads of the CTA; writes the inverse in
// natural order to X (row stride kSub).  Thread t holds row t % 64, columns 16 (t / 64) ..
// + 15 of the block in registers for the whole exchange: a step publishes only the pivot
// row (its 4 owners) and the pivot column (one value per row) through shared memory, and the
// next pivot is found as the maximum over the 32 rows of each of the 2 warps that
// hold the next column (warp reductions on a rank key).  Pivot choice: largest magnitude among
// the rows not yet used, the smallest row on ties, a NaN ranking as zero.  Two barriers per step.  Returns true if a
// pivot was zero or non-finite.
template <int Ld = kPivotLd>
__device__ inline bool gauss_jordan_sub(double* S, double* X, double* aux) {
  static_assert(kPivotThreads == 4 * kSub, "one thread per (row, 16-column group)");
  double* prow = aux;
  double* pcol = aux + kSub;
  double* cand_val = aux + 2 * kSub;
  int* cand_row = reinterpret_cast<int*>(cand_val + 4);
  int* perm = cand_row + 4;
  const int t = threadIdx.x, r = t & (kSub - 1), cg = t / kSub, lane = t & 31, half = r >> 5;
  double v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = S[r * Ld + 16 * cg + i];
  bool row_used = false, singular = false;
  // this warp's best row for the next pivot to slot `half`.  Rank: 0 for a used row, else 1 +
  // the bit pattern of the magnitude (a NaN as zero), which orders like the magnitude; the
  // largest rank wins, the smallest row on ties: three warp reductions instead of shuffles.
  unsigned long long* cand_key = reinterpret_cast<unsigned long long*>(cand_val);
  auto candidate = [&](double m, bool excluded) {
    const unsigned long long key = excluded ? 0ull : 1ull + (unsigned long long)__double_as_longlong(m >= 0.0 ? m : 0.0);
    const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
    const unsigned hmax = __reduce_max_sync(0xffffffffu, hi);
    const unsigned lmax = __reduce_max_sync(0xffffffffu, hi == hmax ? lo : 0u);
    const unsigned rmin = __reduce_min_sync(0xffffffffu, (hi == hmax && lo == lmax) ? (unsigned)r : 0xffffffffu);
    if (lane == 0) {
      cand_key[half] = ((unsigned long long)hmax << 32) | lmax;
      cand_row[half] = (int)rmin;
    }
  };
  if (cg == 0) candidate(fabs(v[0]), false);
  __syncthreads();
#pragma unroll 1
  for (int blk = 0; blk < kSub / 16; ++blk) {
#pragma unroll
    for (int jj = 0; jj < 16; ++jj) {
      const int j = 16 * blk + jj;
      const unsigned long long k0 = cand_key[0], k1 = cand_key[1];
      int p = cand_row[0];
      const int p1 = cand_row[1];
      if (k1 > k0 || (k1 == k0 && p1 < p)) p = p1;
      const bool mine = r == p;
      if (mine) {
#pragma unroll
        for (int i = 0; i < 16; ++i) prow[16 * cg + i] = v[i];
        row_used = true;
      }
      if (cg == blk) pcol[r] = v[jj];
      if (t == 0) perm[j] = p;
      __syncthreads();
      double a = prow[j];
      if (!(fabs(a) > 0.0) || !isfinite(a)) {
        singular = true;
        a = 1.0;
      }
      const double inv_a = 1.0 / a;
      const double pc = pcol[r];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int c = 16 * cg + i;
        const double pr = prow[c] * inv_a;
        const double w = (c == j) ? pc * inv_a : v[i] - pc * pr;
        v[i] = mine ? ((c == j) ? inv_a : -pr) : w;
      }
      if (j + 1 < kSub && cg == (j + 1) / 16) candidate(fabs(v[(jj + 1) & 15]), row_used);
      __syncthreads();
    }
  }
#pragma unroll
  for (int i = 0; i < 16; ++i) S[r * Ld + 16 * cg + i] = v[i];
  __syncthreads();
  // inverse element (j, perm[c]) sits at exchange slot (perm[j], c)
  int* iperm = reinterpret_cast<int*>(prow);
  if (t < kSub) iperm[perm[t]] = t;
  __syncthreads();
  for (int e = t; e < kSub * kSub; e += kPivotThreads) {
    const int jj = e / kSub, m = e % kSub;
    X[e] = S[perm[jj] * Ld + iperm[m]];
  }
  __syncthreads();
  return singular;
}

// C (64x64, row stride ldc) = sign * A (64x64, lda) * B (64x64, ldb) [+ C if accumulate];
// 256 threads, 4x4 outputs each.  No aliasing between C and A/B.
__device__ inline void small_gemm64(double* C, int ldc, const double* A, int lda, const double* B, int ldb, double sign, bool accumulate) {
  const int t = threadIdx.x;
  const int i0 = (t >> 4) * 4, m0 = (t & 15) * 4;
  double acc[4][4] = {};
  for (int k = 0; k < kSub; ++k) {
    double a[4], b[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) a[u] = A[(i0 + u) * lda + k];
#pragma unroll
    for (int u = 0; u < 4; ++u) b[u] = B[k * ldb + m0 + u];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int w = 0; w < 4; ++w) acc[u][w] = fma(a[u], b[w], acc[u][w]);
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      double* d = C + (i0 + u) * ldc + m0 + w;
      *d = accumulate ? *d + sign * acc[u][w] : sign * acc[u][w];
    }
  __syncthreads();
}

// Sweep the 128x128 block held in shared memory (row stride kPivotLd) in place:
// P <- -P^{-1}, through its two 64-wide sub-blocks (the same principal pivot transform
// as the outer sweep, one level down).  aux holds two 64x64 temporaries and the
// Gauss-Jordan bookkeeping.
template <bool kSym>
__device__ inline bool sweep_block(double* P, double* aux) {
  double* X = aux;
  double* U = aux + kSub * kSub;
  double* gj = aux + 2 * kSub * kSub;
  bool singular = false;
  for (int s = 0; s < 2; ++s) {
    const int k0 = kSub * s, r0 = kSub * (1 - s);
    double* Pkk = P + k0 * kPivotLd + k0;
    double* Pkr = P + k0 * kPivotLd + r0;
    double* Prk = P + r0 * kPivotLd + k0;
    double* Prr = P + r0 * kPivotLd + r0;
    singular |= gauss_jordan_sub(Pkk, X, gj);
    small_gemm64(U, kSub, X, kSub, Pkr, kPivotLd, 1.0, false);     // U = P_KK^-1 P_KR
    small_gemm64(Prr, kPivotLd, Prk, kPivotLd, U, kSub, -1.0, true);  // P_RR -= P_RK U
    if (kSym) {
      for (int e = threadIdx.x; e < kSub * kSub; e += kPivotThreads) {
        const int i = e / kSub, m = e % kSub;
        Pkr[i * kPivotLd + m] = U[e];
        Prk[m * kPivotLd + i] = U[e];
      }
      __syncthreads();
    } else {
      for (int e = threadIdx.x; e < kSub * kSub; e += kPivotThreads) Pkr[(e / kSub) * kPivotLd + e % kSub] = U[e];
      __syncthreads();
      small_gemm64(U, kSub, Prk, kPivotLd, X, kSub, 1.0, false);     // V = P_RK P_KK^-1
      for (int e = threadIdx.x; e < kSub * kSub; e += kPivotThreads) Prk[(e / kSub) * kPivotLd + e % kSub] = U[e];
      __syncthreads();
    }
    for (int e = threadIdx.x; e < kSub * kSub; e += kPivotThreads) Pkk[(e / kSub) * kPivotLd + e % kSub] = -X[e];
    __syncthreads();
  }
  return singular;
}

// Invert the pivot block of matrix b whose rows/cols start at k0; P is a [128][kStride]
// shared tile already holding the block.  Writes -P^-1 into M_KK and P^-1 (general
// sweep: also its transpose) into the scratch panel; the symmetric sweep symmetrises.
template <bool kSym>
__device__ inline void invert_pivot_block(double* P, double* aux, double* Mb, int ld, int k0, double* pinv, int b, int* status) {
  const bool singular = sweep_block<kSym>(P, aux);
  if (singular && threadIdx.x == 0) report_status(status, kDeviceSingularPivot, b, k0 / kBlock);
  double* Pb = pinv + (long long)b * 2 * kBlock * kBlock;
  for (int idx = threadIdx.x; idx < kBlock * kBlock; idx += blockDim.x) {
    const int j = idx >> 7, m = idx & (kBlock - 1);
    double x = -P[j * kPivotLd + m];
    if (kSym) {
      x = 0.5 * (x - P[m * kPivotLd + j]);
      Pb[idx] = x;
    } else {
      Pb[idx] = x;
      Pb[kBlock * kBlock + m * kBlock + j] = x;
    }
    Mb[(long long)(k0 + j) * ld + k0 + m] = -x;
  }
}

// With `split` (a sweep whose first step runs on tcgen05: 0 < *reduced_blocks), P^-1 also goes
// out as that step's pivot panel (slot 0) for the row-panel products.
template <bool kSym>
__global__ void __launch_bounds__(kPivotThreads) sweep_pivot_kernel(double* __restrict__ M, long long mstride, int ld, int k0, double* __restrict__ pinv, int* status, float* split = nullptr,
                                                                    const int* reduced_blocks = nullptr, int batch = 0) {
  extern __shared__ double smem[];
  double* P = smem;
  double* aux = smem + kBlock * kPivotLd;
  const int b = blockIdx.x;
  double* Mb = M + (long long)b * mstride;
  // 128 x 128 block as double2 pieces, 8 loads in flight per thread
#pragma unroll 1
  for (int base = 0; base < kBlock * 64; base += 8 * kPivotThreads) {
    double2 m[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int piece = base + u * kPivotThreads + threadIdx.x;
      m[u] = *reinterpret_cast<const double2*>(Mb + (long long)(k0 + (piece >> 6)) * ld + k0 + (piece & 63) * 2);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int piece = base + u * kPivotThreads + threadIdx.x;
      double* d = P + (piece >> 6) * kPivotLd + (piece & 63) * 2;
      d[0] = m[u].x;
      d[1] = m[u].y;
    }
  }
  __syncthreads();
  invert_pivot_block<kSym>(P, aux, Mb, ld, k0, pinv, b, status);
  if (split != nullptr && reduced_blocks != nullptr && 0 < *reduced_blocks) {
    __syncthreads();
    tc_write_panel_at(split + (long long)tc_pinv_block(b, 0, ld / kBlock, batch) * kTcArrayFloats, pinv + (long long)b * 2 * kBlock * kBlock, kBlock, 0);
  }
}

// Sweep of a single-block matrix whose channels fill at most the leading 64 rows and
// columns (the rest is identity padding): only the 64x64 block is inverted, in a CTA with
// 69 KB of shared memory so that three matrices share an SM; the padding becomes -I.
constexpr int kSmallLd = kSub + 4;
constexpr size_t kPivot64SmemBytes = (size_t(kSub) * kSmallLd + size_t(kSub) * kSub + kGJAuxDoubles) * sizeof(double) + (4 + kSub) * sizeof(int);
template <bool kSym>
__global__ void __launch_bounds__(kPivotThreads) sweep_pivot64_kernel(double* __restrict__ M, long long mstride, int ld, int* status) {
  extern __shared__ double smem[];
  double* S = smem;
  double* X = S + kSub * kSmallLd;
  double* gj = X + kSub * kSub;
  const int b = blockIdx.x;
  double* Mb = M + (long long)b * mstride;
#pragma unroll
  for (int u = 0; u < kSub * kSub / 2 / kPivotThreads; ++u) {
    const int piece = u * kPivotThreads + threadIdx.x;
    const double2 m = *reinterpret_cast<const double2*>(Mb + (long long)(piece >> 5) * ld + (piece & 31) * 2);
    double* d = S + (piece >> 5) * kSmallLd + (piece & 31) * 2;
    d[0] = m.x;
    d[1] = m.y;
  }
  __syncthreads();
  const bool singular = gauss_jordan_sub<kSmallLd>(S, X, gj);
  if (singular && threadIdx.x == 0) report_status(status, kDeviceSingularPivot, b, 0);
  for (int idx = threadIdx.x; idx < ld * ld; idx += kPivotThreads) {
    const int i = idx / ld, j = idx % ld;
    double x;
    if (i < kSub && j < kSub) {
      x = X[i * kSub + j];
      if (kSym) x = 0.5 * (x + X[j * kSub + i]);
      x = -x;
    } else {
      x = (i == j) ? -1.0 : 0.0;
    }
    Mb[(long long)i * ld + j] = x;
  }
}

// Cs[r][c] += M[r0 + r][c0 + c] for a 128x128 tile; 8 global loads in flight per batch.
__device__ inline void add_tile_from_global(double* Cs, const double* Mb, int ld, int r0, int c0) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int base = 0; base < kBlock * 64; base += 8 * kGemmThreads) {
    double2 m[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int piece = base + u * kGemmThreads + tid;
      m[u] = *reinterpret_cast<const double2*>(Mb + (long long)(r0 + (piece >> 6)) * ld + c0 + (piece & 63) * 2);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int piece = base + u * kGemmThreads + tid;
      double* d = Cs + (piece >> 6) * kStride + (piece & 63) * 2;
      d[0] += m[u].x;
      d[1] += m[u].y;
    }
  }
}

// dst[dr0 + r][dc0 + c] = src[sr0 + r][sc0 + c] for a 128x128 tile (global to global).
__device__ inline void copy_tile(double* dst, int ldd, int dr0, int dc0, const double* src, int lds, int sr0, int sc0) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int base = 0; base < kBlock * 64; base += 8 * kGemmThreads) {
    double2 m[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int piece = base + u * kGemmThreads + tid;
      m[u] = __ldcg(reinterpret_cast<const double2*>(src + (long long)(sr0 + (piece >> 6)) * lds + sc0 + (piece & 63) * 2));
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int piece = base + u * kGemmThreads + tid;
      *reinterpret_cast<double2*>(dst + (long long)(dr0 + (piece >> 6)) * ldd + dc0 + (piece & 63) * 2) = m[u];
    }
  }
}

// dst[k][dc0 + c] = src[sr0 + c][sc0 + k] for a 128x128 tile, through a shared tile of row
// stride 129 (conflict-free column reads; one double per thread and step, so the global
// writes of a warp are 256 contiguous bytes).  Ends with a __syncthreads().
constexpr int kTransLd = kBlock + 1;
__device__ inline void copy_tile_transposed(double* dst, int ldd, int dc0, const double* src, int lds, int sr0, int sc0, double* smem) {
  const int tid = threadIdx.x;
#pragma unroll 1
  for (int base = 0; base < kBlock * 64; base += 8 * kGemmThreads) {
    double2 m[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int piece = base + u * kGemmThreads + tid;
      m[u] = __ldcg(reinterpret_cast<const double2*>(src + (long long)(sr0 + (piece >> 6)) * lds + sc0 + (piece & 63) * 2));
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int piece = base + u * kGemmThreads + tid;
      double* d = smem + (piece >> 6) * kTransLd + (piece & 63) * 2;
      d[0] = m[u].x;
      d[1] = m[u].y;
    }
  }
  __syncthreads();
#pragma unroll 4
  for (int e = tid; e < kBlock * kBlock; e += kGemmThreads) {
    const int k = e >> 7, c = e & (kBlock - 1);
    dst[(long long)k * ldd + dc0 + c] = smem[c * kTransLd + k];
  }
  __syncthreads();
}

// The old rows K over column tile jt (M_KR, the tile that U = P^-1 M_KR needs) into cold.
// Only the lower and diagonal 128-tiles of a symmetric work matrix are current, so for
// jt > kb the tile is read as the transpose of (jt, kb).  Ends with a __syncthreads().
__device__ inline void load_cold_tile(double* Cb, int ld, const double* Mb, int kb, int jt, double* smem) {
  const int k0 = kb * kBlock, c0 = jt * kBlock;
  if (jt < kb) {
    copy_tile(Cb, ld, 0, c0, Mb, ld, k0, c0);
    __syncthreads();
  } else {
    copy_tile_transposed(Cb, ld, c0, Mb, ld, c0, k0, smem);
  }
}

// Write a finished 128x128 tile from shared memory to M at (r0, c0).
__device__ inline void store_tile(double* Mb, int ld, int r0, int c0, const double* Cs) {
  const int tid = threadIdx.x;
  for (int piece = tid; piece < kBlock * 64; piece += kGemmThreads) {
    const int r = piece >> 6;
    const int c = (piece & 63) * 2;
    double2 v;
    v.x = Cs[r * kStride + c];
    v.y = Cs[r * kStride + c + 1];
    *reinterpret_cast<double2*>(Mb + (long long)(r0 + r) * ld + c0 + c) = v;
  }
}

// Row panel: U = P^-1 M_KR for one 128-column tile of the rows K.  The symmetric
// sweep also keeps the old rows (= old columns K, transposed) in `cold` and mirrors U^T
// into the columns K; the general sweep leaves the columns to the column-panel kernel.
template <bool kSym>
__global__ void __launch_bounds__(kGemmThreads) sweep_rowpanel_kernel(double* __restrict__ M, long long mstride, int ld, int kb, const double* __restrict__ pinv, double* __restrict__ cold, long long cstride, int* queue) {
  extern __shared__ double smem[];
  const int b = blockIdx.y;
  const int jt = blockIdx.x + (blockIdx.x >= kb ? 1 : 0);
  const int k0 = kb * kBlock, c0 = jt * kBlock;
  double* Mb = M + (long long)b * mstride;
  double* Cb = cold + (long long)b * cstride;
  const int tid = threadIdx.x;
  if (kSym) load_cold_tile(Cb, ld, Mb, kb, jt, smem);
  const double* Pt = pinv + (long long)b * 2 * kBlock * kBlock + (kSym ? 0 : kBlock * kBlock);
  TileAcc acc;
  // the symmetric sweep reads M_KR from cold (current for every jt), the general one from M
  tile_gemm_tn(acc, Pt, kBlock, kSym ? Cb + c0 : Mb + (long long)k0 * ld + c0, ld, kBlock, smem);
  // U^T into the columns K from registers where (jt, kb) is a lower tile, U rows (for jt > kb
  // the otherwise unused upper tile, read by this step's update) from shared memory
  acc_to_smem_mirror(acc, smem, Mb + (long long)c0 * ld + k0, ld, kSym && jt > kb);
  __syncthreads();
  store_tile(Mb, ld, k0, c0, smem);
  if (blockIdx.x == 0 && blockIdx.y == 0 && tid == 0) *queue = 0;  // the step's update tile queue
}

// Column panel of the general sweep: M_RK <- M_RK P^-1 for one 128-row tile, keeping
// the old columns transposed in `cold` (cold[k][i] = M[i][k0 + k]).
__global__ void __launch_bounds__(kGemmThreads) sweep_colpanel_kernel(double* __restrict__ M, long long mstride, int ld, int kb, const double* __restrict__ pinv, double* __restrict__ cold, long long cstride) {
  extern __shared__ double smem[];
  const int b = blockIdx.y;
  const int it = blockIdx.x + (blockIdx.x >= kb ? 1 : 0);
  const int k0 = kb * kBlock, r0 = it * kBlock;
  double* Mb = M + (long long)b * mstride;
  double* Cb = cold + (long long)b * cstride;
  const int tid = threadIdx.x;
  for (int e = tid; e < kBlock * kBlock; e += kGemmThreads) smem[(e >> 7) * kStride + (e & (kBlock - 1))] = 0.0;
  __syncthreads();
  add_tile_from_global(smem, Mb, ld, r0, k0);
  __syncthreads();
  for (int piece = tid; piece < kBlock * 64; piece += kGemmThreads) {
    const int k = piece >> 6, i = (piece & 63) * 2;
    double2 v;
    v.x = smem[i * kStride + k];
    v.y = smem[(i + 1) * kStride + k];
    *reinterpret_cast<double2*>(Cb + (long long)k * ld + r0 + i) = v;
  }
  __syncthreads();
  TileAcc acc;
  tile_gemm_tn(acc, Cb + r0, ld, pinv + (long long)b * 2 * kBlock * kBlock, kBlock, kBlock, smem);
  acc_to_smem(acc, smem, 1.0);
  __syncthreads();
  store_tile(Mb, ld, r0, k0, smem);
}

__device__ __forceinline__ void lower_pair(int idx, int& a, int& b) {
  int r = static_cast<int>((sqrt(8.0 * idx + 1.0) - 1.0) * 0.5);
  while ((r + 1) * (r + 2) / 2 <= idx) ++r;
  while (r * (r + 1) / 2 > idx) --r;
  a = r;
  b = idx - r * (r + 1) / 2;
}

// Matrix b and lower (symmetric sweep) or any (general sweep) tile (ta, tb) of update item g,
// skipping the pivot row/column kb.
template <bool kSym>
__device__ __forceinline__ void update_tile_of(int g, int per, int t, int kb, int& b, int& ta, int& tb) {
  b = g / per;
  const int local = g - b * per;
  if (kSym) {
    lower_pair(local, ta, tb);
  } else {
    ta = local / t;
    tb = local % t;
  }
  ta += (ta >= kb) ? 1 : 0;
  tb += (tb >= kb) ? 1 : 0;
}

// Persistent tile loop of the trailing update: tiles come from the step's atomic queue; the
// next tile's first K-chunk is issued before the current tile's epilogue and its C tile
// right after, so only the product itself is on the critical path of a CTA.
template <bool kSym, class Acc>
__device__ inline void update_tiles(double* M, long long mstride, int ld, int kb, const double* cold, long long cstride, int t, int per, int total, bool skip_pivot, int* queue,
                                    double* smem) {
  const int tid = threadIdx.x;
  double* Cs = smem + kUpdStageDoubles;
  int* slot = reinterpret_cast<int*>(Cs + kBlock * kStride);
  const int k0 = kb * kBlock;
  auto fetch = [&]() {
    if (tid == 0) {
      int g = atomicAdd(queue, 1);
      for (;;) {
        if (g >= total || !skip_pivot) break;
        int b, ta, tb;
        update_tile_of<kSym>(g, per, t, kb, b, ta, tb);
        if (ta != kb + 1 || tb != kb + 1) break;
        g = atomicAdd(queue, 1);  // the pivot tile belongs to a pivot CTA
      }
      *slot = g;
    }
    __syncthreads();
    const int g = *slot;
    __syncthreads();
    return g;
  };
  int g = fetch();
  if (g >= total) return;
  int b, ta, tb;
  update_tile_of<kSym>(g, per, t, kb, b, ta, tb);
  issue_update_chunk0(cold + (long long)b * cstride + ta * kBlock, ld, M + (long long)b * mstride + (long long)k0 * ld + tb * kBlock, ld, smem);
  issue_update_ctile(Cs, M + (long long)b * mstride + (long long)ta * kBlock * ld + tb * kBlock, ld);
  for (;;) {
    double* Mb = M + (long long)b * mstride;
    const int r0 = ta * kBlock, c0 = tb * kBlock;
    Acc acc;
    update_mainloop(acc, cold + (long long)b * cstride + r0, ld, Mb + (long long)k0 * ld + c0, ld, kBlock, smem);
    const int gn = fetch();
    int bn = 0, tan = 0, tbn = 0;
    if (gn < total) {
      update_tile_of<kSym>(gn, per, t, kb, bn, tan, tbn);
      issue_update_chunk0(cold + (long long)bn * cstride + tan * kBlock, ld, M + (long long)bn * mstride + (long long)k0 * ld + tbn * kBlock, ld, smem);
    }
    // C - acc straight from registers (with the transpose of an off-diagonal tile of the
    // symmetric sweep, a diagonal tile symmetrised from its lower half); Cs is free after
    acc_epilogue_direct(acc, Cs, Mb, ld, r0, c0, kSym);
    __syncthreads();
    if (gn >= total) break;
    issue_update_ctile(Cs, M + (long long)bn * mstride + (long long)tan * kBlock * ld + tbn * kBlock, ld);
    b = bn;
    ta = tan;
    tb = tbn;
  }
}

// The same persistent tile loop for the TF32x3 steps, with the operands split while staging:
// the next tile's first chunk goes into registers before the current tile's epilogue.
template <bool kSym>
__device__ inline void update_tiles_split(double* M, long long mstride, int ld, int kb, const double* cold, long long cstride, int t, int per, int total, bool skip_pivot,
                                          int* queue, double* smem) {
  const int tid = threadIdx.x;
  double* Cs = smem + kUpdStageDoubles;
  unsigned* stages = reinterpret_cast<unsigned*>(smem);
  int* slot = reinterpret_cast<int*>(Cs + kBlock * kStride);
  const int k0 = kb * kBlock;
  auto fetch = [&]() {
    if (tid == 0) {
      int g = atomicAdd(queue, 1);
      for (;;) {
        if (g >= total || !skip_pivot) break;
        int b, ta, tb;
        update_tile_of<kSym>(g, per, t, kb, b, ta, tb);
        if (ta != kb + 1 || tb != kb + 1) break;
        g = atomicAdd(queue, 1);  // the pivot tile belongs to a pivot CTA
      }
      *slot = g;
    }
    __syncthreads();
    const int g = *slot;
    __syncthreads();
    return g;
  };
  int g = fetch();
  if (g >= total) return;
  int b, ta, tb;
  update_tile_of<kSym>(g, per, t, kb, b, ta, tb);
  SplitChunk r;
  load_split_chunk(r, cold + (long long)b * cstride + ta * kBlock, ld, M + (long long)b * mstride + (long long)k0 * ld + tb * kBlock, ld, 0);
  issue_update_ctile(Cs, M + (long long)b * mstride + (long long)ta * kBlock * ld + tb * kBlock, ld);
  for (;;) {
    double* Mb = M + (long long)b * mstride;
    const int r0 = ta * kBlock, c0 = tb * kBlock;
    TileAcc32 acc;
    split_mainloop(acc, r, cold + (long long)b * cstride + r0, ld, Mb + (long long)k0 * ld + c0, ld, stages);
    const int gn = fetch();
    int bn = 0, tan = 0, tbn = 0;
    if (gn < total) {
      update_tile_of<kSym>(gn, per, t, kb, bn, tan, tbn);
      load_split_chunk(r, cold + (long long)bn * cstride + tan * kBlock, ld, M + (long long)bn * mstride + (long long)k0 * ld + tbn * kBlock, ld, 0);
    }
    cp_async_wait<0>();  // the C tile
    __syncthreads();
    acc_epilogue_direct(acc, Cs, Mb, ld, r0, c0, kSym);
    __syncthreads();
    if (gn >= total) break;
    issue_update_ctile(Cs, M + (long long)bn * mstride + (long long)tan * kBlock * ld + tbn * kBlock, ld);
    b = bn;
    ta = tan;
    tb = tbn;
  }
}

// Trailing update M_RR -= cold^T U: the symmetric sweep visits the lower-triangular tiles
// and mirrors them, the general sweep visits every tile.  Persistent: about one CTA per SM.
// The first `batch` CTAs first update the next pivot block (kb+1, kb+1) of their matrix and
// invert it in place, so the next step's row panel needs no separate pivot launch, then
// join the tile queue (reset to 0 by this step's row-panel kernel).
template <bool kSym>
__global__ void __launch_bounds__(kGemmThreads, 1) sweep_update_kernel(double* __restrict__ M, long long mstride, int ld, int kb, const double* __restrict__ cold, long long cstride, int tiles_per_dim, int batch, int fuse_next, double* __restrict__ pinv, int* status, const int* __restrict__ reduced_blocks, int* queue) {
  extern __shared__ double smem[];
  const int t = tiles_per_dim;  // tiles per dimension excluding the pivot block kb
  const int per = kSym ? t * (t + 1) / 2 : t * t;
  const int total = per * batch;
  const int tid = threadIdx.x;
  const int k0 = kb * kBlock;
  double* Cs = smem + kUpdStageDoubles;  // [A/B stages | C tile]; the inversion's scratch reuses the stages
  // the leading `*reduced_blocks` pivot blocks (channels closed beyond the threshold of the
  // mixed-precision mode) take the FP32-accurate TF32x3 product; all others FP64 DMMA
  const bool reduced = reduced_blocks != nullptr && kb < *reduced_blocks;
  if (fuse_next && (int)blockIdx.x < batch) {
    const int b = blockIdx.x;
    const int p0 = (kb + 1) * kBlock;
    double* Mb = M + (long long)b * mstride;
    const double* A = cold + (long long)b * cstride + p0;
    const double* B = Mb + (long long)k0 * ld + p0;
    const double* Cg = Mb + (long long)p0 * ld + p0;
    if (reduced) {
      TileAcc32 acc;
      tile_update_product(acc, A, ld, B, ld, kBlock, smem, Cs, Cg, ld);
      acc_sub_smem(acc, Cs);
    } else {
      TileAcc acc;
      tile_update_product(acc, A, ld, B, ld, kBlock, smem, Cs, Cg, ld);
      acc_sub_smem(acc, Cs);
    }
    __syncthreads();
    if (kSym) {  // symmetrise the pivot block from its lower half, as store_tile would
      for (int e = tid; e < kBlock * kBlock; e += kGemmThreads) {
        const int r = e >> 7, c = e & (kBlock - 1);
        if (r < c) Cs[r * kStride + c] = Cs[c * kStride + r];
      }
      __syncthreads();
    }
    invert_pivot_block<kSym>(Cs, smem, Mb, ld, p0, pinv, b, status);
    __syncthreads();
  }
  if (reduced) {
    update_tiles_split<kSym>(M, mstride, ld, kb, cold, cstride, t, per, total, fuse_next != 0, queue, smem);
  } else {
    update_tiles<kSym, TileAcc>(M, mstride, ld, kb, cold, cstride, t, per, total, fuse_next != 0, queue, smem);
  }
}

// ---- one persistent launch per step of the symmetric sweep ---------------------------------
// Work units from one queue, in order: the step's row-panel tiles (matrix b, column tile jt),
// then the fused next-pivot units (one per matrix), then the trailing-update tiles.  A unit
// waits only for row-panel tiles, which come earlier in the queue and so were fetched by
// CTAs that are already running: the waits cannot deadlock.  Each wait is still bounded; on
// timeout the CTA raises a shared abort flag, reports kDeviceStalled and skips the unit.
// Flags hold the step number + 1 of the last finished row-panel tile; queues alternate by
// step parity (each step resets the next step's) and so do the two P^-1 slots of a matrix
// (a pivot unit writes the next step's slot while row-panel tiles still read this one).
// Per-matrix integer area (the 16-double tail of the sweep scratch): [0..1] queues (matrix 0),
// [2] abort flag (matrix 0), [4 .. 4 + nt) row-panel flags.
constexpr int kStepFlagOffset = 4;
constexpr int kStepIntsPerMatrix = 32;
constexpr long long kStepSpinLimit = 1LL << 22;

__device__ __forceinline__ int load_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void store_release(int* p, int v) { asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory"); }

// Polls a wait may spend before it gives up (kStepSpinLimit unless a test lowers it through
// ticc_debug_set_step_poll_limit; 0 makes every wait give up before its first poll).
__device__ long long g_step_poll_limit = kStepSpinLimit;

// Thread 0 waits until both flags reach `target`; the CTA learns the outcome.
__device__ inline bool step_wait(const int* f0, const int* f1, int target, int* abort_flag, int* status, int b, int* slot) {
  if (threadIdx.x == 0) {
    int ok = 1;
    const long long limit = g_step_poll_limit;
    for (long long it = 0;; ++it) {
      if (it >= limit || load_acquire(abort_flag) != 0) {
        if (atomicExch(abort_flag, 1) == 0) report_status(status, kDeviceStalled, b, target);
        ok = 0;
        break;
      }
      if (load_acquire(f0) >= target && load_acquire(f1) >= target) break;
      __nanosleep(128);
    }
    *slot = ok;
  }
  __syncthreads();
  const bool ok = *slot != 0;
  __syncthreads();
  return ok;
}

// ---- streamed update phase of a tensor-core step ------------------------------------------------
// Once a CTA of a reduced step has claimed its first trailing-update unit, it stops working unit
// by unit and streams every further update unit it can claim through warp-specialised roles:
//   thread 0   claims units, waits for their row-panel flags and keeps the operand ring full
//              across unit boundaries (chunk g of the CTA in stage g % 4, as in tc_product),
//              refilling a stage as soon as its products are done;
//   warps 1-2  split the landed chunks into TF32 hi/lo;
//   thread 96  (warp 3) issues each unit's MMAs into TMEM accumulator j % 2 and never waits
//              for a product to finish;
//   warps 4-7  run the epilogues (one TMEM lane = one row each): C <- C - D in the C buffer, then
//              their leader (thread 128) stores the tile by TMA and, once the store has read
//              the buffer, loads the next unit's C tile into it.
// So unit j + 1's loads and products overlap unit j's epilogue and store.  Units reach the
// roles through a ring of kTcDescSlots descriptors (b < 0 ends the stream).  Every wait is
// bounded and gives up once another thread of the CTA has; decisions are warp-uniform, and
// the roles meet only in mbarriers, so a role that gives up leaves no other waiting for ever.
struct TcUnitDesc {
  int b, ta, tb, pad;
};

__device__ __forceinline__ volatile TcUnitDesc* tc_desc_slot(const TcState& s, int j) { return reinterpret_cast<volatile TcUnitDesc*>(s.base + kTcDescOffset) + (j % kTcDescSlots); }

__device__ __forceinline__ int load_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Bounded poll of two row-panel flags by one thread (thread 0 of the streaming CTA): both
// loads in flight together, then one acquire fence once both are set.
__device__ inline bool tc_flags_ready(const int* fa, const int* fb, int target, int* abort_flag, int* status, int b) {
  const long long limit = g_step_poll_limit;
  for (long long it = 0;; ++it) {
    const int va = load_relaxed(fa), vb = load_relaxed(fb);
    if (va >= target && vb >= target) {
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
      return true;
    }
    if (it >= limit || load_acquire(abort_flag) != 0) {
      if (atomicExch(abort_flag, 1) == 0) report_status(status, kDeviceStalled, b, target);
      return false;
    }
    __nanosleep(128);
  }
}

// Issue the TMA loads of the C tile of unit d into the C buffer (the leader of the epilogue warps).
__device__ __forceinline__ void tc_stream_load_c(const TcState& s, const TcMaps& maps, const TcUnitDesc& d) {
  const uint32_t cbar = tc_bar(s, kTcCFull);
  fence_proxy_async_shared();
  mbar_expect_tx(cbar, kTcCBytes);
  const uint64_t once = l2_policy_evict_first();
  for (int q = 0; q < 8; ++q) tma_load_3d(s.base_u + (uint32_t)q * kTcCChunkBytes, &maps.matrix, d.tb * kBlock + 16 * q, d.ta * kBlock, d.b, cbar, once);
}

// Unit (b0, ta0, tb0) has been claimed and its flags acquired by the whole CTA; the rest of the
// step's queue (units first_update .. total - 1) is claimed here.  Returns false (on every
// thread) if a wait gave up: the abort flag and status are then set and the issued work has
// been drained.
__device__ inline bool tc_update_stream(TcState& s, const TcMaps& maps, int b0, int ta0, int tb0, int* queue, int first_update, int total, int per, int t, int kb, bool fuse_next,
                                        const int* ints, int* abort_flag, int* status) {
  constexpr int nchunks = kBlock / kTcChunk;  // 8
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t g0 = s.chunk, tile0 = s.tile;
  const uint32_t cbar = tc_bar(s, kTcCFull);
  if (tid == 0) {
    // ---- producer: claims units and keeps the operand ring full
    int ok = 1, n_units = 0;
    uint32_t g_next = g0;  // next chunk to load
    TcUnitDesc units[kTcDescSlots];
    // units are claimed two at a time; the row-panel flags already seen set for the current
    // matrix are remembered (bit ct of `seen` for matrix seen_b)
    int claim_next = 0, claim_left = 0, seen_b = -1;
    uint32_t seen = 0;
    auto publish = [&](int j, int b, int ta, int tb) -> bool {
      // the slot's previous descriptor (unit j - kTcDescSlots) has been read by every role
      if (j >= kTcDescSlots && !mbar_wait_or_abort(tc_bar(s, kTcDescEmpty + j % kTcDescSlots), ((j - kTcDescSlots) / kTcDescSlots) & 1u, s.abort)) return false;
      volatile TcUnitDesc* d = tc_desc_slot(s, j);
      d->b = b;
      d->ta = ta;
      d->tb = tb;
      mbar_arrive(tc_bar(s, kTcDescFull + j % kTcDescSlots));
      return true;
    };
    fence_proxy_async_shared();
    fence_proxy_async_global();
    units[0] = TcUnitDesc{b0, ta0, tb0, 0};
    if (publish(0, b0, ta0, tb0)) n_units = 1;
    else ok = 0;
    while (ok) {
      const int j = (int)((g_next - g0) / nchunks), c = (int)((g_next - g0) % nchunks);
      if (j == n_units) {  // the next unit: claim it (or end the stream)
        if (claim_left == 0) {
          claim_next = atomicAdd(queue, 2);
          claim_left = 2;
        }
        const int u = claim_next++;
        --claim_left;
        if (u >= total) {
          if (!publish(n_units, -1, 0, 0)) ok = 0;
          break;
        }
        int b, ta, tb;
        update_tile_of<true>(u - first_update, per, t, kb, b, ta, tb);
        if (fuse_next && ta == kb + 1 && tb == kb + 1) continue;  // the pivot unit's tile
        const int* fl = ints + b * kStepIntsPerMatrix + kStepFlagOffset;
        if (b != seen_b) {
          seen_b = b;
          seen = 0;
        }
        const uint32_t need = (1u << ta) | (1u << tb);
        if ((seen & need) != need) {
          if (!tc_flags_ready(fl + ta, fl + tb, kb + 1, abort_flag, status, b)) {
            ok = 0;
            break;
          }
          seen |= need;
          fence_proxy_async_global();  // the released panels are read next by TMA
        }
        units[n_units % kTcDescSlots] = TcUnitDesc{b, ta, tb, 0};
        if (!publish(n_units, b, ta, tb)) {
          ok = 0;
          break;
        }
        ++n_units;
      }
      // the MMAs that last read this stage (chunk g_next - kTcStages) have completed
      const int stage = g_next % kTcStages;
      if (g_next >= (uint32_t)kTcStages && !mbar_wait_or_abort(tc_bar(s, kTcEmpty + stage), ((g_next - kTcStages) / kTcStages) & 1u, s.abort)) {
        ok = 0;
        break;
      }
      const TcUnitDesc& d = units[j % kTcDescSlots];
      tc_issue_chunk(s, &maps.split, tc_split_block(d.b, 0, s.nt, d.ta, 0), tc_split_block(d.b, 1, s.nt, d.tb, 0), c, stage);
      ++g_next;
    }
    if (!ok) {
      *s.abort = 1;  // the other roles stop waiting
      if (atomicExch(abort_flag, 1) == 0) report_status(status, kDeviceStalled, -1, -1);
      // the last kTcStages loads issued land before the CTA moves on (earlier ones were
      // waited for through their stages' empty phases)
      for (uint32_t g = (g_next > g0 + kTcStages ? g_next - kTcStages : g0); g < g_next; ++g) mbar_wait(tc_bar(s, kTcFull + g % kTcStages), (g / kTcStages) & 1u);
    }
  } else if (tid == 32 * kTcMmaWarp) {
    // ---- MMA issuer: unit j into TMEM accumulator j % 2, never waiting for a product
    bool ok = true, mma_issued = false;
    for (int j = 0; ok; ++j) {
      if (!mbar_wait_or_abort(tc_bar(s, kTcDescFull + j % kTcDescSlots), (j / kTcDescSlots) & 1u, s.abort)) {
        ok = false;
        break;
      }
      const int b = tc_desc_slot(s, j)->b;
      mbar_arrive(tc_bar(s, kTcDescEmpty + j % kTcDescSlots));
      if (b < 0) break;
      const uint32_t d_tmem = s.tmem + (uint32_t)((j & 1) * kBlock);
      for (int c = 0; c < nchunks; ++c) {
        const uint32_t g = g0 + (uint32_t)(j * nchunks + c);
        const int stage = g % kTcStages;
        if (!mbar_wait_or_abort(tc_bar(s, kTcConv + stage), (g / kTcStages) & 1u, s.abort)) {
          ok = false;
          break;
        }
        // accumulator j % 2 has been read out by the epilogue of unit j - 2
        if (c == 0 && j >= 2 && !mbar_wait_or_abort(tc_bar(s, kTcAccEmpty + (j & 1)), ((j - 2) / 2) & 1u, s.abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t st = s.base_u + kTcStageOffset + (uint32_t)stage * kTcStageBytes;
        const uint32_t lo = s.base_u + kTcLoOffset + (uint32_t)(g % kTcLoBufs) * kTcStageBytes;
#pragma unroll
        for (int kg = 0; kg < kTcChunk / 8; ++kg) {
          const uint64_t a_hi = tc_desc(st, kg), a_lo = tc_desc(lo, kg);
          const uint64_t b_hi = tc_desc(st + kTcArrayBytes, kg), b_lo = tc_desc(lo + kTcArrayBytes, kg);
          tc_mma_tf32(d_tmem, a_lo, b_hi, (c > 0 || kg > 0) ? 1u : 0u);
          tc_mma_tf32(d_tmem, a_hi, b_lo, 1u);
          tc_mma_tf32(d_tmem, a_hi, b_hi, 1u);
        }
        mma_issued = true;
        tc_commit(tc_bar(s, kTcEmpty + stage));
        if (c == nchunks - 1) tc_commit(tc_bar(s, kTcAccFull + (j & 1)));
      }
    }
    if (!ok) {
      *s.abort = 1;
      if (mma_issued) {  // the products land before the CTA moves on or frees TMEM
        tc_commit(tc_bar(s, kTcDrain));
        mbar_wait(tc_bar(s, kTcDrain), 0u);
      }
    }
  } else if (warp >= 1 && warp <= kTcStreamConvWarps) {
    // ---- warps 1-3: split the chunks of every unit (lanes 1-31 of warp 0 have no role)
    bool ok = true;
    for (int j = 0; ok; ++j) {
      ok = __all_sync(0xffffffffu, mbar_wait_or_abort(tc_bar(s, kTcDescFull + j % kTcDescSlots), (j / kTcDescSlots) & 1u, s.abort));
      if (!ok) break;
      const int b = tc_desc_slot(s, j)->b;
      __syncwarp();
      if (lane == 0) mbar_arrive(tc_bar(s, kTcDescEmpty + j % kTcDescSlots));
      if (b < 0) break;
      for (int c = 0; c < nchunks; ++c) {
        const uint32_t g = g0 + (uint32_t)(j * nchunks + c);
        const int stage = g % kTcStages;
        bool w = mbar_wait_or_abort(tc_bar(s, kTcFull + stage), (g / kTcStages) & 1u, s.abort);
        if (w && g >= (uint32_t)kTcLoBufs) {
          const uint32_t gp = g - kTcLoBufs;
          w = mbar_wait_or_abort(tc_bar(s, kTcEmpty + gp % kTcStages), (gp / kTcStages) & 1u, s.abort);
        }
        if (!__all_sync(0xffffffffu, w)) {
          ok = false;
          break;
        }
        tc_split_stage_all<32 * kTcStreamConvWarps>(s, stage, g % kTcLoBufs);
        fence_proxy_async_shared();  // read next by the tensor core
        __syncwarp();
        // the conversion barrier counts kTcConvWarps warp arrivals: warp 1 stands in for the rest
        if (lane == 0) mbar_arrive_count(tc_bar(s, kTcConv + stage), warp == 1 ? kTcConvWarps - (kTcStreamConvWarps - 1) : 1);
      }
    }
    if (!ok) *s.abort = 1;
  } else if (warp > kTcMmaWarp) {
    // ---- warps 4-7: epilogues, in two column halves of the C buffer; thread 128 moves the C
    // tiles half by half, so that the next tile's first half loads while this tile's second
    // half is still being formed and stored
    const bool leader = tid == 32 * (kTcMmaWarp + 1);
    const int r = 32 * (warp & 3) + lane;  // TMEM lane = tile row of this thread
    const uint32_t cbar_hi = tc_bar(s, kTcCFullHi);
    bool ok = true;
    unsigned c_pending = 0;  // halves whose load this thread issued and no epilogue has waited for
    uint32_t c_phase[2] = {0, 0};
    auto load_half = [&](const TcUnitDesc& d, int h, uint32_t bar) {
      fence_proxy_async_shared();
      mbar_expect_tx(bar, kTcCBytes / 2);
      const uint64_t once = l2_policy_evict_first();
      for (int q = 4 * h; q < 4 * h + 4; ++q) tma_load_3d(s.base_u + (uint32_t)q * kTcCChunkBytes, &maps.matrix, d.tb * kBlock + 16 * q, d.ta * kBlock, d.b, bar, once);
    };
    for (int j = 0; ok; ++j) {
      ok = __all_sync(0xffffffffu, mbar_wait_or_abort(tc_bar(s, kTcDescFull + j % kTcDescSlots), (j / kTcDescSlots) & 1u, s.abort));
      if (!ok) break;
      TcUnitDesc d;
      d.b = tc_desc_slot(s, j)->b;
      d.ta = tc_desc_slot(s, j)->ta;
      d.tb = tc_desc_slot(s, j)->tb;
      __syncwarp();
      if (lane == 0) mbar_arrive(tc_bar(s, kTcDescEmpty + j % kTcDescSlots));
      if (d.b < 0) break;
      const uint32_t ph_lo = (tile0 + (uint32_t)j) & 1u, ph_hi = (uint32_t)j & 1u;
      if (leader && j == 0) {  // the C buffer is free: earlier units of this CTA left no store pending
        load_half(d, 0, cbar);
        load_half(d, 1, cbar_hi);
        c_pending = 3u;
        c_phase[0] = ph_lo;
        c_phase[1] = ph_hi;
      }
      const bool diagonal = d.ta == d.tb;
      // a diagonal tile's mirror writes reach the second half from the first
      bool w = mbar_wait_or_abort(tc_bar(s, kTcAccFull + (j & 1)), (j / 2) & 1u, s.abort);
      if (w) w = mbar_wait_or_abort(cbar, ph_lo, s.abort);
      if (w && diagonal) w = mbar_wait_or_abort(cbar_hi, ph_hi, s.abort);
      if (!__all_sync(0xffffffffu, w)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t row_tmem = s.tmem + (uint32_t)((j & 1) * kBlock) + ((uint32_t)(32 * (warp & 3)) << 16);
      for (int h = 0; h < 2 && ok; ++h) {
        if (h == 1 && !diagonal && !__all_sync(0xffffffffu, mbar_wait_or_abort(cbar_hi, ph_hi, s.abort))) {
          ok = false;
          break;
        }
        if (h == 1) tc_fence_after();
#pragma unroll 1
        for (int q = 0; q < 2; ++q) {
          const int col = 64 * h + 32 * q;
          float dv[32];
          tc_ld_32(row_tmem + (uint32_t)col, dv);
          if (!diagonal) {
            double2 v[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) v[u] = *reinterpret_cast<const double2*>(s.base + tc_c_offset(r, col + 2 * u));
#pragma unroll
            for (int u = 0; u < 16; ++u) {
              v[u].x -= (double)dv[2 * u];
              v[u].y -= (double)dv[2 * u + 1];
              *reinterpret_cast<double2*>(s.base + tc_c_offset(r, col + 2 * u)) = v[u];
            }
          } else if (col <= r) {
            // a diagonal tile keeps its lower half and mirrors it: row r writes (r, n) and
            // (n, r) for n <= r; the upper elements of row r are written by the rows below
#pragma unroll
            for (int u = 0; u < 32; ++u) {
              const int n = col + u;
              if (n <= r) {
                double* p = reinterpret_cast<double*>(s.base + tc_c_offset(r, n));
                const double v = *p - (double)dv[u];
                *p = v;
                *reinterpret_cast<double*>(s.base + tc_c_offset(n, r)) = v;
              }
            }
          }
        }
        if (h == 1) tc_fence_before();
        fence_proxy_async_shared();  // the rows are read next by the TMA store
        __syncwarp();
        if (lane == 0) {
          if (h == 1) mbar_arrive(tc_bar(s, kTcAccEmpty + (j & 1)));
          mbar_arrive(tc_bar(s, h == 0 ? kTcEpiDone : kTcEpiDoneHi));
        }
        if (leader) {
          // every epilogue warp has written this half (a diagonal tile's first half is final
          // once every row has done its first half; its second half, once every row is done)
          bool l = mbar_wait_or_abort(tc_bar(s, h == 0 ? kTcEpiDone : kTcEpiDoneHi), (uint32_t)j & 1u, s.abort);
          if (l) {
            c_pending &= ~(1u << h);
            const uint64_t once = l2_policy_evict_first();
            for (int q = 4 * h; q < 4 * h + 4; ++q) tma_store_3d(&maps.matrix, s.base_u + (uint32_t)q * kTcCChunkBytes, d.tb * kBlock + 16 * q, d.ta * kBlock, d.b, once);
            bulk_commit();
          }
          ok = l;
        }
        ok = __all_sync(0xffffffffu, ok);
      }
      if (!ok) break;
      if (leader) {
        // the next unit's C tile, half by half as this tile's stores read the buffer out
        bool l = mbar_wait_or_abort(tc_bar(s, kTcDescFull + (j + 1) % kTcDescSlots), ((j + 1) / kTcDescSlots) & 1u, s.abort);
        if (l) {
          TcUnitDesc nd;
          nd.b = tc_desc_slot(s, j + 1)->b;
          nd.ta = tc_desc_slot(s, j + 1)->ta;
          nd.tb = tc_desc_slot(s, j + 1)->tb;
          if (nd.b >= 0) {
            asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");  // the first half's store
            load_half(nd, 0, cbar);
            bulk_wait_read_all();
            load_half(nd, 1, cbar_hi);
            c_pending = 3u;
            c_phase[0] = (tile0 + (uint32_t)j + 1) & 1u;
            c_phase[1] = (uint32_t)(j + 1) & 1u;
          }
        }
        ok = l;
      }
      ok = __all_sync(0xffffffffu, ok);
    }
    if (leader) {
      bulk_wait_all();  // this thread's stores are complete before the CTA moves on
      if (c_pending & 1u) mbar_wait(cbar, c_phase[0]);
      if (c_pending & 2u) mbar_wait(cbar_hi, c_phase[1]);
    }
    if (!ok) *s.abort = 1;
  }
  __syncthreads();
  return *s.abort == 0;
}

// Row-panel tile (b, jt) of step kb: keep the old rows K in `cold`, U = P^-1 M_KR, U into
// the rows K and, where (jt, kb) is a lower tile, U^T into the columns K.  Pt is this
// matrix's P^-1 for the step.  When the
// pivot block K is strongly closed (`reduced`), U takes the same FP32-accurate TF32x3
// product as the step's trailing update.
// With `split` (a reduced step whose trailing update runs on tcgen05), the old rows and U of
// this column tile also go out as FP32 panels for the update's TMA loads.
__device__ inline void rowpanel_unit(double* Mb, int ld, int kb, int jt, const double* Pt, double* Cb, double* smem, bool reduced, float* split, int b) {
  const int k0 = kb * kBlock, c0 = jt * kBlock;
  load_cold_tile(Cb, ld, Mb, kb, jt, smem);
  if (reduced) {
    TileAcc32 acc;
    tile_gemm_tn_tf32x3(acc, Pt, kBlock, Cb + c0, ld, kBlock, smem);
    acc32_to_smem_mirror(acc, smem, Mb + (long long)c0 * ld + k0, ld, jt > kb);
  } else {
    TileAcc acc;
    tile_gemm_tn(acc, Pt, kBlock, Cb + c0, ld, kBlock, smem);
    acc_to_smem_mirror(acc, smem, Mb + (long long)c0 * ld + k0, ld, jt > kb);
  }
  __syncthreads();
  store_tile(Mb, ld, k0, c0, smem);
  if (split != nullptr) {
    tc_write_panel(split, b, 0, ld, Cb, ld, c0, jt);          // A = the old rows K
    tc_write_panel(split, b, 1, ld, smem, kStride, 0, jt);    // B = U = P^-1 (old rows K)
    fence_proxy_async_global();                               // read next by TMA (async proxy)
  }
}

template <class Acc>
__device__ inline void update_unit(Acc& acc, double* Mb, int ld, int k0, int r0, int c0, const double* Cb, double* smem) {
  double* Cs = smem + kUpdStageDoubles;
  tile_update_product(acc, Cb + r0, ld, Mb + (long long)k0 * ld + c0, ld, kBlock, smem, Cs, Mb + (long long)r0 * ld + c0, ld);
  acc_epilogue_direct(acc, Cs, Mb, ld, r0, c0, true);
  __syncthreads();
}

__device__ inline void update_unit_split(double* Mb, int ld, int k0, int r0, int c0, const double* Cb, double* smem) {
  double* Cs = smem + kUpdStageDoubles;
  SplitChunk r;
  load_split_chunk(r, Cb + r0, ld, Mb + (long long)k0 * ld + c0, ld, 0);
  issue_update_ctile(Cs, Mb + (long long)r0 * ld + c0, ld);
  TileAcc32 acc;
  split_mainloop(acc, r, Cb + r0, ld, Mb + (long long)k0 * ld + c0, ld, reinterpret_cast<unsigned*>(smem));
  cp_async_wait<0>();
  __syncthreads();
  acc_epilogue_direct(acc, Cs, Mb, ld, r0, c0, true);
  __syncthreads();
}

// Dynamic shared memory of the step kernel: the FP64 units use the first kUpdTileSmemBytes,
// a reduced step's tcgen05 units the first kTcSmemBytes; the unit queue's broadcast slot
// sits after both.
constexpr size_t kStepSlotOffset = (size_t(kTcSmemBytes) > kUpdTileSmemBytes ? size_t(kTcSmemBytes) : kUpdTileSmemBytes);
constexpr size_t kStepSmemBytes = kStepSlotOffset + 16;
// The FP64 units (row panels, pivots, mma.sync updates) that share a CTA with the tcgen05
// units overwrite shared memory below kUpdTileSmemBytes between them: the tcgen05 barriers
// and TMEM slot, which live across units, must sit above it.
static_assert(size_t(kTcBarOffset) >= kUpdTileSmemBytes, "tcgen05 barriers must lie beyond the FP64 units' shared memory");

// In a reduced step with `split` (and tensor maps over it and M), the trailing-update tiles
// run on the tcgen05 tensor core (tc_update_unit); otherwise on the mma.sync paths.
__global__ void __launch_bounds__(kGemmThreads, 1) sweep_step_kernel(double* __restrict__ M, long long mstride, int ld, int kb, double* __restrict__ cold, long long cstride, int t, int batch, int fuse_next, double* __restrict__ pinv, int* status, const int* __restrict__ reduced_blocks, int* ints,
                                                                     float* __restrict__ split, const __grid_constant__ TcMaps maps) {
  extern __shared__ double smem[];
  const int tid = threadIdx.x;
  int* slot = reinterpret_cast<int*>(reinterpret_cast<char*>(smem) + kStepSlotOffset);
  int* queue = ints + (kb & 1);
  int* abort_flag = ints + 2;
  if (blockIdx.x == 0 && tid == 0) ints[(kb + 1) & 1] = 0;  // the next step's queue
  const int per = t * (t + 1) / 2;
  const int n_panel = t * batch;
  const int n_pivot = fuse_next ? batch : 0;
  const int total = n_panel + n_pivot + per * batch;
  const int k0 = kb * kBlock;
  const int pslot = kb & 1, nslot = (kb + 1) & 1;
  const bool reduced = reduced_blocks != nullptr && kb < *reduced_blocks;
  const bool tensor_core = reduced && split != nullptr;
  TcState tcs;
  bool tc_live = false;
  if (tensor_core) {
    tc_setup(tcs, smem, ld);
    tc_live = true;
  }
  for (;;) {
    // the previous unit's generic shared-memory writes come before any TMA load of the next
    if (tensor_core) fence_proxy_async_shared();
    if (tid == 0) *slot = atomicAdd(queue, 1);
    __syncthreads();
    const int u = *slot;
    __syncthreads();
    if (u >= total) break;
    if (u < n_panel) {
      const int b = u / t, j = u % t;
      const int jt = j + (j >= kb ? 1 : 0);
      double* Mb = M + (long long)b * mstride;
      if (tc_live) {
        if (!tc_rowpanel_unit(tcs, maps, split, tc_pinv_block(b, pslot, t + 1, batch), b, kb, jt, Mb, ld, cold + (long long)b * cstride, abort_flag, status)) tc_live = false;
      } else {
        rowpanel_unit(Mb, ld, kb, jt, pinv + (long long)b * 2 * kBlock * kBlock + pslot * kBlock * kBlock, cold + (long long)b * cstride, smem, reduced, tensor_core ? split : nullptr, b);
      }
      __syncthreads();
      if (tid == 0) {
        __threadfence();
        store_release(ints + b * kStepIntsPerMatrix + kStepFlagOffset + jt, kb + 1);
      }
      continue;
    }
    if (u < n_panel + n_pivot) {
      const int b = u - n_panel;
      const int p0 = (kb + 1) * kBlock;
      const int* f = ints + b * kStepIntsPerMatrix + kStepFlagOffset + kb + 1;
      if (!step_wait(f, f, kb + 1, abort_flag, status, b, slot)) continue;
      double* Mb = M + (long long)b * mstride;
      double* Cs = smem + kUpdStageDoubles;
      const double* A = cold + (long long)b * cstride + p0;
      const double* B = Mb + (long long)k0 * ld + p0;
      const double* Cg = Mb + (long long)p0 * ld + p0;
      if (reduced) {
        TileAcc32 acc;
        tile_update_product(acc, A, ld, B, ld, kBlock, smem, Cs, Cg, ld);
        acc_sub_smem(acc, Cs);
      } else {
        TileAcc acc;
        tile_update_product(acc, A, ld, B, ld, kBlock, smem, Cs, Cg, ld);
        acc_sub_smem(acc, Cs);
      }
      __syncthreads();
      for (int e = tid; e < kBlock * kBlock; e += kGemmThreads) {  // symmetrise from the lower half
        const int r = e >> 7, c = e & (kBlock - 1);
        if (r < c) Cs[r * kStride + c] = Cs[c * kStride + r];
      }
      __syncthreads();
      invert_pivot_block<true>(Cs, smem, Mb, ld, p0, pinv + nslot * kBlock * kBlock, b, status);
      __syncthreads();
      if (split != nullptr && kb + 1 < *reduced_blocks) {  // the next step's row panels run on tcgen05
        tc_write_panel_at(split + (long long)tc_pinv_block(b, nslot, t + 1, batch) * kTcArrayFloats, pinv + nslot * kBlock * kBlock + (long long)b * 2 * kBlock * kBlock, kBlock, 0);
        fence_proxy_async_global();
        __syncthreads();
      }
      continue;
    }
    const int g = u - n_panel - n_pivot;
    int b, ta, tb;
    update_tile_of<true>(g, per, t, kb, b, ta, tb);
    if (fuse_next && ta == kb + 1 && tb == kb + 1) continue;  // the pivot unit's tile
    const int* fa = ints + b * kStepIntsPerMatrix + kStepFlagOffset + ta;
    const int* fb = ints + b * kStepIntsPerMatrix + kStepFlagOffset + tb;
    if (!step_wait(fa, fb, kb + 1, abort_flag, status, b, slot)) continue;
    double* Mb = M + (long long)b * mstride;
    const double* Cb = cold + (long long)b * cstride;
    if (tensor_core) {
      // units come in queue order (row panels, pivots, then updates): from its first update
      // unit on, the CTA streams the rest of the queue's update units; after a failure this
      // CTA's tensor-core state is unknown and it only drains the queue
      if (tc_live) {
        if (!tc_update_stream(tcs, maps, b, ta, tb, queue, n_panel + n_pivot, total, per, t, kb, fuse_next != 0, ints, abort_flag, status)) tc_live = false;
        break;
      }
    } else if (reduced) {
      update_unit_split(Mb, ld, k0, ta * kBlock, tb * kBlock, Cb, smem);
    } else {
      TileAcc acc;
      update_unit(acc, Mb, ld, k0, ta * kBlock, tb * kBlock, Cb, smem);
    }
  }
  if (tensor_core) tc_teardown(tcs);
}

// Scratch per matrix: cold (kBlock x np) + P^-1 and its transpose (2 x kBlock x kBlock).
// The last 16 doubles of each matrix's share hold the update kernel's tile queue (one int).
inline size_t sweep_scratch_doubles(int np) { return size_t(kBlock) * np + size_t(2) * kBlock * kBlock + 16; }

template <bool kSym>
inline cudaError_t sweep_configure_variant() {
  cudaError_t e = cudaFuncSetAttribute(sweep_pivot_kernel<kSym>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPivotSmemBytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(sweep_pivot64_kernel<kSym>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPivot64SmemBytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(sweep_rowpanel_kernel<kSym>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmemBytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(sweep_update_kernel<kSym>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUpdateSmemBytes);
}

inline cudaError_t sweep_configure_step() { return cudaFuncSetAttribute(sweep_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStepSmemBytes); }

inline cudaError_t sweep_configure() {
  // per-device attribute: cheap to repeat, so no process-wide cache is kept
  cudaError_t e = sweep_configure_variant<true>();
  if (e != cudaSuccess) return e;
  e = sweep_configure_variant<false>();
  if (e != cudaSuccess) return e;
  e = sweep_configure_step();
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(sweep_colpanel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmemBytes);
}

// Sweep every block of `batch` matrices of padded size np (a multiple of kBlock):
// M <- -M^{-1}.  scratch holds batch * sweep_scratch_doubles(np) doubles.
// Launches: one pivot kernel, then per block a row panel (and column panel for the
// general sweep) and an update that also inverts the next pivot block.
// With reduced_blocks and `split` (tc_split_floats(np, batch) floats, 16-byte aligned), the
// reduced steps' trailing updates run on the tcgen05 tensor core.
template <bool kSym>
inline cudaError_t sweep_batched(double* M, long long mstride, int np, int batch, double* scratch, int* status, cudaStream_t stream, const int* reduced_blocks = nullptr, int n_used = 0,
                                 float* split = nullptr) {
  cudaError_t e = sweep_configure();
  if (e != cudaSuccess) return e;
  const int nt = np / kBlock;
  if (nt == 1 && n_used > 0 && n_used <= kSub) {
    sweep_pivot64_kernel<kSym><<<batch, kPivotThreads, kPivot64SmemBytes, stream>>>(M, mstride, np, status);
    note_launch();
    return cudaGetLastError();
  }
  const long long cstride = (long long)kBlock * np;
  double* cold = scratch;
  double* pinv = scratch + (long long)batch * cstride;
  int* queue = reinterpret_cast<int*>(pinv + (long long)batch * 2 * kBlock * kBlock);
  int sms = 0;
  if (nt > 1) {
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
  }
  const bool fused = kSym && nt >= 2 && nt <= kStepIntsPerMatrix - kStepFlagOffset;
  if (fused) {
    e = cudaMemsetAsync(queue, 0, sizeof(int) * kStepIntsPerMatrix * (size_t)batch, stream);
    if (e != cudaSuccess) return e;
  }
  const bool tc_steps = kSym && reduced_blocks != nullptr && split != nullptr && nt >= 2 && nt <= kStepIntsPerMatrix - kStepFlagOffset;
  sweep_pivot_kernel<kSym><<<batch, kPivotThreads, kPivotSmemBytes, stream>>>(M, mstride, np, 0, pinv, status, tc_steps ? split : nullptr, reduced_blocks, batch);
  note_launch();
  if (fused) {
    TcMaps maps{};
    float* tc_split = (reduced_blocks != nullptr) ? split : nullptr;
    if (tc_split != nullptr) {
      e = tc_make_maps(maps, tc_split, M, np, mstride, batch);
      if (e != cudaSuccess) return e;
    }
    const int t = nt - 1;
    const long long per = (long long)t * (t + 1) / 2;
    for (int kb = 0; kb < nt; ++kb) {
      const int fuse = (kb + 1 < nt) ? 1 : 0;
      const long long work = (long long)t * batch + (fuse ? batch : 0) + per * batch;
      const long long blocks = work < sms ? work : sms;
      sweep_step_kernel<<<(unsigned)blocks, kGemmThreads, kStepSmemBytes, stream>>>(M, mstride, np, kb, cold, cstride, t, batch, fuse, pinv, status, reduced_blocks, queue, tc_split, maps);
      note_launch();
    }
    return cudaGetLastError();
  }
  for (int kb = 0; kb < nt; ++kb) {
    if (nt == 1) break;
    const int t = nt - 1;
    sweep_rowpanel_kernel<kSym><<<dim3(t, batch), kGemmThreads, kTileSmemBytes, stream>>>(M, mstride, np, kb, pinv, cold, cstride, queue);
    note_launch();
    if (!kSym) {
      sweep_colpanel_kernel<<<dim3(t, batch), kGemmThreads, kTileSmemBytes, stream>>>(M, mstride, np, kb, pinv, cold, cstride);
      note_launch();
    }
    const int per = kSym ? t * (t + 1) / 2 : t * t;
    const int fuse = (kb + 1 < nt) ? 1 : 0;
    // persistent grid: one CTA per SM (shared memory allows no second), at least one per pivot
    const long long work = (long long)per * batch + (fuse ? batch : 0);
    long long blocks = work < sms ? work : sms;
    if (fuse && blocks < batch) blocks = batch;
    sweep_update_kernel<kSym><<<(unsigned)blocks, kGemmThreads, kUpdateSmemBytes, stream>>>(M, mstride, np, kb, cold, cstride, t, batch, fuse, pinv, status, reduced_blocks, queue);
    note_launch();
  }
  return cudaGetLastError();
}

// n_used > 0 states that only the leading n_used rows and columns differ from the identity.
inline cudaError_t sweep_sym(double* M, long long mstride, int np, int batch, double* scratch, int* status, cudaStream_t stream, const int* reduced_blocks = nullptr, int n_used = 0,
                             float* split = nullptr) {
  return sweep_batched<true>(M, mstride, np, batch, scratch, status, stream, reduced_blocks, n_used, split);
}
inline cudaError_t sweep_general(double* M, long long mstride, int np, int batch, double* scratch, int* status, cudaStream_t stream) {
  return sweep_batched<false>(M, mstride, np, batch, scratch, status, stream);
}

}  // namespace ticc
