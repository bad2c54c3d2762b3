// Batched blocked symmetric sweep: M <- -M^{-1} for a batch of padded symmetric
// matrices, in place.
//
// The sweep (principal pivot transform) over an index block K with P = M_KK:
//     M_KK <- -P^{-1},   M_KR <- P^{-1} M_KR,   M_RK <- M_RK P^{-1},
//     M_RR <- M_RR - M_RK P^{-1} M_KR,
// keeps M symmetric, and sweeping every block in turn yields -M^{-1}.  Per block:
//   1. pivot kernel   : one CTA per matrix inverts the 128x128 block P in shared
//                       memory by Gauss-Jordan exchange with partial pivoting
//                       (pivoting is local to the block), writes -P^{-1} into M_KK
//                       and P^{-1} into a scratch buffer;
//   2. row-panel kernel: U = P^{-1} M_KR per 128-column tile on the FP64 tensor pipe;
//                       keeps the old rows in `cold`, writes U into rows K and U^T
//                       into columns K (exact symmetry);
//   3. update kernel  : lower-triangular tiles M_RR -= cold^T U, mirrored into the
//                       upper triangle, so the matrix stays exactly symmetric and the
//                       update costs N^2 * 128 flops instead of 2 N^2 * 128.
// Total work for an N x N inverse: N^3 flops (vs 2 N^3 for a general inverse).
#pragma once

#include "dmma_tile.cuh"
#include "ticc_common.cuh"

namespace ticc {

constexpr int kPivotLd = kBlock + 1;
constexpr size_t kPivotSmemBytes = size_t(kBlock) * kPivotLd * sizeof(double) + 2 * kBlock * sizeof(double) + 2 * kBlock * sizeof(int);

template <bool kSym>
__global__ void __launch_bounds__(kPivotThreads) sweep_pivot_kernel(double* __restrict__ M, long long mstride, int ld, int k0, double* __restrict__ pinv, int* status) {
  extern __shared__ double smem[];
  double* P = smem;
  double* prow = P + kBlock * kPivotLd;
  double* pcol = prow + kBlock;
  int* used = reinterpret_cast<int*>(pcol + kBlock);
  int* perm = used + kBlock;
  __shared__ int s_row;
  __shared__ double s_val;

  const int b = blockIdx.x;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  double* Mb = M + (long long)b * mstride;

  for (int idx = tid; idx < kBlock * kBlock; idx += kPivotThreads) {
    const int r = idx >> 7, c = idx & (kBlock - 1);
    P[r * kPivotLd + c] = Mb[(long long)(k0 + r) * ld + k0 + c];
  }
  if (tid < kBlock) used[tid] = 0;
  __syncthreads();

  bool singular = false;
  for (int j = 0; j < kBlock; ++j) {
    if (warp == 0) {
      double best = -1.0;
      int best_row = kBlock;
      for (int r = lane; r < kBlock; r += 32) {
        if (!used[r]) {
          const double v = fabs(P[r * kPivotLd + j]);
          if (v > best) {
            best = v;
            best_row = r;
          }
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, best, off);
        const int orow = __shfl_down_sync(0xffffffffu, best_row, off);
        if (ov > best || (ov == best && orow < best_row)) {
          best = ov;
          best_row = orow;
        }
      }
      if (lane == 0) {
        s_row = best_row;
        used[best_row] = 1;
        perm[j] = best_row;
        s_val = P[best_row * kPivotLd + j];
      }
    }
    __syncthreads();
    const int p = s_row;
    double a = s_val;
    if (!(fabs(a) > 0.0) || !isfinite(a)) {
      singular = true;
      a = 1.0;
    }
    if (tid < kBlock) {
      prow[tid] = P[p * kPivotLd + tid];
    } else if (tid < 2 * kBlock) {
      pcol[tid - kBlock] = P[(tid - kBlock) * kPivotLd + j];
    }
    __syncthreads();
    const double inv_a = 1.0 / a;
    for (int idx = tid; idx < kBlock * kBlock; idx += kPivotThreads) {
      const int r = idx >> 7, c = idx & (kBlock - 1);
      double v;
      if (r == p) {
        v = (c == j) ? inv_a : -prow[c] * inv_a;
      } else if (c == j) {
        v = pcol[r] * inv_a;
      } else {
        v = P[r * kPivotLd + c] - pcol[r] * (prow[c] * inv_a);
      }
      P[r * kPivotLd + c] = v;
    }
    __syncthreads();
  }
  if (singular && tid == 0) report_status(status, kDeviceSingularPivot, b, k0 / kBlock);

  // Inverse element (j, perm[c]) sits at exchange slot (perm[j], c).  The symmetric
  // sweep stores the symmetrised inverse once; the general sweep stores P^-1 and
  // its transpose (the k-major operand of the row-panel product).
  int* iperm = used;  // reuse: iperm[perm[c]] = c
  if (tid < kBlock) iperm[perm[tid]] = tid;
  __syncthreads();
  double* Pb = pinv + (long long)b * 2 * kBlock * kBlock;
  for (int idx = tid; idx < kBlock * kBlock; idx += kPivotThreads) {
    const int j = idx >> 7, m = idx & (kBlock - 1);
    const double x = P[perm[j] * kPivotLd + iperm[m]];
    if (kSym) {
      const double y = P[perm[m] * kPivotLd + iperm[j]];
      const double v = 0.5 * (x + y);
      Pb[idx] = v;
      Mb[(long long)(k0 + j) * ld + k0 + m] = -v;
    } else {
      Pb[idx] = x;
      Pb[kBlock * kBlock + m * kBlock + j] = x;
      Mb[(long long)(k0 + j) * ld + k0 + m] = -x;
    }
  }
}

// Write a finished 128x128 tile from shared memory to M at (r0, c0).  With `mirror`
// (symmetric sweep) its transpose also goes to (c0, r0) and a diagonal tile is written
// symmetrised from its lower half.
__device__ inline void store_tile(double* Mb, int ld, int r0, int c0, const double* Cs, bool mirror) {
  const int tid = threadIdx.x;
  const bool diagonal = mirror && (r0 == c0);
  for (int piece = tid; piece < kBlock * 64; piece += kGemmThreads) {
    const int r = piece >> 6;
    const int c = (piece & 63) * 2;
    double2 v;
    if (diagonal) {
      v.x = (r >= c) ? Cs[r * kStride + c] : Cs[c * kStride + r];
      v.y = (r >= c + 1) ? Cs[r * kStride + c + 1] : Cs[(c + 1) * kStride + r];
    } else {
      v.x = Cs[r * kStride + c];
      v.y = Cs[r * kStride + c + 1];
    }
    *reinterpret_cast<double2*>(Mb + (long long)(r0 + r) * ld + c0 + c) = v;
  }
  if (mirror && !diagonal) {
    for (int piece = tid; piece < kBlock * 64; piece += kGemmThreads) {
      const int r = piece >> 6;        // destination row offset (a column of Cs)
      const int c = (piece & 63) * 2;  // destination column offset (a row of Cs)
      double2 v;
      v.x = Cs[c * kStride + r];
      v.y = Cs[(c + 1) * kStride + r];
      *reinterpret_cast<double2*>(Mb + (long long)(c0 + r) * ld + r0 + c) = v;
    }
  }
}

// Row panel: U = P^-1 M_KR for one 128-column tile of the rows K.  The symmetric
// sweep also keeps the old rows (= old columns K, transposed) in `cold` and mirrors U^T
// into the columns K; the general sweep leaves the columns to the column-panel kernel.
template <bool kSym>
__global__ void __launch_bounds__(kGemmThreads) sweep_rowpanel_kernel(double* __restrict__ M, long long mstride, int ld, int kb, const double* __restrict__ pinv, double* __restrict__ cold, long long cstride) {
  extern __shared__ double smem[];
  const int b = blockIdx.y;
  const int jt = blockIdx.x + (blockIdx.x >= kb ? 1 : 0);
  const int k0 = kb * kBlock, c0 = jt * kBlock;
  double* Mb = M + (long long)b * mstride;
  double* Cb = cold + (long long)b * cstride;
  const int tid = threadIdx.x;
  if (kSym) {
    for (int piece = tid; piece < kBlock * 64; piece += kGemmThreads) {
      const int r = piece >> 6, c = (piece & 63) * 2;
      *reinterpret_cast<double2*>(Cb + (long long)r * ld + c0 + c) = *reinterpret_cast<const double2*>(Mb + (long long)(k0 + r) * ld + c0 + c);
    }
  }
  const double* Pt = pinv + (long long)b * 2 * kBlock * kBlock + (kSym ? 0 : kBlock * kBlock);
  TileAcc acc;
  tile_gemm_tn(acc, Pt, kBlock, Mb + (long long)k0 * ld + c0, ld, kBlock, smem);
  acc_to_smem(acc, smem, 1.0);
  __syncthreads();
  store_tile(Mb, ld, k0, c0, smem, kSym);
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
  for (int piece = tid; piece < kBlock * 64; piece += kGemmThreads) {
    const int r = piece >> 6, c = (piece & 63) * 2;
    const double2 v = *reinterpret_cast<const double2*>(Mb + (long long)(r0 + r) * ld + k0 + c);
    smem[r * kStride + c] = v.x;
    smem[r * kStride + c + 1] = v.y;
  }
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
  store_tile(Mb, ld, r0, k0, smem, false);
}

__device__ __forceinline__ void lower_pair(int idx, int& a, int& b) {
  int r = static_cast<int>((sqrt(8.0 * idx + 1.0) - 1.0) * 0.5);
  while ((r + 1) * (r + 2) / 2 <= idx) ++r;
  while (r * (r + 1) / 2 > idx) --r;
  a = r;
  b = idx - r * (r + 1) / 2;
}

// Trailing update M_RR -= cold^T U: the symmetric sweep visits the lower-triangular
// tiles and mirrors them, the general sweep visits every tile.
template <bool kSym>
__global__ void __launch_bounds__(kGemmThreads) sweep_update_kernel(double* __restrict__ M, long long mstride, int ld, int kb, const double* __restrict__ cold, long long cstride, int tiles_per_dim) {
  extern __shared__ double smem[];
  const int b = blockIdx.y;
  int ta, tb;
  if (kSym) {
    lower_pair(blockIdx.x, ta, tb);
  } else {
    ta = blockIdx.x / tiles_per_dim;
    tb = blockIdx.x % tiles_per_dim;
  }
  ta += (ta >= kb) ? 1 : 0;
  tb += (tb >= kb) ? 1 : 0;
  const int r0 = ta * kBlock, c0 = tb * kBlock, k0 = kb * kBlock;
  double* Mb = M + (long long)b * mstride;
  const double* Cb = cold + (long long)b * cstride;
  TileAcc acc;
  tile_gemm_tn(acc, Cb + r0, ld, Mb + (long long)k0 * ld + c0, ld, kBlock, smem);
  // C = M_tile - acc, staged in shared memory for the (mirrored) store
  const int tid = threadIdx.x;
  acc_to_smem(acc, smem, -1.0);
  __syncthreads();
  for (int piece = tid; piece < kBlock * 64; piece += kGemmThreads) {
    const int r = piece >> 6, c = (piece & 63) * 2;
    const double2 m = *reinterpret_cast<const double2*>(Mb + (long long)(r0 + r) * ld + c0 + c);
    smem[r * kStride + c] += m.x;
    smem[r * kStride + c + 1] += m.y;
  }
  __syncthreads();
  store_tile(Mb, ld, r0, c0, smem, kSym);
}

// Scratch per matrix: cold (kBlock x np) + P^-1 and its transpose (2 x kBlock x kBlock).
inline size_t sweep_scratch_doubles(int np) { return size_t(kBlock) * np + size_t(2) * kBlock * kBlock; }

template <bool kSym>
inline cudaError_t sweep_configure_variant() {
  cudaError_t e = cudaFuncSetAttribute(sweep_pivot_kernel<kSym>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPivotSmemBytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(sweep_rowpanel_kernel<kSym>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmemBytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(sweep_update_kernel<kSym>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmemBytes);
}

inline cudaError_t sweep_configure() {
  // per-device attribute: cheap to repeat, so no process-wide cache is kept
  cudaError_t e = sweep_configure_variant<true>();
  if (e != cudaSuccess) return e;
  e = sweep_configure_variant<false>();
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(sweep_colpanel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmemBytes);
}

// Sweep every block of `batch` matrices of padded size np (a multiple of kBlock):
// M <- -M^{-1}.  scratch holds batch * sweep_scratch_doubles(np) doubles.
template <bool kSym>
inline cudaError_t sweep_batched(double* M, long long mstride, int np, int batch, double* scratch, int* status, cudaStream_t stream) {
  cudaError_t e = sweep_configure();
  if (e != cudaSuccess) return e;
  const int nt = np / kBlock;
  const long long cstride = (long long)kBlock * np;
  double* cold = scratch;
  double* pinv = scratch + (long long)batch * cstride;
  for (int kb = 0; kb < nt; ++kb) {
    sweep_pivot_kernel<kSym><<<batch, kPivotThreads, kPivotSmemBytes, stream>>>(M, mstride, np, kb * kBlock, pinv, status);
    if (nt > 1) {
      const int t = nt - 1;
      sweep_rowpanel_kernel<kSym><<<dim3(t, batch), kGemmThreads, kTileSmemBytes, stream>>>(M, mstride, np, kb, pinv, cold, cstride);
      if (!kSym) sweep_colpanel_kernel<<<dim3(t, batch), kGemmThreads, kTileSmemBytes, stream>>>(M, mstride, np, kb, pinv, cold, cstride);
      const int tiles = kSym ? t * (t + 1) / 2 : t * t;
      sweep_update_kernel<kSym><<<dim3(tiles, batch), kGemmThreads, kTileSmemBytes, stream>>>(M, mstride, np, kb, cold, cstride, t);
    }
  }
  return cudaGetLastError();
}

inline cudaError_t sweep_sym(double* M, long long mstride, int np, int batch, double* scratch, int* status, cudaStream_t stream) {
  return sweep_batched<true>(M, mstride, np, batch, scratch, status, stream);
}
inline cudaError_t sweep_general(double* M, long long mstride, int np, int batch, double* scratch, int* status, cudaStream_t stream) {
  return sweep_batched<false>(M, mstride, np, batch, scratch, status, stream);
}

}  // namespace ticc
