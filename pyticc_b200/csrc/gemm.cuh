// Batched FP64 GEMM C = alpha * A^T B on the DMMA tile core, for padded operands
// (M, N multiples of 128, K a multiple of 32).  A and B are k-major (row k holds
// A^T[k][:] and B[k][:]).  The result is stored as is or transposed.
#pragma once

#include "dmma_tile.cuh"
#include "ticc_common.cuh"

namespace ticc {

struct GemmBatch {
  const double* A;
  long long lda, strideA;
  const double* B;
  long long ldb, strideB;
  double* C;
  long long ldc, strideC;
  int K;
  double alpha;
  int transpose_store;
};

__global__ void __launch_bounds__(kGemmThreads) gemm_tn_kernel(GemmBatch g) {
  extern __shared__ double smem[];
  const int m0 = blockIdx.x * kBlock, n0 = blockIdx.y * kBlock, b = blockIdx.z;
  TileAcc acc;
  tile_gemm_tn(acc, g.A + b * g.strideA + m0, g.lda, g.B + b * g.strideB + n0, g.ldb, g.K, smem);
  acc_to_smem(acc, smem, g.alpha);
  __syncthreads();
  double* C = g.C + b * g.strideC;
  for (int piece = threadIdx.x; piece < kBlock * 64; piece += kGemmThreads) {
    const int r = piece >> 6, c = (piece & 63) * 2;
    double2 v;
    if (g.transpose_store) {
      // destination row n0 + r, columns m0 + c, m0 + c + 1
      v.x = smem[c * kStride + r];
      v.y = smem[(c + 1) * kStride + r];
      *reinterpret_cast<double2*>(C + (long long)(n0 + r) * g.ldc + m0 + c) = v;
    } else {
      v.x = smem[r * kStride + c];
      v.y = smem[r * kStride + c + 1];
      *reinterpret_cast<double2*>(C + (long long)(m0 + r) * g.ldc + n0 + c) = v;
    }
  }
}

inline cudaError_t gemm_tn(const GemmBatch& g, int M, int N, int batch, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(gemm_tn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmemBytes);
  if (e != cudaSuccess) return e;
  gemm_tn_kernel<<<dim3(M / kBlock, N / kBlock, batch), kGemmThreads, kTileSmemBytes, stream>>>(g);
  note_launch();
  return cudaGetLastError();
}

// Copy a batch of n x n matrices (complex interleaved when is_complex: `part` 0 = real,
// 1 = imaginary plane) into zero-padded np x np planes.
__global__ void pad_plane_kernel(const double* src, int n, int is_complex, int part, double* dst, int np) {
  const int b = blockIdx.y;
  const double* s = src + (long long)b * n * n * (is_complex ? 2 : 1);
  double* d = dst + (long long)b * np * np;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)np * np; idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / np), j = (int)(idx % np);
    double v = 0.0;
    if (i < n && j < n) v = is_complex ? s[2 * ((long long)i * n + j) + part] : s[(long long)i * n + j];
    d[idx] = v;
  }
}

__global__ void unpad_plane_kernel(const double* src, int np, double* dst, int n, int is_complex, int part) {
  const int b = blockIdx.y;
  const double* s = src + (long long)b * np * np;
  double* d = dst + (long long)b * n * n * (is_complex ? 2 : 1);
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)n * n; idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / n), j = (int)(idx % n);
    const double v = s[(long long)i * np + j];
    if (is_complex) {
      d[2 * idx + part] = v;
    } else {
      d[idx] = v;
    }
  }
}

}  // namespace ticc
