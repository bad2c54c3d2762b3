// FP64 tensor-core tile core: one CTA computes a 128x128 tile of A^T B with
// mma.sync m8n8k4 f64 (DMMA), operands staged into shared memory by cp.async.
//
// B200 has no tcgen05 kind for FP64; the FP64 tensor pipe is reached through the
// warp-level DMMA instruction.  A CTA of 8 warps (2 x 4) owns a 128 x 128 tile, each
// warp a 64 x 32 sub-tile held as 8 x 4 DMMA accumulators (64 doubles per lane).
// Operands are "k-major": row k of A holds A^T[k][m0 .. m0+127], which is how every
// caller stores them (the sweep's panels are rows of a symmetric matrix).
#pragma once

#include "ticc_common.cuh"

namespace ticc {

constexpr size_t kTileSmemBytes = size_t(4) * kChunk * kStride * sizeof(double);  // 135168

__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

struct TileAcc {
  double v[8][4][2];
};

// Stage rows [k, k + kC) of a k-major operand (128 contiguous doubles per row).
template <int kC = kChunk>
__device__ __forceinline__ void stage_rows(double* dst, const double* src, long long ld, int k, int tid) {
#pragma unroll
  for (int i = 0; i < (kC * 64) / kGemmThreads; ++i) {
    const int piece = tid + i * kGemmThreads;
    const int r = piece >> 6;
    const int c = (piece & 63) * 2;
    cp_async16(dst + r * kStride + c, src + (long long)(k + r) * ld + c);
  }
}

template <int kC = kChunk>
__device__ __forceinline__ void mma_chunk(TileAcc& acc, const double* As, const double* Bs, int warp, int lane) {
  const int wm = (warp >> 2) * 64;
  const int wn = (warp & 3) * 32;
  const int kr = lane & 3;
  const int mr = lane >> 2;
#pragma unroll
  for (int kk = 0; kk < kC; kk += 4) {
    double a[8], b[4];
    const double* arow = As + (kk + kr) * kStride + wm + mr;
    const double* brow = Bs + (kk + kr) * kStride + wn + mr;
#pragma unroll
    for (int mt = 0; mt < 8; ++mt) a[mt] = arow[mt * 8];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) b[nt] = brow[nt * 8];
#pragma unroll
    for (int mt = 0; mt < 8; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) dmma_8x8x4(acc.v[mt][nt], a[mt], b[nt]);
  }
}

// acc = sum_{k < K} A[k][0..127]^T B[k][0..127]; A, B already offset to their tile column.
// K must be a multiple of kChunk.  Ends with a __syncthreads(), so smem is free afterwards.
__device__ inline void tile_gemm_tn(TileAcc& acc, const double* A, long long lda, const double* B, long long ldb, int K, double* smem) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
#pragma unroll
  for (int mt = 0; mt < 8; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) acc.v[mt][nt][0] = acc.v[mt][nt][1] = 0.0;

  // stage s of the double buffer: A at smem + s * 2 * kChunk * kStride, B right after it
  constexpr int kStage = 2 * kChunk * kStride;
  const int nchunks = K / kChunk;
  stage_rows(smem, A, lda, 0, tid);
  stage_rows(smem + kChunk * kStride, B, ldb, 0, tid);
  cp_async_commit();
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) {
      double* next = smem + ((c + 1) & 1) * kStage;
      stage_rows(next, A, lda, (c + 1) * kChunk, tid);
      stage_rows(next + kChunk * kStride, B, ldb, (c + 1) * kChunk, tid);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* cur = smem + (c & 1) * kStage;
    mma_chunk(acc, cur, cur + kChunk * kStride, warp, lane);
    __syncthreads();
  }
}

// Write the accumulator into a [128][kStride] shared tile: Cs[row][col] = scale * acc.
__device__ __forceinline__ void acc_to_smem(const TileAcc& acc, double* Cs, double scale) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int wm = (warp >> 2) * 64;
  const int wn = (warp & 3) * 32;
#pragma unroll
  for (int mt = 0; mt < 8; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int row = wm + mt * 8 + (lane >> 2);
      const int col = wn + nt * 8 + 2 * (lane & 3);
      Cs[row * kStride + col] = scale * acc.v[mt][nt][0];
      Cs[row * kStride + col + 1] = scale * acc.v[mt][nt][1];
    }
}

// Cs[row][col] = acc and, with `mirror`, the same value straight from registers to the
// transposed position Mt[col * ld + row] (8 lanes of a column write 64 contiguous bytes).
__device__ __forceinline__ void acc_to_smem_mirror(const TileAcc& acc, double* Cs, double* Mt, long long ld, bool mirror) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int wm = (warp >> 2) * 64;
  const int wn = (warp & 3) * 32;
#pragma unroll
  for (int mt = 0; mt < 8; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int row = wm + mt * 8 + (lane >> 2);
      const int col = wn + nt * 8 + 2 * (lane & 3);
      Cs[row * kStride + col] = acc.v[mt][nt][0];
      Cs[row * kStride + col + 1] = acc.v[mt][nt][1];
      if (mirror) {
        Mt[(long long)col * ld + row] = acc.v[mt][nt][0];
        Mt[(long long)(col + 1) * ld + row] = acc.v[mt][nt][1];
      }
    }
}

// ---- FP32-accurate tile product on the TF32 tensor pipe ---------------------------------
// The same staged FP64 operands, split on the fly as x = hi + lo with hi, lo TF32
// (cvt.rna), and D += A_hi B_hi + A_hi B_lo + A_lo B_hi with mma.sync m16n8k8 TF32 and
// FP32 accumulation: ~2^-21 relative per product, about 2.5x the FP64 DMMA rate on B200.
// Warp w owns rows (w/4)*64 .. +63 and cols (w%4)*32 .. +31 as 4 x 4 m16n8 tiles.
struct TileAcc32 {
  float v[4][4][4];
};

__device__ __forceinline__ void split_tf32(double x, unsigned& hi, unsigned& lo) {
  const float f = static_cast<float>(x);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(f));
  const float r = f - __uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int kC = kChunk>
__device__ __forceinline__ void mma_chunk_tf32x3(TileAcc32& acc, const double* As, const double* Bs, int warp, int lane) {
  const int wm = (warp >> 2) * 64;
  const int wn = (warp & 3) * 32;
  const int t = lane & 3;
  const int g = lane >> 2;
#pragma unroll
  for (int kk = 0; kk < kC; kk += 8) {
    unsigned ah[4][4], al[4][4], bh[4][2], bl[4][2];
    const double* a0 = As + (kk + t) * kStride + wm + g;
    const double* a4 = As + (kk + t + 4) * kStride + wm + g;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
      split_tf32(a0[mt * 16], ah[mt][0], al[mt][0]);
      split_tf32(a0[mt * 16 + 8], ah[mt][1], al[mt][1]);
      split_tf32(a4[mt * 16], ah[mt][2], al[mt][2]);
      split_tf32(a4[mt * 16 + 8], ah[mt][3], al[mt][3]);
    }
    const double* b0 = Bs + (kk + t) * kStride + wn + g;
    const double* b4 = Bs + (kk + t + 4) * kStride + wn + g;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      split_tf32(b0[nt * 8], bh[nt][0], bl[nt][0]);
      split_tf32(b4[nt * 8], bh[nt][1], bl[nt][1]);
    }
    // each term across the 16 accumulators before the next, so that consecutive mma are
    // independent; every accumulator still takes lo*hi, hi*lo, hi*hi in that order
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) mma_tf32(acc.v[mt][nt], al[mt], bh[nt][0], bh[nt][1]);
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) mma_tf32(acc.v[mt][nt], ah[mt], bl[nt][0], bl[nt][1]);
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) mma_tf32(acc.v[mt][nt], ah[mt], bh[nt][0], bh[nt][1]);
  }
}

// acc = sum_{k < K} A[k][0..127]^T B[k][0..127] in FP32-accurate TF32x3; same staging and
// contract as tile_gemm_tn.
__device__ inline void tile_gemm_tn_tf32x3(TileAcc32& acc, const double* A, long long lda, const double* B, long long ldb, int K, double* smem) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc.v[mt][nt][q] = 0.0f;
  constexpr int kStage = 2 * kChunk * kStride;
  const int nchunks = K / kChunk;
  stage_rows(smem, A, lda, 0, tid);
  stage_rows(smem + kChunk * kStride, B, ldb, 0, tid);
  cp_async_commit();
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) {
      double* next = smem + ((c + 1) & 1) * kStage;
      stage_rows(next, A, lda, (c + 1) * kChunk, tid);
      stage_rows(next + kChunk * kStride, B, ldb, (c + 1) * kChunk, tid);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* cur = smem + (c & 1) * kStage;
    mma_chunk_tf32x3(acc, cur, cur + kChunk * kStride, warp, lane);
    __syncthreads();
  }
}

// acc32 into a [128][kStride] shared tile and, with `mirror`, its transpose to Mt (row
// stride ld) straight from registers, as acc_to_smem_mirror.
__device__ __forceinline__ void acc32_to_smem_mirror(const TileAcc32& acc, double* Cs, double* Mt, long long ld, bool mirror) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int wm = (warp >> 2) * 64;
  const int wn = (warp & 3) * 32;
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = wm + mt * 16 + g + 8 * h, col = wn + nt * 8 + 2 * t;
        const double v0 = acc.v[mt][nt][2 * h], v1 = acc.v[mt][nt][2 * h + 1];
        Cs[row * kStride + col] = v0;
        Cs[row * kStride + col + 1] = v1;
        if (mirror) {
          Mt[(long long)col * ld + row] = v0;
          Mt[(long long)(col + 1) * ld + row] = v1;
        }
      }
}

// ---- trailing-update tile with the C tile staged during the product ----------------------
// The update M_tile -= A^T B of the sweep reads the 128 x 128 FP64 tile of M once; here it
// is copied into shared memory by cp.async while the first K-chunk is multiplied, so the
// epilogue is an in-place shared-memory subtraction instead of a global read after the
// product.  K-chunks of kUpdChunk rows keep both staging buffers and the C tile resident:
//   [ A/B stages: 2 x 2 x kUpdChunk x kStride ][ C tile: 128 x kStride ]   (doubles)
constexpr int kUpdChunk = 16;
// TF32x3 operands split once while staging: per stage A_hi, A_lo, B_hi, B_lo as 32-bit words,
// kUpdChunk rows of kSplitLd words (136 = 8 mod 32: conflict-free tf32 fragment loads)
constexpr int kSplitLd = kBlock + 8;
constexpr int kSplitArray = kUpdChunk * kSplitLd;
constexpr int kSplitStageWords = 4 * kSplitArray;
constexpr int kUpdStageDoubles64 = 2 * 2 * kUpdChunk * kStride;  // FP64 stages: 8448 doubles
constexpr int kUpdStageDoubles = kUpdStageDoubles64 > kSplitStageWords ? kUpdStageDoubles64 : kSplitStageWords;  // 2 split stages = 8704 doubles
constexpr size_t kUpdTileSmemBytes = (size_t(kUpdStageDoubles) + size_t(kBlock) * kStride) * sizeof(double);  // 204800

__device__ __forceinline__ void mma_chunk_any(TileAcc& acc, const double* As, const double* Bs, int warp, int lane) { mma_chunk<kUpdChunk>(acc, As, Bs, warp, lane); }
__device__ __forceinline__ void mma_chunk_any(TileAcc32& acc, const double* As, const double* Bs, int warp, int lane) { mma_chunk_tf32x3<kUpdChunk>(acc, As, Bs, warp, lane); }
__device__ __forceinline__ void acc_zero(TileAcc& acc) {
#pragma unroll
  for (int mt = 0; mt < 8; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) acc.v[mt][nt][0] = acc.v[mt][nt][1] = 0.0;
}
__device__ __forceinline__ void acc_zero(TileAcc32& acc) {
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc.v[mt][nt][q] = 0.0f;
}

// The product is split so that a persistent CTA can start the next tile's loads early:
// issue_update_chunk0 and issue_update_ctile each commit one cp.async group, and
// update_mainloop expects exactly that order of groups in flight (chunk 0, C tile) and
// then commits chunks 1 .. K/kUpdChunk - 1 itself.
__device__ __forceinline__ void issue_update_chunk0(const double* A, long long lda, const double* B, long long ldb, double* stages) {
  const int tid = threadIdx.x;
  stage_rows<kUpdChunk>(stages, A, lda, 0, tid);
  stage_rows<kUpdChunk>(stages + kUpdChunk * kStride, B, ldb, 0, tid);
  cp_async_commit();
}
__device__ __forceinline__ void issue_update_ctile(double* Cs, const double* Cg, long long ldc) {
  const int tid = threadIdx.x;
#pragma unroll 4
  for (int i = 0; i < (kBlock * 64) / kGemmThreads; ++i) {
    const int piece = tid + i * kGemmThreads;
    cp_async16(Cs + (piece >> 6) * kStride + (piece & 63) * 2, Cg + (long long)(piece >> 6) * ldc + (piece & 63) * 2);
  }
  cp_async_commit();
}

// acc = sum_{k < K} A[k][.]^T B[k][.] (K a multiple of kUpdChunk, at least 2 chunks), with
// chunk 0 and the C tile already issued.  On return Cs holds C and the staging region is
// free (ends with a __syncthreads()).
template <class Acc>
__device__ inline void update_mainloop(Acc& acc, const double* A, long long lda, const double* B, long long ldb, int K, double* stages) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  acc_zero(acc);
  constexpr int kStage = 2 * kUpdChunk * kStride;
  const int nchunks = K / kUpdChunk;
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) {
      double* next = stages + ((c + 1) & 1) * kStage;
      stage_rows<kUpdChunk>(next, A, lda, (c + 1) * kUpdChunk, tid);
      stage_rows<kUpdChunk>(next + kUpdChunk * kStride, B, ldb, (c + 1) * kUpdChunk, tid);
      cp_async_commit();
    }
    // groups newer than chunk c that may stay in flight: c = 0 -> C tile and chunk 1;
    // later -> chunk c + 1 only; the last chunk waits for everything
    if (c + 1 >= nchunks) {
      cp_async_wait<0>();
    } else if (c == 0) {
      cp_async_wait<2>();
    } else {
      cp_async_wait<1>();
    }
    __syncthreads();
    const double* cur = stages + (c & 1) * kStage;
    mma_chunk_any(acc, cur, cur + kUpdChunk * kStride, warp, lane);
    __syncthreads();
  }
}

// The whole product in one call: Cs <- C tile while acc = A^T B.
template <class Acc>
__device__ inline void tile_update_product(Acc& acc, const double* A, long long lda, const double* B, long long ldb, int K, double* stages, double* Cs, const double* Cg, long long ldc) {
  issue_update_chunk0(A, lda, B, ldb, stages);
  issue_update_ctile(Cs, Cg, ldc);
  update_mainloop(acc, A, lda, B, ldb, K, stages);
}

// Cs[row][col] -= acc in the accumulator's own fragment layout (the pivot tile of a fused
// next-pivot update, inverted in shared memory afterwards).
__device__ __forceinline__ void acc_sub_smem(const TileAcc& acc, double* Cs) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int wm = (warp >> 2) * 64;
  const int wn = (warp & 3) * 32;
#pragma unroll
  for (int mt = 0; mt < 8; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int row = wm + mt * 8 + (lane >> 2), col = wn + nt * 8 + 2 * (lane & 3);
      double* d = Cs + row * kStride + col;
      d[0] -= acc.v[mt][nt][0];
      d[1] -= acc.v[mt][nt][1];
    }
}
__device__ __forceinline__ void acc_sub_smem(const TileAcc32& acc, double* Cs) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int wm = (warp >> 2) * 64;
  const int wn = (warp & 3) * 32;
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = wm + mt * 16 + g + 8 * h, col = wn + nt * 8 + 2 * t;
        double* d = Cs + row * kStride + col;
        d[0] -= acc.v[mt][nt][2 * h];
        d[1] -= acc.v[mt][nt][2 * h + 1];
      }
}

// Epilogue written straight from the accumulator registers: M[r0 + row][c0 + col] = C - acc
// with C from the staged tile Cs (a double2 per lane pair of columns).  The symmetric sweep
// keeps only the lower and diagonal 128-tiles current, so an off-diagonal tile writes no
// transpose; a diagonal tile writes each lower-half value (row >= col) to both of its
// positions, so the tile stays exactly symmetric.  Cs is only read.
__device__ __forceinline__ void put_updated(double* Mb, long long ld, int r0, int c0, int row, int col, double v0, double v1, bool sym) {
  if (!sym || r0 != c0) {
    *reinterpret_cast<double2*>(Mb + (long long)(r0 + row) * ld + c0 + col) = make_double2(v0, v1);
  } else {
    if (row >= col) {
      Mb[(long long)(r0 + row) * ld + c0 + col] = v0;
      Mb[(long long)(c0 + col) * ld + r0 + row] = v0;
    }
    if (row >= col + 1) {
      Mb[(long long)(r0 + row) * ld + c0 + col + 1] = v1;
      Mb[(long long)(c0 + col + 1) * ld + r0 + row] = v1;
    }
  }
}
__device__ __forceinline__ void acc_epilogue_direct(const TileAcc& acc, const double* Cs, double* Mb, long long ld, int r0, int c0, bool sym) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int wm = (warp >> 2) * 64;
  const int wn = (warp & 3) * 32;
#pragma unroll
  for (int mt = 0; mt < 8; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int row = wm + mt * 8 + (lane >> 2), col = wn + nt * 8 + 2 * (lane & 3);
      const double2 c = *reinterpret_cast<const double2*>(Cs + row * kStride + col);
      put_updated(Mb, ld, r0, c0, row, col, c.x - acc.v[mt][nt][0], c.y - acc.v[mt][nt][1], sym);
    }
}
__device__ __forceinline__ void acc_epilogue_direct(const TileAcc32& acc, const double* Cs, double* Mb, long long ld, int r0, int c0, bool sym) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int wm = (warp >> 2) * 64;
  const int wn = (warp & 3) * 32;
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = wm + mt * 16 + g + 8 * h, col = wn + nt * 8 + 2 * t;
        const double2 c = *reinterpret_cast<const double2*>(Cs + row * kStride + col);
        put_updated(Mb, ld, r0, c0, row, col, c.x - (double)acc.v[mt][nt][2 * h], c.y - (double)acc.v[mt][nt][2 * h + 1], sym);
      }
}

// ---- TF32x3 trailing update with the split done once per CTA while staging ---------------
// Chunk c + 1 of A (cold rows) and B (U rows) is loaded into registers while chunk c is
// multiplied, then split into hi/lo TF32 words in the other stage: every operand value is
// split once per tile instead of once per warp that reads it, and the inner loop is only
// 32-bit shared loads and mma.sync.  Same split and product order as mma_chunk_tf32x3.
struct SplitChunk {
  double2 a[4], b[4];  // this thread's 8 of the chunk's 2 x 16 x 64 double2 pieces
};

__device__ __forceinline__ void load_split_chunk(SplitChunk& r, const double* A, long long lda, const double* B, long long ldb, int k_row0) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int piece = tid + i * kGemmThreads;
    const long long off_a = (long long)(k_row0 + (piece >> 6)) * lda + (piece & 63) * 2;
    const long long off_b = (long long)(k_row0 + (piece >> 6)) * ldb + (piece & 63) * 2;
    r.a[i] = __ldcg(reinterpret_cast<const double2*>(A + off_a));  // L2: written by other CTAs of a fused step
    r.b[i] = __ldcg(reinterpret_cast<const double2*>(B + off_b));
  }
}

__device__ __forceinline__ void store_split_chunk(const SplitChunk& r, unsigned* stage) {
  const int tid = threadIdx.x;
  unsigned* Ahi = stage;
  unsigned* Alo = stage + kSplitArray;
  unsigned* Bhi = stage + 2 * kSplitArray;
  unsigned* Blo = stage + 3 * kSplitArray;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int piece = tid + i * kGemmThreads;
    const int at = (piece >> 6) * kSplitLd + (piece & 63) * 2;
    unsigned h0, l0, h1, l1;
    split_tf32(r.a[i].x, h0, l0);
    split_tf32(r.a[i].y, h1, l1);
    *reinterpret_cast<uint2*>(Ahi + at) = make_uint2(h0, h1);
    *reinterpret_cast<uint2*>(Alo + at) = make_uint2(l0, l1);
    split_tf32(r.b[i].x, h0, l0);
    split_tf32(r.b[i].y, h1, l1);
    *reinterpret_cast<uint2*>(Bhi + at) = make_uint2(h0, h1);
    *reinterpret_cast<uint2*>(Blo + at) = make_uint2(l0, l1);
  }
}

__device__ __forceinline__ void mma_chunk_split(TileAcc32& acc, const unsigned* stage, int warp, int lane) {
  const unsigned* Ahi = stage;
  const unsigned* Alo = stage + kSplitArray;
  const unsigned* Bhi = stage + 2 * kSplitArray;
  const unsigned* Blo = stage + 3 * kSplitArray;
  const int wm = (warp >> 2) * 64;
  const int wn = (warp & 3) * 32;
  const int t = lane & 3;
  const int g = lane >> 2;
#pragma unroll
  for (int kk = 0; kk < kUpdChunk; kk += 8) {
    unsigned ah[4][4], al[4][4], bh[4][2], bl[4][2];
    const int r0 = (kk + t) * kSplitLd, r4 = (kk + t + 4) * kSplitLd;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
      const int m = wm + mt * 16 + g;
      ah[mt][0] = Ahi[r0 + m];
      ah[mt][1] = Ahi[r0 + m + 8];
      ah[mt][2] = Ahi[r4 + m];
      ah[mt][3] = Ahi[r4 + m + 8];
      al[mt][0] = Alo[r0 + m];
      al[mt][1] = Alo[r0 + m + 8];
      al[mt][2] = Alo[r4 + m];
      al[mt][3] = Alo[r4 + m + 8];
    }
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int n = wn + nt * 8 + g;
      bh[nt][0] = Bhi[r0 + n];
      bh[nt][1] = Bhi[r4 + n];
      bl[nt][0] = Blo[r0 + n];
      bl[nt][1] = Blo[r4 + n];
    }
    // each term across the 16 accumulators before the next, so that consecutive mma are
    // independent; every accumulator still takes lo*hi, hi*lo, hi*hi in that order
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) mma_tf32(acc.v[mt][nt], al[mt], bh[nt][0], bh[nt][1]);
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) mma_tf32(acc.v[mt][nt], ah[mt], bl[nt][0], bl[nt][1]);
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) mma_tf32(acc.v[mt][nt], ah[mt], bh[nt][0], bh[nt][1]);
  }
}

// acc = A^T B over K = kBlock rows with chunk 0 already in `r`; on return `r` is free, the
// stages are free (ends with a __syncthreads()) and the C tile's cp.async group is untouched.
__device__ inline void split_mainloop(TileAcc32& acc, SplitChunk& r, const double* A, long long lda, const double* B, long long ldb, unsigned* stages) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  constexpr int nchunks = kBlock / kUpdChunk;
  acc_zero(acc);
  store_split_chunk(r, stages);
  __syncthreads();
#pragma unroll 1
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) load_split_chunk(r, A, lda, B, ldb, (c + 1) * kUpdChunk);
    mma_chunk_split(acc, stages + (c & 1) * kSplitStageWords, warp, lane);
    if (c + 1 < nchunks) store_split_chunk(r, stages + ((c + 1) & 1) * kSplitStageWords);
    __syncthreads();
  }
}

}  // namespace ticc
