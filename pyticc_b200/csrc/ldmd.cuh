// LDMD log-derivative propagation (two half-steps per sector, diagonal reference
// potential at the sector midpoint), batched over energies, driven sector by sector.
//
// Per sector s with half-step h, ref = diag(W_mid), p^2 = ref - 2 mu E:
//   y1 = p coth(ph) | |p| cot(|p|h),  y2 = p csch(ph) | |p| csc(|p|h)   (series if |ph| < 1e-5)
//   Q_start = h (W_start - diag ref)/3,  Q_end = h (W_end - diag ref)/3,
//   Q_mid = (4/h) [(I - h^2 (W_mid - diag ref)/6)^{-1} - I]        (energy independent)
//   Y_mid = Q_mid + y1 - y2 (Y + Q_start + y1)^{-1} y2
//   Y_end = Q_end + y1 - y2 (Y_mid + Q_mid + y1)^{-1} y2
// The sweep returns S = -A^{-1}, so "- y2 A^{-1} y2" is "+ y2 S y2": every step
// between two inversions is one fused elementwise pass over the work matrices.
//
// Several channel blocks of one size (the K blocks of a coupled-states or NNCC system,
// padded to a common n) propagate together: the batch is (block g, energy e) with
// b = g * n_energy + e, block g reads its W at offset g * wb_stride, and Q_mid is one
// energy-shared matrix per (sector, block).
#pragma once

#include "sweep.cuh"
#include "ticc_common.cuh"

namespace ticc {

struct LdmdSectors {
  const double* h;        // [n_sector] half-steps (device)
  const double* Ws;       // W_base at sector starts, sector stride ws_stride, row stride n
  const double* Wm;
  const double* We;
  long long ws_stride, wm_stride, we_stride;
  int n_sector;
  long long wb_stride;    // offset between the W of consecutive channel blocks (0: one block)
};

struct LdmdLayout {
  int n;          // logical channels
  int n_energy;
  int n_block;    // channel blocks; the batch of work matrices is n_block * n_energy
  int is_complex;
  int np;         // padded sweep size of the per-energy work matrix
  int npr;        // padded sweep size of the real, energy-shared Q_mid matrix
  double* M;      // [n_block * n_energy][np][np]
  double* Qm;     // [n_sector][n_block][npr][npr]
  double* y1;     // [n_sector][n_block * n_energy][n]
  double* y2;
  double* scratch;
  size_t scratch_doubles;
  int* reduced;   // [n_sector] leading sweep blocks taken in TF32x3 (mixed mode), else null
  float* split;   // FP32 operand panels of the reduced steps' tcgen05 update (mixed mode), else null
};

// Mixed precision: a channel whose local wavenumber at the sector midpoint exceeds this
// (for the highest energy of the batch, p^2 = W_mid,ii - 2 mu E_max > kappa^2) is closed
// strongly enough that the FP32-level error of its block's trailing update decays before
// it reaches the open channels.  30 bohr^-1 keeps max|dS| ~1e-8 in the tested systems.
constexpr double kMixedKappa = 30.0;

inline int ldmd_np(int n, int is_complex) { return (int)round_up((long long)(is_complex ? 2 * n : n), kBlock); }

__device__ __forceinline__ void reference_pair(double h, double p2, double& y1, double& y2) {
  const double mag = sqrt(fabs(p2));
  const double arg = mag * h;
  if (fabs(arg) < 1.0e-5) {
    y1 = 1.0 / h + p2 * h / 3.0 - p2 * p2 * h * h * h / 45.0;
    y2 = 1.0 / h - p2 * h / 6.0 + 7.0 * p2 * p2 * h * h * h / 360.0;
  } else if (p2 >= 0.0) {
    y1 = mag / tanh(arg);
    y2 = mag / sinh(arg);
  } else {
    y1 = mag / tan(arg);
    y2 = mag / sin(arg);
  }
}

// y1/y2 for every (sector, block, energy, channel).
__global__ void ldmd_reference_kernel(LdmdSectors sec, const double* energies, double mu, int n, int n_energy, int n_block, double* y1, double* y2) {
  const long long total = (long long)sec.n_sector * n_block * n_energy * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n);
    const long long sb = idx / n;
    const int e = (int)(sb % n_energy);
    const long long sg = sb / n_energy;
    const int g = (int)(sg % n_block);
    const int s = (int)(sg / n_block);
    const double ref = sec.Wm[s * sec.wm_stride + g * sec.wb_stride + (long long)i * n + i];
    double a, b;
    reference_pair(sec.h[s], ref - 2.0 * mu * energies[e], a, b);
    y1[idx] = a;
    y2[idx] = b;
  }
}

__device__ __forceinline__ double sym(const double* W, int n, int i, int j) { return 0.5 * (W[(long long)i * n + j] + W[(long long)j * n + i]); }

// Number of leading 128-blocks of the (closed-first ordered) work matrix whose channels
// are all closed beyond kMixedKappa at the highest energy, in every channel block; one CTA
// per sector.
__global__ void ldmd_reduced_blocks_kernel(LdmdSectors sec, const double* energies, double mu, int n, int n_energy, int n_block, int np, int is_complex, int* reduced) {
  __shared__ double e_max;
  __shared__ int first_open;
  const int s = blockIdx.x;
  if (threadIdx.x == 0) {
    double m = energies[0];
    for (int e = 1; e < n_energy; ++e) m = fmax(m, energies[e]);
    e_max = m;
    first_open = n;
  }
  __syncthreads();
  for (int g = 0; g < n_block; ++g) {
    const double* Wm = sec.Wm + s * sec.wm_stride + g * sec.wb_stride;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const double p2 = Wm[(long long)i * n + i] - 2.0 * mu * e_max;
      if (!(p2 > kMixedKappa * kMixedKappa)) atomicMin(&first_open, i);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int rows = (first_open == n) ? np : first_open * (is_complex ? 2 : 1);
    reduced[s] = rows / kBlock;
  }
}

// Mq = I - h^2 (W_mid - diag ref)/6 (padded identity), batched over (sector, block):
// blockIdx.y = s * n_block + g.
__global__ void ldmd_qmid_build_kernel(LdmdSectors sec, int n, int n_block, int npr, double* Qm) {
  const int sg = blockIdx.y;
  const int s = sg / n_block, g = sg % n_block;
  const double h = sec.h[s];
  const double* Wm = sec.Wm + s * sec.wm_stride + g * sec.wb_stride;
  double* Q = Qm + (long long)sg * npr * npr;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)npr * npr; idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / npr), j = (int)(idx % npr);
    double v;
    if (i < n && j < n) {
      v = (i == j) ? 1.0 : -h * h * sym(Wm, n, i, j) / 6.0;
    } else {
      v = (i == j) ? 1.0 : 0.0;
    }
    Q[idx] = v;
  }
}

// Q_mid = (4/h)(X - I) from the swept matrix -X.
__global__ void ldmd_qmid_finish_kernel(LdmdSectors sec, int n, int n_block, int npr, double* Qm) {
  const int sg = blockIdx.y;
  const double h = sec.h[sg / n_block];
  double* Q = Qm + (long long)sg * npr * npr;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)npr * npr; idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / npr), j = (int)(idx % npr);
    Q[idx] = (i < n && j < n) ? 4.0 / h * (-Q[idx] - (i == j ? 1.0 : 0.0)) : 0.0;
  }
}

// Store one logical element (X + iZ) of a work matrix, or padding.
__device__ __forceinline__ void put_element(double* Mb, int np, int i, int j, double x, double z, int is_complex) {
  if (is_complex) {
    Mb[(long long)(2 * i) * np + 2 * j] = x;
    Mb[(long long)(2 * i) * np + 2 * j + 1] = z;
    Mb[(long long)(2 * i + 1) * np + 2 * j] = z;
    Mb[(long long)(2 * i + 1) * np + 2 * j + 1] = -x;
  } else {
    Mb[(long long)i * np + j] = x;
  }
}

// Read the swept value S = -A^{-1} at logical (i, j): real part S00 and the imaginary
// companion -S01 (so that -A^{-1} = s_re + i s_im).  The symmetric sweep keeps only the
// lower and diagonal 128-tiles current, so an element of an upper tile is read at (j, i).
__device__ __forceinline__ void get_swept(const double* Mb, int np, int i, int j, int is_complex, double& s_re, double& s_im) {
  const int mi = is_complex ? 2 * i : i, mj = is_complex ? 2 * j : j;
  if ((mi >> 7) < (mj >> 7)) {
    const int x = i;
    i = j;
    j = x;
  }
  if (is_complex) {
    s_re = Mb[(long long)(2 * i) * np + 2 * j];
    s_im = -Mb[(long long)(2 * i) * np + 2 * j + 1];
  } else {
    s_re = Mb[(long long)i * np + j];
    s_im = 0.0;
  }
}

// Work-matrix padding: identity on the padded diagonal of the real sweep matrix.
__device__ __forceinline__ void put_padding(double* Mb, int np, long long r, long long c) { Mb[r * np + c] = (r == c) ? 1.0 : 0.0; }

// W_base must be exactly symmetric (the contraction writes both halves from one value), so
// the per-energy passes read W[i][j] only, row-contiguous across the threads of a warp.
// phase 0: A = Y_in + Q_start + y1          (first sector of the call)
// phase 1: A = [Q_end' + y1' + y2' S y2'] + Q_start + y1   (S from the previous sector)
// phase 2: B = 2 Q_mid + 2 y1 + y2 S y2
// phase 3: Y_out = Q_end + y1 + y2 S y2     (last sector of the call)
// One CTA per (logical row i, channel block g) runs over every energy of the block: the
// row's W (or Q_mid) values are read once into registers and reused for all energies, and
// each thread keeps kRowCols columns of loads in flight per energy.  Every quantity is
// symmetric in (i, j) and the sweep reads only the lower and diagonal 128-tiles, so a row
// is processed up to the end of its diagonal tile; the last pass writes Y_out's upper
// triangle as the transpose of the lower tiles.
constexpr int kRowCols = 4;
__global__ void __launch_bounds__(256, 2) ldmd_elementwise_kernel(int phase, int s, LdmdSectors sec, LdmdLayout L, const double* Yin, double* Yout) {
  const int i = blockIdx.x;
  const int g = blockIdx.y;
  const int ne = L.n_energy;
  const int batch = L.n_block * ne;
  const int n = L.n, np = L.np;
  const int nl = L.is_complex ? np / 2 : np;  // logical-element grid covering the padded matrix
  const int mi = L.is_complex ? 2 * i : i;    // work-matrix row of logical row i
  const int tile_end = ((mi >> 7) + 1) << 7;  // end of row i's diagonal 128-tile (work-matrix columns)
  const int jl = L.is_complex ? tile_end / 2 : tile_end;
  const int jlim = jl < nl ? jl : nl;
  if (i >= n) {  // padding row
    if (phase == 3) return;
    for (int e = 0; e < ne; ++e) {
      double* Mb = L.M + (long long)(g * ne + e) * np * np;
      for (int j = threadIdx.x; j < jlim; j += blockDim.x) {
        if (L.is_complex) {
          for (int a = 0; a < 2; ++a)
            for (int c = 0; c < 2; ++c) put_padding(Mb, np, 2LL * i + a, 2LL * j + c);
        } else {
          put_padding(Mb, np, i, j);
        }
      }
    }
    return;
  }
  const double h = sec.h[s];
  const long long wb = g * sec.wb_stride;
  const double* Ws = sec.Ws + s * sec.ws_stride + wb + (long long)i * n;
  const double* Wm = sec.Wm + s * sec.wm_stride + wb;
  const double* We = sec.We + s * sec.we_stride + wb + (long long)i * n;
  const double ref = Wm[(long long)i * n + i];
  double hp = 0.0, ref_p = 0.0;
  const double* Wep = nullptr;
  if (phase == 1) {
    hp = sec.h[s - 1];
    Wep = sec.We + (s - 1) * sec.we_stride + wb + (long long)i * n;
    ref_p = sec.Wm[(s - 1) * sec.wm_stride + wb + (long long)i * n + i];
  }
  const double* Qrow = L.Qm + ((long long)s * L.n_block + g) * L.npr * L.npr + (long long)i * L.npr;
  for (int j0 = 0; j0 < jlim; j0 += kRowCols * 256) {
    // energy-independent row values of this thread's columns
    double wa[kRowCols], wp[kRowCols];
#pragma unroll
    for (int q = 0; q < kRowCols; ++q) {
      const int j = j0 + q * 256 + threadIdx.x;
      wa[q] = wp[q] = 0.0;
      if (j < n) {
        if (phase <= 1) wa[q] = Ws[j];
        else if (phase == 2) wa[q] = Qrow[j];
        else wa[q] = We[j];
        if (phase == 1) wp[q] = Wep[j];
      }
    }
    if (!L.is_complex && (phase == 1 || phase == 2)) {
      // the per-sector passes of a real work matrix: two energies at a time, all loads of
      // both issued before either's stores (the stores of one energy could alias the next
      // energy's loads as far as the compiler knows, so it would not hoist them itself)
#pragma unroll 1
      for (int e = 0; e < ne; e += 2) {
        const int cnt = (ne - e < 2) ? ne - e : 2;
        double sv[2][kRowCols], yv[2][kRowCols], y1i[2], y2i[2];
        double* Mv[2];
        const double* y2row[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int b = g * ne + e + (u < cnt ? u : 0);
          Mv[u] = L.M + (long long)b * np * np;
          const double* y1 = L.y1 + ((long long)(phase == 1 ? s - 1 : s) * batch + b) * n;
          y2row[u] = L.y2 + ((long long)(phase == 1 ? s - 1 : s) * batch + b) * n;
          y1i[u] = y1[i];
          y2i[u] = y2row[u][i];
#pragma unroll
          for (int q = 0; q < kRowCols; ++q) {
            const int j = j0 + q * 256 + threadIdx.x;
            sv[u][q] = yv[u][q] = 0.0;
            if (j < n && j < jlim) {
              sv[u][q] = Mv[u][(long long)i * np + j];
              yv[u][q] = y2row[u][j];
            }
          }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          if (u >= cnt) break;
          const int b = g * ne + e + u;
          const double* y1c = L.y1 + ((long long)s * batch + b) * n;  // this sector's y1 (phase 1)
          const double y1cur = y1c[i];
#pragma unroll
          for (int q = 0; q < kRowCols; ++q) {
            const int j = j0 + q * 256 + threadIdx.x;
            if (j >= jlim) continue;
            if (j >= n) {  // padding column
              put_padding(Mv[u], np, i, j);
              continue;
            }
            const double d = (i == j) ? 1.0 : 0.0;
            double x;
            if (phase == 1) {
              x = hp * (wp[q] - d * ref_p) / 3.0 + d * y1i[u] + y2i[u] * sv[u][q] * yv[u][q];
              x += h * (wa[q] - d * ref) / 3.0 + d * y1cur;
            } else {
              x = 2.0 * wa[q] + 2.0 * d * y1i[u] + y2i[u] * sv[u][q] * yv[u][q];
            }
            Mv[u][(long long)i * np + j] = x;
          }
        }
      }
      continue;
    }
#pragma unroll 1
    for (int e = 0; e < ne; ++e) {
      const int b = g * ne + e;
      double* Mb = L.M + (long long)b * np * np;
      const double* y1 = L.y1 + ((long long)s * batch + b) * n;
      const double* y2 = L.y2 + ((long long)s * batch + b) * n;
      const double y1i = y1[i], y2i = y2[i];
      double y1pi = 0.0, y2pi = 0.0;
      const double* y2p = nullptr;
      if (phase == 1) {
        const double* y1p = L.y1 + ((long long)(s - 1) * batch + b) * n;
        y2p = L.y2 + ((long long)(s - 1) * batch + b) * n;
        y1pi = y1p[i];
        y2pi = y2p[i];
      }
#pragma unroll
      for (int q = 0; q < kRowCols; ++q) {
        const int j = j0 + q * 256 + threadIdx.x;
        if (j >= jlim) continue;
        if (j >= n) {  // padding column
          if (phase == 3) continue;
          if (L.is_complex) {
            for (int a = 0; a < 2; ++a)
              for (int c = 0; c < 2; ++c) put_padding(Mb, np, 2LL * i + a, 2LL * j + c);
          } else {
            put_padding(Mb, np, i, j);
          }
          continue;
        }
        const double d = (i == j) ? 1.0 : 0.0;
        double x = 0.0, z = 0.0;
        if (phase == 0) {
          if (L.is_complex) {
            const double* Yb = Yin + (long long)b * n * n * 2;
            x = 0.5 * (Yb[2 * ((long long)i * n + j)] + Yb[2 * ((long long)j * n + i)]);
            z = 0.5 * (Yb[2 * ((long long)i * n + j) + 1] + Yb[2 * ((long long)j * n + i) + 1]);
          } else {
            const double* Yb = Yin + (long long)b * n * n;
            x = 0.5 * (Yb[(long long)i * n + j] + Yb[(long long)j * n + i]);
          }
        } else if (phase == 1) {
          double sr, si;
          get_swept(Mb, np, i, j, L.is_complex, sr, si);
          x = hp * (wp[q] - d * ref_p) / 3.0 + d * y1pi + y2pi * sr * y2p[j];
          z = y2pi * si * y2p[j];
        }
        if (phase <= 1) {
          x += h * (wa[q] - d * ref) / 3.0 + d * y1i;
          put_element(Mb, np, i, j, x, z, L.is_complex);
        } else if (phase == 2) {
          double sr, si;
          get_swept(Mb, np, i, j, L.is_complex, sr, si);
          x = 2.0 * wa[q] + 2.0 * d * y1i + y2i * sr * y2[j];
          z = y2i * si * y2[j];
          put_element(Mb, np, i, j, x, z, L.is_complex);
        } else {
          double sr, si;
          get_swept(Mb, np, i, j, L.is_complex, sr, si);
          x = h * (wa[q] - d * ref) / 3.0 + d * y1i + y2i * sr * y2[j];
          z = y2i * si * y2[j];
          const bool below = ((L.is_complex ? 2 * j : j) >> 7) < (mi >> 7);  // (i, j) in a strictly lower tile
          if (L.is_complex) {
            Yout[((long long)b * n * n + (long long)i * n + j) * 2] = x;
            Yout[((long long)b * n * n + (long long)i * n + j) * 2 + 1] = z;
            if (below) {
              Yout[((long long)b * n * n + (long long)j * n + i) * 2] = x;
              Yout[((long long)b * n * n + (long long)j * n + i) * 2 + 1] = z;
            }
          } else {
            Yout[(long long)b * n * n + (long long)i * n + j] = x;
            if (below) Yout[(long long)b * n * n + (long long)j * n + i] = x;
          }
        }
      }
    }
  }
}

inline unsigned grid_for(long long work, int threads, unsigned cap = 1u << 16) {
  long long blocks = (work + threads - 1) / threads;
  if (blocks < 1) blocks = 1;
  return (unsigned)(blocks > cap ? cap : blocks);
}

// Q_mid for every (sector, block) of the call (batched sweep, chunked to fit scratch).
inline cudaError_t ldmd_qmid(const LdmdSectors& sec, LdmdLayout& L, int* status, cudaStream_t stream) {
  const long long per = (long long)L.npr * L.npr;
  const int count = sec.n_sector * L.n_block;
  ldmd_qmid_build_kernel<<<dim3(grid_for(per, 256, 4096), count), 256, 0, stream>>>(sec, L.n, L.n_block, L.npr, L.Qm);
  note_launch();
  const int chunk = (int)(L.scratch_doubles / sweep_scratch_doubles(L.npr));
  for (int s0 = 0; s0 < count; s0 += chunk) {
    const int cnt = (count - s0 < chunk) ? count - s0 : chunk;
    cudaError_t e = sweep_sym(L.Qm + (long long)s0 * per, per, L.npr, cnt, L.scratch, status, stream, nullptr, L.n);
    if (e != cudaSuccess) return e;
  }
  ldmd_qmid_finish_kernel<<<dim3(grid_for(per, 256, 4096), count), 256, 0, stream>>>(sec, L.n, L.n_block, L.npr, L.Qm);
  note_launch();
  return cudaGetLastError();
}

// Propagate every (block, energy) through every sector of the call.  Y (device,
// n_block x n_energy x n x n, complex interleaved when is_complex) is read at the first
// sector start and overwritten with the log-derivative at the last sector end.
inline cudaError_t ldmd_propagate(double* Y, const double* energies, double mu, const LdmdSectors& sec, LdmdLayout& L, int* status, cudaStream_t stream) {
  const int batch = L.n_block * L.n_energy;
  ldmd_reference_kernel<<<grid_for((long long)sec.n_sector * batch * L.n, 256), 256, 0, stream>>>(sec, energies, mu, L.n, L.n_energy, L.n_block, L.y1, L.y2);
  note_launch();
  if (L.reduced != nullptr) {
    ldmd_reduced_blocks_kernel<<<sec.n_sector, 256, 0, stream>>>(sec, energies, mu, L.n, L.n_energy, L.n_block, L.np, L.is_complex, L.reduced);
    note_launch();
  }
  cudaError_t err = ldmd_qmid(sec, L, status, stream);
  if (err != cudaSuccess) return err;
  const long long nl = L.is_complex ? L.np / 2 : L.np;
  const dim3 grid((unsigned)nl, L.n_block);
  const long long mstride = (long long)L.np * L.np;
  const int used = L.is_complex ? 2 * L.n : L.n;  // rows of the work matrix beyond these are identity padding
  for (int s = 0; s < sec.n_sector; ++s) {
    ldmd_elementwise_kernel<<<grid, 256, 0, stream>>>(s == 0 ? 0 : 1, s, sec, L, Y, Y);
    note_launch();
    err = sweep_sym(L.M, mstride, L.np, batch, L.scratch, status, stream, L.reduced ? L.reduced + s : nullptr, used, L.split);
    if (err != cudaSuccess) return err;
    ldmd_elementwise_kernel<<<grid, 256, 0, stream>>>(2, s, sec, L, Y, Y);
    note_launch();
    err = sweep_sym(L.M, mstride, L.np, batch, L.scratch, status, stream, L.reduced ? L.reduced + s : nullptr, used, L.split);
    if (err != cudaSuccess) return err;
  }
  ldmd_elementwise_kernel<<<grid, 256, 0, stream>>>(3, sec.n_sector - 1, sec, L, Y, Y);
  note_launch();
  return cudaGetLastError();
}

}  // namespace ticc
