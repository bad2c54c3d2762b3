// extern "C" entry points of libticc_b200.so (declared in include/ticc_b200.h).
//
// Each entry validates its arguments on the host, carves the caller's workspace into
// 256-byte aligned regions, enqueues the kernels on the caller's stream and returns a
// status code; the message of the last failure is kept per host thread.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/ticc_b200.h"
#include "contract.cuh"
#include "gemm.cuh"
#include "learned.cuh"
#include "ldmd.cuh"
#include "match.cuh"
#include "pes.cuh"
#include "sweep.cuh"
#include "tc_update.cuh"

namespace {

thread_local char g_message[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list args;
  va_start(args, fmt);
  vsnprintf(g_message, sizeof(g_message), fmt, args);
  va_end(args);
  return code;
}

int cuda_fail(cudaError_t e, const char* where) { return fail(TICC_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e)); }

// Bump allocator over the caller's workspace (256-byte aligned regions).
struct Carver {
  char* base;
  size_t used = 0;
  template <class T>
  T* take(size_t count) {
    used = (used + 255) & ~size_t(255);
    T* p = base ? reinterpret_cast<T*>(base + used) : nullptr;
    used += count * sizeof(T);
    return p;
  }
};

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

size_t ldmd_layout(ticc::LdmdLayout& L, int n, int n_energy, int n_block, int n_sector, int is_complex, int precision, char* base) {
  Carver c{base};
  const size_t batch = (size_t)n_block * n_energy;
  L.n = n;
  L.n_energy = n_energy;
  L.n_block = n_block;
  L.is_complex = is_complex;
  L.np = ticc::ldmd_np(n, is_complex);
  L.npr = ticc::ldmd_np(n, 0);
  L.M = c.take<double>(batch * L.np * L.np);
  L.Qm = c.take<double>((size_t)n_sector * n_block * L.npr * L.npr);
  L.y1 = c.take<double>((size_t)n_sector * batch * n);
  L.y2 = c.take<double>((size_t)n_sector * batch * n);
  // one scratch region serves the per-energy sweeps and the per-sector Q_mid sweeps
  // (the latter are chunked to fit); at least one sector's worth is guaranteed
  const size_t need_e = batch * ticc::sweep_scratch_doubles(L.np);
  const size_t need_s = ticc::sweep_scratch_doubles(L.npr) * (size_t)(n_sector < 8 ? n_sector : 8);
  L.scratch_doubles = need_e > need_s ? need_e : need_s;
  L.scratch = c.take<double>(L.scratch_doubles);
  L.reduced = (precision == TICC_PRECISION_MIXED) ? c.take<int>((size_t)n_sector) : nullptr;
  L.split = (precision == TICC_PRECISION_MIXED) ? c.take<float>(ticc::tc_split_floats(L.np, (int)batch)) : nullptr;
  if (base == nullptr) L.reduced = nullptr, L.split = nullptr;
  return c.used + 256;
}

size_t match_layout(ticc::MatchLayout& L, int n, int n_energy, int is_complex, int max_open, char* base) {
  Carver c{base};
  L.n = n;
  L.n_energy = n_energy;
  L.is_complex = is_complex;
  L.max_open = max_open;
  L.npz = ticc::ldmd_np(n, is_complex);
  L.npa = (int)ticc::round_up(2LL * (max_open > 0 ? max_open : 1), ticc::kBlock);
  L.Jv = c.take<double>((size_t)n_energy * n);
  L.Nv = c.take<double>((size_t)n_energy * n);
  L.Jp = c.take<double>((size_t)n_energy * n);
  L.Np = c.take<double>((size_t)n_energy * n);
  L.gamma = c.take<double>((size_t)n_energy * n);
  L.oidx = c.take<int>((size_t)n_energy * n);
  L.Z = c.take<double>((size_t)n_energy * L.npz * L.npz);
  L.A = c.take<double>((size_t)n_energy * L.npa * L.npa);
  L.B = c.take<double>((size_t)n_energy * L.npa * L.npa);
  L.C = c.take<double>((size_t)n_energy * L.npa * L.npa);
  const int np = L.npz > L.npa ? L.npz : L.npa;
  L.scratch = c.take<double>((size_t)n_energy * ticc::sweep_scratch_doubles(np));
  return c.used + 256;
}

}  // namespace

extern "C" {

int ticc_version(void) { return 10000; }

long long ticc_kernel_launches(void) { return ticc::launch_counter().load(); }

int ticc_last_error(char* buf, size_t len) {
  const size_t n = strlen(g_message);
  if (buf && len) {
    strncpy(buf, g_message, len - 1);
    buf[len - 1] = '\0';
  }
  return (int)n;
}

// ---- symmetric inversion ---------------------------------------------------------------
static size_t sym_layout(int n, int batch, int is_complex, double** M, double** scratch, char* base) {
  Carver c{base};
  const int np = ticc::ldmd_np(n, is_complex);
  *M = c.take<double>((size_t)batch * np * np);
  *scratch = c.take<double>((size_t)batch * ticc::sweep_scratch_doubles(np));
  return c.used + 256;
}

int ticc_sym_inverse_workspace_size(int n, int batch, int is_complex, size_t* bytes) {
  if (n < 1 || batch < 1 || bytes == nullptr) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_sym_inverse_workspace_size: n=%d batch=%d", n, batch);
  double *M, *s;
  *bytes = sym_layout(n, batch, is_complex, &M, &s, nullptr);
  return TICC_OK;
}

__global__ void sym_load_kernel(const double* src, int n, int is_complex, double* M, int np) {
  const int b = blockIdx.y;
  const int nl = is_complex ? np / 2 : np;
  double* Mb = M + (long long)b * np * np;
  const double* s = src + (long long)b * n * n * (is_complex ? 2 : 1);
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)nl * nl; idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / nl), j = (int)(idx % nl);
    if (i >= n || j >= n) {
      if (is_complex) {
        for (int a = 0; a < 2; ++a)
          for (int c = 0; c < 2; ++c) ticc::put_padding(Mb, np, 2LL * i + a, 2LL * j + c);
      } else {
        ticc::put_padding(Mb, np, i, j);
      }
      continue;
    }
    double x, z = 0.0;
    if (is_complex) {
      x = 0.5 * (s[2 * ((long long)i * n + j)] + s[2 * ((long long)j * n + i)]);
      z = 0.5 * (s[2 * ((long long)i * n + j) + 1] + s[2 * ((long long)j * n + i) + 1]);
    } else {
      x = 0.5 * (s[(long long)i * n + j] + s[(long long)j * n + i]);
    }
    ticc::put_element(Mb, np, i, j, x, z, is_complex);
  }
}

__global__ void sym_store_kernel(const double* M, int np, double* dst, int n, int is_complex) {
  const int b = blockIdx.y;
  const double* Mb = M + (long long)b * np * np;
  double* d = dst + (long long)b * n * n * (is_complex ? 2 : 1);
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)n * n; idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / n), j = (int)(idx % n);
    double sr, si;
    ticc::get_swept(Mb, np, i, j, is_complex, sr, si);
    if (is_complex) {
      d[2 * idx] = -sr;
      d[2 * idx + 1] = -si;
    } else {
      d[idx] = -sr;
    }
  }
}

int ticc_sym_inverse(void* M, int n, int batch, int is_complex, void* workspace, size_t workspace_bytes, int* device_status, void* stream) {
  if (M == nullptr || n < 1 || batch < 1) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_sym_inverse: M=%p n=%d batch=%d", M, n, batch);
  double *Mw, *scratch;
  const size_t need = sym_layout(n, batch, is_complex, &Mw, &scratch, nullptr);
  if (workspace == nullptr || workspace_bytes < need) return fail(TICC_ERR_WORKSPACE, "ticc_sym_inverse: workspace of %zu bytes given, %zu needed", workspace_bytes, need);
  sym_layout(n, batch, is_complex, &Mw, &scratch, static_cast<char*>(workspace));
  const int np = ticc::ldmd_np(n, is_complex);
  const long long nl = is_complex ? np / 2 : np;
  cudaStream_t s = as_stream(stream);
  sym_load_kernel<<<dim3(ticc::grid_for(nl * nl, 256, 8192), batch), 256, 0, s>>>(static_cast<double*>(M), n, is_complex, Mw, np);
  ticc::note_launch();
  cudaError_t e = ticc::sweep_sym(Mw, (long long)np * np, np, batch, scratch, device_status, s, nullptr, is_complex ? 2 * n : n);
  if (e != cudaSuccess) return cuda_fail(e, "ticc_sym_inverse");
  sym_store_kernel<<<dim3(ticc::grid_for((long long)n * n, 256, 8192), batch), 256, 0, s>>>(Mw, np, static_cast<double*>(M), n, is_complex);
  ticc::note_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_sym_inverse");
}

// ---- LDMD propagation ----------------------------------------------------------------------
static int ldmd_check_sizes(const char* who, int n_channel, int n_energy, int n_block, int n_sector, int precision) {
  if (n_channel < 1 || n_energy < 1 || n_block < 1 || n_sector < 1)
    return fail(TICC_ERR_INVALID_ARGUMENT, "%s: n_channel=%d n_energy=%d n_block=%d n_sector=%d must be positive", who, n_channel, n_energy, n_block, n_sector);
  if ((long long)n_block * n_energy > 65535 || (long long)n_block * n_sector > 65535)
    return fail(TICC_ERR_INVALID_ARGUMENT, "%s: n_block*n_energy=%lld and n_block*n_sector=%lld must not exceed 65535 per call", who, (long long)n_block * n_energy,
                (long long)n_block * n_sector);
  if (precision != TICC_PRECISION_FP64 && precision != TICC_PRECISION_MIXED) return fail(TICC_ERR_UNSUPPORTED, "%s: precision mode %d is not available", who, precision);
  return TICC_OK;
}

static int ldmd_run(const char* who, void* Y, int is_complex, const double* energies, int n_energy, double reduced_mass, const double* half_steps,
                    const double* W_start, long long W_start_stride, const double* W_mid, long long W_mid_stride, const double* W_end, long long W_end_stride,
                    long long W_block_stride, int n_sector, int n_channel, int n_block, int precision, void* workspace, size_t workspace_bytes, int* device_status,
                    void* stream) {
  if (Y == nullptr || energies == nullptr || half_steps == nullptr || W_start == nullptr || W_mid == nullptr || W_end == nullptr)
    return fail(TICC_ERR_INVALID_ARGUMENT, "%s: null input pointer", who);
  const int rc = ldmd_check_sizes(who, n_channel, n_energy, n_block, n_sector, precision);
  if (rc != TICC_OK) return rc;
  if (!(reduced_mass > 0.0)) return fail(TICC_ERR_INVALID_ARGUMENT, "%s: reduced_mass must be positive, got %g", who, reduced_mass);
  ticc::LdmdLayout L{};
  const size_t need = ldmd_layout(L, n_channel, n_energy, n_block, n_sector, is_complex, precision, nullptr);
  if (workspace == nullptr || workspace_bytes < need) return fail(TICC_ERR_WORKSPACE, "%s: workspace of %zu bytes given, %zu needed", who, workspace_bytes, need);
  ldmd_layout(L, n_channel, n_energy, n_block, n_sector, is_complex, precision, static_cast<char*>(workspace));
  ticc::LdmdSectors sec{half_steps, W_start, W_mid, W_end, W_start_stride, W_mid_stride, W_end_stride, n_sector, W_block_stride};
  cudaError_t e = ticc::ldmd_propagate(static_cast<double*>(Y), energies, reduced_mass, sec, L, device_status, as_stream(stream));
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, who);
}

int ticc_ldmd_workspace_size(int n_channel, int n_energy, int n_sector, int is_complex, int precision, size_t* bytes) {
  if (bytes == nullptr) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_ldmd_workspace_size: null output pointer");
  const int rc = ldmd_check_sizes("ticc_ldmd_workspace_size", n_channel, n_energy, 1, n_sector, precision);
  if (rc != TICC_OK) return rc;
  ticc::LdmdLayout L{};
  *bytes = ldmd_layout(L, n_channel, n_energy, 1, n_sector, is_complex, precision, nullptr);
  return TICC_OK;
}

int ticc_ldmd_propagate(void* Y, int is_complex, const double* energies, int n_energy, double reduced_mass, const double* half_steps, const double* W_start,
                        long long W_start_stride, const double* W_mid, long long W_mid_stride, const double* W_end, long long W_end_stride, int n_sector,
                        int n_channel, int precision, void* workspace, size_t workspace_bytes, int* device_status, void* stream) {
  return ldmd_run("ticc_ldmd_propagate", Y, is_complex, energies, n_energy, reduced_mass, half_steps, W_start, W_start_stride, W_mid, W_mid_stride, W_end,
                  W_end_stride, 0, n_sector, n_channel, 1, precision, workspace, workspace_bytes, device_status, stream);
}

int ticc_ldmd_reduced_blocks(const void* workspace, size_t workspace_bytes, int n_channel, int n_energy, int n_block, int n_sector, int is_complex, int precision,
                             int* counts, void* stream) {
  if (workspace == nullptr || counts == nullptr) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_ldmd_reduced_blocks: null pointer");
  const int rc = ldmd_check_sizes("ticc_ldmd_reduced_blocks", n_channel, n_energy, n_block, n_sector, precision);
  if (rc != TICC_OK) return rc;
  if (precision != TICC_PRECISION_MIXED) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_ldmd_reduced_blocks: only mixed-precision calls reduce sweep blocks");
  ticc::LdmdLayout L{};
  const size_t need = ldmd_layout(L, n_channel, n_energy, n_block, n_sector, is_complex, precision, nullptr);
  if (workspace_bytes < need) return fail(TICC_ERR_WORKSPACE, "ticc_ldmd_reduced_blocks: workspace of %zu bytes given, %zu needed", workspace_bytes, need);
  ldmd_layout(L, n_channel, n_energy, n_block, n_sector, is_complex, precision, static_cast<char*>(const_cast<void*>(workspace)));
  const cudaError_t e = cudaMemcpyAsync(counts, L.reduced, sizeof(int) * (size_t)n_sector, cudaMemcpyDeviceToHost, as_stream(stream));
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_ldmd_reduced_blocks");
}

int ticc_ldmd_blocks_workspace_size(int n_channel, int n_energy, int n_block, int n_sector, int is_complex, int precision, size_t* bytes) {
  if (bytes == nullptr) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_ldmd_blocks_workspace_size: null output pointer");
  const int rc = ldmd_check_sizes("ticc_ldmd_blocks_workspace_size", n_channel, n_energy, n_block, n_sector, precision);
  if (rc != TICC_OK) return rc;
  ticc::LdmdLayout L{};
  *bytes = ldmd_layout(L, n_channel, n_energy, n_block, n_sector, is_complex, precision, nullptr);
  return TICC_OK;
}

int ticc_ldmd_propagate_blocks(void* Y, int is_complex, const double* energies, int n_energy, double reduced_mass, const double* half_steps,
                               const double* W_start, long long W_start_stride, const double* W_mid, long long W_mid_stride, const double* W_end,
                               long long W_end_stride, long long W_block_stride, int n_sector, int n_channel, int n_block, int precision, void* workspace,
                               size_t workspace_bytes, int* device_status, void* stream) {
  return ldmd_run("ticc_ldmd_propagate_blocks", Y, is_complex, energies, n_energy, reduced_mass, half_steps, W_start, W_start_stride, W_mid, W_mid_stride,
                  W_end, W_end_stride, W_block_stride, n_sector, n_channel, n_block, precision, workspace, workspace_bytes, device_status, stream);
}

// ---- contraction ---------------------------------------------------------------------------------
int ticc_contract(const double* rows_real, const double* rows_imag, const int* group_offsets, int n_groups, const int* row_out, int n_grid,
                  double normalization, const double* potential, long long pot_stride, int n_R, int n_channel, const double* radial_points, const double* U,
                  const double* E_int, double reduced_mass, double* out, void* stream) {
  if (rows_real == nullptr || group_offsets == nullptr || row_out == nullptr || potential == nullptr || out == nullptr)
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_contract: null input pointer");
  if (n_groups < 0 || n_grid < 1 || n_R < 0 || n_channel < 1 || pot_stride < n_grid)
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_contract: n_groups=%d n_grid=%d n_R=%d n_channel=%d pot_stride=%lld", n_groups, n_grid, n_R, n_channel, pot_stride);
  if (U != nullptr && (radial_points == nullptr || E_int == nullptr || !(reduced_mass > 0.0)))
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_contract: W assembly needs radial_points, E_int and a positive reduced_mass");
  for (int g = 0; g < n_groups; ++g)
    if (group_offsets[g + 1] < group_offsets[g]) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_contract: group_offsets must be non-decreasing");
  if (n_R == 0) return TICC_OK;
  cudaStream_t s = as_stream(stream);
  ticc::contract_init_kernel<<<ticc::grid_for((long long)n_R * n_channel * n_channel, 256), 256, 0, s>>>(out, n_channel, n_R, radial_points, U, E_int, reduced_mass);
  ticc::note_launch();
  const double scale = normalization * (U != nullptr ? 2.0 * reduced_mass : 1.0);
  cudaError_t e = cudaFuncSetAttribute(ticc::contract_group_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ticc::kVSmemBytes);
  if (e != cudaSuccess) return cuda_fail(e, "ticc_contract");
  // one launch per kVMaxGroups non-empty groups (and per 65535 radial points)
  ticc::ContractTiles tiles{};
  auto flush = [&]() {
    const int n_tiles = tiles.tile_start[tiles.n_groups];
    for (int r0 = 0; r0 < n_R; r0 += 65535) {
      ticc::contract_group_kernel<<<dim3(n_tiles, std::min(65535, n_R - r0)), 256, ticc::kVSmemBytes, s>>>(tiles, rows_real, rows_imag, row_out, n_grid, scale, potential,
                                                                                                     pot_stride, r0, n_channel, out);
      ticc::note_launch();
    }
    tiles.n_groups = 0;
    tiles.tile_start[0] = 0;
  };
  for (int g = 0; g < n_groups; ++g) {
    const int rows = group_offsets[g + 1] - group_offsets[g];
    if (rows == 0) continue;
    const int t = (rows + ticc::kVTile - 1) / ticc::kVTile;
    const int k = tiles.n_groups++;
    tiles.row0[k] = group_offsets[g];
    tiles.rows[k] = rows;
    tiles.tile_start[k + 1] = tiles.tile_start[k] + t * (t + 1) / 2;
    if (tiles.n_groups == ticc::kVMaxGroups) flush();
  }
  if (tiles.n_groups > 0) flush();
  e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_contract");
}

// ---- one block of a state-resolved contraction ----------------------------------------------------
int ticc_contract_block(const double* A, int n_a, const double* B, int n_b, int n_grid, const double* weights, long long w_stride, int n_R, const int* pos_a,
                        const int* pos_b, int symmetric, int mirror, int n, double* out, void* stream) {
  if (A == nullptr || B == nullptr || weights == nullptr || pos_a == nullptr || pos_b == nullptr || out == nullptr)
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_contract_block: null pointer");
  if (n_a < 0 || n_b < 0 || n_grid < 1 || n_R < 0 || n < 1 || w_stride < n_grid || (symmetric && (n_a != n_b || A != B || pos_a != pos_b)))
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_contract_block: n_a=%d n_b=%d n_grid=%d n_R=%d n=%d w_stride=%lld symmetric=%d (a symmetric block has B = A)", n_a, n_b,
                n_grid, n_R, n, w_stride, symmetric);
  if (n_a == 0 || n_b == 0 || n_R == 0) return TICC_OK;
  cudaError_t e = cudaFuncSetAttribute(ticc::weighted_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ticc::kVSmemBytes);
  if (e != cudaSuccess) return cuda_fail(e, "ticc_contract_block");
  for (int r0 = 0; r0 < n_R; r0 += 65535) {
    const dim3 grid((n_a + ticc::kVTile - 1) / ticc::kVTile, (n_b + ticc::kVTile - 1) / ticc::kVTile, std::min(65535, n_R - r0));
    ticc::weighted_block_kernel<<<grid, 256, ticc::kVSmemBytes, as_stream(stream)>>>(A, n_a, B, n_b, n_grid, weights, w_stride, r0, pos_a, pos_b, symmetric, mirror, n, out);
    ticc::note_launch();
  }
  e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_contract_block");
}

// ---- packed channel pairs into matrices (fine-structure families) --------------------------------
int ticc_pairs_to_matrix(const double* src, int is_complex, long long src_stride, int n_pairs, const int* pair_rows, const int* pair_cols,
                         const unsigned char* reversed, int n, int n_R, double* out, void* stream) {
  if (src == nullptr || pair_rows == nullptr || pair_cols == nullptr || out == nullptr) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_pairs_to_matrix: null pointer");
  if (n_pairs < 0 || n < 1 || n_R < 0 || src_stride < (long long)n_pairs * (is_complex ? 2 : 1))
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_pairs_to_matrix: n_pairs=%d n=%d n_R=%d src_stride=%lld", n_pairs, n, n_R, src_stride);
  if (n_pairs == 0 || n_R == 0) return TICC_OK;
  ticc::pairs_to_matrix_kernel<<<ticc::grid_for((long long)n_R * n_pairs, 256), 256, 0, as_stream(stream)>>>(src, is_complex, src_stride, n_pairs, pair_rows, pair_cols, reversed, n,
                                                                                                          n_R, out);
  ticc::note_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_pairs_to_matrix");
}

// ---- analytic PES on the device -----------------------------------------------------------------
int ticc_pes_legendre_grid(const double* R, int n_R, const double* r, int n_r, const double* x, int n_x, int n_terms, const int* lam, const int* n_prim,
                           const int* prim_kind, const double* prim_params, const int* n_poly, const double* poly, double re, double* V, void* stream) {
  if (R == nullptr || r == nullptr || x == nullptr || V == nullptr || lam == nullptr || n_prim == nullptr || prim_kind == nullptr || prim_params == nullptr ||
      n_poly == nullptr || poly == nullptr)
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_pes_legendre_grid: null pointer");
  if (n_R < 0 || n_r < 1 || n_x < 1 || n_terms < 1 || n_terms > ticc::kPesMaxTerms)
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_pes_legendre_grid: n_R=%d n_r=%d n_x=%d n_terms=%d (at most %d terms)", n_R, n_r, n_x, n_terms, ticc::kPesMaxTerms);
  ticc::PesTable tab{};
  tab.n_terms = n_terms;
  tab.re = re;
  tab.lmax = 0;
  for (int t = 0; t < n_terms; ++t) {
    if (lam[t] < 0 || lam[t] > ticc::kPesMaxLam || n_prim[t] < 0 || n_prim[t] > ticc::kPesMaxPrim || n_poly[t] < 0 || n_poly[t] > ticc::kPesMaxPoly)
      return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_pes_legendre_grid: term %d has lam=%d, %d primitives, %d polynomial coefficients (at most %d, %d, %d)", t, lam[t],
                  n_prim[t], n_poly[t], ticc::kPesMaxLam, ticc::kPesMaxPrim, ticc::kPesMaxPoly);
    tab.lam[t] = lam[t];
    tab.lmax = lam[t] > tab.lmax ? lam[t] : tab.lmax;
    tab.n_prim[t] = n_prim[t];
    tab.n_poly[t] = n_poly[t];
    for (int p = 0; p < n_prim[t]; ++p) {
      const int k = prim_kind[t * ticc::kPesMaxPrim + p];
      if (k < ticc::kPesPower || k > ticc::kPesLJ) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_pes_legendre_grid: term %d primitive %d has unknown kind %d", t, p, k);
      tab.kind[t][p] = k;
      tab.a[t][p] = prim_params[(t * ticc::kPesMaxPrim + p) * 3 + 0];
      tab.b[t][p] = prim_params[(t * ticc::kPesMaxPrim + p) * 3 + 1];
      tab.c[t][p] = prim_params[(t * ticc::kPesMaxPrim + p) * 3 + 2];
    }
    for (int q = 0; q < n_poly[t]; ++q) tab.poly[t][q] = poly[t * ticc::kPesMaxPoly + q];
  }
  if (n_R == 0) return TICC_OK;
  const long long total = (long long)n_R * n_r * n_x;
  ticc::pes_legendre_kernel<<<ticc::grid_for(total, 256), 256, 0, as_stream(stream)>>>(tab, R, n_R, r, n_r, x, n_x, V);
  ticc::note_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_pes_legendre_grid");
}

// ---- BF -> SF transform ------------------------------------------------------------------------------
static size_t transform_layout(int n, int batch, double** Bp, double** P, double** T, char* base) {
  Carver c{base};
  const int np = ticc::ldmd_np(n, 0);
  *Bp = c.take<double>((size_t)np * np);
  *P = c.take<double>((size_t)batch * np * np);
  *T = c.take<double>((size_t)batch * np * np);
  return c.used + 256;
}

int ticc_transform_workspace_size(int n, int batch, int is_complex, size_t* bytes) {
  if (n < 1 || batch < 1 || bytes == nullptr) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_transform_workspace_size: n=%d batch=%d", n, batch);
  double *a, *b, *c;
  *bytes = transform_layout(n, batch, &a, &b, &c, nullptr);
  return TICC_OK;
}

int ticc_transform_bf_to_sf(const void* Y, void* Y_out, const double* B, int n, int batch, int is_complex, void* workspace, size_t workspace_bytes, void* stream) {
  if (Y == nullptr || Y_out == nullptr || B == nullptr || n < 1 || batch < 1) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_transform_bf_to_sf: bad arguments");
  double *Bp, *P, *T;
  const size_t need = transform_layout(n, batch, &Bp, &P, &T, nullptr);
  if (workspace == nullptr || workspace_bytes < need) return fail(TICC_ERR_WORKSPACE, "ticc_transform_bf_to_sf: workspace of %zu bytes given, %zu needed", workspace_bytes, need);
  transform_layout(n, batch, &Bp, &P, &T, static_cast<char*>(workspace));
  const int np = ticc::ldmd_np(n, 0);
  cudaStream_t s = as_stream(stream);
  const long long area = (long long)np * np;
  ticc::pad_plane_kernel<<<dim3(ticc::grid_for(area, 256, 8192), 1), 256, 0, s>>>(B, n, 0, 0, Bp, np);
  ticc::note_launch();
  for (int part = 0; part < (is_complex ? 2 : 1); ++part) {
    ticc::pad_plane_kernel<<<dim3(ticc::grid_for(area, 256, 8192), batch), 256, 0, s>>>(static_cast<const double*>(Y), n, is_complex, part, P, np);
    ticc::note_launch();
    // T^T = (B^T Y)^T, then (B^T T^T)^T = T B = B^T Y B
    ticc::GemmBatch g1{Bp, np, 0, P, np, area, T, np, area, np, 1.0, 1};
    cudaError_t e = ticc::gemm_tn(g1, np, np, batch, s);
    if (e != cudaSuccess) return cuda_fail(e, "ticc_transform_bf_to_sf");
    ticc::GemmBatch g2{Bp, np, 0, T, np, area, P, np, area, np, 1.0, 1};
    e = ticc::gemm_tn(g2, np, np, batch, s);
    if (e != cudaSuccess) return cuda_fail(e, "ticc_transform_bf_to_sf");
    ticc::unpad_plane_kernel<<<dim3(ticc::grid_for((long long)n * n, 256, 8192), batch), 256, 0, s>>>(P, np, static_cast<double*>(Y_out), n, is_complex, part);
    ticc::note_launch();
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_transform_bf_to_sf");
}

// ---- Bessel functions -------------------------------------------------------------------------------------
__global__ void riccati_kernel(const double* ell, const double* x, int n, double* out, int* status) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const ticc::BesselJY r = ticc::riccati_bessel(ell[i], x[i]);
    if (!r.ok) ticc::report_status(status, ticc::kDeviceBesselFailed, 0, i);
    out[4 * i] = r.J;
    out[4 * i + 1] = r.Y;
    out[4 * i + 2] = r.Jp;
    out[4 * i + 3] = r.Yp;
  }
}

__global__ void k_logd_kernel(const double* nu, const double* x, int n, double* out, int* status) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = ticc::bessel_k_logd(nu[i], x[i]);
    if (!isfinite(v)) ticc::report_status(status, ticc::kDeviceBesselFailed, 0, i);
    out[i] = v;
  }
}

int ticc_riccati_bessel_jy(const double* ell, const double* x, int n, double* out, int* device_status, void* stream) {
  if (ell == nullptr || x == nullptr || out == nullptr || n < 0) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_riccati_bessel_jy: bad arguments");
  if (n == 0) return TICC_OK;
  riccati_kernel<<<ticc::grid_for(n, 128), 128, 0, as_stream(stream)>>>(ell, x, n, out, device_status);
  ticc::note_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_riccati_bessel_jy");
}

int ticc_bessel_k_logd(const double* nu, const double* x, int n, double* out, int* device_status, void* stream) {
  if (nu == nullptr || x == nullptr || out == nullptr || n < 0) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_bessel_k_logd: bad arguments");
  if (n == 0) return TICC_OK;
  k_logd_kernel<<<ticc::grid_for(n, 128), 128, 0, as_stream(stream)>>>(nu, x, n, out, device_status);
  ticc::note_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_bessel_k_logd");
}

// ---- matching ---------------------------------------------------------------------------------------------
int ticc_match_workspace_size(int n_channel, int n_energy, int is_complex, int max_open, size_t* bytes) {
  if (n_channel < 1 || n_energy < 1 || max_open < 0 || max_open > n_channel || bytes == nullptr)
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_match_workspace_size: n_channel=%d n_energy=%d max_open=%d", n_channel, n_energy, max_open);
  ticc::MatchLayout L{};
  *bytes = match_layout(L, n_channel, n_energy, is_complex, max_open, nullptr);
  return TICC_OK;
}

int ticc_match_smatrix(const void* Y, int is_complex, double Rmatch, const double* energies, int n_energy, double reduced_mass, const double* E_int, const double* L,
                       int n_channel, int max_open, double* S, int* n_open, void* workspace, size_t workspace_bytes, int* device_status, void* stream) {
  if (Y == nullptr || energies == nullptr || E_int == nullptr || L == nullptr || S == nullptr || n_open == nullptr)
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_match_smatrix: null input pointer");
  if (n_channel < 1 || n_energy < 1 || max_open < 0 || max_open > n_channel)
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_match_smatrix: n_channel=%d n_energy=%d max_open=%d", n_channel, n_energy, max_open);
  if (!(Rmatch > 0.0) || !(reduced_mass > 0.0))
    return fail(TICC_ERR_INVALID_ARGUMENT, "Rmatch and reduced_mass must be positive, but got Rmatch=%g, reduced_mass=%g", Rmatch, reduced_mass);
  ticc::MatchLayout Lay{};
  const size_t need = match_layout(Lay, n_channel, n_energy, is_complex, max_open, nullptr);
  if (workspace == nullptr || workspace_bytes < need) return fail(TICC_ERR_WORKSPACE, "ticc_match_smatrix: workspace of %zu bytes given, %zu needed", workspace_bytes, need);
  match_layout(Lay, n_channel, n_energy, is_complex, max_open, static_cast<char*>(workspace));
  cudaError_t e = ticc::match_smatrix(static_cast<const double*>(Y), Rmatch, energies, reduced_mass, E_int, L, S, n_open, Lay, device_status, as_stream(stream));
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_match_smatrix");
}

// ---- learned sector widths -------------------------------------------------------------------------
int ticc_mlp_shape(int* n_feature, int* n_hidden, int* n_param) {
  if (n_feature == nullptr || n_hidden == nullptr || n_param == nullptr) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_mlp_shape: null output pointer");
  *n_feature = ticc::kFeat;
  *n_hidden = ticc::kHidden;
  *n_param = ticc::kParams;
  return TICC_OK;
}

int ticc_step_features(const double* W_start, long long W_start_stride, const double* W_mid, long long W_mid_stride, const double* W_end, long long W_end_stride,
                       const double* half_steps, int n_sector, int n_channel, double two_mu_emax, double two_mu_emin, float* features, void* stream) {
  if (W_start == nullptr || W_mid == nullptr || W_end == nullptr || half_steps == nullptr || features == nullptr)
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_step_features: null pointer");
  if (n_sector < 0 || n_channel < 1) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_step_features: n_sector=%d n_channel=%d", n_sector, n_channel);
  if (n_sector == 0) return TICC_OK;
  ticc::step_features_kernel<<<n_sector, ticc::kFeatureThreads, 0, as_stream(stream)>>>(W_start, W_start_stride, W_mid, W_mid_stride, W_end, W_end_stride, half_steps, n_channel,
                                                                                        two_mu_emax, two_mu_emin, features);
  ticc::note_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_step_features");
}

int ticc_mlp_forward(const float* params, const float* norm, const float* x, int n, float* y, void* stream) {
  if (params == nullptr || norm == nullptr || x == nullptr || y == nullptr) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_mlp_forward: null pointer");
  if (n < 0) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_mlp_forward: n=%d", n);
  if (n == 0) return TICC_OK;
  ticc::mlp_forward_kernel<<<(n + 127) / 128, 128, 0, as_stream(stream)>>>(params, norm, x, n, y);
  ticc::note_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_mlp_forward");
}

int ticc_mlp_workspace_size(int n, size_t* bytes) {
  if (n < 1 || bytes == nullptr) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_mlp_workspace_size: n=%d", n);
  *bytes = ticc::mlp_workspace_floats(n) * sizeof(float) + 256;
  return TICC_OK;
}

int ticc_mlp_gradient(const float* params, const float* norm, const float* x, const float* target, const float* weight, int n, float over_weight, float inv_weight_sum,
                      float* grads, float* loss, void* workspace, size_t workspace_bytes, void* stream) {
  if (params == nullptr || norm == nullptr || x == nullptr || target == nullptr || weight == nullptr || grads == nullptr || loss == nullptr)
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_mlp_gradient: null pointer");
  if (n < 1 || !(over_weight > 0.0f) || !(inv_weight_sum > 0.0f))
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_mlp_gradient: n=%d over_weight=%g inv_weight_sum=%g", n, over_weight, inv_weight_sum);
  const size_t need = ticc::mlp_workspace_floats(n) * sizeof(float) + 256;
  if (workspace == nullptr || workspace_bytes < need) return fail(TICC_ERR_WORKSPACE, "ticc_mlp_gradient: workspace of %zu bytes given, %zu needed", workspace_bytes, need);
  Carver c{static_cast<char*>(workspace)};
  const int nb = ticc::mlp_grad_blocks(n);
  float* partials = c.take<float>((size_t)nb * ticc::kParams);
  float* loss_partials = c.take<float>((size_t)nb);
  cudaError_t e = cudaFuncSetAttribute(ticc::mlp_partial_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ticc::kMlpGradSmemBytes);
  if (e != cudaSuccess) return cuda_fail(e, "ticc_mlp_gradient");
  cudaStream_t s = as_stream(stream);
  ticc::mlp_partial_grad_kernel<<<nb, ticc::kMlpSamples, ticc::kMlpGradSmemBytes, s>>>(params, norm, x, target, weight, n, over_weight, inv_weight_sum, partials, loss_partials);
  ticc::note_launch();
  ticc::mlp_reduce_kernel<<<(ticc::kParams + 255) / 256, 256, 0, s>>>(partials, loss_partials, nb, grads, loss);
  ticc::note_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_mlp_gradient");
}

int ticc_mlp_adam(float* params, const float* grads, float* moments, int step, float lr, float beta1, float beta2, float eps, void* stream) {
  if (params == nullptr || grads == nullptr || moments == nullptr) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_mlp_adam: null pointer");
  if (step < 1 || !(lr > 0.0f) || !(beta1 >= 0.0f && beta1 < 1.0f) || !(beta2 >= 0.0f && beta2 < 1.0f) || !(eps > 0.0f))
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_mlp_adam: step=%d lr=%g beta1=%g beta2=%g eps=%g", step, lr, beta1, beta2, eps);
  ticc::mlp_adam_kernel<<<(ticc::kParams + 255) / 256, 256, 0, as_stream(stream)>>>(params, grads, moments, step, lr, beta1, beta2, eps);
  ticc::note_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_mlp_adam");
}

// ---- test hook: the tcgen05 TF32x3 update tile on its own -------------------------------------
static size_t tc_debug_layout(int np, int batch, float** split, int** flag, char* base) {
  Carver c{base};
  *split = c.take<float>(ticc::tc_split_floats(np, batch));
  *flag = c.take<int>(4);
  return c.used + 256;
}

int ticc_debug_tc_update_workspace_size(int np, int batch, size_t* bytes) {
  if (bytes == nullptr || np < ticc::kBlock || np % ticc::kBlock != 0 || batch < 1)
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_debug_tc_update_workspace_size: np=%d (a positive multiple of 128) batch=%d", np, batch);
  float* split;
  int* flag;
  *bytes = tc_debug_layout(np, batch, &split, &flag, nullptr);
  return TICC_OK;
}

int ticc_debug_tc_update(double* M, int np, int batch, const double* cold, const double* U, const int* tiles, int n_tiles, void* workspace, size_t workspace_bytes,
                         int* device_status, void* stream) {
  if (M == nullptr || cold == nullptr || U == nullptr || tiles == nullptr || n_tiles < 0 || np < ticc::kBlock || np % ticc::kBlock != 0 || batch < 1)
    return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_debug_tc_update: bad arguments (np=%d batch=%d n_tiles=%d)", np, batch, n_tiles);
  float* split;
  int* flag;
  const size_t need = tc_debug_layout(np, batch, &split, &flag, nullptr);
  if (workspace == nullptr || workspace_bytes < need) return fail(TICC_ERR_WORKSPACE, "ticc_debug_tc_update: workspace of %zu bytes given, %zu needed", workspace_bytes, need);
  tc_debug_layout(np, batch, &split, &flag, static_cast<char*>(workspace));
  cudaStream_t s = as_stream(stream);
  cudaError_t e = cudaMemsetAsync(flag, 0, 4 * sizeof(int), s);
  if (e != cudaSuccess) return cuda_fail(e, "ticc_debug_tc_update: memset");
  ticc::tc_split_panels_kernel<<<dim3(np / ticc::kBlock, batch), 256, 0, s>>>(cold, U, np, batch, split);
  ticc::note_launch();
  if (n_tiles == 0) return TICC_OK;
  ticc::TcMaps maps;
  e = ticc::tc_make_maps(maps, split, M, np, (long long)np * np, batch);
  if (e != cudaSuccess) return cuda_fail(e, "ticc_debug_tc_update: tensor maps");
  e = cudaFuncSetAttribute(ticc::tc_tiles_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, ticc::kTcSmemBytes);
  if (e != cudaSuccess) return cuda_fail(e, "ticc_debug_tc_update: shared memory");
  int dev = 0, sms = 0;
  e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return cuda_fail(e, "ticc_debug_tc_update: device");
  const int blocks = n_tiles < sms ? n_tiles : sms;
  ticc::tc_tiles_kernel<<<blocks, 256, ticc::kTcSmemBytes, s>>>(maps, np, tiles, n_tiles, flag, device_status);
  ticc::note_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_debug_tc_update");
}

// ---- test hook: bounded waits ------------------------------------------------------------------
int ticc_debug_set_step_poll_limit(long long polls) {
  if (polls < 0) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_debug_set_step_poll_limit: polls=%lld must be non-negative", polls);
  cudaError_t e = cudaMemcpyToSymbol(ticc::g_step_poll_limit, &polls, sizeof(polls));
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_debug_set_step_poll_limit");
}

// ---- allocation-free symmetric inversion -------------------------------------------------
// For callers that cannot allocate device memory themselves: plugin hosts that hand this
// library only the buffers they already own, runtimes that fix their device memory budget
// at start-up, and drivers written in languages without a device allocator of their own (a
// Fortran or C program that links just this ABI).  The scratch lives in a fixed array
// compiled into the library instead of a caller workspace.

}  // extern "C"

namespace {

// 32 MiB of scratch; every GPU that loads the library holds it until the process exits.
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
__device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double)];

// Device address of g_noalloc_scratch per device ordinal (host code cannot use the symbol
// itself: on the host it names a stand-in, not device memory).
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_address[kMaxDevices] = {};

}  // namespace

extern "C" {

int ticc_sym_inverse_noalloc(void* M, int n, int batch, int is_complex, int* device_status, void* stream) {
  if (M == nullptr || n < 1 || batch < 1) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_sym_inverse_noalloc: M=%p n=%d batch=%d", M, n, batch);
  double *Mw, *scratch;
  const size_t need = sym_layout(n, batch, is_complex, &Mw, &scratch, nullptr);
  if (need > kNoAllocScratchBytes)
    return fail(TICC_ERR_INVALID_ARGUMENT,
                "ticc_sym_inverse_noalloc: n=%d batch=%d is_complex=%d needs %zu bytes of scratch, but the fixed device array holds %zu bytes "
                "(batch * (Np^2 + 128 Np + 32784) doubles with Np = n, or 2n when complex, rounded up to 128)",
                n, batch, is_complex, need, kNoAllocScratchBytes);
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return cuda_fail(e, "ticc_sym_inverse_noalloc: cudaGetDevice");
  if (device < 0 || device >= kMaxDevices) return fail(TICC_ERR_INVALID_ARGUMENT, "ticc_sym_inverse_noalloc: device ordinal %d beyond %d", device, kMaxDevices);
  double* base = nullptr;
  {
    // first call on a device: look up the array's device address with that device current
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_address[device] == nullptr) {
      void* address = nullptr;
      e = cudaGetSymbolAddress(&address, g_noalloc_scratch);
      if (e != cudaSuccess) return cuda_fail(e, "ticc_sym_inverse_noalloc: cudaGetSymbolAddress");
      g_noalloc_address[device] = static_cast<double*>(address);
    }
    base = g_noalloc_address[device];
  }
  // the array keeps the previous call's contents: the work matrix and the panel regions are
  // fully written before they are read (the load kernel fills the whole padded matrix, the
  // sweep writes each panel before using it), and the words that must start at zero (the
  // fused step's work queues, abort flag and row-panel tile flags) are zeroed by
  // sweep_batched on every call
  sym_layout(n, batch, is_complex, &Mw, &scratch, reinterpret_cast<char*>(base));
  const int np = ticc::ldmd_np(n, is_complex);
  const long long nl = is_complex ? np / 2 : np;
  cudaStream_t s = as_stream(stream);
  sym_load_kernel<<<dim3(ticc::grid_for(nl * nl, 256, 8192), batch), 256, 0, s>>>(static_cast<double*>(M), n, is_complex, Mw, np);
  ticc::note_launch();
  e = ticc::sweep_sym(Mw, (long long)np * np, np, batch, scratch, device_status, s);
  if (e != cudaSuccess) return cuda_fail(e, "ticc_sym_inverse_noalloc");
  sym_store_kernel<<<dim3(ticc::grid_for((long long)n * n, 256, 8192), batch), 256, 0, s>>>(Mw, np, static_cast<double*>(M), n, is_complex);
  ticc::note_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? TICC_OK : cuda_fail(e, "ticc_sym_inverse_noalloc");
}

}  // extern "C"
