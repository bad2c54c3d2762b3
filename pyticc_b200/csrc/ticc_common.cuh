// Shared definitions for the B200 coupled-channel kernels.
//
// Layout conventions used by every kernel in this library:
//  * matrices are row-major doubles; a "batch" of matrices is a base pointer plus a
//    batch stride in elements;
//  * matrices that go through the blocked symmetric sweep are padded to a multiple
//    of kBlock (128) rows and columns; padding carries the identity on the diagonal
//    and zeros elsewhere, so sweeping it leaves -1 on the padded diagonal and never
//    couples it to the logical channels;
//  * complex symmetric matrices A = X + iZ are swept through the real symmetric
//    embedding with 2x2 blocks [[X, Z], [Z, -X]] interleaved per channel, which is
//    invertible exactly when A is and keeps every 2x2 diagonal block nonsingular.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>

namespace ticc {

constexpr int kBlock = 128;          // sweep pivot block = GEMM output tile edge
constexpr int kChunk = 32;           // K rows staged per shared-memory stage
constexpr int kPad = 4;              // shared-memory row padding (doubles)
constexpr int kStride = kBlock + kPad;  // 132: conflict-free DMMA fragment loads
constexpr int kGemmThreads = 256;    // 8 warps: 2 (rows of 64) x 4 (cols of 32)
constexpr int kPivotThreads = 256;

// Device status codes written into the caller's status word (first error wins).
enum DeviceStatus : int {
  kDeviceOk = 0,
  kDeviceSingularPivot = 1,   // a pivot block of the sweep was singular or non-finite
  kDeviceNonFinite = 2,       // a non-finite value reached an output
  kDeviceBesselFailed = 3,    // a Bessel continued fraction did not converge
  kDeviceThreshold = 4,       // a total energy sits exactly on a channel threshold
  kDeviceStalled = 6,         // a fused sweep step gave up waiting for a row-panel tile (bounded wait)
};

// Host-side count of kernels this library has enqueued (process lifetime).
inline std::atomic<long long>& launch_counter() {
  static std::atomic<long long> count{0};
  return count;
}
inline void note_launch(long long n = 1) { launch_counter().fetch_add(n, std::memory_order_relaxed); }

inline __host__ __device__ long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

// Record the first device-side error: status[0] = code, status[1] = batch item,
// status[2] = detail (block or channel index).  Later errors are dropped.
__device__ inline void report_status(int* status, int code, int item, int detail) {
  if (status == nullptr) return;
  if (atomicCAS(status, 0, code) == 0) {
    status[1] = item;
    status[2] = detail;
  }
}

}  // namespace ticc
