// TF32x3 trailing-update tiles on the 5th-generation tensor core (tcgen05 + TMA + TMEM).
//
// One unit computes C <- C - A^T B for a 128 x 128 FP64 tile C of a work matrix, with
// A = the old pivot rows (cold, 128 x 128 block of columns ta) and B = U = P^-1 cold
// (columns tb), both given as FP32 panels and split in shared memory as x = hi + lo in TF32:
//   D = A_lo B_hi + A_hi B_lo + A_hi B_hi      (FP32 accumulation in TMEM, ~2^-20 relative)
// Operand chunks of kTcChunk k-rows arrive by TMA (cp.async.bulk.tensor) in the canonical
// K-major no-swizzle layout through a ring of kTcStages raw stages.  Warps 1-7 split a landed
// chunk: the TF32 MMA reads an FP32 word through its leading 19 bits, so the raw word serves as
// hi = trunc_tf32(x), and lo = x - hi goes into one of kTcLoBufs lo buffers.
// Thread 0 issues the loads and tcgen05.mma.cta_group::1.kind::tf32 (M = N = 128, K = 8
// per instruction) into a 128-column TMEM accumulator, and commits to mbarriers that free
// the stages.  So the panels cost 4 bytes per element in global memory and on the way into
// the SM, half of what pre-split hi/lo panels cost.  The FP64 C tile is loaded by TMA
// (128-byte swizzle) into shared memory while the products run, C - D is formed there (D
// read from TMEM with tcgen05.ld, one TMEM lane = one row), and the tile goes back by TMA
// store.  A diagonal tile is symmetrised from its lower half before the store.
//
// The row panels of such a step run on the same machinery (tc_rowpanel_unit): U = P^-1 cold
// with P^-1 from a pivot panel (written by the unit that inverted the pivot) and cold, the
// unit's FP64 tile of M loaded into the C buffer, turned into the B operand by the converter
// warps, which write the update's A panel on the way; U leaves as FP64 (TMA store) and as the
// update's B panel (one bulk copy).
//
// Panel layout in global memory (read by TMA), one 8 KB block per (matrix b, panel which,
// 128-column tile ct, 16-row k chunk kc):
//   block = ((b * 2 + which) * (np / 128) + ct) * 8 + kc,    which = 0: A (old rows K), 1: B (U)
//   element (k, c), m = c % 128, kk = k % 16, at float block * 2048 + ((m / 8) * 4 + kk / 4) * 32 + (m % 8) * 4 + kk % 4
// i.e. 8-row x 16-byte core matrices, the four along k 128 bytes apart (LBO), the sixteen
// 8-row groups along m 512 bytes apart (SBO): the MMA's K-major operand layout, so a block
// is copied into shared memory as it is and split there element by element.  After the
// panels of all matrices come two pivot panels per matrix (tc_pinv_block: P^-1[k][m] as
// element (k, m), slot = step parity).
//
// Every mbarrier wait is bounded (kTcSpinLimit polls, about a second) and also gives up once
// another thread of the CTA has given up; the unit then raises the call's abort flag,
// reports kDeviceStalled, waits (bounded again) for the loads and products it issued, and
// the CTA frees its TMEM before it exits.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "ticc_common.cuh"

namespace ticc {

constexpr int kTcChunk = 16;                                       // k rows per stage
constexpr int kTcStages = 4;                                       // raw stages (A, B), hi in place
constexpr int kTcLoBufs = 2;                                       // lo buffers (A_lo, B_lo); chunk g uses g % 2
constexpr int kTcArrayBytes = kBlock * kTcChunk * 4;               // 8 KB: one operand's chunk (one panel block)
constexpr int kTcArrayFloats = kTcArrayBytes / 4;
constexpr int kTcStageBytes = 2 * kTcArrayBytes;                   // 16 KB: A then B
constexpr int kTcCBytes = kBlock * kBlock * 8;                     // 128 KB FP64 C tile (8 chunks of 16 columns)
constexpr int kTcCChunkBytes = kBlock * 16 * 8;                    // 16 KB
constexpr int kTcStageOffset = kTcCBytes;
constexpr int kTcLoOffset = kTcStageOffset + kTcStages * kTcStageBytes;
constexpr int kTcBarOffset = kTcLoOffset + kTcLoBufs * kTcStageBytes;  // 229376
constexpr int kTcConvWarps = 7;                                    // warps 1-7 split the chunks
constexpr int kTcFull = 0, kTcEmpty = kTcStages, kTcConv = 2 * kTcStages, kTcAcc = 3 * kTcStages, kTcCFull = 3 * kTcStages + 1, kTcDrain = 3 * kTcStages + 2;
// the streamed update phase (tc_update_stream): two TMEM accumulators, a ring of unit
// descriptors, and the epilogue warps' hand-over of a finished C tile to its store
constexpr int kTcDescSlots = 4;
constexpr int kTcAccFull = 3 * kTcStages + 3, kTcAccEmpty = kTcAccFull + 2, kTcDescFull = kTcAccEmpty + 2, kTcDescEmpty = kTcDescFull + kTcDescSlots, kTcEpiDone = kTcDescEmpty + kTcDescSlots;
constexpr int kTcEpiDoneHi = kTcEpiDone + 1, kTcCFullHi = kTcEpiDone + 2;  // the C buffer's second column half
constexpr int kTcBarriers = kTcEpiDone + 3;
constexpr int kTcEpiWarps = 4;     // warps 4-7 (TMEM lanes 0-127) in the streamed phase
constexpr int kTcStreamConvWarps = 2;  // warps 1-2 split the chunks there
constexpr int kTcMmaWarp = 3;           // and lane 0 of warp 3 issues the MMAs
static_assert(kTcStages % kTcLoBufs == 0, "a stage must always pair with the same lo buffer");
static_assert(kGemmThreads == 32 * (kTcConvWarps + 1), "the units run with thread 0 issuing and warps 1-7 converting");
static_assert(kTcMmaWarp == kTcStreamConvWarps + 1 && kTcMmaWarp + 1 + kTcEpiWarps == kGemmThreads / 32 && kTcEpiWarps == 4, "the streamed phase: warp 0 loads, then converter warps, the MMA warp, four epilogue warps (TMEM lanes 0-127)");
constexpr int kTcTmemSlotOffset = kTcBarOffset + 8 * kTcBarriers;   // TMEM address, then the abort flag at + 8
constexpr int kTcDescOffset = kTcTmemSlotOffset + 16;                // kTcDescSlots x 16 bytes
constexpr int kTcRegionBytes = kTcDescOffset + 16 * kTcDescSlots;
constexpr int kTcSmemBytes = kTcRegionBytes + 1024;                // + alignment slack of the dynamic base
constexpr int kTcTmemColumns = 256;  // two 128-column FP32 accumulators
constexpr long long kTcSpinLimit = 1LL << 20;                      // try_wait polls (each may suspend briefly): about a second
// instruction descriptor: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12 = 2), A and B
// K-major (bits 15, 16 clear), N = 128 (bits 17-22 = N >> 3), M = 128 (bits 24-28 = M >> 4)
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kBlock >> 3) << 17) | ((uint32_t)(kBlock >> 4) << 24);
constexpr uint32_t kTcLBO = 128;  // bytes between the k-adjacent core matrices of a split block
constexpr uint32_t kTcSBO = 512;  // bytes between its 8-row groups
static_assert(kTcRegionBytes + 1024 <= 232448, "tcgen05 update region must fit the 227 KB shared-memory limit");

// ---- PTX wrappers ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) { asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory"); }
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of parity `parity` to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long long it = 0; it < kTcSpinLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// The same, giving up early once *abort (a CTA-wide flag in shared memory) is set.
__device__ __forceinline__ bool mbar_wait_or_abort(uint32_t bar, uint32_t parity, const volatile int* abort) {
  for (long long it = 0; it < kTcSpinLimit; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort) return false;
  }
  return false;
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) { asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory"); }
__device__ __forceinline__ void mbar_arrive_count(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// L2 policies: the split operand panels are re-read by every tile of their row or column
// (keep them), the FP64 C tiles pass through once (let them go first).
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar, uint64_t policy) {
  asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, {%2, %3, %4}], [%5], %6;" ::"r"(dst),
               "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar), "l"(policy)
               : "memory");
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, uint32_t src, int x, int y, int z, uint64_t policy) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group.L2::cache_hint [%0, {%2, %3, %4}], [%1], %5;" ::"l"(reinterpret_cast<uint64_t>(map)), "r"(src),
               "r"(x), "r"(y), "r"(z), "l"(policy)
               : "memory");
}
__device__ __forceinline__ void bulk_copy_s2g(void* dst, uint32_t src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t columns) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(columns) : "memory");
}
__device__ __forceinline__ void tmem_relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t columns) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(columns) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_ld_32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, "
      "%27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tc_ld_16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor of one K-major, unswizzled stage array (a split block);
// `kgroup` selects the 8 k values of one instruction (two core matrices, 256 bytes on).
__device__ __forceinline__ uint64_t tc_desc(uint32_t array_addr, int kgroup) {
  const uint32_t start = array_addr + (uint32_t)kgroup * 2u * kTcLBO;
  uint64_t d = 0;
  d |= (uint64_t)((start >> 4) & 0x3FFFu);
  d |= (uint64_t)((kTcLBO >> 4) & 0x3FFFu) << 16;  // LBO: next core matrix along k
  d |= (uint64_t)((kTcSBO >> 4) & 0x3FFFu) << 32;  // SBO: next 8-row group along m / n
  d |= (uint64_t)1 << 46;                          // descriptor version (sm_100); no swizzle
  return d;
}

// Byte offset of C(r, j) inside the shared C tile: 8 chunks of 16 columns, each 128 rows of
// 128 bytes with the 128-byte swizzle TMA applies (16-byte unit index XOR row % 8).
__device__ __forceinline__ int tc_c_offset(int r, int j) { return (j >> 4) * kTcCChunkBytes + r * 128 + ((((j & 15) >> 1) ^ (r & 7)) << 4) + (j & 1) * 8; }

// Per-CTA state of the tcgen05 unit: the aligned region, its barriers, TMEM and the running
// chunk / tile counters that give every barrier wait its phase parity.
struct TcState {
  char* base;       // 1024-aligned start of the region
  uint32_t base_u;  // its shared-window address
  uint32_t tmem;    // accumulator (lane 0, first column)
  uint32_t chunk;   // operand chunks of finished tiles (every thread keeps the count)
  uint32_t tile;    // tiles finished so far
  int nt;           // 128-column tiles per matrix (np / 128)
  volatile int* abort;  // CTA-wide give-up flag in shared memory
};

// Panel block of (matrix b, panel which, column tile ct, k chunk kc) when a matrix has nt tiles.
__device__ __forceinline__ int tc_split_block(int b, int which, int nt, int ct, int kc) { return ((b * 2 + which) * nt + ct) * (kBlock / kTcChunk) + kc; }

__device__ __forceinline__ uint32_t tc_bar(const TcState& s, int i) { return s.base_u + kTcBarOffset + 8u * (uint32_t)i; }

// Set up the region (thread 0 initialises the barriers, warp 0 allocates TMEM).  Every
// thread of the CTA calls it once, before the first unit.
__device__ inline void tc_setup(TcState& s, void* dynamic_smem, int np) {
  const uintptr_t raw = reinterpret_cast<uintptr_t>(dynamic_smem);
  const uint32_t raw_u = smem_u32(dynamic_smem);
  const uint32_t pad = (1024u - (raw_u & 1023u)) & 1023u;
  s.base = reinterpret_cast<char*>(raw + pad);
  s.base_u = raw_u + pad;
  s.chunk = 0;
  s.tile = 0;
  s.nt = np / kBlock;
  s.abort = reinterpret_cast<volatile int*>(s.base + kTcTmemSlotOffset + 8);
  if (threadIdx.x == 0) {
    for (int i = 0; i < kTcBarriers; ++i) {
      uint32_t count = 1;
      if (i >= kTcConv && i < kTcConv + kTcStages) count = kTcConvWarps;            // a warp-level arrival of every converter warp
      if (i >= kTcAccEmpty && i < kTcAccEmpty + 2) count = kTcEpiWarps;             // every epilogue warp has read the accumulator
      if (i >= kTcDescEmpty && i < kTcDescEmpty + kTcDescSlots) count = kTcStreamConvWarps + 1 + kTcEpiWarps;  // every reader has the descriptor
      if (i == kTcEpiDone || i == kTcEpiDoneHi) count = kTcEpiWarps;                 // every epilogue warp has written its rows
      mbar_init(tc_bar(s, i), count);
    }
    mbar_fence_init();
    *s.abort = 0;
  }
  if (threadIdx.x < 32) {
    tmem_alloc(s.base_u + kTcTmemSlotOffset, kTcTmemColumns);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  s.tmem = *reinterpret_cast<volatile uint32_t*>(s.base + kTcTmemSlotOffset);
}

// Free TMEM; every thread calls it once, after its last unit (and after any failure).
__device__ inline void tc_teardown(TcState& s) {
  if (threadIdx.x == 0) bulk_wait_all();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32) tmem_dealloc(s.tmem, kTcTmemColumns);
}

struct TcMaps {
  CUtensorMap split;   // 3-D {256, 8, blocks} over the split blocks, box {256, 8, 1} (one block)
  CUtensorMap matrix;  // 3-D {np, np, batch} over the FP64 work matrices, box {16, 128, 1}
};

// Issue the TMA loads of operand chunk `c` (k rows c * kTcChunk ..) into raw stage `stage`:
// A from panel block a0 + c and, when b0 >= 0, B from panel block b0 + c (a row-panel unit
// builds B itself); thread 0 only.
__device__ __forceinline__ void tc_issue_chunk(const TcState& s, const CUtensorMap* split, int a0, int b0, int c, int stage) {
  const uint32_t dst = s.base_u + kTcStageOffset + (uint32_t)stage * kTcStageBytes;
  const uint32_t full = tc_bar(s, kTcFull + stage);
  mbar_expect_tx(full, b0 >= 0 ? kTcStageBytes : kTcArrayBytes);
  const uint64_t keep = l2_policy_evict_last();
  tma_load_3d(dst, split, 0, 0, a0 + c, full, keep);
  if (b0 >= 0) tma_load_3d(dst + kTcArrayBytes, split, 0, 0, b0 + c, full, keep);
}

// The TF32 MMA reads an FP32 operand word through its leading 19 bits (sign, exponent, 10
// mantissa bits), so the word itself serves as hi = trunc_tf32(x), and lo = x - hi (exact in
// FP32) is written as it is: the MMA reads its leading 19 bits in turn, so hi + trunc_tf32(lo)
// carries x to 2^-20 relative.
__device__ __forceinline__ float tc_lo_value(float x) { return x - __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }
__device__ __forceinline__ float4 tc_lo4(const float4& x) { return make_float4(tc_lo_value(x.x), tc_lo_value(x.y), tc_lo_value(x.z), tc_lo_value(x.w)); }

// Split the first `vecs` float4 of the landed raw chunk of `stage`: hi is the raw word (left in
// place), lo goes to lo buffer `lo`; the converter threads (warps 1 .. from thread 32 on).
__device__ __forceinline__ void tc_split_stage(const TcState& s, int stage, int lo, int vecs, int stride = 32 * kTcConvWarps) {
  float4* raw = reinterpret_cast<float4*>(s.base + kTcStageOffset + stage * kTcStageBytes);
  float4* low = reinterpret_cast<float4*>(s.base + kTcLoOffset + lo * kTcStageBytes);
#pragma unroll 4
  for (int i = (int)threadIdx.x - 32; i < vecs; i += stride) low[i] = tc_lo4(raw[i]);
}

// The same for a whole 16 KB stage with kThreads converter threads (from thread 32 on), each
// taking kStageVecs / kThreads float4: all loads first, then the differences and stores, so
// that one shared-memory latency covers the chunk.
template <int kThreads>
__device__ __forceinline__ void tc_split_stage_all(const TcState& s, int stage, int lo) {
  constexpr int kVecs = kTcStageBytes / 16, kPer = kVecs / kThreads;
  static_assert(kVecs % kThreads == 0, "every converter thread takes the same number of float4");
  const float4* raw = reinterpret_cast<const float4*>(s.base + kTcStageOffset + stage * kTcStageBytes);
  float4* low = reinterpret_cast<float4*>(s.base + kTcLoOffset + lo * kTcStageBytes);
  const int i0 = (int)threadIdx.x - 32;
  float4 x[kPer];
#pragma unroll
  for (int k = 0; k < kPer; ++k) x[k] = raw[i0 + k * kThreads];
#pragma unroll
  for (int k = 0; k < kPer; ++k) low[i0 + k * kThreads] = tc_lo4(x[k]);
}

// Element (k, n) of the FP64 tile in the C buffer, stored with rows k (`rows_k`) or rows n.
__device__ __forceinline__ double tc_c_at(const TcState& s, bool rows_k, int k, int n) {
  return *reinterpret_cast<const double*>(s.base + (rows_k ? tc_c_offset(k, n) : tc_c_offset(n, k)));
}

// Row-panel chunk c: B_kmajor[n][k] = cold(k, n) for the 16 k rows of the chunk, from the FP64
// cold tile in the C buffer, split into the stage's B array (hi) and the lo buffer; the FP32
// values also go to `out` (the update's A panel block of this chunk).  Threads of warps 1-7.
__device__ __forceinline__ void tc_build_cold_chunk(const TcState& s, int stage, int lo, int c, bool rows_k, float* out) {
  float* hi_b = reinterpret_cast<float*>(s.base + kTcStageOffset + stage * kTcStageBytes + kTcArrayBytes);
  float* lo_b = reinterpret_cast<float*>(s.base + kTcLoOffset + lo * kTcStageBytes + kTcArrayBytes);
  for (int i = (int)threadIdx.x - 32; i < kBlock * (kTcChunk / 4); i += 32 * kTcConvWarps) {
    const int n = i & (kBlock - 1), j = i >> 7;  // k = c * 16 + 4 j .. + 3
    const int k = c * kTcChunk + 4 * j;
    float4 x = make_float4(static_cast<float>(tc_c_at(s, rows_k, k, n)), static_cast<float>(tc_c_at(s, rows_k, k + 1, n)), static_cast<float>(tc_c_at(s, rows_k, k + 2, n)),
                           static_cast<float>(tc_c_at(s, rows_k, k + 3, n)));
    const int o = ((n >> 3) * 4 + j) * 32 + (n & 7) * 4;
    *reinterpret_cast<float4*>(out + o) = x;
    *reinterpret_cast<float4*>(hi_b + o) = x;
    *reinterpret_cast<float4*>(lo_b + o) = tc_lo4(x);
  }
}

// The product of one unit, D = A^T B over k = 0..127 into TMEM, with the unit's FP64 tile
// loaded by TMA into the C buffer (tile coordinates (cx, cy) of matrix b): before the operand
// ring when `c_first` (a row-panel unit turns it into its B operand), else after it.  Thread 0
// issues the loads and the MMAs; warps 1-7 split the chunks and, for a row-panel unit
// (b0 < 0), build B from the tile, writing the update's A panel to `a_out` on the way.
// Returns false on every thread if a wait gave up; the abort flag and status are then set and
// the unit's issued work has been drained (bounded waits).
//
// Chunk g (counted over the CTA's units, g = s.chunk + c) lives in raw stage g % kTcStages
// and lo buffer g % kTcLoBufs.  Phases: full[stage] completes when its loads land, conv[stage]
// when warps 1-7 have split it, empty[stage] when its MMAs have read it.  Thread 0 refills a
// stage after its empty phase; a converter writes lo buffer g % 2 after chunk g - 2's empty
// phase.  Every wait is for the phase right after one this thread has already waited for
// (or the first), so the parity of a wait always names the phase it means.
__device__ inline bool tc_product(TcState& s, const TcMaps& maps, int a0, int b0, int b, int cx, int cy, bool c_first, bool rows_k, float* a_out, int* abort_flag, int* status) {
  constexpr int nchunks = kBlock / kTcChunk;  // 8
  const int tid = threadIdx.x;
  const uint32_t g0 = s.chunk;
  const uint32_t cbar = tc_bar(s, kTcCFull);
  if (tid == 0) {
    int ok = 1;
    unsigned loads_pending = 0;  // stages whose TMA load was issued and not yet seen complete
    uint32_t pending_parity[kTcStages] = {};
    bool c_pending = false, c_issued = false, mma_issued = false;
    // panels written by other CTAs of this launch were released to this thread by the flag
    // it acquired; the stages were last read by the previous unit's MMAs (waited for)
    fence_proxy_async_shared();
    fence_proxy_async_global();
    auto issue = [&](int c, uint32_t g) {
      const int stage = g % kTcStages;
      tc_issue_chunk(s, &maps.split, a0, b0, c, stage);
      loads_pending |= 1u << stage;
      pending_parity[stage] = (g / kTcStages) & 1u;
    };
    // the tile, once the previous unit's TMA store has read the C buffer out (its generic
    // writes were ordered before that store by a proxy fence and a barrier)
    auto load_tile = [&]() {
      bulk_wait_read_all();
      fence_proxy_async_shared();
      mbar_expect_tx(cbar, kTcCBytes);
      const uint64_t once = l2_policy_evict_first();
      for (int q = 0; q < 8; ++q) tma_load_3d(s.base_u + (uint32_t)q * kTcCChunkBytes, &maps.matrix, cx + 16 * q, cy, b, cbar, once);
      c_pending = c_issued = true;
    };
    if (c_first) load_tile();
    for (int c = 0; c < kTcStages && c < nchunks && ok; ++c) {
      const uint32_t g = g0 + c;
      // the MMAs that last read this stage (chunk g - kTcStages) have completed
      if (g >= (uint32_t)kTcStages && !mbar_wait_or_abort(tc_bar(s, kTcEmpty + g % kTcStages), ((g - kTcStages) / kTcStages) & 1u, s.abort)) ok = 0;
      if (ok) issue(c, g);
    }
    // an update unit's C tile goes behind the operand loads in the TMA queue (after the last
    // refill): needed only by the epilogue, it would otherwise hold back chunks 4-7
    for (int c = 0; c < nchunks && ok; ++c) {
      const uint32_t g = g0 + c;
      const int stage = g % kTcStages;
      if (!mbar_wait_or_abort(tc_bar(s, kTcConv + stage), (g / kTcStages) & 1u, s.abort)) {
        ok = 0;
        break;
      }
      loads_pending &= ~(1u << stage);  // split, so landed
      tc_fence_after();
      const uint32_t st = s.base_u + kTcStageOffset + (uint32_t)stage * kTcStageBytes;
      const uint32_t lo = s.base_u + kTcLoOffset + (uint32_t)(g % kTcLoBufs) * kTcStageBytes;
#pragma unroll
      for (int kg = 0; kg < kTcChunk / 8; ++kg) {
        const uint64_t a_hi = tc_desc(st, kg), a_lo = tc_desc(lo, kg);
        const uint64_t b_hi = tc_desc(st + kTcArrayBytes, kg), b_lo = tc_desc(lo + kTcArrayBytes, kg);
        tc_mma_tf32(s.tmem, a_lo, b_hi, (c > 0 || kg > 0) ? 1u : 0u);
        tc_mma_tf32(s.tmem, a_hi, b_lo, 1u);
        tc_mma_tf32(s.tmem, a_hi, b_hi, 1u);
      }
      mma_issued = true;
      tc_commit(tc_bar(s, kTcEmpty + stage));
      // refill the stage of the previous chunk (its MMAs precede this chunk's in the pipe)
      if (c >= 1 && c - 1 + kTcStages < nchunks) {
        const uint32_t gp = g - 1;
        if (!mbar_wait_or_abort(tc_bar(s, kTcEmpty + gp % kTcStages), (gp / kTcStages) & 1u, s.abort)) {
          ok = 0;
          break;
        }
        issue(c - 1 + kTcStages, gp + kTcStages);
        if (c - 1 + kTcStages == nchunks - 1 && !c_issued) load_tile();
      }
    }
    if (ok && !c_issued) load_tile();
    if (ok) {
      tc_commit(tc_bar(s, kTcAcc));
      mma_issued = false;
      if (!mbar_wait_or_abort(tc_bar(s, kTcAcc), s.tile & 1u, s.abort)) ok = 0;
      if (ok && mbar_wait_or_abort(cbar, s.tile & 1u, s.abort)) c_pending = false;
      else ok = 0;
    }
    if (!ok) {
      *s.abort = 1;  // the converters stop waiting
      if (atomicExch(abort_flag, 1) == 0) report_status(status, kDeviceStalled, b, -1);
      // drain: the issued loads and products land before the CTA moves on or frees TMEM
      for (int st = 0; st < kTcStages; ++st)
        if (loads_pending & (1u << st)) mbar_wait(tc_bar(s, kTcFull + st), pending_parity[st]);
      if (c_pending) mbar_wait(cbar, s.tile & 1u);
      if (mma_issued) {
        tc_commit(tc_bar(s, kTcDrain));
        mbar_wait(tc_bar(s, kTcDrain), 0u);
      }
    }
  } else if (tid >= 32) {
    // a row-panel unit reads its tile from the first chunk on
    // (decisions are made warp-uniform, so that a warp's lanes reach __syncwarp together)
    bool ok = __all_sync(0xffffffffu, b0 >= 0 || mbar_wait_or_abort(cbar, s.tile & 1u, s.abort));
    for (int c = 0; c < nchunks && ok; ++c) {
      const uint32_t g = g0 + c;
      const int stage = g % kTcStages;
      // the raw chunk has landed, and the MMAs of chunk g - kTcLoBufs (the lo buffer's last
      // reader) have completed
      ok = mbar_wait_or_abort(tc_bar(s, kTcFull + stage), (g / kTcStages) & 1u, s.abort);
      if (ok && g >= (uint32_t)kTcLoBufs) {
        const uint32_t gp = g - kTcLoBufs;
        ok = mbar_wait_or_abort(tc_bar(s, kTcEmpty + gp % kTcStages), (gp / kTcStages) & 1u, s.abort);
      }
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      const int lo = g % kTcLoBufs;
      if (b0 >= 0) {
        tc_split_stage(s, stage, lo, kTcStageBytes / 16);
      } else {
        tc_split_stage(s, stage, lo, kTcArrayBytes / 16);
        tc_build_cold_chunk(s, stage, lo, c, rows_k, a_out + c * kTcArrayFloats);
        fence_proxy_async_global();  // the A panel is read next by other CTAs' TMA loads
      }
      fence_proxy_async_shared();  // the split chunk is read next by the tensor core
      __syncwarp();
      if ((tid & 31) == 0) mbar_arrive(tc_bar(s, kTcConv + stage));
    }
    if (!ok) *s.abort = 1;  // thread 0 stops waiting for this warp's conversion
  }
  __syncthreads();
  if (*s.abort) return false;
  s.chunk = g0 + nchunks;
  // every thread observes the completed tile load itself (acquire of the async-proxy writes)
  mbar_wait(cbar, s.tile & 1u);
  tc_fence_after();
  return true;
}

// One update tile C <- C - A^T B: C = tile (ta, tb) of matrix b, A = the A panel of column tile
// ta, B = the B panel of column tile tb.  Returns false (on every thread) if a wait gave up.
__device__ inline bool tc_update_unit(TcState& s, const TcMaps& maps, int b, int ta, int tb, int* abort_flag, int* status) {
  const int tid = threadIdx.x;
  const int r0 = ta * kBlock, c0 = tb * kBlock;
  if (!tc_product(s, maps, tc_split_block(b, 0, s.nt, ta, 0), tc_split_block(b, 1, s.nt, tb, 0), b, c0, r0, false, true, nullptr, abort_flag, status)) return false;
  // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (one row each), columns of half w / 4
  const int warp = tid >> 5, lane = tid & 31;
  const int r = 32 * (warp & 3) + lane;
  const int half = warp >> 2;
#pragma unroll 1
  for (int q = 0; q < 4; ++q) {
    const int col = 64 * half + 16 * q;
    float d[16];
    tc_ld_16(s.tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)col, d);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      double2* p = reinterpret_cast<double2*>(s.base + tc_c_offset(r, col + 2 * u));
      double2 v = *p;
      v.x -= (double)d[2 * u];
      v.y -= (double)d[2 * u + 1];
      *p = v;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (ta == tb) {  // keep a diagonal tile exactly symmetric: upper half from the lower half
    for (int e = tid; e < kBlock * kBlock; e += blockDim.x) {
      const int rr = e >> 7, cc = e & (kBlock - 1);
      if (rr < cc) *reinterpret_cast<double*>(s.base + tc_c_offset(rr, cc)) = *reinterpret_cast<const double*>(s.base + tc_c_offset(cc, rr));
    }
    __syncthreads();
  }
  fence_proxy_async_shared();
  __syncthreads();
  if (tid == 0) {
    // the next unit waits for this store to have read the buffer before it reloads C
    const uint64_t once = l2_policy_evict_first();
    for (int q = 0; q < 8; ++q) tma_store_3d(&maps.matrix, s.base_u + (uint32_t)q * kTcCChunkBytes, c0 + 16 * q, r0, b, once);
    bulk_commit();
  }
  ++s.tile;
  __syncthreads();
  return true;
}

// Row panel of a tensor-core step for column tile jt of matrix b: U = P^-1 cold on tcgen05,
// with cold = the old rows K over the tile (tile (kb, jt) of M for jt < kb, the transpose of
// the lower tile (jt, kb) for jt > kb) and P^-1 from the pivot panel at pinv_block0.  Writes
// the update's A panel (cold) and B panel (U) of column tile jt, U into that lower tile and,
// for jt = kb + 1, the old rows into `Cb` and U into the rows K (both read by the next
// pivot's update later in this launch).  Ends with the panels written and the shared buffers
// free; the store of U's tile may still be in flight (this thread waits for it before exit).
__device__ inline bool tc_rowpanel_unit(TcState& s, const TcMaps& maps, float* split, int pinv_block0, int b, int kb, int jt, double* Mb, long long ld, double* Cb, int* abort_flag,
                                        int* status) {
  const int tid = threadIdx.x;
  const int k0 = kb * kBlock, c0 = jt * kBlock;
  const bool rows_k = jt < kb;  // the tile in the C buffer: (kb, jt) (rows k) or (jt, kb) (rows n)
  const int cx = rows_k ? c0 : k0, cy = rows_k ? k0 : c0;
  float* a_panel = split + (long long)tc_split_block(b, 0, s.nt, jt, 0) * kTcArrayFloats;
  if (!tc_product(s, maps, pinv_block0, -1, b, cx, cy, true, rows_k, a_panel, abort_flag, status)) return false;
  const bool pivot_next = jt == kb + 1;
  if (pivot_next) {  // the old rows over tile kb + 1: cold[k][c0 + n]
    for (int e = tid; e < kBlock * kBlock; e += blockDim.x) {
      const int k = e >> 7, n = e & (kBlock - 1);
      Cb[(long long)k * ld + c0 + n] = tc_c_at(s, rows_k, k, n);
    }
  }
  __syncthreads();
  // U = D from TMEM into the C buffer as FP64, oriented like the tile it replaces
  const int warp = tid >> 5, lane = tid & 31;
  const int m = 32 * (warp & 3) + lane;  // row of U (k within the pivot block)
  const int half = warp >> 2;
#pragma unroll 1
  for (int q = 0; q < 4; ++q) {
    const int col = 64 * half + 16 * q;
    float d[16];
    tc_ld_16(s.tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)col, d);
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int n = col + u;
      *reinterpret_cast<double*>(s.base + (rows_k ? tc_c_offset(m, n) : tc_c_offset(n, m))) = (double)d[u];
    }
  }
  tc_fence_before();
  __syncthreads();
  // the B panel (U rounded to FP32) into the free stage area for one bulk copy, and U into the
  // rows K for the pivot unit
  float* b_stage = reinterpret_cast<float*>(s.base + kTcStageOffset);
  for (int e = tid; e < kBlock * (kBlock / 4); e += blockDim.x) {
    const int n = e & (kBlock - 1), k = 4 * (e >> 7);
    const int kk = k % kTcChunk;
    const float4 v = make_float4(static_cast<float>(tc_c_at(s, rows_k, k, n)), static_cast<float>(tc_c_at(s, rows_k, k + 1, n)), static_cast<float>(tc_c_at(s, rows_k, k + 2, n)),
                                 static_cast<float>(tc_c_at(s, rows_k, k + 3, n)));
    *reinterpret_cast<float4*>(b_stage + (k / kTcChunk) * kTcArrayFloats + ((n >> 3) * 4 + (kk >> 2)) * 32 + (n & 7) * 4) = v;
  }
  if (pivot_next) {
    for (int e = tid; e < kBlock * kBlock; e += blockDim.x) {
      const int k = e >> 7, n = e & (kBlock - 1);
      Mb[(long long)(k0 + k) * ld + c0 + n] = tc_c_at(s, rows_k, k, n);
    }
  }
  fence_proxy_async_shared();
  __syncthreads();
  if (tid == 0) {
    // the B panel first, in a bulk group of its own: it must be written before the unit's flag
    // is released; U's tile is read in this launch by nobody, so its store only has to have
    // read the C buffer before the buffers are reused
    bulk_copy_s2g(split + (long long)tc_split_block(b, 1, s.nt, jt, 0) * kTcArrayFloats, s.base_u + kTcStageOffset, kTcStages * kTcStageBytes);
    bulk_commit();
    const uint64_t once = l2_policy_evict_first();
    for (int q = 0; q < 8; ++q) tma_store_3d(&maps.matrix, s.base_u + (uint32_t)q * kTcCChunkBytes, cx + 16 * q, cy, b, once);
    bulk_commit();
    asm volatile("cp.async.bulk.wait_group 1;" ::: "memory");  // the B panel is written
    fence_proxy_async_global();
    bulk_wait_read_all();  // and both buffers have been read out
  }
  ++s.tile;
  __syncthreads();
  return true;
}

// Write one 128 x 128 block of a panel (k rows 0..127 of src at row stride ld, columns
// src_c0 .. src_c0 + 127), rounded to FP32, into the 8 panel blocks from blk0 on (k chunk kc
// in block kc).  All threads of the CTA; a thread takes 4 consecutive k of one column
// (coalesced loads across the warp's consecutive columns) and stores them as one 16-byte row
// of a core matrix.
__device__ inline void tc_write_panel_at(float* blk0, const double* src, long long ld, int src_c0) {
  for (int e = threadIdx.x; e < kBlock * (kBlock / 4); e += blockDim.x) {
    const int k4 = e / kBlock, m = e % kBlock;
    const int k = 4 * k4;
    float v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = static_cast<float>(src[(long long)(k + j) * ld + src_c0 + m]);
    const int kk = k % kTcChunk;
    const long long inner = ((m >> 3) * 4 + (kk >> 2)) * 32 + (m & 7) * 4;
    *reinterpret_cast<float4*>(blk0 + (long long)(k / kTcChunk) * kTcArrayFloats + inner) = make_float4(v[0], v[1], v[2], v[3]);
  }
}
// The same into panel `which` of column tile ct of matrix b.
__device__ inline void tc_write_panel(float* split, int b, int which, int np, const double* src, long long ld, int src_c0, int ct) {
  tc_write_panel_at(split + (long long)tc_split_block(b, which, np / kBlock, ct, 0) * kTcArrayFloats, src, ld, src_c0);
}

// After the A and B panels of all `batch` matrices come two pivot panels per matrix (P^-1 as
// the row-panel product's A operand; slot = step parity): the first of their 8 blocks.
__host__ __device__ inline int tc_pinv_block(int b, int slot, int nt, int batch) { return batch * 2 * nt * (kBlock / kTcChunk) + (b * 2 + slot) * (kBlock / kTcChunk); }
inline size_t tc_split_blocks(int np, int batch) { return (size_t)tc_pinv_block(batch, 0, np / kBlock, batch); }

inline size_t tc_split_floats(int np, int batch) { return tc_split_blocks(np, batch) * kTcArrayFloats; }

// ---- host: tensor maps ----------------------------------------------------------------------------
typedef CUresult (*TcEncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                   CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline TcEncodeTiled tc_encoder() {
  static TcEncodeTiled fn = []() -> TcEncodeTiled {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess) return nullptr;
    return reinterpret_cast<TcEncodeTiled>(p);
  }();
  return fn;
}

// Tensor maps over the split panels of `batch` matrices and over the matrices themselves
// (FP64, row stride np, matrix stride mstride elements).
inline cudaError_t tc_make_maps(TcMaps& maps, const float* split, const double* M, int np, long long mstride, int batch) {
  TcEncodeTiled encode = tc_encoder();
  if (encode == nullptr) return cudaErrorNotSupported;
  if (np % kBlock != 0 || (reinterpret_cast<uintptr_t>(split) & 15) || (reinterpret_cast<uintptr_t>(M) & 15) || (mstride * 8) % 16 != 0) return cudaErrorInvalidValue;
  const cuuint64_t blocks = (cuuint64_t)tc_split_blocks(np, batch);
  const cuuint64_t sdim[3] = {256, (cuuint64_t)(kTcArrayFloats / 256), blocks};
  const cuuint64_t sstride[2] = {256 * 4, (cuuint64_t)kTcArrayBytes};
  const cuuint32_t sbox[3] = {256, (cuuint32_t)(kTcArrayFloats / 256), 1};
  const cuuint32_t ones[4] = {1, 1, 1, 1};
  CUresult r = encode(&maps.split, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(split), sdim, sstride, sbox, ones, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  const cuuint64_t mdim[3] = {(cuuint64_t)np, (cuuint64_t)np, (cuuint64_t)batch};
  const cuuint64_t mstr[2] = {(cuuint64_t)np * 8, (cuuint64_t)mstride * 8};
  const cuuint32_t mbox[3] = {16, (cuuint32_t)kBlock, 1};
  r = encode(&maps.matrix, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(M), mdim, mstr, mbox, ones, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// ---- bring-up path: split two panels, then update a list of tiles ---------------------------------
// cold and U: [batch][128][np]; one CTA per (128-column block, matrix).
__global__ void __launch_bounds__(256) tc_split_panels_kernel(const double* cold, const double* U, int np, int batch, float* split) {
  const int jt = blockIdx.x, b = blockIdx.y;
  tc_write_panel(split, b, 0, np, cold + (long long)b * kBlock * np, np, jt * kBlock, jt);
  tc_write_panel(split, b, 1, np, U + (long long)b * kBlock * np, np, jt * kBlock, jt);
}

// tiles[3 t .. 3 t + 2] = (matrix, row tile, column tile); every CTA takes tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ...
__global__ void __launch_bounds__(256, 1) tc_tiles_kernel(const __grid_constant__ TcMaps maps, int np, const int* tiles, int n_tiles, int* abort_flag, int* status) {
  extern __shared__ __align__(1024) char tc_smem[];
  TcState s;
  tc_setup(s, tc_smem, np);
  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    if (!tc_update_unit(s, maps, tiles[3 * t], tiles[3 * t + 1], tiles[3 * t + 2], abort_flag, status)) break;
  }
  tc_teardown(s);
}

}  // namespace ticc
