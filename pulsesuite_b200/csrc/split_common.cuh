// split_common.cuh -- constants and PTX helpers shared by the split-precision
// tensor-core kernels (sbe_split.cu: one Coulomb matrix shared by a group of
// wires; sbe_split_wire.cu: one matrix per wire).  sm_100a only.
#pragma once

#include <math.h>
#include <stdint.h>

#include "psb_common.cuh"

namespace psb {
namespace split {

constexpr int kEpiWarps = 8;    // warps 0..7: drain + epilogue (warpgroups 0, 1)
constexpr int kGenWarp0 = 8;    // warps 8..11: A-tile generators (warpgroup 2)
constexpr int kGenWarps = 4;
constexpr int kMmaWarp = 12;    // warp 12: TMEM owner + MMA issuer (warpgroup 3;
                                // warps 13..15 only complete that warpgroup)
constexpr int kThreadsS = 32 * 16;
constexpr int kEpiThreads = 32 * kEpiWarps;
// Registers per thread: 128 at launch (65536 / 512 threads); after the
// set-up the generator and MMA warpgroups give theirs down to kRegsLow and
// the two epilogue warpgroups take them: 256 kRegsHigh + 256 kRegsLow =
// 512 * kRegsLaunch, so the increase always finds its registers.
constexpr int kRegsLaunch = 128;
constexpr int kRegsLow = 64;
constexpr int kRegsHigh = 2 * kRegsLaunch - kRegsLow;  // 192
static_assert(kEpiWarps * 32 * kRegsHigh + (kThreadsS - kEpiWarps * 32) * kRegsLow <=
                  kThreadsS * kRegsLaunch,
              "register split exceeds the launch allocation");
constexpr int kTileRows = 128;  // M of one MMA
constexpr int kTileK = 64;      // k' per A tile
constexpr int kDigits = 3;
constexpr int kPlaneCols = kTileK / 4;            // TMEM columns of one digit plane of a tile
constexpr int kTileCols = kDigits * kPlaneCols;   // 48
constexpr int kTmemCols = 512;
constexpr double kBase = 254.0;
// Polls of one bounded hand-off wait before it gives up (the default of
// psb_split_set_wait_limit; the teardown wait for the last MMAs always uses
// this value).
constexpr uint32_t kSpinLimit = 1u << 26;
// dynamic shared memory per CTA (the 227 KiB limit less the static
// shared memory and alignment padding)
constexpr uint32_t kMaxDynSmem = 226 * 1024;

// ---------------------------------------------------------------------------
// PTX helpers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Non-blocking probe of a phase (no suspension of the waiting thread).
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded spin on a phase; false when the limit ran out (which also sets
// abort) or another role aborted.  Spinning with test_wait rather than
// suspending in try_wait keeps the hand-off latency between the MMA issuer,
// the generators and the drain warps short.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort,
                                          uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i) {
    if (mbar_test_wait(bar, parity)) return true;
    if (*abort) return false;
  }
  *abort = 1;
  return false;
}
// Bounded wait that suspends in try_wait between probes instead of
// spinning: for roles that wait long (issuers and generators waiting on the
// epilogue), so that their polling does not take issue slots from the warps
// doing the arithmetic.  Same contract as mbar_wait.
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t* bar, uint32_t parity,
                                                volatile int* abort, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort) return false;
  }
  *abort = 1;
  return false;
}
// D[tmem] (+)= A[tmem] * B[smem desc], int8 x int8 -> int32
__device__ __forceinline__ void umma_i8(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accum));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void named_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
// 8 consecutive TMEM columns of this thread's lane (no wait: pair with
// tmem_ld_wait before the registers are used)
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t* r) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
      "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15])
      : "memory");
}

// Three balanced base-254 digits of v, |v| < 1/2 (so |254 v| < 127): each
// remainder is formed exactly with an FMA, every digit lies in [-127, 127].
// (Values outside the range give meaningless digits; the callers detect
// them and re-digitise the column with a wider scale.)
__device__ __forceinline__ void digits3(float v, int& d1, int& d2, int& d3) {
  // x + 1.5 * 2^23 rounds x (|x| < 2^22) to the nearest integer in one FMA
  // rounding, and that integer is the sum's bit pattern less the constant's:
  // plain FP32 and integer arithmetic instead of a conversion per digit.
  constexpr float kMagic = 12582912.f;
  constexpr int kMagicBits = 0x4B400000;
  const float t1 = fmaf(v, 254.f, kMagic);
  const float r1 = fmaf(v, 254.f, -(t1 - kMagic));
  const float t2 = fmaf(r1, 254.f, kMagic);
  const float r2 = fmaf(r1, 254.f, -(t2 - kMagic));
  const float t3 = fmaf(r2, 254.f, kMagic);
  d1 = __float_as_int(t1) - kMagicBits;
  d2 = __float_as_int(t2) - kMagicBits;
  d3 = __float_as_int(t3) - kMagicBits;
}

// One step of a halving max-butterfly over a warp: each lane holds C
// values, sends half of them to the lane `o` apart and keeps the maxima of
// the other half (the lane with bit o set keeps the upper half).
template <int C>
__device__ __forceinline__ void colmax_halve(float* v, int o, int lane) {
  const bool up = (lane & o) != 0;
#pragma unroll
  for (int i = 0; i < C / 2; ++i) {
    const float send = up ? v[i] : v[i + C / 2];
    const float keep = up ? v[i + C / 2] : v[i];
    v[i] = fmaxf(keep, __shfl_xor_sync(0xffffffffu, send, o));
  }
}

// Shared-memory matrix descriptor, no swizzle (canonical layout of 8-row x
// 16-byte core matrices): start address, leading-dimension (K) byte offset,
// stride-dimension (M/N) byte offset, descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::i8: D s32, A and B signed 8-bit, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_i8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(kTileRows >> 4) << 24);
}

__host__ __device__ inline int kpad_of(int nk) { return (nk + kTileK - 1) / kTileK * kTileK; }
__host__ __device__ inline int mtiles_of(int nk) { return (nk + kTileRows - 1) / kTileRows; }
// Distinct A tiles of a grid: one per value of 2 mi - kj.
__host__ __device__ inline int ntiles_of(int nk) {
  return kpad_of(nk) / kTileK + 2 * (mtiles_of(nk) - 1);
}

// Polls of a bounded hand-off wait for launches issued now (set by
// psb_split_set_wait_limit; host side).
uint32_t wait_limit();

}  // namespace split
}  // namespace psb
