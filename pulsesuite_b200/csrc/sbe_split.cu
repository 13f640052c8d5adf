// sbe_split.cu -- split-precision batched SBE RK4 step on the 5th-generation
// tensor cores (tcgen05 / TMEM), sm_100a.
//
// The exchange sums of every right-hand side (pulsesuite/PSTD3D/SBEs.py:
// 896-921) are, for W wires sharing one k grid, one dense contraction
//     D[k][(w,v)] = sum_k' T[k][k'] X[k'][(w,v)],   T[k][k'] = V(|k-k'|)/vscale
// with X the stage state (v: p_re, p_im, ne, nh).  T and X are split into
// bf16 hi + lo parts and D = Th Xh + Th Xl + Tl Xh is accumulated in FP32 in
// tensor memory (the lo*lo term is below FP32 resolution of the sum).
//
// One CTA owns a group of W wires for all `nsteps` RK4 steps:
//   * X (bf16 hi and lo, the MMA B operand, N = 4W columns, wire-major) lives
//     in shared memory for the whole call;
//   * the T tiles (MMA A operand, 128 k rows x 64 k' per tile, built once per
//     grid by psb_split_prepare and L2-resident) stream through a two-slot
//     ring filled with cp.async.bulk by a producer warp;
//   * one thread of the MMA warp issues tcgen05.mma (M = 128, N = 4W, K = 16)
//     into one TMEM accumulator block per 128-row tile of k;
//   * eight epilogue warps read the accumulators (tcgen05.ld), evaluate the
//     diagonal SBE right-hand side in FP32, combine the RK4 stages in FP64
//     (stage order of libpulsesuite/integrator.py:143-157), and write the next
//     stage's X back into shared memory.
// Every mbarrier wait is bounded; on a timeout the CTA records
// PSB_ERR_TIMEOUT in its wires' status, drains, frees TMEM and returns.
#include <cuda_bf16.h>
#include <math.h>

#include "psb_common.cuh"

namespace psb {
namespace split {

constexpr int kEpiWarps = 8;
constexpr int kProducerWarp = 8;
constexpr int kMmaWarp = 9;
constexpr int kThreadsS = 32 * 10;
constexpr int kNSlot = 2;
constexpr int kTileRows = 128;  // M of one MMA / rows of a T tile
constexpr int kTileK = 64;      // k' per T tile
constexpr int kLimbBytes = kTileRows * kTileK * 2;  // 16 KiB per bf16 limb
constexpr uint32_t kSpinLimit = 1u << 26;

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
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
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
// Bounded wait; false when the limit ran out or another role aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort) return false;
  }
  *abort = 1;
  return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accum) {
  uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
          d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum), "r"(m0), "r"(m1), "r"(m2), "r"(m3));
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
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor, no swizzle (canonical interleaved layout
// of 8 x 16-byte core matrices): start address, leading-dimension (K) and
// stride-dimension (M/N) byte offsets, descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: D f32, A and B bf16, A K-major,
// B MN-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 16) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(kTileRows >> 4) << 24);
}

// Byte offset of element (row r, k c) in a 128 x 64 T tile (K-major):
// K-groups of 8 at 2048 B, row groups of 8 at 128 B, rows at 16 B.
__host__ __device__ __forceinline__ uint32_t tile_off(int r, int c) {
  return (uint32_t)((c >> 3) * 2048 + (r >> 3) * 128 + (r & 7) * 16 + (c & 7) * 2);
}
// Byte offset of element (k, col) in the X operand (MN-major, N columns
// contiguous inside a core matrix): column groups at sbo, k groups at 128 B.
__device__ __forceinline__ uint32_t x_off(int k, int col, uint32_t sbo) {
  return (uint32_t)((col >> 3) * sbo + (k >> 3) * 128 + (k & 7) * 16 + (col & 7) * 2);
}

__host__ __device__ inline int kpad_of(int nk) { return (nk + kTileK - 1) / kTileK * kTileK; }
__host__ __device__ inline int mtiles_of(int nk) { return (nk + kTileRows - 1) / kTileRows; }

struct Args {
  const PsbTable* tables;
  int ntab;
  const double* tabdata;
  int64_t n_tabdata;
  PsbWire* wires;
  int nw;
  const PsbSplitTable* stab;
  const uint8_t* tiles;
  int64_t n_tiles;
  const PsbSplitGroup* groups;
  int ngroups;
  double* y;
  int64_t n_state;
  float4* ws_ys;
  double4* ws_acc;
  int nsteps;
  double dt;
  double* P;
  int64_t n_P;
  int p_stride;
  int p_cap;
  double hbar;
};

template <int W>
struct Layout {
  static constexpr int N = 4 * W;
  uint32_t x_hi, x_lo, ring, bars, misc, total;
  __host__ __device__ Layout(int kpad) {
    uint32_t xb = (uint32_t)kpad * N * 2;
    x_hi = 0;
    x_lo = x_hi + xb;
    ring = x_lo + xb;
    bars = ring + kNSlot * 2 * kLimbBytes;
    misc = bars + 8 * (2 * kNSlot + 2);  // full[], empty[], dready, final
    // misc: tmem base (16 B), abort (16 B), M re/im float2[W], wire params
    // (gap, gamma, mscale, pscale: float4[W]), t double[W], off int64[W],
    // P partials double[2][4][W]
    total = misc + 32 + 8 * W + 16 * W + 8 * W + 8 * W + 64 * W;
  }
};

// ---------------------------------------------------------------------------
// The kernel.
// ---------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(kThreadsS, 1) split_rk4_kernel(Args a) {
  constexpr int N = 4 * W;
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const PsbSplitGroup grp = a.groups[blockIdx.x];

  // ---- validate the group (uniform across the CTA) -------------------------
  bool ok = grp.table >= 0 && grp.table < a.ntab && grp.nw >= 1 && grp.nw <= W;
  PsbTable tb{};
  PsbSplitTable st{};
  if (ok) {
    tb = a.tables[grp.table];
    st = a.stab[grp.table];
    ok = tb.nk >= 2 && tb.nk <= PSB_MAX_NK && st.kpad == kpad_of(tb.nk) &&
         (st.tile_off & 15) == 0 && st.kpad * N * 4 <= 128 * 1024 &&
         st.mtiles == mtiles_of(tb.nk) && st.mtiles * N <= 512 && st.tile_off >= 0 &&
         st.tile_off + (int64_t)st.mtiles * (st.kpad / kTileK) * 2 * kLimbBytes <= a.n_tiles &&
         tb.off >= 0 && tb.off + 9 * (int64_t)tb.nk <= a.n_tabdata &&
         (tb.flags & PSB_TAB_EXCITONS) && (tb.flags & PSB_TAB_SHARED_V) &&
         !(tb.flags & PSB_TAB_SCREENED);
    for (int i = 0; ok && i < grp.nw; ++i) {
      int wi = grp.wire[i];
      ok = wi >= 0 && wi < a.nw && a.wires[wi].table == grp.table && a.wires[wi].off >= 0 &&
           a.wires[wi].off + tb.nk <= a.n_state;
    }
  }
  if (!ok) {
    if (tid < W && tid < grp.nw && grp.wire[tid] >= 0 && grp.wire[tid] < a.nw)
      a.wires[grp.wire[tid]].status = PSB_ERR_INVALID;
    return;
  }
  const int nk = tb.nk, kpad = st.kpad, nM = st.mtiles, nK = kpad / kTileK;
  const Layout<W> L(kpad);
  uint8_t* xh = smem + L.x_hi;
  uint8_t* xl = smem + L.x_lo;
  uint8_t* ring = smem + L.ring;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.bars);
  uint64_t* empty = full + kNSlot;
  uint64_t* dready = empty + kNSlot;
  uint64_t* final_bar = dready + 1;  // teardown: all MMAs of this CTA done
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + L.misc);
  volatile int* abort = reinterpret_cast<volatile int*>(smem + L.misc + 16);
  // abort as seen at each stage's end barrier (written by one participant
  // before the barrier, read by all after it, so every role breaks together)
  volatile int* snap = reinterpret_cast<volatile int*>(smem + L.misc + 20);
  float2* Msh = reinterpret_cast<float2*>(smem + L.misc + 32);
  float4* wpar = reinterpret_cast<float4*>(smem + L.misc + 32 + 8 * W);
  double* wt = reinterpret_cast<double*>(smem + L.misc + 32 + 24 * W);
  int64_t* woff = reinterpret_cast<int64_t*>(smem + L.misc + 32 + 32 * W);
  double* ppart = reinterpret_cast<double*>(smem + L.misc + 32 + 40 * W);
  const uint32_t xsbo = (uint32_t)(kpad / 8) * 128;

  // ---- set-up ---------------------------------------------------------------
  for (uint32_t i = tid * 16; i < 2 * (uint32_t)kpad * N * 2; i += kThreadsS * 16)
    *reinterpret_cast<uint4*>(smem + i) = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    for (int s = 0; s < kNSlot; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(dready, 1);
    mbar_init(final_bar, 1);
    *abort = 0;
    snap[0] = 0;
    snap[1] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < W) {
    if (tid < grp.nw) {
      const PsbWire& w = a.wires[grp.wire[tid]];
      wpar[tid] = make_float4((float)w.gap, (float)w.gamma, (float)w.mscale, (float)w.pscale);
      wt[tid] = w.t;
      woff[tid] = w.off;
    } else {
      wpar[tid] = make_float4(0.f, 0.f, 0.f, 0.f);
      wt[tid] = 0.0;
      woff[tid] = -1;
    }
  }
  int ncols = 32;
  while (ncols < nM * N) ncols <<= 1;
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const double* blk = a.tabdata + tb.off;
  const double* Ee = blk + 3 * nk;
  const double* Eh = blk + 4 * nk;
  const float vscale = (float)st.vscale;
  const float inv_hbar = (float)(1.0 / a.hbar);
  const double h = a.dt;

  // ---- epilogue-role helpers --------------------------------------------------
  const int q = warp & 3;                // TMEM lane quarter
  const int hh = warp >> 2;              // wire half
  const int w0 = hh * (W / 2);           // first wire of this warp
  auto store_x = [&](int k, int w, const float v[4]) {
    __nv_bfloat16 hi[4], lo[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      hi[c] = __float2bfloat16_rn(v[c]);
      lo[c] = __float2bfloat16_rn(v[c] - __bfloat162float(hi[c]));
    }
    uint32_t o = x_off(k, 4 * w, xsbo);
    uint2 ph, pl;
    ph.x = (uint32_t)__bfloat16_as_ushort(hi[0]) | ((uint32_t)__bfloat16_as_ushort(hi[1]) << 16);
    ph.y = (uint32_t)__bfloat16_as_ushort(hi[2]) | ((uint32_t)__bfloat16_as_ushort(hi[3]) << 16);
    pl.x = (uint32_t)__bfloat16_as_ushort(lo[0]) | ((uint32_t)__bfloat16_as_ushort(lo[1]) << 16);
    pl.y = (uint32_t)__bfloat16_as_ushort(lo[2]) | ((uint32_t)__bfloat16_as_ushort(lo[3]) << 16);
    *reinterpret_cast<uint2*>(xh + o) = ph;
    *reinterpret_cast<uint2*>(xl + o) = pl;
  };

  // Stage-0 input: X = split(y), ys = y (fp32), for this thread's elements.
  if (warp < kEpiWarps) {
    for (int mi = 0; mi < nM; ++mi) {
      const int k = mi * kTileRows + 32 * q + lane;
      if (k >= nk) continue;
      for (int j = 0; j < W / 2; ++j) {
        const int w = w0 + j;
        if (w >= grp.nw) break;
        const int64_t e = woff[w] + k;
        const double4 yv = reinterpret_cast<const double4*>(a.y)[e];
        float v[4] = {(float)yv.x, (float)yv.y, (float)yv.z, (float)yv.w};
        a.ws_ys[e] = make_float4(v[0], v[1], v[2], v[3]);
        store_x(k, w, v);
      }
    }
    fence_async_smem();
  }
  __syncthreads();

  const uint32_t idesc = idesc_bf16(N);
  const int total_iters = a.nsteps * 4;  // stages

  if (warp == kProducerWarp) {
    // ---- producer: stream the T tiles of every stage through the ring -------
    if (lane == 0) {
      const uint8_t* tiles = a.tiles + st.tile_off;
      uint32_t it = 0;
      for (int s = 0; s < total_iters && !*abort; ++s) {
        for (int mi = 0; mi < nM && !*abort; ++mi) {
          for (int kj = 0; kj < nK; ++kj, ++it) {
            const int slot = it % kNSlot;
            const uint32_t round = it / kNSlot;
            if (round > 0 && !mbar_wait(&empty[slot], (round - 1) & 1, abort)) break;
            uint8_t* dst = ring + slot * 2 * kLimbBytes;
            const uint8_t* src = tiles + ((size_t)(mi * nK + kj) * 2) * kLimbBytes;
            mbar_arrive_expect_tx(&full[slot], 2 * kLimbBytes);
            bulk_g2s(dst, src, kLimbBytes, &full[slot]);
            bulk_g2s(dst + kLimbBytes, src + kLimbBytes, kLimbBytes, &full[slot]);
          }
        }
      }
      // Drain: wait (bounded) until the consumer released every slot we
      // filled, so no bulk copy is in flight when the CTA exits.
      for (uint32_t j = (it > kNSlot ? it - kNSlot : 0); j < it; ++j) {
        const int slot = j % kNSlot;
        for (uint32_t i = 0; i < kSpinLimit; ++i)
          if (mbar_try_wait(&full[slot], (j / kNSlot) & 1)) break;
      }
    }
  } else if (warp == kMmaWarp) {
    // ---- MMA issuer -----------------------------------------------------------
    uint32_t it = 0;
    for (int s = 0; s < total_iters; ++s) {
      if (lane == 0 && !*abort) {
        tc_fence_after();
        for (int mi = 0; mi < nM; ++mi) {
          const uint32_t dcol = tmem + (uint32_t)(mi * N);
          for (int kj = 0; kj < nK; ++kj, ++it) {
            const int slot = it % kNSlot;
            if (!mbar_wait(&full[slot], (it / kNSlot) & 1, abort)) break;
            tc_fence_after();
            const uint32_t ah = smem_u32(ring + slot * 2 * kLimbBytes);
            const uint32_t al = ah + kLimbBytes;
#pragma unroll
            for (int ks = 0; ks < kTileK / 16; ++ks) {
              const int k0 = kj * kTileK + ks * 16;
              const uint64_t dah = smem_desc(ah + ks * 4096, 2048, 128);
              const uint64_t dal = smem_desc(al + ks * 4096, 2048, 128);
              const uint64_t dbh = smem_desc(smem_u32(xh) + (k0 >> 3) * 128, 128, xsbo);
              const uint64_t dbl = smem_desc(smem_u32(xl) + (k0 >> 3) * 128, 128, xsbo);
              umma_bf16(dcol, dah, dbh, idesc, (kj | ks) != 0);
              umma_bf16(dcol, dah, dbl, idesc, 1);
              umma_bf16(dcol, dal, dbh, idesc, 1);
            }
            umma_commit(&empty[slot]);  // slot reusable once these MMAs finish
          }
          if (*abort) break;
        }
        umma_commit(dready);
      }
      __syncwarp();
      // wait for the epilogue to publish the next stage's X
      named_sync(1, 32 * (kEpiWarps + 1));
      if (snap[s & 1]) break;
    }
  } else {
    // ---- epilogue warps ---------------------------------------------------------
    for (int s = 0; s < total_iters; ++s) {
      const int stg = s & 3;
      // drive of this stage for the group's wires (fp32 is enough: M enters
      // the RHS as an additive fp32 term)
      if (warp == 0 && lane < grp.nw) {
        const PsbWire& w = a.wires[grp.wire[lane]];
        const double t = wt[lane] + (stg == 0 ? 0.0 : (stg == 3 ? h : h / 2.0));
        double er = 0.0, ei = 0.0;
        for (int j = 0; j < w.npulse && j < 2; ++j) {
          const double u = (t - w.t0[j]) / w.fwhm[j];
          const double env = w.amp[j] * exp(-4.0 * log(2.0) * u * u);
          double sn, cs;
          sincos(w.phase[j], &sn, &cs);
          er += env * cs;
          ei += env * sn;
        }
        Msh[lane] = make_float2((float)(-w.mscale * er), (float)(-w.mscale * ei));
      }
      named_sync(2, 32 * kEpiWarps);
      const bool got = mbar_wait(dready, s & 1, abort);
      tc_fence_after();
      if (got) {
        double pr[W / 2], pim[W / 2];
#pragma unroll
        for (int j = 0; j < W / 2; ++j) pr[j] = pim[j] = 0.0;
        for (int mi = 0; mi < nM; ++mi) {
          const int k = mi * kTileRows + 32 * q + lane;
          float d[2 * W];
#pragma unroll
          for (int c = 0; c < 2 * W; c += 16)
            tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(mi * N + 2 * W * hh + c),
                      d + c);
          if (k >= nk) continue;
          const float ee = (float)Ee[k], eh = (float)Eh[k];
#pragma unroll
          for (int j = 0; j < W / 2; ++j) {
            const int w = w0 + j;
            if (w >= grp.nw) break;
            const int64_t e = woff[w] + k;
            const float4 par = wpar[w];
            const float2 M = Msh[w];
            const float4 ys = a.ws_ys[e];
            // exchange sums (SBEs.py:896-921) and the diagonal RHS
            // (SBEs.py:1962-1975, 2325-2337, 2623-2636) in fp32
            const float omr = M.x + vscale * d[4 * j + 0];
            const float omi = M.y + vscale * d[4 * j + 1];
            const float se = (ee + par.x) - vscale * d[4 * j + 2];
            const float sh = eh - vscale * d[4 * j + 3];
            const float sum = se + sh;
            const float nn = ys.z + ys.w - 1.0f;
            const float xr = sum * ys.x - omr * nn;
            const float xi = sum * ys.y - omi * nn;
            const float hg = par.y;  // gamma
            float f[4];
            f[0] = xi * inv_hbar - hg * ys.x;
            f[1] = -xr * inv_hbar - hg * ys.y;
            const float u = omi * ys.x - omr * ys.y;
            f[2] = 2.0f * u * inv_hbar;
            f[3] = f[2];
            // RK4 stage combination in fp64 (integrator.py:143-157):
            // acc = k1 + 2 k2 + 2 k3, y += h/6 (acc + k4)
            double4 yv = reinterpret_cast<const double4*>(a.y)[e];
            double4 acc;
            double nxt[4];
            const double yy[4] = {yv.x, yv.y, yv.z, yv.w};
            if (stg == 0) {
              acc = make_double4(f[0], f[1], f[2], f[3]);
#pragma unroll
              for (int c = 0; c < 4; ++c) nxt[c] = yy[c] + (h / 2.0) * (double)f[c];
            } else if (stg == 3) {
              acc = a.ws_acc[e];
              const double ac[4] = {acc.x, acc.y, acc.z, acc.w};
#pragma unroll
              for (int c = 0; c < 4; ++c) nxt[c] = yy[c] + (h / 6.0) * (ac[c] + (double)f[c]);
              // state stored with p rounded to fp32 (the split form's
              // working precision), densities in fp64
              yv = make_double4((double)(float)nxt[0], (double)(float)nxt[1], nxt[2], nxt[3]);
              reinterpret_cast<double4*>(a.y)[e] = yv;
              pr[j] += yv.x;
              pim[j] += yv.y;
            } else {
              acc = a.ws_acc[e];
              acc.x += 2.0 * (double)f[0];
              acc.y += 2.0 * (double)f[1];
              acc.z += 2.0 * (double)f[2];
              acc.w += 2.0 * (double)f[3];
              const double c2 = stg == 1 ? h / 2.0 : h;
#pragma unroll
              for (int c = 0; c < 4; ++c) nxt[c] = yy[c] + c2 * (double)f[c];
            }
            if (stg != 3) a.ws_acc[e] = acc;
            float v[4] = {(float)nxt[0], (float)nxt[1], (float)nxt[2], (float)nxt[3]};
            if (stg == 3) {
              v[0] = (float)yv.x;
              v[1] = (float)yv.y;
              v[2] = (float)yv.z;
              v[3] = (float)yv.w;
            }
            a.ws_ys[e] = make_float4(v[0], v[1], v[2], v[3]);
            store_x(k, w, v);
          }
        }
        if (stg == 3) {
          // P(t) = pscale * sum_k p_k, reduced in a fixed order
#pragma unroll
          for (int j = 0; j < W / 2; ++j) {
            double sr = pr[j], si = pim[j];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
              sr += __shfl_xor_sync(0xffffffffu, sr, o);
              si += __shfl_xor_sync(0xffffffffu, si, o);
            }
            if (lane == 0) {
              ppart[(0 * 4 + q) * W + w0 + j] = sr;
              ppart[(1 * 4 + q) * W + w0 + j] = si;
            }
          }
        }
      }
      fence_async_smem();
      tc_fence_before();
      named_sync(2, 32 * kEpiWarps);
      if (stg == 3 && warp == 0 && lane < grp.nw) {
        const int w = lane;
        const int step = s >> 2;
        wt[w] = wt[w] + h;
        if (a.P && a.p_stride > 0 && (step + 1) % a.p_stride == 0) {
          const int r = (step + 1) / a.p_stride - 1;
          const PsbWire& wd = a.wires[grp.wire[w]];
          if (r < a.p_cap && wd.p_off >= 0 && wd.p_off + r < a.n_P) {
            double sr = 0.0, si = 0.0;
            for (int qq = 0; qq < 4; ++qq) {
              sr += ppart[(0 * 4 + qq) * W + w];
              si += ppart[(1 * 4 + qq) * W + w];
            }
            a.P[2 * (wd.p_off + r)] = (double)wpar[w].w * sr;
            a.P[2 * (wd.p_off + r) + 1] = (double)wpar[w].w * si;
          }
        }
      }
      if (warp == 0 && lane == 0) snap[s & 1] = *abort;
      named_sync(1, 32 * (kEpiWarps + 1));
      if (snap[s & 1]) break;
    }
  }

  // ---- teardown -----------------------------------------------------------------
  if (warp == kMmaWarp && lane == 0) {
    // every MMA this thread issued has completed before TMEM is released
    umma_commit(final_bar);
    for (uint32_t i = 0; i < kSpinLimit; ++i)
      if (mbar_try_wait(final_bar, 0)) break;
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(ncols));
  if (tid < grp.nw) {
    PsbWire* wp = a.wires + grp.wire[tid];
    if (*abort) {
      wp->status = PSB_ERR_TIMEOUT;
    } else {
      wp->t = wt[tid];
      wp->steps += a.nsteps;
      bool bad = false;
      for (int k = 0; k < nk; ++k) {
        const double4 yv = reinterpret_cast<const double4*>(a.y)[woff[tid] + k];
        bad |= !(isfinite(yv.x) && isfinite(yv.y) && isfinite(yv.z) && isfinite(yv.w));
      }
      if (bad && wp->status == PSB_OK) wp->status = PSB_ERR_NONFINITE;
    }
  }
}

// T tiles of one grid: tile (mi, kj) holds rows k = 128 mi + r and columns
// k' = 64 kj + c of T[k][k'] = V(|k - k'|)/vscale (0 on the diagonal, the
// excluded q = 0 term, and outside the grid), hi limb then lo limb.
__global__ void prepare_tiles_kernel(const double* __restrict__ V, int nk, double vscale,
                                     uint8_t* __restrict__ tiles) {
  const int kpad = kpad_of(nk), nK = kpad / kTileK, nM = mtiles_of(nk);
  const int64_t total = (int64_t)nM * nK * kTileRows * kTileK;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % kTileK);
    const int r = (int)((i / kTileK) % kTileRows);
    const int64_t t = i / ((int64_t)kTileK * kTileRows);
    const int kj = (int)(t % nK), mi = (int)(t / nK);
    const int k = mi * kTileRows + r, kp = kj * kTileK + c;
    float v = 0.f;
    if (k < nk && kp < nk && k != kp) v = (float)(V[k > kp ? k - kp : kp - k] / vscale);
    const __nv_bfloat16 hi = __float2bfloat16_rn(v);
    const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
    uint8_t* tb = tiles + (size_t)(mi * nK + kj) * 2 * kLimbBytes;
    *reinterpret_cast<__nv_bfloat16*>(tb + tile_off(r, c)) = hi;
    *reinterpret_cast<__nv_bfloat16*>(tb + kLimbBytes + tile_off(r, c)) = lo;
  }
}

template <int W>
int launch(const Args& a, int kpad_max, cudaStream_t s) {
  const Layout<W> L(kpad_max);
  if (L.total > 227 * 1024)
    return set_error(PSB_ERR_SIZE, "split form: %u bytes of shared memory for kpad %d, W %d",
                     L.total, kpad_max, W);
  cudaError_t e = cudaFuncSetAttribute(split_rk4_kernel<W>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
  if (e != cudaSuccess)
    return set_error(PSB_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
  split_rk4_kernel<W><<<a.ngroups, kThreadsS, L.total, s>>>(a);
  return check_cuda("split_rk4_kernel");
}

}  // namespace split
}  // namespace psb

using namespace psb;

extern "C" int64_t psb_split_tile_bytes(int nk) {
  if (nk < 2 || nk > PSB_MAX_NK) return set_error(PSB_ERR_SIZE, "nk %d out of range", nk);
  return (int64_t)split::mtiles_of(nk) * (split::kpad_of(nk) / split::kTileK) * 2 *
         split::kLimbBytes;
}

extern "C" int64_t psb_split_ws_bytes(int64_t n_state) {
  if (n_state < 0) return set_error(PSB_ERR_INVALID, "n_state < 0");
  return 48 * n_state + 32;
}

extern "C" int psb_split_smem_bytes(int nk, int wgroup) {
  if (nk < 2 || nk > PSB_MAX_NK) return set_error(PSB_ERR_SIZE, "nk %d out of range", nk);
  const int kp = split::kpad_of(nk);
  if (wgroup == 16) return (int)split::Layout<16>(kp).total;
  if (wgroup == 8) return (int)split::Layout<8>(kp).total;
  return set_error(PSB_ERR_INVALID, "wgroup must be 8 or 16");
}

extern "C" int psb_split_prepare(const double* d_V, int nk, double vscale, void* d_tiles,
                                 int64_t n_tiles_bytes, void* stream) {
  if (!d_V || !d_tiles || !(vscale > 0.0))
    return set_error(PSB_ERR_INVALID, "psb_split_prepare: bad arguments");
  if (nk < 2 || nk > PSB_MAX_NK) return set_error(PSB_ERR_SIZE, "nk %d out of range", nk);
  if (((uintptr_t)d_tiles & 15) != 0)
    return set_error(PSB_ERR_INVALID, "psb_split_prepare: tiles must be 16-byte aligned");
  if (n_tiles_bytes < psb_split_tile_bytes(nk))
    return set_error(PSB_ERR_SIZE, "psb_split_prepare: tile buffer too small");
  split::prepare_tiles_kernel<<<148 * 4, 256, 0, (cudaStream_t)stream>>>(d_V, nk, vscale,
                                                                          (uint8_t*)d_tiles);
  return check_cuda("psb_split_prepare");
}

extern "C" int psb_rk4_split(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                             int64_t n_tabdata, PsbWire* d_wires, int nw,
                             const PsbSplitTable* d_stab, const void* d_tiles,
                             int64_t n_tiles_bytes, const PsbSplitGroup* d_groups, int ngroups,
                             int wgroup, int nkmax, double* d_y, int64_t n_state, void* d_ws,
                             int64_t n_ws_bytes, int nsteps, double dt, double* d_P, int64_t n_P,
                             int p_stride, int p_cap, const PsbModel* model, void* stream) {
  if (!d_tables || !d_tabdata || !d_wires || !d_stab || !d_tiles || !d_groups || !d_y ||
      !d_ws || !model || ntab <= 0 || nw < 0 || ngroups < 0)
    return set_error(PSB_ERR_INVALID, "psb_rk4_split: null pointer or bad count");
  if (wgroup != 8 && wgroup != 16)
    return set_error(PSB_ERR_INVALID, "psb_rk4_split: wgroup must be 8 or 16");
  if (nkmax < 2 || nkmax > PSB_MAX_NK || (wgroup == 16 && nkmax > 512))
    return set_error(PSB_ERR_SIZE, "psb_rk4_split: nkmax %d too large for wgroup %d", nkmax,
                     wgroup);
  if (n_ws_bytes < psb_split_ws_bytes(n_state))
    return set_error(PSB_ERR_SIZE, "psb_rk4_split: workspace needs psb_split_ws_bytes(n_state)");
  if (((uintptr_t)d_ws & 31) != 0 || ((uintptr_t)d_y & 31) != 0)
    return set_error(PSB_ERR_INVALID, "psb_rk4_split: state and workspace must be 32-byte aligned");
  if (!(model->hbar > 0.0)) return set_error(PSB_ERR_INVALID, "model.hbar must be > 0");
  if (nsteps < 0) return set_error(PSB_ERR_INVALID, "nsteps < 0");
  if (nsteps == 0 || ngroups == 0) return PSB_OK;
  split::Args a{};
  a.tables = d_tables;
  a.ntab = ntab;
  a.tabdata = d_tabdata;
  a.n_tabdata = n_tabdata;
  a.wires = d_wires;
  a.nw = nw;
  a.stab = d_stab;
  a.tiles = (const uint8_t*)d_tiles;
  a.n_tiles = n_tiles_bytes;
  a.groups = d_groups;
  a.ngroups = ngroups;
  a.y = d_y;
  a.n_state = n_state;
  a.ws_ys = (float4*)d_ws;
  a.ws_acc = (double4*)((uint8_t*)d_ws + ((16 * n_state + 31) & ~(int64_t)31));
  a.nsteps = nsteps;
  a.dt = dt;
  a.P = d_P;
  a.n_P = n_P;
  a.p_stride = p_stride;
  a.p_cap = p_cap;
  a.hbar = model->hbar;
  const int kp = split::kpad_of(nkmax);
  return wgroup == 16 ? split::launch<16>(a, kp, (cudaStream_t)stream)
                      : split::launch<8>(a, kp, (cudaStream_t)stream);
}
