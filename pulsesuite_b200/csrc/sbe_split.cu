// sbe_split.cu -- split-precision batched SBE RK4 step on the 5th-generation
// tensor cores (tcgen05 / TMEM), sm_100a.
//
// The exchange sums of every right-hand side (pulsesuite/PSTD3D/SBEs.py:
// 896-921) are, for W wires sharing one k grid, one dense contraction
//     D[k][(w,v)] = sum_k' T[k][k'] X[k'][(w,v)],   T[k][k'] = V(|k-k'|)/vscale
// with X the stage state (v: p_re, p_im, ne, nh).  T and X are split into
// bf16 hi + lo parts and D = Th Xh + (Th Xl + Tl Xh) is accumulated in FP32
// in tensor memory, the main product and the two corrections in separate
// accumulators that the epilogue adds in FP64 (Tl Xl is below the FP32
// resolution of the sum).
//
// One CTA owns a group of W (4, 8 or 16) wires for all `nsteps` RK4 steps:
//   * X (bf16 hi and lo, the MMA B operand, N = 4W columns, wire-major) lives
//     in shared memory for the whole call;
//   * T is Toeplitz, so it is never stored as a matrix: each 128 x 64 tile
//     of the MMA A operand is generated straight into tensor memory from a
//     table of bf16 pairs (Tv(d), Tv(d-1)) in shared memory -- one 32-bit
//     lookup per TMEM cell -- double buffered, and the MMA reads A from TMEM;
//   * one thread issues tcgen05.mma (M = 128, N = 4W, K = 16) into one TMEM
//     accumulator block per 128-row tile of k;
//   * eight warps generate the T tiles during the MMA phase and, once the
//     accumulators are complete, evaluate the diagonal SBE right-hand side,
//     combine the RK4 stages (stage order of libpulsesuite/integrator.py:
//     143-157) and write the next stage's X back into shared memory.
// The right-hand side and the stage state are FP64 (O(Nk) work per wire);
// only the O(Nk^2) exchange contraction runs in split bf16.
// Every mbarrier wait is bounded; on a timeout the CTA records
// PSB_ERR_TIMEOUT in its wires' status, waits for its MMAs, frees TMEM and
// returns.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <math.h>

#include "psb_common.cuh"

namespace psb {
namespace split {

constexpr int kEpiWarps = 8;
constexpr int kMmaWarp = 8;
constexpr int kThreadsS = 32 * 9;
constexpr int kTileRows = 128;  // M of one MMA
constexpr int kTileK = 64;      // k' per generated A tile
constexpr int kACols = kTileK / 2;  // TMEM columns of one bf16 limb of an A tile
constexpr uint32_t kSpinLimit = 1u << 26;
// dynamic shared memory per CTA (the 227 KiB limit less the static reduction
// buffer and its alignment padding)
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
// Bounded wait; false when the limit ran out (which also sets abort) or
// another role aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort) return false;
  }
  *abort = 1;
  return false;
}
// D[tmem] (+)= A[tmem] * B[smem desc]
__device__ __forceinline__ void umma_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accum) {
  uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
          d_tmem),
      "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accum), "r"(m0), "r"(m1), "r"(m2), "r"(m3));
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

// One 16-bit limb of the split: bf16 (8 significant bits) or fp16 (11
// significant bits; values are O(1) after the vscale normalisation).
template <bool F16>
__device__ __forceinline__ uint16_t limb_bits(float v, float& back) {
  if (F16) {
    const __half hv = __float2half_rn(v);
    back = __half2float(hv);
    return __half_as_ushort(hv);
  }
  const __nv_bfloat16 bv = __float2bfloat16_rn(v);
  back = __bfloat162float(bv);
  return __bfloat16_as_ushort(bv);
}
// hi and lo limbs of v (v ~ hi + lo)
template <bool F16>
__device__ __forceinline__ void split2(float v, uint16_t& hi, uint16_t& lo) {
  float b;
  hi = limb_bits<F16>(v, b);
  float b2;
  lo = limb_bits<F16>(v - b, b2);
}

// Shared-memory matrix descriptor, no swizzle (canonical interleaved layout
// of 8 x 16-byte core matrices): start address, leading-dimension (K) and
// stride-dimension (M/N) byte offsets, descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: D f32, A and B bf16 (format 1) or
// fp16 (format 0), A K-major (required for A in TMEM), B MN-major, M = 128,
// N = n.
__host__ __device__ constexpr uint32_t idesc_f16(int n, bool f16) {
  return (1u << 4) | ((f16 ? 0u : 1u) << 7) | ((f16 ? 0u : 1u) << 10) | (1u << 16) |
         ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTileRows >> 4) << 24);
}

// Byte offset of element (k, col) in the X operand (MN-major, N columns
// contiguous inside a core matrix): column groups at sbo, k groups at 128 B.
__device__ __forceinline__ uint32_t x_off(int k, int col, uint32_t sbo) {
  return (uint32_t)((col >> 3) * sbo + (k >> 3) * 128 + (k & 7) * 16 + (col & 7) * 2);
}

__host__ __device__ inline int kpad_of(int nk) { return (nk + kTileK - 1) / kTileK * kTileK; }
__host__ __device__ inline int mtiles_of(int nk) { return (nk + kTileRows - 1) / kTileRows; }
// TMEM columns: main accumulators Th*Xh (mtiles x N), correction
// accumulators Th*Xl + Tl*Xh (mtiles x N), then two A buffers (hi + lo).
// Keeping the small corrections out of the main accumulator stops every
// FP32 accumulate from dropping their low-order bits.
__host__ __device__ inline int tmem_need(int nk, int n) {
  return 2 * mtiles_of(nk) * n + 4 * kACols;
}
__host__ __device__ inline int tmem_cols(int nk, int n) {
  int need = tmem_need(nk, n);
  int c = 32;
  while (c < need) c <<= 1;
  return c;
}

struct Args {
  const PsbTable* tables;
  int ntab;
  const double* tabdata;
  int64_t n_tabdata;
  PsbWire* wires;
  int nw;
  const PsbSplitGroup* groups;
  int ngroups;
  double* y;
  int64_t n_state;
  double4* ws_ys;
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
  uint32_t x_hi, x_lo, tab, bars, misc, total;
  int ntab_words;
  __host__ __device__ Layout(int nk) {
    const int kpad = kpad_of(nk), nM = mtiles_of(nk);
    const uint32_t xb = (uint32_t)kpad * N * 2;
    x_hi = 0;
    x_lo = x_hi + xb;
    tab = x_lo + xb;
    ntab_words = kTileRows * nM + kpad;
    bars = tab + 2 * 4 * (uint32_t)ntab_words;  // hi and lo pair tables
    bars = (bars + 15) & ~15u;
    misc = bars + 8 * 8;  // afull[2], afree[2], dready, final
    // misc: tmem base (16 B), abort + snapshots (16 B), M re/im double2[W],
    // wire params (gap, gamma, mscale, pscale: double4[W]), t double[W],
    // off int64[W], P partials double[2][4][W]
    total = misc + 32 + 128 * W;
  }
};

// ---------------------------------------------------------------------------
// The kernel.
// ---------------------------------------------------------------------------
template <int W, bool F16>
__global__ void __launch_bounds__(kThreadsS, 1) split_rk4_kernel(Args a) {
  constexpr int N = 4 * W;
  constexpr int WH = W / 2;  // wires per epilogue warp
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const PsbSplitGroup grp = a.groups[blockIdx.x];

  // ---- validate the group (uniform across the CTA) -------------------------
  bool ok = grp.table >= 0 && grp.table < a.ntab && grp.nw >= 1 && grp.nw <= W;
  PsbTable tb{};
  if (ok) {
    tb = a.tables[grp.table];
    ok = tb.nk >= 2 && tb.nk <= PSB_MAX_NK && tmem_need(tb.nk, N) <= 512 &&
         tb.off >= 0 && tb.off + 9 * (int64_t)tb.nk <= a.n_tabdata &&
         (tb.flags & PSB_TAB_EXCITONS) && (tb.flags & PSB_TAB_SHARED_V) &&
         !(tb.flags & PSB_TAB_SCREENED);
    for (int i = 0; ok && i < grp.nw; ++i) {
      const int wi = grp.wire[i];
      ok = wi >= 0 && wi < a.nw && a.wires[wi].table == grp.table && a.wires[wi].off >= 0 &&
           a.wires[wi].off + tb.nk <= a.n_state;
    }
  }
  if (!ok) {
    if (tid < W && tid < grp.nw && grp.wire[tid] >= 0 && grp.wire[tid] < a.nw)
      a.wires[grp.wire[tid]].status = PSB_ERR_INVALID;
    return;
  }
  const int nk = tb.nk, kpad = kpad_of(nk), nM = mtiles_of(nk), nK = kpad / kTileK;
  const Layout<W> L(nk);
  uint8_t* xh = smem + L.x_hi;
  uint8_t* xl = smem + L.x_lo;
  uint32_t* tab_hi = reinterpret_cast<uint32_t*>(smem + L.tab);
  uint32_t* tab_lo = tab_hi + L.ntab_words;
  uint64_t* afull = reinterpret_cast<uint64_t*>(smem + L.bars);
  uint64_t* afree = afull + 2;
  uint64_t* dready = afree + 2;
  uint64_t* final_bar = dready + 1;  // teardown: all MMAs of this CTA done
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + L.misc);
  volatile int* abort = reinterpret_cast<volatile int*>(smem + L.misc + 16);
  // abort as seen at each stage's end barrier (written by one participant
  // before the barrier, read by all after it, so every role breaks together)
  volatile int* snap = reinterpret_cast<volatile int*>(smem + L.misc + 20);
  double2* Msh = reinterpret_cast<double2*>(smem + L.misc + 32);
  double4* wpar = reinterpret_cast<double4*>(smem + L.misc + 32 + 16 * W);
  double* wt = reinterpret_cast<double*>(smem + L.misc + 32 + 48 * W);
  int64_t* woff = reinterpret_cast<int64_t*>(smem + L.misc + 32 + 56 * W);
  double* ppart = reinterpret_cast<double*>(smem + L.misc + 32 + 64 * W);
  const uint32_t xsbo = (uint32_t)(kpad / 8) * 128;
  const double* blk = a.tabdata + tb.off;
  const double* Ee = blk + 3 * nk;
  const double* Eh = blk + 4 * nk;

  // ---- set-up ---------------------------------------------------------------
  // vscale: the power of two at or above max V, so T = V/vscale is exact.
  __shared__ double vmax_w[kThreadsS / 32];
  double vm = 0.0;
  for (int qq = 1 + tid; qq < nk; qq += kThreadsS) vm = fmax(vm, fabs(blk[qq]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) vm = fmax(vm, __shfl_xor_sync(0xffffffffu, vm, o));
  if (lane == 0) vmax_w[warp] = vm;
  for (uint32_t i = tid * 16; i < 2 * (uint32_t)kpad * N * 2; i += kThreadsS * 16)
    *reinterpret_cast<uint4*>(smem + i) = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    mbar_init(&afull[0], kEpiWarps);
    mbar_init(&afull[1], kEpiWarps);
    mbar_init(&afree[0], 1);
    mbar_init(&afree[1], 1);
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
      wpar[tid] = make_double4(w.gap, w.gamma, w.mscale, w.pscale);
      wt[tid] = w.t;
      woff[tid] = w.off;
    } else {
      wpar[tid] = make_double4(0.0, 0.0, 0.0, 0.0);
      wt[tid] = 0.0;
      woff[tid] = -1;
    }
  }
  const int ncols = tmem_cols(nk, N);
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
  double vmax = 0.0;
#pragma unroll
  for (int i = 0; i < kThreadsS / 32; ++i) vmax = fmax(vmax, vmax_w[i]);
  int ex = 0;
  frexp(vmax > 0.0 ? vmax : 1.0, &ex);
  const double vscale = ldexp(1.0, ex);
  const double inv_vscale = ldexp(1.0, -ex);
  // Pair tables: word(d) = (Tv(d), Tv(d-1)) for d in [2 - kpad, 128 nM - 1],
  // Tv(d) = bf16 limb of V(|d|)/vscale (0 at d = 0 and outside the grid).
  const int dlo = 2 - kpad;
  auto tv = [&](int d, uint16_t& hi, uint16_t& lo) {
    const int ad = d < 0 ? -d : d;
    const float v = (ad > 0 && ad < nk) ? (float)(blk[ad] * inv_vscale) : 0.f;
    split2<F16>(v, hi, lo);
  };
  for (int i = tid; i < L.ntab_words; i += kThreadsS) {
    const int d = dlo + i;
    uint16_t h0, l0, h1, l1;
    tv(d, h0, l0);
    tv(d - 1, h1, l1);
    tab_hi[i] = (uint32_t)h0 | ((uint32_t)h1 << 16);
    tab_lo[i] = (uint32_t)l0 | ((uint32_t)l1 << 16);
  }

  // ---- epilogue-role helpers --------------------------------------------------
  const int q = warp & 3;          // TMEM lane quarter
  const int hh = (warp >> 2) & 1;  // wire half / A column half
  const int w0 = hh * WH;          // first wire of this warp
  auto store_x = [&](int k, int w, const float v[4]) {
    uint16_t hi[4], lo[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) split2<F16>(v[c], hi[c], lo[c]);
    const uint32_t o = x_off(k, 4 * w, xsbo);
    uint2 ph, pl;
    ph.x = (uint32_t)hi[0] | ((uint32_t)hi[1] << 16);
    ph.y = (uint32_t)hi[2] | ((uint32_t)hi[3] << 16);
    pl.x = (uint32_t)lo[0] | ((uint32_t)lo[1] << 16);
    pl.y = (uint32_t)lo[2] | ((uint32_t)lo[3] << 16);
    *reinterpret_cast<uint2*>(xh + o) = ph;
    *reinterpret_cast<uint2*>(xl + o) = pl;
  };

  // Stage-0 input: X = split(y), ys = y, for this thread's elements.
  if (warp < kEpiWarps) {
    for (int mi = 0; mi < nM; ++mi) {
      const int k = mi * kTileRows + 32 * q + lane;
      if (k >= nk) continue;
      for (int j = 0; j < WH; ++j) {
        const int w = w0 + j;
        if (w >= grp.nw) break;
        const int64_t e = woff[w] + k;
        const double4 yv = reinterpret_cast<const double4*>(a.y)[e];
        const float v[4] = {(float)yv.x, (float)yv.y, (float)yv.z, (float)yv.w};
        a.ws_ys[e] = yv;
        store_x(k, w, v);
      }
    }
    fence_async_smem();
  }
  __syncthreads();

  const uint32_t idesc = idesc_f16(N, F16);
  const int total_stages = a.nsteps * 4;
  const uint32_t ccol0 = (uint32_t)(nM * N);      // first correction-accumulator column
  const uint32_t acol0 = (uint32_t)(2 * nM * N);  // first A-buffer column
  const double h = a.dt;
  const double hbar = a.hbar;

  if (warp == kMmaWarp) {
    // ---- MMA issuer -----------------------------------------------------------
    uint32_t it = 0;
    for (int s = 0; s < total_stages; ++s) {
      if (lane == 0 && !*abort) {
        tc_fence_after();
        for (int mi = 0; mi < nM; ++mi) {
          const uint32_t dcol = tmem + (uint32_t)(mi * N);
          const uint32_t ccol = tmem + ccol0 + (uint32_t)(mi * N);
          for (int kj = 0; kj < nK; ++kj, ++it) {
            const int b = it & 1;
            if (!mbar_wait(&afull[b], (it >> 1) & 1, abort)) break;
            tc_fence_after();
            const uint32_t ah = tmem + acol0 + (uint32_t)(b * 2 * kACols);
            const uint32_t al = ah + kACols;
#pragma unroll
            for (int ks = 0; ks < kTileK / 16; ++ks) {
              const int k0 = kj * kTileK + ks * 16;
              const uint64_t dbh = smem_desc(smem_u32(xh) + (k0 >> 3) * 128, 128, xsbo);
              const uint64_t dbl = smem_desc(smem_u32(xl) + (k0 >> 3) * 128, 128, xsbo);
              umma_ts(dcol, ah + ks * 8, dbh, idesc, (kj | ks) != 0);
              umma_ts(ccol, ah + ks * 8, dbl, idesc, (kj | ks) != 0);
              umma_ts(ccol, al + ks * 8, dbh, idesc, 1);
            }
            umma_commit(&afree[b]);  // buffer reusable once these MMAs finish
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
    // ---- generator / epilogue warps -----------------------------------------------
    uint32_t it = 0;
    for (int s = 0; s < total_stages; ++s) {
      const int stg = s & 3;
      // drive of this stage for the group's wires
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
        Msh[lane] = make_double2(-w.mscale * er, -w.mscale * ei);
      }
      // Generate this stage's A tiles into the two TMEM buffers, in the order
      // the MMA thread consumes them.  Row r = 32q + lane of tile (mi, kj) is
      // Tv(d0 - c), c = 0..63, d0 = 128 mi + r - 64 kj; TMEM column j of a limb
      // holds c = 2j, 2j+1, i.e. word(d0 - 2j).  This warp writes columns
      // 16 hh .. 16 hh + 15 of both limbs.
      for (int mi = 0; mi < nM && !*abort; ++mi) {
        for (int kj = 0; kj < nK; ++kj, ++it) {
          const int b = it & 1;
          const uint32_t round = it >> 1;
          if (round > 0 && !mbar_wait(&afree[b], (round - 1) & 1, abort)) break;
          const int d0 = mi * kTileRows + 32 * q + lane - kj * kTileK;
          const int base = d0 - 32 * hh - dlo;  // table index of word(d0 - 2*(16 hh))
          uint32_t rh[16], rl[16];
#pragma unroll
          for (int jj = 0; jj < 16; ++jj) {
            rh[jj] = tab_hi[base - 2 * jj];
            rl[jj] = tab_lo[base - 2 * jj];
          }
          const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16) + acol0 +
                              (uint32_t)(b * 2 * kACols + 16 * hh);
          tmem_st16(ta, rh);
          tmem_st16(ta + kACols, rl);
          asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&afull[b]);
        }
      }
      named_sync(2, 32 * kEpiWarps);
      const bool got = mbar_wait(dready, s & 1, abort);
      tc_fence_after();
      if (got) {
        double pr[WH], pim[WH];
#pragma unroll
        for (int j = 0; j < WH; ++j) pr[j] = pim[j] = 0.0;
        for (int mi = 0; mi < nM; ++mi) {
          const int k = mi * kTileRows + 32 * q + lane;
          const uint32_t lrow = tmem + ((uint32_t)(32 * q) << 16);
          const double ee = k < nk ? Ee[k] : 0.0, eh = k < nk ? Eh[k] : 0.0;
          // wires in pairs: one 8-column TMEM load per accumulator, and the
          // pair's element state loaded together for memory parallelism
#pragma unroll 1
          for (int jp = 0; jp < WH; jp += 2) {
          uint32_t d1[8], d2[8];
          tmem_ld8(lrow + (uint32_t)(mi * N + 4 * (w0 + jp)), d1);
          tmem_ld8(lrow + ccol0 + (uint32_t)(mi * N + 4 * (w0 + jp)), d2);
          tmem_ld_wait();
          if (k >= nk) continue;
          double4 ysv[2], yvv[2], accv[2];
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            if (w0 + jp + u < grp.nw) {
              const int64_t e = woff[w0 + jp + u] + k;
              ysv[u] = a.ws_ys[e];
              yvv[u] = reinterpret_cast<const double4*>(a.y)[e];
              if (stg != 0) accv[u] = a.ws_acc[e];
            }
          }
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int j = jp + u;
            const int w = w0 + j;
            if (w >= grp.nw) break;
            const int64_t e = woff[w] + k;
            const double4 par = wpar[w];
            const double2 M = Msh[w];
            const double4 ys = ysv[u];
            double ex[4];
#pragma unroll
            for (int c = 0; c < 4; ++c)
              ex[c] = vscale * ((double)__uint_as_float(d1[4 * u + c]) +
                                (double)__uint_as_float(d2[4 * u + c]));
            // exchange sums (SBEs.py:896-921) from the tensor cores, the
            // diagonal RHS (SBEs.py:1962-1975, 2325-2337, 2623-2636) in fp64
            const double omr = M.x + ex[0];
            const double omi = M.y + ex[1];
            const double se = (ee + par.x) - ex[2];
            const double sh = eh - ex[3];
            const double sum = se + sh;
            const double nn = ys.z + ys.w - 1.0;
            const double xr = sum * ys.x - omr * nn;
            const double xi = sum * ys.y - omi * nn;
            const double hg = par.y;  // gamma
            double f[4];
            f[0] = xi / hbar - hg * ys.x;
            f[1] = -xr / hbar - hg * ys.y;
            const double uu = omi * ys.x - omr * ys.y;
            f[2] = 2.0 * uu / hbar;
            f[3] = f[2];
            // RK4 stage combination in fp64 (integrator.py:143-157):
            // acc = k1 + 2 k2 + 2 k3, y += h/6 (acc + k4)
            const double4 yv = yvv[u];
            const double yy[4] = {yv.x, yv.y, yv.z, yv.w};
            double4 acc;
            double nxt[4];
            if (stg == 0) {
              acc = make_double4(f[0], f[1], f[2], f[3]);
#pragma unroll
              for (int c = 0; c < 4; ++c) nxt[c] = yy[c] + (h / 2.0) * f[c];
            } else if (stg == 3) {
              acc = accv[u];
              const double ac[4] = {acc.x, acc.y, acc.z, acc.w};
#pragma unroll
              for (int c = 0; c < 4; ++c) nxt[c] = yy[c] + (h / 6.0) * (ac[c] + f[c]);
              reinterpret_cast<double4*>(a.y)[e] = make_double4(nxt[0], nxt[1], nxt[2], nxt[3]);
              pr[j] += nxt[0];
              pim[j] += nxt[1];
            } else {
              acc = accv[u];
              acc.x += 2.0 * f[0];
              acc.y += 2.0 * f[1];
              acc.z += 2.0 * f[2];
              acc.w += 2.0 * f[3];
              const double c2 = stg == 1 ? h / 2.0 : h;
#pragma unroll
              for (int c = 0; c < 4; ++c) nxt[c] = yy[c] + c2 * f[c];
            }
            if (stg != 3) a.ws_acc[e] = acc;
            const float v[4] = {(float)nxt[0], (float)nxt[1], (float)nxt[2], (float)nxt[3]};
            a.ws_ys[e] = make_double4(nxt[0], nxt[1], nxt[2], nxt[3]);
            store_x(k, w, v);
          }
          }
        }
        if (stg == 3) {
          // P(t) = pscale * sum_k p_k, reduced in a fixed order
#pragma unroll
          for (int j = 0; j < WH; ++j) {
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
            a.P[2 * (wd.p_off + r)] = wpar[w].w * sr;
            a.P[2 * (wd.p_off + r) + 1] = wpar[w].w * si;
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

template <int W, bool F16>
int launch(const Args& a, int nkmax, cudaStream_t s) {
  uint32_t smem = 0;
  for (int nk = 2; nk <= nkmax; ++nk) {
    const uint32_t t = Layout<W>(nk).total;
    if (t > smem) smem = t;
  }
  if (smem > kMaxDynSmem || tmem_need(nkmax, 4 * W) > 512)
    return set_error(PSB_ERR_SIZE, "split form: nk %d does not fit a group of %d wires", nkmax,
                     W);
  cudaError_t e = cudaFuncSetAttribute(split_rk4_kernel<W, F16>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess)
    return set_error(PSB_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
  split_rk4_kernel<W, F16><<<a.ngroups, kThreadsS, smem, s>>>(a);
  return check_cuda("split_rk4_kernel");
}

}  // namespace split
}  // namespace psb

using namespace psb;

extern "C" int64_t psb_split_ws_bytes(int64_t n_state) {
  if (n_state < 0) return set_error(PSB_ERR_INVALID, "n_state < 0");
  return 64 * n_state + 32;
}

extern "C" int psb_split_smem_bytes(int nk, int wgroup) {
  if (nk < 2 || nk > PSB_MAX_NK) return set_error(PSB_ERR_SIZE, "nk %d out of range", nk);
  if (wgroup == 16) return (int)split::Layout<16>(nk).total;
  if (wgroup == 8) return (int)split::Layout<8>(nk).total;
  if (wgroup == 4) return (int)split::Layout<4>(nk).total;
  return set_error(PSB_ERR_INVALID, "wgroup must be 4, 8 or 16");
}

extern "C" int psb_split_max_nk(int wgroup) {
  if (wgroup != 4 && wgroup != 8 && wgroup != 16)
    return set_error(PSB_ERR_INVALID, "wgroup must be 4, 8 or 16");
  int best = 0;
  for (int nk = 2; nk <= PSB_MAX_NK; ++nk) {
    const uint32_t sm = wgroup == 16 ? split::Layout<16>(nk).total
                                     : (wgroup == 8 ? split::Layout<8>(nk).total
                                                    : split::Layout<4>(nk).total);
    if (sm <= split::kMaxDynSmem && split::tmem_need(nk, 4 * wgroup) <= 512) best = nk;
  }
  return best;
}

extern "C" int psb_rk4_split(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                             int64_t n_tabdata, PsbWire* d_wires, int nw,
                             const PsbSplitGroup* d_groups, int ngroups, int wgroup, int nkmax,
                             int limb, double* d_y, int64_t n_state, void* d_ws,
                             int64_t n_ws_bytes,
                             int nsteps, double dt, double* d_P, int64_t n_P, int p_stride,
                             int p_cap, const PsbModel* model, void* stream) {
  if (!d_tables || !d_tabdata || !d_wires || !d_groups || !d_y || !d_ws || !model || ntab <= 0 ||
      nw < 0 || ngroups < 0)
    return set_error(PSB_ERR_INVALID, "psb_rk4_split: null pointer or bad count");
  if (wgroup != 4 && wgroup != 8 && wgroup != 16)
    return set_error(PSB_ERR_INVALID, "psb_rk4_split: wgroup must be 4, 8 or 16");
  if (limb != PSB_LIMB_BF16 && limb != PSB_LIMB_FP16)
    return set_error(PSB_ERR_INVALID, "psb_rk4_split: limb must be PSB_LIMB_BF16 or _FP16");
  if (nkmax < 2 || nkmax > psb_split_max_nk(wgroup))
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
  a.groups = d_groups;
  a.ngroups = ngroups;
  a.y = d_y;
  a.n_state = n_state;
  a.ws_ys = (double4*)d_ws;
  a.ws_acc = (double4*)((uint8_t*)d_ws + 32 * n_state);
  a.nsteps = nsteps;
  a.dt = dt;
  a.P = d_P;
  a.n_P = n_P;
  a.p_stride = p_stride;
  a.p_cap = p_cap;
  a.hbar = model->hbar;
  cudaStream_t st = (cudaStream_t)stream;
  if (limb == PSB_LIMB_FP16) {
    if (wgroup == 16) return split::launch<16, true>(a, nkmax, st);
    if (wgroup == 8) return split::launch<8, true>(a, nkmax, st);
    return split::launch<4, true>(a, nkmax, st);
  }
  if (wgroup == 16) return split::launch<16, false>(a, nkmax, st);
  if (wgroup == 8) return split::launch<8, false>(a, nkmax, st);
  return split::launch<4, false>(a, nkmax, st);
}
