// sbe_split.cu -- split-precision batched SBE RK4 step on the 5th-generation
// tensor cores (tcgen05 / TMEM, kind::i8), sm_100a.
//
// The exchange sums of every right-hand side (pulsesuite/PSTD3D/SBEs.py:
// 896-921) are, for W wires sharing one k grid, one dense contraction
//     D[k][(w,v)] = sum_k' T[k][k'] X[k'][(w,v)],   T[k][k'] = V(|k-k'|)
// with X the stage point (v: p_re, p_im, ne, nh).  T and X are written as
// three signed base-254 digits each (Ozaki-style slicing onto the integer
// tensor cores):
//     t = V / VS  (|t| < 1/2),    254 t  ~ a1 + a2/254 + a3/254^2
//     x' = x * sc (|x'| < 1/2),   254 x' ~ b1 + b2/254 + b3/254^2
// with int8 digits in [-127, 127], VS just above twice the largest |V| and sc a power of two
// per X column (wire, variable) chosen each stage from the column's largest
// value.  The products of digit weight i + j <= 4,
//     D2 = sum a1 b1,  D3 = sum a1 b2 + a2 b1,  D4 = sum a1 b3 + a2 b2 + a3 b1,
// are exact in int32 (|D| < 3 * 1024 * 127^2 < 2^31), so the tensor cores
// add no rounding at all; the exchange sum is
//     VS / (254^2 sc) * (D2 + D3/254 + D4/254^2)
// (rounded once to FP32).  The digits represent t and x' to 2^-24.6 of
// their scale (the static part, from T, is ~5e-8 of a sum); the dropped
// products are below that.  (FP32 accumulation of 16-bit limbs was measured
// to truncate every K = 16 step with a bias of ~1e-7 of the sum, which
// compounds into the phase of p.)  The three digit products of one K step
// are issued as three MMAs with the X digit planes stacked along N:
// T1 [X1|X2|X3] -> (D2|D3|D4), T2 [X1|X2] -> (D3|D4), T3 X1 -> D4.
//
// Precision of the right-hand side.  The phase of p is set by the band
// energies: (Se + Sh)/hbar * p and the dephasing gamma p are formed in FP64
// (rounding a static energy to FP32 drifts the phase linearly in time).  The
// Rabi frequency and the exchange terms are formed as Omega/hbar in FP32
// (Omega itself, ~V p, leaves the FP32 range once p has dephased), the
// stage point, the RK accumulator and an FP32 copy of y in FP32, the state y
// and the P(t) sums in FP64.
//
// One CTA owns a group of W (4, 8 or 16) wires for all `nsteps` RK4 steps,
// 128-row tiles of k at a time:
//   * X (the MMA B operand: three int8 digit planes, K-major, N = 4W
//     columns) lives in shared memory, double buffered: stage s reads
//     X[s & 1] while its epilogue writes the digits of the next stage point
//     into X[(s+1) & 1], with each column's scale taken from the previous
//     stage's column maximum and one bit of headroom; a column whose values
//     outgrow that headroom is re-digitised with its exact scale at the end
//     of the stage;
//   * T is Toeplitz and never stored as a matrix: each 128 x 64 tile of the
//     A operand (three digit planes) is generated straight into tensor
//     memory by four generator warps from tables of digit quads
//     (a(d), a(d-1), a(d-2), a(d-3)) in shared memory -- one 32-bit lookup
//     per TMEM cell.  A tile depends only on 2 mi - kj (mi the row tile, kj
//     the 64-wide k' slice); when all distinct tiles fit in tensor memory
//     they are generated once per call, else they stream through a double
//     buffer;
//   * one thread issues tcgen05.mma (M = 128, N = 4W, K = 32), six digit
//     products per K step, into the three accumulators of a row tile; the
//     accumulators are double buffered per row tile, so the epilogue of
//     tile mi overlaps the MMAs of tile mi + 1;
//   * eight drain/epilogue warps read a finished tile's accumulators and
//     evaluate the diagonal SBE right-hand side and the RK4 stage
//     combination (stage order of libpulsesuite/integrator.py:143-157);
//   * the per-element state (y FP64, FP32 copy of y, stage point and
//     accumulator FP32) stays
//     in shared memory for the whole call when it fits (psb_split_max_nk_
//     resident), else in the caller's workspace.
// Every mbarrier wait is bounded; on a timeout the CTA records
// PSB_ERR_TIMEOUT in its wires' status, waits for its MMAs, frees TMEM and
// returns.
#include <math.h>

#include <atomic>

#include "split_common.cuh"

namespace psb {
namespace split {

// Byte offset of element (k, col) in one digit plane of X (K-major: 16 k of
// a column contiguous in a core-matrix row, 8 columns per core matrix; core
// matrices at 128 B along k, column groups at sbo = 8 kpad).
__device__ __forceinline__ uint32_t x_off(int k, int col, uint32_t sbo) {
  return (uint32_t)((col >> 3) * sbo + (k >> 4) * 128 + (col & 7) * 16 + (k & 15));
}

// MMA-issuing warps: one thread issues a tcgen05.mma only every ~100-120
// cycles whatever N is (measured on B200, M = 128, K = 32 int8, N <= 128),
// so a group of 4 wires (N = 16, the narrowest MMAs) splits the K slices of
// every row tile between two issuing warps, each into its own partial
// accumulators, which the epilogue adds (exact int32 sums).  Wider groups
// keep one issuer: their accumulators leave no tensor memory for a second
// set.
__host__ __device__ constexpr int issuers_of(int n) { return n == 16 ? 2 : 1; }
// TMEM columns: two row-tile buffers of issuers_of(n) accumulator sets
// (D2, D3, D4: 3 N each), then the A slots (3 digit planes): all distinct
// tiles when they fit (persistent), else streamed slots in the remaining
// columns (up to kMaxSlots), used as two buffers of nslot / 2 slots: the
// generators fill one group while the MMAs read the other.
constexpr int kMaxSlots = 8;
__host__ __device__ inline int acc_cols(int n) { return 6 * n * issuers_of(n); }
__host__ __device__ inline bool persistent_tiles(int nk, int n) {
  return acc_cols(n) + kTileCols * ntiles_of(nk) <= kTmemCols;
}
__host__ __device__ inline int ring_slots(int n) {
  const int r = (kTmemCols - acc_cols(n)) / kTileCols;
  return r < kMaxSlots ? r : kMaxSlots;
}
__host__ __device__ inline int tmem_cols(int nk, int n) {
  const int slots = persistent_tiles(nk, n) ? ntiles_of(nk) : ring_slots(n);
  const int need = acc_cols(n) + kTileCols * slots;
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
  float4* ws_ys;   // stage point per element (workspace layout)
  float4* ws_acc;  // RK accumulator per element (workspace layout)
  float4* ws_yf;   // FP32 copy of y per element (workspace layout)
  int nsteps;
  double dt;
  double* P;
  int64_t n_P;
  int p_stride;
  int p_cap;
  double hbar;
  uint32_t smem_bytes;  // dynamic shared memory of the launch
  uint32_t spin_limit;  // polls of a bounded hand-off wait (>= 1)
};

// Shared-memory layout of one CTA.  RES: the element state (y double4,
// stage point, accumulator and FP32 copy of y float4 per (wire, k)) is
// resident here.
template <int W, bool RES>
struct Layout {
  static constexpr int N = 4 * W;
  uint32_t plane, xbuf, st, tab, bars, misc, total;
  int ntab_words;
  __host__ __device__ Layout(int nk) {
    const int kpad = kpad_of(nk), nM = mtiles_of(nk);
    plane = (uint32_t)kpad * N;  // one digit plane of X
    xbuf = kDigits * plane;      // one stage buffer
    st = 2 * xbuf;
    tab = st + (RES ? 80u * W * (uint32_t)kpad : 0u);
    ntab_words = kTileRows * nM + kpad;
    bars = tab + kDigits * 4 * (uint32_t)ntab_words;  // digit-quad tables
    bars = (bars + 15) & ~15u;
    misc = bars + 8 * 24;  // afull[8], afree[8], dfull[2], dfree[2], final
    // misc: tmem base (16 B), abort + snapshots (16 B), pulse constants
    // double[W][2][4], wire params double4[W], t double[W], off int64[W],
    // P partials double[2][4][W], X column decode factors float[2][N],
    // column maxima float[4][N], column write scales float[N], column
    // overflow flags int[2][N], gap/hbar double[W]
    total = misc + 32 + 328 * W + 16;  // + any-overflow flags int[2]
  }
};

// ---------------------------------------------------------------------------
// The kernel.
// ---------------------------------------------------------------------------
template <int W, bool RES>
__global__ void __launch_bounds__(kThreadsS, 1) split_rk4_kernel(Args a) {
  constexpr int N = 4 * W;
  constexpr int NI = issuers_of(N);  // MMA-issuing warps (kMmaWarp ..)
  constexpr int WH = W / 2;  // wires per drain/epilogue warp
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const PsbSplitGroup grp = a.groups[blockIdx.x];

  // ---- validate the group (uniform across the CTA) -------------------------
  bool ok = grp.table >= 0 && grp.table < a.ntab && grp.nw >= 1 && grp.nw <= W;
  PsbTable tb{};
  if (ok) {
    tb = a.tables[grp.table];
    ok = tb.nk >= 2 && tb.nk <= PSB_MAX_NK && tb.off >= 0 &&
         tb.off + 9 * (int64_t)tb.nk <= a.n_tabdata && (tb.flags & PSB_TAB_EXCITONS) &&
         (tb.flags & PSB_TAB_SHARED_V) && !(tb.flags & PSB_TAB_SCREENED) &&
         Layout<W, RES>(tb.nk).total <= a.smem_bytes;
    for (int i = 0; ok && i < grp.nw; ++i) {
      const int wi = grp.wire[i];
      ok = wi >= 0 && wi < a.nw && a.wires[wi].table == grp.table && a.wires[wi].off >= 0 &&
           a.wires[wi].off + tb.nk <= a.n_state && a.wires[wi].npulse >= 0 &&
           a.wires[wi].npulse <= 2;
    }
  }
  if (!ok) {
    if (tid < W && tid < grp.nw && grp.wire[tid] >= 0 && grp.wire[tid] < a.nw)
      a.wires[grp.wire[tid]].status = PSB_ERR_INVALID;
    return;
  }
  const int nk = tb.nk, kpad = kpad_of(nk), nM = mtiles_of(nk), nK = kpad / kTileK;
  const Layout<W, RES> L(nk);
  const bool persist = persistent_tiles(nk, N);
  const int nslot = ring_slots(N);  // streamed A slots
  const int ntile = ntiles_of(nk);
  uint8_t* xbase = smem;  // X[b] digit plane p at xbase + b xbuf + p plane
  double4* s_y = reinterpret_cast<double4*>(smem + L.st);
  float4* s_ys = reinterpret_cast<float4*>(smem + L.st + 32u * W * kpad);
  float4* s_acc = reinterpret_cast<float4*>(smem + L.st + 48u * W * kpad);
  float4* s_yf = reinterpret_cast<float4*>(smem + L.st + 64u * W * kpad);
  uint32_t* tabq = reinterpret_cast<uint32_t*>(smem + L.tab);  // [digit][word]
  uint64_t* afull = reinterpret_cast<uint64_t*>(smem + L.bars);
  uint64_t* afree = afull + kMaxSlots;
  uint64_t* dfull = afree + kMaxSlots;
  uint64_t* dfree = dfull + 2;
  uint64_t* final_bar = dfree + 2;  // teardown: all MMAs of this CTA done
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + L.misc);
  volatile int* abort = reinterpret_cast<volatile int*>(smem + L.misc + 16);
  // abort as seen at each stage's end barrier (written by one participant
  // before the barrier, read by all after it, so every role breaks together)
  volatile int* snap = reinterpret_cast<volatile int*>(smem + L.misc + 20);
  double* pulse = reinterpret_cast<double*>(smem + L.misc + 32);  // [W][2][4]
  double4* wpar = reinterpret_cast<double4*>(smem + L.misc + 32 + 64 * W);
  double* wt = reinterpret_cast<double*>(smem + L.misc + 32 + 96 * W);
  int64_t* woff = reinterpret_cast<int64_t*>(smem + L.misc + 32 + 104 * W);
  double* ppart = reinterpret_cast<double*>(smem + L.misc + 32 + 112 * W);
  float* xfach = reinterpret_cast<float*>(smem + L.misc + 32 + 176 * W);  // [2][N]
  float* colmax = reinterpret_cast<float*>(smem + L.misc + 32 + 208 * W);  // [4][N]
  float* scw = reinterpret_cast<float*>(smem + L.misc + 32 + 272 * W);     // [N]
  int* ovf = reinterpret_cast<int*>(smem + L.misc + 32 + 288 * W);         // [2][N]
  double* gaph = reinterpret_cast<double*>(smem + L.misc + 32 + 320 * W);  // [W]
  volatile int* ovf_any = reinterpret_cast<volatile int*>(smem + L.misc + 32 + 328 * W);  // [2]
  const double inv_hbar = 1.0 / a.hbar;
  const uint32_t xsbo = (uint32_t)kpad * 8;
  const double* blk = a.tabdata + tb.off;
  const double* Ee = blk + 3 * nk;
  const double* Eh = blk + 4 * nk;

  // ---- set-up ---------------------------------------------------------------
  // VS: just above 2 max V, so |t| < 1/2.
  __shared__ double vmax_w[kThreadsS / 32];
  double vm = 0.0;
  for (int qq = 1 + tid; qq < nk; qq += kThreadsS) vm = fmax(vm, fabs(blk[qq]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) vm = fmax(vm, __shfl_xor_sync(0xffffffffu, vm, o));
  if (lane == 0) vmax_w[warp] = vm;
  for (uint32_t i = tid * 16; i < 2 * L.xbuf; i += kThreadsS * 16)
    *reinterpret_cast<uint4*>(xbase + i) = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    for (int b = 0; b < kMaxSlots; ++b) {
      mbar_init(&afull[b], kGenWarps);
      mbar_init(&afree[b], NI);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&dfull[b], NI);
      mbar_init(&dfree[b], kEpiWarps);
    }
    mbar_init(final_bar, NI);
    *abort = 0;
    snap[0] = 0;
    snap[1] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < W) {
    // per pulse: t0, -4 ln2 / fwhm^2, and -mscale * amp * (cos, sin)(phase),
    // so M(t) = sum (c2, c3) exp(c1 (t - t0)^2)  (SBEs drive, E(t) Gaussian)
    double* pc = pulse + tid * 8;
    if (tid < grp.nw) {
      const PsbWire& w = a.wires[grp.wire[tid]];
      wpar[tid] = make_double4(w.gap, w.gamma, w.mscale, w.pscale);
      gaph[tid] = w.gap * inv_hbar;
      wt[tid] = w.t;
      woff[tid] = w.off;
      for (int j = 0; j < 2; ++j) {
        if (j < w.npulse) {
          double sn, cs;
          sincos(w.phase[j], &sn, &cs);
          pc[4 * j + 0] = w.t0[j];
          pc[4 * j + 1] = -4.0 * log(2.0) / (w.fwhm[j] * w.fwhm[j]);
          pc[4 * j + 2] = -w.mscale * w.amp[j] * cs;
          pc[4 * j + 3] = -w.mscale * w.amp[j] * sn;
        } else {
          pc[4 * j + 0] = pc[4 * j + 1] = pc[4 * j + 2] = pc[4 * j + 3] = 0.0;
        }
      }
    } else {
      wpar[tid] = make_double4(0.0, 0.0, 0.0, 0.0);
      gaph[tid] = 0.0;
      wt[tid] = 0.0;
      woff[tid] = -1;
      for (int j = 0; j < 8; ++j) pc[j] = 0.0;
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
  // TMEM column map: accumulator set b at 3 N b (D2, D3, D4 at +0, +N,
  // +2N); A slot i at acol0 + kTileCols i (digit plane p at + kPlaneCols p).
  const uint32_t acol0 = (uint32_t)acc_cols(N);
  double vmax = 0.0;
#pragma unroll
  for (int i = 0; i < kThreadsS / 32; ++i) vmax = fmax(vmax, vmax_w[i]);
  // V is static, so its scale needs no headroom: VS = 2 vmax (1 + 2^-20)
  // puts the largest |t| just below 1/2 and uses the full digit range (a
  // power-of-two scale would leave up to a factor 2 of the precision
  // unused; the static representation error of V drifts the phase of p)
  const double VS = vmax > 0.0 ? 2.0 * vmax * (1.0 + 0x1p-20) : 1.0;
  const double inv_VS = 1.0 / VS;
  // Digit-quad tables: word(d) = bytes (a(d), a(d-1), a(d-2), a(d-3)) of one
  // digit plane for d in [dlo, dlo + ntab_words), a(d) = digit of
  // V(|d|)/VS (0 at d = 0 and outside the grid).
  const int dlo = 4 - kpad;
  for (int i = tid; i < L.ntab_words; i += kThreadsS) {
    const int d = dlo + i;
    uint32_t wq[kDigits] = {0u, 0u, 0u};
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int dd = d - u;
      const int ad = dd < 0 ? -dd : dd;
      const double t = (ad > 0 && ad < nk) ? blk[ad] * inv_VS : 0.0;
      // digits of t from its FP64 value
      const double f1 = rint(t * kBase);
      const double r1 = t * kBase - f1;
      const double f2 = rint(r1 * kBase);
      const double r2 = r1 * kBase - f2;
      const double f3 = rint(r2 * kBase);
      const int dg[3] = {(int)f1, (int)f2, (int)f3};
#pragma unroll
      for (int p = 0; p < kDigits; ++p) wq[p] |= ((uint32_t)(dg[p] & 0xFF)) << (8 * u);
    }
#pragma unroll
    for (int p = 0; p < kDigits; ++p) tabq[p * L.ntab_words + i] = wq[p];
  }

  // ---- element ownership of the drain/epilogue warps -----------------------------
  // warp (q, hh): rows 128 mi + 32 q + lane (q = TMEM lane quarter), wires
  // w0 .. w0 + WH - 1.
  const int q = warp & 3;
  const int hh = (warp >> 2) & 1;
  const int w0 = hh * WH;
  double4* g_y = reinterpret_cast<double4*>(a.y);
  // Largest |value| of each of this warp's X columns, per lane quarter q.
  // Halving butterfly (colmax_halve): the 4 WH columns need 4 WH shuffles
  // in all, not 5 per column; afterwards lane L holds column
  // (L >> (5 - m)) & (4 WH - 1), m = log2(4 WH).
  auto publish_colmax = [&](const float* cm) {
    constexpr int C = 4 * WH;  // 8, 16 or 32
    static_assert(C == 8 || C == 16 || C == 32, "column count of a drain warp");
    float v[C];
#pragma unroll
    for (int c = 0; c < C; ++c) v[c] = cm[c];
    if constexpr (C == 32) {
      // five halvings leave lane L with column L
      colmax_halve<32>(v, 16, lane);
      colmax_halve<16>(v, 8, lane);
      colmax_halve<8>(v, 4, lane);
      colmax_halve<4>(v, 2, lane);
      colmax_halve<2>(v, 1, lane);
      colmax[q * N + 4 * w0 + lane] = v[0];
    } else if constexpr (C == 16) {
      colmax_halve<16>(v, 16, lane);
      colmax_halve<8>(v, 8, lane);
      colmax_halve<4>(v, 4, lane);
      colmax_halve<2>(v, 2, lane);
      v[0] = fmaxf(v[0], __shfl_xor_sync(0xffffffffu, v[0], 1));
      if ((lane & 1) == 0) colmax[q * N + 4 * w0 + ((lane >> 1) & 15)] = v[0];
    } else {
      colmax_halve<8>(v, 16, lane);
      colmax_halve<4>(v, 8, lane);
      colmax_halve<2>(v, 4, lane);
      v[0] = fmaxf(v[0], __shfl_xor_sync(0xffffffffu, v[0], 2));
      v[0] = fmaxf(v[0], __shfl_xor_sync(0xffffffffu, v[0], 1));
      if ((lane & 3) == 0) colmax[q * N + 4 * w0 + ((lane >> 2) & 7)] = v[0];
    }
  };
  auto track = [&](float* cm, int j, float4 v) {
    cm[4 * j + 0] = fmaxf(cm[4 * j + 0], fabsf(v.x));
    cm[4 * j + 1] = fmaxf(cm[4 * j + 1], fabsf(v.y));
    cm[4 * j + 2] = fmaxf(cm[4 * j + 2], fabsf(v.z));
    cm[4 * j + 3] = fmaxf(cm[4 * j + 3], fabsf(v.w));
  };
  auto ws_ptrs = [&](int w, int k, float4*& ysp, float4*& accp, float4*& yfp) {
    if (RES) {
      const int es = w * kpad + k;
      ysp = s_ys + es;
      accp = s_acc + es;
      yfp = s_yf + es;
    } else {
      const int64_t eg = woff[w] + k;
      ysp = a.ws_ys + eg;
      accp = a.ws_acc + eg;
      yfp = a.ws_yf + eg;
    }
  };
  // Largest |value| of column col over the four lane quarters.
  auto col_max = [&](int col) -> float {
    return fmaxf(fmaxf(colmax[col], colmax[N + col]),
                 fmaxf(colmax[2 * N + col], colmax[3 * N + col]));
  };
  // Exact column scale: the power of two that puts the column's largest
  // value m in [1/4, 1/2).  Lagged scale (for values of the next stage,
  // which may grow): m in [1/8, 1/4), and 1/4 for an all-zero column
  // (|p| <= 1/2 and n <= 1 for any physical state).
  auto sexp_exact = [](float m) -> int {
    int e2 = 0;
    if (!(m > 0.f) || !isfinite(m)) return 0;
    frexpf(m, &e2);  // m < 2^e2
    return min(max(-1 - e2, -120), 120);
  };
  auto sexp_lag = [](float m) -> int {
    int e2 = 0;
    if (!(m > 0.f) || !isfinite(m)) return -2;
    frexpf(m, &e2);
    return min(max(-2 - e2, -120), 120);
  };
  // Decode factor of a column digitised with scale 2^sexp: exchange sum / hbar
  // = VS / (hbar 254^2) 2^-sexp (D2 + (D3 + D4/254)/254).
  const double dec0 = VS * inv_hbar / (kBase * kBase);
  // Digitise the stage points of X[b] column by column with the exact scale
  // of each column: all columns (only_flagged false) or the columns whose
  // lagged scale overflowed (ovf[b][col] set).  One item = 4 consecutive k
  // of one column (a 32-bit word per digit plane).  Sets xfach[b][col].
  auto x_pass = [&](int b, bool only_flagged) {
    const int nq = (nk + 3) >> 2;
    uint8_t* xb = xbase + b * L.xbuf;
    for (int item = tid; item < 4 * grp.nw * nq; item += kEpiThreads) {
      const int col = item / nq;
      const int k0 = (item - col * nq) * 4;
      if (only_flagged && !ovf[b * N + col]) continue;
      const int sexp = sexp_exact(col_max(col));
      if (k0 == 0) xfach[b * N + col] = (float)ldexp(dec0, -sexp);
      const float sc = ldexpf(1.f, sexp);
      const int w = col >> 2, v = col & 3;
      uint32_t word[kDigits] = {0u, 0u, 0u};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (k0 + u >= nk) break;
        float4* ysp; float4* accp; float4* yfp;
        ws_ptrs(w, k0 + u, ysp, accp, yfp);
        const float4 yv = *ysp;
        const float x = v == 0 ? yv.x : (v == 1 ? yv.y : (v == 2 ? yv.z : yv.w));
        int d1, d2, d3;
        digits3(x * sc, d1, d2, d3);
        word[0] |= ((uint32_t)(d1 & 0xFF)) << (8 * u);
        word[1] |= ((uint32_t)(d2 & 0xFF)) << (8 * u);
        word[2] |= ((uint32_t)(d3 & 0xFF)) << (8 * u);
      }
      const uint32_t o = x_off(k0, col, xsbo);
#pragma unroll
      for (int p = 0; p < kDigits; ++p) *reinterpret_cast<uint32_t*>(xb + p * L.plane + o) = word[p];
    }
  };
  // Lagged write scales for the next stage's digits (from this stage's column
  // maxima) and their decode factors xfach[b]; run by threads < N.
  const float dec0f = (float)dec0;
  auto set_write_scales = [&](int b) {
    if (tid < N) {
      const int sexp = sexp_lag(col_max(tid));
      scw[tid] = ldexpf(1.f, sexp);
      xfach[b * N + tid] = ldexpf(dec0f, -sexp);
    }
  };

  // Stage-0 input: stage point = FP32 copy of y = y, X[0] = digits(y) with
  // exact column scales, write scales of stage 0 from the same maxima.
  if (warp < kEpiWarps) {
    float cm0[4 * WH];
#pragma unroll
    for (int c = 0; c < 4 * WH; ++c) cm0[c] = 0.f;
    for (int mi = 0; mi < nM; ++mi) {
      const int k = mi * kTileRows + 32 * q + lane;
      if (k >= nk) continue;
#pragma unroll
      for (int j = 0; j < WH; ++j) {
        const int w = w0 + j;
        if (w >= grp.nw) break;
        const double4 yv = g_y[woff[w] + k];
        const float4 yf = make_float4((float)yv.x, (float)yv.y, (float)yv.z, (float)yv.w);
        if (RES) s_y[w * kpad + k] = yv;
        float4* ysp; float4* accp; float4* yfp;
        ws_ptrs(w, k, ysp, accp, yfp);
        *ysp = yf;
        *yfp = yf;
        track(cm0, j, yf);
      }
    }
    if (tid < 2 * N) ovf[tid] = 0;
    if (tid < 2) ovf_any[tid] = 0;
    publish_colmax(cm0);
    named_sync(2, kEpiThreads);
    x_pass(0, false);
    set_write_scales(1);
    fence_async_smem();
  }
  __syncthreads();

  static_assert(3 * N <= 256, "stacked MMA width 3N must be <= 256");
  const uint32_t idesc1 = idesc_i8(N), idesc2 = idesc_i8(2 * N), idesc3 = idesc_i8(3 * N);
  const int total_stages = a.nsteps * 4;
  const double h = a.dt;

  // Roles.  Each warpgroup changes its register allocation once, at the top
  // of its branch (all four warps at the same instruction): warpgroups 2
  // and 3 down to kRegsLow, the epilogue warpgroups 0 and 1 up to kRegsHigh.
  if (warp >= kMmaWarp) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kRegsLow));
    if (warp < kMmaWarp + NI) {
    // ---- MMA issuers ----------------------------------------------------------
    // The whole warp polls the barriers (uniform control flow) and lane 0
    // alone issues the MMAs and commits.  One thread issues every MMA, and
    // these narrow MMAs are short, so the issuing thread's own instructions
    // between them set the rate: a barrier poll whose result it branches on
    // stalls the issue for ~150-180 cycles (measured), about the time of
    // three MMAs.  So the MMAs of a row tile (persistent A) or of a group of
    // streamed slots go out in one unbroken sequence, with one poll before
    // it; descriptors and TMEM addresses advance incrementally.
    // With NI = 2 issuer ik takes the slices kj = ik (mod 2) of every row
    // tile into accumulator set ik; with streamed A both issuers read every
    // group (and both release it), so the generators keep filling one
    // buffer while the issuers read the other.
    const int ik = warp - kMmaWarp;
    const bool issuer = lane == 0;
    uint32_t it = 0;  // row tiles issued
    int gb = 0;       // streamed group buffer of the next slices (two of G slots)
    uint32_t gph = 0; // parity of that buffer's current fill
    const int G = nslot / 2;
    auto warp_wait = [&](uint64_t* bar, uint32_t parity) -> bool {
      const bool got = mbar_wait(bar, parity, abort, a.spin_limit);
      return __all_sync(0xffffffffu, got);
    };
    // (an abort is seen through the stage-end snapshot and inside every
    // wait, so the stage start needs no vote of its own)
    for (int s = 0; s < total_stages; ++s) {
      {
        bool ok = !(s == 0 && persist) || warp_wait(&afull[0], 0);
        tc_fence_after();
        // B descriptor of X[s & 1] at k' = 0; +32 per 64-wide slice, +16 per
        // K step (start address in 16-byte units: 256 B per 32 k')
        const uint64_t bdesc0 = smem_desc(smem_u32(xbase + (s & 1) * L.xbuf), 128, xsbo);
        for (int mi = 0; ok && mi < nM; ++mi, ++it) {
          const int b = it & 1;
          // every lane polls; the vote on the outcome comes at the tile end
          if (it >= 2 && !mbar_wait(&dfree[b], ((it >> 1) - 1) & 1, abort, a.spin_limit))
            ok = false;
          tc_fence_after();
          const uint32_t d2 = tmem + (uint32_t)(3 * N * (b * NI + ik));
          const uint32_t d3 = d2 + (uint32_t)N;
          const uint32_t d4 = d2 + (uint32_t)(2 * N);
          // one 64-wide K slice: K step 0 (the tile's first slice overwrites
          // its accumulators), then K step 1
          auto slice = [&](uint32_t a1, uint64_t bd, bool acc) {
            umma_i8(d2, a1, bd, idesc3, acc);                // T1 [X1|X2|X3] -> D2|D3|D4
            umma_i8(d3, a1 + kPlaneCols, bd, idesc2, 1);     // T2 [X1|X2] -> D3|D4
            umma_i8(d4, a1 + 2 * kPlaneCols, bd, idesc1, 1); // T3 X1 -> D4
            umma_i8(d2, a1 + 8, bd + 16, idesc3, 1);
            umma_i8(d3, a1 + kPlaneCols + 8, bd + 16, idesc2, 1);
            umma_i8(d4, a1 + 2 * kPlaneCols + 8, bd + 16, idesc1, 1);
          };
          uint64_t bd = bdesc0;
          if (persist) {
            // persistent slot of slice kj is 2 mi - kj + nK - 1
            if (issuer && ok) {
              uint32_t a1 = tmem + acol0 + (uint32_t)((2 * mi + nK - 1 - ik) * kTileCols);
              bd += 32 * ik;
              for (int kj = ik; kj < nK; kj += NI, a1 -= NI * kTileCols, bd += 32 * NI)
                slice(a1, bd, kj != ik);
            }
          } else {
            // streamed: slices k0 .. k0 + gn - 1 sit in slots gb G .. gb G + gn - 1.
            // Every lane polls the group and the warp reconverges after it
            // (so no lane can fall a buffer cycle behind and test a parity
            // that has come round again), but it votes on the outcome only
            // once per row tile: a vote costs the issuing lane about as much
            // as the poll.
            bool first = true;  // this issuer's first slice of the row tile
            for (int k0 = 0; ok && k0 < nK; k0 += G, bd += 32 * G) {
              const int gn = min(G, nK - k0);
              if (!mbar_wait(&afull[gb], gph, abort, a.spin_limit)) {
                ok = false;
                break;
              }
              tc_fence_after();
              if (issuer) {
                uint32_t a1 = tmem + acol0 + (uint32_t)(gb * G * kTileCols);
                uint64_t bj = bd;
                for (int j = 0; j < gn; ++j, a1 += kTileCols, bj += 32) {
                  if (((k0 + j) & (NI - 1)) != ik) continue;
                  slice(a1, bj, !first);
                  first = false;
                }
                umma_commit(&afree[gb]);  // the group's slots are reusable once these finish
              }
              __syncwarp();
              if (++gb == 2) {
                gb = 0;
                gph ^= 1u;
              }
            }
          }
          ok = __all_sync(0xffffffffu, ok);
          if (!ok) break;
          if (issuer) umma_commit(&dfull[b]);  // the row tile is ready to drain
          __syncwarp();
        }
      }
      __syncwarp();
      // wait for the epilogue to publish the next stage's X
      named_sync(1, kEpiThreads + 32 * NI);
      if (snap[s & 1]) break;
    }
    }
  } else if (warp >= kGenWarp0) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kRegsLow));
    // ---- A-tile generators ------------------------------------------------------
    // Row r = 32 gq + lane of the tile for 2 mi - kj = dl is a(d0 - c),
    // c = 0..63, d0 = 64 dl + r; TMEM column j of a digit plane holds
    // c = 4j .. 4j+3, i.e. word(d0 - 4j).
    const int gq = warp - kGenWarp0;
    auto gen_tile = [&](int dl, int slot) {
      const int base = 64 * dl + 32 * gq + lane - dlo;
      const uint32_t ta = tmem + ((uint32_t)(32 * gq) << 16) + acol0 +
                          (uint32_t)(slot * kTileCols);
#pragma unroll
      for (int p = 0; p < kDigits; ++p) {
        uint32_t r[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) r[j] = tabq[p * L.ntab_words + base - 4 * j];
        tmem_st16(ta + p * kPlaneCols, r);
      }
    };
    if (persist) {
      for (int sl = 0; sl < ntile; ++sl) gen_tile(sl - (nK - 1), sl);
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&afull[0]);
    } else {
      // the issuer's group sequence: per row tile, slices in groups of at
      // most G, alternating between two buffers of G slots
      const int G = nslot / 2;
      int gb = 0;           // group buffer of the next group
      uint32_t gph = 0;     // parity of that buffer's current fill
      bool first = true;    // first pass over both buffers: nothing to wait for
      for (int s = 0; s < total_stages && !*abort; ++s) {
        for (int mi = 0; mi < nM && !*abort; ++mi) {
          for (int k0 = 0; k0 < nK; k0 += G) {
            const int gn = min(G, nK - k0);
            bool got = first || mbar_wait(&afree[gb], gph ^ 1u, abort, a.spin_limit);
            got = __all_sync(0xffffffffu, got);
            if (!got) break;
            tc_fence_after();
            for (int j = 0; j < gn; ++j) gen_tile(2 * mi - (k0 + j), gb * G + j);
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&afull[gb]);
            if (++gb == 2) {
              gb = 0;
              gph ^= 1u;
              first = false;
            }
          }
        }
      }
    }
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kRegsHigh));
    // ---- drain / epilogue warps -----------------------------------------------------
    uint32_t it = 0;
    const uint32_t lrow = tmem + ((uint32_t)(32 * q) << 16);
    const float inv_base = 1.f / 254.f;
    const float hf = (float)h, h2f = (float)(h / 2.0), h6f = (float)(h / 6.0);
    // lane j < WH keeps the time of wire w0 + j
    double tj = (lane < WH) ? wt[w0 + lane] : 0.0;
    for (int s = 0; s < total_stages; ++s) {
      const int stg = s & 3;
      const int bn = (s + 1) & 1;  // X buffer this stage's epilogue writes
      // drive of this stage as M/hbar: lane j < WH evaluates wire w0 + j
      float Mr = 0.f, Mi = 0.f;
      if (lane < WH) {
        const double t = tj + (stg == 0 ? 0.0 : (stg == 3 ? h : h / 2.0));
        const double* pc = pulse + (w0 + lane) * 8;
        double mr = 0.0, mim = 0.0;
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) {
          const double u = t - pc[4 * jj + 0];
          const double env = exp(pc[4 * jj + 1] * u * u);
          mr += pc[4 * jj + 2] * env;
          mim += pc[4 * jj + 3] * env;
        }
        Mr = (float)(mr * inv_hbar);
        Mi = (float)(mim * inv_hbar);
      }
      double pr[WH], pim[WH];
#pragma unroll
      for (int jj = 0; jj < WH; ++jj) pr[jj] = pim[jj] = 0.0;
      float cm[4 * WH];
#pragma unroll
      for (int c = 0; c < 4 * WH; ++c) cm[c] = 0.f;
      const float* fx = xfach + (s & 1) * N;
      uint8_t* xn = xbase + bn * L.xbuf;
      int* ovn = ovf + bn * N;
      for (int mi = 0; mi < nM; ++mi, ++it) {
        const int k = mi * kTileRows + 32 * q + lane;
        const int b = it & 1;
        // band energies of this row: loaded before the wait, which hides them
        const double ekh = k < nk ? (Ee[k] + Eh[k]) * inv_hbar : 0.0;
        bool got = mbar_wait(&dfull[b], (it >> 1) & 1, abort, a.spin_limit);
        got = __all_sync(0xffffffffu, got);
        if (got) tc_fence_after();
        // this lane's row takes part in this tile (abort read once per tile)
        const bool live = got && k < nk && !*abort;
        const uint32_t kofs = (uint32_t)(k >> 4) * 128 + (uint32_t)(k & 15);
#pragma unroll
        for (int jp = 0; jp < WH; jp += 2) {
          // accumulators of wires w0+jp, w0+jp+1 (8 columns each)
          uint32_t r2[8], r3[8], r4[8];
          if (got) {
            const uint32_t col = lrow + (uint32_t)(3 * N * b * NI + 4 * (w0 + jp));
            tmem_ld8(col, r2);
            tmem_ld8(col + N, r3);
            tmem_ld8(col + 2 * N, r4);
            if (NI == 2 && nK > 1) {
              // the second issuer's partial sums (every row tile has slices
              // of both issuers when nK > 1)
              uint32_t s2[8], s3[8], s4[8];
              tmem_ld8(col + 3 * N, s2);
              tmem_ld8(col + 4 * N, s3);
              tmem_ld8(col + 5 * N, s4);
              tmem_ld_wait();
#pragma unroll
              for (int c = 0; c < 8; ++c) {
                r2[c] += s2[c];
                r3[c] += s3[c];
                r4[c] += s4[c];
              }
            }
            tmem_ld_wait();
          }
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int j = jp + u;
            const int w = w0 + j;
            const float Mjr = __shfl_sync(0xffffffffu, Mr, j);
            const float Mji = __shfl_sync(0xffffffffu, Mi, j);
            if (!live || w >= grp.nw) continue;
            // exchange sums / hbar (SBEs.py:896-921) from the exact digit
            // products, rounded once to FP32
            float exh[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              const int cc = 4 * u + c;
              const float e = (float)(int)r2[cc] +
                              ((float)(int)r3[cc] + (float)(int)r4[cc] * inv_base) * inv_base;
              exh[c] = e * fx[4 * w + c];
            }
            float4* ysp; float4* accp; float4* yfp;
            ws_ptrs(w, k, ysp, accp, yfp);
            const float4 ysf = *ysp;
            // diagonal RHS (SBEs.py:1962-1975, 2325-2337, 2623-2636) / hbar:
            // phase and dephasing terms in FP64, Rabi terms in FP32
            const float omr = Mjr + exh[0];
            const float omi = Mji + exh[1];
            const double sumh = (ekh + gaph[w]) - (double)(exh[2] + exh[3]);
            const float nn = ysf.z + ysf.w - 1.f;
            const double prd = ysf.x, pid = ysf.y;
            const double gw = wpar[w].y;  // gamma
            const float f0 = (float)(sumh * pid - gw * prd) - omi * nn;
            const float f1 = (float)(-(sumh * prd) - gw * pid) + omr * nn;
            const float f2 = 2.f * (omi * ysf.x - omr * ysf.y);
            // RK4 stage combination (integrator.py:143-157): acc = k1 + 2 k2
            // + 2 k3 and the stage points in FP32, y += h/6 (acc + k4) in FP64
            float4 nxt;
            if (stg == 0) {
              *accp = make_float4(f0, f1, f2, f2);
              // the stage-0 point is the FP32 copy of y
              nxt = make_float4(ysf.x + h2f * f0, ysf.y + h2f * f1, ysf.z + h2f * f2,
                                ysf.w + h2f * f2);
            } else if (stg == 3) {
              const float4 af = *accp;
              double4* yp = RES ? s_y + (w * kpad + k) : g_y + (woff[w] + k);
              double4 yv = *yp;
              yv.x += (double)(h6f * (af.x + f0));
              yv.y += (double)(h6f * (af.y + f1));
              yv.z += (double)(h6f * (af.z + f2));
              yv.w += (double)(h6f * (af.w + f2));
              *yp = yv;
              nxt = make_float4((float)yv.x, (float)yv.y, (float)yv.z, (float)yv.w);
              *yfp = nxt;
              pr[j] += yv.x;
              pim[j] += yv.y;
            } else {
              const float4 af = *accp;
              *accp = make_float4(af.x + 2.f * f0, af.y + 2.f * f1, af.z + 2.f * f2,
                                  af.w + 2.f * f2);
              const float4 yf = *yfp;
              const float c2 = stg == 1 ? h2f : hf;
              nxt = make_float4(yf.x + c2 * f0, yf.y + c2 * f1, yf.z + c2 * f2, yf.w + c2 * f2);
            }
            *ysp = nxt;
            track(cm, j, nxt);
            // digits of the next stage point with the lagged column scales
            const float4 sc = *reinterpret_cast<const float4*>(scw + 4 * w);
            const float xv[4] = {nxt.x * sc.x, nxt.y * sc.y, nxt.z * sc.z, nxt.w * sc.w};
            // x_off(k, 4w + c): columns 4w..4w+3 share a core matrix
            const uint32_t obase = (uint32_t)(w >> 1) * xsbo + (uint32_t)(w & 1) * 64 + kofs;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              int d1, d2, d3;
              digits3(xv[c], d1, d2, d3);
              const uint32_t o = obase + 16 * c;
              xn[o] = (uint8_t)d1;
              xn[L.plane + o] = (uint8_t)d2;
              xn[2 * L.plane + o] = (uint8_t)d3;
              if (!(fabsf(xv[c]) < 0.5f)) {
                ovn[4 * w + c] = 1;
                ovf_any[bn] = 1;
              }
            }
          }
        }
        // accumulators of this row tile are free again
        tc_fence_before();
        __syncwarp();
        if (lane == 0 && got) mbar_arrive(&dfree[b]);
      }
      publish_colmax(cm);
      if (stg == 3) {
        // P(t) = pscale * sum_k p_k, reduced in a fixed order
#pragma unroll
        for (int jj = 0; jj < WH; ++jj) {
          double sr = pr[jj], si = pim[jj];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            sr += __shfl_xor_sync(0xffffffffu, sr, o);
            si += __shfl_xor_sync(0xffffffffu, si, o);
          }
          if (lane == 0) {
            ppart[(0 * 4 + q) * W + w0 + jj] = sr;
            ppart[(1 * 4 + q) * W + w0 + jj] = si;
          }
        }
      }
      named_sync(2, kEpiThreads);
      if (!*abort) {
        // columns whose values outgrew the lagged scale: exact re-digitising
        if (ovf_any[bn]) x_pass(bn, true);
        // flags of X[s & 1] were consumed at the end of the previous stage
        if (tid < N) ovf[(s & 1) * N + tid] = 0;
        if (tid == 0) ovf_any[s & 1] = 0;
        // write scales of the next stage (digits into X[s & 1])
        set_write_scales(s & 1);
      }
      if (stg == 3) {
        if (q == 0 && lane < WH && w0 + lane < grp.nw) {
          const int w = w0 + lane;
          const int step = s >> 2;
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
        tj = tj + h;
      }
      // this thread's digit stores become visible to the tensor cores
      fence_async_smem();
      if (warp == 0 && lane == 0) snap[s & 1] = *abort;
      named_sync(1, kEpiThreads + 32 * NI);
      if (snap[s & 1]) break;
    }
    if (!*abort) {
      if (q == 0 && lane < WH) wt[w0 + lane] = tj;
      // resident state back to the caller's y
      if (RES) {
        for (int mi = 0; mi < nM; ++mi) {
          const int k = mi * kTileRows + 32 * q + lane;
          if (k >= nk) continue;
          for (int j = 0; j < WH; ++j) {
            const int w = w0 + j;
            if (w >= grp.nw) break;
            g_y[woff[w] + k] = s_y[w * kpad + k];
          }
        }
      }
    }
  }

  // ---- teardown -----------------------------------------------------------------
  // every MMA of every issuer has completed before TMEM is released
  if (warp >= kMmaWarp && warp < kMmaWarp + NI && lane == 0) umma_commit(final_bar);
  if (warp == kMmaWarp && lane == 0) {
    bool done = false;
    for (uint32_t i = 0; i < kSpinLimit && !done; ++i) done = mbar_try_wait(final_bar, 0);
    // MMAs still in flight after the bounded wait: the wires' results are
    // not trustworthy, so they report PSB_ERR_TIMEOUT
    if (!done) *abort = 1;
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
        const double4 yv = g_y[woff[tid] + k];
        bad |= !(isfinite(yv.x) && isfinite(yv.y) && isfinite(yv.z) && isfinite(yv.w));
      }
      if (bad && wp->status == PSB_OK) wp->status = PSB_ERR_NONFINITE;
    }
  }
}

template <int W, bool RES>
int max_nk() {
  int best = 0;
  for (int nk = 2; nk <= PSB_MAX_NK; ++nk)
    if (Layout<W, RES>(nk).total <= kMaxDynSmem) best = nk;
  return best;
}

template <int W, bool RES>
int launch_res(Args a, int nkmax, cudaStream_t s) {
  const uint32_t smem = Layout<W, RES>(nkmax).total;  // monotone in nk
  if (smem > kMaxDynSmem)
    return set_error(PSB_ERR_SIZE, "split form: nk %d does not fit a group of %d wires", nkmax,
                     W);
  // the register reallocation inside the kernel assumes exactly kRegsLaunch
  // registers per thread at launch (an increase beyond what the warpgroups
  // gave down would never complete), so a build that differs is refused
  cudaFuncAttributes fa{};
  cudaError_t e = cudaFuncGetAttributes(&fa, split_rk4_kernel<W, RES>);
  if (e != cudaSuccess)
    return set_error(PSB_ERR_CUDA, "cudaFuncGetAttributes: %s", cudaGetErrorString(e));
  if (fa.numRegs != kRegsLaunch || fa.maxThreadsPerBlock < kThreadsS)
    return set_error(PSB_ERR_UNSUPPORTED,
                     "split_rk4_kernel built with %d registers per thread (needs %d) and at "
                     "most %d threads (needs %d)",
                     fa.numRegs, kRegsLaunch, fa.maxThreadsPerBlock, kThreadsS);
  e = cudaFuncSetAttribute(split_rk4_kernel<W, RES>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess)
    return set_error(PSB_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
  a.smem_bytes = smem;
  split_rk4_kernel<W, RES><<<a.ngroups, kThreadsS, smem, s>>>(a);
  return check_cuda("split_rk4_kernel");
}

template <int W>
int launch(const Args& a, int nkmax, cudaStream_t s) {
  if (nkmax <= max_nk<W, true>()) return launch_res<W, true>(a, nkmax, s);
  return launch_res<W, false>(a, nkmax, s);
}

}  // namespace split
}  // namespace psb

using namespace psb;

namespace psb {
namespace split {
static std::atomic<uint32_t> g_spin_limit{kSpinLimit};
uint32_t wait_limit() { return g_spin_limit.load(); }
}  // namespace split
}  // namespace psb

extern "C" int psb_split_set_wait_limit(uint32_t spins) {
  split::g_spin_limit.store(spins == 0 ? split::kSpinLimit : spins);
  return PSB_OK;
}

extern "C" int64_t psb_split_ws_bytes(int64_t n_state) {
  if (n_state < 0) return set_error(PSB_ERR_INVALID, "n_state < 0");
  return 64 * n_state + 32;
}

extern "C" int psb_split_max_nk(int wgroup) {
  if (wgroup == 16) return split::max_nk<16, false>();
  if (wgroup == 8) return split::max_nk<8, false>();
  if (wgroup == 4) return split::max_nk<4, false>();
  return set_error(PSB_ERR_INVALID, "wgroup must be 4, 8 or 16");
}

extern "C" int psb_split_max_nk_resident(int wgroup) {
  if (wgroup == 16) return split::max_nk<16, true>();
  if (wgroup == 8) return split::max_nk<8, true>();
  if (wgroup == 4) return split::max_nk<4, true>();
  return set_error(PSB_ERR_INVALID, "wgroup must be 4, 8 or 16");
}

namespace psb {
namespace split {
template <int W>
int smem_bytes(int nk) {
  return (int)(nk <= max_nk<W, true>() ? Layout<W, true>(nk).total : Layout<W, false>(nk).total);
}
}  // namespace split
}  // namespace psb

extern "C" int psb_split_smem_bytes(int nk, int wgroup) {
  if (nk < 2 || nk > PSB_MAX_NK) return set_error(PSB_ERR_SIZE, "nk %d out of range", nk);
  if (wgroup == 16) return split::smem_bytes<16>(nk);
  if (wgroup == 8) return split::smem_bytes<8>(nk);
  if (wgroup == 4) return split::smem_bytes<4>(nk);
  return set_error(PSB_ERR_INVALID, "wgroup must be 4, 8 or 16");
}

extern "C" int psb_rk4_split(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                             int64_t n_tabdata, PsbWire* d_wires, int nw,
                             const PsbSplitGroup* d_groups, int ngroups, int wgroup, int nkmax,
                             double* d_y, int64_t n_state, void* d_ws, int64_t n_ws_bytes,
                             int nsteps, double dt, double* d_P, int64_t n_P, int p_stride,
                             int p_cap, const PsbModel* model, void* stream) {
  if (!d_tables || !d_tabdata || !d_wires || !d_groups || !d_y || !d_ws || !model || ntab <= 0 ||
      nw < 0 || ngroups < 0)
    return set_error(PSB_ERR_INVALID, "psb_rk4_split: null pointer or bad count");
  if (wgroup != 4 && wgroup != 8 && wgroup != 16)
    return set_error(PSB_ERR_INVALID, "psb_rk4_split: wgroup must be 4, 8 or 16");
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
  a.ws_ys = (float4*)d_ws;
  a.ws_acc = (float4*)((uint8_t*)d_ws + 16 * n_state);
  a.ws_yf = (float4*)((uint8_t*)d_ws + 32 * n_state);
  a.nsteps = nsteps;
  a.dt = dt;
  a.P = d_P;
  a.n_P = n_P;
  a.p_stride = p_stride;
  a.p_cap = p_cap;
  a.hbar = model->hbar;
  a.spin_limit = split::wait_limit();
  cudaStream_t st = (cudaStream_t)stream;
  if (wgroup == 16) return split::launch<16>(a, nkmax, st);
  return wgroup == 8 ? split::launch<8>(a, nkmax, st) : split::launch<4>(a, nkmax, st);
}

// ---------------------------------------------------------------------------
// psb_rk4_split without a caller workspace: the workspace is one file-scope
// device array (held by every GPU that loads the library).  Host code only
// sees a host-side stand-in under the array's name, so its device address
// is looked up once per device with cudaGetSymbolAddress and cached,
// together with the context it was looked up in: a call from another
// context of that device looks it up again.  (A device reset that gives the
// new primary context the old handle is not detected: resetting a device
// between calls is not supported.)
// ---------------------------------------------------------------------------
#include <mutex>

namespace psb {
namespace split {
static __device__ __align__(256) uint8_t g_noalloc_ws[PSB_SPLIT_NOALLOC_SCRATCH_BYTES];
constexpr int kMaxDevices = 64;
static void* g_noalloc_ptr[kMaxDevices] = {};
static void* g_noalloc_ctx[kMaxDevices] = {};
static std::mutex g_noalloc_mu;

// The current driver context (CUcontext as void*), or null when the driver
// entry point is unavailable; fetched through the runtime, so the library
// does not link the driver library.  Called with g_noalloc_mu held.
static void* current_context() {
  typedef int (*CtxGetCurrent)(void**);
  static CtxGetCurrent fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrent>(p);
  }
  void* ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

// Device address of g_noalloc_ws on the current device (set-up on first use).
static int noalloc_scratch(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return set_error(PSB_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(PSB_ERR_UNSUPPORTED, "device ordinal %d beyond %d", dev, kMaxDevices);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  const void* ctx = current_context();
  if (!g_noalloc_ptr[dev] || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_ws);
    if (e != cudaSuccess || !p)
      return set_error(PSB_ERR_CUDA, "cudaGetSymbolAddress(workspace): %s",
                       cudaGetErrorString(e));
    g_noalloc_ptr[dev] = p;
    g_noalloc_ctx[dev] = current_context();  // the lookup may have created the context
  }
  *out = g_noalloc_ptr[dev];
  return PSB_OK;
}
}  // namespace split
}  // namespace psb

extern "C" int psb_rk4_split_noalloc(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                                     int64_t n_tabdata, PsbWire* d_wires, int nw,
                                     const PsbSplitGroup* d_groups, int ngroups, int wgroup,
                                     int nkmax, double* d_y, int64_t n_state, int nsteps,
                                     double dt, double* d_P, int64_t n_P, int p_stride,
                                     int p_cap, const PsbModel* model, void* stream) {
  if (n_state < 0) return set_error(PSB_ERR_INVALID, "psb_rk4_split_noalloc: n_state < 0");
  if (n_state > PSB_SPLIT_NOALLOC_MAX_STATE)
    return set_error(PSB_ERR_SIZE,
                     "psb_rk4_split_noalloc: n_state %lld exceeds the built-in workspace "
                     "(at most %lld elements); use psb_rk4_split with a caller workspace",
                     (long long)n_state, (long long)PSB_SPLIT_NOALLOC_MAX_STATE);
  void* ws = nullptr;
  const int rc = split::noalloc_scratch(&ws);
  if (rc != PSB_OK) return rc;
  return psb_rk4_split(d_tables, ntab, d_tabdata, n_tabdata, d_wires, nw, d_groups, ngroups,
                       wgroup, nkmax, d_y, n_state, ws, PSB_SPLIT_NOALLOC_SCRATCH_BYTES, nsteps,
                       dt, d_P, n_P, p_stride, p_cap, model, stream);
}
