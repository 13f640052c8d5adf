// sbe_split_wire.cu -- the split-precision batched RK4 step with one Coulomb
// matrix per wire, sm_100a (tcgen05 kind::i8, TMEM accumulators).
//
// sbe_split.cu shares one Toeplitz matrix V(|k-k'|) between the W wires of
// a CTA and stacks their columns along N.  That needs every wire of a group
// to use the same matrix for all four state columns.  Two cases of the
// reference do not:
//   * static screening (coulomb.py:1212-1230, CalcScreenedArrays): every
//     right-hand-side evaluation divides V(q) by eps(q; n1D), n1D =
//     sum_k (ne_k + nh_k) / 2 / L of that wire's current stage point, so the
//     matrix differs per wire and per RK stage;
//   * distinct electron-hole, electron-electron and hole-hole matrices
//     (CalcCoulombArrays, coulomb.py:502-577: Veh for p, Vee for ne, Vhh for
//     nh), where each state column has its own matrix.
// This kernel contracts one wire at a time with that wire's own matrices.
//
// Arithmetic: exactly that of sbe_split.cu -- T = V / VS and the stage point
// X (scaled per column by a power of two) as three balanced base-254 int8
// digits, the six digit products of weight <= 4 accumulated exactly in
// int32, the sum decoded once to FP32; the phase-setting terms FP64, the
// stage point and RK accumulator FP32, the state y and P(t) FP64.
// Differences: the column scales are exact (the stage point of a wire is
// complete before its digits are written, so no lagged scale and no
// re-digitising), and VS is taken per wire and stage from the screened
// matrix.
//
// Layout of one wire's contraction.  X is stored per wire as a "sequence"
// of 24 N-rows per 16-k block, rows 4g + v (v the state column, g = 0..5):
// g = 0, 1 and 5 are zero, g = 2, 3, 4 hold the digit planes X1, X2, X3.
// The B operand of A-digit p (T1, T2, T3) is the 16-row window starting at
// row 8 - 4p, i.e. [X1|X2|X3|0], [0|X1|X2|X3], [0|0|X1|X2], so the three
// MMAs of one K step add T1X1 | T1X2 + T2X1 | T1X3 + T2X2 + T3X1 into one
// 16-column accumulator (D2 | D3 | D4 | unused) per 128-row tile.  With
// distinct matrices each matrix has its own sequence holding only its
// columns (zeros elsewhere) and all three add into the same accumulator.
// A tiles (128 x 64, three digit planes) are generated into TMEM from
// per-digit-plane byte arrays (table_scaled / table_digits below); a tile
// depends on d = 2 mi - kj
// only, so the MMAs run d by d: each distinct tile is generated once per
// wire and stage and used for every (row tile, k' slice) pair it serves,
// with the accumulators of all row tiles of the wire live at once (double
// buffered between consecutive wires).
//
// One CTA owns a group of up to 16 wires (one grid) for all steps and
// visits them round robin, stage by stage.  Roles (16 warps):
//   warps 0..7   drain + epilogue: the whole wire per item (8 warps share
//                its row tiles), FP64 right-hand side and RK4 stage
//                combination, then the exact column scales and the digits
//                of the next stage point, the n1D and P(t) sums; for
//                screened tables, then n1D -> eps(q) (coulomb.py:1172-1193)
//                -> V/eps and VS of the wire's next stage;
//   warps 8..11  A-tile generators; for a screened wire they first write
//                the digits of its V/eps / VS into its byte arrays;
//   warps 12..15 MMA issuers, one per row tile mi (mod 4); warp 12 owns
//                TMEM.  One thread issues a tcgen05.mma about every 100-120
//                cycles whatever N is (measured on B200 for M = 128, K = 32
//                int8, N <= 128), while four issuing warps reach about four
//                times that rate, so the narrow per-wire MMAs are spread
//                over four issuers with disjoint accumulators.
// While one wire's epilogue and table run, the tensor cores work on the
// other wires of the group.  Every mbarrier wait is bounded (as in
// sbe_split.cu); a CTA that runs out records PSB_ERR_TIMEOUT in its wires'
// status, waits for its MMAs, frees TMEM and returns.
#include <math.h>

#include "split_common.cuh"

namespace psb {
namespace splitw {

using namespace psb::split;

constexpr int kIssuers = 4;  // warps 12..15 issue MMAs (row tiles mi = k mod 4)
constexpr int kMaxW = PSB_SPLIT_WMAX;
constexpr int kSeqRows = 24;                // N rows of a sequence per 16-k block
constexpr int kSeqBlock = kSeqRows * 16;    // bytes per 16-k block (K-direction stride)
constexpr int kMaxTilesPerWarp = 4;         // row tiles per epilogue warp (nk <= 1024)
constexpr int kMaxNkW = 2 * kMaxTilesPerWarp * kTileRows;  // 1024
constexpr int kMaxSlotsW = 8;

// Fixed part of the shared-memory map (bytes from `misc`).
constexpr uint32_t kOffAbort = 4, kOffSnap = 8;
constexpr uint32_t kOffPulse = 32;                          // double[16][8]
constexpr uint32_t kOffWpar = kOffPulse + 64 * kMaxW;      // double4[16]
constexpr uint32_t kOffGaph = kOffWpar + 32 * kMaxW;       // double[16]
constexpr uint32_t kOffWt = kOffGaph + 8 * kMaxW;          // double[16][2]
constexpr uint32_t kOffWoff = kOffWt + 16 * kMaxW;         // int64[16]
constexpr uint32_t kOffVs = kOffWoff + 8 * kMaxW;          // double[16][3]
constexpr uint32_t kOffSx = kOffVs + 24 * kMaxW;           // int[8 warps][16][4]
constexpr uint32_t kOffRed = kOffSx + 16 * kEpiWarps * kMaxW;  // [2][8 warps] x 48 B
constexpr uint32_t kOffSred = kOffRed + 2 * kEpiWarps * 48;    // double[16][4]
constexpr uint32_t kMiscBytes = kOffSred + 8 * 4 * 16;
constexpr int kNumBars = 2 * kMaxSlotsW + 5 + 3 * kMaxW;

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
  float4* ws_ys;
  float4* ws_acc;
  float4* ws_yf;
  int nsteps;
  double dt;
  double* P;
  int64_t n_P;
  int p_stride;
  int p_cap;
  double hbar;
  int wgroup;           // wires per group the shared memory is sized for
  int screened;         // tables of this launch are screened (per-wire tables)
  uint32_t smem_bytes;
  uint32_t spin_limit;
};

// Shared-memory map of one CTA for a grid of nk, W wires, NT matrices.
template <int NT>
struct WLayout {
  uint32_t seq, tab, tabsz, plane, sv, svsz, qc, vt, bars, misc, total;
  int ntab_words;
  __host__ __device__ WLayout(int nk, int W, bool scr) {
    const int kpad = kpad_of(nk), nM = mtiles_of(nk);
    seq = (uint32_t)(kpad / 16) * kSeqBlock;
    tab = (uint32_t)(W * NT) * seq;
    ntab_words = kTileRows * nM + kpad;
    plane = (uint32_t)ntab_words + 16u;  // one digit plane's byte array (see table_digits)
    tabsz = 3u * plane;
    sv = tab + (uint32_t)((scr ? W : 1) * NT) * tabsz;  // V / eps per wire (screened)
    svsz = 8u * (uint32_t)(NT * nk);
    qc = sv + (uint32_t)(scr ? W : 1) * svsz;          // qe, qh, 2 chi_e, 2 chi_h
    vt = qc + (scr ? 32u * (uint32_t)nk : 0u);          // V_t
    bars = (vt + svsz + 15u) & ~15u;
    misc = (bars + 8u * kNumBars + 127u) & ~127u;
    total = misc + kMiscBytes;
  }
};

// TMEM: two accumulator buffers of 16 columns per row tile, then A slots of
// NT tiles (48 columns each), an even number of them (two groups).
__host__ __device__ inline int dcols_of(int nk) { return 2 * 16 * mtiles_of(nk); }
template <int NT>
__host__ __device__ inline int slots_of(int nk) {
  int r = (kTmemCols - dcols_of(nk)) / (NT * kTileCols);
  r = r < kMaxSlotsW ? r : kMaxSlotsW;
  return r & ~1;
}
template <int NT>
__host__ __device__ inline int tmem_cols_w(int nk) {
  const int need = dcols_of(nk) + slots_of<NT>(nk) * NT * kTileCols;
  int c = 32;
  while (c < need) c <<= 1;
  return c;
}

// Matrix of state column v: Veh for p (v = 0, 1), Vee for ne, Vhh for nh;
// one shared matrix when NT == 1.
template <int NT>
__host__ __device__ constexpr int mat_of(int v) {
  return NT == 1 ? 0 : (v < 2 ? 0 : v - 1);
}

// log|(qc - pn) / (qc + n)| of Eps1D, pn = pi n (see table_scaled).
__device__ __forceinline__ double screen_log(double qc, double pn, double n) {
  const double den = qc + n;
  if (qc - pn < 0.5 * den) return log(fabs((qc - pn) / den));
  return (double)log1pf((float)(-(pn + n) / den));
}

// Digit tables of the NT matrices of one wire (screened: V / eps(q; n1d))
// or of one grid (unscreened).  Digit plane p of matrix t is a byte array
// R = tq + (t * 3 + p) * plane with R[c0 - d] = a(d), c0 = dlo + ntab_words
// - 1 (the largest d a generator reads), a(d) = digit p of V_t(|d|) /
// eps(|d|) / VS_t, 0 at d = 0 and outside the grid: the word of the four
// bytes (a(d), a(d-1), a(d-2), a(d-3)) a generator stores into tensor
// memory is then the four consecutive bytes from R[c0 - d].  The zeros are
// written once (the arrays start zeroed); a build rewrites a(+q) and a(-q)
// for 0 < q < nk.  It runs in two passes: table_scaled (the epilogue warps,
// after a wire's stage) and table_digits (the generator warps, before they
// generate that wire's tiles).
//
// Pass 1: sv[t][q] = V_t(q) / eps(q) with eps of Eps1D (coulomb.py:
// 1172-1193; qc holds qe, qh, 2 chi_e, 2 chi_h per q, vt the matrices) and
// VS_t = 2 max |sv_t| (1 + 2^-20) into vs[t] (every thread writes the same
// value).  Two q per iteration.  The logarithm of R = (qc - pi n) / (qc +
// n) is FP64 where R < 1/2 (q -> 0, where the clamped n brings qc - pi n
// close to zero); elsewhere it is log1pf of R - 1 = -(pi + 1) n / (qc + n),
// formed without cancellation, whose FP32 error (~1e-7 of log R, itself of
// order R - 1) moves eps by about 1e-8 -- below the 2^-24.6 at which the
// digits represent V / eps.  nthr threads from t0 on, named barrier `bar`.
template <int NT>
__device__ void table_scaled(const double* qc, const double* vt, int nk, bool scr, double n1d,
                             double* sv, double* vs, double* red, int t0, int nthr, int bar) {
  const int t = (int)threadIdx.x - t0;
  const int lane = threadIdx.x & 31, wl = t >> 5;
  double vm[NT];
#pragma unroll
  for (int m = 0; m < NT; ++m) vm[m] = 0.0;
  const double pn = kPi * n1d;
  for (int q0 = t; q0 < nk; q0 += 2 * nthr) {
    double ie[2] = {1.0, 1.0};
    if (scr) {
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int qq = min(q0 + u * nthr, nk - 1);
        const double le = screen_log(qc[qq], pn, n1d);
        const double lh = screen_log(qc[nk + qq], pn, n1d);
        ie[u] = 1.0 / ((1.0 - __dmul_rn(qc[2 * nk + qq], le)) - __dmul_rn(qc[3 * nk + qq], lh));
      }
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int q = q0 + u * nthr;
      if (q >= nk) continue;
#pragma unroll
      for (int m = 0; m < NT; ++m) {
        const double v = vt[m * nk + q] * ie[u];
        sv[m * nk + q] = v;
        if (q > 0) vm[m] = fmax(vm[m], fabs(v));
      }
    }
  }
#pragma unroll
  for (int m = 0; m < NT; ++m) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vm[m] = fmax(vm[m], __shfl_xor_sync(0xffffffffu, vm[m], o));
    if (lane == 0) red[wl * 4 + m] = vm[m];
  }
  named_sync(bar, nthr);
#pragma unroll
  for (int m = 0; m < NT; ++m) {
    double mx = 0.0;
    for (int i = 0; i < nthr / 32; ++i) mx = fmax(mx, red[i * 4 + m]);
    vs[m] = mx > 0.0 ? 2.0 * mx * (1.0 + 0x1p-20) : 1.0;
  }
}

// Pass 2: the three digits of sv_t(q) / VS_t into the byte arrays (threads
// t0 .. t0 + nthr - 1; the caller synchronises before the tables are read).
template <int NT>
__device__ void table_digits(const double* sv, const double* vs, int nk, int c0, uint8_t* tq,
                             uint32_t plane, int t0, int nthr) {
  const int t = (int)threadIdx.x - t0;
  double ivs[NT];
#pragma unroll
  for (int m = 0; m < NT; ++m) ivs[m] = 1.0 / vs[m];
  for (int q = 1 + t; q < nk; q += nthr) {
#pragma unroll
    for (int m = 0; m < NT; ++m) {
      const double x = sv[m * nk + q] * ivs[m];
      const double f1 = rint(x * kBase);
      const double r1 = x * kBase - f1;
      const double f2 = rint(r1 * kBase);
      const double r2 = r1 * kBase - f2;
      const double f3 = rint(r2 * kBase);
      const uint8_t dg[3] = {(uint8_t)(int)f1, (uint8_t)(int)f2, (uint8_t)(int)f3};
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        uint8_t* R = tq + (uint32_t)(m * 3 + p) * plane;
        R[c0 - q] = dg[p];  // d = +q
        R[c0 + q] = dg[p];  // d = -q
      }
    }
  }
}

template <int NT>
__global__ void __launch_bounds__(kThreadsS, 1) split_wire_kernel(Args a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const PsbSplitGroup grp = a.groups[blockIdx.x];
  const bool scr = a.screened != 0;

  // ---- validate the group (uniform across the CTA) -------------------------
  bool ok = grp.table >= 0 && grp.table < a.ntab && grp.nw >= 1 && grp.nw <= a.wgroup &&
            a.wgroup <= kMaxW;
  PsbTable tb{};
  if (ok) {
    tb = a.tables[grp.table];
    ok = tb.nk >= 2 && tb.nk <= kMaxNkW && tb.off >= 0 &&
         tb.off + 9 * (int64_t)tb.nk <= a.n_tabdata && (tb.flags & PSB_TAB_EXCITONS) &&
         (NT == 3 || (tb.flags & PSB_TAB_SHARED_V)) &&
         (((tb.flags & PSB_TAB_SCREENED) != 0) == scr) &&
         (NT == 1 || mtiles_of(tb.nk) <= 4) &&
         WLayout<NT>(tb.nk, a.wgroup, scr).total <= a.smem_bytes && slots_of<NT>(tb.nk) >= 2;
    for (int i = 0; ok && i < grp.nw; ++i) {
      const int wi = grp.wire[i];
      ok = wi >= 0 && wi < a.nw && a.wires[wi].table == grp.table && a.wires[wi].off >= 0 &&
           a.wires[wi].off + tb.nk <= a.n_state && a.wires[wi].npulse >= 0 &&
           a.wires[wi].npulse <= 2;
    }
  }
  if (!ok) {
    if (tid < kMaxW && tid < grp.nw && grp.wire[tid] >= 0 && grp.wire[tid] < a.nw)
      a.wires[grp.wire[tid]].status = PSB_ERR_INVALID;
    return;
  }
  const int nk = tb.nk, nw = grp.nw, kpad = kpad_of(nk), nM = mtiles_of(nk);
  const int nK = kpad / kTileK;
  const WLayout<NT> L(nk, a.wgroup, scr);
  const int nslot = slots_of<NT>(nk), G = nslot / 2;
  const int dmin = -(nK - 1), dmax = 2 * (nM - 1);
  const int dlo = 4 - kpad;
  const uint32_t c0 = (uint32_t)(dlo + L.ntab_words - 1);  // R[c0 - d] = a(d)
  uint8_t* xbase = smem;  // sequence (j, t) at xbase + (j NT + t) seq
  uint8_t* tabq = smem + L.tab;  // digit byte arrays (see table_scaled)
  double* svb = reinterpret_cast<double*>(smem + L.sv);  // V_t(q) / eps(q) per wire
  double* qcs = reinterpret_cast<double*>(smem + L.qc);  // screening constants per q
  double* vts = reinterpret_cast<double*>(smem + L.vt);  // V_t(q)
  uint64_t* afull = reinterpret_cast<uint64_t*>(smem + L.bars);
  uint64_t* afree = afull + kMaxSlotsW;
  uint64_t* dfull = afree + kMaxSlotsW;
  uint64_t* dfree = dfull + 2;
  uint64_t* final_bar = dfree + 2;
  uint64_t* xfull = final_bar + 1;     // [W] next stage's digits of wire j written
  uint64_t* svfull = xfull + kMaxW;    // [W] V/eps and VS of wire j's next stage written
  uint64_t* gdone = svfull + kMaxW;    // [W] every generator warp wrote its share of j's digits
  uint8_t* misc = smem + L.misc;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(misc);
  volatile int* abort = reinterpret_cast<volatile int*>(misc + kOffAbort);
  volatile int* snap = reinterpret_cast<volatile int*>(misc + kOffSnap);  // [2]
  double* pulse = reinterpret_cast<double*>(misc + kOffPulse);
  double4* wpar = reinterpret_cast<double4*>(misc + kOffWpar);
  double* gaph = reinterpret_cast<double*>(misc + kOffGaph);
  double* wtb = reinterpret_cast<double*>(misc + kOffWt);  // [W][2] by step parity
  int64_t* woff = reinterpret_cast<int64_t*>(misc + kOffWoff);
  double* vsw = reinterpret_cast<double*>(misc + kOffVs);  // [W][3] (unscreened: row 0)
  int* sx = reinterpret_cast<int*>(misc + kOffSx);  // [epilogue warp][W][4] column scales
  uint8_t* red = misc + kOffRed;                      // [2][8] {float cm[4], double n1, pr, pi}
  double* sred = reinterpret_cast<double*>(misc + kOffSred);
  const double inv_hbar = 1.0 / a.hbar;
  const double* blk = a.tabdata + tb.off;
  const double* Ee = blk + 3 * nk;
  const double* Eh = blk + 4 * nk;
  double4* g_y = reinterpret_cast<double4*>(a.y);
  const uint32_t lim = a.spin_limit;

  // ---- set-up ---------------------------------------------------------------
  if (tid == 0) {
    for (int b = 0; b < kMaxSlotsW; ++b) {
      mbar_init(&afull[b], kGenWarps);
      mbar_init(&afree[b], kIssuers);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&dfull[b], kIssuers);
      mbar_init(&dfree[b], kEpiWarps);
    }
    mbar_init(final_bar, kIssuers);
    for (int j = 0; j < kMaxW; ++j) {
      mbar_init(&xfull[j], kEpiWarps);
      mbar_init(&svfull[j], 1);
      mbar_init(&gdone[j], kGenWarps);
    }
    *abort = 0;
    snap[0] = 0;
    snap[1] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < kMaxW) {
    double* pc = pulse + tid * 8;
    if (tid < nw) {
      const PsbWire& w = a.wires[grp.wire[tid]];
      wpar[tid] = make_double4(w.gap, w.gamma, w.mscale, w.pscale);
      gaph[tid] = w.gap * inv_hbar;
      wtb[2 * tid] = w.t;
      wtb[2 * tid + 1] = w.t;
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
      wtb[2 * tid] = wtb[2 * tid + 1] = 0.0;
      woff[tid] = -1;
      for (int j = 0; j < 8; ++j) pc[j] = 0.0;
    }
  }
  // X sequences and digit tables start at zero: the entries no digit is
  // written to stay zero
  for (uint32_t i = tid * 16; i < L.sv; i += kThreadsS * 16)
    *reinterpret_cast<uint4*>(xbase + i) = make_uint4(0, 0, 0, 0);
  // the matrices and screening constants of the grid, per q
  for (int q = tid; q < nk; q += kThreadsS) {
#pragma unroll
    for (int m = 0; m < NT; ++m) vts[m * nk + q] = blk[m * nk + q];
    if (scr) {
      qcs[q] = blk[7 * nk + q];
      qcs[nk + q] = blk[8 * nk + q];
      qcs[2 * nk + q] = 2.0 * blk[5 * nk + q];
      qcs[3 * nk + q] = 2.0 * blk[6 * nk + q];
    }
  }
  __syncthreads();
  // Wire j's stage-0 point (the FP32 copy of y) into the workspace, its
  // column maxima and n1D sum; then (screened) its tables, and its digits.
  for (int j = 0; j < nw; ++j) {
    float cm[4] = {0.f, 0.f, 0.f, 0.f};
    double sn = 0.0;
    for (int k = tid; k < nk; k += kThreadsS) {
      const double4 yv = g_y[woff[j] + k];
      const float4 yf = make_float4((float)yv.x, (float)yv.y, (float)yv.z, (float)yv.w);
      a.ws_ys[woff[j] + k] = yf;
      a.ws_yf[woff[j] + k] = yf;
      cm[0] = fmaxf(cm[0], fabsf(yf.x));
      cm[1] = fmaxf(cm[1], fabsf(yf.y));
      cm[2] = fmaxf(cm[2], fabsf(yf.z));
      cm[3] = fmaxf(cm[3], fabsf(yf.w));
      sn += yv.z + yv.w;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sn += __shfl_xor_sync(0xffffffffu, sn, o);
#pragma unroll
      for (int v = 0; v < 4; ++v) cm[v] = fmaxf(cm[v], __shfl_xor_sync(0xffffffffu, cm[v], o));
    }
    if (lane == 0) {
      sred[warp * 4 + 0] = sn;
      float* f = reinterpret_cast<float*>(sred + warp * 4 + 1);
      for (int v = 0; v < 4; ++v) f[v] = cm[v];
    }
    __syncthreads();
    double tot = 0.0;
    float cma[4] = {0.f, 0.f, 0.f, 0.f};
    for (int i = 0; i < kThreadsS / 32; ++i) {
      tot += sred[i * 4 + 0];
      const float* f = reinterpret_cast<const float*>(sred + i * 4 + 1);
      for (int v = 0; v < 4; ++v) cma[v] = fmaxf(cma[v], f[v]);
    }
    __syncthreads();
    if (scr) {
      double n1d = tot / 2.0 / tb.L;
      n1d = n1d < tb.dens_max ? n1d : tb.dens_max;
      double* svj = svb + (uint32_t)j * (L.svsz / 8);
      table_scaled<NT>(qcs, vts, nk, true, n1d, svj, vsw + 3 * j, sred, 0, kThreadsS, 0);
      __syncthreads();
      table_digits<NT>(svj, vsw + 3 * j, nk, (int)c0, tabq + (uint32_t)(j * NT) * L.tabsz,
                       L.plane, 0, kThreadsS);
      __syncthreads();
    }
    int se[4];
    float sc[4];
    for (int v = 0; v < 4; ++v) {
      int e2 = 0;
      const float m = cma[v];
      se[v] = 0;
      if (m > 0.f && isfinite(m)) {
        frexpf(m, &e2);
        se[v] = min(max(-1 - e2, -120), 120);
      }
      sc[v] = ldexpf(1.f, se[v]);
    }
    for (int k = tid; k < nk; k += kThreadsS) {
      const float4 yf = a.ws_ys[woff[j] + k];
      const float xv[4] = {yf.x * sc[0], yf.y * sc[1], yf.z * sc[2], yf.w * sc[3]};
      const uint32_t ob = (uint32_t)(k >> 4) * kSeqBlock + (uint32_t)(k & 15);
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        int d1, d2, d3;
        digits3(xv[v], d1, d2, d3);
        uint8_t* xq = xbase + (uint32_t)(j * NT + mat_of<NT>(v)) * L.seq + ob + 16 * v;
        xq[8 * 16] = (uint8_t)d1;
        xq[12 * 16] = (uint8_t)d2;
        xq[16 * 16] = (uint8_t)d3;
      }
    }
    if (tid < 4 * kEpiWarps) sx[((tid >> 2) * kMaxW + j) * 4 + (tid & 3)] = se[tid & 3];
  }
  if (!scr) {
    table_scaled<NT>(qcs, vts, nk, false, 0.0, svb, vsw, sred, 0, kThreadsS, 0);
    __syncthreads();
    table_digits<NT>(svb, vsw, nk, (int)c0, tabq, L.plane, 0, kThreadsS);
  }
  fence_async_smem();
  const int ncols = tmem_cols_w<NT>(nk);
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
  const uint32_t dstride = (uint32_t)(16 * nM);       // columns of one accumulator buffer
  const uint32_t acol0 = 2u * dstride;                // first A slot
  const uint32_t idesc16 = idesc_i8(16);
  const int total_stages = a.nsteps * 4;
  const double h = a.dt;

  if (warp >= kMmaWarp) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kRegsLow));
    // ---- MMA issuers: items (stage, wire) in order; per item the distinct
    // tiles d in groups of G slots; issuer k takes the row tiles mi = k
    // (mod 4) of every (row tile, k' slice) pair of a tile: two K steps,
    // three digit planes per pair, into that row tile's own accumulator.
    // Every issuer commits each group (afree) and each item (dfull), so
    // those barriers expect kIssuers arrivals.  Lane 0 issues.
    const int ik = warp - kMmaWarp;
    const bool issuer = lane == 0;
    uint32_t it = 0;
    int gb = 0;
    uint32_t gph = 0;
    bool go = true;
    const uint64_t bdesc0 = smem_desc(smem_u32(xbase), kSeqBlock, 128);
    for (int s = 0; s < total_stages && go; ++s) {
      for (int j = 0; j < nw && go; ++j, ++it) {
        const int b = it & 1;
        bool w8 = true;
        if (s >= 1) w8 = mbar_wait_sleep(&xfull[j], (s - 1) & 1, abort, lim);
        if (w8 && it >= 2) w8 = mbar_wait_sleep(&dfree[b], ((it >> 1) - 1) & 1, abort, lim);
        go = __all_sync(0xffffffffu, w8);
        if (!go) break;
        tc_fence_after();
        const uint32_t dbase = tmem + (uint32_t)b * dstride;
        // descriptor start addresses count 16-byte units
        const uint64_t bwire = bdesc0 + (uint64_t)(((uint32_t)(j * NT) * L.seq) >> 4);
        for (int d0 = dmin; d0 <= dmax; d0 += G) {
          const int gn = min(G, dmax - d0 + 1);
          go = __all_sync(0xffffffffu, mbar_wait_sleep(&afull[gb], gph, abort, lim));
          if (!go) break;
          tc_fence_after();
          if (issuer) {
            for (int jj = 0; jj < gn; ++jj) {
              const int d = d0 + jj;
              const int mlo = max(0, (d + 1) >> 1), mhi = min(nM - 1, (d + nK - 1) >> 1);
              // first row tile >= mlo of this issuer
              const int m0 = mlo + ((ik - mlo) % kIssuers + kIssuers) % kIssuers;
              const uint32_t aslot = tmem + acol0 + (uint32_t)((gb * G + jj) * NT * kTileCols);
#pragma unroll
              for (int t = 0; t < NT; ++t) {
                const uint32_t at = aslot + (uint32_t)(t * kTileCols);
                const uint64_t bt = bwire + (uint64_t)(((uint32_t)t * L.seq) >> 4);
                for (int mi = m0; mi <= mhi; mi += kIssuers) {
                  const int kj = 2 * mi - d;
                  const uint32_t dcol = dbase + 16u * (uint32_t)mi;
                  // the first product into a row tile's accumulator overwrites it
                  const uint32_t acc0 = (t == 0 && kj == nK - 1) ? 0u : 1u;
                  const uint64_t bk = bt + (uint64_t)((4 * kj) * (kSeqBlock >> 4));
                  // K step 0: windows at rows 8, 4, 0 (8 - 4p) of the sequence
                  umma_i8(dcol, at, bk + 8, idesc16, acc0);
                  umma_i8(dcol, at + kPlaneCols, bk + 4, idesc16, 1);
                  umma_i8(dcol, at + 2 * kPlaneCols, bk, idesc16, 1);
                  // K step 1: 32 k' further (two 16-k blocks)
                  const uint64_t bk1 = bk + 2 * (kSeqBlock >> 4);
                  umma_i8(dcol, at + 8, bk1 + 8, idesc16, 1);
                  umma_i8(dcol, at + kPlaneCols + 8, bk1 + 4, idesc16, 1);
                  umma_i8(dcol, at + 2 * kPlaneCols + 8, bk1, idesc16, 1);
                }
              }
            }
            umma_commit(&afree[gb]);  // the group's slots are free once these finish
          }
          __syncwarp();
          if (++gb == 2) {
            gb = 0;
            gph ^= 1u;
          }
        }
        if (!go) break;
        if (issuer) umma_commit(&dfull[b]);  // this issuer's accumulators are complete
        __syncwarp();
      }
    }
  } else if (warp >= kGenWarp0) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kRegsLow));
    // ---- A-tile generators: row r = 32 gq + lane of tile d is a(64 d + r - c),
    // c = 0..63; TMEM column jc of a digit plane holds c = 4 jc .. 4 jc + 3,
    // the four bytes from R[c0 - 64 d - r + 4 jc]: 17 aligned words and a
    // funnel shift give the 16 columns.
    const int gq = warp - kGenWarp0;
    const uint32_t lrow = tmem + ((uint32_t)(32 * gq) << 16);
    int gb = 0;
    uint32_t gph = 0;
    bool first = true, go = true;
    for (int s = 0; s < total_stages && go; ++s) {
      for (int j = 0; j < nw && go; ++j) {
        if (scr && s >= 1) {
          // the wire's next-stage digits, from the V/eps the epilogue wrote
          go = __all_sync(0xffffffffu, mbar_wait_sleep(&svfull[j], (s - 1) & 1, abort, lim));
          if (!go) break;
          table_digits<NT>(svb + (uint32_t)j * (L.svsz / 8), vsw + 3 * j, nk, (int)c0,
                           tabq + (uint32_t)(j * NT) * L.tabsz, L.plane, 32 * kGenWarp0,
                           32 * kGenWarps);
          // all four warps' digits are written before any tile reads them (a
          // bounded mbarrier, not a named barrier: a warp that stops on an
          // abort must not leave the others waiting)
          __syncwarp();
          if (lane == 0) mbar_arrive(&gdone[j]);
          go = __all_sync(0xffffffffu, mbar_wait(&gdone[j], (s - 1) & 1, abort, lim));
          if (!go) break;
        }
        const uint8_t* tq = tabq + (scr ? (uint32_t)(j * NT) * L.tabsz : 0u);
        for (int d0 = dmin; d0 <= dmax; d0 += G) {
          const int gn = min(G, dmax - d0 + 1);
          if (!first) {
            go = __all_sync(0xffffffffu, mbar_wait_sleep(&afree[gb], gph ^ 1u, abort, lim));
            if (!go) break;
          }
          tc_fence_after();
          for (int jj = 0; jj < gn; ++jj) {
            const uint32_t y0 = c0 - (uint32_t)(64 * (d0 + jj) + 32 * gq + lane);
            const uint32_t sh = 8u * (y0 & 3u);
#pragma unroll
            for (int t = 0; t < NT; ++t) {
              const uint32_t ta =
                  lrow + acol0 + (uint32_t)(((gb * G + jj) * NT + t) * kTileCols);
#pragma unroll
              for (int p = 0; p < kDigits; ++p) {
                const uint32_t* tw = reinterpret_cast<const uint32_t*>(
                                         tq + (uint32_t)(t * 3 + p) * L.plane) +
                                     (y0 >> 2);
                uint32_t w[17], r[16];
#pragma unroll
                for (int k = 0; k < 17; ++k) w[k] = tw[k];
#pragma unroll
                for (int jc = 0; jc < 16; ++jc) r[jc] = __funnelshift_r(w[jc], w[jc + 1], sh);
                tmem_st16(ta + p * kPlaneCols, r);
              }
            }
          }
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
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kRegsHigh));
    // ---- drain / epilogue: warp (q, hh) takes rows 128 mi + 32 q + lane of
    // the row tiles mi = hh, hh + 2, ... of the current wire.
    const int q = warp & 3, hh = warp >> 2;
    const uint32_t lrow = tmem + ((uint32_t)(32 * q) << 16);
    const float inv_base = 1.f / 254.f;
    const float hf = (float)h, h2f = (float)(h / 2.0), h6f = (float)(h / 6.0);
    const double dec_hb = inv_hbar / (kBase * kBase);
    uint32_t it = 0;
    bool go = true;
    for (int s = 0; s < total_stages && go; ++s) {
      const int stg = s & 3, step = s >> 2;
      for (int j = 0; j < nw; ++j, ++it) {
        const int b = it & 1;
        bool got = true;
        // decode factors VS_t / (hbar 254^2) 2^-sexp (VS of a screened wire's
        // stage was set by these warps when they built its table); scaling a
        // float by a power of two is exact
        float fac[4];
#pragma unroll
        for (int v = 0; v < 4; ++v)
          fac[v] = (float)(vsw[(scr ? 3 * j : 0) + mat_of<NT>(v)] * dec_hb) *
                   ldexpf(1.f, -sx[(warp * kMaxW + j) * 4 + v]);
        // drive M(t)/hbar of this stage: lane 0 evaluates pulse 0, lane 1
        // pulse 1, summed in that order
        double mr = 0.0, mim = 0.0;
        if (lane < 2) {
          const double tt = wtb[2 * j + (step & 1)] + (stg == 0 ? 0.0 : (stg == 3 ? h : h / 2.0));
          const double* pc = pulse + j * 8 + 4 * lane;
          const double u = tt - pc[0];
          const double env = exp(pc[1] * u * u);
          mr = pc[2] * env;
          mim = pc[3] * env;
        }
        const float Mr = (float)((__shfl_sync(0xffffffffu, mr, 0) + __shfl_sync(0xffffffffu, mr, 1)) *
                                 inv_hbar);
        const float Mi = (float)((__shfl_sync(0xffffffffu, mim, 0) +
                                  __shfl_sync(0xffffffffu, mim, 1)) *
                                 inv_hbar);
        const double gw = wpar[j].y, gj = gaph[j];
        const int64_t wo = woff[j];
        // this thread's elements: loads issued before the accumulator wait
        float4 ysv[kMaxTilesPerWarp], accv[kMaxTilesPerWarp], yfv[kMaxTilesPerWarp];
        double ekh[kMaxTilesPerWarp];
#pragma unroll
        for (int i = 0; i < kMaxTilesPerWarp; ++i) {
          const int k = (hh + 2 * i) * kTileRows + 32 * q + lane;
          if (k < nk) {
            ysv[i] = a.ws_ys[wo + k];
            accv[i] = a.ws_acc[wo + k];
            yfv[i] = a.ws_yf[wo + k];
            ekh[i] = (Ee[k] + Eh[k]) * inv_hbar;
          }
        }
        if (got) got = mbar_wait(&dfull[b], (it >> 1) & 1, abort, lim);
        got = __all_sync(0xffffffffu, got);
        if (got) tc_fence_after();
        float cm[4] = {0.f, 0.f, 0.f, 0.f};
        double n1 = 0.0, pr = 0.0, pim = 0.0;
        float4 nx[kMaxTilesPerWarp];
#pragma unroll
        for (int i = 0; i < kMaxTilesPerWarp; ++i) {
          const int mi = hh + 2 * i;
          nx[i] = make_float4(0.f, 0.f, 0.f, 0.f);
          if (mi >= nM) break;
          uint32_t r[16];
          if (got) {
            const uint32_t col = lrow + (uint32_t)b * dstride + 16u * (uint32_t)mi;
            tmem_ld8(col, r);
            tmem_ld8(col + 8, r + 8);
            tmem_ld_wait();
          }
          const int k = mi * kTileRows + 32 * q + lane;
          if (!got || k >= nk) continue;
          // exchange sums / hbar from the exact digit products (D2 | D3 | D4)
          float exh[4];
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const float e = (float)(int)r[c] +
                            ((float)(int)r[4 + c] + (float)(int)r[8 + c] * inv_base) * inv_base;
            exh[c] = e * fac[c];
          }
          const float4 ysf = ysv[i];
          // diagonal RHS (SBEs.py:1962-1975, 2325-2337, 2623-2636) / hbar
          const float omr = Mr + exh[0];
          const float omi = Mi + exh[1];
          const double sumh = (ekh[i] + gj) - (double)(exh[2] + exh[3]);
          const float nn = ysf.z + ysf.w - 1.f;
          const double prd = ysf.x, pid = ysf.y;
          const float f0 = (float)(sumh * pid - gw * prd) - omi * nn;
          const float f1 = (float)(-(sumh * prd) - gw * pid) + omr * nn;
          const float f2 = 2.f * (omi * ysf.x - omr * ysf.y);
          // RK4 stage combination (integrator.py:143-157)
          float4 nxt;
          const int64_t e = wo + k;
          if (stg == 0) {
            a.ws_acc[e] = make_float4(f0, f1, f2, f2);
            nxt = make_float4(ysf.x + h2f * f0, ysf.y + h2f * f1, ysf.z + h2f * f2,
                              ysf.w + h2f * f2);
            n1 += (double)nxt.z + (double)nxt.w;
          } else if (stg == 3) {
            const float4 af = accv[i];
            double4 yv = g_y[e];
            yv.x += (double)(h6f * (af.x + f0));
            yv.y += (double)(h6f * (af.y + f1));
            yv.z += (double)(h6f * (af.z + f2));
            yv.w += (double)(h6f * (af.w + f2));
            g_y[e] = yv;
            nxt = make_float4((float)yv.x, (float)yv.y, (float)yv.z, (float)yv.w);
            a.ws_yf[e] = nxt;
            n1 += yv.z + yv.w;
            pr += yv.x;
            pim += yv.y;
          } else {
            const float4 af = accv[i];
            a.ws_acc[e] = make_float4(af.x + 2.f * f0, af.y + 2.f * f1, af.z + 2.f * f2,
                                      af.w + 2.f * f2);
            const float4 yf = yfv[i];
            const float c2 = stg == 1 ? h2f : hf;
            nxt = make_float4(yf.x + c2 * f0, yf.y + c2 * f1, yf.z + c2 * f2, yf.w + c2 * f2);
            n1 += (double)nxt.z + (double)nxt.w;
          }
          a.ws_ys[e] = nxt;
          nx[i] = nxt;
          cm[0] = fmaxf(cm[0], fabsf(nxt.x));
          cm[1] = fmaxf(cm[1], fabsf(nxt.y));
          cm[2] = fmaxf(cm[2], fabsf(nxt.z));
          cm[3] = fmaxf(cm[3], fabsf(nxt.w));
        }
        // the wire's accumulators are free again
        tc_fence_before();
        __syncwarp();
        if (lane == 0 && got) mbar_arrive(&dfree[b]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
          for (int v = 0; v < 4; ++v) cm[v] = fmaxf(cm[v], __shfl_xor_sync(0xffffffffu, cm[v], o));
          n1 += __shfl_xor_sync(0xffffffffu, n1, o);
          pr += __shfl_xor_sync(0xffffffffu, pr, o);
          pim += __shfl_xor_sync(0xffffffffu, pim, o);
        }
        uint8_t* rb = red + ((it & 1) * kEpiWarps) * 48;
        if (lane == 0) {
          float* rf = reinterpret_cast<float*>(rb + warp * 48);
          double* rd = reinterpret_cast<double*>(rb + warp * 48 + 16);
          rf[0] = cm[0];
          rf[1] = cm[1];
          rf[2] = cm[2];
          rf[3] = cm[3];
          rd[0] = n1;
          rd[1] = pr;
          rd[2] = pim;
        }
        if (stg == 3 && tid == 0) wtb[2 * j + ((step + 1) & 1)] = wtb[2 * j + (step & 1)] + h;
        if (tid == 0) snap[it & 1] = *abort;
        named_sync(1, kEpiThreads);
        if (snap[it & 1]) {
          go = false;
          break;
        }
        // exact column scales of the next stage point (largest |x| in [1/4, 1/2))
        float cma[4] = {0.f, 0.f, 0.f, 0.f};
        for (int wq = 0; wq < kEpiWarps; ++wq) {
          const float* rf = reinterpret_cast<const float*>(rb + wq * 48);
#pragma unroll
          for (int v = 0; v < 4; ++v) cma[v] = fmaxf(cma[v], rf[v]);
        }
        int se[4];
        float sc[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          int e2 = 0;
          se[v] = 0;
          if (cma[v] > 0.f && isfinite(cma[v])) {
            frexpf(cma[v], &e2);
            se[v] = min(max(-1 - e2, -120), 120);
          }
          sc[v] = ldexpf(1.f, se[v]);
        }
        if (s + 1 < total_stages) {
#pragma unroll
          for (int i = 0; i < kMaxTilesPerWarp; ++i) {
            const int k = (hh + 2 * i) * kTileRows + 32 * q + lane;
            if (k >= nk) continue;
            const float xv[4] = {nx[i].x * sc[0], nx[i].y * sc[1], nx[i].z * sc[2],
                                 nx[i].w * sc[3]};
            const uint32_t ob = (uint32_t)(k >> 4) * kSeqBlock + (uint32_t)(k & 15);
#pragma unroll
            for (int v = 0; v < 4; ++v) {
              int d1, d2, d3;
              digits3(xv[v], d1, d2, d3);
              uint8_t* xq = xbase + (uint32_t)(j * NT + mat_of<NT>(v)) * L.seq + ob + 16 * v;
              xq[8 * 16] = (uint8_t)d1;
              xq[12 * 16] = (uint8_t)d2;
              xq[16 * 16] = (uint8_t)d3;
            }
          }
          if (lane < 4) {
            const int sv = lane == 0 ? se[0] : (lane == 1 ? se[1] : (lane == 2 ? se[2] : se[3]));
            sx[(warp * kMaxW + j) * 4 + lane] = sv;
          }
          // digit stores become visible to the tensor cores
          fence_async_smem();
          __syncwarp();
          if (lane == 0) mbar_arrive(&xfull[j]);
        }
        double n1t = 0.0, prt = 0.0, pit = 0.0;
        for (int wq = 0; wq < kEpiWarps; ++wq) {
          const double* rd = reinterpret_cast<const double*>(rb + wq * 48 + 16);
          n1t += rd[0];
          prt += rd[1];
          pit += rd[2];
        }
        if (tid == 0) {
          if (stg == 3 && a.P && a.p_stride > 0 && (step + 1) % a.p_stride == 0) {
            const int rr = (step + 1) / a.p_stride - 1;
            const PsbWire& wd = a.wires[grp.wire[j]];
            if (rr < a.p_cap && wd.p_off >= 0 && wd.p_off + rr < a.n_P) {
              a.P[2 * (wd.p_off + rr)] = wpar[j].w * prt;
              a.P[2 * (wd.p_off + rr) + 1] = wpar[j].w * pit;
            }
          }
        }
        // screened: this wire's table for its next stage, from the n1D of the
        // stage point just written (CalcScreenedArrays, coulomb.py:1218-1223)
        if (scr && s + 1 < total_stages) {
          double n1d = n1t / 2.0 / tb.L;
          n1d = n1d < tb.dens_max ? n1d : tb.dens_max;
          table_scaled<NT>(qcs, vts, nk, true, n1d, svb + (uint32_t)j * (L.svsz / 8), vsw + 3 * j,
                           sred, 0, kEpiThreads, 1);
          if (tid == 0) mbar_arrive(&svfull[j]);
        }
      }
    }
  }

  // ---- teardown -----------------------------------------------------------------
  // every MMA of every issuer has completed before TMEM is released
  if (warp >= kMmaWarp && lane == 0) umma_commit(final_bar);
  if (warp == kMmaWarp && lane == 0) {
    bool done = false;
    for (uint32_t i = 0; i < kSpinLimit && !done; ++i) done = mbar_try_wait(final_bar, 0);
    if (!done) *abort = 1;
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(ncols));
  if (tid < nw) {
    PsbWire* wp = a.wires + grp.wire[tid];
    if (*abort) {
      wp->status = PSB_ERR_TIMEOUT;
    } else {
      wp->t = wtb[2 * tid + (a.nsteps & 1)];
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

template <int NT>
int smem_total(int nk, int wgroup, bool scr) {
  return (int)WLayout<NT>(nk, wgroup, scr).total;
}

template <int NT>
bool fits(int nk, int wgroup, bool scr) {
  return nk >= 2 && nk <= kMaxNkW && wgroup >= 1 && wgroup <= kMaxW &&
         (NT == 1 || mtiles_of(nk) <= 4) && slots_of<NT>(nk) >= 2 &&
         WLayout<NT>(nk, wgroup, scr).total <= kMaxDynSmem;
}

template <int NT>
int launch(Args a, int nkmax, cudaStream_t s) {
  const bool scr = a.screened != 0;
  if (!fits<NT>(nkmax, a.wgroup, scr))
    return set_error(PSB_ERR_SIZE,
                     "per-wire split form: nk %d with %d wires per group does not fit", nkmax,
                     a.wgroup);
  const uint32_t smem = WLayout<NT>(nkmax, a.wgroup, scr).total;
  cudaFuncAttributes fa{};
  cudaError_t e = cudaFuncGetAttributes(&fa, split_wire_kernel<NT>);
  if (e != cudaSuccess)
    return set_error(PSB_ERR_CUDA, "cudaFuncGetAttributes: %s", cudaGetErrorString(e));
  if (fa.numRegs != kRegsLaunch || fa.maxThreadsPerBlock < kThreadsS)
    return set_error(PSB_ERR_UNSUPPORTED,
                     "split_wire_kernel built with %d registers per thread (needs %d) and at "
                     "most %d threads (needs %d)",
                     fa.numRegs, kRegsLaunch, fa.maxThreadsPerBlock, kThreadsS);
  e = cudaFuncSetAttribute(split_wire_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
  if (e != cudaSuccess)
    return set_error(PSB_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
  a.smem_bytes = smem;
  split_wire_kernel<NT><<<a.ngroups, kThreadsS, smem, s>>>(a);
  return check_cuda("split_wire_kernel");
}

}  // namespace splitw
}  // namespace psb

using namespace psb;

extern "C" int psb_split_wire_max_group(int nk, int tab_flags) {
  const bool scr = (tab_flags & PSB_TAB_SCREENED) != 0;
  const bool shared = (tab_flags & PSB_TAB_SHARED_V) != 0;
  for (int w = splitw::kMaxW; w >= 1; --w)
    if (shared ? splitw::fits<1>(nk, w, scr) : splitw::fits<3>(nk, w, scr)) return w;
  return 0;
}

extern "C" int psb_split_wire_smem_bytes(int nk, int wgroup, int tab_flags) {
  const bool scr = (tab_flags & PSB_TAB_SCREENED) != 0;
  const bool shared = (tab_flags & PSB_TAB_SHARED_V) != 0;
  if (nk < 2 || nk > splitw::kMaxNkW || wgroup < 1 || wgroup > splitw::kMaxW)
    return set_error(PSB_ERR_SIZE, "nk %d or wgroup %d out of range", nk, wgroup);
  return shared ? splitw::smem_total<1>(nk, wgroup, scr) : splitw::smem_total<3>(nk, wgroup, scr);
}

extern "C" int psb_rk4_split_wire(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                                  int64_t n_tabdata, PsbWire* d_wires, int nw,
                                  const PsbSplitGroup* d_groups, int ngroups, int wgroup,
                                  int nkmax, int tab_flags, double* d_y, int64_t n_state,
                                  void* d_ws, int64_t n_ws_bytes, int nsteps, double dt,
                                  double* d_P, int64_t n_P, int p_stride, int p_cap,
                                  const PsbModel* model, void* stream) {
  if (!d_tables || !d_tabdata || !d_wires || !d_groups || !d_y || !d_ws || !model || ntab <= 0 ||
      nw < 0 || ngroups < 0)
    return set_error(PSB_ERR_INVALID, "psb_rk4_split_wire: null pointer or bad count");
  if (wgroup < 1 || wgroup > splitw::kMaxW)
    return set_error(PSB_ERR_INVALID, "psb_rk4_split_wire: wgroup must be 1..%d", splitw::kMaxW);
  if (!(tab_flags & PSB_TAB_EXCITONS))
    return set_error(PSB_ERR_INVALID, "psb_rk4_split_wire: tables without excitons");
  if (nkmax < 2 || wgroup > psb_split_wire_max_group(nkmax, tab_flags))
    return set_error(PSB_ERR_SIZE, "psb_rk4_split_wire: nkmax %d too large for wgroup %d",
                     nkmax, wgroup);
  if (n_ws_bytes < psb_split_ws_bytes(n_state))
    return set_error(PSB_ERR_SIZE,
                     "psb_rk4_split_wire: workspace needs psb_split_ws_bytes(n_state)");
  if (((uintptr_t)d_ws & 31) != 0 || ((uintptr_t)d_y & 31) != 0)
    return set_error(PSB_ERR_INVALID,
                     "psb_rk4_split_wire: state and workspace must be 32-byte aligned");
  if (!(model->hbar > 0.0)) return set_error(PSB_ERR_INVALID, "model.hbar must be > 0");
  if (nsteps < 0) return set_error(PSB_ERR_INVALID, "nsteps < 0");
  if (nsteps == 0 || ngroups == 0) return PSB_OK;
  splitw::Args a{};
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
  a.wgroup = wgroup;
  a.screened = (tab_flags & PSB_TAB_SCREENED) ? 1 : 0;
  a.spin_limit = split::wait_limit();
  cudaStream_t st = (cudaStream_t)stream;
  if (tab_flags & PSB_TAB_SHARED_V) return splitw::launch<1>(a, nkmax, st);
  return splitw::launch<3>(a, nkmax, st);
}
