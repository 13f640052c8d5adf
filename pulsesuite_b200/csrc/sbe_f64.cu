// sbe_f64.cu -- fused FP64 SBE right-hand side, RK4 step and leapfrog step.
//
// One CTA owns one wire for the whole call: the wire's state stays in shared
// memory and registers across all `nsteps` steps, so HBM sees the state once
// in and once out per call.  Work per right-hand side is dominated by the
// three Toeplitz exchange sums (pulsesuite/PSTD3D/SBEs.py:896-921):
//   Omega_k += sum_k' Veh(|k-k'|) p_k'   Se_k -= sum Vee ne   Sh_k -= sum Vhh nh
// i.e. 4 FP64 FMAs per (k, k') pair.
//
// Exchange mapping.  Thread (ob, kc) owns R consecutive outputs
// k = ob*R .. ob*R+R-1 and a chunk of sources k' (kc selects the chunk).  For
// each k' it loads the 4 source values (a shared-memory broadcast) and keeps
// the R values V(k - k') of each table in a register window that slides by one
// entry per k', so one new table value per table and k' is loaded.  The
// symmetric tables Vs[d + doff] = V(|d|) (0 at d = 0, the excluded q = 0 term,
// and beyond the grid) are stored with one pad double every R entries, which
// makes the stride-R reads of a warp bank-conflict free.  When the three
// tables are equal (PSB_TAB_SHARED_V, the regularised-wire potential) only one
// window is kept.  Partial sums of the kc chunks meet in shared memory and are
// added in a fixed order, so a wire's result never depends on the other wires
// of the launch.
#include <math.h>

#include "psb_common.cuh"

namespace psb {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

enum Mode { kRhs = 0, kRk4 = 1, kLeapfrog = 2, kCalcH = 3 };

struct Geo {
  int nk, nkp, nb, kc, chunk, yslen, doff, vlen, vphys;
};

template <int R>
__host__ __device__ inline Geo geometry(int nk) {
  Geo g;
  g.nk = nk;
  g.nkp = (nk + R - 1) / R * R;
  g.nb = g.nkp / R;
  int kc = kThreads / g.nb;
  if (kc < 1) kc = 1;
  int c = (g.nkp + kc - 1) / kc;
  c = (c + R - 1) / R * R;
  g.chunk = c;
  g.kc = (g.nkp + c - 1) / c;
  g.yslen = g.kc * g.chunk;
  g.doff = g.yslen + 1;
  g.vlen = g.nkp + g.yslen + 2;
  g.vphys = g.vlen + g.vlen / R + 1;
  return g;
}

// Shared-memory layout (doubles) of one wire.
struct Smem {
  int ys, red, v, eps, stage, scratch, total;
};

template <int R>
__host__ __device__ inline Smem smem_layout(const Geo& g, int ntab) {
  Smem s;
  s.ys = 0;                          // 4 SoA arrays of yslen: p_re, p_im, ne, nh
  s.red = s.ys + 4 * g.yslen;        // [kc][4][nkp] partial exchange sums
  s.v = s.red + 4 * g.kc * g.nkp;    // ntab skewed symmetric tables of vphys
  s.eps = s.v + ntab * g.vphys;      // eps(q) when screened (nkp)
  s.stage = s.eps + g.nkp;           // [8][nkp]: RK4 k1 and k2/k2+k3, leapfrog X3
  s.scratch = s.stage + 8 * g.nkp;   // block reductions: kWarps*4 + 4
  s.total = s.scratch + kWarps * 4 + 4;
  return s;
}

template <int R>
__device__ __forceinline__ int skew(int i) {
  return i + i / R;
}

struct Batch {
  const PsbTable* tables;
  int ntab;
  const double* tabdata;
  int64_t n_tabdata;
  PsbWire* wires;
  int nw;
  const int32_t* order;
  double* y;   // RK4 state, leapfrog X2, RHS input
  double* y1;  // leapfrog X1
  double* dy;  // RHS output
  int64_t n_state;
  const double* field;
  int64_t field_stride;
  int64_t n_field;
  int nsteps;
  double dt;
  double* P;
  int64_t n_P;
  int p_stride;
  int p_cap;
  double hbar;
  int nk_limit;  // largest nk the launch's shared memory was sized for
};

// Sum of n <= 4 values over the block; every thread returns the same totals.
__device__ __forceinline__ void block_sum(double* v, int n, double* scratch) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = 0; i < n; ++i) v[i] = warp_sum(v[i]);
  if (lane == 0)
    for (int i = 0; i < n; ++i) scratch[warp * 4 + i] = v[i];
  __syncthreads();
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) s += scratch[w * 4 + i];
    v[i] = s;
  }
  __syncthreads();
}

// Drive E(t) of a wire (PsbWire doc): sum of up to two Gaussian pulses.
__device__ __forceinline__ void drive(const PsbWire& w, double t, double& er, double& ei) {
  er = 0.0;
  ei = 0.0;
  for (int j = 0; j < w.npulse && j < 2; ++j) {
    double u = (t - w.t0[j]) / w.fwhm[j];
    double env = w.amp[j] * exp(-4.0 * log(2.0) * u * u);
    double s, c;
    sincos(w.phase[j], &s, &c);
    er += env * c;
    ei += env * s;
  }
}

// Fill the symmetric tables of a wire, screened by eps when given.
template <int R, int NT, bool SCREEN>
__device__ void fill_tables(const Geo& g, const double* __restrict__ blk, double* vs,
                            const double* eps) {
  for (int i = threadIdx.x; i < g.vlen; i += kThreads) {
    int d = i - g.doff;
    d = d < 0 ? -d : d;
    const bool in = d > 0 && d < g.nk;
    const double e = (SCREEN && in) ? eps[d] : 1.0;
    const int p = skew<R>(i);
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      double v = in ? blk[t * g.nk + d] : 0.0;
      if (SCREEN) v = v / e;
      vs[t * g.vphys + p] = v;
    }
  }
}

// Static screening of the current stage state (coulomb.py:1218-1230): n1D
// from the stage densities, then eps(q) for q < nk.
__device__ void screen_stage(const Geo& g, const PsbTable& tb, const double* __restrict__ blk,
                             const double* ys, double* eps, double* scratch) {
  double s[1] = {0.0};
  for (int k = threadIdx.x; k < g.nk; k += kThreads)
    s[0] += ys[2 * g.yslen + k] + ys[3 * g.yslen + k];
  block_sum(s, 1, scratch);
  double n1d = s[0] / 2.0 / tb.L;
  n1d = n1d < tb.dens_max ? n1d : tb.dens_max;
  const int nk = g.nk;
  for (int q = threadIdx.x; q < nk; q += kThreads) {
    double chie = blk[5 * nk + q], chih = blk[6 * nk + q];
    double qe = blk[7 * nk + q], qh = blk[8 * nk + q];
    double le = log(fabs((qe - kPi * n1d) / (qe + n1d)));
    double lh = log(fabs((qh - kPi * n1d) / (qh + n1d)));
    eps[q] = (1.0 - __dmul_rn(__dmul_rn(chie, 2.0), le)) - __dmul_rn(__dmul_rn(chih, 2.0), lh);
  }
  __syncthreads();
}

// Exchange sums of one stage into red[kc][c][k] (c: Omega_re, Omega_im,
// sum Vee ne, sum Vhh nh).
template <int R, int NT>
__device__ __forceinline__ void exchange(const Geo& g, const double* ys, const double* vs,
                                         double* red) {
  const int t = threadIdx.x;
  const int ob = t % g.nb;
  const int kc = t / g.nb;
  if (kc >= g.kc) return;
  const int k0 = kc * g.chunk;
  const int kout0 = ob * R;
  const double* __restrict__ VE = vs;
  const double* __restrict__ VW = vs + (NT == 3 ? g.vphys : 0);
  const double* __restrict__ VH = vs + (NT == 3 ? 2 * g.vphys : 0);
  const double* __restrict__ A = ys;
  const double* __restrict__ B = ys + g.yslen;
  const double* __restrict__ NE = ys + 2 * g.yslen;
  const double* __restrict__ NH = ys + 3 * g.yslen;
  double ar[R], ai[R], ae[R], ah[R];
  double we[R], ww[R], wh[R];
#pragma unroll
  for (int r = 0; r < R; ++r) ar[r] = ai[r] = ae[r] = ah[r] = 0.0;
  int j = kout0 - k0 + g.doff;  // table index of r = 0 at k' = k0
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int p = skew<R>(j + r);
    we[r] = VE[p];
    if (NT == 3) {
      ww[r] = VW[p];
      wh[r] = VH[p];
    }
  }
  for (int kk = 0; kk < g.chunk; kk += R) {
#pragma unroll
    for (int u = 0; u < R; ++u) {
      const int kp = k0 + kk + u;
      const double a = A[kp], b = B[kp], ne = NE[kp], nh = NH[kp];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        ar[r] = fma(we[r], a, ar[r]);
        ai[r] = fma(we[r], b, ai[r]);
        ae[r] = fma(NT == 3 ? ww[r] : we[r], ne, ae[r]);
        ah[r] = fma(NT == 3 ? wh[r] : we[r], nh, ah[r]);
      }
#pragma unroll
      for (int r = R - 1; r > 0; --r) {
        we[r] = we[r - 1];
        if (NT == 3) {
          ww[r] = ww[r - 1];
          wh[r] = wh[r - 1];
        }
      }
      --j;
      const int p = skew<R>(j);
      we[0] = VE[p];
      if (NT == 3) {
        ww[0] = VW[p];
        wh[0] = VH[p];
      }
    }
  }
  double* rr = red + (size_t)kc * 4 * g.nkp;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    rr[kout0 + r] = ar[r];
    rr[g.nkp + kout0 + r] = ai[r];
    rr[2 * g.nkp + kout0 + r] = ae[r];
    rr[3 * g.nkp + kout0 + r] = ah[r];
  }
}

// f(k) of element k from the reduced exchange sums (the diagonal of dpdt,
// dCdt, dDdt: SBEs.py:1962-1975, 2325-2337, 2623-2636).
__device__ __forceinline__ void rhs_element(const Geo& g, int k, const double* ys,
                                            const double* red, const double* __restrict__ Ee,
                                            const double* __restrict__ Eh, double gap,
                                            double hg, double hbar, double mr, double mi,
                                            bool exc, double f[4]) {
  double omr = mr, omi = mi, xe = 0.0, xh = 0.0;
  if (exc) {
    for (int c = 0; c < g.kc; ++c) {
      const double* rr = red + (size_t)c * 4 * g.nkp;
      omr += rr[k];
      omi += rr[g.nkp + k];
      xe += rr[2 * g.nkp + k];
      xh += rr[3 * g.nkp + k];
    }
  }
  double se = (Ee[k] + gap) - xe;
  double sh = Eh[k] - xh;
  double a = ys[k], b = ys[g.yslen + k];
  double ne = ys[2 * g.yslen + k], nh = ys[3 * g.yslen + k];
  double xr = sh * a + se * a;
  double xi = sh * b + se * b;
  xr = xr - omr * ne;
  xi = xi - omi * ne;
  xr = xr - omr * nh;
  xi = xi - omi * nh;
  xr = xr + omr;
  xi = xi + omi;
  xr = xr + hg * b;
  xi = xi - hg * a;
  f[0] = xi / hbar;
  f[1] = -xr / hbar;
  double u = omi * a - omr * b;
  double dn = (u + u) / hbar;
  f[2] = dn;
  f[3] = dn;
}

template <int R, int EPT, int MODE, bool SCREEN, int NT>
__global__ void __launch_bounds__(kThreads, EPT <= 2 ? 2 : 1) sbe_f64_kernel(Batch bt) {
  extern __shared__ double smem[];
  const int wi = bt.order ? bt.order[blockIdx.x] : (int)blockIdx.x;
  if (wi < 0 || wi >= bt.nw) return;
  PsbWire* wp = bt.wires + wi;
  const PsbWire w = *wp;
  if (w.table < 0 || w.table >= bt.ntab) {
    if (threadIdx.x == 0) wp->status = PSB_ERR_INVALID;
    return;
  }
  const PsbTable tb = bt.tables[w.table];
  if (tb.nk < 2 || tb.nk > bt.nk_limit || w.off < 0 || w.off + tb.nk > bt.n_state ||
      tb.off < 0 || tb.off + 9 * (int64_t)tb.nk > bt.n_tabdata) {
    if (threadIdx.x == 0) wp->status = PSB_ERR_SIZE;
    return;
  }
  if (NT == 1 && (tb.flags & PSB_TAB_SHARED_V) == 0) {
    if (threadIdx.x == 0) wp->status = PSB_ERR_INVALID;
    return;
  }
  const Geo g = geometry<R>(tb.nk);
  const Smem L = smem_layout<R>(g, NT);
  double* ys = smem + L.ys;
  double* red = smem + L.red;
  double* vs = smem + L.v;
  double* eps = smem + L.eps;
  double* stage = smem + L.stage;
  double* scratch = smem + L.scratch;
  const double* blk = bt.tabdata + tb.off;
  const double* Ee = blk + 3 * tb.nk;
  const double* Eh = blk + 4 * tb.nk;
  const bool exc = (tb.flags & PSB_TAB_EXCITONS) != 0;
  const bool scr = SCREEN && (tb.flags & PSB_TAB_SCREENED) != 0;
  const double hbar = bt.hbar;
  const double hg = hbar * w.gamma;
  const int tid = threadIdx.x;
  const int nkp = g.nkp;

  // Zero the padded sources, load the state.
  for (int i = tid; i < 4 * g.yslen; i += kThreads) ys[i] = 0.0;
  __syncthreads();
  double yb[EPT][4];  // RK4 base state / leapfrog X1
  const double2* y2 = reinterpret_cast<const double2*>(bt.y + 4 * w.off);
  const double2* y1g = MODE == kLeapfrog ? reinterpret_cast<const double2*>(bt.y1 + 4 * w.off)
                                         : nullptr;
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    int k = tid + e * kThreads;
    if (k < g.nk) {
      double2 pa = y2[2 * k], pb = y2[2 * k + 1];
      ys[k] = pa.x;
      ys[g.yslen + k] = pa.y;
      ys[2 * g.yslen + k] = pb.x;
      ys[3 * g.yslen + k] = pb.y;
      if (MODE == kLeapfrog) {
        double2 qa = y1g[2 * k], qb = y1g[2 * k + 1];
        yb[e][0] = qa.x;
        yb[e][1] = qa.y;
        yb[e][2] = qb.x;
        yb[e][3] = qb.y;
      } else {
        yb[e][0] = pa.x;
        yb[e][1] = pa.y;
        yb[e][2] = pb.x;
        yb[e][3] = pb.y;
      }
    }
  }
  if (exc && !scr) fill_tables<R, NT, false>(g, blk, vs, eps);
  __syncthreads();

  const int nst = (MODE == kRhs || MODE == kCalcH) ? 1 : bt.nsteps;
  const int nstage = MODE == kRk4 ? 4 : 1;
  const double h = bt.dt;
  double t = w.t;
  int steps = w.steps;
  for (int s = 0; s < nst; ++s) {
    double er_lf = 0.0, ei_lf = 0.0;
    if (MODE == kLeapfrog) {
      int64_t fi = (int64_t)wi * bt.field_stride + 2 * (int64_t)steps;
      if (bt.field && fi >= 0 && fi + 1 < bt.n_field) {
        er_lf = bt.field[fi];
        ei_lf = bt.field[fi + 1];
      }
    }
    for (int st = 0; st < nstage; ++st) {
      if (exc) {
        if (scr) {
          screen_stage(g, tb, blk, ys, eps, scratch);
          fill_tables<R, NT, true>(g, blk, vs, eps);
          __syncthreads();
        }
        exchange<R, NT>(g, ys, vs, red);
      }
      __syncthreads();
      double er, ei;
      if (MODE == kLeapfrog) {
        er = er_lf;
        ei = ei_lf;
      } else {
        double ts = st == 0 ? t : (st == 3 ? t + h : t + h / 2.0);
        drive(w, ts, er, ei);
      }
      const double mr = -w.mscale * er, mi = -w.mscale * ei;
#pragma unroll
      for (int e = 0; e < EPT; ++e) {
        const int k = tid + e * kThreads;
        if (k >= g.nk) continue;
        double f[4];
        if (MODE == kCalcH) {
          // renormalised H diagonals (CalcH, SBEs.py:819-935): Heh (Rabi
          // frequency), Hee, Hhh in the slots of dy
          double omr = mr, omi = mi, xe = 0.0, xh = 0.0;
          if (exc) {
            for (int c = 0; c < g.kc; ++c) {
              const double* rr = red + (size_t)c * 4 * g.nkp;
              omr += rr[k];
              omi += rr[g.nkp + k];
              xe += rr[2 * g.nkp + k];
              xh += rr[3 * g.nkp + k];
            }
          }
          double2* d2 = reinterpret_cast<double2*>(bt.dy + 4 * w.off);
          d2[2 * k] = make_double2(omr, omi);
          d2[2 * k + 1] = make_double2((Ee[k] + w.gap) - xe, Eh[k] - xh);
          continue;
        }
        rhs_element(g, k, ys, red, Ee, Eh, w.gap, hg, hbar, mr, mi, exc, f);
        if (MODE == kRhs) {
          double2* d2 = reinterpret_cast<double2*>(bt.dy + 4 * w.off);
          d2[2 * k] = make_double2(f[0], f[1]);
          d2[2 * k + 1] = make_double2(f[2], f[3]);
        } else if (MODE == kRk4) {
          // Stage order of integrator.py:143-157; k1 in stage[c], k2 and
          // then k3 + k2 in stage[4 + c] (owner-thread slots, no sync needed).
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            double* k1 = stage + c * nkp + k;
            double* dym = stage + (4 + c) * nkp + k;
            double v;
            if (st == 0) {
              *k1 = f[c];
              v = yb[e][c] + (h / 2.0) * f[c];
            } else if (st == 1) {
              *dym = f[c];
              v = yb[e][c] + (h / 2.0) * f[c];
            } else if (st == 2) {
              v = yb[e][c] + h * f[c];
              *dym = f[c] + *dym;
            } else {
              yb[e][c] = yb[e][c] + (h / 6.0) * ((*k1 + f[c]) + 2.0 * *dym);
              v = yb[e][c];
            }
            ys[c * g.yslen + k] = v;
          }
        } else {
          // Leapfrog X3 = X1 + 2 dt f(X2) (SBEs.py:5685-5687), kept in stage[c].
#pragma unroll
          for (int c = 0; c < 4; ++c) stage[c * nkp + k] = yb[e][c] + f[c] * h * 2.0;
        }
      }
      __syncthreads();
    }
    if (MODE == kRhs || MODE == kCalcH) break;
    if (MODE == kLeapfrog) {
      // Population neutrality and reshuffle (SBEs.py:5704-5718).
      double v[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int e = 0; e < EPT; ++e) {
        const int k = tid + e * kThreads;
        if (k < g.nk) {
          double a = fabs(stage[2 * nkp + k]), b = fabs(stage[3 * nkp + k]);
          stage[2 * nkp + k] = a;
          stage[3 * nkp + k] = b;
          v[0] += a;
          v[1] += b;
        }
      }
      block_sum(v, 2, scratch);
      const double total = (v[0] + v[1]) / 2.0;
      const double small = 1e-200;
#pragma unroll
      for (int e = 0; e < EPT; ++e) {
        const int k = tid + e * kThreads;
        if (k < g.nk) {
          stage[2 * nkp + k] = stage[2 * nkp + k] * total / (v[0] + small);
          stage[3 * nkp + k] = stage[3 * nkp + k] * total / (v[1] + small);
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const double x3 = stage[c * nkp + k];
            yb[e][c] = (yb[e][c] + x3) / 2.0;
            ys[c * g.yslen + k] = x3;
          }
        }
      }
      __syncthreads();
    }
    t = t + h;
    steps += 1;
    // P(t) record (qwoptics.py:815-946, diagonal: pscale * sum_k p_k).
    if (bt.P && bt.p_stride > 0 && (s + 1) % bt.p_stride == 0) {
      const int r = (s + 1) / bt.p_stride - 1;
      double v[2] = {0.0, 0.0};
#pragma unroll
      for (int e = 0; e < EPT; ++e) {
        const int k = tid + e * kThreads;
        if (k < g.nk) {
          v[0] += ys[k];
          v[1] += ys[g.yslen + k];
        }
      }
      block_sum(v, 2, scratch);
      if (tid == 0 && r < bt.p_cap && w.p_off >= 0 && w.p_off + r < bt.n_P) {
        bt.P[2 * (w.p_off + r)] = w.pscale * v[0];
        bt.P[2 * (w.p_off + r) + 1] = w.pscale * v[1];
      }
    }
  }
  if (MODE == kRhs || MODE == kCalcH) return;

  // Write the state back; flag non-finite wires.
  bool bad = false;
  double2* yo = reinterpret_cast<double2*>(bt.y + 4 * w.off);
  double2* y1o = MODE == kLeapfrog ? reinterpret_cast<double2*>(bt.y1 + 4 * w.off) : nullptr;
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int k = tid + e * kThreads;
    if (k < g.nk) {
      double a = ys[k], b = ys[g.yslen + k], c = ys[2 * g.yslen + k], d = ys[3 * g.yslen + k];
      if (MODE == kRk4) {
        a = yb[e][0];
        b = yb[e][1];
        c = yb[e][2];
        d = yb[e][3];
      }
      yo[2 * k] = make_double2(a, b);
      yo[2 * k + 1] = make_double2(c, d);
      bad |= !(isfinite(a) && isfinite(b) && isfinite(c) && isfinite(d));
      if (MODE == kLeapfrog) {
        y1o[2 * k] = make_double2(yb[e][0], yb[e][1]);
        y1o[2 * k + 1] = make_double2(yb[e][2], yb[e][3]);
        bad |= !(isfinite(yb[e][0]) && isfinite(yb[e][1]) && isfinite(yb[e][2]) &&
                 isfinite(yb[e][3]));
      }
    }
  }
  bad = __syncthreads_or(bad);
  if (tid == 0) {
    wp->t = t;
    wp->steps = steps;
    if (bad && wp->status == PSB_OK) wp->status = PSB_ERR_NONFINITE;
  }
}

constexpr int kR = 4;

size_t smem_bytes_for(int nk, int ntab) {
  Geo g = geometry<kR>(nk);
  return sizeof(double) * (size_t)smem_layout<kR>(g, ntab).total;
}

template <int MODE, bool SCREEN, int NT>
static int launch_ept(const Batch& bt, int ept, int grid, size_t smem, cudaStream_t st) {
  void (*kern)(Batch) = nullptr;
  switch (ept) {
    case 1: kern = sbe_f64_kernel<kR, 1, MODE, SCREEN, NT>; break;
    case 2: kern = sbe_f64_kernel<kR, 2, MODE, SCREEN, NT>; break;
    case 4: kern = sbe_f64_kernel<kR, 4, MODE, SCREEN, NT>; break;
    default: return set_error(PSB_ERR_SIZE, "unsupported elements per thread %d", ept);
  }
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess)
    return set_error(PSB_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
  kern<<<grid, kThreads, smem, st>>>(bt);
  return check_cuda("sbe_f64_kernel");
}

template <int MODE>
static int launch_mode(const Batch& bt, int ept, int grid, size_t smem, bool screened,
                       bool shared, cudaStream_t st) {
  if (screened)
    return shared ? launch_ept<MODE, true, 1>(bt, ept, grid, smem, st)
                  : launch_ept<MODE, true, 3>(bt, ept, grid, smem, st);
  return shared ? launch_ept<MODE, false, 1>(bt, ept, grid, smem, st)
                : launch_ept<MODE, false, 3>(bt, ept, grid, smem, st);
}

// Host-side launch: sizes shared memory for the largest grid of the launch.
int launch_sbe_f64(Batch bt, int mode, int n_order, int nkmax, int tab_flags, cudaStream_t st) {
  if (nkmax < 2 || nkmax > PSB_MAX_NK)
    return set_error(PSB_ERR_SIZE, "nk %d outside [2, %d]", nkmax, PSB_MAX_NK);
  const bool screened = (tab_flags & PSB_TAB_SCREENED) != 0;
  const bool shared = (tab_flags & PSB_TAB_SHARED_V) != 0;
  bt.nk_limit = nkmax;
  size_t smem = 0;
  for (int nk = 2; nk <= nkmax; ++nk) {
    size_t b = smem_bytes_for(nk, shared ? 1 : 3);
    if (b > smem) smem = b;
  }
  int ept = (nkmax + kThreads - 1) / kThreads;
  if (ept == 3) ept = 4;
  const int grid = bt.order ? n_order : bt.nw;
  if (grid <= 0) return PSB_OK;
  if (mode == kRhs) return launch_mode<kRhs>(bt, ept, grid, smem, screened, shared, st);
  if (mode == kCalcH) return launch_mode<kCalcH>(bt, ept, grid, smem, screened, shared, st);
  if (mode == kRk4) return launch_mode<kRk4>(bt, ept, grid, smem, screened, shared, st);
  return launch_mode<kLeapfrog>(bt, ept, grid, smem, screened, shared, st);
}

}  // namespace psb

using namespace psb;

extern "C" int psb_f64_smem_bytes(int nk, int tab_flags) {
  if (nk < 2 || nk > PSB_MAX_NK) return set_error(PSB_ERR_SIZE, "nk %d out of range", nk);
  return (int)smem_bytes_for(nk, (tab_flags & PSB_TAB_SHARED_V) ? 1 : 3);
}

static int common_checks(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                         const PsbWire* d_wires, int nw, const double* d_y,
                         const PsbModel* model, int nkmax) {
  if (!d_tables || !d_tabdata || !d_wires || !d_y || !model || ntab <= 0 || nw < 0)
    return set_error(PSB_ERR_INVALID, "null pointer or bad count");
  if (nkmax < 2 || nkmax > PSB_MAX_NK)
    return set_error(PSB_ERR_SIZE, "nkmax %d outside [2, %d]", nkmax, PSB_MAX_NK);
  if (!(model->hbar > 0.0)) return set_error(PSB_ERR_INVALID, "model.hbar must be > 0");
  return PSB_OK;
}

extern "C" int psb_rhs_f64(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                           int64_t n_tabdata, const PsbWire* d_wires, int nw, const double* d_y,
                           double* d_dy, int64_t n_state, int nkmax, int tab_flags,
                           const PsbModel* model, void* stream) {
  int rc = common_checks(d_tables, ntab, d_tabdata, d_wires, nw, d_y, model, nkmax);
  if (rc) return rc;
  if (!d_dy) return set_error(PSB_ERR_INVALID, "d_dy is null");
  Batch bt{};
  bt.tables = d_tables;
  bt.ntab = ntab;
  bt.tabdata = d_tabdata;
  bt.n_tabdata = n_tabdata;
  bt.wires = const_cast<PsbWire*>(d_wires);
  bt.nw = nw;
  bt.y = const_cast<double*>(d_y);
  bt.dy = d_dy;
  bt.n_state = n_state;
  bt.nsteps = 1;
  bt.hbar = model->hbar;
  return launch_sbe_f64(bt, kRhs, 0, nkmax, tab_flags, (cudaStream_t)stream);
}

extern "C" int psb_calch_f64(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                             int64_t n_tabdata, const PsbWire* d_wires, int nw, const double* d_y,
                             double* d_h, int64_t n_state, int nkmax, int tab_flags,
                             const PsbModel* model, void* stream) {
  int rc = common_checks(d_tables, ntab, d_tabdata, d_wires, nw, d_y, model, nkmax);
  if (rc) return rc;
  if (!d_h) return set_error(PSB_ERR_INVALID, "d_h is null");
  Batch bt{};
  bt.tables = d_tables;
  bt.ntab = ntab;
  bt.tabdata = d_tabdata;
  bt.n_tabdata = n_tabdata;
  bt.wires = const_cast<PsbWire*>(d_wires);
  bt.nw = nw;
  bt.y = const_cast<double*>(d_y);
  bt.dy = d_h;
  bt.n_state = n_state;
  bt.nsteps = 1;
  bt.hbar = model->hbar;
  return launch_sbe_f64(bt, kCalcH, 0, nkmax, tab_flags, (cudaStream_t)stream);
}

extern "C" int psb_rk4_f64(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                           int64_t n_tabdata, PsbWire* d_wires, int nw, const int32_t* d_order,
                           int n_order, double* d_y, int64_t n_state, int nkmax, int tab_flags,
                           int nsteps, double dt, double* d_P, int64_t n_P, int p_stride,
                           int p_cap, const PsbModel* model, void* stream) {
  int rc = common_checks(d_tables, ntab, d_tabdata, d_wires, nw, d_y, model, nkmax);
  if (rc) return rc;
  if (nsteps < 0 || (d_order && n_order < 0))
    return set_error(PSB_ERR_INVALID, "nsteps or n_order < 0");
  if (nsteps == 0) return PSB_OK;
  Batch bt{};
  bt.tables = d_tables;
  bt.ntab = ntab;
  bt.tabdata = d_tabdata;
  bt.n_tabdata = n_tabdata;
  bt.wires = d_wires;
  bt.nw = nw;
  bt.order = d_order;
  bt.y = d_y;
  bt.n_state = n_state;
  bt.nsteps = nsteps;
  bt.dt = dt;
  bt.P = d_P;
  bt.n_P = n_P;
  bt.p_stride = p_stride;
  bt.p_cap = p_cap;
  bt.hbar = model->hbar;
  return launch_sbe_f64(bt, kRk4, n_order, nkmax, tab_flags, (cudaStream_t)stream);
}

extern "C" int psb_leapfrog_f64(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                                int64_t n_tabdata, PsbWire* d_wires, int nw,
                                const int32_t* d_order, int n_order, double* d_y1, double* d_y2,
                                int64_t n_state, int nkmax, int tab_flags,
                                const double* d_field, int64_t field_stride, int64_t n_field,
                                int nsteps, double dt, double* d_P, int64_t n_P, int p_stride,
                                int p_cap, const PsbModel* model, void* stream) {
  int rc = common_checks(d_tables, ntab, d_tabdata, d_wires, nw, d_y2, model, nkmax);
  if (rc) return rc;
  if (!d_y1 || !d_field) return set_error(PSB_ERR_INVALID, "d_y1 or d_field is null");
  if (nsteps < 0 || (d_order && n_order < 0))
    return set_error(PSB_ERR_INVALID, "nsteps or n_order < 0");
  if (nsteps == 0) return PSB_OK;
  Batch bt{};
  bt.tables = d_tables;
  bt.ntab = ntab;
  bt.tabdata = d_tabdata;
  bt.n_tabdata = n_tabdata;
  bt.wires = d_wires;
  bt.nw = nw;
  bt.order = d_order;
  bt.y = d_y2;
  bt.y1 = d_y1;
  bt.n_state = n_state;
  bt.field = d_field;
  bt.field_stride = field_stride;
  bt.n_field = n_field;
  bt.nsteps = nsteps;
  bt.dt = dt;
  bt.P = d_P;
  bt.n_P = n_P;
  bt.p_stride = p_stride;
  bt.p_cap = p_cap;
  bt.hbar = model->hbar;
  return launch_sbe_f64(bt, kLeapfrog, n_order, nkmax, tab_flags, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Elementwise diagonal derivatives from given Hamiltonian diagonals (the
// diagonal of dpdt / dCdt / dDdt for diagonal states, SBEs.py:1958-1975,
// 2325-2337, 2623-2636), in the reference's association order:
//   i hbar dp = ((((Hhh p + Hee p) - Heh C) - Heh D) + Heh) - (i hbar g) p + Off
//   i hbar dC = i hbar dD = Heh conj(p) - conj(Heh) p
// (the Hee / Hhh commutators vanish on the diagonal).
// ---------------------------------------------------------------------------
namespace psb {
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
// x / (i hbar) = (x.im / hbar, -x.re / hbar)
__device__ __forceinline__ double2 div_ihbar(double2 x, double hb) {
  return make_double2(x.y / hb, -x.x / hb);
}

__global__ void diag_derivs_kernel(const double2* __restrict__ h, const double2* __restrict__ st,
                                   const double* __restrict__ g, const double2* __restrict__ off,
                                   double hb, double2* __restrict__ out, int64_t n) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double2 heh = h[3 * k], hee = h[3 * k + 1], hhh = h[3 * k + 2];
  const double2 p = st[3 * k], c = st[3 * k + 1], d = st[3 * k + 2];
  double2 acc = cadd(cmul(hhh, p), cmul(hee, p));
  acc = csub(acc, cmul(heh, c));
  acc = csub(acc, cmul(heh, d));
  acc = cadd(acc, heh);
  // (i hbar) g = (0, hbar g) as a complex scalar, times p
  acc = csub(acc, cmul(make_double2(0.0 * g[k], hb * g[k]), p));
  if (off) acc = cadd(acc, off[k]);
  out[3 * k] = div_ihbar(acc, hb);
  const double2 pc = make_double2(p.x, -p.y), hc = make_double2(heh.x, -heh.y);
  const double2 dn = div_ihbar(csub(cmul(heh, pc), cmul(hc, p)), hb);
  out[3 * k + 1] = dn;
  out[3 * k + 2] = dn;
}
}  // namespace psb

extern "C" int psb_diag_derivs_f64(const double* d_h, const double* d_state, const double* d_gam,
                                   const double* d_off, double hbar, double* d_out, int64_t n,
                                   void* stream) {
  if (!d_h || !d_state || !d_gam || !d_out || n < 0 || !(hbar > 0.0))
    return psb::set_error(PSB_ERR_INVALID, "psb_diag_derivs_f64: null pointer or bad size");
  if (n == 0) return PSB_OK;
  const int threads = 256;
  const int64_t blocks = (n + threads - 1) / threads;
  psb::diag_derivs_kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(
      reinterpret_cast<const double2*>(d_h), reinterpret_cast<const double2*>(d_state), d_gam,
      reinterpret_cast<const double2*>(d_off), hbar, reinterpret_cast<double2*>(d_out), n);
  return psb::check_cuda("diag_derivs_kernel");
}
