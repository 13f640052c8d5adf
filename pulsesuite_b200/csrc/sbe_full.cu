// sbe_full.cu -- the full-matrix (Nk x Nk) SBE step of one quantum wire in
// FP64, for drives that vary along the wire: the reference's general case.
//
// A wire's state is three complex matrices p[kh][ke] (YY), C[k1][k2] (CC)
// and D[k1][k2] (DD) per stored level (SBEs.py:4782-4790); with a field that
// is not uniform along the wire the coupling Meh and the Hamiltonians are
// full matrices and the right-hand side is O(Nk^3).  One call of
// psb_full_step_f64 is one step of the reference's integrator for one wire
// (SBESolver._sbe_calculator, SBEs.py:5624-5836) with the flags Optics,
// Excitons, LF and Screened:
//   Meh   = CalcMeh of the wire-space fields (SBEs.py:5165-5175)
//   H     = CalcH with the exchange (and, with LF, direct) Coulomb sums
//           along the diagonals of p, C, D (SBEs.py:819-935, lf branch)
//   dX    = dpdt, dCdt, dDdt (SBEs.py:1952-1975, 2318-2337, 2617-2636)
//   X3    = X1 + 2 dt dX, occupations |C3_kk|, |D3_kk| rescaled to a common
//           total, X2 = (X1 + X3) / 2 (SBEs.py:5681-5718)
// psb_full_step_mb_f64 adds the many-body terms mb.params switches on
// (DiagDph, OffDiagDph: k-dependent and off-diagonal dephasing in dpdt;
// EHs, Phonon: carrier-carrier and LO-phonon relaxation of the new
// occupations before the rescale; Recomb: spontaneous emission after that
// relaxation; DCTrans: the DC-field shift of X3 in k); see the mb_* kernels.
// psb_full_sources_f64 evaluates the wire-space source terms of the new
// level: the polarisation components of QWPolarization3 and the charge
// densities of QWRho5 before their transforms (qwoptics.py:56-84, 367-381).
// Every sum runs in the reference's order; results agree with it to
// rounding (numpy's pairwise sums and the kernels' sequential ones differ
// in the last bits).
#include <mutex>

#include "psb_common.cuh"

namespace psb {
namespace full {

__device__ __forceinline__ double2 cm(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 ca(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 cs(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 rs(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
// x / (i hbar)
__device__ __forceinline__ double2 div_ih(double2 x, double hb) {
  return make_double2(x.y / hb, -x.x / hb);
}

struct Step {
  int nk, nr, nq0;
  const double* kr;     // [nk] (unused by the step; kept for symmetry)
  const double* V3;     // [3][nk]: V_eh, V_ee, V_hh at index distance q
  const double* Ee;     // [nk]
  const double* Eh;     // [nk]
  const double2* E;     // [3][nr] wire-space fields Ex, Ey, Ez (q space)
  PsbFullParams prm;
  double2* L1;          // levels, [3][nk][nk] each: p, C, D
  double2* L2;
  double2* L3;
  double2* Meh;         // work [nk][nk]
  double2* H;           // work [3][nk][nk]: Heh, Hee, Hhh
  double2* dX;          // work [3][nk][nk]: dp, dC, dD
  // many-body terms (null when off): k-dependent dephasing rates, the
  // off-diagonal dephasing term of dpdt, and X3 written out so that the
  // relaxation can change its occupations before the neutrality rescale
  const double* GamE;   // [nk]
  const double* GamH;   // [nk]
  const double2* OffP;  // [nk][nk], OffP[kh][ke]
  const double2* X3;    // [3][nk][nk]
  // a batch of wires of one grid, wire = blockIdx.y: byte strides between
  // the wires' V3, fields, levels, work and many-body scratch, and the
  // per-wire [nw][4] = yw, (-1)^w, dc_dk, 0 (null: prm.yw, prm.sgnw)
  int64_t st_v3, st_e, st_lv, st_wk, st_sc;
  const double* wpar;
};

template <class T>
__device__ __forceinline__ T* bump(T* p, int64_t bytes) {
  return p ? reinterpret_cast<T*>(reinterpret_cast<uintptr_t>(p) + bytes) : p;
}

// the Step of wire blockIdx.y of a batch
__device__ __forceinline__ Step at_wire(Step s) {
  const int64_t w = blockIdx.y;
  s.V3 = bump(s.V3, w * s.st_v3);
  s.E = bump(s.E, w * s.st_e);
  s.L1 = bump(s.L1, w * s.st_lv);
  s.L2 = bump(s.L2, w * s.st_lv);
  s.L3 = bump(s.L3, w * s.st_lv);
  s.Meh = bump(s.Meh, w * s.st_wk);
  s.H = bump(s.H, w * s.st_wk);
  s.dX = bump(s.dX, w * s.st_wk);
  s.GamE = bump(s.GamE, w * s.st_sc);
  s.GamH = bump(s.GamH, w * s.st_sc);
  s.OffP = bump(s.OffP, w * s.st_sc);
  s.X3 = bump(s.X3, w * s.st_sc);
  if (s.wpar) {
    s.prm.yw = s.wpar[4 * w];
    s.prm.sgnw = s.wpar[4 * w + 1];
  }
  return s;
}

// Meh[ke][kh] = -ehint (Xcv Ex[q] + Ycv Ey[q] yw + Zcv Ez[q] (-1)^w),
// q = kkp[ke][kh] = ke - kh + NQ0, Xcv = dcv (-1)^(kh+1), Ycv = dcv,
// Zcv = -dcv (QWOptics dipoles, qwoptics.py:619-623).
__global__ void meh_kernel(Step s0) {
  const Step s = at_wire(s0);
  const int nk = s.nk;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nk * nk) return;
  const int ke = e / nk, kh = e - ke * nk;
  const int q = ke - kh + s.nq0;
  double2 ex = make_double2(0.0, 0.0), ey = ex, ez = ex;
  if (q >= 0 && q < s.nr) {
    ex = s.E[q];
    ey = s.E[s.nr + q];
    ez = s.E[2 * s.nr + q];
  }
  const double dcv = s.prm.dcv, eh = s.prm.ehint;
  const double xcv = ((kh + 1) & 1) ? -dcv : dcv;
  double2 m = rs(-eh * xcv, ex);
  m = cs(m, rs(s.prm.yw, rs(eh * dcv, ey)));
  m = cs(m, rs(s.prm.sgnw, rs(eh * -dcv, ez)));
  s.Meh[e] = m;
}

__device__ __forceinline__ double vq(const double* V, int n, int nk, int q) {
  const int a = q < 0 ? -q : q;
  return (a > 0 && a < nk) ? V[n * nk + a] : 0.0;
}

// CalcH (SBEs.py:819-935): every element (k1, k2) sums along its diagonal
// d = k1 - k2 of p, C, D (the exchange terms) and, with LF, along the
// diagonals d and -d of C and D (the direct terms), each in the reference's
// order.  One CTA per diagonal and wire: the five diagonals it reads are
// loaded once into shared memory (they are strided in the row-major
// matrices), then thread t sums for the element at position t.
constexpr int kHThreads = 128;
__global__ void __launch_bounds__(kHThreads) calch_kernel(Step s0) {
  const Step s = at_wire(s0);
  const int nk = s.nk, n2 = nk * nk;
  const int d = (int)blockIdx.x - (nk - 1);     // k1 - k2
  const int ad = d < 0 ? -d : d, len = nk - ad;  // elements on the diagonal
  const int o1 = d > 0 ? d : 0, o2 = d < 0 ? -d : 0;  // k1 = t + o1, k2 = t + o2
  extern __shared__ double2 hsm[];  // [5][len]: p, C, D at row - col = -d; C, D at +d
  double2* pd = hsm;
  double2* cd = pd + len;
  double2* dd = cd + len;
  double2* cm_ = dd + len;
  double2* dm = cm_ + len;
  const double2* p = s.L3;
  const double2* C = s.L3 + n2;
  const double2* D = s.L3 + 2 * n2;
  for (int u = threadIdx.x; u < len; u += kHThreads) {
    // element u of the run: row o2 + u, column o1 + u (col - row = d), and
    // the mirrored run row o1 + u, column o2 + u
    const int a = (o2 + u) * nk + (o1 + u), b = (o1 + u) * nk + (o2 + u);
    pd[u] = p[a];
    cd[u] = C[a];
    dd[u] = D[a];
    cm_[u] = C[b];
    dm[u] = D[b];
  }
  __syncthreads();
  const double* V = s.V3;
  for (int t = threadIdx.x; t < len; t += kHThreads) {
    const int k1 = t + o1, k2 = t + o2, e = k1 * nk + k2;
    double2 heh = s.Meh[e];
    double2 hee = make_double2(0.0, 0.0), hhh = hee;
    if (k1 == k2) {
      hee = make_double2(s.Ee[k1] + s.prm.gap, 0.0);
      hhh = make_double2(s.Eh[k1], 0.0);
    }
    if (s.prm.excitons) {
      // q runs over qmin .. qmax, i.e. positions u = t + q = 0 .. len - 1
      // H^eh: sum_q V_eh(q) p^T[k1+q][k2+q] = p[k2+q][k1+q]
      for (int u = 0; u < len; ++u)
        if (u != t) heh = ca(heh, rs(vq(V, 0, nk, u - t), pd[u]));
      if (s.prm.lf) {
        for (int u = 0; u < len; ++u)
          if (u != t) hee = cs(hee, rs(vq(V, 1, nk, u - t), cd[u]));
        if (d != 0) {
          // direct terms: k = kmin .. kmax, C[k][k + d] and D[k + d][k]
          const double v1 = vq(V, 1, nk, d), v0 = vq(V, 0, nk, d), v2 = vq(V, 2, nk, d);
          // with k = kmin + u: C[k][k + d] = cd[u], D[k + d][k] = dm[u],
          // D[k][k + d] = dd[u], C[k + d][k] = cm_[u]
          for (int u = 0; u < len; ++u) hee = ca(hee, cs(rs(v1, cd[u]), rs(v0, dm[u])));
          for (int u = 0; u < len; ++u)
            if (u != t) hhh = cs(hhh, rs(vq(V, 2, nk, u - t), dd[u]));
          for (int u = 0; u < len; ++u) hhh = ca(hhh, cs(rs(v2, dd[u]), rs(v0, cm_[u])));
        } else {
          for (int u = 0; u < len; ++u)
            if (u != t) hhh = cs(hhh, rs(vq(V, 2, nk, u - t), dd[u]));
        }
      } else if (k1 == k2) {
        for (int u = 0; u < len; ++u)
          if (u != t) hee = cs(hee, rs(vq(V, 1, nk, u - t), cd[u]));
        for (int u = 0; u < len; ++u)
          if (u != t) hhh = cs(hhh, rs(vq(V, 2, nk, u - t), dd[u]));
      }
    }
    s.H[e] = heh;
    s.H[n2 + e] = hee;
    s.H[2 * n2 + e] = hhh;
  }
}

// dpdt / dCdt / dDdt (SBEs.py:1952-1975, 2318-2337, 2617-2636): one thread
// per (i, j), the four dot products of each in the reference's order (each
// accumulator runs over k = 0 .. nk-1 in sequence).  One CTA computes a
// kDT x kDT block of elements: per chunk of kDT values of k, the 18 operand
// tiles the block's 12 dot products read are staged in shared memory
// (rows padded by one element against bank conflicts).
constexpr int kDT = 16, kDTP = kDT + 1;
enum DTile {  // tile [row block][col block]; I, J the element block, K the k chunk
  T_HHH_IK, T_HHH_JK, T_HHH_KI, T_HEE_JK, T_HEE_KI, T_HEH_KI, T_HEH_JK, T_HEH_IK, T_HEH_KJ,
  T_P_KJ, T_P_IK, T_P_KI, T_P_JK, T_C_KJ, T_C_IK, T_D_KI, T_D_IK, T_D_KJ, T_NUM
};
constexpr size_t kDerivsSmem = (size_t)T_NUM * kDT * kDTP * sizeof(double2);

__global__ void __launch_bounds__(kDT* kDT) derivs_kernel(Step s0) {
  const Step s = at_wire(s0);
  const int nk = s.nk, n2 = nk * nk;
  extern __shared__ double2 dsm[];
  const int tx = threadIdx.x % kDT, ty = threadIdx.x / kDT;
  const int I0 = blockIdx.x * kDT, J0 = blockIdx.z * kDT;
  const int i = I0 + ty, j = J0 + tx;
  const double2* p = s.L3;
  const double2* C = s.L3 + n2;
  const double2* D = s.L3 + 2 * n2;
  const double2* Heh = s.H;
  const double2* Hee = s.H + n2;
  const double2* Hhh = s.H + 2 * n2;
  const double2 z = make_double2(0.0, 0.0);
  auto tile = [&](int t, int r, int c) -> double2& { return dsm[(t * kDT + r) * kDTP + c]; };
  // tile t of matrix M: rows from block R0 (or the k chunk), columns likewise
  auto load = [&](int t, const double2* M, int R0, int C0) {
    const int r = R0 + ty, c = C0 + tx;
    tile(t, ty, tx) = (r < nk && c < nk) ? M[r * nk + c] : z;
  };
  double2 a1 = z, a2 = z, a3 = z, a4 = z;  // dp
  double2 b1 = z, b2 = z, b3 = z, b4 = z;  // dC
  double2 c1 = z, c2 = z, c3 = z, c4 = z;  // dD
  for (int k0 = 0; k0 < nk; k0 += kDT) {
    load(T_HHH_IK, Hhh, I0, k0);
    load(T_HHH_JK, Hhh, J0, k0);
    load(T_HHH_KI, Hhh, k0, I0);
    load(T_HEE_JK, Hee, J0, k0);
    load(T_HEE_KI, Hee, k0, I0);
    load(T_HEH_KI, Heh, k0, I0);
    load(T_HEH_JK, Heh, J0, k0);
    load(T_HEH_IK, Heh, I0, k0);
    load(T_HEH_KJ, Heh, k0, J0);
    load(T_P_KJ, p, k0, J0);
    load(T_P_IK, p, I0, k0);
    load(T_P_KI, p, k0, I0);
    load(T_P_JK, p, J0, k0);
    load(T_C_KJ, C, k0, J0);
    load(T_C_IK, C, I0, k0);
    load(T_D_KI, D, k0, I0);
    load(T_D_IK, D, I0, k0);
    load(T_D_KJ, D, k0, J0);
    __syncthreads();
    const int kn = min(kDT, nk - k0);
    for (int kk = 0; kk < kn; ++kk) {
      // dp[kh = i][ke = j]
      a1 = ca(a1, cm(tile(T_HHH_IK, ty, kk), tile(T_P_KJ, kk, tx)));
      a2 = ca(a2, cm(tile(T_HEE_JK, tx, kk), tile(T_P_IK, ty, kk)));
      a3 = ca(a3, cm(tile(T_HEH_KI, kk, ty), tile(T_C_KJ, kk, tx)));
      a4 = ca(a4, cm(tile(T_HEH_JK, tx, kk), tile(T_D_KI, kk, ty)));
      // dC[k1 = i][k2 = j]
      b1 = ca(b1, cm(tile(T_HEE_JK, tx, kk), tile(T_C_IK, ty, kk)));
      b2 = ca(b2, cm(tile(T_HEE_KI, kk, ty), tile(T_C_KJ, kk, tx)));
      b3 = ca(b3, cm(tile(T_HEH_JK, tx, kk), cconj(tile(T_P_KI, kk, ty))));
      b4 = ca(b4, cm(cconj(tile(T_HEH_IK, ty, kk)), tile(T_P_KJ, kk, tx)));
      // dD[k1 = i][k2 = j]
      c1 = ca(c1, cm(tile(T_HHH_JK, tx, kk), tile(T_D_IK, ty, kk)));
      c2 = ca(c2, cm(tile(T_HHH_KI, kk, ty), tile(T_D_KJ, kk, tx)));
      c3 = ca(c3, cm(tile(T_HEH_KJ, kk, tx), cconj(tile(T_P_IK, ty, kk))));
      c4 = ca(c4, cm(cconj(tile(T_HEH_KI, kk, ty)), tile(T_P_JK, tx, kk)));
    }
    __syncthreads();
  }
  if (i >= nk || j >= nk) return;
  const int e = i * nk + j;
  const double hb = s.prm.hbar;
  {
    double2 r = cs(cs(ca(a1, a2), a3), a4);
    r = ca(r, Heh[j * nk + i]);
    // GamE[ke] + GamH[kh]: the constant rates, or CalcGammaE/H's
    const double g = s.GamE ? s.GamE[j] + s.GamH[i] : s.prm.gam_e + s.prm.gam_h;
    r = cs(r, cm(make_double2(0.0 * g, hb * g), p[i * nk + j]));
    if (s.OffP) r = ca(r, s.OffP[e]);  // + OffP[kh][ke]
    s.dX[e] = div_ih(r, hb);
  }
  s.dX[n2 + e] = div_ih(cs(ca(cs(b1, b2), b3), b4), hb);
  s.dX[2 * n2 + e] = div_ih(cs(ca(cs(c1, c2), c3), c4), hb);
}

// Leapfrog with neutrality and reshuffle (SBEs.py:5681-5718), one CTA.
constexpr int kLfThreads = 256;
__global__ void __launch_bounds__(kLfThreads) leapfrog_kernel(Step s0) {
  const Step s = at_wire(s0);
  const int nk = s.nk, n2 = nk * nk;
  const double dt = s.prm.dt, small = 1e-200;
  __shared__ double red_e[kLfThreads], red_h[kLfThreads];
  __shared__ double fac[3];
  auto x3_of = [&](int e) -> double2 {
    if (s.X3) return s.X3[e];  // relaxed occupations (many-body terms)
    return ca(s.L2[e], rs(2.0, rs(dt, s.dX[e])));  // X1 + dX dt 2
  };
  double se = 0.0, sh = 0.0;
  for (int k = threadIdx.x; k < nk; k += kLfThreads) {
    const double2 c3 = x3_of(n2 + k * nk + k), d3 = x3_of(2 * n2 + k * nk + k);
    se += hypot(c3.x, c3.y);
    sh += hypot(d3.x, d3.y);
  }
  red_e[threadIdx.x] = se;
  red_h[threadIdx.x] = sh;
  __syncthreads();
  for (int o = kLfThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red_e[threadIdx.x] += red_e[threadIdx.x + o];
      red_h[threadIdx.x] += red_h[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double total = (red_e[0] + red_h[0]) / 2.0;
    fac[0] = total;
    fac[1] = red_e[0] + small;
    fac[2] = red_h[0] + small;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 3 * n2; e += kLfThreads) {
    const double2 x1 = s.L2[e];
    double2 x3 = x3_of(e);
    const int m = e / n2, r = e - m * n2;
    if (m > 0 && r / nk == r % nk)  // occupation: |X3_kk| total / sum
      x3 = make_double2(hypot(x3.x, x3.y) * fac[0] / fac[m], 0.0);
    s.L1[e] = x1;
    s.L3[e] = x3;
    s.L2[e] = make_double2((x1.x + x3.x) / 2.0, (x1.y + x3.y) / 2.0);
  }
}

// Wire-space sources of one level: the QWPolarization3 sums (before the
// 2 ehint / (area L) factor and the transform) and the QWRho5 sums (before
// the boundary offset, normalisation and transform),
//   Px(r) = W(r) sum_{kh,ke} Re(conj(Xcv[ke][kh]) p[kh][ke] E[ke] conj(E[kh])),
//   Py, Pz likewise with dcv yw, -dcv (-1)^w,
//   Re(r) = W(r)/(2L) sum_{k1,k2} C[k1][k2] conj(E[k1]) E[k2],
//   Rh(r) = W(r)/(2L) sum_{k1,k2} conj(D[k1][k2]) conj(E[k1]) E[k2],
// E[k] = exp(i kr[k] r) (qwoptics.py:56-84, 367-381).  One CTA per
// kSrcR positions and wire (blockIdx.y of a batch: levels [nw][3][nk][nk],
// out [nw][5][nr], yw and (-1)^w from wpar[4 w], wpar[4 w + 1] when set):
// the phases of its positions in shared memory, threads over the column
// (ke, k2) so the rows of p, C, D are read coalesced, each element once for
// all kSrcR positions, then a block reduction.  The sums run in this tree
// order, not the reference's sequential one (they agree to rounding).
constexpr int kSrcThreads = 128, kSrcR = 4;
__global__ void __launch_bounds__(kSrcThreads) sources_kernel(
    int nk, int nr, const double* kr, const double* rpos, const double* window, double L,
    double dcv, double yw, double sgnw, const double* wpar, const double2* lev, double2* out) {
  extern __shared__ double2 ph[];  // [kSrcR][nk]
  __shared__ double red[kSrcR][6][kSrcThreads / 32];
  const int n2 = nk * nk, r0 = blockIdx.x * kSrcR;
  const int64_t w = blockIdx.y;
  lev += w * 3 * n2;
  out += w * 5 * nr;
  if (wpar) {
    yw = wpar[4 * w];
    sgnw = wpar[4 * w + 1];
  }
  for (int e = threadIdx.x; e < kSrcR * nk; e += kSrcThreads) {
    const int j = e / nk, k = e - j * nk;
    const int r = min(r0 + j, nr - 1);
    double sn, cn;
    sincos(kr[k] * rpos[r], &sn, &cn);
    ph[e] = make_double2(cn, sn);
  }
  __syncthreads();
  const double2* p = lev;
  const double2* C = lev + n2;
  const double2* D = lev + 2 * n2;
  double sx[kSrcR], sp[kSrcR];
  double2 se[kSrcR], sh[kSrcR];
#pragma unroll
  for (int j = 0; j < kSrcR; ++j) {
    sx[j] = sp[j] = 0.0;
    se[j] = sh[j] = make_double2(0.0, 0.0);
  }
  for (int c = threadIdx.x; c < nk; c += kSrcThreads) {
    double2 ec[kSrcR];
#pragma unroll
    for (int j = 0; j < kSrcR; ++j) ec[j] = ph[j * nk + c];
    for (int i = 0; i < nk; ++i) {
      const double2 pv = p[i * nk + c], cv = C[i * nk + c], dv = cconj(D[i * nk + c]);
      const double xs = ((i + 1) & 1) ? -1.0 : 1.0;  // conj(Xcv) / dcv at kh = i
#pragma unroll
      for (int j = 0; j < kSrcR; ++j) {
        const double2 ei = cconj(ph[j * nk + i]);
        const double t = cm(cm(pv, ec[j]), ei).x;
        sx[j] += xs * t;
        sp[j] += t;
        se[j] = ca(se[j], cm(cm(cv, ei), ec[j]));
        sh[j] = ca(sh[j], cm(cm(dv, ei), ec[j]));
      }
    }
  }
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < kSrcR; ++j) {
    const double v[6] = {sx[j], sp[j], se[j].x, se[j].y, sh[j].x, sh[j].y};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const double u = warp_sum(v[q]);
      if (lane == 0) red[j][q][wp] = u;
    }
  }
  __syncthreads();
  if (threadIdx.x < kSrcR) {
    const int j = threadIdx.x, r = r0 + j;
    if (r < nr) {
      double t[6];
      for (int q = 0; q < 6; ++q) {
        t[q] = 0.0;
        for (int u = 0; u < kSrcThreads / 32; ++u) t[q] += red[j][q][u];
      }
      const double W = window[r], h = W / (2.0 * L);
      out[r] = make_double2(W * dcv * t[0], 0.0);
      out[nr + r] = make_double2(W * yw * dcv * t[1], 0.0);
      out[2 * nr + r] = make_double2(W * sgnw * -dcv * t[1], 0.0);
      out[3 * nr + r] = make_double2(h * t[2], h * t[3]);
      out[4 * nr + r] = make_double2(h * t[4], h * t[5]);
    }
  }
}

// ---------------------------------------------------------------------------
// Many-body terms switched on by mb.params (PsbFullMB).  Each kernel keeps
// the reference's loop order for every accumulated value.
// ---------------------------------------------------------------------------
struct MBView {
  int nk;
  const double* V3;    // screened [3][nk] (VC[q, 0, n])
  const double* Ee;
  const double* Eh;
  const double2* L;    // the level the right-hand side reads (p2, C2, D2)
  double hbar;
  PsbFullMB mb;
  double* GamE;
  double* GamH;
  double* De;          // [(2 nk + 1)][nk]
  double* Dh;
  double2* OffP;
  double2* X3;         // [3][nk][nk]
  double* rates;       // [5][nk]: WinE, WoutE, WinH, WoutH, Rsp
  double2* shift;      // [nk]: circulant kernel of the DC shift
  double2* tr;         // [3][nk][nk]: DC-shift intermediate
  double gap;          // J
  int lf;
  // a batch of wires (blockIdx.y): byte strides of V3, the levels, the
  // scratch and eps between wires; wpar[4 w + 2] = dc_dk of wire w
  int64_t st_v3, st_lv, st_sc, st_eps;
  const double* wpar;
};

// the MBView of wire blockIdx.y of a batch
__device__ __forceinline__ MBView at_wire(MBView v) {
  const int64_t w = blockIdx.y;
  v.V3 = bump(v.V3, w * v.st_v3);
  v.L = bump(v.L, w * v.st_lv);
  const int64_t b = w * v.st_sc;
  v.GamE = bump(v.GamE, b);
  v.GamH = bump(v.GamH, b);
  v.De = bump(v.De, b);
  v.Dh = bump(v.Dh, b);
  v.OffP = bump(v.OffP, b);
  v.X3 = bump(v.X3, b);
  v.rates = bump(v.rates, b);
  v.shift = bump(v.shift, b);
  v.tr = bump(v.tr, b);
  v.mb.eps = bump(v.mb.eps, w * v.st_eps);
  if (v.wpar) v.mb.dc_dk = v.wpar[4 * w + 2];
  return v;
}

// CalcGammaE / CalcGammaH (dephasing.py:28-105): ne, nh the real parts of
// the diagonal of C2, D2; Vxx2[q] = V(iq[q])^2; one thread per k.
__global__ void mb_gamma_kernel(MBView v0) {
  const MBView v = at_wire(v0);
  const int nk = v.nk, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nk) return;
  const int n2 = nk * nk;
  const int32_t* kpq = v.mb.maps;
  const int32_t* kmq = kpq + n2;
  const int32_t* k1p = kpq + 2 * n2;
  const int32_t* k1pmq = kpq + 3 * n2;
  const int32_t* k1 = kpq + 4 * n2;
  const int32_t* k1mq = kpq + 5 * n2;
  const double2* C = v.L + n2;
  const double2* D = v.L + 2 * n2;
  auto ne = [&](int i) { return C[i * nk + i].x; };
  auto nh = [&](int i) { return D[i * nk + i].x; };
  auto in = [&](int i) { return i >= 0 && i < nk; };
  const double ph = kPi / v.hbar;
  double ge = 0.0, gh = 0.0;
  // electron-electron, then electron-hole scattering of electrons
  for (int q = 0; q < nk; ++q) {
    const int a = kpq[k * nk + q];
    if (in(a)) {
      const double vv = v.V3[nk + v.mb.iq[q]];
      ge = ge + ph * (vv * vv) * ne(a) * (1.0 - ne(a)) * fabs(v.mb.xe[q]);
    }
  }
  for (int q = 0; q < nk; ++q) {
    const int a = k1pmq[k * nk + q], b = k1p[k * nk + q], c = kmq[k * nk + q];
    if (in(a) && in(b) && in(c)) {
      const double vv = v.V3[v.mb.iq[q]];
      ge = ge + ph * (vv * vv) *
                    (nh(a) * (1.0 - nh(b)) * ne(c) + (1.0 - nh(a)) * nh(b) * (1.0 - ne(c))) *
                    fabs(v.mb.xh[q]);
    }
  }
  // hole-hole, then electron-hole scattering of holes
  for (int q = 0; q < nk; ++q) {
    const int a = kpq[k * nk + q];
    if (in(a)) {
      const double vv = v.V3[2 * nk + v.mb.iq[q]];
      gh = gh + ph * (vv * vv) * nh(a) * (1.0 - nh(a)) * fabs(v.mb.xh[q]);
    }
  }
  for (int q = 0; q < nk; ++q) {
    const int a = k1mq[k * nk + q], b = k1[k * nk + q], c = kmq[k * nk + q];
    if (in(a) && in(b) && in(c)) {
      const double vv = v.V3[v.mb.iq[q]];
      gh = gh + ph * (vv * vv) *
                    (ne(a) * (1.0 - ne(b)) * nh(c) + (1.0 - ne(a)) * ne(b) * (1.0 - nh(c))) *
                    fabs(v.mb.xe[q]);
    }
  }
  v.GamE[k] = ge;
  v.GamH[k] = gh;
}

__device__ __forceinline__ double lrtz(double a, double b) { return (b / kPi) / (a * a + b * b); }

// CalcOffDiagDeph_E2 / _H2 (dephasing.py:226-318): De[q + nk][k] and
// Dh[q + nk][k] for q in [-nk, nk], with |C_kk|, |D_kk| as occupations and
// Vsq(q) = V(|q|)^2 for 0 < |q| < nk; one thread per (q, k), the partner
// momentum p in the reference's order, then the factor pi / hbar.  The
// occupations and band energies are staged in shared memory per CTA.
__global__ void mb_offd_kernel(MBView v0) {
  const MBView v = at_wire(v0);
  const int nk = v.nk, n2 = nk * nk;
  extern __shared__ double osm[];  // [4][nk]: |C_kk|, |D_kk|, Ee, Eh
  for (int i = threadIdx.x; i < nk; i += blockDim.x) {
    const double2 c = v.L[n2 + i * nk + i], d = v.L[2 * n2 + i * nk + i];
    osm[i] = hypot(c.x, c.y);
    osm[nk + i] = hypot(d.x, d.y);
    osm[2 * nk + i] = v.Ee[i];
    osm[3 * nk + i] = v.Eh[i];
  }
  __syncthreads();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (2 * nk + 1) * nk) return;
  const int qi = e / nk, k = e - qi * nk, q = qi - nk;
  const double* Ee = osm + 2 * nk;
  const double* Eh = osm + 3 * nk;
  auto ne = [&](int i) { return osm[i]; };
  auto nh = [&](int i) { return osm[nk + i]; };
  const int aq = q < 0 ? -q : q;
  auto vsq = [&](int t) {
    const double x = (aq > 0 && aq < nk) ? v.V3[t * nk + aq] : 0.0;
    return x * x;
  };
  const double hb = v.hbar;
  const double b_ee = hb * v.mb.gam_eh, b_eh = hb * v.mb.gam_h;  // De: gee = g[0], geh = g[2]
  const double b_hh = hb * v.mb.gam_e;                            // Dh: ghh = g[1], geh = g[2]
  double de = 0.0, dh = 0.0;
  const int kq = k + q;
  const bool kin = kq >= 0 && kq < nk;
  // same-band scattering: q in [max(p - nk, -k), min(p - 1, nk - k - 1)]
  for (int p = 0; p < nk && kin; ++p) {
    const int pm = p - q;
    if (q < max(p - nk, -k) || q > min(p - 1, nk - k - 1) || pm < 0 || pm >= nk) continue;
    const double Ed = ((Ee[kq] + Ee[pm]) - Ee[p]) - Ee[k];
    de = de + vsq(1) * lrtz(Ed, b_ee) *
                  (ne(pm) * (1.0 - ne(p)) * (1.0 - ne(k)) + (1.0 - ne(pm)) * ne(p) * ne(k));
  }
  // electron-hole scattering: q in [max(-p, -k), min(nk - p - 1, nk - k - 1)]
  for (int p = 0; p < nk && kin; ++p) {
    const int pp = p + q;
    if (q < max(-p, -k) || q > min(nk - p - 1, nk - k - 1) || pp < 0 || pp >= nk) continue;
    const double Ed = ((Ee[kq] + Eh[pp]) - Eh[p]) - Ee[k];
    de = de + vsq(0) * lrtz(Ed, b_eh) *
                  (nh(pp) * (1.0 - nh(p)) * (1.0 - ne(k)) + (1.0 - nh(pp)) * nh(p) * ne(k));
  }
  for (int p = 0; p < nk && kin; ++p) {
    const int pm = p - q;
    if (q < max(p - nk, -k) || q > min(p - 1, nk - k - 1) || pm < 0 || pm >= nk) continue;
    const double Ed = ((Eh[kq] + Eh[pm]) - Eh[p]) - Eh[k];
    dh = dh + vsq(2) * lrtz(Ed, b_hh) *
                  (nh(pm) * (1.0 - nh(p)) * (1.0 - nh(k)) + (1.0 - nh(pm)) * nh(p) * nh(k));
  }
  for (int p = 0; p < nk && kin; ++p) {
    const int pp = p + q;
    if (q < max(-p, -k) || q > min(nk - p - 1, nk - k - 1) || pp < 0 || pp >= nk) continue;
    const double Ed = ((Eh[kq] + Ee[pp]) - Ee[p]) - Eh[k];
    dh = dh + vsq(0) * lrtz(Ed, b_eh) *
                  (ne(pp) * (1.0 - ne(p)) * (1.0 - nh(k)) + (1.0 - ne(pp)) * ne(p) * nh(k));
  }
  v.De[e] = de * kPi / hb;
  v.Dh[e] = dh * kPi / hb;
}

// OffDiagDephasing2 (dephasing.py:320-359): x[kh][ke] = i hbar (sum_q
// Dh[q][kh] p[kh + q][ke] + sum_q De[q][ke] p[kh][ke + q]), q != 0; one
// thread per (kh, ke).
__global__ void mb_offp_kernel(MBView v0) {
  const MBView v = at_wire(v0);
  const int nk = v.nk, e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nk * nk) return;
  const int kh = e / nk, ke = e - kh * nk;
  const double2* p = v.L;
  double2 x = make_double2(0.0, 0.0);
  for (int q = -kh; q <= nk - kh - 1; ++q) {
    const double u = q == 0 ? 0.0 : 1.0;  // undel
    const double d = v.Dh[(q + nk) * nk + kh];
    const double2 pv = p[(kh + q) * nk + ke];
    x = ca(x, make_double2(d * pv.x * u, d * pv.y * u));
  }
  for (int q = -ke; q <= nk - ke - 1; ++q) {
    const double u = q == 0 ? 0.0 : 1.0;
    const double d = v.De[(q + nk) * nk + ke];
    const double2 pv = p[kh * nk + ke + q];  // p^T[ke + q][kh]
    x = ca(x, make_double2(d * pv.x * u, d * pv.y * u));
  }
  // x * i * hbar
  v.OffP[e] = make_double2(-x.y * v.hbar, x.x * v.hbar);
}

// X3 = X1 + 2 dt dX, written out for the relaxation (SBEs.py:5685-5687).
__global__ void mb_x3_kernel(Step s0, MBView v0) {
  const Step s = at_wire(s0);
  double2* X3 = at_wire(v0).X3;
  const int n3 = 3 * s.nk * s.nk, e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n3) return;
  X3[e] = ca(s.L2[e], rs(2.0, rs(s.prm.dt, s.dX[e])));
}

// In/out scattering rates of the new occupations (SBESolver._relaxation_E/H,
// SBEs.py:5248-5291): MBCE / MBCH (coulomb.py:957-1071) with |Re n| on the
// 1-based grid, k3(a, b, c) = a + b - c (1-based, 0 when outside), and the
// reference's C arrays read at [k - 1][..][..]; then MBPE / MBPH
// (phonons.py:140-271) with Re n; with recomb also SpontEmission's Rsp.
// One CTA per (k, wire): the occupations and V^2 in shared memory, threads
// over the inner index of each double sum (so C[k][q1][q2] is read along
// q2), block reductions.  The sums run in this tree order, not the
// reference's sequential one (they agree to rounding).
constexpr int kRateThreads = 128;

// sum of K values over the CTA (kRateThreads threads); every thread gets them
template <int K>
__device__ __forceinline__ void rate_block_sum(double (&v)[K], double (*red)[kRateThreads / 32]) {
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < K; ++q) {
    const double u = warp_sum(v[q]);
    if (lane == 0) red[q][wp] = u;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < K; ++q) {
    double t = 0.0;
    for (int u = 0; u < kRateThreads / 32; ++u) t += red[q][u];
    v[q] = t;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kRateThreads) mb_rates_kernel(MBView v0) {
  const MBView v = at_wire(v0);
  const int nk = v.nk, k0 = blockIdx.x;
  const int n2 = nk * nk, N1 = nk + 1;
  extern __shared__ double sm[];
  double* ne1 = sm;             // [nk + 1] |Re n_e|, 1-based, [0] = 0
  double* nh1 = ne1 + N1;       // [nk + 1]
  double* v2 = nh1 + N1;        // [3][nk] V(q)^2
  __shared__ double red[5][kRateThreads / 32];
  const double2* C3 = v.X3 + n2;
  const double2* D3 = v.X3 + 2 * n2;
  for (int i = threadIdx.x; i <= nk; i += kRateThreads) {
    ne1[i] = i == 0 ? 0.0 : fabs(C3[(i - 1) * nk + i - 1].x);
    nh1[i] = i == 0 ? 0.0 : fabs(D3[(i - 1) * nk + i - 1].x);
  }
  for (int i = threadIdx.x; i < 3 * nk; i += kRateThreads) {
    const double x = v.V3[i];
    v2[i] = x * x;
  }
  __syncthreads();
  auto k3 = [&](int a, int b, int c) {  // 0-based arguments, 1-based result
    const int r = (a + 1) + (b + 1) - (c + 1);
    return (r < 1 || r > nk) ? 0 : r;
  };
  auto vv2 = [&](int t, int a, int b) { return v2[t * nk + (a > b ? a - b : b - a)]; };
  const size_t cs3 = (size_t)N1 * N1 * N1;
  const double* Ceh = v.mb.C;
  const double* Cee = Ceh + cs3;
  const double* Chh = Ceh + 2 * cs3;
  auto cix = [&](int a, int b, int c) { return ((size_t)a * N1 + b) * N1 + c; };
  double acc[4] = {0.0, 0.0, 0.0, 0.0};  // WinE, WoutE, WinH, WoutH
  if (v.mb.ehs) {
    const int k = k0 + 1;  // MBCE: k; MBCH: kp
    // two q1 per iteration keep twice the C reads in flight (each
    // accumulator still adds in q1 order)
#pragma unroll 2
    for (int q1 = 1; q1 <= nk; ++q1) {
      for (int q2 = threadIdx.x + 1; q2 <= nk; q2 += kRateThreads) {
        {  // electrons (MBCE)
          const int kp = q1, k1 = q2;
          int r = k3(kp - 1, k1 - 1, k - 1);
          if (r > 0)
            acc[0] += vv2(0, k - 1, k1 - 1) * (1.0 - nh1[kp]) * nh1[r] * ne1[k1] *
                      Ceh[cix(k - 1, kp - 1, k1 - 1)];
          r = k3(kp - 1, k - 1, k1 - 1);
          if (r > 0)
            acc[1] += vv2(0, k1 - 1, k - 1) * (1.0 - ne1[k1]) * (1.0 - nh1[kp]) * nh1[r] *
                      Ceh[cix(k1 - 1, kp - 1, k - 1)];
          const int k2 = q1, k4 = q2;
          r = k3(k - 1, k2 - 1, k4 - 1);
          if (r > 0)
            acc[0] += vv2(1, k - 1, k4 - 1) * (1.0 - ne1[k2]) * ne1[r] * ne1[k4] *
                      Cee[cix(k - 1, k2 - 1, k4 - 1)];
          r = k3(k4 - 1, k2 - 1, k - 1);
          if (r > 0)
            acc[1] += vv2(1, k4 - 1, k - 1) * (1.0 - ne1[k4]) * (1.0 - ne1[k2]) * ne1[r] *
                      Cee[cix(k4 - 1, k2 - 1, k - 1)];
        }
        {  // holes (MBCH): kp is this CTA's momentum
          const int kp = k, kk = q1, k1 = q2;
          int r = k3(kp - 1, k1 - 1, kk - 1);
          if (r > 0)
            acc[2] += vv2(0, kk - 1, k1 - 1) * (1.0 - ne1[kk]) * nh1[r] * ne1[k1] *
                      Ceh[cix(kk - 1, kp - 1, k1 - 1)];
          r = k3(kp - 1, kk - 1, k1 - 1);
          if (r > 0)
            acc[3] += vv2(0, k1 - 1, kk - 1) * (1.0 - ne1[kk]) * (1.0 - nh1[r]) * ne1[k1] *
                      Ceh[cix(kk - 1, r - 1, k1 - 1)];
          const int k2p = q1, k4p = q2;
          r = k3(kp - 1, k2p - 1, k4p - 1);
          if (r > 0)
            acc[2] += vv2(2, kp - 1, k4p - 1) * (1.0 - nh1[k2p]) * nh1[r] * nh1[k4p] *
                      Chh[cix(kp - 1, k2p - 1, k4p - 1)];
          r = k3(k4p - 1, k2p - 1, kp - 1);
          if (r > 0)
            acc[3] += vv2(2, k4p - 1, kp - 1) * (1.0 - nh1[k4p]) * (1.0 - nh1[k2p]) * nh1[r] *
                      Chh[cix(k4p - 1, k2p - 1, kp - 1)];
        }
      }
    }
  }
  rate_block_sum<4>(acc, red);
  if (v.mb.phonon) {
    // Vep[k][i] = VC_ee[k][i] / E1D[k][i] * Vscale (VC already screened)
    const double* EP = v.mb.ph;
    const double* EPT = EP + n2;
    const double* HP = EP + 2 * n2;
    const double* HPT = EP + 3 * n2;
    double ph[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < nk; i += kRateThreads) {
      const int d = i > k0 ? i - k0 : k0 - i;
      const double e = v.mb.eps ? v.mb.eps[d] : 1.0;
      const double vep = v.V3[nk + d] / e * v.mb.vscale;
      const double vhp = v.V3[2 * nk + d] / e * v.mb.vscale;
      const double nei = C3[i * nk + i].x, nhi = D3[i * nk + i].x;
      ph[0] += vep * nei * EPT[i * nk + k0];
      ph[1] += vep * (1.0 - nei) * EP[i * nk + k0];
      ph[2] += vhp * nhi * HPT[i * nk + k0];
      ph[3] += vhp * (1.0 - nhi) * HP[i * nk + k0];
    }
    rate_block_sum<4>(ph, red);
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = acc[q] + ph[q];
  }
  double rsp = 0.0;
  if (v.mb.recomb) {
    // SpontEmission (emission.py:94-131) from the level the right-hand side
    // reads (SBEs.py:5237-5238): Ec (emission.py:133-172) with Re n and the
    // screened V, Ek = gap + Ee + Eh + Ec, then SpontIntegral
    // (emission.py:174-199): sum_n x rho0(x) square_n dhw, x = HOmega_n + Ek,
    // rho0(x) = x^2 / (c0^3 pi^2 hbar^3)
    const double2* C2 = v.L + n2;
    const double2* D2 = v.L + 2 * n2;
    const double veh0 = v.V3[0], vee0 = v.V3[nk], vhh0 = v.V3[2 * nk];
    double ec[2] = {0.0, 0.0};
    for (int i = threadIdx.x; i < nk; i += kRateThreads) {
      const int d = i > k0 ? i - k0 : k0 - i;
      const double ne = C2[i * nk + i].x, nh = D2[i * nk + i].x;
      ec[0] += ne * (vee0 - v.V3[nk + d]) + nh * (vhh0 - v.V3[2 * nk + d]);
      const double id = i == k0 ? 0.0 : 1.0;
      ec[1] += ne * veh0 * id - nh * veh0 * id;
    }
    rate_block_sum<2>(ec, red);
    const double ek = ((v.gap + v.Ee[k0]) + v.Eh[k0]) + ((ec[0] + ec[1]) - veh0);
    const double* hw = v.mb.emis;
    const double* sq = hw + v.mb.n_hw;
    double it[1] = {0.0};
    for (int n = threadIdx.x; n < v.mb.n_hw; n += kRateThreads) {
      const double x = hw[n] + ek;
      it[0] += x * (x * x / v.mb.rho0_den) * sq[n];
    }
    rate_block_sum<1>(it, red);
    rsp = it[0] * v.mb.dhw;
  }
  if (threadIdx.x == 0) {
    v.rates[k0] = acc[0];
    v.rates[nk + k0] = acc[1];
    v.rates[2 * nk + k0] = acc[2];
    v.rates[3 * nk + k0] = acc[3];
    if (v.mb.recomb) v.rates[4 * nk + k0] = rsp;
  }
}

// n <- exp(-W dt) ((-1 + exp(W dt) + n) Win + n Wout) / (W + small), W = Win
// + Wout, on the diagonal of C3 and D3 (SBEs.py:5322-5331).
__global__ void mb_relax_kernel(MBView v0, double dt) {
  const MBView v = at_wire(v0);
  const int nk = v.nk, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nk) return;
  const int n2 = nk * nk;
  const double small = 1e-200;
  for (int b = 0; b < 2; ++b) {
    const double win = v.rates[2 * b * nk + k], wout = v.rates[(2 * b + 1) * nk + k];
    const double W = win + wout;
    double2* c = v.X3 + (1 + b) * n2 + k * nk + k;
    const double2 n = *c;
    const double em = exp(-W * dt), ep = exp(W * dt);
    const double2 s1 = make_double2((-1.0 + ep) + n.x, n.y);
    const double2 s = make_double2(s1.x * win + n.x * wout, s1.y * win + n.y * wout);
    const double den = W + small;
    *c = make_double2(em * s.x / den, em * s.y / den);
  }
  if (v.mb.recomb) {
    // n_e *= exp(-Rsp n_h dt), then n_h *= exp(-Rsp n_e dt) with the new
    // n_e (SBEs.py:5335-5337), complex as the reference's ne3, nh3
    const double r = v.rates[4 * nk + k];
    double2* ce = v.X3 + n2 + k * nk + k;
    double2* ch = v.X3 + 2 * n2 + k * nk + k;
    auto cexp_ = [](double x, double y) {
      const double m = exp(x);
      return make_double2(m * cos(y), m * sin(y));
    };
    const double2 nh = *ch;
    const double2 ne = cm(*ce, cexp_(-r * nh.x * dt, -r * nh.y * dt));
    *ce = ne;
    *ch = cm(nh, cexp_(-r * ne.x * dt, -r * ne.y * dt));
  }
}

// DC transport (Transport, dcfield.py:1213-1247): ShiftN1D / ShiftN2D move
// a vector or matrix in k by fft -> times exp(-i Y dk) -> ifft
// (dcfield.py:1169-1211), i.e. a circular convolution with
//   s[d] = (1/nk) sum_m exp(-i Y_m dk) exp(2 pi i m d / nk),
// applied along both indices of each matrix (lf) or to its diagonal.
__global__ void mb_shift_kernel(MBView v0) {
  const MBView v = at_wire(v0);
  const int nk = v.nk, d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= nk) return;
  double re = 0.0, im = 0.0;
  for (int m = 0; m < nk; ++m) {
    double sy, cy, sw, cw;
    sincos(-v.mb.Y[m] * v.mb.dc_dk, &sy, &cy);
    const int r = (int)(((long long)m * d) % nk);
    sincospi(2.0 * r / nk, &sw, &cw);
    re += cy * cw - sy * sw;
    im += cy * sw + sy * cw;
  }
  v.shift[d] = make_double2(re / nk, im / nk);
}

// The two circulant products of the shift, tiled: one CTA per kST x kST
// block of one matrix (x) of one wire; per chunk of kST summation indices
// the block's operand tile and the 2 kST - 1 coefficients s[(j - b) mod nk]
// it needs sit in shared memory.  Each element sums in the old order (the
// summation index ascending).
constexpr int kST = 16;

// T[x][a][j] = sum_b X3[x][a][b] s[(j - b) mod nk]
__global__ void __launch_bounds__(kST* kST) mb_shift_rows_kernel(MBView v0) {
  const MBView v = at_wire(v0);
  const int nk = v.nk, n2 = nk * nk, nb = (nk + kST - 1) / kST;
  const int x = blockIdx.x / (nb * nb), t = blockIdx.x % (nb * nb);
  const int A0 = (t / nb) * kST, J0 = (t % nb) * kST;
  const int tx = threadIdx.x % kST, ty = threadIdx.x / kST;
  __shared__ double2 xt[kST][kST + 1];
  __shared__ double2 sv[2 * kST - 1];
  const double2* X = v.X3 + (size_t)x * n2;
  const int a = A0 + ty, j = J0 + tx;
  double2 acc = make_double2(0.0, 0.0);
  for (int b0 = 0; b0 < nk; b0 += kST) {
    const int r = A0 + ty, c = b0 + tx;
    xt[ty][tx] = (r < nk && c < nk) ? X[r * nk + c] : make_double2(0.0, 0.0);
    if (threadIdx.x < 2 * kST - 1) {
      // sv[u] = s[(J0 - b0 - (kST - 1) + u) mod nk]
      int d = (J0 - b0 - (kST - 1) + (int)threadIdx.x) % nk;
      if (d < 0) d += nk;
      sv[threadIdx.x] = v.shift[d];
    }
    __syncthreads();
    const int bn = min(kST, nk - b0);
    for (int bb = 0; bb < bn; ++bb) acc = ca(acc, cm(xt[ty][bb], sv[tx - bb + kST - 1]));
    __syncthreads();
  }
  if (a < nk && j < nk) v.tr[(size_t)x * n2 + a * nk + j] = acc;
}

// X3[x][i][j] = sum_a s[(i - a) mod nk] T[x][a][j]
__global__ void __launch_bounds__(kST* kST) mb_shift_cols_kernel(MBView v0) {
  const MBView v = at_wire(v0);
  const int nk = v.nk, n2 = nk * nk, nb = (nk + kST - 1) / kST;
  const int x = blockIdx.x / (nb * nb), t = blockIdx.x % (nb * nb);
  const int I0 = (t / nb) * kST, J0 = (t % nb) * kST;
  const int tx = threadIdx.x % kST, ty = threadIdx.x / kST;
  __shared__ double2 tt[kST][kST + 1];
  __shared__ double2 sv[2 * kST - 1];
  const double2* T = v.tr + (size_t)x * n2;
  const int i = I0 + ty, j = J0 + tx;
  double2 acc = make_double2(0.0, 0.0);
  for (int a0 = 0; a0 < nk; a0 += kST) {
    const int r = a0 + ty, c = J0 + tx;
    tt[ty][tx] = (r < nk && c < nk) ? T[r * nk + c] : make_double2(0.0, 0.0);
    if (threadIdx.x < 2 * kST - 1) {
      // sv[u] = s[(I0 - a0 - (kST - 1) + u) mod nk]
      int d = (I0 - a0 - (kST - 1) + (int)threadIdx.x) % nk;
      if (d < 0) d += nk;
      sv[threadIdx.x] = v.shift[d];
    }
    __syncthreads();
    const int an = min(kST, nk - a0);
    for (int aa = 0; aa < an; ++aa) acc = ca(acc, cm(sv[ty - aa + kST - 1], tt[aa][tx]));
    __syncthreads();
  }
  if (i < nk && j < nk) v.X3[(size_t)x * n2 + i * nk + j] = acc;
}

// without lf only the diagonals move: T[x][a] = sum_n s[(a - n) mod nk] X3[x][n][n]
__global__ void mb_shift_diag_kernel(MBView v0) {
  const MBView v = at_wire(v0);
  const int nk = v.nk, n2 = nk * nk, e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3 * nk) return;
  const int x = e / nk, a = e % nk;
  const double2* X = v.X3 + (size_t)x * n2;
  double2 acc = make_double2(0.0, 0.0);
  for (int n = 0; n < nk; ++n) {
    const int d = a - n < 0 ? a - n + nk : a - n;
    acc = ca(acc, cm(v.shift[d], X[n * nk + n]));
  }
  v.tr[e] = acc;
}

__global__ void mb_shift_diag_store_kernel(MBView v0) {
  const MBView v = at_wire(v0);
  const int nk = v.nk, e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3 * nk) return;
  const int x = e / nk, a = e % nk;
  v.X3[(size_t)x * nk * nk + a * nk + a] = v.tr[e];
}

// CalcMBArrays (coulomb.py:367-499) on the (nk+1)^3 grid the reference
// allocates (index 0 unused); UnDel(i, j) = 0 on row/column 0 and the
// diagonal, else 1 (coulomb.py:336-366).  One thread per entry.
__global__ void mb_tables_kernel(int nk, const double* Ee, const double* Eh, double ge,
                                 double gh, double hb, int lorentz, double* Ceh) {
  const int N1 = nk + 1;
  const size_t n3 = (size_t)N1 * N1 * N1;
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n3) return;
  double* Cee = Ceh + n3;
  double* Chh = Ceh + 2 * n3;
  const int a = (int)(e / ((size_t)N1 * N1)), bb = (int)((e / N1) % N1), c = (int)(e % N1);
  Ceh[e] = Cee[e] = Chh[e] = 0.0;
  if (a == 0 || bb == 0 || c == 0) return;
  const int k1 = a - 1, k2 = bb - 1, k4 = c - 1;
  auto undel = [&](int i, int j) { return (i == 0 || j == 0 || i == j) ? 0.0 : 1.0; };
  auto gdelta = [&](double x, double w) {
    if (fabs(w) < 1e-300) return 0.0;
    return 1.0 / (sqrt(kPi) * w) * exp(-((x / w) * (x / w)));
  };
  const double geh = (ge + gh) / 2.0;
  const double twopi = 2.0 * kPi;
  // Veh(k1, k2, k30, k4), k30 = k3[k4, k2, k1]
  int r = (k4 + 1) + (k2 + 1) - (k1 + 1);
  if (r >= 1 && r <= nk) {
    const int k30 = r - 1;
    const double Ed = Ee[k1] + Eh[k2] - Eh[k30] - Ee[k4];
    if (lorentz) {
      const double h2 = (hb * geh) * (hb * geh);
      Ceh[e] = 2.0 * geh * undel(a, c) * undel(bb, r) / (Ed * Ed + h2);
    } else {
      Ceh[e] = twopi / hb * undel(a, c) * undel(bb, r) * gdelta(Ed, hb * geh);
    }
  }
  // Vee / Vhh(k1, k2, k30, k4), k30 = k3[k1, k2, k4]
  r = (k1 + 1) + (k2 + 1) - (k4 + 1);
  if (r >= 1 && r <= nk) {
    const int k30 = r - 1;
    const double Ede = Ee[k1] + Ee[k2] - Ee[k30] - Ee[k4];
    const double Edh = Eh[k1] + Eh[k2] - Eh[k30] - Eh[k4];
    if (lorentz) {
      Cee[e] = 2.0 * ge * undel(a, c) * undel(bb, r) / (Ede * Ede + (hb * ge) * (hb * ge));
      Chh[e] = 2.0 * gh * undel(a, c) * undel(bb, r) / (Edh * Edh + (hb * gh) * (hb * gh));
    } else {
      Cee[e] = twopi / hb * undel(a, c) * undel(bb, r) * gdelta(Ede, hb * ge);
      Chh[e] = twopi / hb * undel(a, c) * undel(bb, r) * gdelta(Edh, hb * gh);
    }
  }
}

// Screening of a batch (CalcScreenedArrays, coulomb.py:1195-1230), one CTA
// per wire: n1D from the diagonals of the level the right-hand side reads,
// eps(q; n1D) of the grid's table block and V3 = V0 / eps.  The n1D sum
// has psb_screen_f64's thread mapping and tree, so a wire's V3 is the same
// bits as the one-wire path's.
constexpr int kScrThreads = 256;
__global__ void __launch_bounds__(kScrThreads) screen_batch_kernel(Step s0, const double* tab,
                                                                   double L, double dens_max,
                                                                   double* eps, double* V3) {
  const Step s = at_wire(s0);
  const int nk = s.nk, n2 = nk * nk;
  const int64_t w = blockIdx.y;
  eps = bump(eps, w * s.st_v3);
  V3 = bump(V3, w * s.st_v3);
  const double2* C = s.L3 + n2;
  const double2* D = s.L3 + 2 * n2;
  double t = 0.0;
  for (int k = threadIdx.x; k < nk; k += kScrThreads) t += C[k * nk + k].x + D[k * nk + k].x;
  __shared__ double red[kScrThreads / 32];
  __shared__ double n1d_s;
  t = warp_sum(t);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double u = 0.0;
    for (int i = 0; i < kScrThreads / 32; ++i) u += red[i];
    const double n1d = u / 2.0 / L;
    n1d_s = n1d < dens_max ? n1d : dens_max;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nk; q += kScrThreads) {
    const double e = eps1d(tab, nk, q, n1d_s);
    eps[q] = e;
    V3[q] = tab[q] / e;
    V3[nk + q] = tab[nk + q] / e;
    V3[2 * nk + q] = tab[2 * nk + q] / e;
  }
}

}  // namespace full
}  // namespace psb

using namespace psb;

extern "C" int64_t psb_full_work_bytes(int nk) {
  if (nk < 2 || nk > PSB_MAX_NK) return set_error(PSB_ERR_SIZE, "nk %d out of range", nk);
  return (int64_t)7 * nk * nk * 16;
}

namespace {
// scratch of the many-body terms: GamE, GamH, De, Dh, OffP, X3, rates
// (+ Rsp), the DC-shift kernel and intermediate
struct MBScratch {
  size_t gam, de, dh, offp, x3, rates, shift, tr, total;
  explicit MBScratch(int nk) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t n = (size_t)nk, n2 = n * n, nd = (2 * n + 1) * n;
    gam = 0;
    de = al(gam + 2 * n * 8);
    dh = al(de + nd * 8);
    offp = al(dh + nd * 8);
    x3 = al(offp + n2 * 16);
    rates = al(x3 + 3 * n2 * 16);
    shift = al(rates + 5 * n * 8);
    tr = al(shift + n * 16);
    total = al(tr + 3 * n2 * 16);
  }
};
}  // namespace

extern "C" int64_t psb_full_mb_scratch_bytes(int nk) {
  if (nk < 2 || nk > PSB_MAX_NK) return set_error(PSB_ERR_SIZE, "nk %d out of range", nk);
  return (int64_t)MBScratch(nk).total;
}

extern "C" int psb_mb_tables_f64(int nk, const double* d_Ee, const double* d_Eh, double ge,
                                 double gh, double hbar, int lorentz, double* d_C,
                                 void* stream) {
  if (!d_Ee || !d_Eh || !d_C) return set_error(PSB_ERR_INVALID, "psb_mb_tables_f64: null pointer");
  if (nk < 2 || nk > PSB_MAX_NK) return set_error(PSB_ERR_SIZE, "psb_mb_tables_f64: nk %d", nk);
  if (!(hbar > 0.0)) return set_error(PSB_ERR_INVALID, "hbar must be > 0");
  const size_t n3 = (size_t)(nk + 1) * (nk + 1) * (nk + 1);
  const int th = 256;
  const unsigned bl = (unsigned)((n3 + th - 1) / th);
  full::mb_tables_kernel<<<bl, th, 0, (cudaStream_t)stream>>>(nk, d_Ee, d_Eh, ge, gh, hbar,
                                                               lorentz ? 1 : 0, d_C);
  return check_cuda("psb_mb_tables_f64");
}

namespace {
// per-wire work of a batch: Meh, H, dX, then the screened V3 and eps
struct BatchWork {
  size_t v3, eps, total;
  explicit BatchWork(int nk) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    v3 = al((size_t)7 * nk * nk * 16);
    eps = al(v3 + 3 * (size_t)nk * 8);
    total = al(eps + (size_t)nk * 8);
  }
};

// one full-matrix step of nw wires of one grid (nw = 1: the one-wire entry)
struct Launch {
  int nw, nk, nr, nq0;
  const double* V3;
  int64_t st_v3;         // bytes between wires' V3 (0: shared)
  const double* Ee;
  const double* Eh;
  const double* fields;  // [nw][3][nr] complex
  const PsbFullParams* params;
  const double* wpar;    // [nw][4] or null
  const PsbFullMB* mb;
  double* L1;
  double* L2;
  double* L3;
  void* work;
  int64_t st_wk;         // bytes between wires' work
  const double* tab;     // screened batch: the grid's table block, else null
  double L, dens_max;
};

int check_mb(const PsbFullMB* mb, bool deph, bool relax, bool dct) {
  if (!(deph || relax || dct)) return PSB_OK;
  if (!mb->scratch) return set_error(PSB_ERR_INVALID, "PsbFullMB.scratch is null");
  if (mb->diag_dph && (!mb->maps || !mb->iq || !mb->xe || !mb->xh))
    return set_error(PSB_ERR_INVALID, "PsbFullMB: dephasing tables missing");
  if ((mb->ehs && !mb->C) || (mb->phonon && !mb->ph))
    return set_error(PSB_ERR_INVALID, "PsbFullMB: relaxation tables missing");
  if (relax && mb->recomb && (!mb->emis || mb->n_hw < 2 || !(mb->rho0_den > 0.0)))
    return set_error(PSB_ERR_INVALID, "PsbFullMB: emission tables missing");
  if (dct && !mb->Y) return set_error(PSB_ERR_INVALID, "PsbFullMB: DC wavenumbers missing");
  return PSB_OK;
}

int full_launch(const Launch& a, cudaStream_t st) {
  const int nk = a.nk, nw = a.nw, n2 = nk * nk;
  const PsbFullMB* mb = a.mb;
  const bool deph = mb && (mb->diag_dph || mb->offdiag_dph);
  const bool relax = mb && (mb->ehs || mb->phonon);
  const bool dct = mb && mb->dctrans;
  const int rc = check_mb(mb, deph, relax, dct);
  if (rc != PSB_OK) return rc;
  full::Step s{};
  s.nk = nk;
  s.nr = a.nr;
  s.nq0 = a.nq0;
  s.V3 = a.V3;
  s.Ee = a.Ee;
  s.Eh = a.Eh;
  s.E = reinterpret_cast<const double2*>(a.fields);
  s.prm = *a.params;
  s.L1 = reinterpret_cast<double2*>(a.L1);
  s.L2 = reinterpret_cast<double2*>(a.L2);
  s.L3 = reinterpret_cast<double2*>(a.L3);
  double2* w = reinterpret_cast<double2*>(a.work);
  s.Meh = w;
  s.H = w + n2;
  s.dX = w + 4 * n2;
  s.st_v3 = a.st_v3;
  s.st_e = (int64_t)3 * a.nr * 16;
  s.st_lv = (int64_t)3 * n2 * 16;
  s.st_wk = a.st_wk;
  s.st_sc = (int64_t)MBScratch(nk).total;
  s.wpar = a.wpar;
  const dim3 one(1, nw);
  const double* eps = mb ? mb->eps : nullptr;
  int64_t st_eps = 0;
  if (a.tab) {
    // each wire's V3 and eps from its own densities, into its work
    const BatchWork bw(nk);
    double* v3w = reinterpret_cast<double*>(reinterpret_cast<uint8_t*>(a.work) + bw.v3);
    double* epsw = reinterpret_cast<double*>(reinterpret_cast<uint8_t*>(a.work) + bw.eps);
    s.V3 = v3w;
    s.st_v3 = a.st_wk;
    full::screen_batch_kernel<<<one, full::kScrThreads, 0, st>>>(s, a.tab, a.L, a.dens_max,
                                                                  epsw, v3w);
    eps = epsw;
    st_eps = a.st_wk;
  }
  full::MBView v{};
  if (deph || relax || dct) {
    const MBScratch L(nk);
    uint8_t* sc = reinterpret_cast<uint8_t*>(mb->scratch);
    v.nk = nk;
    v.V3 = s.V3;
    v.Ee = a.Ee;
    v.Eh = a.Eh;
    v.L = s.L3;
    v.hbar = a.params->hbar;
    v.mb = *mb;
    v.mb.eps = eps;
    v.GamE = reinterpret_cast<double*>(sc + L.gam);
    v.GamH = v.GamE + nk;
    v.De = reinterpret_cast<double*>(sc + L.de);
    v.Dh = reinterpret_cast<double*>(sc + L.dh);
    v.OffP = reinterpret_cast<double2*>(sc + L.offp);
    v.X3 = reinterpret_cast<double2*>(sc + L.x3);
    v.rates = reinterpret_cast<double*>(sc + L.rates);
    v.shift = reinterpret_cast<double2*>(sc + L.shift);
    v.tr = reinterpret_cast<double2*>(sc + L.tr);
    v.gap = a.params->gap;
    v.lf = a.params->lf;
    v.st_v3 = s.st_v3;
    v.st_lv = s.st_lv;
    v.st_sc = s.st_sc;
    v.st_eps = st_eps;
    v.wpar = a.wpar;
  }
  const int th = 128;
  const dim3 bl((n2 + th - 1) / th, nw), blk((nk + th - 1) / th, nw);
  full::meh_kernel<<<bl, th, 0, st>>>(s);
  {
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
      attr = cudaFuncSetAttribute(full::calch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  5 * PSB_MAX_NK * 16);
    });
    if (attr != cudaSuccess) return set_error(PSB_ERR_CUDA, "calch_kernel: shared memory");
    full::calch_kernel<<<dim3(2 * nk - 1, nw), full::kHThreads, 5 * (size_t)nk * 16, st>>>(s);
  }
  // dephasing from the level the right-hand side reads (SBEs.py:5225-5232)
  if (mb && mb->diag_dph) {
    full::mb_gamma_kernel<<<blk, th, 0, st>>>(v);
    s.GamE = v.GamE;
    s.GamH = v.GamH;
  }
  if (mb && mb->offdiag_dph) {
    const int nd = (2 * nk + 1) * nk;
    full::mb_offd_kernel<<<dim3((nd + th - 1) / th, nw), th, 4 * (size_t)nk * 8, st>>>(v);
    full::mb_offp_kernel<<<bl, th, 0, st>>>(v);
    s.OffP = v.OffP;
  }
  {
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
      attr = cudaFuncSetAttribute(full::derivs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)full::kDerivsSmem);
    });
    if (attr != cudaSuccess) return set_error(PSB_ERR_CUDA, "derivs_kernel: shared memory");
    const int nb = (nk + full::kDT - 1) / full::kDT;
    full::derivs_kernel<<<dim3(nb, nw, nb), full::kDT * full::kDT, full::kDerivsSmem, st>>>(s);
  }
  if (relax || dct) {
    // X3, its occupations relaxed (SBEs.py:5688-5695) and shifted by the DC
    // field (SBEs.py:5698-5702), then the rescale
    const dim3 b3((3 * n2 + th - 1) / th, nw);
    full::mb_x3_kernel<<<b3, th, 0, st>>>(s, v);
    if (relax) {
      const size_t smr = (2 * (size_t)(nk + 1) + 3 * (size_t)nk) * 8;
      full::mb_rates_kernel<<<dim3(nk, nw), full::kRateThreads, smr, st>>>(v);
      full::mb_relax_kernel<<<blk, th, 0, st>>>(v, a.params->dt);
    }
    if (dct) {
      full::mb_shift_kernel<<<blk, th, 0, st>>>(v);
      if (a.params->lf) {
        const int nb = (nk + full::kST - 1) / full::kST;
        const dim3 bt(3 * nb * nb, nw);
        full::mb_shift_rows_kernel<<<bt, full::kST * full::kST, 0, st>>>(v);
        full::mb_shift_cols_kernel<<<bt, full::kST * full::kST, 0, st>>>(v);
      } else {
        const dim3 bd((3 * nk + th - 1) / th, nw);
        full::mb_shift_diag_kernel<<<bd, th, 0, st>>>(v);
        full::mb_shift_diag_store_kernel<<<bd, th, 0, st>>>(v);
      }
    }
    s.X3 = v.X3;
  }
  full::leapfrog_kernel<<<one, full::kLfThreads, 0, st>>>(s);
  return PSB_OK;
}
}  // namespace

extern "C" int psb_full_step_mb_f64(int nk, int nr, int nq0, const double* d_V3,
                                    const double* d_Ee, const double* d_Eh,
                                    const double* d_fields, const PsbFullParams* params,
                                    const PsbFullMB* mb, double* d_L1, double* d_L2,
                                    double* d_L3, void* d_work, int64_t n_work_bytes,
                                    void* stream) {
  if (!d_V3 || !d_Ee || !d_Eh || !d_fields || !params || !d_L1 || !d_L2 || !d_L3 || !d_work)
    return set_error(PSB_ERR_INVALID, "psb_full_step_f64: null pointer");
  if (nk < 2 || nk > PSB_MAX_NK || nr < 1 || nq0 < 0 || nq0 >= nr)
    return set_error(PSB_ERR_SIZE, "psb_full_step_f64: nk %d / nr %d / nq0 %d out of range", nk,
                     nr, nq0);
  if (n_work_bytes < psb_full_work_bytes(nk))
    return set_error(PSB_ERR_SIZE, "psb_full_step_f64: work needs psb_full_work_bytes(nk)");
  if (!(params->hbar > 0.0)) return set_error(PSB_ERR_INVALID, "hbar must be > 0");
  Launch a{};
  a.nw = 1;
  a.nk = nk;
  a.nr = nr;
  a.nq0 = nq0;
  a.V3 = d_V3;
  a.Ee = d_Ee;
  a.Eh = d_Eh;
  a.fields = d_fields;
  a.params = params;
  a.mb = mb;
  a.L1 = d_L1;
  a.L2 = d_L2;
  a.L3 = d_L3;
  a.work = d_work;
  const int rc = full_launch(a, (cudaStream_t)stream);
  if (rc != PSB_OK) return rc;
  return check_cuda("psb_full_step_f64");
}

extern "C" int psb_full_step_f64(int nk, int nr, int nq0, const double* d_V3, const double* d_Ee,
                                 const double* d_Eh, const double* d_fields,
                                 const PsbFullParams* params, double* d_L1, double* d_L2,
                                 double* d_L3, void* d_work, int64_t n_work_bytes,
                                 void* stream) {
  return psb_full_step_mb_f64(nk, nr, nq0, d_V3, d_Ee, d_Eh, d_fields, params, nullptr, d_L1,
                              d_L2, d_L3, d_work, n_work_bytes, stream);
}

extern "C" int64_t psb_full_batch_work_bytes(int nw, int nk) {
  if (nk < 2 || nk > PSB_MAX_NK) return set_error(PSB_ERR_SIZE, "nk %d out of range", nk);
  if (nw < 1 || nw > PSB_FULL_MAX_WIRES) return set_error(PSB_ERR_SIZE, "nw %d out of range", nw);
  return (int64_t)nw * (int64_t)BatchWork(nk).total;
}

extern "C" int psb_full_step_batch_f64(int nw, int nk, int nr, int nq0, const double* d_tab,
                                       double L, double dens_max, int screened,
                                       const double* d_fields, const PsbFullParams* params,
                                       const double* d_wpar, const PsbFullMB* mb, double* d_L1,
                                       double* d_L2, double* d_L3, void* d_work,
                                       int64_t n_work_bytes, void* stream) {
  if (!d_tab || !d_fields || !params || !d_wpar || !d_L1 || !d_L2 || !d_L3 || !d_work)
    return set_error(PSB_ERR_INVALID, "psb_full_step_batch_f64: null pointer");
  if (nk < 2 || nk > PSB_MAX_NK || nr < 1 || nq0 < 0 || nq0 >= nr || nw < 1 ||
      nw > PSB_FULL_MAX_WIRES)
    return set_error(PSB_ERR_SIZE, "psb_full_step_batch_f64: nw %d / nk %d / nr %d / nq0 %d", nw,
                     nk, nr, nq0);
  if (n_work_bytes < psb_full_batch_work_bytes(nw, nk))
    return set_error(PSB_ERR_SIZE, "psb_full_step_batch_f64: work needs "
                                   "psb_full_batch_work_bytes(nw, nk)");
  if (!(params->hbar > 0.0)) return set_error(PSB_ERR_INVALID, "hbar must be > 0");
  if (screened && !(L > 0.0)) return set_error(PSB_ERR_INVALID, "screening needs L > 0");
  Launch a{};
  a.nw = nw;
  a.nk = nk;
  a.nr = nr;
  a.nq0 = nq0;
  a.V3 = d_tab;  // V_eh, V_ee, V_hh rows of the table block, shared when unscreened
  a.Ee = d_tab + 3 * (size_t)nk;
  a.Eh = d_tab + 4 * (size_t)nk;
  a.fields = d_fields;
  a.params = params;
  a.wpar = d_wpar;
  a.mb = mb;
  a.L1 = d_L1;
  a.L2 = d_L2;
  a.L3 = d_L3;
  a.work = d_work;
  a.st_wk = (int64_t)BatchWork(nk).total;
  if (screened) {
    a.tab = d_tab;
    a.L = L;
    a.dens_max = dens_max;
  }
  const int rc = full_launch(a, (cudaStream_t)stream);
  if (rc != PSB_OK) return rc;
  return check_cuda("psb_full_step_batch_f64");
}

namespace {
// dynamic shared memory of sources_kernel (the phases of its positions),
// with the opt-in above 48 KB set on first use; 0 if that fails
size_t sources_smem(int nk) {
  const size_t sm = (size_t)full::kSrcR * nk * 16;
  static std::once_flag once;
  static bool ok = true;
  if (sm > 48 * 1024)
    std::call_once(once, [] {
      ok = cudaFuncSetAttribute(full::sources_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                full::kSrcR * PSB_MAX_NK * 16) == cudaSuccess;
    });
  return ok ? sm : 0;
}
}  // namespace

extern "C" int psb_full_sources_f64(int nk, int nr, const double* d_kr, const double* d_r,
                                    const double* d_window, double L, double dcv, double yw,
                                    double sgnw, const double* d_level, double* d_out,
                                    void* stream) {
  if (!d_kr || !d_r || !d_window || !d_level || !d_out)
    return set_error(PSB_ERR_INVALID, "psb_full_sources_f64: null pointer");
  if (nk < 2 || nk > PSB_MAX_NK || nr < 1)
    return set_error(PSB_ERR_SIZE, "psb_full_sources_f64: nk %d / nr %d out of range", nk, nr);
  const size_t sm = sources_smem(nk);
  if (!sm) return set_error(PSB_ERR_CUDA, "psb_full_sources_f64: shared memory");
  full::sources_kernel<<<(nr + full::kSrcR - 1) / full::kSrcR, full::kSrcThreads, sm,
                         (cudaStream_t)stream>>>(
      nk, nr, d_kr, d_r, d_window, L, dcv, yw, sgnw, nullptr,
      reinterpret_cast<const double2*>(d_level), reinterpret_cast<double2*>(d_out));
  return check_cuda("psb_full_sources_f64");
}

extern "C" int psb_full_sources_batch_f64(int nw, int nk, int nr, const double* d_kr,
                                          const double* d_r, const double* d_window, double L,
                                          double dcv, const double* d_wpar,
                                          const double* d_levels, double* d_out, void* stream) {
  if (!d_kr || !d_r || !d_window || !d_wpar || !d_levels || !d_out)
    return set_error(PSB_ERR_INVALID, "psb_full_sources_batch_f64: null pointer");
  if (nk < 2 || nk > PSB_MAX_NK || nr < 1 || nw < 1 || nw > PSB_FULL_MAX_WIRES)
    return set_error(PSB_ERR_SIZE, "psb_full_sources_batch_f64: nw %d / nk %d / nr %d", nw, nk,
                     nr);
  const size_t sm = sources_smem(nk);
  if (!sm) return set_error(PSB_ERR_CUDA, "psb_full_sources_batch_f64: shared memory");
  const dim3 bl((nr + full::kSrcR - 1) / full::kSrcR, nw);
  full::sources_kernel<<<bl, full::kSrcThreads, sm, (cudaStream_t)stream>>>(
      nk, nr, d_kr, d_r, d_window, L, dcv, 0.0, 0.0, d_wpar,
      reinterpret_cast<const double2*>(d_levels), reinterpret_cast<double2*>(d_out));
  return check_cuda("psb_full_sources_batch_f64");
}
