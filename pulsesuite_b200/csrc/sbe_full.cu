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
// psb_full_sources_f64 evaluates the wire-space source terms of the new
// level: the polarisation components of QWPolarization3 and the charge
// densities of QWRho5 before their transforms (qwoptics.py:56-84, 367-381).
// Every sum runs in the reference's order; results agree with it to
// rounding (numpy's pairwise sums and the kernels' sequential ones differ
// in the last bits).
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
};

// Meh[ke][kh] = -ehint (Xcv Ex[q] + Ycv Ey[q] yw + Zcv Ez[q] (-1)^w),
// q = kkp[ke][kh] = ke - kh + NQ0, Xcv = dcv (-1)^(kh+1), Ycv = dcv,
// Zcv = -dcv (QWOptics dipoles, qwoptics.py:619-623).
__global__ void meh_kernel(Step s) {
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

// CalcH (SBEs.py:819-935): one thread per (k1, k2).
__global__ void calch_kernel(Step s) {
  const int nk = s.nk, n2 = nk * nk;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n2) return;
  const int k1 = e / nk, k2 = e - k1 * nk;
  const double2* p = s.L3;
  const double2* C = s.L3 + n2;
  const double2* D = s.L3 + 2 * n2;
  const double* V = s.V3;
  double2 heh = s.Meh[e];
  double2 hee = make_double2(0.0, 0.0), hhh = hee;
  if (k1 == k2) {
    hee = make_double2(s.Ee[k1] + s.prm.gap, 0.0);
    hhh = make_double2(s.Eh[k1], 0.0);
  }
  if (s.prm.excitons) {
    const int qmin = max(-k1, -k2), qmax = min(nk - 1 - k1, nk - 1 - k2);
    // H^eh: sum_q V_eh(q) p^T[k1+q][k2+q]
    for (int q = qmin; q <= qmax; ++q)
      if (q != 0) heh = ca(heh, rs(vq(V, 0, nk, q), p[(k2 + q) * nk + (k1 + q)]));
    if (s.prm.lf) {
      for (int q = qmin; q <= qmax; ++q)
        if (q != 0) hee = cs(hee, rs(vq(V, 1, nk, q), C[(k2 + q) * nk + (k1 + q)]));
      const int qd = k1 - k2;
      if (qd != 0) {
        const int kmin = max(0, -qd), kmax = min(nk - 1, nk - 1 - qd);
        const double v1 = vq(V, 1, nk, qd), v0 = vq(V, 0, nk, qd), v2 = vq(V, 2, nk, qd);
        for (int k = kmin; k <= kmax; ++k)
          hee = ca(hee, cs(rs(v1, C[k * nk + k + qd]), rs(v0, D[(k + qd) * nk + k])));
        for (int q = qmin; q <= qmax; ++q)
          if (q != 0) hhh = cs(hhh, rs(vq(V, 2, nk, q), D[(k2 + q) * nk + (k1 + q)]));
        for (int k = kmin; k <= kmax; ++k)
          hhh = ca(hhh, cs(rs(v2, D[k * nk + k + qd]), rs(v0, C[(k + qd) * nk + k])));
      } else {
        for (int q = qmin; q <= qmax; ++q)
          if (q != 0) hhh = cs(hhh, rs(vq(V, 2, nk, q), D[(k2 + q) * nk + (k1 + q)]));
      }
    } else if (k1 == k2) {
      for (int q = -k1; q <= nk - 1 - k1; ++q)
        if (q != 0) hee = cs(hee, rs(vq(V, 1, nk, q), C[(k2 + q) * nk + (k1 + q)]));
      for (int q = -k1; q <= nk - 1 - k1; ++q)
        if (q != 0) hhh = cs(hhh, rs(vq(V, 2, nk, q), D[(k2 + q) * nk + (k1 + q)]));
    }
  }
  s.H[e] = heh;
  s.H[n2 + e] = hee;
  s.H[2 * n2 + e] = hhh;
}

// dpdt / dCdt / dDdt (SBEs.py:1952-1975, 2318-2337, 2617-2636): one thread
// per (i, j), the four dot products of each in the reference's order.
__global__ void derivs_kernel(Step s) {
  const int nk = s.nk, n2 = nk * nk;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n2) return;
  const int i = e / nk, j = e - i * nk;
  const double2* p = s.L3;
  const double2* C = s.L3 + n2;
  const double2* D = s.L3 + 2 * n2;
  const double2* Heh = s.H;
  const double2* Hee = s.H + n2;
  const double2* Hhh = s.H + 2 * n2;
  const double hb = s.prm.hbar;
  const double2 z = make_double2(0.0, 0.0);
  // dp[kh = i][ke = j]
  {
    double2 t1 = z, t2 = z, t3 = z, t4 = z;
    for (int k = 0; k < nk; ++k) t1 = ca(t1, cm(Hhh[i * nk + k], p[k * nk + j]));
    for (int k = 0; k < nk; ++k) t2 = ca(t2, cm(Hee[j * nk + k], p[i * nk + k]));
    for (int k = 0; k < nk; ++k) t3 = ca(t3, cm(Heh[k * nk + i], C[k * nk + j]));
    for (int k = 0; k < nk; ++k) t4 = ca(t4, cm(Heh[j * nk + k], D[k * nk + i]));
    double2 r = cs(cs(ca(t1, t2), t3), t4);
    r = ca(r, Heh[j * nk + i]);
    const double g = s.prm.gam_e + s.prm.gam_h;  // GamE[ke] + GamH[kh]
    r = cs(r, cm(make_double2(0.0 * g, hb * g), p[i * nk + j]));
    s.dX[e] = div_ih(r, hb);
  }
  // dC[k1 = i][k2 = j]
  {
    double2 t1 = z, t2 = z, t3 = z, t4 = z;
    for (int k = 0; k < nk; ++k) t1 = ca(t1, cm(Hee[j * nk + k], C[i * nk + k]));
    for (int k = 0; k < nk; ++k) t2 = ca(t2, cm(Hee[k * nk + i], C[k * nk + j]));
    for (int k = 0; k < nk; ++k) t3 = ca(t3, cm(Heh[j * nk + k], cconj(p[k * nk + i])));
    for (int k = 0; k < nk; ++k) t4 = ca(t4, cm(cconj(Heh[i * nk + k]), p[k * nk + j]));
    s.dX[n2 + e] = div_ih(cs(ca(cs(t1, t2), t3), t4), hb);
  }
  // dD[k1 = i][k2 = j]
  {
    double2 t1 = z, t2 = z, t3 = z, t4 = z;
    for (int k = 0; k < nk; ++k) t1 = ca(t1, cm(Hhh[j * nk + k], D[i * nk + k]));
    for (int k = 0; k < nk; ++k) t2 = ca(t2, cm(Hhh[k * nk + i], D[k * nk + j]));
    for (int k = 0; k < nk; ++k) t3 = ca(t3, cm(Heh[k * nk + j], cconj(p[i * nk + k])));
    for (int k = 0; k < nk; ++k) t4 = ca(t4, cm(cconj(Heh[k * nk + i]), p[j * nk + k]));
    s.dX[2 * n2 + e] = div_ih(cs(ca(cs(t1, t2), t3), t4), hb);
  }
}

// Leapfrog with neutrality and reshuffle (SBEs.py:5681-5718), one CTA.
constexpr int kLfThreads = 256;
__global__ void __launch_bounds__(kLfThreads) leapfrog_kernel(Step s) {
  const int nk = s.nk, n2 = nk * nk;
  const double dt = s.prm.dt, small = 1e-200;
  __shared__ double red_e[kLfThreads], red_h[kLfThreads];
  __shared__ double fac[3];
  auto x3_of = [&](int e) -> double2 {
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

// Wire-space sources of one level (one thread per r): the QWPolarization3
// sums (before the 2 ehint / (area L) factor and the transform) and the
// QWRho5 sums (before the boundary offset, normalisation and transform).
__global__ void sources_kernel(int nk, int nr, const double* kr, const double* rpos,
                               const double* window, double L, double dcv, double yw,
                               double sgnw, const double2* lev, double2* out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nr) return;
  const int n2 = nk * nk;
  const double2* p = lev;
  const double2* C = lev + n2;
  const double2* D = lev + 2 * n2;
  const double W = window[r], y = rpos[r];
  double px = 0.0, py = 0.0, pz = 0.0;
  for (int ke = 0; ke < nk; ++ke) {
    double se, ce;
    sincos(kr[ke] * y, &se, &ce);
    const double2 Ek = make_double2(ce, se);
    for (int kh = 0; kh < nk; ++kh) {
      double sh, ch;
      sincos(kr[kh] * y, &sh, &ch);
      const double2 Ekc = make_double2(ch, -sh);
      const double2 pk = p[kh * nk + ke];
      const double xvc = ((kh + 1) & 1) ? -dcv : dcv;  // conj(Xcv[ke][kh])
      px = px + cm(cm(rs(xvc, pk), Ek), Ekc).x * W;
      py = py + cm(cm(rs(dcv, pk), Ek), Ekc).x * W * yw;
      pz = pz + cm(cm(rs(-dcv, pk), Ek), Ekc).x * W * sgnw;
    }
  }
  double2 re = make_double2(0.0, 0.0), rh = re;
  for (int k2 = 0; k2 < nk; ++k2) {
    double s2, c2;
    sincos(kr[k2] * y, &s2, &c2);
    const double2 E2 = make_double2(c2, s2);
    for (int k1 = 0; k1 < nk; ++k1) {
      double s1, c1;
      sincos(kr[k1] * y, &s1, &c1);
      const double2 E1c = make_double2(c1, -s1);
      const double2 a = rs(W, cm(cm(C[k1 * nk + k2], E1c), E2));
      const double2 b = rs(W, cm(cm(cconj(D[k1 * nk + k2]), E1c), E2));
      re = ca(re, make_double2(a.x / (2.0 * L), a.y / (2.0 * L)));
      rh = ca(rh, make_double2(b.x / (2.0 * L), b.y / (2.0 * L)));
    }
  }
  out[r] = make_double2(px, 0.0);
  out[nr + r] = make_double2(py, 0.0);
  out[2 * nr + r] = make_double2(pz, 0.0);
  out[3 * nr + r] = re;
  out[4 * nr + r] = rh;
}

}  // namespace full
}  // namespace psb

using namespace psb;

extern "C" int64_t psb_full_work_bytes(int nk) {
  if (nk < 2 || nk > PSB_MAX_NK) return set_error(PSB_ERR_SIZE, "nk %d out of range", nk);
  return (int64_t)7 * nk * nk * 16;
}

extern "C" int psb_full_step_f64(int nk, int nr, int nq0, const double* d_V3, const double* d_Ee,
                                 const double* d_Eh, const double* d_fields,
                                 const PsbFullParams* params, double* d_L1, double* d_L2,
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
  full::Step s{};
  s.nk = nk;
  s.nr = nr;
  s.nq0 = nq0;
  s.V3 = d_V3;
  s.Ee = d_Ee;
  s.Eh = d_Eh;
  s.E = reinterpret_cast<const double2*>(d_fields);
  s.prm = *params;
  s.L1 = reinterpret_cast<double2*>(d_L1);
  s.L2 = reinterpret_cast<double2*>(d_L2);
  s.L3 = reinterpret_cast<double2*>(d_L3);
  double2* w = reinterpret_cast<double2*>(d_work);
  const int n2 = nk * nk;
  s.Meh = w;
  s.H = w + n2;
  s.dX = w + 4 * n2;
  cudaStream_t st = (cudaStream_t)stream;
  const int th = 128, bl = (n2 + th - 1) / th;
  full::meh_kernel<<<bl, th, 0, st>>>(s);
  full::calch_kernel<<<bl, th, 0, st>>>(s);
  full::derivs_kernel<<<bl, th, 0, st>>>(s);
  full::leapfrog_kernel<<<1, full::kLfThreads, 0, st>>>(s);
  return check_cuda("psb_full_step_f64");
}

extern "C" int psb_full_sources_f64(int nk, int nr, const double* d_kr, const double* d_r,
                                    const double* d_window, double L, double dcv, double yw,
                                    double sgnw, const double* d_level, double* d_out,
                                    void* stream) {
  if (!d_kr || !d_r || !d_window || !d_level || !d_out)
    return set_error(PSB_ERR_INVALID, "psb_full_sources_f64: null pointer");
  if (nk < 2 || nk > PSB_MAX_NK || nr < 1)
    return set_error(PSB_ERR_SIZE, "psb_full_sources_f64: nk %d / nr %d out of range", nk, nr);
  const int th = 64, bl = (nr + th - 1) / th;
  full::sources_kernel<<<bl, th, 0, (cudaStream_t)stream>>>(
      nk, nr, d_kr, d_r, d_window, L, dcv, yw, sgnw,
      reinterpret_cast<const double2*>(d_level), reinterpret_cast<double2*>(d_out));
  return check_cuda("psb_full_sources_f64");
}
