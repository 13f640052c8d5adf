/*
 * sbe_oracle.c -- CPU restatement of the reference quantum-wire SBE path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  See
 * sbe_oracle.h for the list of reference functions restated here.  Paths
 * in citations are relative to the reference project's src/pulsesuite.
 *
 * The right-hand side follows the reference's floating-point operation order
 * for diagonal states: the exchange sums run sequentially over q ascending as
 * in _CalcH_jit (PSTD3D/SBEs.py:896-913), and the dpdt/dCdt/dDdt
 * expressions keep the reference's association (SBEs.py:1958-1975,
 * 2325-2337, 2623-2636) after removing the exact zeros that diagonal matrices
 * contribute.  Build with -ffp-contract=off so no FMA changes the rounding.
 */
#include "sbe_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static const double kPi = 3.14159265358979323846;
static const double kEuler = 0.5772156649015329;

/* ---------------------------------------------------------------------------
 * Bessel K0.
 * ------------------------------------------------------------------------- */

/* The reference's JIT-friendly K0 approximation used inside Vint
 * (PSTD3D/coulomb.py:38-66), restated as written: 23 below 1e-10, a 19-term
 * series with (1/k - gamma) weights below 2, bare asymptote above, 0 past 100. */
double orc_k03_crude(double x) {
  if (x > 100.0) return 0.0;
  if (x < 1e-10) return 23.0;
  if (x < 2.0) {
    double x2 = x * x;
    double result = -log(0.5 * x) - kEuler;
    double term = 1.0;
    for (int k = 1; k < 20; ++k) {
      term = term * 0.25 * x2 / (double)(k * k);
      result = result + term * (1.0 / (double)k - kEuler);
      if (fabs(term) < 1e-15) break;
    }
    return result;
  }
  return sqrt(kPi / (2.0 * x)) * exp(-x);
}

/* The reference evaluates cik01 on numpy complex scalars with zero imaginary
 * part (K03 forms z = x + 0j from a numpy float).  For such values numpy's
 * complex division a/b is a * (1/b) and an integer power is a binary
 * exponentiation; these helpers restate that arithmetic on the real parts so
 * the rounding (which the K0 series amplifies for x in 6..9) matches. */
static double np_div(double a, double b) { return a * (1.0 / b); }

static double np_powi(double a, int n) {
  if (n == 1) return a;
  if (n == 2) return a * a;
  if (n == 3) return a * (a * a);
  double aa = 1.0, p = a;
  int mask = 1;
  for (;;) {
    if (n & mask) aa = aa * p;
    mask <<= 1;
    if (n < mask) break;
    p = p * p;
  }
  return aa;
}

/* I0(x), x > 0, by the Zhang & Jin method used in cik01
 * (PSTD3D/usefulsubs.py:1712-1748): power series up to 18, Hankel
 * asymptotic series above with 12/9/7 terms.  The asymptotic coefficients
 * a_k = ((2k-1)!!)^2 / (k! 8^k) are generated here from that formula. */
double orc_i0(double x) {
  if (x <= 18.0) {
    double z2 = x * x;
    double s = 1.0, cr = 1.0;
    for (int k = 1; k <= 50; ++k) {
      cr = np_div(0.25 * cr * z2, (double)(k * k));
      s = s + cr;
      if (fabs(np_div(cr, s)) < 1e-15) break;
    }
    return s;
  }
  int k0 = x < 35.0 ? 12 : (x < 50.0 ? 9 : 7);
  double ca = np_div(exp(x), sqrt(2.0 * kPi * x));
  double zr = np_div(1.0, x), s = 1.0, ak = 1.0;
  for (int k = 1; k <= k0; ++k) {
    double odd = (double)(2 * k - 1);
    ak = ak * odd * odd / ((double)k * 8.0);
    s = s + ak * np_powi(zr, k);
  }
  return ca * s;
}

/* K0(x), x > 0, as the reference's K03 computes it through cik01
 * (PSTD3D/usefulsubs.py:1750-1772, 1794-1820): series in (x/2)^2 with
 * harmonic weights up to 9; above 9, K0 = (1/(2x)) (1 + sum_k b_k x^-2k) / I0
 * with the ten coefficients of the I0*K0 asymptotic product,
 * b_k = [(2k-1)!!/(2k)!!] ((2k-1)!!)^2 / 4^k.  0 past 100 as K03 does. */
double orc_k0(double x) {
  if (x > 100.0) return 0.0;
  if (x <= 0.0) return 1e30;
  if (x <= 9.0) {
    double z2 = x * x;
    double ct = -log(0.5 * x) - kEuler;
    double w0 = 0.0, cr = 1.0, cs = 0.0, cw = 0.0;
    for (int k = 1; k <= 50; ++k) {
      w0 = w0 + 1.0 / (double)k;
      cr = np_div(0.25 * cr, (double)(k * k)) * z2;
      cs = cs + cr * (w0 + ct);
      if (fabs(np_div(cs - cw, cs)) < 1e-15) break;
      cw = cs;
    }
    return ct + cs;
  }
  double cb = np_div(0.5, x);
  double zr2 = np_div(1.0, x * x), s = 1.0, ratio = 1.0, dfac = 1.0;
  for (int k = 1; k <= 10; ++k) {
    double odd = (double)(2 * k - 1);
    ratio = ratio * odd / (double)(2 * k);
    dfac = dfac * odd * odd / 4.0;
    s = s + ratio * dfac * np_powi(zr2, k);
  }
  return np_div(cb * s, orc_i0(x));
}

/* ---------------------------------------------------------------------------
 * Coulomb tables.
 * ------------------------------------------------------------------------- */

/* prefactor * Vint(qy[i]) for every i: the Gaussian-confined double sum of
 * PSTD3D/coulomb.py:69-104 over y indices [Ny/4, 3Ny/4], as called by
 * CalcCoulombArrays (coulomb.py:548-557). */
void orc_vint_table(const double* qy, int nq, const double* y, int ny, double alpha1,
                    double alpha2, double delta0, double prefactor, double* out) {
  int n1 = ny / 4, n2 = 3 * ny / 4;
  double* a1 = (double*)malloc(sizeof(double) * (size_t)ny);
  double* a2 = (double*)malloc(sizeof(double) * (size_t)ny);
  for (int i = 0; i < ny; ++i) {
    a1[i] = (alpha1 * y[i]) * (alpha1 * y[i]);
    a2[i] = (alpha2 * y[i]) * (alpha2 * y[i]);
  }
  double kmin = (alpha1 + alpha2) / 4.0;
  double dy = y[1] - y[0];
  double mult = alpha1 * alpha2 / kPi * (dy * dy);
#pragma omp parallel for schedule(dynamic)
  for (int iq = 0; iq < nq; ++iq) {
    double dk = fabs(qy[iq]) > kmin ? fabs(qy[iq]) : kmin;
    double v = 0.0;
    for (int i = n1; i <= n2; ++i) {
      for (int j = n1; j <= n2; ++j) {
        double d = y[i] - y[j];
        double r = sqrt(d * d + delta0 * delta0);
        double ef = exp(-a1[i] - a2[j]);
        v += ef * mult * orc_k03_crude(dk * r);
      }
    }
    out[iq] = prefactor * v;
  }
  free(a1);
  free(a2);
}

void orc_k0_table(const double* q, int nq, double radius, double prefactor, double* out) {
  for (int i = 0; i < nq; ++i)
    out[i] = q[i] == 0.0 ? 0.0 : prefactor * orc_k0(fabs(q[i]) * radius);
}

/* CalcChi1D at [q, 0] (PSTD3D/coulomb.py:612-628). */
void orc_chi1d_table(const double* qc, int nq, double alpha, double delta0, double mass,
                     double scale, double* out) {
  double R = sqrt((2.0 / alpha) * (2.0 / alpha) + delta0 * delta0);
  for (int i = 0; i < nq; ++i) out[i] = mass * orc_k0(qc[i] * R) / qc[i] * scale;
}

/* ---------------------------------------------------------------------------
 * Right-hand side of one wire.
 * ------------------------------------------------------------------------- */

static void drive(const PsbWire* w, double t, double* er, double* ei) {
  double re = 0.0, im = 0.0;
  for (int j = 0; j < w->npulse && j < 2; ++j) {
    double u = (t - w->t0[j]) / w->fwhm[j];
    double env = w->amp[j] * exp(-4.0 * log(2.0) * u * u);
    re += env * cos(w->phase[j]);
    im += env * sin(w->phase[j]);
  }
  *er = re;
  *ei = im;
}

/* Screened (or plain) V tables of a wire at its current densities, with the
 * q = 0 entry zeroed: CalcScreenedArrays + Eps1D (coulomb.py:1172-1230). */
static void wire_tables(const PsbTable* tb, const double* td, const double* y, double* veh,
                        double* vee, double* vhh) {
  int nk = tb->nk;
  const double* V = td + tb->off;
  if (tb->flags & PSB_TAB_SCREENED) {
    const double* chie = V + 5 * (size_t)nk;
    const double* chih = V + 6 * (size_t)nk;
    const double* qe = V + 7 * (size_t)nk;
    const double* qh = V + 8 * (size_t)nk;
    double s = 0.0;
    for (int k = 0; k < nk; ++k) s += y[4 * k + 2] + y[4 * k + 3];
    double n1d = s / 2.0 / tb->L;
    if (n1d > tb->dens_max) n1d = tb->dens_max;
    for (int q = 0; q < nk; ++q) {
      double eps = 1.0 - chie[q] * 2.0 * log(fabs((qe[q] - kPi * n1d) / (qe[q] + n1d))) -
                   chih[q] * 2.0 * log(fabs((qh[q] - kPi * n1d) / (qh[q] + n1d)));
      veh[q] = V[q] / eps;
      vee[q] = V[nk + q] / eps;
      vhh[q] = V[2 * nk + q] / eps;
    }
  } else {
    for (int q = 0; q < nk; ++q) {
      veh[q] = V[q];
      vee[q] = V[nk + q];
      vhh[q] = V[2 * nk + q];
    }
  }
  veh[0] = vee[0] = vhh[0] = 0.0;
}

/* f(t, y) of one wire; scratch holds 3*nk doubles. */
static void rhs_wire(const PsbTable* tb, const double* td, const PsbWire* w, double mr, double mi,
                     const double* y, double* dy, double hbar, double* scratch) {
  int nk = tb->nk;
  const double* Ee = td + tb->off + 3 * (size_t)nk;
  const double* Eh = td + tb->off + 4 * (size_t)nk;
  double* veh = scratch;
  double* vee = scratch + nk;
  double* vhh = scratch + 2 * nk;
  int exc = (tb->flags & PSB_TAB_EXCITONS) != 0;
  if (exc) wire_tables(tb, td, y, veh, vee, vhh);
  double hg = hbar * w->gamma;
  for (int k = 0; k < nk; ++k) {
    /* CalcH, excitons & !LF branch (SBEs.py:896-921): Heh[k,k] = Meh + sum,
     * Hee[k,k] = Ee+gap - sum, Hhh[k,k] = Eh - sum, q ascending. */
    double omr = mr, omi = mi;
    double se = Ee[k] + w->gap;
    double sh = Eh[k];
    if (exc) {
      for (int kp = 0; kp < nk; ++kp) {
        if (kp == k) continue;
        int d = kp > k ? kp - k : k - kp;
        omr = omr + veh[d] * y[4 * kp + 0];
        omi = omi + veh[d] * y[4 * kp + 1];
        se = se - vee[d] * y[4 * kp + 2];
        sh = sh - vhh[d] * y[4 * kp + 3];
      }
    }
    double a = y[4 * k + 0], b = y[4 * k + 1];
    double ne = y[4 * k + 2], nh = y[4 * k + 3];
    /* dpdt (SBEs.py:1962-1975): X = Hhh p + Hee p - Heh C - Heh D + Heh
     * - i hbar gamma p, then X / (i hbar). */
    double xr = sh * a + se * a;
    double xi = sh * b + se * b;
    xr = xr - omr * ne;
    xi = xi - omi * ne;
    xr = xr - omr * nh;
    xi = xi - omi * nh;
    xr = xr + omr;
    xi = xi + omi;
    xr = xr - (-(hg * b));
    xi = xi - hg * a;
    dy[4 * k + 0] = xi / hbar;
    dy[4 * k + 1] = -xr / hbar;
    /* dCdt / dDdt (SBEs.py:2325-2337, 2623-2636): Heh p* - Heh^* p over i hbar. */
    double u = omi * a - omr * b;
    double dn = (u + u) / hbar;
    dy[4 * k + 2] = dn;
    dy[4 * k + 3] = dn;
  }
}

static int check_tables(const PsbTable* tables, int ntab, const PsbWire* wires, int nw) {
  if (!tables || !wires || ntab <= 0 || nw < 0) return PSB_ERR_INVALID;
  for (int i = 0; i < nw; ++i) {
    if (wires[i].table < 0 || wires[i].table >= ntab) return PSB_ERR_INVALID;
    int nk = tables[wires[i].table].nk;
    if (nk < 2 || nk > PSB_MAX_NK) return PSB_ERR_SIZE;
  }
  return PSB_OK;
}

int orc_rhs(const PsbTable* tables, int ntab, const double* td, const PsbWire* wires, int nw,
            const double* t, const double* y, double* dy, const PsbModel* model) {
  int rc = check_tables(tables, ntab, wires, nw);
  if (rc) return rc;
#pragma omp parallel
  {
    double* scratch = (double*)malloc(sizeof(double) * 3 * PSB_MAX_NK);
#pragma omp for schedule(dynamic)
    for (int i = 0; i < nw; ++i) {
      const PsbWire* w = &wires[i];
      const PsbTable* tb = &tables[w->table];
      double mr, mi;
      drive(w, t ? t[i] : w->t, &mr, &mi);
      mr = -w->mscale * mr;
      mi = -w->mscale * mi;
      rhs_wire(tb, td, w, mr, mi, y + 4 * w->off, dy + 4 * w->off, model->hbar, scratch);
    }
    free(scratch);
  }
  return PSB_OK;
}

/* P(t) record of the call-local step s (0-based): every p_stride-th step. */
static void record_P(const PsbWire* w, int s, int nk, const double* y, double* P, int p_stride,
                     int p_cap) {
  if (!P || p_stride <= 0 || ((s + 1) % p_stride) != 0) return;
  int r = (s + 1) / p_stride - 1;
  if (r < 0 || r >= p_cap) return;
  double sr = 0.0, si = 0.0;
  for (int k = 0; k < nk; ++k) {
    sr += y[4 * k + 0];
    si += y[4 * k + 1];
  }
  P[2 * (w->p_off + r) + 0] = w->pscale * sr;
  P[2 * (w->p_off + r) + 1] = w->pscale * si;
}

static void check_finite(PsbWire* w, int nk, const double* y) {
  for (int k = 0; k < 4 * nk; ++k)
    if (!isfinite(y[k])) {
      w->status = PSB_ERR_NONFINITE;
      return;
    }
}

/* Classical RK4 in the stage order of _rk4 (libpulsesuite/integrator.py:143-157),
 * with dydt = D(t, y) computed first as rk4_dpc's callers do. */
int orc_rk4(const PsbTable* tables, int ntab, const double* td, PsbWire* wires, int nw,
            double* y, int nsteps, double dt, double* P, int p_stride, int p_cap,
            const PsbModel* model, int nthreads) {
  int rc = check_tables(tables, ntab, wires, nw);
  if (rc) return rc;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  double hbar = model->hbar;
#pragma omp parallel
  {
    size_t n4 = 4 * (size_t)PSB_MAX_NK;
    double* buf = (double*)malloc(sizeof(double) * (5 * n4 + 3 * PSB_MAX_NK));
    double *k1 = buf, *k2 = buf + n4, *k3 = buf + 2 * n4, *k4 = buf + 3 * n4;
    double* yt = buf + 4 * n4;
    double* scratch = buf + 5 * n4;
#pragma omp for schedule(dynamic)
    for (int i = 0; i < nw; ++i) {
      PsbWire* w = &wires[i];
      const PsbTable* tb = &tables[w->table];
      int nk = tb->nk, n = 4 * nk;
      double* yw = y + 4 * w->off;
      double h = dt;
      for (int s = 0; s < nsteps; ++s) {
        double t = w->t, er, ei;
        drive(w, t, &er, &ei);
        rhs_wire(tb, td, w, -w->mscale * er, -w->mscale * ei, yw, k1, hbar, scratch);
        for (int j = 0; j < n; ++j) yt[j] = yw[j] + (h / 2.0) * k1[j];
        drive(w, t + h / 2.0, &er, &ei);
        rhs_wire(tb, td, w, -w->mscale * er, -w->mscale * ei, yt, k2, hbar, scratch);
        for (int j = 0; j < n; ++j) yt[j] = yw[j] + (h / 2.0) * k2[j];
        rhs_wire(tb, td, w, -w->mscale * er, -w->mscale * ei, yt, k3, hbar, scratch);
        for (int j = 0; j < n; ++j) yt[j] = yw[j] + h * k3[j];
        for (int j = 0; j < n; ++j) k3[j] = k3[j] + k2[j];
        drive(w, t + h, &er, &ei);
        rhs_wire(tb, td, w, -w->mscale * er, -w->mscale * ei, yt, k4, hbar, scratch);
        for (int j = 0; j < n; ++j) yw[j] = yw[j] + (h / 6.0) * (k1[j] + k4[j] + 2.0 * k3[j]);
        w->t = t + h;
        w->steps += 1;
        record_P(w, s, nk, yw, P, p_stride, p_cap);
      }
      check_finite(w, nk, yw);
    }
    free(buf);
  }
  return PSB_OK;
}

/* The reference's own integrator, SBESolver._sbe_calculator
 * (PSTD3D/SBEs.py:5681-5718): leapfrog X3 = X1 + 2 dt f(X2), population
 * neutrality on diag(X3), then X1 <- (X1+X3)/2, X2 <- X3. */
int orc_leapfrog(const PsbTable* tables, int ntab, const double* td, PsbWire* wires, int nw,
                 double* y1, double* y2, const double* field, int field_stride, int nsteps,
                 double dt, double* P, int p_stride, int p_cap, const PsbModel* model,
                 int nthreads) {
  int rc = check_tables(tables, ntab, wires, nw);
  if (rc) return rc;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  double hbar = model->hbar;
  const double small = 1e-200; /* SBEs.py:4717 */
#pragma omp parallel
  {
    size_t n4 = 4 * (size_t)PSB_MAX_NK;
    double* buf = (double*)malloc(sizeof(double) * (2 * n4 + 3 * PSB_MAX_NK));
    double* f = buf;
    double* x3 = buf + n4;
    double* scratch = buf + 2 * n4;
#pragma omp for schedule(dynamic)
    for (int i = 0; i < nw; ++i) {
      PsbWire* w = &wires[i];
      const PsbTable* tb = &tables[w->table];
      int nk = tb->nk, n = 4 * nk;
      double* a = y1 + 4 * w->off;
      double* b = y2 + 4 * w->off;
      for (int s = 0; s < nsteps; ++s) {
        const double* e = field + (size_t)i * (size_t)field_stride + 2 * (size_t)w->steps;
        rhs_wire(tb, td, w, -w->mscale * e[0], -w->mscale * e[1], b, f, hbar, scratch);
        for (int j = 0; j < n; ++j) x3[j] = a[j] + f[j] * dt * 2.0;
        double se = 0.0, sh = 0.0;
        for (int k = 0; k < nk; ++k) {
          x3[4 * k + 2] = fabs(x3[4 * k + 2]);
          x3[4 * k + 3] = fabs(x3[4 * k + 3]);
          se += x3[4 * k + 2];
          sh += x3[4 * k + 3];
        }
        double total = (se + sh) / 2.0;
        for (int k = 0; k < nk; ++k) {
          x3[4 * k + 2] = x3[4 * k + 2] * total / (se + small);
          x3[4 * k + 3] = x3[4 * k + 3] * total / (sh + small);
        }
        for (int j = 0; j < n; ++j) {
          a[j] = (a[j] + x3[j]) / 2.0;
          b[j] = x3[j];
        }
        w->t = w->t + dt;
        w->steps += 1;
        record_P(w, s, nk, b, P, p_stride, p_cap);
      }
      check_finite(w, nk, b);
    }
    free(buf);
  }
  return PSB_OK;
}
