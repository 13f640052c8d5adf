/*
 * pulsesuite_b200.h -- C ABI of the B200 (sm_100a) quantum-wire SBE step.
 *
 * Drop-in boundary for the reference's SBE hot path (pulsesuite, pure
 * Python).  The reference binds its kernels through Python call signatures;
 * each entry point below names the reference interface it replaces
 * (file:line, paths relative to the reference project's src/pulsesuite).
 * The Python facade (pulsesuite_b200/SBEs.py, coulomb.py) binds these with
 * ctypes, the way a maintainer of the reference would bind them.
 *
 * Conventions
 *   - Every function returns PSB_OK (0) or a negative PSB_ERR_* code and never
 *     aborts; psb_last_error() returns a thread-local message for the last
 *     failure.
 *   - Pointers named d_* are device pointers (CUDA global memory on the
 *     current device); the caller allocates and owns every buffer, and the
 *     step entry points allocate nothing.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *     Calls are asynchronous with respect to the host unless stated.
 *   - All arithmetic of the *_f64 entry points is IEEE binary64.
 *
 * Diagonal SBE model (what the reference's full-matrix SBEs reduce to when
 * p, C, D and the drive are diagonal in k; SBEs.py:843-935, 1958-1975,
 * 2325-2337, 2623-2636):
 *   Omega_k = M(t) + sum_{k'!=k} Veh(|k-k'|) p_k'
 *   Se_k    = Ee_k + gap - sum_{k'!=k} Vee(|k-k'|) ne_k'
 *   Sh_k    = Eh_k       - sum_{k'!=k} Vhh(|k-k'|) nh_k'
 *   i hbar dp_k/dt  = (Se_k+Sh_k) p_k - Omega_k (ne_k+nh_k) + Omega_k - i hbar gamma p_k
 *   i hbar dne_k/dt = i hbar dnh_k/dt = Omega_k p_k^* - Omega_k^* p_k
 *   M(t) = -mscale * E(t)
 * V(q) may be statically screened per wire and per right-hand-side
 * evaluation: V_n(q) <- V_n(q) / eps(q; n1D)  (coulomb.py:1195-1230).
 */
#ifndef PULSESUITE_B200_H
#define PULSESUITE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSB_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
#define PSB_OK 0
#define PSB_ERR_INVALID (-1)     /* bad argument (null pointer, bad size)      */
#define PSB_ERR_CUDA (-2)        /* CUDA runtime error (message in last_error)  */
#define PSB_ERR_SIZE (-3)        /* size beyond the supported maximum           */
#define PSB_ERR_NONFINITE (-4)   /* per-wire status: state became NaN/Inf       */
#define PSB_ERR_UNSUPPORTED (-5) /* feature not available on this device/build  */
#define PSB_ERR_TIMEOUT (-6)     /* per-wire status: a bounded on-chip wait ran out */

/* Largest k grid one wire may have (one CTA holds a wire's state). */
#define PSB_MAX_NK 1024

/* ---- table flags --------------------------------------------------------- */
#define PSB_TAB_EXCITONS 1 /* include the Hartree-Fock exchange sums (mb.params Excitons) */
#define PSB_TAB_SCREENED 2 /* screen V per wire and per RHS (mb.params Screened)         */
#define PSB_TAB_SHARED_V 4 /* Veh == Vee == Vhh (one table serves all three sums)        */

/*
 * One k grid with its Coulomb/energy tables.  The doubles live in a packed
 * device array `tabdata`, starting at `off`, each block nk long:
 *   [0] Veh(q)  [1] Vee(q)  [2] Vhh(q)   q = index distance 0..nk-1
 *       (the q = 0 entry is never used: the reference excludes q = 0,
 *        SBEs.py:829-834, 876-878)
 *   [3] Ee(k)   [4] Eh(k)                band energies (J), SBEs.py:4834-4835
 *   [5] chi_e(q) [6] chi_h(q) [7] qe(q) [8] qh(q)
 *       screening blocks, read only with PSB_TAB_SCREENED
 *       (coulomb.py:302-333 MakeQs and 580-630 CalcChi1D at [q, 0]).
 */
typedef struct PsbTable {
  int32_t nk;       /* k points (even, 2..PSB_MAX_NK)                              */
  int32_t flags;    /* PSB_TAB_*                                                   */
  int64_t off;      /* offset (doubles) of this table's blocks in tabdata          */
  double L;         /* wire length (m): n1D = sum_k(ne_k+nh_k)/2/L (coulomb.py:1221) */
  double dens_max;  /* n1D clamp min(qe[1,1],qh[1,1])/pi*0.99 (coulomb.py:1222)    */
} PsbTable;

/*
 * One wire.  The wire's k block occupies state elements [off, off+nk) of
 * the packed state, each element 4 doubles {p_re, p_im, ne, nh}.
 * Analytic drive (RK4 entry points):
 *   E(t) = sum_{j<npulse} amp_j exp(-4 ln2 (t-t0_j)^2 / fwhm_j^2) exp(i phase_j)
 * The leapfrog entry point takes sampled E(t_n) instead (field array).
 */
typedef struct PsbWire {
  int32_t table;     /* index of this wire's PsbTable                               */
  int32_t npulse;    /* Gaussian pulses in the analytic drive, 0..2                 */
  int64_t off;       /* first state element of this wire                            */
  double gap;        /* energy added to Ee (J); rotating frame: gap - hbar*omega_L  */
  double gamma;      /* gam_e + gam_h (1/s); dephasing of p (SBEs.py:1974)           */
  double mscale;     /* M_k(t) = -mscale * E(t)                                     */
  double pscale;     /* P(t) = pscale * sum_k p_k                                   */
  double t;          /* time (s) at the start of the next step; advanced by calls   */
  double amp[2];     /* pulse amplitudes (V/m)                                      */
  double t0[2];      /* pulse centres (s)                                           */
  double fwhm[2];    /* pulse intensity FWHM of the field envelope (s)              */
  double phase[2];   /* pulse carrier-envelope phases (rad)                         */
  int64_t p_off;     /* first P(t) record (complex sample) of this wire             */
  int32_t status;    /* PSB_OK, or PSB_ERR_NONFINITE once the state is not finite   */
  int32_t steps;     /* steps taken so far (advanced by the step entry points)      */
} PsbWire;

/* Model constants shared by every wire of a call. */
typedef struct PsbModel {
  double hbar;       /* reduced Planck constant (J s)                               */
  int32_t flags;     /* reserved, 0                                                 */
  int32_t reserved;
} PsbModel;

/* ---- library ------------------------------------------------------------ */
int psb_abi_version(void);
/* Message of the last failing call on this thread ("" when none). */
const char* psb_last_error(void);
/* Compute capability of the current device, e.g. 100 for sm_100a. */
int psb_device_arch(int* arch);

/* ---- Coulomb tables (init-time, FP64) ------------------------------------ */
/*
 * Unscreened 1D Coulomb matrix elements with Gaussian confinement,
 *   out[i] = prefactor * Vint(qy[i], y, alpha1, alpha2, delta0)
 * Replaces coulomb.py:69-104 (_Vint_jit, with its _K03_jit Bessel
 * approximation, coulomb.py:38-66) as called by CalcCoulombArrays
 * (coulomb.py:548-557).  prefactor = e^2/(2 pi eps0 epsr L).
 */
int psb_coulomb_vint(const double* d_qy, int nq, const double* d_y, int ny, double alpha1,
                     double alpha2, double delta0, double prefactor, double* d_out,
                     void* stream);
/*
 * Regularised wire potential out[i] = prefactor * K0(|q_i| * radius)
 * (K0 by the Zhang & Jin series/asymptotic method that the reference's
 * K03 uses, usefulsubs.py:1669-1820).  Entries with q_i == 0 are set to 0.
 */
int psb_coulomb_k0(const double* d_q, int nq, double radius, double prefactor, double* d_out,
                   void* stream);
/*
 * 1D susceptibility at momentum transfers qc[i] (already clamped at alpha/2,
 * coulomb.py:325-331): out[i] = scale * mass * K03(qc[i]*R)/qc[i] with
 * R = sqrt((2/alpha)^2 + delta0^2).  Replaces CalcChi1D (coulomb.py:580-630).
 */
int psb_chi1d(const double* d_qc, int nq, double alpha, double delta0, double mass,
              double scale, double* d_out, void* stream);
/*
 * Static screening of every wire for its current densities:
 *   d_eps[w*ldeps + q] = eps(q; n1D_w), q < nk of the wire's table,
 * n1D_w = min(sum_k(ne+nh)/(2L), dens_max).  Replaces Eps1D / the
 * screening branch of CalcScreenedArrays (coulomb.py:1172-1193, 1218-1230).
 */
int psb_screen_f64(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                   const PsbWire* d_wires, int nw, const double* d_y, double* d_eps, int ldeps,
                   void* stream);

/* ---- SBE right-hand side and steps (FP64) -------------------------------- */
/*
 * Shared arguments of the SBE entry points:
 *   d_tables[ntab], d_tabdata[n_tabdata]  device tables (PsbTable doc)
 *   d_wires[nw]                           device wire descriptors (PsbWire doc)
 *   d_y (and d_y1)                        packed state, n_state elements of
 *                                         4 doubles {p_re, p_im, ne, nh}
 *   d_order, n_order                      optional list of wire indices to
 *                                         advance (one CTA each, in this
 *                                         order; largest grids first balances
 *                                         uneven batches), or NULL for all nw
 *   nkmax                                 largest table nk of the wires
 *                                         launched (sizes shared memory and
 *                                         registers: launch size classes
 *                                         separately for speed)
 *   tab_flags                             PSB_TAB_SCREENED if any launched
 *                                         table is screened; PSB_TAB_SHARED_V
 *                                         only if every launched table has it
 * Descriptors are validated on the device: a wire whose table index, grid
 * size or state range is invalid is skipped and its status set to
 * PSB_ERR_INVALID / PSB_ERR_SIZE.  A wire whose state stops being finite gets
 * PSB_ERR_NONFINITE; other wires of the launch are unaffected (each wire's
 * arithmetic is independent of its neighbours, so results are bitwise the
 * same alone and in any batch).
 */

/*
 * Right-hand side of every wire at the wire's own t: d_dy = f(t_w, d_y).
 * Replaces the diagonal action of CalcH + dpdt + dCdt + dDdt
 * (SBEs.py:669-935, 1850-1975, 2221-2337, 2513-2636) including the per-call
 * screening of _preparation (SBEs.py:5185-5238).
 */
int psb_rhs_f64(const PsbTable* d_tables, int ntab, const double* d_tabdata, int64_t n_tabdata,
                const PsbWire* d_wires, int nw, const double* d_y, double* d_dy,
                int64_t n_state, int nkmax, int tab_flags, const PsbModel* model, void* stream);
/*
 * Renormalised single-particle Hamiltonian diagonals of every wire (the
 * diagonal of CalcH, SBEs.py:669-935 / _CalcH_jit SBEs.py:819-935, with the
 * exchange sums over k' and, for screened tables, the per-call screening):
 * d_h[e] = (Re Heh, Im Heh, Hee, Hhh) per element, where Heh = M(t_w) +
 * sum_{q!=0} Veh(q) p_{k+q}, Hee = Ee + gap - sum Vee(q) n_e,k+q and
 * Hhh = Eh - sum Vhh(q) n_h,k+q.  M(t_w) is the wire's drive at its own t
 * (zero for npulse = 0).
 */
int psb_calch_f64(const PsbTable* d_tables, int ntab, const double* d_tabdata, int64_t n_tabdata,
                  const PsbWire* d_wires, int nw, const double* d_y, double* d_h,
                  int64_t n_state, int nkmax, int tab_flags, const PsbModel* model,
                  void* stream);
/*
 * Diagonal time derivatives of n k-points from given Hamiltonian diagonals:
 * the diagonal of dpdt, dCdt and dDdt (SBEs.py:1850-1975, 2221-2337,
 * 2513-2636) for diagonal states, in the reference's association order,
 *   i hbar dp = Hhh p + Hee p - Heh C - Heh D + Heh - i hbar g p + Off
 *   i hbar dC = i hbar dD = Heh conj(p) - conj(Heh) p
 * d_h[3k..3k+2] = (Heh, Hee, Hhh) and d_state[3k..3k+2] = (p, C, D) as
 * complex (re, im) pairs; d_gam[k] = GamE_k + GamH_k; d_off[k] = OffP_kk
 * (complex) or NULL; d_out[3k..3k+2] = (dp, dC, dD) complex.
 */
int psb_diag_derivs_f64(const double* d_h, const double* d_state, const double* d_gam,
                        const double* d_off, double hbar, double* d_out, int64_t n,
                        void* stream);
/*
 * nsteps classical RK4 steps of size dt on every wire, in the stage order of
 * the reference integrator (libpulsesuite/integrator.py:143-157, rk4_dpc),
 * the whole step fused in one kernel with the wire's state resident on chip.
 * Advances each wire's t and steps.  Every p_stride-th step of the call
 * (s = 1..nsteps, counted from the start of this call) writes
 * P(t) = pscale * sum_k p_k to d_P[p_off + s/p_stride - 1] (complex: 2
 * doubles) while s/p_stride <= p_cap and the record lies inside d_P[0, n_P)
 * (qwoptics.py:815-946, diagonal form).  A caller advancing a solve in
 * chunks copies each chunk's records out before the next call.
 */
int psb_rk4_f64(const PsbTable* d_tables, int ntab, const double* d_tabdata, int64_t n_tabdata,
                PsbWire* d_wires, int nw, const int32_t* d_order, int n_order, double* d_y,
                int64_t n_state, int nkmax, int tab_flags, int nsteps, double dt, double* d_P,
                int64_t n_P, int p_stride, int p_cap, const PsbModel* model, void* stream);
/*
 * nsteps steps of the reference's own integrator (SBEs.py:5681-5718):
 *   X3 = X1 + 2 dt f(X2);  ne3 = |ne3|, nh3 = |nh3| rescaled to a common
 *   total;  X1 <- (X1 + X3)/2;  X2 <- X3.
 * d_y1 / d_y2 are the two stored levels (YY2/CC2/DD2 and YY3/CC3/DD3 of
 * SBESolver, SBEs.py:5073-5092).  The drive of a wire's step n is the
 * sampled field d_field[w*field_stride + 2*steps_n] (re, im; n_field doubles
 * in all), the q = 0 component the reference passes as Ey[NQ0] to CalcMeh
 * (SBEs.py:5165-5175).  P(t) of the new level X3 is recorded as in
 * psb_rk4_f64 (QWPolarization3 of p3, SBEs.py:5729-5742).
 */
int psb_leapfrog_f64(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                     int64_t n_tabdata, PsbWire* d_wires, int nw, const int32_t* d_order,
                     int n_order, double* d_y1, double* d_y2, int64_t n_state, int nkmax,
                     int tab_flags, const double* d_field, int64_t field_stride,
                     int64_t n_field, int nsteps, double dt, double* d_P, int64_t n_P,
                     int p_stride, int p_cap, const PsbModel* model, void* stream);
/* Dynamic shared memory (bytes) one CTA of the FP64 step kernels uses for a
 * grid of nk points (for capacity planning; tab_flags as above). */
int psb_f64_smem_bytes(int nk, int tab_flags);

/* ---- full-matrix form (FP64): fields that vary along the wire ------------- */
/*
 * Constants of one wire's full-matrix step.  gam_e + gam_h is the dephasing
 * of p (GamE, GamH of _preparation without k-dependent dephasing,
 * SBEs.py:5213-5214); yw = yw(w) and sgnw = (-1)^w are the wire's dipole
 * signs (qwoptics.py:1099-1112, SBEs.py:5171-5174).
 */
typedef struct PsbFullParams {
  double ehint;     /* electron-hole overlap integral                          */
  double dcv;       /* interband dipole (C m)                                  */
  double yw;        /* yw(w)                                                   */
  double sgnw;      /* (-1)^w                                                  */
  double gap;       /* band gap (J), added to Ee on the diagonal of Hee         */
  double gam_e;     /* 1/s                                                     */
  double gam_h;     /* 1/s                                                     */
  double hbar;      /* J s                                                     */
  double dt;        /* step (s)                                                */
  int32_t excitons; /* mb.params Excitons                                      */
  int32_t lf;       /* mb.params LF: full Hee/Hhh with the direct terms        */
} PsbFullParams;

/* Work bytes psb_full_step_f64 needs for a grid of nk (Meh, H, dX). */
int64_t psb_full_work_bytes(int nk);
/*
 * One step of the reference's integrator for one wire with full Nk x Nk
 * states (SBESolver._sbe_calculator, SBEs.py:5624-5718): Meh from the
 * wire-space fields (CalcMeh, SBEs.py:5165-5175), CalcH with the exchange
 * and, with lf, direct Coulomb sums (SBEs.py:819-935), dpdt / dCdt / dDdt
 * (SBEs.py:1952-1975, 2318-2337, 2617-2636), then X3 = X1 + 2 dt dX with the
 * occupations |C3_kk|, |D3_kk| rescaled to a common total and X2 = (X1+X3)/2
 * (SBEs.py:5681-5718).
 *   d_V3      [3][nk] V_eh, V_ee, V_hh at index distance q (screened if the
 *             caller screened them for this step, coulomb.py:1195-1230)
 *   d_Ee/Eh   [nk] band energies
 *   d_fields  [3][nr] complex: Ex, Ey, Ez in wire q space (after Prop2QW),
 *             q index of k - k' at (k - k') + nq0
 *   d_L1..L3  [3][nk][nk] complex each: the levels (p, C, D); the step reads
 *             L2 (X1) and L3 (X2) and writes L1 = X1, L2 = (X1 + X3)/2,
 *             L3 = X3 (the checkin of SBEs.py:5082-5092)
 *   d_work    psb_full_work_bytes(nk) bytes
 */
int psb_full_step_f64(int nk, int nr, int nq0, const double* d_V3, const double* d_Ee,
                      const double* d_Eh, const double* d_fields, const PsbFullParams* params,
                      double* d_L1, double* d_L2, double* d_L3, void* d_work,
                      int64_t n_work_bytes, void* stream);
/*
 * Wire-space source terms of one level (d_level = [3][nk][nk] complex p, C,
 * D) on the wire grid r[nr] with the window[nr]: d_out[5][nr] complex =
 * Px, Py, Pz as the sums of QWPolarization3 before the 2 ehint/(area L)
 * factor and the transform (qwoptics.py:56-84), and the electron / hole
 * densities as the sums of QWRho5 before the boundary offset, normalisation
 * and transform (qwoptics.py:367-381, 948-1078).
 */
int psb_full_sources_f64(int nk, int nr, const double* d_kr, const double* d_r,
                         const double* d_window, double L, double dcv, double yw, double sgnw,
                         const double* d_level, double* d_out, void* stream);

/*
 * The many-body terms of the full-matrix step that mb.params switches on,
 * all FP64 and in the reference's summation order:
 *  - diag_dph:    k-dependent dephasing rates GamE, GamH replace gam_e, gam_h
 *                 in dpdt (CalcGammaE / CalcGammaH, dephasing.py:28-105,
 *                 540-625; SBEs.py:5225-5228);
 *  - offdiag_dph: OffDiagDephasing2 added to dpdt (dephasing.py:226-360,
 *                 713-760; widths gam_eh, gam_h for electrons and gam_e,
 *                 gam_h for holes, as SBEs.py:5229-5232 passes them);
 *  - ehs:         carrier-carrier in/out scattering rates MBCE / MBCH
 *                 (coulomb.py:957-1071, 1298-1326) and
 *  - phonon:      LO-phonon rates MBPE / MBPH (phonons.py:157-271),
 *                 applied to the new occupations before the neutrality
 *                 rescale (SBESolver._relaxation, SBEs.py:5248-5336,
 *                 5688-5695);
 *  - recomb:      spontaneous emission (SpontEmission, emission.py:94-199)
 *                 from the level the right-hand side reads, applied after
 *                 that relaxation as n_e *= exp(-Rsp n_h dt), then
 *                 n_h *= exp(-Rsp n_e dt) (SBEs.py:5335-5337; like the
 *                 reference, only when ehs or phonon is on);
 *  - dctrans:     the DC-field transport shift of X3 (Transport,
 *                 dcfield.py:1169-1247; SBEs.py:5698-5702): with lf the
 *                 full matrices, else their diagonals, each moved by dc_dk
 *                 in k as fft -> exp(-i Y dc_dk) -> ifft does, here as the
 *                 equivalent circular convolution.
 * Tables (made once per grid by the caller):
 *   maps   int32 [6][nk][nk]: k_p_q, k_m_q, k1p, k1p_m_q, k1, k1_m_q of
 *          InitializeDephasing (dephasing.py:471-538), 0-based, any value
 *          outside [0, nk) meaning "no partner";
 *   iq     int32 [nk]: round(|ky / dk|), the index Vxx2 reads (dephasing.py:362);
 *   xe, xh double [nk] (InitializeDephasing);
 *   C      double [3][(nk+1)^3]: Ceh, Cee, Chh of CalcMBArrays
 *          (coulomb.py:367-499), psb_mb_tables_f64;
 *   ph     double [4][nk][nk]: EP, EPT, HP, HPT of InitializePhonons
 *          (phonons.py:55-136), vscale its _Vscale;
 *   eps    double [nk]: eps(q) the step's V3 was screened with (null: 1);
 *   emis   double [2][n_hw]: HOmega and square of InitializeEmission
 *          (emission.py:35-92, CalcHOmega :220-256), dhw = HOmega[1] -
 *          HOmega[0], rho0_den = c0^3 pi^2 hbar^3 (rho0, :201-218);
 *   Y      double [nk]: the FFT wavenumbers of InitializeDC (GetKArray(nk,
 *          (nk - 1) dky), dcfield.py:39-69, 793).
 * Per step: dc_dk = -e0 (Edc + Re Ex[nq0]) / hbar * dt (dcfield.py:1240).
 * scratch: psb_full_mb_scratch_bytes(nk) bytes, caller-owned.
 */
typedef struct PsbFullMB {
  int32_t diag_dph, offdiag_dph, ehs, phonon;
  double gam_e, gam_h, gam_eh; /* 1/s */
  double vscale;               /* phonon coupling scale (J) */
  const int32_t* maps;
  const int32_t* iq;
  const double* xe;
  const double* xh;
  const double* C;
  const double* ph;
  const double* eps;
  void* scratch;
  int32_t recomb, dctrans;
  double dc_dk;                /* 1/m */
  double dhw;                  /* J */
  double rho0_den;             /* c0^3 pi^2 hbar^3 */
  int32_t n_hw, pad_;
  const double* emis;
  const double* Y;
} PsbFullMB;

int64_t psb_full_mb_scratch_bytes(int nk);
/* Ceh, Cee, Chh of CalcMBArrays into d_C ([3][(nk+1)^3] doubles, every entry
 * written): Gaussian delta, or Lorentzian when lorentz != 0 (mb.params
 * LorentzDelta); ge, gh in 1/s. */
int psb_mb_tables_f64(int nk, const double* d_Ee, const double* d_Eh, double ge, double gh,
                      double hbar, int lorentz, double* d_C, void* stream);
/* psb_full_step_f64 with the many-body terms of *mb (host struct holding
 * device pointers); mb == NULL is psb_full_step_f64. */
int psb_full_step_mb_f64(int nk, int nr, int nq0, const double* d_V3, const double* d_Ee,
                         const double* d_Eh, const double* d_fields,
                         const PsbFullParams* params, const PsbFullMB* mb, double* d_L1,
                         double* d_L2, double* d_L3, void* d_work, int64_t n_work_bytes,
                         void* stream);

/*
 * All wires of one grid in one step (rhoPJ.QuantumWire's loop over wires,
 * rhoPJ.py:311-348, each iteration one SBESolver.QWCalculator step): the
 * kernels of psb_full_step_mb_f64 with the wire as the grid's y index.
 *   d_tab     the grid's table block [9][nk] (V_eh, V_ee, V_hh, Ee, Eh,
 *             chi_e, chi_h, qe, qh), as in PsbTable
 *   screened  each wire's V3 = V / eps(q; n1D) from its own densities
 *             (L, dens_max as in PsbTable), made in the step; unscreened
 *             wires share the table's V
 *   d_fields  [nw][3][nr] complex wire-space fields
 *   d_wpar    [nw][4] doubles per wire: yw(w), (-1)^w, the DC shift dc_dk
 *             of that wire (PsbFullMB.dc_dk and .eps are not read), 0
 *   mb        NULL, or tables shared by the wires with scratch of
 *             nw * psb_full_mb_scratch_bytes(nk) bytes
 *   d_L1..L3  [nw][3][nk][nk] complex each
 *   d_work    psb_full_batch_work_bytes(nw, nk) bytes
 * A wire's result is the same bits as psb_full_step_mb_f64 on that wire
 * alone (with the V3 the one-wire screening gives).
 */
#define PSB_FULL_MAX_WIRES 65535
int64_t psb_full_batch_work_bytes(int nw, int nk);
int psb_full_step_batch_f64(int nw, int nk, int nr, int nq0, const double* d_tab, double L,
                            double dens_max, int screened, const double* d_fields,
                            const PsbFullParams* params, const double* d_wpar,
                            const PsbFullMB* mb, double* d_L1, double* d_L2, double* d_L3,
                            void* d_work, int64_t n_work_bytes, void* stream);
/* psb_full_sources_f64 of nw wires: d_levels [nw][3][nk][nk] complex, d_out
 * [nw][5][nr] complex, yw and (-1)^w of each wire from d_wpar [nw][4]. */
int psb_full_sources_batch_f64(int nw, int nk, int nr, const double* d_kr, const double* d_r,
                               const double* d_window, double L, double dcv,
                               const double* d_wpar, const double* d_levels, double* d_out,
                               void* stream);

/*
 * Host function (no device work): m complex signals z0 [m][n0] on grid
 * x0[n0] resampled onto x1[n1] by their cubic splines, out [m][n1] (0
 * outside [min x0, max x0]) -- rescale_1D_dpc with spline_dpc / seval_dpc
 * (spliner.py:153-188, 1287-1396), the resampling inside Prop2QW / QW2Prop
 * (qwoptics.py:673-812), with numpy's complex arithmetic (the bits of the
 * numpy restatement in pulsesuite_b200.wirespace).  Complex values are
 * interleaved (re, im) doubles.
 */
int psb_spline_rows_c128(const double* x0, int n0, const double* z0, int m, const double* x1,
                         int n1, double* out);

/* ---- split-precision tensor-core form (sm_100a tcgen05, kind::i8) --------- */
/*
 * The batched form of the same RK4 step: per group of wires sharing one k
 * grid, the exchange sums of all wires are one contraction
 *   D[k][(w,v)] = sum_k' V(|k-k'|) X[k'][(w,v)]
 * computed on the integer tensor cores: V and X are written as three
 * signed base-254 int8 digits each (V scaled by a power of two, X by a
 * power of two per column), the six digit products of weight <= 4 are
 * accumulated exactly in int32 and combined in FP64.  The O(Nk) right-hand
 * side is FP64, the stage point and RK accumulator FP32, the state y and the
 * P(t) sums FP64 (FP64 layout of the plain form).  Target accuracy:
 * normwise relative error <= 1e-6 in P(t) and <= 1e-5 in the state against
 * the FP64 form.  Requires PSB_TAB_EXCITONS | PSB_TAB_SHARED_V tables
 * without screening.
 */
#define PSB_SPLIT_WMAX 16
/* One CTA's work: 1..wgroup wires of one table (same k grid); wire slots
 * past nw are ignored.  wgroup is 4, 8 or 16 (wider groups make every MMA
 * wider at the same issue cost; 16 needs nk <= psb_split_max_nk(16)). */
typedef struct PsbSplitGroup {
  int32_t table;
  int32_t nw;
  int32_t wire[PSB_SPLIT_WMAX];
} PsbSplitGroup;

/*
 * Polls a bounded on-chip hand-off wait of the split kernel makes before it
 * gives up (0 restores the default, 2^26).  A wait that runs out makes its
 * CTA stop: it waits (bounded) for its MMAs in flight, frees its tensor
 * memory and reports PSB_ERR_TIMEOUT in the status of its wires; the call
 * and the context stay usable.  Applies to launches issued after the call
 * (process-wide); a small value makes the waits run out on purpose, which
 * is how the timeout path is tested.
 */
int psb_split_set_wait_limit(uint32_t spins);
/* Workspace bytes psb_rk4_split needs for n_state elements. */
int64_t psb_split_ws_bytes(int64_t n_state);
/* Dynamic shared memory (bytes) of one CTA for a grid of nk, wgroup 4, 8
 * or 16 (the layout psb_rk4_split picks for nkmax = nk). */
int psb_split_smem_bytes(int nk, int wgroup);
/* Largest nk a group of wgroup (4, 8 or 16) wires supports. */
int psb_split_max_nk(int wgroup);
/* Largest nk for which the stage state of a group stays resident in shared
 * memory for the whole call (faster; larger grids keep it in the workspace). */
int psb_split_max_nk_resident(int wgroup);
/*
 * nsteps RK4 steps of every group (one CTA each), same contract as
 * psb_rk4_f64 (state, t, steps, status, P(t) records) for the wires of
 * d_groups[0..ngroups).  wgroup (4, 8 or 16) is the group capacity compiled
 * for; nkmax the largest grid among the groups (<= psb_split_max_nk(wgroup)).
 * d_ws: caller-allocated workspace of psb_split_ws_bytes(n_state) bytes,
 * 32-byte aligned (stage state and RK accumulator per element).  On
 * PSB_ERR_TIMEOUT the state of the group's wires is unspecified.  Replaces,
 * like psb_rk4_f64, CalcH + dpdt/dCdt/dDdt (SBEs.py:669-935, 1850-2636)
 * integrated by rk4_dpc (libpulsesuite/integrator.py:143-167).
 */
int psb_rk4_split(const PsbTable* d_tables, int ntab, const double* d_tabdata, int64_t n_tabdata,
                  PsbWire* d_wires, int nw, const PsbSplitGroup* d_groups, int ngroups,
                  int wgroup, int nkmax, double* d_y, int64_t n_state, void* d_ws,
                  int64_t n_ws_bytes, int nsteps, double dt, double* d_P, int64_t n_P,
                  int p_stride, int p_cap, const PsbModel* model, void* stream);

/*
 * psb_rk4_split without a caller workspace, for callers that cannot
 * allocate device memory: code that runs where cudaMalloc is unavailable or
 * forbidden (inside another framework's memory pool or allocator hooks, or a
 * host that owns every allocation and hands this library only its inputs
 * and outputs).  No counterpart in the reference (its step allocates
 * through numpy); this is an addition of this library.
 *
 * The workspace lives in one static device array of
 * PSB_SPLIT_NOALLOC_SCRATCH_BYTES bytes that every GPU loading the library
 * holds until the process exits.  Limit: n_state <=
 * PSB_SPLIT_NOALLOC_MAX_STATE elements; larger batches get PSB_ERR_SIZE
 * (use psb_rk4_split with your own workspace).  Nothing is allocated:
 * no cudaMalloc, cudaFree or allocating library call.
 * - The first call on a device looks up the array's device address
 *   (cudaGetSymbolAddress) with that device current; make that first call
 *   before any stream capture.  The address is cached per device and looked
 *   up again when the calling context changes; resetting the device
 *   (cudaDeviceReset) between calls is not supported, since a new primary
 *   context may reuse the old handle and leave the cached address stale.
 * - All calls share the array, and it keeps what the last call wrote.  The
 *   kernel writes every workspace element before reading it, so nothing
 *   needs to start at zero.  Calls whose kernels overlap on the GPU (other
 *   streams, other host threads) race on the array: serialize them.
 * Other arguments and results as psb_rk4_split.
 */
#define PSB_SPLIT_NOALLOC_SCRATCH_BYTES (8 * 1024 * 1024)
#define PSB_SPLIT_NOALLOC_MAX_STATE ((PSB_SPLIT_NOALLOC_SCRATCH_BYTES - 32) / 64)
int psb_rk4_split_noalloc(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                          int64_t n_tabdata, PsbWire* d_wires, int nw,
                          const PsbSplitGroup* d_groups, int ngroups, int wgroup, int nkmax,
                          double* d_y, int64_t n_state, int nsteps, double dt, double* d_P,
                          int64_t n_P, int p_stride, int p_cap, const PsbModel* model,
                          void* stream);

/*
 * The split form with one Coulomb matrix per wire, for the tables
 * psb_rk4_split does not take:
 *  - screened tables (PSB_TAB_SCREENED): every stage divides V(q) by
 *    eps(q; n1D) of that wire's own stage densities, as psb_rk4_f64 does
 *    (CalcScreenedArrays, coulomb.py:1212-1230, Eps1D coulomb.py:1172-1193;
 *    eps in FP64, its logarithms in FP64 near q -> 0 where their argument
 *    is below 1/2 and as FP32 log1p of the exactly formed argument - 1
 *    elsewhere, ~3e-8 relative in eps);
 *  - distinct Veh, Vee, Vhh (tables without PSB_TAB_SHARED_V; the
 *    reference's CalcCoulombArrays physics, coulomb.py:502-577): p uses Veh,
 *    ne Vee, nh Vhh.
 * Same digit arithmetic, accuracy target, state layout, workspace
 * (psb_split_ws_bytes) and per-wire results as psb_rk4_split; the CTA of a
 * group contracts its wires one after another, so the tensor-core work per
 * wire does not shrink with the group size.  wgroup: wires per group, 1 ..
 * psb_split_wire_max_group(nkmax, tab_flags) (<= PSB_SPLIT_WMAX); nkmax <=
 * 1024 (512 for distinct matrices).  tab_flags: the PSB_TAB_* flags every
 * group's table has (PSB_TAB_EXCITONS required; PSB_TAB_SCREENED and
 * PSB_TAB_SHARED_V as the tables have them).  Replaces, like psb_rk4_f64,
 * CalcH + dpdt/dCdt/dDdt (SBEs.py:669-935, 1850-2636) integrated by rk4_dpc
 * (libpulsesuite/integrator.py:143-167).
 */
int psb_rk4_split_wire(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                       int64_t n_tabdata, PsbWire* d_wires, int nw, const PsbSplitGroup* d_groups,
                       int ngroups, int wgroup, int nkmax, int tab_flags, double* d_y,
                       int64_t n_state, void* d_ws, int64_t n_ws_bytes, int nsteps, double dt,
                       double* d_P, int64_t n_P, int p_stride, int p_cap, const PsbModel* model,
                       void* stream);
/* Largest group (wires per CTA) psb_rk4_split_wire supports for a grid of nk
 * with these table flags; 0 when the grid does not fit. */
int psb_split_wire_max_group(int nk, int tab_flags);
/* Dynamic shared memory (bytes) of one psb_rk4_split_wire CTA. */
int psb_split_wire_smem_bytes(int nk, int wgroup, int tab_flags);

/* ---- measurement --------------------------------------------------------- */
/*
 * FP64 FMA throughput of the current device: runs an in-register FMA loop
 * (iters per thread) on blocks x 256 threads and returns the elapsed device
 * time in *ms (CUDA events on `stream`).  Flops = 2 * 8 * iters * blocks * 256.
 * Used as the measured FP64 roofline peak.
 */
int psb_probe_fp64_fma(int blocks, int iters, double* d_sink, float* ms, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PULSESUITE_B200_H */
