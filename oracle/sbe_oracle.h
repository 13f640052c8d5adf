/*
 * sbe_oracle.h -- CPU restatement of the reference quantum-wire SBE path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product path: only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * --impl reference legs of bench.py may load it.  The product
 * (pulsesuite_b200) never calls it and has no CPU fallback.
 *
 * It restates, in the diagonal (p_k, n_e,k, n_h,k) form, the reference's
 *   - CalcH exchange sums           pulsesuite/PSTD3D/SBEs.py:819-935
 *   - dpdt / dCdt / dDdt            pulsesuite/PSTD3D/SBEs.py:1952-1975, 2319-2337, 2617-2636
 *   - leapfrog + neutrality step    pulsesuite/PSTD3D/SBEs.py:5681-5718
 *   - classical RK4 stage order     pulsesuite/libpulsesuite/integrator.py:143-157
 *   - Coulomb V(q) via Vint/_K03    pulsesuite/PSTD3D/coulomb.py:38-104, 502-577
 *   - 1D susceptibility + screening pulsesuite/PSTD3D/coulomb.py:580-630, 1172-1230
 *   - K0 of cik01 (Zhang & Jin)     pulsesuite/PSTD3D/usefulsubs.py:1669-1820
 *   - P(t) diagonal reduction       pulsesuite/PSTD3D/qwoptics.py:815-946
 * Parity of this restatement is pinned by the golden vectors in tests/golden
 * (generated by importing the reference itself; see make_golden.py there).
 *
 * The structs are the same layout as the product's C-ABI structs
 * (include/pulsesuite_b200.h) so the same host-side tables drive both.
 */
#ifndef PSB_SBE_ORACLE_H
#define PSB_SBE_ORACLE_H
#include <stdint.h>
#include "../include/pulsesuite_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

double orc_k03_crude(double x);
double orc_k0(double x);
double orc_i0(double x);
void orc_vint_table(const double* qy, int nq, const double* y, int ny, double alpha1,
                    double alpha2, double delta0, double prefactor, double* out);
void orc_k0_table(const double* q, int nq, double radius, double prefactor, double* out);
void orc_chi1d_table(const double* q, int nq, double alpha, double delta0, double mass,
                     double scale, double* out);

/* RHS of all wires at per-wire time t[w] (or the wire's own t when t == NULL). */
int orc_rhs(const PsbTable* tables, int ntab, const double* tabdata, const PsbWire* wires,
            int nw, const double* t, const double* y, double* dy, const PsbModel* model);

/* nsteps classical RK4 steps on every wire; y is [p_re, p_im, ne, nh] per k (4 doubles). */
int orc_rk4(const PsbTable* tables, int ntab, const double* tabdata, PsbWire* wires, int nw,
            double* y, int nsteps, double dt, double* P, int p_stride, int p_cap,
            const PsbModel* model, int nthreads);

/* nsteps reference leapfrog steps; y1 = older (averaged) level, y2 = newer level. */
int orc_leapfrog(const PsbTable* tables, int ntab, const double* tabdata, PsbWire* wires,
                 int nw, double* y1, double* y2, const double* field, int field_stride,
                 int nsteps, double dt, double* P, int p_stride, int p_cap,
                 const PsbModel* model, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
