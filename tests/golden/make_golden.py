"""Generate the golden vectors of tests/golden by running the reference itself.

Run in a container that holds the reference source (default
/root/reference/src, override with PULSESUITE_REF_SRC):

    python tests/golden/make_golden.py            # small cases (a few minutes)
    python tests/golden/make_golden.py --full-c0  # + the 4000-step Nk=128 RK4 run (~10 min)
    python tests/golden/make_golden.py --only manybody,transport   # selected groups

The reference does not import cleanly in this image, so three shims are set
up first, exactly the minimum needed:
  * ``pyfftw`` is absent: a package mapping ``pyfftw.interfaces.numpy_fft`` to
    ``numpy.fft`` with a no-op ``cache.enable()`` (FFTs are off the diagonal
    SBE path);
  * ``pulsesuite.PSTD3D.benchmark`` does not exist in the reference but the
    legacy path imports it: a stub module;
  * numba 0.65 mis-compiles the parallel ``_CalcH_jit`` (it drops the exchange
    sums); it is replaced by the serial compile of its own Python source,
    checked against the reference's ``_CalcH_fallback`` before use.
Numba-CUDA / CuPy are disabled (PULSESUITE_USE_CUDA=0): the goldens are the
reference's Numba CPU path.

Cases (all stored as .npz next to this script):
  tables_*.npz    reference Coulomb V(q), chi1D, qe/qh, Eps1D, screened VC
  rhs_*.npz       CalcH + dpdt/dCdt/dDdt on random diagonal states
  rk4_*.npz       reference RHS integrated by libpulsesuite.integrator.rk4_dpc
                  (rotating-frame drive, the benchmark configurations' physics)
  leapfrog_*.npz  SBESolver._sbe_calculator, the reference's own driver
  solver_*.npz    the SBESolver API with LF on: source terms, levels, backup files
  qwcalc_*.npz    QWCalculator driven by propagation-space fields (full-matrix state),
                  plain, with DiagDph/OffDiagDph/EHs/Phonon (qwcalc_manybody_*), and
                  with Recomb and DCTrans in a DC field, LF on and off (qwcalc_mb_dc_*)
  manybody_units_nk32.npz  the many-body functions (CalcGammaE/H, OffDiagDephasing2,
                  MBCE/MBCH, MBPE/MBPH, SpontEmission) on random levels, and the
                  emission / DC host tables of the reference's modules
"""

import argparse
import os
import sys
import tempfile
import time
import types

os.environ["PULSESUITE_USE_CUDA"] = "0"
_TMP = tempfile.mkdtemp(prefix="psb_golden_")
os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(_TMP, "numba_cache"))

import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from pulsesuite_b200 import grid as pgrid  # noqa: E402

REF_SRC = os.environ.get("PULSESUITE_REF_SRC", "/root/reference/src")


def import_reference():
    shim = os.path.join(_TMP, "shim")
    os.makedirs(os.path.join(shim, "pyfftw", "interfaces"), exist_ok=True)
    with open(os.path.join(shim, "pyfftw", "__init__.py"), "w") as f:
        f.write("from . import interfaces\n")
    with open(os.path.join(shim, "pyfftw", "interfaces", "__init__.py"), "w") as f:
        f.write("import numpy.fft as numpy_fft\n\n\nclass cache:\n"
                "    enable = staticmethod(lambda: None)\n")
    sys.path.insert(0, shim)
    sys.path.insert(0, REF_SRC)
    bench = types.ModuleType("pulsesuite.PSTD3D.benchmark")
    bench.profile_start = time.perf_counter
    bench.profile_record = lambda name, t0: None
    sys.modules["pulsesuite.PSTD3D.benchmark"] = bench

    import numba

    from pulsesuite.libpulsesuite import integrator
    from pulsesuite.PSTD3D import SBEs, coulomb, qwoptics, usefulsubs

    SBEs._CalcH_jit = numba.njit(parallel=False)(SBEs._CalcH_jit.py_func)
    _selftest_calch(SBEs)
    return types.SimpleNamespace(SBEs=SBEs, coulomb=coulomb, usefulsubs=usefulsubs,
                                 qwoptics=qwoptics, integrator=integrator)


def _selftest_calch(SBEs):
    rng = np.random.default_rng(7)
    nk = 16
    for lf in (False, True):
        args = [rng.standard_normal((nk, nk)) + 1j * rng.standard_normal((nk, nk))
                for _ in range(6)]
        VC = rng.standard_normal((nk, nk, 3))
        Ee, Eh = rng.standard_normal(nk), rng.standard_normal(nk)
        outs = []
        for fn in (SBEs._CalcH_jit, SBEs._CalcH_fallback):
            H = [np.zeros((nk, nk), complex) for _ in range(3)]
            fn(*args, VC, *H, nk, Ee, Eh, 0.3, True, lf, False)
            outs.append(H)
        for a, b in zip(*outs):
            if np.max(np.abs(a - b)) > 1e-12 * max(1.0, np.max(np.abs(b))):
                raise RuntimeError("patched _CalcH_jit disagrees with _CalcH_fallback")


def kkp_of(kr, dkr, NQ0):
    nk = kr.size
    kkp = np.zeros((nk, nk), dtype=int)
    for k in range(nk):
        for kp in range(nk):
            kkp[k, kp] = int(np.round((kr[k] - kr[kp]) / dkr)) + NQ0
    return kkp


def reference_coulomb(R, g):
    """Reference Coulomb arrays of one reference grid, column [:, 0]."""
    c = R.coulomb
    nr = g.y.size
    Qr = R.SBEs.GetKArray(nr, 2 * g.L)
    Qr = np.roll(Qr, nr // 2)
    Qr[0] = -Qr[0]
    NQ0 = R.usefulsubs.GetArray0Index(Qr)
    kkp = kkp_of(g.kr, g.dk, NQ0)
    Veh0, Vee0, Vhh0 = c.CalcCoulombArrays(g.y, g.kr, g.epsr, g.alphae, g.alphah, g.L,
                                           g.delta0, Qr, kkp)
    qe, qh = c.MakeQs(g.kr, g.alphae, g.alphah)
    Chi1De, Chi1Dh = c.CalcChi1D(g.kr, g.alphae, g.alphah, g.delta0, g.epsr, g.me, g.mh, qe, qh)
    inst = object.__new__(c.CoulombModule)
    inst.qe, inst.qh, inst.Chi1De, inst.Chi1Dh = qe, qh, Chi1De, Chi1Dh
    inst.Veh0, inst.Vee0, inst.Vhh0 = Veh0, Vee0, Vhh0
    return inst, Qr, NQ0, kkp


def reference_k0_vc(R, g):
    """VC[:, :, n] whose [q, 0] column is the synthetic wire's V(q) (K0 via
    the reference's own K03 = cik01)."""
    nk = g.nk
    v = np.array([0.0] + [g.vprefactor * R.usefulsubs.K03(abs(g.kr[q] - g.kr[0]) * g.radius)
                          for q in range(1, nk)])
    VC = np.zeros((nk, nk, 3))
    for n in range(3):
        VC[:, 0, n] = v
    return VC, v


def ref_rhs(R, nk, Ee, Eh, gap, VC, M, p, ne, nh, gamma):
    """Reference diagonal RHS: patched CalcH + dpdt/dCdt/dDdt."""
    S = R.SBEs
    Meh = np.diag(np.full(nk, M, dtype=complex))
    C = np.diag(ne.astype(complex))
    D = np.diag(nh.astype(complex))
    P = np.diag(p.astype(complex))
    Heh, Hee, Hhh = (np.zeros((nk, nk), complex) for _ in range(3))
    Z = np.zeros((nk, nk), complex)
    S._CalcH_jit(Meh, Z, Z, C, D, P, VC, Heh, Hee, Hhh, nk, Ee, Eh, gap, True, False, False)
    G = np.full(nk, gamma / 2.0)
    hb = S.hbar
    dp = S._dpdt_jit(C, D, P, Heh, Hee, Hhh, G, G, Z, 1j, hb)
    dC = S._dCdt_jit(C, D, P, Heh, Hee, Hhh, G, G, Z, 1j, hb)
    dD = S._dDdt_jit(C, D, P, Heh, Hee, Hhh, G, G, Z, 1j, hb)
    off = max(np.max(np.abs(dp - np.diag(np.diag(dp)))), np.max(np.abs(dC - np.diag(np.diag(dC)))))
    return np.diag(dp).copy(), np.diag(dC).copy(), np.diag(dD).copy(), off


def grid_meta(g):
    return dict(nk=g.nk, dk=g.dk, kr=g.kr, L=g.L, me=g.me, mh=g.mh, epsr=g.epsr,
                delta0=g.delta0, alphae=g.alphae, alphah=g.alphah, radius=g.radius,
                gap=g.gap, dcv=g.dcv, ehint=g.ehint, area=g.area)


# ----------------------------------------------------------------------------
def make_tables(R, out):
    rng = np.random.default_rng(11)
    for L in (2.85e-8, 1e-7):
        g = pgrid.reference_grid(L=L)
        inst, Qr, NQ0, kkp = reference_coulomb(R, g)
        ne = rng.uniform(0, 0.3, g.nk)
        nh = rng.uniform(0, 0.3, g.nk)
        VC = np.zeros((g.nk, g.nk, 3))
        E1D = np.zeros((g.nk, g.nk))
        inst.CalcScreenedArrays(True, g.L, ne.astype(complex), nh.astype(complex), VC, E1D)
        dens = [1e5, 1e7, 0.5 * g.dens_max * np.pi]
        eps = np.array([inst.Eps1D(d)[:, 0] for d in dens])
        np.savez_compressed(
            os.path.join(out, f"tables_ref_nk{g.nk}.npz"), **grid_meta(g), y=g.y, Qr=Qr,
            NQ0=NQ0, Veh=inst.Veh0[:, 0], Vee=inst.Vee0[:, 0], Vhh=inst.Vhh0[:, 0],
            chie=inst.Chi1De[:, 0], chih=inst.Chi1Dh[:, 0], qe=inst.qe[:, 0], qh=inst.qh[:, 0],
            dens=np.array(dens), eps=eps, ne=ne, nh=nh, VCs=VC[:, 0, :].copy(),
            E1D=E1D[:, 0].copy())
        print(f"tables_ref_nk{g.nk}: done")
    # K0 of the reference (cik01) at a spread of arguments
    xs = np.concatenate([np.geomspace(1e-6, 1.0, 40), np.linspace(1.0, 99.0, 120)])
    k0 = np.array([R.usefulsubs.K03(x) for x in xs])
    k03j = np.array([R.coulomb._K03_jit(x) for x in xs])
    np.savez_compressed(os.path.join(out, "k0_ref.npz"), x=xs, K03=k0, K03_jit=k03j)
    print("k0_ref: done")


def make_rhs(R, out):
    rng = np.random.default_rng(12)
    cases = []
    for nk in (16, 32, 64, 128):
        g = pgrid.wire_grid(nk)
        VC, v = reference_k0_vc(R, g)
        cases.append(("k0", g, VC, v, None))
    gr = pgrid.reference_grid(L=2.85e-8)
    inst, *_ = reference_coulomb(R, gr)
    cases.append(("ref", gr, None, None, inst))
    for kind, g, VC, v, inst in cases:
        nk = g.nk
        p = 0.05 * (rng.standard_normal(nk) + 1j * rng.standard_normal(nk))
        ne = rng.uniform(0, 0.2, nk)
        nh = rng.uniform(0, 0.2, nk)
        M = complex(rng.standard_normal(), rng.standard_normal()) * 1e-21
        gap = float(rng.uniform(-0.05, 0.05)) * 1.602176634e-19
        gamma = 1.0 / 100e-15
        if kind == "ref":
            VC = np.zeros((nk, nk, 3))
            E1D = np.zeros((nk, nk))
            inst.CalcScreenedArrays(False, g.L, ne.astype(complex), nh.astype(complex), VC, E1D)
            VCs = np.zeros((nk, nk, 3))
            inst.CalcScreenedArrays(True, g.L, ne.astype(complex), nh.astype(complex), VCs, E1D)
            dps, dCs, dDs, offs = ref_rhs(R, nk, g.Ee, g.Eh, gap, VCs, M, p, ne, nh, gamma)
        dp, dC, dD, off = ref_rhs(R, nk, g.Ee, g.Eh, gap, VC, M, p, ne, nh, gamma)
        extra = {}
        if kind == "ref":
            extra = dict(dp_s=dps, dC_s=dCs, dD_s=dDs, VCs=VCs[:, 0, :].copy(),
                         chie=inst.Chi1De[:, 0], chih=inst.Chi1Dh[:, 0])
        np.savez_compressed(
            os.path.join(out, f"rhs_{kind}_nk{nk}.npz"), **grid_meta(g), VC=VC[:, 0, :].copy(),
            p=p, ne=ne, nh=nh, M=M, gap_eff=gap, gamma=gamma, dp=dp, dC=dC, dD=dD,
            offdiag=off, **extra)
        print(f"rhs_{kind}_nk{nk}: off-diagonal |d/dt| = {off:.1e}")


def rwa_case(nk, nsteps, theta=0.5 * np.pi, fwhm=50e-15, T2=100e-15, det_meV=0.0,
             dt=1e-15, screened=False):
    g = pgrid.wire_grid(nk)
    mscale = g.ehint * g.dcv / 2.0
    amp = pgrid.gaussian_amplitude(theta, fwhm, mscale)
    return dict(g=g, nsteps=nsteps, dt=dt, amp=amp, t0=3.0 * fwhm, fwhm=fwhm, mscale=mscale,
                gamma=1.0 / T2, gap_eff=-det_meV * 1e-3 * 1.602176634e-19, screened=screened)


def make_rk4(R, out, name, case):
    """Oracle A: reference RHS kernels + reference rk4_dpc (the diagonal-drive harness)."""
    g = case["g"]
    nk = g.nk
    S = R.SBEs
    Ee, Eh = g.Ee, g.Eh
    VC0, v = reference_k0_vc(R, g)
    inst = None
    if case["screened"]:
        qe, qh = R.coulomb.MakeQs(g.kr, g.alphae, g.alphah)
        Chi1De, Chi1Dh = R.coulomb.CalcChi1D(g.kr, g.alphae, g.alphah, g.delta0, g.epsr, g.me,
                                             g.mh, qe, qh)
        inst = object.__new__(R.coulomb.CoulombModule)
        inst.qe, inst.qh, inst.Chi1De, inst.Chi1Dh = qe, qh, Chi1De, Chi1Dh
        inst.Veh0 = VC0[:, :, 0]
        inst.Vee0 = VC0[:, :, 1]
        inst.Vhh0 = VC0[:, :, 2]
    amp, t0, fwhm, mscale = case["amp"], case["t0"], case["fwhm"], case["mscale"]
    gamma, gap = case["gamma"], case["gap_eff"]

    def D(t, y):
        p, ne, nh = y[:nk], y[nk:2 * nk].real, y[2 * nk:].real
        E = amp * np.exp(-4.0 * np.log(2.0) * ((t - t0) / fwhm) ** 2)
        M = -mscale * E
        VC = VC0
        if inst is not None:
            VC = np.zeros((nk, nk, 3))
            E1D = np.zeros((nk, nk))
            inst.CalcScreenedArrays(True, g.L, ne.astype(complex), nh.astype(complex), VC, E1D)
        dp, dC, dD, _ = ref_rhs(R, nk, Ee, Eh, gap, VC, M, p, ne, nh, gamma)
        return np.concatenate([dp, dC, dD])

    y = np.zeros(3 * nk, dtype=complex)
    t = 0.0
    P = np.zeros(case["nsteps"], dtype=complex)
    pscale = g.pscale
    t_start = time.time()
    for n in range(case["nsteps"]):
        dydt = D(t, y)
        t = R.integrator.rk4_dpc(y, dydt, t, case["dt"], D)
        P[n] = pscale * np.sum(y[:nk])
    el = time.time() - t_start
    np.savez_compressed(os.path.join(out, f"{name}.npz"), **grid_meta(g), V=v, amp=amp, t0=t0,
                        fwhm=fwhm, mscale=mscale, gamma=gamma, gap_eff=gap, dt=case["dt"],
                        nsteps=case["nsteps"], screened=case["screened"], P=P, p=y[:nk],
                        ne=y[nk:2 * nk].real, nh=y[2 * nk:].real, imag_n=np.max(np.abs(
                            y[nk:].imag)), pscale=pscale, seconds=el)
    print(f"{name}: {case['nsteps']} steps in {el:.1f} s, max|P| = {np.max(np.abs(P)):.3e}, "
          f"max ne = {np.max(y[nk:2 * nk].real):.3e}")


QW_PARAMS = """{L}     # L
5e-9       # Delta0
1.5        # gap
0.07       # me
0.45       # mh
100e-3     # HO
{gam}      # gam_e
{gam}      # gam_h
{gam}      # gam_eh
9.1        # epsr
36e-3      # Oph
3e-3       # Gph
0.0        # Edc
1000000    # jmax
20000      # ntmax
"""

MB_PARAMS = "1\n1\n0\n{scr}\n0\n0\n0\n0\n0\n0\n0\n0\n0\n0\n0\n"


def make_leapfrog(R, out, name, L=2.85e-8, screened=False, nsteps=3000, dt=10e-18):
    """Oracle B: the reference's own SBESolver driver with a diagonal drive."""
    cwd = os.getcwd()
    run = tempfile.mkdtemp(prefix="lf_", dir=_TMP)
    os.makedirs(os.path.join(run, "params"))
    gam = 5e12
    with open(os.path.join(run, "params", "qw.params"), "w") as f:
        f.write(QW_PARAMS.format(L=L, gam=gam))
    with open(os.path.join(run, "params", "mb.params"), "w") as f:
        f.write(MB_PARAMS.format(scr=1 if screened else 0))
    os.chdir(run)
    try:
        rr = np.linspace(-5e-7, 5e-7, 64)
        qrr = R.SBEs.GetKArray(64, 64 * (rr[1] - rr[0]))
        s = R.SBEs.SBESolver(qrr, rr, 0.0, 1e7, 800e-9, 1, True)
        nk, nr = s.Nk, s.Nr
        y1 = np.stack([np.diag(s.YY2[:, :, 0]).real, np.diag(s.YY2[:, :, 0]).imag,
                       np.diag(s.CC2[:, :, 0]).real, np.diag(s.DD2[:, :, 0]).real], 1)
        y2 = np.stack([np.diag(s.YY3[:, :, 0]).real, np.diag(s.YY3[:, :, 0]).imag,
                       np.diag(s.CC3[:, :, 0]).real, np.diag(s.DD3[:, :, 0]).real], 1)
        E0, tw, tp = 2e8, 4e-15, 12e-15
        wl = (s.gap + 0.05 * 1.602176634e-19) / R.SBEs.hbar
        field = np.zeros(nsteps, dtype=complex)
        P = np.zeros(nsteps, dtype=complex)
        pscale = 2.0 * s.ehint / s.area / s.L * s.dcv
        Px, Py, Pz = (np.zeros(nr, complex) for _ in range(3))
        Re_, Rh_ = np.zeros(nr, complex), np.zeros(nr, complex)
        t_start = time.time()
        for n in range(nsteps):
            t = n * dt
            E = E0 * np.exp(-(((t - tp) / tw) ** 2)) * np.cos(wl * (t - tp))
            field[n] = E
            Ex = np.zeros(nr, complex)
            Ey = np.zeros(nr, complex)
            Ez = np.zeros(nr, complex)
            Vr = np.zeros(nr, complex)
            Ey[s.NQ0] = E
            s._sbe_calculator(Ex, Ey, Ez, Vr, dt, Px, Py, Pz, Re_, Rh_, False, 1)
            P[n] = pscale * np.sum(np.diag(s.YY3[:, :, 0]))
        el = time.time() - t_start
        Py_space = Py.copy()
        R.usefulsubs.iFFTG(Py_space)
        off = np.max(np.abs(s.YY3[:, :, 0] - np.diag(np.diag(s.YY3[:, :, 0]))))
        z1 = np.stack([np.diag(s.YY2[:, :, 0]).real, np.diag(s.YY2[:, :, 0]).imag,
                       np.diag(s.CC2[:, :, 0]).real, np.diag(s.DD2[:, :, 0]).real], 1)
        z2 = np.stack([np.diag(s.YY3[:, :, 0]).real, np.diag(s.YY3[:, :, 0]).imag,
                       np.diag(s.CC3[:, :, 0]).real, np.diag(s.DD3[:, :, 0]).real], 1)
        g = pgrid.reference_grid(L=L)
        assert g.nk == nk and np.array_equal(g.kr, s.kr)
        VCt = np.zeros((nk, nk, 3))
        E1Dt = np.zeros((nk, nk))
        R.coulomb.CalcScreenedArrays(False, s.L, np.zeros(nk, complex), np.zeros(nk, complex),
                                     VCt, E1Dt)
        chie = R.coulomb._instance.Chi1De[:, 0].copy()
        chih = R.coulomb._instance.Chi1Dh[:, 0].copy()
        np.savez_compressed(
            os.path.join(out, f"{name}.npz"), **grid_meta(g), y=g.y, gam=gam, screened=screened,
            dt=dt, nsteps=nsteps, field=field, y1_init=y1, y2_init=y2, y1=z1, y2=z2, P=P,
            pscale=pscale, mscale=s.ehint * s.dcv, Py_last=Py.copy(), Py_space=Py_space,
            r=s.r.copy(), NQ0=s.NQ0,
            Veh=VCt[:, 0, 0], Vee=VCt[:, 0, 1], Vhh=VCt[:, 0, 2], chie=chie, chih=chih,
            offdiag=off, seconds=el)
        print(f"{name}: Nk={nk} {nsteps} steps in {el:.1f} s, off-diag |p| = {off:.1e}, "
              f"max|P| = {np.max(np.abs(P)):.3e}, max ne = {np.max(z2[:, 2]):.3e}")
    finally:
        os.chdir(cwd)


MB_PARAMS_LF = "1\n1\n0\n0\n0\n0\n1\n0\n0\n0\n0\n0\n0\n0\n0\n"


def make_solver_api(R, out, name="solver_lf_nk32", L=2.85e-8, nsteps=300, dt=10e-18):
    """The reference's SBESolver as a caller uses it, with LF on (so the
    charge densities Re, Rh of QWRho5 are computed): the initial levels, the
    last step's source terms Px, Py, Pz, Re, Rh (q space), the final levels,
    and the text of the backup files write_sbes_data writes at the end."""
    cwd = os.getcwd()
    run = tempfile.mkdtemp(prefix="api_", dir=_TMP)
    os.makedirs(os.path.join(run, "params"))
    gam = 5e12
    with open(os.path.join(run, "params", "qw.params"), "w") as f:
        f.write(QW_PARAMS.format(L=L, gam=gam))
    with open(os.path.join(run, "params", "mb.params"), "w") as f:
        f.write(MB_PARAMS_LF)
    os.chdir(run)
    try:
        rr = np.linspace(-5e-7, 5e-7, 64)
        qrr = R.SBEs.GetKArray(64, 64 * (rr[1] - rr[0]))
        s = R.SBEs.SBESolver(qrr, rr, 0.0, 1e7, 800e-9, 1, True)
        nk, nr = s.Nk, s.Nr

        def levels():
            return np.stack([np.stack([np.diag(a[:, :, 0]) for a in
                                       (s.YY1, s.YY2, s.YY3)]),
                             np.stack([np.diag(a[:, :, 0]) for a in (s.CC1, s.CC2, s.CC3)]),
                             np.stack([np.diag(a[:, :, 0]) for a in (s.DD1, s.DD2, s.DD3)])])

        init = levels()
        E0, tw, tp = 2e8, 4e-15, 1.5e-15
        wl = (s.gap + 0.05 * 1.602176634e-19) / R.SBEs.hbar
        field = np.zeros(nsteps, dtype=complex)
        srcs = [np.zeros(nr, complex) for _ in range(5)]
        for n in range(nsteps):
            t = n * dt
            E = E0 * np.exp(-(((t - tp) / tw) ** 2)) * np.cos(wl * (t - tp))
            field[n] = E
            Ex, Ey, Ez, Vr = (np.zeros(nr, complex) for _ in range(4))
            Ey[s.NQ0] = E
            s._sbe_calculator(Ex, Ey, Ez, Vr, dt, *srcs, False, 1)
        s.write_sbes_data(7)
        texts = {}
        for key in ("CC1", "CC2", "CC3", "DD1", "DD2", "DD3", "YY1", "YY2", "YY3"):
            with open(os.path.join("dataQW", "backup", f"{key}.7.dat")) as f:
                texts[key] = np.array(f.read())
        np.savez_compressed(os.path.join(out, f"{name}.npz"), nk=nk, nr=nr, NQ0=s.NQ0, L=L,
                            gam=gam, dt=dt, nsteps=nsteps, field=field, init=init,
                            final=levels(), Px=srcs[0], Py=srcs[1], Pz=srcs[2], Re=srcs[3],
                            Rh=srcs[4], r=s.r.copy(), Qr=s.Qr.copy(), kr=s.kr.copy(),
                            chiw=s.chiw, qc=s.qc, area=s.area,
                            **{f"backup_{k}": v for k, v in texts.items()})
        print(f"{name}: Nk={nk}, {nsteps} steps, max|Re| = {np.max(np.abs(srcs[3])):.3e}")
    finally:
        os.chdir(cwd)


MB_PARAMS_FULL = "1\n1\n0\n{scr}\n0\n0\n1\n0\n0\n0\n0\n0\n0\n0\n0\n"


def with_edc(params, edc):
    """qw.params text with the DC field line set to edc (V/m)."""
    return params.replace("0.0        # Edc", f"{edc!r}        # Edc")


def make_qwcalculator(R, out, name, L=2.85e-8, screened=True, nsteps=200, dt=10e-18, mb=None,
                      edc=0.0):
    """The reference's QWCalculator as its PSTD caller drives it (rhoPJ.py:311-348):
    propagation-space fields along the wire axis (a Gaussian profile, so the
    windowed wire field has every q component and the state is full-matrix),
    LF on.  Stored: the fields, every step's Pxx/Pyy/Pzz/Rho, and the final
    full Nk x Nk levels."""
    cwd = os.getcwd()
    run = tempfile.mkdtemp(prefix="qwc_", dir=_TMP)
    os.makedirs(os.path.join(run, "params"))
    gam = 5e12
    with open(os.path.join(run, "params", "qw.params"), "w") as f:
        f.write(with_edc(QW_PARAMS.format(L=L, gam=gam), edc))
    with open(os.path.join(run, "params", "mb.params"), "w") as f:
        f.write(mb if mb is not None else MB_PARAMS_FULL.format(scr=1 if screened else 0))
    os.chdir(run)
    try:
        nrr = 64
        rr = np.linspace(-5e-8, 5e-8, nrr)
        qrr = R.SBEs.GetKArray(nrr, nrr * (rr[1] - rr[0]))
        s = R.SBEs.SBESolver(qrr, rr, 0.0, 1e7, 800e-9, 2, True)
        nk = s.Nk
        E0, tw, tp = 2e8, 1.0e-15, 1.0e-15
        wl = (s.gap + 0.05 * 1.602176634e-19) / R.SBEs.hbar
        prof = np.exp(-((rr / 3e-8) ** 2))
        outs = {k: np.zeros((nsteps, 2, nrr), complex) for k in ("Pxx", "Pyy", "Pzz", "Rho")}
        env = np.zeros(nsteps)
        t_start = time.time()
        for n in range(nsteps):
            t = n * dt
            E = E0 * np.exp(-(((t - tp) / tw) ** 2)) * np.cos(wl * (t - tp))
            env[n] = E
            for w in (1, 2):
                Exx = (0.3 * E * prof * (rr / 3e-8)).astype(complex)
                Eyy = (E * prof).astype(complex)
                Ezz = (0.2 * E * prof).astype(complex)
                Vrr = np.zeros(nrr, complex)
                o = [np.zeros(nrr, complex) for _ in range(4)]
                DoQWP, DoQWDl = [False], [False]
                s.QWCalculator(Exx, Eyy, Ezz, Vrr, rr, qrr, dt, w, *o, DoQWP, DoQWDl)
                for k, v in zip(("Pxx", "Pyy", "Pzz", "Rho"), o):
                    outs[k][n, w - 1] = v
        el = time.time() - t_start
        lv = {f"{a}{i}": getattr(s, f"{a}{i}").copy() for a in ("YY", "CC", "DD") for i in (1, 2, 3)}
        np.savez_compressed(os.path.join(out, f"{name}.npz"), nk=nk, nr=s.Nr, L=L, gam=gam,
                            dt=dt, nsteps=nsteps, rr=rr, prof=prof, env=env, edc=edc,
                            screened=screened, seconds=el, **outs, **lv)
        print(f"{name}: Nk={nk}, {nsteps} steps x 2 wires in {el:.1f} s, "
              f"max|Pyy| = {np.max(np.abs(outs['Pyy'])):.3e}, "
              f"offdiag |p| = {np.max(np.abs(lv['YY3'] - np.einsum('iiw->iw', lv['YY3'])[None]*0)):.3e}")
    finally:
        os.chdir(cwd)


MB_PARAMS_MB = ("1\n1\n{ehs}\n{scr}\n{ph}\n{dc}\n{lf}\n0\n{dd}\n{od}\n{rc}\n0\n0\n0\n{lor}\n")


def mb_params(ehs=1, scr=0, ph=1, dc=0, lf=1, dd=1, od=1, rc=0, lor=0):
    """mb.params text: Optics, Excitons on; the many-body flags as given."""
    return MB_PARAMS_MB.format(ehs=ehs, scr=scr, ph=ph, dc=dc, lf=lf, dd=dd, od=od, rc=rc, lor=lor)


def _run_dir(prefix, L, gam, mb):
    run = tempfile.mkdtemp(prefix=prefix, dir=_TMP)
    os.makedirs(os.path.join(run, "params"))
    with open(os.path.join(run, "params", "qw.params"), "w") as f:
        f.write(QW_PARAMS.format(L=L, gam=gam))
    with open(os.path.join(run, "params", "mb.params"), "w") as f:
        f.write(mb)
    return run


def make_manybody_units(R, out, L=2.85e-8, gam=5e12):
    """The reference's many-body functions (CalcGammaE/H, CalcOffDiagDeph_E2
    /H2, OffDiagDephasing2, MBCE/MBCH, MBPE/MBPH, SpontEmission) on random
    levels of its own grid, unscreened, Lorentzian delta: the inputs one
    full-matrix step reads (X1 = level 2, X2 = level 3 of the GPU state,
    dt = 0) and its outputs."""
    from pulsesuite.PSTD3D import coulomb as C
    from pulsesuite.PSTD3D import dephasing as D
    from pulsesuite.PSTD3D import emission as EM
    from pulsesuite.PSTD3D import phonons as P

    cwd = os.getcwd()
    run = _run_dir("mbu_", L, gam, mb_params(rc=1, lor=1))
    os.chdir(run)
    try:
        rr = np.linspace(-5e-8, 5e-8, 64)
        qrr = R.SBEs.GetKArray(64, 64 * (rr[1] - rr[0]))
        s = R.SBEs.SBESolver(qrr, rr, 0.0, 1e7, 800e-9, 1, True)
        nk = s.Nk
        rng = np.random.default_rng(23)

        def level():
            p = 0.05 * (rng.standard_normal((nk, nk)) + 1j * rng.standard_normal((nk, nk)))
            c = 0.02 * (rng.standard_normal((nk, nk)) + 1j * rng.standard_normal((nk, nk)))
            d = 0.02 * (rng.standard_normal((nk, nk)) + 1j * rng.standard_normal((nk, nk)))
            c[np.diag_indices(nk)] = rng.uniform(0.05, 0.6, nk) + 0.01j * rng.standard_normal(nk)
            d[np.diag_indices(nk)] = rng.uniform(0.05, 0.6, nk) + 0.01j * rng.standard_normal(nk)
            return p, c, d

        p1, c1, d1 = level()   # X1 (the new X3 when dt = 0)
        p2, c2, d2 = level()   # X2 (what the right-hand side reads)
        ne2, nh2 = np.diag(c2).copy(), np.diag(d2).copy()
        VC = np.zeros((nk, nk, 3))
        E1D = np.zeros((nk, nk))
        C.CalcScreenedArrays(False, s.L, ne2, nh2, VC, E1D)
        GamE, GamH = np.zeros(nk), np.zeros(nk)
        D.CalcGammaE(s.kr, ne2, nh2, VC, GamE)
        D.CalcGammaH(s.kr, ne2, nh2, VC, GamH)
        g = np.array([s.gam_eh, s.gam_e, s.gam_h])
        De = D.CalcOffDiagDeph_E2(ne2, nh2, s.kr, s.Ee, s.Eh, g[0], g[2], VC, nk)
        Dh = D.CalcOffDiagDeph_H2(ne2, nh2, s.kr, s.Ee, s.Eh, g[1], g[2], VC, nk)
        OffP = np.zeros((nk, nk), complex)
        D.OffDiagDephasing2(ne2, nh2, p2, s.kr, s.Ee, s.Eh, g, VC, 0.0, OffP)
        ne3, nh3 = np.real(np.diag(c1)), np.real(np.diag(d1))
        WinE, WoutE, WinH, WoutH = (np.zeros(nk) for _ in range(4))
        C.MBCE(ne3, nh3, s.kr, s.Ee, s.Eh, VC, s.gam_eh, s.gam_e, WinE, WoutE)
        P.MBPE(ne3, VC, E1D, WinE, WoutE)
        C.MBCH(ne3, nh3, s.kr, s.Ee, s.Eh, VC, s.gam_eh, s.gam_h, WinH, WoutH)
        P.MBPH(nh3, VC, E1D, WinH, WoutH)
        Rsp = np.zeros(nk)
        EM.SpontEmission(ne2, nh2, s.Ee, s.Eh, s.gap, s.gam_eh, VC, Rsp)
        from pulsesuite.PSTD3D import dcfield as DC
        # host tables of InitializeEmission / InitializeDC and their inputs
        host = dict(kr=s.kr, dcv=s.dcv, epsr=s.epsr, gam_eh=s.gam_eh, ehint=s.ehint,
                    HOmega=EM._HOmega, square=EM._square, Ydc=DC._instance.Y)
        np.savez_compressed(os.path.join(out, "manybody_units_nk32.npz"), nk=nk, L=L, gam=gam,
                            p1=p1, c1=c1, d1=d1, p2=p2, c2=c2, d2=d2, GamE=GamE, GamH=GamH,
                            De=De, Dh=Dh, OffP=OffP, WinE=WinE, WoutE=WoutE, WinH=WinH,
                            WoutH=WoutH, Rsp=Rsp, **host)
        print(f"manybody units: Nk={nk}, |GamE| {np.max(np.abs(GamE)):.3e}, |OffP| "
              f"{np.max(np.abs(OffP)):.3e}, |WinE| {np.max(np.abs(WinE)):.3e}, "
              f"|Rsp| {np.max(np.abs(Rsp)):.3e}")
    finally:
        os.chdir(cwd)


def make_glue(R, out):
    """The reference's spline resampling and centred transforms on random
    data (the wire/propagation grid plumbing of QWCalculator)."""
    from pulsesuite.libpulsesuite import spliner

    rng = np.random.default_rng(17)
    x0 = np.linspace(-5e-8, 5e-8, 64)
    z0 = rng.standard_normal(64) + 1j * rng.standard_normal(64)
    x1 = np.linspace(-6e-8, 6e-8, 70)  # reaches beyond x0 on both sides
    z1 = np.zeros(70, complex)
    spliner.rescale_1D(x0, z0, x1, z1)
    F = z0.copy()
    R.usefulsubs.FFTG(F)
    G = z0.copy()
    R.usefulsubs.iFFTG(G)
    np.savez_compressed(os.path.join(out, "glue.npz"), x0=x0, z0=z0, x1=x1, z1=z1, fftg=F,
                        ifftg=G)
    print("glue: done")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--full-c0", action="store_true")
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    R = import_reference()
    out = HERE
    only = set(a.only.split(",")) if a.only else None

    def want(k):
        return only is None or k in only

    if want("tables"):
        make_tables(R, out)
    if want("rhs"):
        make_rhs(R, out)
    if want("rk4"):
        make_rk4(R, out, "rk4_c0_nk32", rwa_case(32, 600))
        make_rk4(R, out, "rk4_c0_nk64", rwa_case(64, 400, theta=1.5 * np.pi, det_meV=20.0,
                                                 fwhm=30e-15, T2=60e-15))
        make_rk4(R, out, "rk4_screened_nk32", rwa_case(32, 400, theta=1.2 * np.pi,
                                                       screened=True))
    if want("leapfrog"):
        make_leapfrog(R, out, "leapfrog_nk32", screened=False)
        make_leapfrog(R, out, "leapfrog_screened_nk32", screened=True, nsteps=2000)
    if want("solver"):
        make_solver_api(R, out)
    if want("glue"):
        make_glue(R, out)
    if want("qwcalc"):
        make_qwcalculator(R, out, "qwcalc_screened_nk32", screened=True)
        make_qwcalculator(R, out, "qwcalc_nk32", screened=False, nsteps=120)
    if want("manybody"):
        make_manybody_units(R, out)
        make_qwcalculator(R, out, "qwcalc_manybody_nk32", screened=True, nsteps=120,
                          mb=mb_params(scr=1))
    if want("transport"):
        # all six many-body flags with a DC field: the whole matrices shifted
        # (LF) or their diagonals only
        for lf in (1, 0):
            make_qwcalculator(R, out, f"qwcalc_mb_dc_{'lf' if lf else 'diag'}_nk32",
                              screened=True, nsteps=120, edc=2e6,
                              mb=mb_params(scr=1, dc=1, rc=1, lf=lf))
    if a.full_c0:
        make_rk4(R, out, "rk4_c0_nk128_full", rwa_case(128, 4000))


if __name__ == "__main__":
    main()
