"""The reference's own Numba CPU path, timed as a CPU baseline.

TEST INFRASTRUCTURE ONLY (a reported baseline, never the product path):
only bench.py's CPU-baseline legs import this module.

Imports the unmodified reference package installed under
``baseline/_ref`` (``pip install --target baseline/_ref``) and drives its
diagonal-drive harness, the same one the goldens come from
(tests/golden/make_golden.py):

  * right-hand side: ``SBEs._CalcH_jit`` (SBEs.py:819-935) +
    ``_dpdt_jit`` / ``_dCdt_jit`` / ``_dDdt_jit`` (SBEs.py:1952-2636) on
    full Nk x Nk matrices (the reference has no diagonal form), with the
    rotating-frame drive Meh = -mscale E_env(t) on the diagonal;
  * integrator: ``libpulsesuite.integrator.rk4_dpc`` (integrator.py:165).

Three adjustments are needed to run the reference in this image, none of
which changes its arithmetic:
  1. ``pyfftw`` is not installed: a shim maps ``pyfftw.interfaces.
     numpy_fft`` to ``numpy.fft`` (the FFTs are off this path);
  2. ``pulsesuite.PSTD3D.benchmark`` does not exist in the reference but is
     imported by its old entry points: a stub module with
     ``profile_start`` / ``profile_record`` stands in;
  3. numba 0.65 (the image's version; the reference pins 0.61.2)
     mis-compiles the ``parallel=True`` build of ``_CalcH_jit``, so the
     same Python source is recompiled with ``parallel=False`` and checked
     against ``_CalcH_fallback`` before use.
"""

import os
import sys
import tempfile
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF_ROOT = os.path.join(REPO, "baseline", "_ref")

_R = None


def available(ref_root=REF_ROOT):
    return os.path.isdir(os.path.join(ref_root, "pulsesuite"))


def load(ref_root=REF_ROOT, threads=None):
    """Import the reference (once per process) with the shims above."""
    global _R
    if _R is not None:
        return _R
    if not available(ref_root):
        raise FileNotFoundError(f"reference package not installed under {ref_root}")
    tmp = tempfile.mkdtemp(prefix="psb_ref_")
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tmp, "numba_cache"))
    os.environ["PULSESUITE_USE_CUDA"] = "0"
    if threads:
        os.environ.setdefault("NUMBA_NUM_THREADS", str(int(threads)))
    shim = os.path.join(tmp, "shim")
    os.makedirs(os.path.join(shim, "pyfftw", "interfaces"), exist_ok=True)
    with open(os.path.join(shim, "pyfftw", "__init__.py"), "w") as f:
        f.write("from . import interfaces\n")
    with open(os.path.join(shim, "pyfftw", "interfaces", "__init__.py"), "w") as f:
        f.write("import numpy.fft as numpy_fft\n\n\nclass cache:\n"
                "    enable = staticmethod(lambda: None)\n")
    sys.path.insert(0, shim)
    sys.path.insert(0, ref_root)
    stub = types.ModuleType("pulsesuite.PSTD3D.benchmark")
    stub.profile_start = time.perf_counter
    stub.profile_record = lambda name, t0: None
    sys.modules["pulsesuite.PSTD3D.benchmark"] = stub

    import numba

    from pulsesuite.libpulsesuite import integrator
    from pulsesuite.PSTD3D import SBEs, usefulsubs

    SBEs._CalcH_jit = numba.njit(parallel=False)(SBEs._CalcH_jit.py_func)
    _selftest_calch(SBEs)
    _R = types.SimpleNamespace(SBEs=SBEs, usefulsubs=usefulsubs, integrator=integrator,
                               numba=numba, threads=numba.config.NUMBA_NUM_THREADS)
    return _R


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
                raise RuntimeError("recompiled _CalcH_jit disagrees with _CalcH_fallback")


def rk4_solver(R, grid, wire):
    """(D, y0) of one wire in the reference's harness: D(t, y) is the
    reference RHS on the diagonal state y = (p, n_e, n_h) (complex 3 Nk)."""
    S = R.SBEs
    nk = grid.nk
    v = np.array([0.0] + [grid.vprefactor * R.usefulsubs.K03(abs(grid.kr[q] - grid.kr[0])
                                                               * grid.radius)
                          for q in range(1, nk)])
    VC = np.zeros((nk, nk, 3))
    for n in range(3):
        VC[:, 0, n] = v
    Ee, Eh = grid.Ee, grid.Eh
    gap = float(wire["gap"])
    G = np.full(nk, float(wire["gamma"]) / 2.0)
    amp, t0, fwhm = float(wire["amp"][0]), float(wire["t0"][0]), float(wire["fwhm"][0])
    mscale = float(wire["mscale"])
    Z = np.zeros((nk, nk), complex)
    Heh, Hee, Hhh = (np.zeros((nk, nk), complex) for _ in range(3))

    def D(t, y):
        p, ne, nh = y[:nk], y[nk:2 * nk].real, y[2 * nk:].real
        E = amp * np.exp(-4.0 * np.log(2.0) * ((t - t0) / fwhm) ** 2)
        Meh = np.diag(np.full(nk, -mscale * E, dtype=complex))
        C = np.diag(ne.astype(complex))
        Dm = np.diag(nh.astype(complex))
        P = np.diag(p.astype(complex))
        S._CalcH_jit(Meh, Z, Z, C, Dm, P, VC, Heh, Hee, Hhh, nk, Ee, Eh, gap, True, False, False)
        dp = S._dpdt_jit(C, Dm, P, Heh, Hee, Hhh, G, G, Z, 1j, S.hbar)
        dC = S._dCdt_jit(C, Dm, P, Heh, Hee, Hhh, G, G, Z, 1j, S.hbar)
        dD = S._dDdt_jit(C, Dm, P, Heh, Hee, Hhh, G, G, Z, 1j, S.hbar)
        return np.concatenate([np.diag(dp), np.diag(dC), np.diag(dD)])

    return D, np.zeros(3 * nk, dtype=complex)


def seconds_per_step(R, grid, wire, dt, nsteps=1):
    """Wall seconds of one RK4 step of one wire (after a warm-up step that
    compiles the kernels)."""
    D, y = rk4_solver(R, grid, wire)
    t = 0.0
    t = R.integrator.rk4_dpc(y, D(t, y), t, dt, D)  # warm-up / JIT
    t0 = time.perf_counter()
    for _ in range(nsteps):
        t = R.integrator.rk4_dpc(y, D(t, y), t, dt, D)
    return (time.perf_counter() - t0) / nsteps


def qwcalc_seconds_per_wire_step(R, qw_params, mb_params, nrr=64, nsteps=2, E0=1e8):
    """Wall seconds of one call of the reference's SBESolver.QWCalculator
    (SBEs.py:5838-6001) for one wire -- the step the PSTD caller makes per
    wire per Maxwell step (rhoPJ.py:311-348) -- with the given params-file
    texts, driven by fields along the wire with a Gaussian profile (the
    full-matrix state with every many-body term mb.params switches on).
    The solver is built in a scratch directory (it reads params/ and writes
    dataQW/ there); one untimed call compiles the Numba kernels.  Returns
    (seconds, Nk)."""
    run = tempfile.mkdtemp(prefix="psb_qwc_")
    os.makedirs(os.path.join(run, "params"))
    with open(os.path.join(run, "params", "qw.params"), "w") as f:
        f.write(qw_params)
    with open(os.path.join(run, "params", "mb.params"), "w") as f:
        f.write(mb_params)
    cwd = os.getcwd()
    os.chdir(run)
    try:
        rr = np.linspace(-5e-8, 5e-8, nrr)
        qrr = R.SBEs.GetKArray(nrr, nrr * (rr[1] - rr[0]))
        s = R.SBEs.SBESolver(qrr, rr, 0.0, 1e7, 800e-9, 1, True)
        prof = np.exp(-((rr / 3e-8) ** 2))
        dt = 1e-17

        def call():
            o = [np.zeros(nrr, complex) for _ in range(4)]
            s.QWCalculator((0.3 * E0 * prof * (rr / 3e-8)).astype(complex),
                           (E0 * prof).astype(complex), (0.2 * E0 * prof).astype(complex),
                           np.zeros(nrr, complex), rr, qrr, dt, 1, *o, [False], [False])

        call()
        t0 = time.perf_counter()
        for _ in range(nsteps):
            call()
        return (time.perf_counter() - t0) / nsteps, int(s.Nk)
    finally:
        os.chdir(cwd)
